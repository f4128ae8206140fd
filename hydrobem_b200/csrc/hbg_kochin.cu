// hbg_kochin.cu -- Kochin functions of the radiation and scattered waves and the mean drift by momentum
// conservation, from the solved potentials of a frequency batch (lo_frequency.rs:1277-1374,
// low_order.rs:1417-1452, response.rs:51-300).
#include <cstring>

#include "../../include/hydrobem_gpu.h"
#include "hbg_device.cuh"
#include "hbg_internal.h"

namespace hbg {

__device__ __forceinline__ double2 zmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

constexpr int KO_COLS = 8;  // columns (radiation modes and headings) a block accumulates

// One block per (angle t, frequency f, chunk of KO_COLS columns): over the wetted panels (the interior
// panels take no part) the far-field kernel g = Z(z) e^{i k (x cos + y sin)} of the global angle
// theta_t = 2 pi t / T, its normal derivative gn and their theta-derivatives (low_order.rs:1417-1431),
// times the panel area, then for a radiation column c H += phi_c Dx - Sx u_c and for a heading h (the
// scattered formulation: the total potential with the dipole column) H += (phi_S + phi_I) Dx, the
// derivative H_t with the theta-derivatives.  The frame is global with no yaw (kochin_global the identity).
__global__ void __launch_bounds__(256) k_kochin(PanelsView pv, const FreqInfo* __restrict__ fi, int T, int H,
                                                double depth, const double2* __restrict__ phi, int ldphi,
                                                const double2* __restrict__ u, const double2* __restrict__ phiI,
                                                double2* __restrict__ kr, double2* __restrict__ krt,
                                                double2* __restrict__ kd, double2* __restrict__ kdt) {
    __shared__ double red[8][4 * KO_COLS];
    const int t = blockIdx.x, f = blockIdx.y, c0 = blockIdx.z * KO_COLS, N = pv.N;
    const int D = 6 * pv.nbod, nrhs = D + H;
    double s, c;
    sincospi(2.0 * t / T, &s, &c);
    const double k = fi[f].k;
    const bool finite = depth > 0.0;
    double acc[4 * KO_COLS];
#pragma unroll
    for (int q = 0; q < 4 * KO_COLS; q++) acc[q] = 0.0;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        if (pv.kind[j] != 0) continue;
        const double x = pv.at(P_C, j), y = pv.at(P_C + 1, j), z = pv.at(P_C + 2, j);
        const double nx = pv.at(P_N, j), ny = pv.at(P_N + 1, j), nz = pv.at(P_N + 2, j), ar = pv.at(P_AREA, j);
        double Z = exp(k * z), Zz = k * Z;
        if (finite) {  // low_order.rs:1401-1412
            const double b = exp(-k * (z + 2.0 * depth)), dd = 1.0 + exp(-2.0 * k * depth);
            Zz = k * (Z - b) / dd;
            Z = (Z + b) / dd;
        }
        double sp, cp;
        sincos(k * (x * c + y * s), &sp, &cp);
        const double2 e = make_double2(cp, sp);
        const double dt = -x * s + y * c, dnt = -nx * s + ny * c;
        const double2 g = zscale(e, Z);
        const double2 gn = zmul(e, make_double2(Zz * nz, Z * k * (nx * c + ny * s)));
        const double2 gt = zmul(g, make_double2(0.0, k * dt));
        const double2 gnt = zadd(zmul(gn, make_double2(0.0, k * dt)), zmul(e, make_double2(0.0, Z * k * dnt)));
        const double2 Sx = zscale(g, ar), Dx = zscale(gn, ar), St = zscale(gt, ar), Dt = zscale(gnt, ar);
#pragma unroll
        for (int q = 0; q < KO_COLS; q++) {
            const int col = c0 + q;
            if (col >= nrhs) break;
            double2 p = phi[((size_t)f * nrhs + col) * ldphi + j];
            double2 hv, ht;
            if (col < D) {
                const double2 uc = u[((size_t)f * nrhs + col) * N + j];
                hv = zadd(zmul(p, Dx), zscale(zmul(Sx, uc), -1.0));
                ht = zadd(zmul(p, Dt), zscale(zmul(St, uc), -1.0));
            } else {
                p = zadd(p, phiI[((size_t)f * H + (col - D)) * N + j]);
                hv = zmul(p, Dx);
                ht = zmul(p, Dt);
            }
            acc[4 * q] += hv.x;
            acc[4 * q + 1] += hv.y;
            acc[4 * q + 2] += ht.x;
            acc[4 * q + 3] += ht.y;
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 4 * KO_COLS; q++) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < KO_COLS) {
        const int q = threadIdx.x, col = c0 + q;
        if (col < nrhs) {
            double v[4] = {0.0, 0.0, 0.0, 0.0};
            for (int w = 0; w < (int)(blockDim.x >> 5); w++)
                for (int i = 0; i < 4; i++) v[i] += red[w][4 * q + i];
            if (col < D) {
                kr[((size_t)f * T + t) * D + col] = make_double2(v[0], v[1]);
                krt[((size_t)f * T + t) * D + col] = make_double2(v[2], v[3]);
            } else {
                kd[((size_t)f * T + t) * H + (col - D)] = make_double2(v[0], v[1]);
                kdt[((size_t)f * T + t) * H + (col - D)] = make_double2(v[2], v[3]);
            }
        }
    }
}

// The mean drift by momentum conservation of every heading pair, one block per frequency
// (response.rs:183-300): b_h(theta) = fac (H_D + sum_c i w H_c xi_c) with the motions xi of the
// radiation columns (none for a fixed body), fac the far-field amplitude of the propagating mode; the
// quadratic far-field flux of the pair over the T angles, and the interaction with the incident waves
// through b's trigonometric interpolant at the headings (the T-mode interpolant of the reference's Trig:
// modes -(T-1)/2 .. (T-1)/2 and, for even T, the Nyquist term; written here as its Dirichlet kernel
// D(phi) = sin(M phi / 2) / sin(phi / 2), M the odd mode count).  drift [F][H][H][3]: surge, sway, yaw;
// the equal pairs keep their real parts.  Shared memory: b, bt and the interpolation weights, H T each.
__global__ void __launch_bounds__(256) k_drift(int D, int H, int T, const FreqInfo* __restrict__ fi, double depth,
                                               double grav, double rho, const double* __restrict__ heads,
                                               const double2* __restrict__ kr, const double2* __restrict__ krt,
                                               const double2* __restrict__ kd, const double2* __restrict__ kdt,
                                               const double2* __restrict__ xi, double2* __restrict__ drift) {
    extern __shared__ double2 dr_smem[];
    double2* b = dr_smem;           // [H][T]
    double2* bt = b + H * T;        // [H][T]
    double* Wt = reinterpret_cast<double*>(bt + H * T);  // [H][T]: the interpolation weights at the headings
    const int f = blockIdx.x;
    const double w = fi[f].omega, k = fi[f].k, K0 = w * w / grav;
    double C = 2.0 * PI * K0, Ke = K0;
    if (depth > 0.0) {
        const double x = k * depth;
        const double A0 = 2.0 * PI * k / (-expm1(-4.0 * x) + 4.0 * x * exp(-2.0 * x));
        const double ch = cosh(x), e2 = 1.0 + exp(-2.0 * x);
        C = A0 * e2 * e2;
        Ke = K0 + k * k * depth / (ch * ch);
    }
    // fac = -(i C / (4 pi)) sqrt(2 / (pi k)) e^{i pi / 4}
    const double fm = -C / (4.0 * PI) * sqrt(2.0 / (PI * k));
    const double2 fac = zmul(make_double2(0.0, fm), make_double2(cos(0.25 * PI), sin(0.25 * PI)));
    const int M = 2 * ((T - 1) / 2) + 1;  // modes -(T-1)/2 .. (T-1)/2
    for (int idx = threadIdx.x; idx < H * T; idx += blockDim.x) {
        const int h = idx / T, t = idx % T;
        double2 v = kd[((size_t)f * T + t) * H + h], vt = kdt[((size_t)f * T + t) * H + h];
        if (xi)
            for (int c = 0; c < D; c++) {
                const double2 x = zmul(make_double2(0.0, w), xi[((size_t)f * H + h) * D + c]);
                v = zadd(v, zmul(kr[((size_t)f * T + t) * D + c], x));
                vt = zadd(vt, zmul(krt[((size_t)f * T + t) * D + c], x));
            }
        b[h * T + t] = zmul(fac, v);
        bt[h * T + t] = zmul(fac, vt);
        // weight of angle t in the interpolant at heading h
        const double ph = heads[h] - 2.0 * PI * t / T, sh = sin(0.5 * ph);
        double dk = fabs(sh) > 1e-12 ? sin(0.5 * M * ph) / sh : (double)M;  // the limit is M for odd M
        if (T % 2 == 0) dk += ((t & 1) ? -1.0 : 1.0) * cos(0.5 * T * heads[h]);
        Wt[h * T + t] = dk / T;
    }
    __syncthreads();
    const double s = rho * Ke / 4.0, q = sqrt(2.0 * PI / k), dth = 2.0 * PI / T;
    const double2 a = make_double2(0.0, grav / w), e = make_double2(cos(-0.25 * PI), sin(-0.25 * PI));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int p = warp; p < H * H; p += nw) {
        const int i = p / H, j = p % H;
        double2 sx = {0, 0}, sy = {0, 0}, dd = {0, 0}, bbij = {0, 0}, bbji = {0, 0}, btij = {0, 0}, btji = {0, 0};
        for (int t = lane; t < T; t += 32) {
            double st, ct;
            sincospi(2.0 * t / T, &st, &ct);
            const double2 bi = b[i * T + t], bj = b[j * T + t], ti = bt[i * T + t], tj = bt[j * T + t];
            const double2 pij = zmul(bi, zconj(bj));
            sx = zadd(sx, zscale(pij, ct));
            sy = zadd(sy, zscale(pij, st));
            dd = zadd(dd, zadd(zmul(ti, zconj(bj)), zscale(zmul(bi, zconj(tj)), -1.0)));
            bbij = zadd(bbij, zscale(bi, Wt[j * T + t]));
            bbji = zadd(bbji, zscale(bj, Wt[i * T + t]));
            btij = zadd(btij, zscale(ti, Wt[j * T + t]));
            btji = zadd(btji, zscale(tj, Wt[i * T + t]));
        }
        double r[14] = {sx.x, sx.y, sy.x, sy.y, dd.x, dd.y, bbij.x, bbij.y, bbji.x, bbji.y, btij.x, btij.y, btji.x, btji.y};
#pragma unroll
        for (int m = 0; m < 14; m++)
            for (int o = 16; o > 0; o >>= 1) r[m] += __shfl_xor_sync(0xffffffffu, r[m], o);
        if (lane == 0) {
            sx = make_double2(r[0], r[1]);
            sy = make_double2(r[2], r[3]);
            dd = zmul(make_double2(r[4], r[5]), make_double2(0.0, -0.5));  // / (2 i)
            bbij = make_double2(r[6], r[7]);
            bbji = make_double2(r[8], r[9]);
            btij = make_double2(r[10], r[11]);
            btji = make_double2(r[12], r[13]);
            const double2 ae = zmul(zconj(a), e), ea = zmul(a, zconj(e));
            const double2 cx = zscale(zmul(ae, bbij), -s * q);          // incident j, disturbance i
            const double2 cy = zscale(zmul(ea, zconj(bbji)), -s * q);   // incident i, disturbance j
            const double cbi = cos(heads[i]), sbi = sin(heads[i]), cbj = cos(heads[j]), sbj = sin(heads[j]);
            double2 o0 = zadd(zadd(zscale(sx, -s * dth), zscale(cx, cbj)), zscale(cy, cbi));
            double2 o1 = zadd(zadd(zscale(sy, -s * dth), zscale(cx, sbj)), zscale(cy, sbi));
            const double2 term = zadd(zmul(make_double2(0.0, 1.0), zmul(ae, btij)),
                                      zscale(zmul(make_double2(0.0, 1.0), zmul(ea, zconj(btji))), -1.0));
            double2 o2 = zadd(zscale(dd, s / k * dth), zscale(term, -(s / k) * q));
            if (i == j) {
                o0.y = 0.0;
                o1.y = 0.0;
                o2.y = 0.0;
            }
            double2* o = drift + (((size_t)f * H + i) * H + j) * 3;
            o[0] = o0;
            o[1] = o1;
            o[2] = o2;
        }
    }
}

size_t drift_smem_bytes(int H, int T) { return (size_t)H * T * (2 * sizeof(double2) + sizeof(double)); }

void launch_kochin(const PanelsView& pv, int F, const FreqInfo* fi, int T, int H, double depth, const double2* phi,
                   int ldphi, const double2* u, const double2* phiI, double2* kr, double2* krt, double2* kd,
                   double2* kdt, cudaStream_t s) {
    const int nrhs = 6 * pv.nbod + H;
    k_kochin<<<dim3(T, F, (nrhs + KO_COLS - 1) / KO_COLS), 256, 0, s>>>(pv, fi, T, H, depth, phi, ldphi, u, phiI, kr,
                                                                          krt, kd, kdt);
}

void launch_drift(int F, int D, int H, int T, const FreqInfo* fi, double depth, double grav, double rho,
                  const double* heads, const double2* kr, const double2* krt, const double2* kd, const double2* kdt,
                  const double2* xi, double2* drift, cudaStream_t s) {
    const size_t sm = drift_smem_bytes(H, T);
    cudaFuncSetAttribute(k_drift, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_drift<<<F, 256, sm, s>>>(D, H, T, fi, depth, grav, rho, heads, kr, krt, kd, kdt, xi, drift);
}

// The Kochin functions and the drift of frequency i of a batch of nb (host copy of the device layout
// [kr nb][krt nb][kd nb][kdt nb][drift nb], complex) into the caller's arrays at frequency fo.
void copy_kochin(const HbgOutputs& o, const double* h, int T, int D, int H, int nb, int i, size_t fo) {
    const size_t rd = (size_t)T * D * 2, rh = (size_t)T * H * 2, rr = (size_t)H * H * 3 * 2;
    const double* kr = h;
    const double* krt = kr + rd * nb;
    const double* kd = krt + rd * nb;
    const double* kdt = kd + rh * nb;
    const double* dr = kdt + rh * nb;
    if (o.kochin_radiation) memcpy(o.kochin_radiation + fo * rd, kr + rd * i, rd * sizeof(double));
    if (o.kochin_radiation_derivative) memcpy(o.kochin_radiation_derivative + fo * rd, krt + rd * i, rd * sizeof(double));
    if (o.kochin_diffraction) memcpy(o.kochin_diffraction + fo * rh, kd + rh * i, rh * sizeof(double));
    if (o.kochin_diffraction_derivative)
        memcpy(o.kochin_diffraction_derivative + fo * rh, kdt + rh * i, rh * sizeof(double));
    if (o.drift) memcpy(o.drift + fo * rr, dr + rr * i, rr * sizeof(double));
}

}  // namespace hbg
