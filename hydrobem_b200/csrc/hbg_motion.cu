// hbg_motion.cu -- the hydrostatics of each body and the rigid-body motions of each frequency, on the
// device beside the forces (crates/hydrobem/src/hydrostatics.rs, motion.rs).
#include "hbg_device.cuh"
#include "hbg_internal.h"
#include "../../include/hydrobem_gpu.h"

namespace hbg {

// ------------------------------------------------------------------ hydrostatics
// hydrostatics.rs:116-141 (Acc) and 143-313 (Problem::hydrostatics) on the wetted panels of body b: one
// quadrature point per low-order panel, its centroid with n dS = area times the normal into the fluid
// (quadrature.rs:152-159); x, y relative to the rotation centre R, z the global depth coordinate.
// Block b reduces the twelve sums (warp shuffles, then the warps in a fixed order), then thread 0 forms the
// record of the body (HBG_HS doubles), its restoring matrix with the weight terms and its rigid inertia about
// R (hydrostatics.rs:315-356) into the block-diagonal D x D matrices C and M; C also receives the additional
// stiffness rows of the body and B_ext the additional damping rows.
__global__ void __launch_bounds__(256) k_hydrostatics(PanelsView pv, const double* __restrict__ rig,
                                                      const double* __restrict__ cext, const double* __restrict__ bext,
                                                      double rho, double grav, double* __restrict__ hs,
                                                      double* __restrict__ MM, double* __restrict__ CC,
                                                      double* __restrict__ BB) {
    __shared__ double red[8][12];
    const int b = blockIdx.x, N = pv.N, D = 6 * pv.nbod;
    const double R0 = pv.rcen ? pv.rcen[3 * b] : 0.0, R1 = pv.rcen ? pv.rcen[3 * b + 1] : 0.0,
                 R2 = pv.rcen ? pv.rcen[3 * b + 2] : 0.0;
    double a[12];
#pragma unroll
    for (int k = 0; k < 12; k++) a[k] = 0.0;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        if (pv.kind[j] != 0 || (pv.body ? pv.body[j] : 0) != b) continue;
        const double x = pv.at(P_C, j) - R0, y = pv.at(P_C + 1, j) - R1, z = pv.at(P_C + 2, j);
        const double ar = pv.at(P_AREA, j);
        const double n0 = ar * pv.at(P_N, j), n1 = ar * pv.at(P_N + 1, j), n2 = ar * pv.at(P_N + 2, j);
        a[0] += x * n0;  // vx
        a[1] += y * n1;  // vy
        a[2] += z * n2;  // vz
        a[3] += 0.5 * x * x * n0;  // mx
        a[4] += 0.5 * y * y * n1;  // my
        a[5] += 0.5 * z * z * n2;  // mz
        a[6] -= n2;                // aw
        a[7] -= x * n2;            // ax
        a[8] -= y * n2;            // ay
        a[9] -= x * x * n2;        // axx
        a[10] -= y * y * n2;       // ayy
        a[11] -= x * y * n2;       // axy
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 12; k++) {
        double v = a[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double s[12];
    for (int k = 0; k < 12; k++) {
        s[k] = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s[k] += red[w][k];
    }
    const double vx = s[0], vy = s[1], V = s[2], mx = s[3], my = s[4], mz = s[5], aw = s[6], ax = s[7], ay = s[8],
                 axx = s[9], ayy = s[10], axy = s[11];
    double* h = hs + (size_t)b * HBG_HS;
    h[0] = vx;
    h[1] = vy;
    h[2] = V;
    h[3] = mx / V + R0;
    h[4] = my / V + R1;
    h[5] = mz / V;
    h[6] = aw;
    h[7] = ax / aw + R0;
    h[8] = ay / aw + R1;
    const double rg = rho * grav, Vzb = mz - R2 * V;
    double c[36];
    for (int k = 0; k < 36; k++) c[k] = 0.0;
    c[2 * 6 + 2] = rg * aw;
    c[2 * 6 + 3] = rg * ay;
    c[3 * 6 + 2] = c[2 * 6 + 3];
    c[2 * 6 + 4] = -rg * ax;
    c[4 * 6 + 2] = c[2 * 6 + 4];
    c[3 * 6 + 3] = rg * (ayy + Vzb);
    c[3 * 6 + 4] = -rg * axy;
    c[4 * 6 + 3] = c[3 * 6 + 4];
    c[3 * 6 + 5] = -rg * mx;
    c[4 * 6 + 4] = rg * (axx + Vzb);
    c[4 * 6 + 5] = -rg * my;
    for (int k = 0; k < 36; k++) h[9 + k] = c[k];
    // the mass in use: given, or the displaced mass rho V_x; the weight terms with G
    const double* r = rig ? rig + (size_t)b * RIGID_PER_BODY : nullptr;
    const double mass = r ? (isnan(r[0]) ? rho * vx : r[0]) : __longlong_as_double(0x7ff8000000000000ll);
    double M[36];
    for (int k = 0; k < 36; k++) M[k] = 0.0;
    if (r) {
        const double g0 = r[1] - R0, g1 = r[2] - R1, g2 = r[3] - R2;
        const double mg = mass * grav;
        c[3 * 6 + 3] -= mg * g2;
        c[3 * 6 + 5] += mg * g0;
        c[4 * 6 + 4] -= mg * g2;
        c[4 * 6 + 5] += mg * g1;
        // rigid inertia about R: J about the origin o (components, or m r |r| from radii of gyration),
        // moved to G and from G to R (hydrostatics.rs:319-356)
        double J[9];
        for (int k = 0; k < 9; k++) J[k] = r[4] == HBG_INERTIA_GYRATION ? mass * r[5 + k] * fabs(r[5 + k]) : r[5 + k];
        const double cg[3] = {r[1], r[2], r[3]}, cc[3] = {g0, g1, g2};
        const double aa[3] = {cg[0] - r[14], cg[1] - r[15], cg[2] - r[16]};
        const double a2 = aa[0] * aa[0] + aa[1] * aa[1] + aa[2] * aa[2], c2 = cc[0] * cc[0] + cc[1] * cc[1] + cc[2] * cc[2];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                J[3 * i + j] += -mass * ((i == j ? a2 : 0.0) - aa[i] * aa[j]) + mass * ((i == j ? c2 : 0.0) - cc[i] * cc[j]);
        const double S[9] = {0.0, -cc[2], cc[1], cc[2], 0.0, -cc[0], -cc[1], cc[0], 0.0};
        for (int i = 0; i < 3; i++) {
            M[i * 6 + i] = mass;
            for (int j = 0; j < 3; j++) {
                M[i * 6 + 3 + j] = -mass * S[3 * i + j];
                M[(3 + i) * 6 + j] = mass * S[3 * i + j];
                M[(3 + i) * 6 + 3 + j] = J[3 * i + j];
            }
        }
    }
    for (int k = 0; k < 36; k++) h[45 + k] = c[k];
    h[81] = mass;
    h[82] = rho * vx;
    // rows 6 b .. 6 b + 5 of the motion matrices
    for (int i = 6 * b; i < 6 * b + 6; i++)
        for (int j = 0; j < D; j++) {
            const bool own = j >= 6 * b && j < 6 * b + 6;
            const int k = (i - 6 * b) * 6 + (j - 6 * b);
            MM[(size_t)i * D + j] = own ? M[k] : 0.0;
            CC[(size_t)i * D + j] = (own ? c[k] : 0.0) + (cext ? cext[(size_t)i * D + j] : 0.0);
            BB[(size_t)i * D + j] = bext ? bext[(size_t)i * D + j] : 0.0;
        }
}

void launch_hydrostatics(const PanelsView& pv, const double* rig, const double* cext, const double* bext, double rho,
                         double grav, double* hs, double* MM, double* CC, double* BB, cudaStream_t s) {
    k_hydrostatics<<<pv.nbod, 256, 0, s>>>(pv, rig, cext, bext, rho, grav, hs, MM, CC, BB);
}

// ------------------------------------------------------------------ motions
// motion.rs:121-158: (C - w^2 (M + A) + i w (B + B_ext)) xi = X for the H headings of frequency f (one block
// per frequency), Gaussian elimination with partial pivoting (the first largest modulus) in shared memory,
// then back substitution.  A zero pivot sets *err = 11 and leaves the frequency's motions unset.
constexpr int MOT_D = 32, MOT_H = 32;

__global__ void __launch_bounds__(128) k_motions(int D, int H, const FreqInfo* __restrict__ fi,
                                                 const double* __restrict__ A, const double* __restrict__ B,
                                                 const double2* __restrict__ X, const double* __restrict__ MM,
                                                 const double* __restrict__ CC, const double* __restrict__ BB,
                                                 double2* __restrict__ xi, int* __restrict__ err) {
    __shared__ double2 Z[MOT_D][MOT_D + 1];
    __shared__ double2 rhs[MOT_D][MOT_H];
    __shared__ double2 lf[MOT_D];
    __shared__ int piv, bad;
    const int f = blockIdx.x, t = threadIdx.x, nt = blockDim.x;
    const double w = fi[f].omega;
    for (int e = t; e < D * D; e += nt) {
        const int i = e / D, j = e % D;
        const size_t o = (size_t)f * D * D + e;
        Z[i][j] = make_double2(CC[e] - w * w * (MM[e] + A[o]), w * (B[o] + BB[e]));
    }
    for (int e = t; e < D * H; e += nt) {
        const int h = e / D, i = e % D;
        rhs[i][h] = X[((size_t)f * H + h) * D + i];
    }
    if (t == 0) bad = 0;
    __syncthreads();
    for (int k = 0; k < D; k++) {
        if (t == 0) {
            int p = k;
            double best = -1.0;
            for (int i = k; i < D; i++) {
                const double m = hypot(Z[i][k].x, Z[i][k].y);
                if (m > best) {
                    best = m;
                    p = i;
                }
            }
            piv = p;
            if (!(best > 0.0)) bad = 1;
        }
        __syncthreads();
        if (bad) break;
        const int p = piv;
        if (p != k) {
            for (int j = t; j < D; j += nt) {
                const double2 v = Z[k][j];
                Z[k][j] = Z[p][j];
                Z[p][j] = v;
            }
            for (int h = t; h < H; h += nt) {
                const double2 v = rhs[k][h];
                rhs[k][h] = rhs[p][h];
                rhs[p][h] = v;
            }
        }
        __syncthreads();
        const double2 d = Z[k][k];
        const double dd = d.x * d.x + d.y * d.y;
        for (int i = k + 1 + t; i < D; i += nt) {  // l_i = Z[i][k] / Z[k][k]
            const double2 z = Z[i][k];
            lf[i] = make_double2((z.x * d.x + z.y * d.y) / dd, (z.y * d.x - z.x * d.y) / dd);
        }
        __syncthreads();
        const int W = D - k - 1;
        for (int e = t; e < W * (D - k - 1 + H); e += nt) {
            const int i = k + 1 + e % W, c = e / W;
            const double2 l = lf[i];
            if (c < D - k - 1) {
                const int j = k + 1 + c;
                const double2 u = Z[k][j];
                Z[i][j].x -= l.x * u.x - l.y * u.y;
                Z[i][j].y -= l.x * u.y + l.y * u.x;
            } else {
                const int h = c - (D - k - 1);
                const double2 u = rhs[k][h];
                rhs[i][h].x -= l.x * u.x - l.y * u.y;
                rhs[i][h].y -= l.x * u.y + l.y * u.x;
            }
        }
        __syncthreads();
    }
    if (bad) {
        if (t == 0) atomicExch(err, 11);
        return;
    }
    // back substitution, one thread per heading
    for (int h = t; h < H; h += nt) {
        for (int k = D - 1; k >= 0; k--) {
            double2 v = rhs[k][h];
            for (int j = k + 1; j < D; j++) {
                const double2 z = Z[k][j], y = rhs[j][h];
                v.x -= z.x * y.x - z.y * y.y;
                v.y -= z.x * y.y + z.y * y.x;
            }
            const double2 d = Z[k][k];
            const double dd = d.x * d.x + d.y * d.y;
            rhs[k][h] = make_double2((v.x * d.x + v.y * d.y) / dd, (v.y * d.x - v.x * d.y) / dd);
        }
        for (int i = 0; i < D; i++) xi[((size_t)f * H + h) * D + i] = rhs[i][h];
    }
}

void launch_motions(int F, int D, int H, const FreqInfo* fi, const double* A, const double* B, const double2* X,
                    const double* MM, const double* CC, const double* BB, double2* xi, int* err, cudaStream_t s) {
    k_motions<<<F, 128, 0, s>>>(D, H, fi, A, B, X, MM, CC, BB, xi, err);
}

}  // namespace hbg
