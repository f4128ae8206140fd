// hbg_freq.cu -- the per-frequency kernels of the FP64 form: finite-depth tiles and fin points,
// assembly of S and A = 2 pi I - D, boundary values, right-hand sides -S u, pressure forces.
#include "hbg_device.cuh"
#include "hbg_internal.h"

namespace hbg {

void set_constants(const double glx[17][16], const double glw[17][16], const Tables& tab) {
    cudaMemcpyToSymbol(c_glx, glx, sizeof(double) * 17 * 16);
    cudaMemcpyToSymbol(c_glw, glw, sizeof(double) * 17 * 16);
    cudaMemcpyToSymbol(c_tab, &tab, sizeof(Tables));
}

// ------------------------------------------------------------------ finite-depth tiles
// green_fin.rs:493-564 build_tiles: the values and both derivatives of Phi1, Phi2 at the
// first-kind Chebyshev nodes of each tile (one thread per node), then per tile and quantity the
// discrete cosine transform to Chebyshev coefficients and the power basis (one thread each).
constexpr int NODES1 = TS * TW * TN * TN, NODES2 = TS * TV * TN * TN, NODES = NODES1 + NODES2;

__device__ __forceinline__ double cheb_node(int i) { return cos(PI * (i + 0.5) / TN); }

__global__ void k_fd_nodes(int F, const FdParams* __restrict__ fdp, double* __restrict__ scratch) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int f = blockIdx.y;
    if (t >= NODES || f >= F) return;
    const FdParams& fd = fdp[f];
    int which = t < NODES1 ? 1 : 2;
    int id = t < NODES1 ? t : t - NODES1;
    int ny = which == 1 ? TW : TV;
    double ymax = which == 1 ? 1.0 : 2.0;
    int j = id % TN, i = (id / TN) % TN, iy = (id / (TN * TN)) % ny, ix = id / (TN * TN * ny);
    double dx = XMAX / TS, dy = ymax / ny;
    double v[3];
    phi_direct(fd, which, dx * (ix + 0.5 * (cheb_node(i) + 1.0)), dy * (iy + 0.5 * (cheb_node(j) + 1.0)), v);
    double* o = scratch + ((size_t)f * NODES + t) * 3;
    o[0] = v[0];
    o[1] = v[1];
    o[2] = v[2];
}

__global__ void k_fd_fit(int F, const double* __restrict__ scratch, double* __restrict__ tiles) {
    constexpr int N = TN;
    constexpr int TILES1 = TS * TW, TILES2 = TS * TV;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int f = blockIdx.y;
    if (t >= 3 * (TILES1 + TILES2) || f >= F) return;
    int q = t % 3, tile = t / 3;
    int which = tile < TILES1 ? 1 : 2;
    int tid = tile < TILES1 ? tile : tile - TILES1;
    const double* s = scratch + (size_t)f * NODES * 3 + (which == 1 ? 0 : (size_t)NODES1 * 3) + (size_t)tid * N * N * 3;
    double fv[N][N];
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) fv[i][j] = s[(i * N + j) * 3 + q];
    double cs[N][N], a[N][N];
    for (int jj = 0; jj < N; jj++)
        for (int i = 0; i < N; i++) cs[jj][i] = cos(PI * jj * (i + 0.5) / N);
    for (int jj = 0; jj < N; jj++)
        for (int k = 0; k < N; k++) a[jj][k] = 0.0;
    a[0][0] = 1.0;
    a[1][1] = 1.0;
    for (int jj = 2; jj < N; jj++)
        for (int k = 0; k < N; k++) a[jj][k] = (k > 0 ? 2.0 * a[jj - 1][k - 1] : 0.0) - a[jj - 2][k];
    double c[N][N];
    for (int ji = 0; ji < N; ji++)
        for (int jj = 0; jj < N; jj++) {
            double acc = 0.0;
            for (int i = 0; i < N; i++)
                for (int j = 0; j < N; j++) acc += fv[i][j] * cs[ji][i] * cs[jj][j];
            c[ji][jj] = acc * (ji != 0 ? 2.0 : 1.0) * (jj != 0 ? 2.0 : 1.0) / (double)(N * N);
        }
    double pw[N * N];
    for (int k = 0; k < N * N; k++) pw[k] = 0.0;
    for (int ji = 0; ji < N; ji++)
        for (int jj = 0; jj < N; jj++)
            for (int ki = 0; ki <= ji; ki++)
                for (int kj = 0; kj <= jj; kj++) pw[ki * N + kj] += c[ji][jj] * a[ji][ki] * a[jj][kj];
    double* o = tiles + (size_t)f * (T1_SIZE + T2_SIZE) + (which == 1 ? 0 : T1_SIZE) + ((size_t)tid * 3 + q) * N * N;
    for (int k = 0; k < N * N; k++) o[k] = pw[k];
}

void launch_fd_tiles(int F, const FdParams* fd, double* tiles, double* scratch, cudaStream_t s) {
    k_fd_nodes<<<dim3((NODES + 127) / 128, F), 128, 0, s>>>(F, fd, scratch);
    int nfit = 3 * (TS * TW + TS * TV);
    k_fd_fit<<<dim3((nfit + 63) / 64, F), 64, 0, s>>>(F, scratch, tiles);
}

// green_fin.rs:937-952 fin_point, planes [F][FP_PLANES][N]: d a b c, then cos, sin k_n (z + h)
__global__ void k_fin_points(PanelsView pv, int F, const FdParams* __restrict__ fdp, double* __restrict__ fpt) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    int f = blockIdx.y;
    if (j >= pv.N) return;
    const FdParams& fd = fdp[f];
    int N = pv.N;
    double z = pv.at(P_C + 2, j), h = fd.h, k0 = fd.k0;
    double* o = fpt + (size_t)f * FP_PLANES * N;
    double d = 0, a = 0, b = 0, c = 0;
    if (fd.mode == 0) {
        d = exp(k0 * z);
        a = exp(-k0 * (z + h));
        b = exp(-k0 * (h - z));
        c = exp(-k0 * (z + 2.0 * h));
    }
    o[0 * N + j] = d;
    o[1 * N + j] = a;
    o[2 * N + j] = b;
    o[3 * N + j] = c;
    for (int n = 0; n < FIN_ROOTS; n++) {
        double sn, cn;
        sincos(fd.kn[n] * (z + h), &sn, &cn);
        o[(4 + 2 * n) * N + j] = cn;
        o[(5 + 2 * n) * N + j] = sn;
    }
}

void launch_fin_points(const PanelsView& pv, int F, const FdParams* fd, double* fpt, cudaStream_t s) {
    k_fin_points<<<dim3((pv.N + 127) / 128, F), 128, 0, s>>>(pv, F, fd, fpt);
}

// ------------------------------------------------------------------ assembly
// low_order.rs:738-769 apply_kernel + 781-790 kind_column: (S, D-column) of panel j at x.
__device__ __forceinline__ void apply_kernel(double rs, double rd, double dl, double dd, double area, double nx,
                                             double ny, double nz, int kindj, const double* x, const double* cj,
                                             double K, double logc, const Kern& k, double R, bool swapped,
                                             double2& S, double2& D) {
    double a = R > 0.0 ? ((x[0] - cj[0]) * nx + (x[1] - cj[1]) * ny) / R : 0.0;
    double rz = swapped ? k.Wrz : k.WrZ;
    double iz = swapped ? k.Wiz : k.WiZ;
    S.x = rs + area * k.Wr - 2.0 * K * logc * dl;
    S.y = area * k.Wi;
    D.x = rd + area * (-k.WrR * a + rz * nz) - 2.0 * K * logc * dd;
    D.y = area * (-k.WiR * a + iz * nz);
    if (kindj == 1) {  // interior free surface: K S (dG/dzeta = K G on zeta = 0)
        D.x = K * S.x;
        D.y = K * S.y;
    }
}

__device__ __forceinline__ double free_term(int kind) { return kind == 1 ? -4.0 * PI : 2.0 * PI; }

// One tile pair (K0 <= N0) of 32 x 32 panels for one frequency: the pair kernel once per
// unordered pair (G(x, xi) = G(xi, x), the swapped source derivative for (n, k):
// lo_frequency.rs:399-537), the (n, k) statics read and the (n, k) entries written through shared
// memory transposes so that every global access is coalesced along the rows.
// Output policies of the assembly: complex128 column-major N x N (the FP64 form), or two FP32 planes
// column-major with leading dimension Np (the mixed form; entry (k, n) at n Np + k).
struct OutF64 {
    static constexpr bool kF32 = false;  // FP64 coefficient tables
    static constexpr int kT1 = T1_SIZE, kT2 = T2_SIZE;
    using Tile = double;
    double2* S;
    double2* A;
    size_t stride;
    int N;
    __device__ __forceinline__ void put(int f, int k, int n, double2 s, double2 a) const {
        size_t o = (size_t)f * stride + (size_t)k + (size_t)n * N;
        S[o] = s;
        A[o] = a;
    }
};

struct OutF32 {
    static constexpr bool kF32 = true;  // FP32 coefficient tables and tiles
    static constexpr int kT1 = T1F_SIZE, kT2 = T2F_SIZE;
    using Tile = float;
    float* S;
    float* A;
    size_t bstride;  // per frequency: two planes of Np * Np
    int Np;
    __device__ __forceinline__ void put(int f, int k, int n, double2 s, double2 a) const {
        size_t o = (size_t)f * bstride + (size_t)n * Np + k, pl = (size_t)Np * Np;
        S[o] = (float)s.x;
        S[o + pl] = (float)s.y;
        A[o] = (float)a.x;
        A[o + pl] = (float)a.y;
    }
};

// Symmetry sectors (SECT, G = pv.G > 1): block y = f G + g assembles the image block g of frequency f,
// M_g(k, n) = S(x_k, panel g n), over the Ns = N / G sector panels; a reflection keeps depths and
// horizontal distances, so (k, g n) and (n, g k) still share one pair kernel.  The statics of the image
// block are the Ns x Ns block g of the Ns x N statics; the free term sits on the diagonal of block 0.
// k_sectors then combines the G blocks of a frequency into its G sector matrices.
template <bool FINITE, class Out, bool SECT>
__global__ void __launch_bounds__(256, Out::kF32 ? 3 : 2) k_assemble(PanelsView pv, const double* __restrict__ st,
                                                  const FreqInfo* __restrict__ fi, const FdParams* __restrict__ fdp,
                                                  const typename Out::Tile* __restrict__ tiles,
                                                  const double* __restrict__ fpt, Out out) {
    // statics (n, k) [q][k_local][n_local]; each (k_local, n_local) slot is read and then
    // overwritten with the results (S, A) of entry (n, k) by the one thread that owns it
    __shared__ double sT[4][32][33];
    if (pv.invalid()) return;  // invalid panels: the solve reports them
    const int G = SECT ? pv.G : 1, Nf = pv.N, N = SECT ? Nf / G : Nf;
    const int nt = (N + 31) / 32;
    // tile pair from the linear index: row-block kb <= column-block nb
    int idx = blockIdx.x, kb = 0;
    while (idx >= nt - kb) {
        idx -= nt - kb;
        kb++;
    }
    const int nb = kb + idx;
    const int y = blockIdx.y, f = SECT ? y / G : y, g = SECT ? y - f * G : 0;
    const int K0 = kb * 32, N0 = nb * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const size_t NN = (size_t)N * Nf;  // one statics plane
    const double* stg = st + (size_t)g * N * N;
    const FreqInfo info = fi[f];
    const double K = info.K, logc = info.logc;
    // statics of (n, g k): rows n in N0, panels k in K0
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int n = N0 + tx, k = K0 + ty + 8 * i;
        if (n < N && k < N)
#pragma unroll
            for (int q = 0; q < 4; q++) sT[q][ty + 8 * i][tx] = __ldg(stg + q * NN + (size_t)n + (size_t)k * N);
    }
    __syncthreads();
    const int k = K0 + tx;
    // xk: the field point of row k; ck, nk, ak: panel g k (the source of entry (n, g k)); kept in shared
    // memory (read where used: short live ranges instead of ten doubles held across the pairs)
    __shared__ double sKd[10][32], sNd[10][32];
    __shared__ int sKind[32], sNKind[32];
    if (ty == 1) {  // the same for the column panels n = N0 + tx: xn, cn, nn, an
        const int nn = N0 + tx;
        double xn[3] = {0, 0, 0}, cn[3] = {0, 0, 0}, nv3[3] = {0, 0, 0}, an = 0;
        int kindn = 0;
        if (nn < N) {
            const int gn = g * N + nn;
            for (int d = 0; d < 3; d++) {
                cn[d] = pv.at(P_C + d, gn);
                nv3[d] = pv.at(P_N + d, gn);
                xn[d] = SECT ? pv.at(P_C + d, nn) : cn[d];
            }
            an = pv.at(P_AREA, gn);
            kindn = pv.kind[nn];
        }
        for (int d = 0; d < 3; d++) sNd[d][tx] = xn[d], sNd[3 + d][tx] = cn[d], sNd[6 + d][tx] = nv3[d];
        sNd[9][tx] = an;
        sNKind[tx] = kindn;
    }
    if (ty == 0) {
        double xk[3] = {0, 0, 0}, ck[3] = {0, 0, 0}, nk[3] = {0, 0, 0}, ak = 0;
        int kindk = 0;
        if (k < N) {
            const int gk = g * N + k;
            for (int d = 0; d < 3; d++) {
                ck[d] = pv.at(P_C + d, gk);
                nk[d] = pv.at(P_N + d, gk);
                xk[d] = SECT ? pv.at(P_C + d, k) : ck[d];
            }
            ak = pv.at(P_AREA, gk);
            kindk = pv.kind[k];
        }
        for (int d = 0; d < 3; d++) sKd[d][tx] = xk[d], sKd[3 + d][tx] = ck[d], sKd[6 + d][tx] = nk[d];
        sKd[9][tx] = ak;
        sKind[tx] = kindk;
    }
    __syncthreads();
    const volatile double(*vK)[32] = sKd;
    const volatile double(*vN)[32] = sNd;
    const FdParams* fd = FINITE ? fdp + f : nullptr;
    const typename Out::Tile* T1 = FINITE ? tiles + (size_t)f * (Out::kT1 + Out::kT2) : nullptr;
    const typename Out::Tile* T2 = FINITE ? T1 + Out::kT1 : nullptr;
    const double* fp = FINITE ? fpt + (size_t)f * FP_PLANES * Nf : nullptr;
#pragma unroll 1
    for (int i = 0; i < 4; i++) {
        const int nl = ty + 8 * i, n = N0 + nl;
        bool live = k < N && n < N && (kb != nb || k <= n);
        if (!live) continue;
        // cn, nn3, an: panel g n (the source of entry (k, g n)); xn: the field point of row n
        // R without contraction: the finite-depth kernel switches form at R = h/2 exactly
        const double xk[3] = {vK[0][tx], vK[1][tx], vK[2][tx]};
        double R, zn;
        {
            const double dx = xk[0] - vN[3][nl], dy = xk[1] - vN[4][nl];
            R = sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
            zn = vN[5][nl];
        }
        Kern w;
        if (FINITE) {
            w = finite_kernel<Out::kF32>(*fd, T1, T2, R, xk[2], zn, fp + k, fp + n, Nf);
        } else {
            w = pair_kernel_inf<Out::kF32>(K, R, xk[2], zn);
        }
        const double xn[3] = {vN[0][nl], vN[1][nl], vN[2][nl]}, cn[3] = {vN[3][nl], vN[4][nl], vN[5][nl]};
        const double nn3[3] = {vN[6][nl], vN[7][nl], vN[8][nl]}, an = vN[9][nl];
        const int kindn = sNKind[nl];
        // entry (k, n): the field point x_k against panel g n
        size_t o1 = (size_t)k + (size_t)n * N;
        double2 s1, d1;
        {
            const double xk2[3] = {vK[0][tx], vK[1][tx], vK[2][tx]};
            apply_kernel(__ldg(stg + o1), __ldg(stg + NN + o1), __ldg(stg + 2 * NN + o1), __ldg(stg + 3 * NN + o1),
                         an, nn3[0], nn3[1], nn3[2], kindn, xk2, cn, K, logc, w, R, false, s1, d1);
        }
        out.put(y, k, n, s1, make_double2((g == 0 && k == n ? free_term(sKind[tx]) : 0.0) - d1.x, -d1.y));
        if (n != k) {
            double2 s2, d2;
            const double ck[3] = {vK[3][tx], vK[4][tx], vK[5][tx]};
            apply_kernel(sT[0][tx][nl], sT[1][tx][nl], sT[2][tx][nl], sT[3][tx][nl], vK[9][tx], vK[6][tx], vK[7][tx],
                         vK[8][tx], sKind[tx], xn, ck, K, logc, w, R, true, s2, d2);
            sT[0][tx][nl] = s2.x;
            sT[1][tx][nl] = s2.y;
            sT[2][tx][nl] = -d2.x;
            sT[3][tx][nl] = -d2.y;
        }
    }
    __syncthreads();
    // write the (n, k) entries: n = N0 + tx (coalesced), k = K0 + ty + 8 i
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int n = N0 + tx, kl = ty + 8 * i, kk = K0 + kl;
        if (n < N && kk < N && (kb != nb || n > kk))
            out.put(y, n, kk, make_double2(sT[0][kl][tx], sT[1][kl][tx]), make_double2(sT[2][kl][tx], sT[3][kl][tx]));
    }
}

template <class Out>
static void assemble(const PanelsView& pv, const double* st, int F, const FreqInfo* fi, const FdParams* fd,
                     const typename Out::Tile* tiles, const double* fpt, bool finite, Out o, cudaStream_t s) {
    const int nt = (pv.N / pv.G + 31) / 32;
    dim3 grid(nt * (nt + 1) / 2, F * pv.G), blk(32, 8);
    if (pv.G > 1) {
        if (finite)
            k_assemble<true, Out, true><<<grid, blk, 0, s>>>(pv, st, fi, fd, tiles, fpt, o);
        else
            k_assemble<false, Out, true><<<grid, blk, 0, s>>>(pv, st, fi, fd, tiles, fpt, o);
    } else if (finite) {
        k_assemble<true, Out, false><<<grid, blk, 0, s>>>(pv, st, fi, fd, tiles, fpt, o);
    } else {
        k_assemble<false, Out, false><<<grid, blk, 0, s>>>(pv, st, fi, fd, tiles, fpt, o);
    }
}

void launch_assemble_f64(const PanelsView& pv, const double* st, int F, const FreqInfo* fi, const FdParams* fd,
                         const double* tiles, const double* fpt, bool finite, double2* S, double2* A,
                         size_t mat_stride, cudaStream_t s) {
    assemble(pv, st, F, fi, fd, tiles, fpt, finite, OutF64{S, A, mat_stride, pv.N / pv.G}, s);
}

// ------------------------------------------------------------------ field points
// The fin_point data of the panels' depths followed by those of the field points, planes of N + P per
// frequency (green_fin.rs:937-952), so that the finite-depth pair kernel reads both with one stride.
__global__ void k_field_fin(PanelsView pv, const double* __restrict__ pts, int P, int F,
                            const FdParams* __restrict__ fdp, double* __restrict__ fq) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x, f = blockIdx.y, N = pv.N, L = N + P;
    if (t >= L || f >= F) return;
    const FdParams& fd = fdp[f];
    const double z = t < N ? pv.at(P_C + 2, t) : pts[3 * (t - N) + 2], h = fd.h, k0 = fd.k0;
    double* o = fq + (size_t)f * FP_PLANES * L + t;
    double d = 0, a = 0, b = 0, c = 0;
    if (fd.mode == 0) {
        d = exp(k0 * z);
        a = exp(-k0 * (z + h));
        b = exp(-k0 * (h - z));
        c = exp(-k0 * (z + 2.0 * h));
    }
    o[0] = d;
    o[(size_t)L] = a;
    o[2 * (size_t)L] = b;
    o[3 * (size_t)L] = c;
    for (int n = 0; n < FIN_ROOTS; n++) {
        double sn, cn;
        sincos(fd.kn[n] * (z + h), &sn, &cn);
        o[(size_t)(4 + 2 * n) * L] = cn;
        o[(size_t)(5 + 2 * n) * L] = sn;
    }
}

void launch_field_fin(const PanelsView& pv, const double* pts, int P, int F, const FdParams* fd, double* fq,
                      cudaStream_t s) {
    k_field_fin<<<dim3((pv.N + P + 127) / 128, F), 128, 0, s>>>(pv, pts, P, F, fd, fq);
}

// lo_frequency.rs:1392-1470 field_values at one point (block) of one frequency: over the panels (the
// interior ones take no part) the influence (S, D) of panel j at the point, from the point's statics row
// and the FP64 pair kernel; per radiation column c the sum of phi_c D - S u_c, per heading the sum of
// (phi_S + phi_I) D; then the elevation (z = 0) or p / (rho g): radiation w^2/g (1/4 pi) sum, incident
// (-i w / g) phi_I(x), scattered (-i w / g) (1/4 pi) sum, and their total.  The sums: per thread over
// its panels, then warp shuffles and the warps in a fixed order (deterministic).
constexpr int FIELD_COLS = 32;

template <bool FINITE>
__global__ void __launch_bounds__(256) k_field(PanelsView pv, const double* __restrict__ pts, int P,
                                               const double* __restrict__ stp, const FreqInfo* __restrict__ fi,
                                               const FdParams* __restrict__ fdp, const double* __restrict__ tiles,
                                               const double* __restrict__ fq, int H, const double* __restrict__ heads,
                                               double depth, double grav, const double2* __restrict__ phi, int ldphi,
                                               const double2* __restrict__ u, const double2* __restrict__ phiI,
                                               double2* __restrict__ frad, double2* __restrict__ finc,
                                               double2* __restrict__ fsca, double2* __restrict__ fdif) {
    __shared__ double2 red[8][FIELD_COLS];
    const int p = blockIdx.x, f = blockIdx.y, N = pv.N, nrad = 6 * pv.nbod, nrhs = nrad + H;
    const double x[3] = {pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]};
    const FreqInfo info = fi[f];
    const double K = info.K, logc = info.logc;
    const size_t NP = (size_t)P * N;
    const double2* ph = phi + (size_t)f * nrhs * ldphi;
    const double2* uf = u + (size_t)f * nrhs * N;
    const double2* pI = phiI + (size_t)f * H * N;
    const double* T1 = FINITE ? tiles + (size_t)f * (T1_SIZE + T2_SIZE) : nullptr;
    const double* fqf = FINITE ? fq + (size_t)f * FP_PLANES * (N + P) : nullptr;
    double2 acc[FIELD_COLS];
#pragma unroll
    for (int c = 0; c < FIELD_COLS; c++) acc[c] = make_double2(0.0, 0.0);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        if (pv.kind[j] != 0) continue;
        const double cj[3] = {pv.at(P_C, j), pv.at(P_C + 1, j), pv.at(P_C + 2, j)};
        const double dx = x[0] - cj[0], dy = x[1] - cj[1];
        const double R = sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
        const Kern w = FINITE ? finite_kernel<false>(fdp[f], T1, T1 + T1_SIZE, R, x[2], cj[2], fqf + N + p, fqf + j, N + P)
                              : pair_kernel_inf<false>(K, R, x[2], cj[2]);
        const size_t o = (size_t)p + (size_t)j * P;
        double2 S, D;
        apply_kernel(stp[o], stp[NP + o], stp[2 * NP + o], stp[3 * NP + o], pv.at(P_AREA, j), pv.at(P_N, j),
                     pv.at(P_N + 1, j), pv.at(P_N + 2, j), 0, x, cj, K, logc, w, R, false, S, D);
#pragma unroll
        for (int c = 0; c < FIELD_COLS; c++) {
            if (c >= nrhs) break;
            double2 v = ph[(size_t)c * ldphi + j];
            if (c < nrad) {  // phi_c D - S u_c
                const double2 uc = uf[(size_t)c * N + j];
                acc[c].x += v.x * D.x - v.y * D.y - (S.x * uc.x - S.y * uc.y);
                acc[c].y += v.x * D.y + v.y * D.x - (S.x * uc.y + S.y * uc.x);
            } else {  // (phi_S + phi_I) D on the wetted panels
                const double2 vi = pI[(size_t)(c - nrad) * N + j];
                v.x += vi.x;
                v.y += vi.y;
                acc[c].x += v.x * D.x - v.y * D.y;
                acc[c].y += v.x * D.y + v.y * D.x;
            }
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < FIELD_COLS; c++) {
        double a = acc[c].x, b = acc[c].y;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane == 0) red[warp][c] = make_double2(a, b);
    }
    __syncthreads();
    const int c = threadIdx.x;
    if (c >= nrhs) return;
    double2 v = make_double2(0.0, 0.0);
    for (int w8 = 0; w8 < (int)(blockDim.x >> 5); w8++) {
        v.x += red[w8][c].x;
        v.y += red[w8][c].y;
    }
    const double wv = info.omega, q = 1.0 / (4.0 * PI);
    if (c < nrad) {
        const double s = wv * wv / grav * q;
        frad[((size_t)f * P + p) * nrad + c] = make_double2(s * v.x, s * v.y);
        return;
    }
    // the incident wave at the point (low_order.rs:1441-1459), as the boundary values
    const int h = c - nrad;
    const double k = info.k;
    double Z = exp(k * x[2]);
    if (depth > 0.0) Z = (Z + exp(-k * (x[2] + 2.0 * depth))) / (1.0 + exp(-2.0 * k * depth));
    double sb, cb;
    sincos(heads[h], &sb, &cb);
    double sp, cp;
    sincos(-k * (x[0] * cb + x[1] * sb), &sp, &cp);
    const double pir = -(grav / wv) * sp * Z, pii = (grav / wv) * cp * Z;
    // (-i w / g) times phi_I and times phi_S = v / 4 pi
    const double2 ei = make_double2(wv / grav * pii, -wv / grav * pir);
    const double2 es = make_double2(wv / grav * q * v.y, -wv / grav * q * v.x);
    const size_t oh = ((size_t)f * P + p) * H + h;
    finc[oh] = ei;
    fsca[oh] = es;
    fdif[oh] = make_double2(ei.x + es.x, ei.y + es.y);
}

void launch_field(const PanelsView& pv, const double* pts, int P, const double* stp, int F, const FreqInfo* fi,
                  const FdParams* fd, const double* tiles, const double* fq, bool finite, int H, const double* heads,
                  double depth, double grav, const double2* phi, int ldphi, const double2* u, const double2* phiI,
                  double2* frad, double2* finc, double2* fsca, double2* fdif, cudaStream_t s) {
    if (finite)
        k_field<true><<<dim3(P, F), 256, 0, s>>>(pv, pts, P, stp, fi, fd, tiles, fq, H, heads, depth, grav, phi, ldphi,
                                                 u, phiI, frad, finc, fsca, fdif);
    else
        k_field<false><<<dim3(P, F), 256, 0, s>>>(pv, pts, P, stp, fi, fd, tiles, fq, H, heads, depth, grav, phi,
                                                  ldphi, u, phiI, frad, finc, fsca, fdif);
}

// ------------------------------------------------------------------ symmetry sectors
// Characters of the reflection group, elements e, x, y, xy reflections (lo_geometry.rs:25-36):
// chi_c(g) = (-1)^popc(c & g) for G = 2 and 4.
__device__ __forceinline__ bool chi_neg(int c, int g) { return __popc(c & g) & 1; }

// The G image blocks M_g of each frequency (matrices f G .. f G + G - 1 of S and of A) replaced in
// place by the sector matrices sum_g chi_c(g) M_g (lo_frequency.rs:276-346: S_c(k, n) =
// sum_g chi_c(g) S(k, g n), A_c likewise; the free term of block 0 enters every sector).  Entries
// (k, n) < Nm of `nplanes` planes, each entry `comps` consecutive T at (n ld + k) comps; sums in FP64.
template <typename T>
__global__ void k_sectors(T* __restrict__ S, T* __restrict__ A, int G, int Nm, int ld, int comps, size_t plane,
                          int nplanes, size_t mstride) {
    const int f = blockIdx.y;
    const size_t per = (size_t)Nm * Nm * comps * nplanes;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < 2 * per; t += (size_t)gridDim.x * blockDim.x) {
        const size_t e = t < per ? t : t - per;
        T* M = t < per ? S : A;
        const int c = (int)(e % comps);
        const size_t r = e / comps;
        const int k = (int)(r % Nm), n = (int)((r / Nm) % Nm), p = (int)(r / ((size_t)Nm * Nm));
        T* b = M + (size_t)f * G * mstride + (size_t)p * plane + ((size_t)n * ld + k) * comps + c;
        double v[4];
        for (int g = 0; g < G; g++) v[g] = (double)b[(size_t)g * mstride];
        for (int cc = 0; cc < G; cc++) {
            double w = 0.0;
            for (int g = 0; g < G; g++) w += chi_neg(cc, g) ? -v[g] : v[g];
            b[(size_t)cc * mstride] = (T)w;
        }
    }
}

void launch_sectors_f64(double2* S, double2* A, int F, int G, int Nm, size_t mat_stride, cudaStream_t s) {
    k_sectors<double><<<dim3(296, F), 256, 0, s>>>(reinterpret_cast<double*>(S), reinterpret_cast<double*>(A), G, Nm,
                                                    Nm, 2, 0, 1, 2 * mat_stride);
}

void launch_sectors_f32(float* S, float* A, int F, int G, int Nm, int Np, cudaStream_t s) {
    const size_t plane = (size_t)Np * Np;
    k_sectors<float><<<dim3(296, F), 256, 0, s>>>(S, A, G, Nm, Np, 1, plane, 2, 2 * plane);
}

// Right-hand-side vectors projected on the sectors (lo_frequency.rs:875-884): up[f G + c][col][n] =
// (1/G) sum_g chi_c(g) u[f][col][g Nm + n]; u holds every panel (Nf = G Nm), up has leading dimension ldp.
__global__ void k_project(const double2* __restrict__ u, double2* __restrict__ up, int G, int Nm, int nrhs, int ldp) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x, col = blockIdx.y, sys = blockIdx.z;
    if (n >= Nm) return;
    const int f = sys / G, c = sys - f * G, Nf = G * Nm;
    const double2* uf = u + ((size_t)f * nrhs + col) * Nf + n;
    double re = 0.0, im = 0.0;
    for (int g = 0; g < G; g++) {
        const double2 v = uf[(size_t)g * Nm];
        re += chi_neg(c, g) ? -v.x : v.x;
        im += chi_neg(c, g) ? -v.y : v.y;
    }
    up[((size_t)sys * nrhs + col) * ldp + n] = make_double2(re / G, im / G);
}

void launch_project(const double2* u, double2* up, int F, int G, int Nm, int nrhs, int ldp, cudaStream_t s) {
    k_project<<<dim3((Nm + 127) / 128, nrhs, F * G), 128, 0, s>>>(u, up, G, Nm, nrhs, ldp);
}

// The potentials on every panel from the sector solutions (lo_frequency.rs:931-943):
// phi[f][col][g Nm + n] = sum_c chi_c(g) x[f G + c][col][n] (x with leading dimension ldx).
__global__ void k_recombine(const double2* __restrict__ x, double2* __restrict__ phi, int G, int Nm, int nrhs,
                            int ldx) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x, col = blockIdx.y, f = blockIdx.z / G,
              g = blockIdx.z - f * G;
    if (n >= Nm) return;
    double re = 0.0, im = 0.0;
    for (int c = 0; c < G; c++) {
        const double2 v = x[((size_t)(f * G + c) * nrhs + col) * ldx + n];
        re += chi_neg(c, g) ? -v.x : v.x;
        im += chi_neg(c, g) ? -v.y : v.y;
    }
    phi[((size_t)f * nrhs + col) * G * Nm + (size_t)g * Nm + n] = make_double2(re, im);
}

void launch_recombine(const double2* x, double2* phi, int F, int G, int Nm, int nrhs, int ldx, cudaStream_t s) {
    k_recombine<<<dim3((Nm + 127) / 128, nrhs, F * G), 128, 0, s>>>(x, phi, G, Nm, nrhs, ldx);
}

// The finite-depth tiles of a batch for the mixed form: per tile and quantity (one thread each) the
// power-basis block of degree TN - 1 taken back to Chebyshev coefficients, the series truncated to
// degree TFD in each variable, returned to the power basis and rounded to FP32.
__global__ void k_tiles_f32(int F, const double* __restrict__ a, float* __restrict__ b) {
    constexpr int N = TN, M = TFN, BLOCKS = 3 * (TS * TW + TS * TV);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = t / BLOCKS, blk = t % BLOCKS;
    if (f >= F) return;
    // cp[j][k]: coefficient of t^k in the Chebyshev polynomial T_j
    double cp[N][N];
    for (int j = 0; j < N; j++)
        for (int k = 0; k < N; k++) cp[j][k] = 0.0;
    cp[0][0] = 1.0;
    cp[1][1] = 1.0;
    for (int j = 2; j < N; j++)
        for (int k = 0; k < N; k++) cp[j][k] = (k > 0 ? 2.0 * cp[j - 1][k - 1] : 0.0) - cp[j - 2][k];
    double c[N][N];
    const double* p = a + (size_t)f * (T1_SIZE + T2_SIZE) + (size_t)blk * N * N;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) c[i][j] = p[i * N + j];
    // power -> Chebyshev along the second variable (rows), then the first (columns): the triangular
    // system p_k = sum_j c_j cp[j][k], solved from the top degree down
    for (int i = 0; i < N; i++)
        for (int j = N - 1; j >= 0; j--) {
            double cj = c[i][j] / cp[j][j];
            for (int k = 0; k < j; k++) c[i][k] -= cj * cp[j][k];
            c[i][j] = cj;
        }
    for (int j = 0; j < N; j++)
        for (int i = N - 1; i >= 0; i--) {
            double ci = c[i][j] / cp[i][i];
            for (int k = 0; k < i; k++) c[k][j] -= ci * cp[i][k];
            c[i][j] = ci;
        }
    // the truncated series back in the power basis
    float* o = b + (size_t)f * (T1F_SIZE + T2F_SIZE) + (size_t)blk * TFB;
    for (int ki = 0; ki < M; ki++)
        for (int kj = 0; kj < M; kj++) {
            double acc = 0.0;
            for (int ji = ki; ji < M; ji++)
                for (int jj = kj; jj < M; jj++) acc += c[ji][jj] * cp[ji][ki] * cp[jj][kj];
            o[ki * M + kj] = (float)acc;
        }
    for (int k = M * M; k < TFB; k++) o[k] = 0.f;
}

void launch_tiles_f32(int F, const double* tiles, float* tiles_f, cudaStream_t s) {
    int n = F * 3 * (TS * TW + TS * TV);
    k_tiles_f32<<<(n + 127) / 128, 128, 0, s>>>(F, tiles, tiles_f);
}

void launch_assemble_f32(const PanelsView& pv, const double* st, int F, const FreqInfo* fi, const FdParams* fd,
                         const float* tiles, const double* fpt, bool finite, float* S, float* A, int Np,
                         cudaStream_t s) {
    assemble(pv, st, F, fi, fd, tiles, fpt, finite, OutF32{S, A, 2 * (size_t)Np * Np, Np}, s);
}

// ------------------------------------------------------------------ boundary values
// low_order.rs:1401-1459 depth factor and incident wave; lo_frequency.rs:214-273 boundary values
// (scattered formulation, one rigid body, rotation centre at the origin).
__global__ void k_boundary(PanelsView pv, int F, const FreqInfo* __restrict__ fi, int H,
                           const double* __restrict__ heads, double depth, double grav, double2* __restrict__ u,
                           double2* __restrict__ phiI) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    int f = blockIdx.y;
    int N = pv.N;
    if (j >= N) return;
    const int nrad = 6 * pv.nbod, nrhs = nrad + H;
    double c[3], n[3];
    for (int d = 0; d < 3; d++) {
        c[d] = pv.at(P_C + d, j);
        n[d] = pv.at(P_N + d, j);
    }
    bool wet = pv.kind[j] == 0;
    double2* uf = u + (size_t)f * nrhs * N;
    // radiation columns: the generalized normal of each rigid mode of each body (lo_frequency.rs:236-251)
    for (int m = 0; m < nrad; m++) uf[(size_t)m * N + j] = make_double2(wet ? pv.gen_normal(j, m) : 0.0, 0.0);
    double k = fi[f].k, w = fi[f].omega;
    double Z = exp(k * c[2]), Zz = k * Z;
    if (depth > 0.0) {
        double b = exp(-k * (c[2] + 2.0 * depth));
        double dd = 1.0 + exp(-2.0 * k * depth);
        Zz = k * (Z - b) / dd;
        Z = (Z + b) / dd;
    }
    for (int h = 0; h < H; h++) {
        double sb, cb;
        sincos(heads[h], &sb, &cb);
        double phase = -k * (c[0] * cb + c[1] * sb);
        double sp, cp;
        sincos(phase, &sp, &cp);
        // e = (i g / w) (cos + i sin)
        double er = -(grav / w) * sp, ei = (grav / w) * cp;
        double pr = er * Z, pi = ei * Z;
        // grad: phi (-i k cb), phi (-i k sb), e Zz ; dphi/dn
        double gxr = pi * k * cb, gxi = -pr * k * cb;
        double gyr = pi * k * sb, gyi = -pr * k * sb;
        double gzr = er * Zz, gzi = ei * Zz;
        double dr = gxr * n[0] + gyr * n[1] + gzr * n[2];
        double di = gxi * n[0] + gyi * n[1] + gzi * n[2];
        phiI[((size_t)f * H + h) * N + j] = make_double2(pr, pi);
        uf[(size_t)(nrad + h) * N + j] = make_double2(wet ? -dr : 0.0, wet ? -di : 0.0);
    }
}

void launch_boundary(const PanelsView& pv, int F, const FreqInfo* fi, int H, const double* heads, double depth,
                     double grav, double2* u, double2* phiI, cudaStream_t s) {
    k_boundary<<<dim3((pv.N + 127) / 128, F), 128, 0, s>>>(pv, F, fi, H, heads, depth, grav, u, phiI);
}

// ------------------------------------------------------------------ right-hand sides -S u
// One thread per row k holds the nrhs sums; S is read once, column by column (coalesced along k),
// u staged in shared memory (lo_frequency.rs:875-892: the product S U with U = -u).
template <int NR>
__global__ void __launch_bounds__(128) k_rhs_f64(int N, int nrhs, const double2* __restrict__ S, size_t mat_stride,
                                                 const double2* __restrict__ u, double2* __restrict__ rhs) {
    constexpr int CH = 32;
    __shared__ double2 su[CH][NR];
    int f = blockIdx.y;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    const double2* Sf = S + (size_t)f * mat_stride;
    const double2* uf = u + (size_t)f * nrhs * N;
    double2 acc[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = make_double2(0.0, 0.0);
    for (int n0 = 0; n0 < N; n0 += CH) {
        __syncthreads();
        for (int t = threadIdx.x; t < CH * NR; t += blockDim.x) {
            int nn = t % CH, c = t / CH;
            su[nn][c] = (n0 + nn < N && c < nrhs) ? uf[(size_t)c * N + n0 + nn] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        if (k < N) {
            int lim = min(CH, N - n0);
            for (int nn = 0; nn < lim; nn++) {
                double2 s = Sf[(size_t)k + (size_t)(n0 + nn) * N];
#pragma unroll
                for (int c = 0; c < NR; c++) {
                    double2 v = su[nn][c];
                    acc[c].x += s.x * v.x - s.y * v.y;
                    acc[c].y += s.x * v.y + s.y * v.x;
                }
            }
        }
    }
    if (k < N)
        for (int c = 0; c < nrhs && c < NR; c++) rhs[((size_t)f * nrhs + c) * N + k] = make_double2(-acc[c].x, -acc[c].y);
}

void launch_rhs_f64(int N, int F, int nrhs, const double2* S, size_t mat_stride, const double2* u, double2* rhs,
                    cudaStream_t s) {
    dim3 grid((N + 127) / 128, F);
    if (nrhs <= 8)
        k_rhs_f64<8><<<grid, 128, 0, s>>>(N, nrhs, S, mat_stride, u, rhs);
    else if (nrhs <= 16)
        k_rhs_f64<16><<<grid, 128, 0, s>>>(N, nrhs, S, mat_stride, u, rhs);
    else
        k_rhs_f64<32><<<grid, 128, 0, s>>>(N, nrhs, S, mat_stride, u, rhs);
}

// ------------------------------------------------------------------ forces
// lo_frequency.rs:1039-1115: z = sum_j n_i phi_c A_j over the wetted panels; A = Re(-rho z),
// B = -w Im(-rho z); X = i w rho sum n_i (phi_S + phi_I) A_j, FK the phi_I part, SC = X - FK.
// One block per (column, body, frequency): each thread accumulates the body's six coordinates (and for a
// diffraction column the incident part beside the total) over its panels in one pass, then warp
// shuffles and a fixed-order sum over the warps (deterministic).
__global__ void __launch_bounds__(256) k_forces(PanelsView pv, const FreqInfo* __restrict__ fi, int H,
                                                const double2* __restrict__ phi, int ldphi,
                                                const double2* __restrict__ phiI,
                                                double rho, double* __restrict__ Aout, double* __restrict__ Bout,
                                                double2* __restrict__ X, double2* __restrict__ FK,
                                                double2* __restrict__ SC) {
    __shared__ double red[8][24];
    const int col = blockIdx.x, b = blockIdx.y, f = blockIdx.z, N = pv.N;
    const int D = 6 * pv.nbod, nrhs = D + H;
    const bool diff = col >= D;
    const double2* pc = phi + ((size_t)f * nrhs + col) * ldphi;
    const double2* pI = diff ? phiI + ((size_t)f * H + (col - D)) * N : nullptr;
    const double r0 = pv.rcen ? pv.rcen[3 * b] : 0.0, r1 = pv.rcen ? pv.rcen[3 * b + 1] : 0.0,
                 r2 = pv.rcen ? pv.rcen[3 * b + 2] : 0.0;
    double acc[24];
#pragma unroll
    for (int k = 0; k < 24; k++) acc[k] = 0.0;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        if (pv.kind[j] != 0 || (pv.body ? pv.body[j] : 0) != b) continue;
        const double nx = pv.at(P_N, j), ny = pv.at(P_N + 1, j), nz = pv.at(P_N + 2, j);
        const double cx = pv.at(P_C, j) - r0, cy = pv.at(P_C + 1, j) - r1, cz = pv.at(P_C + 2, j) - r2;
        const double ar = pv.at(P_AREA, j);
        const double nj[6] = {nx, ny, nz, cy * nz - cz * ny, cz * nx - cx * nz, cx * ny - cy * nx};
        double2 v = pc[j], vi = make_double2(0.0, 0.0);
        if (diff) {
            vi = pI[j];
            v.x += vi.x;
            v.y += vi.y;
        }
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const double wgt = nj[m] * ar;
            acc[2 * m] += wgt * v.x;
            acc[2 * m + 1] += wgt * v.y;
            acc[12 + 2 * m] += wgt * vi.x;
            acc[12 + 2 * m + 1] += wgt * vi.y;
        }
    }
    const int nv = diff ? 24 : 12, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 24; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    __shared__ double tot[24];
    if (threadIdx.x < nv) {
        double t = 0.0;
        for (int w8 = 0; w8 < (int)(blockDim.x >> 5); w8++) t += red[w8][threadIdx.x];
        tot[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int m = threadIdx.x, i = 6 * b + m;
        const double w = fi[f].omega;
        const double sr = tot[2 * m], si = tot[2 * m + 1];
        if (!diff) {
            Aout[((size_t)f * D + i) * D + col] = -rho * sr;
            Bout[((size_t)f * D + i) * D + col] = -w * (-rho * si);
        } else {
            // i w rho (sr + i si) = (-w rho si, w rho sr)
            const size_t o = ((size_t)f * H + (col - D)) * D + i;
            const double fr = tot[12 + 2 * m], fim = tot[12 + 2 * m + 1];
            const double2 x = make_double2(-w * rho * si, w * rho * sr), fk = make_double2(-w * rho * fim, w * rho * fr);
            X[o] = x;
            FK[o] = fk;
            SC[o] = make_double2(x.x - fk.x, x.y - fk.y);
        }
    }
}

void launch_forces(const PanelsView& pv, int F, const FreqInfo* fi, int H, const double2* phi, int ldphi,
                   const double2* phiI, double rho, double* A, double* B, double2* X, double2* FK, double2* SC,
                   cudaStream_t s) {
    k_forces<<<dim3(6 * pv.nbod + H, pv.nbod, F), 256, 0, s>>>(pv, fi, H, phi, ldphi, phiI, rho, A, B, X, FK, SC);
}

// ------------------------------------------------------------------ Haskind excitation
// lo_frequency.rs:1118-1171 on this route's panels (wetted and interior; interior panels take no part):
// HK(h, c) = i w rho sum over wetted j of (n_c(j) phi_I(h, j) - phi_c(j) dphi_I/dn(h, j)) A_j, with n_c the
// generalized normal of radiation column c (zero off its body) and dphi_I/dn = -u(D + h, j), the boundary
// value of diffraction column h on a wetted panel.  One block per (radiation column, frequency); the
// headings in chunks of eight, each chunk one pass over the panels, warp shuffles and a fixed-order sum
// over the warps.  Output [F][H][D] as the other exciting forces (solve_driver.rs:376-383).
__global__ void __launch_bounds__(256) k_haskind(PanelsView pv, const FreqInfo* __restrict__ fi, int H,
                                                 const double2* __restrict__ phi, int ldphi,
                                                 const double2* __restrict__ u, const double2* __restrict__ phiI,
                                                 double rho, double2* __restrict__ HK) {
    __shared__ double red[8][16];
    __shared__ double tot[16];
    const int c = blockIdx.x, f = blockIdx.y, N = pv.N;
    const int D = 6 * pv.nbod, nrhs = D + H;
    const double2* pc = phi + ((size_t)f * nrhs + c) * ldphi;
    const double2* ud = u + ((size_t)f * nrhs + D) * N;
    const double2* pI = phiI + (size_t)f * H * N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int h0 = 0; h0 < H; h0 += 8) {
        const int nh = min(8, H - h0);
        double acc[16];
#pragma unroll
        for (int k = 0; k < 16; k++) acc[k] = 0.0;
        for (int j = threadIdx.x; j < N; j += blockDim.x) {
            if (pv.kind[j] != 0) continue;
            const double ar = pv.at(P_AREA, j);
            const double nc = pv.gen_normal(j, c) * ar;
            const double2 p = pc[j];
            const double px = p.x * ar, py = p.y * ar;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (q < nh) {
                    const double2 I = pI[(size_t)(h0 + q) * N + j];
                    const double2 un = ud[(size_t)(h0 + q) * N + j];  // -dphi_I/dn
                    acc[2 * q] += nc * I.x + (px * un.x - py * un.y);
                    acc[2 * q + 1] += nc * I.y + (px * un.y + py * un.x);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 16; k++) {
            double v = acc[k];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][k] = v;
        }
        __syncthreads();
        if (threadIdx.x < 2 * nh) {
            double t = 0.0;
            for (int w8 = 0; w8 < (int)(blockDim.x >> 5); w8++) t += red[w8][threadIdx.x];
            tot[threadIdx.x] = t;
        }
        __syncthreads();
        if (threadIdx.x < nh) {
            const double w = fi[f].omega, vr = tot[2 * threadIdx.x], vi = tot[2 * threadIdx.x + 1];
            // i w rho (vr + i vi)
            HK[((size_t)f * H + h0 + threadIdx.x) * D + c] = make_double2(-w * rho * vi, w * rho * vr);
        }
        __syncthreads();
    }
}

void launch_haskind(const PanelsView& pv, int F, const FreqInfo* fi, int H, const double2* phi, int ldphi,
                    const double2* u, const double2* phiI, double rho, double2* HK, cudaStream_t s) {
    if (H <= 0) return;
    k_haskind<<<dim3(6 * pv.nbod, F), 256, 0, s>>>(pv, fi, H, phi, ldphi, u, phiI, rho, HK);
}

}  // namespace hbg
