// hbg_mixed_kernels.cuh -- kernels of the mixed-precision form.
//
// Storage: every matrix of a frequency is two FP32 planes (real, imaginary), Np x Np with Np the
// panel count rounded up to a multiple of 128, column-major as the assembly writes it: entry (k, n)
// of A at n Np + k.  Read row-major, that buffer is M = A^T, and the LU runs on M without pivoting
// (blocked by NBL = 128 columns): M = L U, so A = U^T L^T and A x = b is U^T y = b, L^T x = y.
// Per block step k0 (m = n = Np - k0 - NBL):
//   diag      M11 = L11 U11 in shared memory; L11^-1 and U11^-1 into small operand buffers
//   prep2     the block row M12 in the block-real K-major form the GEMM's B operand takes
//   GEMM1     L21 = M21 U11^-1                    (in place)
//   GEMM2     U12 = L11^-1 M12                    (in place; also the B operand of GEMM3)
//   GEMM3     M22 -= L21 U12
// A complex product C = A B runs as one real product [Cr | Ci] = [Ar | Ai] [[Br, Bi], [-Bi, Br]]
// on the tensor cores (kind::tf32, FP32 accumulation); the refinement in FP64 restores the
// accuracy of the solution (iterative refinement against the stored complex64 matrix).
#pragma once
#include "hbg_tc.cuh"

namespace hbg {

constexpr int NBL = 128;  // LU block width (complex columns)
constexpr int GBM = 128, GBK = 32, GSTAGES = 4, GBN = 256;

struct GemmArgs {
    int M, Nc, Kp;         // rows, real output columns, real inner dimension
    int a_planar;          // A from the planar matrix (x = a_x0 + kk % a_kc, plane = kk / a_kc) or a packed buffer
    int a_x0, a_kc, a_row0;
    int mode;              // 0 store, 1 store and scatter into the GEMM3 operand, 2 subtract
    float* out;            // planar matrices [F][2][Np][Np] (row-major view)
    size_t out_bstride, plane_stride;
    int ld, o_row0, o_col0, o_nc;
    float* p3;             // GEMM3's B operand [F][2n][2 NBL] (mode 1)
    size_t p3_bstride;
    int p3_n;
    int* err;
};

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
    return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

constexpr size_t gemm_smem_bytes() {
    return 1024 + (size_t)GSTAGES * (GBM + GBN) * GBK * 4 + 256;
}

// One 128 x 256 output tile per block: warp 0 lane 0 issues the TMA loads (4-stage ring), warp 1
// lane 0 the tcgen05.mma chain, then all four warps read the accumulator from TMEM (warp w owns
// rows 32w..32w+31) and apply the epilogue.
__global__ void __launch_bounds__(128, 1) k_gemm_tf32(const __grid_constant__ CUtensorMap mapA,
                                                      const __grid_constant__ CUtensorMap mapB, GemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = align1024(smem_raw);
    float* sA = reinterpret_cast<float*>(base);
    float* sB = sA + GSTAGES * GBM * GBK;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + GSTAGES * GBN * GBK);
    uint64_t* empty = full + GSTAGES;
    uint64_t* done = empty + GSTAGES;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * GBM, n0 = blockIdx.y * GBN, f = blockIdx.z;
    const int nk = g.Kp / GBK;
    if (threadIdx.x == 0) {
        for (int s = 0; s < GSTAGES; s++) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(done, 1);
        tc::fence_barrier_init();
        tc::prefetch_tensormap(&mapA);
        tc::prefetch_tensormap(&mapB);
    }
    if (warp == 0) tc::tmem_alloc(tslot, GBN);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tslot;
    if (warp == 0 && lane == 0) {
        const uint32_t bytes = (GBM + GBN) * GBK * 4;
        for (int kc = 0; kc < nk; kc++) {
            const int s = kc % GSTAGES;
            if (kc >= GSTAGES && !tc::mbar_wait(&empty[s], ((kc / GSTAGES) - 1) & 1)) {
                atomicExch(g.err, 1);
                break;
            }
            tc::mbar_arrive_expect_tx(&full[s], bytes);
            const int kk = kc * GBK;
            int ax = kk, plane = 0;
            if (g.a_planar) {
                ax = g.a_x0 + kk % g.a_kc;
                plane = kk / g.a_kc;
            }
            tc::tma_load_4d(sA + s * GBM * GBK, &mapA, &full[s], ax, g.a_row0 + m0, plane, f);
            tc::tma_load_4d(sB + s * GBN * GBK, &mapB, &full[s], kk, n0, 0, f);
        }
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = tc::idesc_tf32(GBM, GBN);
        for (int kc = 0; kc < nk; kc++) {
            const int s = kc % GSTAGES;
            if (!tc::mbar_wait(&full[s], (kc / GSTAGES) & 1)) {
                atomicExch(g.err, 2);
                break;
            }
            tc::tc_fence_after();
            const uint32_t a0 = tc::smem_u32(sA + s * GBM * GBK), b0 = tc::smem_u32(sB + s * GBN * GBK);
#pragma unroll
            for (int k8 = 0; k8 < GBK / 8; k8++)
                tc::mma_tf32(tmem, tc::desc_kmajor_sw128(a0 + 32 * k8), tc::desc_kmajor_sw128(b0 + 32 * k8), idesc,
                             (kc | k8) != 0);
            tc::mma_commit(&empty[s]);
        }
        tc::mma_commit(done);
    }
    __syncwarp();
    const bool ok = tc::mbar_wait(done, 0);
    if (!ok) atomicExch(g.err, 3);
    __syncwarp();
    tc::tc_fence_after();
    const int row = m0 + warp * 32 + lane;
    float* outf = g.out + (size_t)f * g.out_bstride;
    float* p3f = g.p3 ? g.p3 + (size_t)f * g.p3_bstride : nullptr;
    for (int c = 0; c < GBN / 32; c++) {
        float v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + c * 32, v);
        const int jg0 = n0 + c * 32;
        if (!ok || row >= g.M || jg0 >= g.Nc) continue;
        const int plane = jg0 >= g.o_nc ? 1 : 0;
        const int col0 = jg0 - plane * g.o_nc;
        float* p = outf + plane * g.plane_stride + (size_t)(g.o_row0 + row) * g.ld + g.o_col0 + col0;
        float4* p4 = reinterpret_cast<float4*>(p);
        if (g.mode == 2) {
#pragma unroll
            for (int q = 0; q < 8; q++) {
                float4 o = p4[q];
                o.x -= v[4 * q];
                o.y -= v[4 * q + 1];
                o.z -= v[4 * q + 2];
                o.w -= v[4 * q + 3];
                p4[q] = o;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 8; q++) p4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            if (g.mode == 1) {
                // U12(kk = row, j) into the block-real K-major operand of GEMM3 (rows 2n, 2 NBL wide)
                const int n = g.p3_n;
#pragma unroll 4
                for (int i = 0; i < 32; i++) {
                    const int j = col0 + i;
                    if (plane == 0) {
                        p3f[(size_t)j * (2 * NBL) + row] = v[i];
                        p3f[(size_t)(n + j) * (2 * NBL) + NBL + row] = v[i];
                    } else {
                        p3f[(size_t)j * (2 * NBL) + NBL + row] = -v[i];
                        p3f[(size_t)(n + j) * (2 * NBL) + row] = v[i];
                    }
                }
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, GBN);
}

// ---- diagonal block: M11 = L11 U11 (no pivoting) in shared memory, then L11^-1 and U11^-1.
// One block per matrix.  Writes the factors back, L11^-1 as [Lr | Li] rows (the A operand of
// GEMM2, [F][NBL][2 NBL]) and U11^-1 in the block-real K-major form (the B operand of GEMM1,
// [F][2 NBL][2 NBL]).  A pivot of modulus below 1e-30 of the block's largest sets err (the
// mixed form then reports the frequency; the FP64 form pivots).
__global__ void __launch_bounds__(1024) k_diag_factor(float* __restrict__ W, int Np, size_t bstride, int k0,
                                                      float* __restrict__ PL, float* __restrict__ PU,
                                                      float2* __restrict__ DINV, int* __restrict__ err) {
    extern __shared__ float2 blk[];  // [NBL][NBL + 1]
    const int f = blockIdx.x;
    float* Wr = W + (size_t)f * bstride;
    float* Wi = Wr + (size_t)Np * Np;
    constexpr int LD = NBL + 1;
    for (int t = threadIdx.x; t < NBL * NBL; t += blockDim.x) {
        int r = t / NBL, c = t % NBL;
        size_t o = (size_t)(k0 + r) * Np + k0 + c;
        blk[r * LD + c] = make_float2(Wr[o], Wi[o]);
    }
    __syncthreads();
    for (int j = 0; j < NBL; j++) {
        float2 d = blk[j * LD + j];
        float dd = d.x * d.x + d.y * d.y;
        if (threadIdx.x == 0 && !(dd > 1e-30f)) atomicExch(err, 10);
        float2 inv = make_float2(d.x / dd, -d.y / dd);
        for (int i = j + 1 + threadIdx.x; i < NBL; i += blockDim.x) {
            float2 a = blk[i * LD + j];
            blk[i * LD + j] = make_float2(a.x * inv.x - a.y * inv.y, a.x * inv.y + a.y * inv.x);
        }
        __syncthreads();
        const int rem = NBL - 1 - j;
        for (int t = threadIdx.x; t < rem * rem; t += blockDim.x) {
            int i = j + 1 + t / rem, c = j + 1 + t % rem;
            float2 l = blk[i * LD + j], u = blk[j * LD + c], a = blk[i * LD + c];
            a.x -= l.x * u.x - l.y * u.y;
            a.y -= l.x * u.y + l.y * u.x;
            blk[i * LD + c] = a;
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < NBL * NBL; t += blockDim.x) {
        int r = t / NBL, c = t % NBL;
        size_t o = (size_t)(k0 + r) * Np + k0 + c;
        Wr[o] = blk[r * LD + c].x;
        Wi[o] = blk[r * LD + c].y;
    }
    __syncthreads();
    // In-place inversion of U11 (upper) and L11 (unit lower), column by column: for column j of
    // U^-1 the leading block is already inverted, U^-1(0:j, j) = -U^-1(0:j, 0:j) U(0:j, j) / U(j, j);
    // for L^-1 from the last column, L^-1(j+1:, j) = -L^-1(j+1:, j+1:) L(j+1:, j).  Eight threads
    // per row share each dot product (shuffle reduction).
    const int row = threadIdx.x >> 3, part = threadIdx.x & 7;
    for (int j = 0; j < NBL; j++) {
        float2 d = blk[j * LD + j];
        float dd = d.x * d.x + d.y * d.y;
        float2 inv = make_float2(d.x / dd, -d.y / dd);
        float2 acc = make_float2(0.f, 0.f);
        if (row < j)
            for (int p = row + part; p < j; p += 8) {
                float2 t = blk[row * LD + p], v = blk[p * LD + j];
                acc.x += t.x * v.x - t.y * v.y;
                acc.y += t.x * v.y + t.y * v.x;
            }
        for (int o = 4; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        __syncthreads();
        if (row < j && part == 0)  // -acc / U(j, j) = -acc * inv
            blk[row * LD + j] = make_float2(-(acc.x * inv.x - acc.y * inv.y), -(acc.x * inv.y + acc.y * inv.x));
        if (row == j && part == 0) blk[j * LD + j] = inv;
        __syncthreads();
    }
    for (int j = NBL - 2; j >= 0; j--) {
        float2 acc = make_float2(0.f, 0.f);
        if (row > j) {
            // L^-1(row, j) = -(L(row, j) + sum_{j < p < row} L^-1(row, p) L(p, j))
            if (part == 0) acc = blk[row * LD + j];
            for (int p = j + 1 + part; p < row; p += 8) {
                float2 t = blk[row * LD + p], v = blk[p * LD + j];
                acc.x += t.x * v.x - t.y * v.y;
                acc.y += t.x * v.y + t.y * v.x;
            }
        }
        for (int o = 4; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        __syncthreads();
        if (row > j && part == 0) blk[row * LD + j] = make_float2(-acc.x, -acc.y);
        __syncthreads();
    }
    // blk now holds L^-1 (strictly below the diagonal, unit diagonal) and U^-1 (upper); kept per
    // block for the triangular solves ([F][Np / NBL][NBL][NBL], row-major)
    {
        float2* D = DINV + ((size_t)f * (Np / NBL) + k0 / NBL) * NBL * NBL;
        for (int t = threadIdx.x; t < NBL * NBL; t += blockDim.x) D[t] = blk[(t / NBL) * LD + t % NBL];
    }
    float* PLf = PL + (size_t)f * NBL * 2 * NBL;
    float* PUf = PU + (size_t)f * 2 * NBL * 2 * NBL;
    for (int t = threadIdx.x; t < NBL * NBL; t += blockDim.x) {
        const int i = t / NBL, c = t % NBL;
        // [Lr | Li] rows of L^-1
        float2 l = i > c ? blk[i * LD + c] : make_float2(i == c ? 1.f : 0.f, 0.f);
        PLf[(size_t)i * 2 * NBL + c] = l.x;
        PLf[(size_t)i * 2 * NBL + NBL + c] = l.y;
        // U^-1 block-real K-major: row c: [Ur(:, c); -Ui(:, c)], row NBL + c: [Ui(:, c); Ur(:, c)]
        float2 u = i <= c ? blk[i * LD + c] : make_float2(0.f, 0.f);  // U^-1(i, c)
        PUf[(size_t)c * 2 * NBL + i] = u.x;
        PUf[(size_t)c * 2 * NBL + NBL + i] = -u.y;
        PUf[(size_t)(NBL + c) * 2 * NBL + i] = u.y;
        PUf[(size_t)(NBL + c) * 2 * NBL + NBL + i] = u.x;
    }
}

// The block row M12 = rows k0..k0+NBL, columns k0+NBL..k0+NBL+n in the block-real K-major form
// [F][2n][2 NBL]: row j: [Br(:, j); -Bi(:, j)], row n + j: [Bi(:, j); Br(:, j)] (32 x 32 tiles
// transposed through shared memory).
__global__ void k_prep_block_row(const float* __restrict__ W, int Np, size_t bstride, int k0, int n,
                                 float* __restrict__ P2, size_t p2_bstride) {
    __shared__ float tr[32][33], ti[32][33];
    const int f = blockIdx.z;
    const int j0 = blockIdx.x * 32, kk0 = blockIdx.y * 32;
    const float* Wr = W + (size_t)f * bstride;
    const float* Wi = Wr + (size_t)Np * Np;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += blockDim.y) {
        size_t o = (size_t)(k0 + kk0 + r) * Np + k0 + NBL + j0 + tx;
        tr[r][tx] = Wr[o];
        ti[r][tx] = Wi[o];
    }
    __syncthreads();
    float* Pf = P2 + (size_t)f * p2_bstride;
    for (int r = ty; r < 32; r += blockDim.y) {
        const int j = j0 + r, kk = kk0 + tx;
        float br = tr[tx][r], bi = ti[tx][r];
        Pf[(size_t)j * 2 * NBL + kk] = br;
        Pf[(size_t)j * 2 * NBL + NBL + kk] = -bi;
        Pf[(size_t)(n + j) * 2 * NBL + kk] = bi;
        Pf[(size_t)(n + j) * 2 * NBL + NBL + kk] = br;
    }
}

// Partial products of y = M x over column chunks: part[z][f][c][k] = sum_{n in chunk z} M(k, n) x[f][c][n],
// M column-major planar FP32 (entry (k, n) at n Np + k), x FP64 complex [F][nrhs][ldx]; one thread
// per row (M read once, coalesced along k), FP64 accumulation.  k_gemv_reduce then forms
// out = bias - sum_z part[z] in a fixed order (deterministic).
constexpr int GEMV_CHUNK = 512;
template <int NR>
__global__ void __launch_bounds__(128) k_cgemv_part(int N, int Np, size_t bstride, int nrhs,
                                                    const float* __restrict__ Mall, const double2* __restrict__ xall,
                                                    int ldx, double2* __restrict__ part, int F) {
    constexpr int CH = 32;
    __shared__ double2 sx[CH][NR];
    const int f = blockIdx.y, z = blockIdx.z;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const float* Mr = Mall + (size_t)f * bstride;
    const float* Mi = Mr + (size_t)Np * Np;
    const double2* x = xall + (size_t)f * nrhs * ldx;
    const int nbeg = z * GEMV_CHUNK, nend = min(N, nbeg + GEMV_CHUNK);
    double2 acc[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = make_double2(0.0, 0.0);
    for (int n0 = nbeg; n0 < nend; n0 += CH) {
        __syncthreads();
        for (int t = threadIdx.x; t < CH * NR; t += blockDim.x) {
            int nn = t % CH, c = t / CH;
            sx[nn][c] = (n0 + nn < nend && c < nrhs) ? x[(size_t)c * ldx + n0 + nn] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        if (k < N) {
            const int lim = min(CH, nend - n0);
#pragma unroll 4
            for (int nn = 0; nn < lim; nn++) {
                const size_t o = (size_t)(n0 + nn) * Np + k;
                const double mr = Mr[o], mi = Mi[o];
#pragma unroll
                for (int c = 0; c < NR; c++) {
                    double2 v = sx[nn][c];
                    acc[c].x += mr * v.x - mi * v.y;
                    acc[c].y += mr * v.y + mi * v.x;
                }
            }
        }
    }
    if (k < N)
        for (int c = 0; c < nrhs && c < NR; c++) part[(((size_t)z * F + f) * nrhs + c) * N + k] = acc[c];
}

__global__ void k_gemv_reduce(int N, int nrhs, int F, int nz, const double2* __restrict__ part,
                              const double2* __restrict__ bias, int ldb, double2* __restrict__ out, int ldo) {
    const int f = blockIdx.y;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nrhs * N) return;
    const int c = (int)(t / N), k = (int)(t % N);
    double sr = 0.0, si = 0.0;
    for (int z = 0; z < nz; z++) {
        double2 v = part[(((size_t)z * F + f) * nrhs + c) * N + k];
        sr += v.x;
        si += v.y;
    }
    double2 b = bias ? bias[((size_t)f * nrhs + c) * ldb + k] : make_double2(0.0, 0.0);
    out[((size_t)f * nrhs + c) * ldo + k] = make_double2(b.x - sr, b.y - si);
}

// x = A^-1 r with the factors of M = A^T = L U (FP32 planar, row-major in W): U^T y = r, then
// L^T x = y, FP64 vectors [F][nrhs][Np] in place, in blocks of TB = 128 rows.  One launch per
// block step: every CTA of the step owns 128 rows, subtracts the contribution of the block solved
// by the previous step (row b0 + p of W read along its rows: coalesced), and the CTA that owns the
// next diagonal block then solves it (a warp per right-hand side, 32-row sub-blocks).
constexpr int TB = 128;

// The diagonal block b of U^T (upper_t) or L^T, solved by its stored inverse: y_b = D^T r_b with
// D = U_bb^-1 (upper part of the stored block, with the diagonal) or L_bb^-1 (lower part, unit
// diagonal).  Rows b0..b0+TB of X in place; thread t computes column t % TB for a set of right-hand sides.
template <int NR>
__device__ __forceinline__ void tri_block_inv(const float2* __restrict__ D, double2* X, int Np, int nrhs, int b0,
                                              bool upper_t, double2 (*rs)[NR]) {
    for (int t = threadIdx.x; t < TB * nrhs; t += blockDim.x) {
        int p = t % TB, c = t / TB;
        rs[p][c] = X[(size_t)c * Np + b0 + p];
    }
    __syncthreads();
    const int i = threadIdx.x % TB, c0 = threadIdx.x / TB, cs = blockDim.x / TB;
    double2 acc[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = make_double2(0.0, 0.0);
    const int pbeg = upper_t ? 0 : i, pend = upper_t ? i + 1 : TB;
    for (int p = pbeg; p < pend; p++) {
        float2 dv = D[p * TB + i];
        double dr = dv.x, di = dv.y;
        if (!upper_t && p == i) {  // the unit diagonal of L^-1
            dr = 1.0;
            di = 0.0;
        }
#pragma unroll
        for (int c = 0; c < NR; c++)
            if ((c % cs) == c0) {
                double2 v = rs[p][c];
                acc[c].x += dr * v.x - di * v.y;
                acc[c].y += dr * v.y + di * v.x;
            }
    }
    __syncthreads();
    for (int c = c0; c < nrhs; c += cs) X[(size_t)c * Np + b0 + i] = acc[c];
}

// One block step of the forward (upper_t) or backward solve.  step = index of the block solved by
// the previous launch (-1: none, only the first diagonal block is solved).
template <int NR>
__global__ void __launch_bounds__(256) k_tri_step(int Np, size_t bstride, const float* __restrict__ W,
                                                  const float2* __restrict__ DINV, int nrhs,
                                                  double2* __restrict__ Xall, int step, int upper_t) {
    extern __shared__ double2 tri_smem[];  // ys [TB][NR]
    double2(*ys)[NR] = reinterpret_cast<double2(*)[NR]>(tri_smem);
    const int f = blockIdx.y;
    const float* Mr = W + (size_t)f * bstride;
    const float* Mi = Mr + (size_t)Np * Np;
    double2* X = Xall + (size_t)f * nrhs * Np;
    const int nblk = Np / TB;
    const float2* Df = DINV + (size_t)f * nblk * TB * TB;
    if (step < 0) {
        const int first = upper_t ? 0 : nblk - 1;
        tri_block_inv<NR>(Df + (size_t)first * TB * TB, X, Np, nrhs, first * TB, upper_t, ys);
        return;
    }
    // block solved last: rows s0 = step TB; this CTA's rows: the c-th block after it (forward) or
    // before it (backward)
    const int s0 = step * TB;
    const int cb = upper_t ? step + 1 + blockIdx.x : step - 1 - blockIdx.x;
    const int r0 = cb * TB;
    for (int t = threadIdx.x; t < TB * nrhs; t += blockDim.x) {
        int p = t % TB, c = t / TB;
        ys[p][c] = X[(size_t)c * Np + s0 + p];
    }
    __syncthreads();
    // rows r0 .. r0 + TB: two threads a row, each a half of the block's 128 terms
    const int i = r0 + (threadIdx.x >> 1), half = threadIdx.x & 1;
    double2 acc[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = make_double2(0.0, 0.0);
    for (int p = half * (TB / 2); p < (half + 1) * (TB / 2); p++) {
        const size_t o = (size_t)(s0 + p) * Np + i;
        const double mr = Mr[o], mi = Mi[o];
#pragma unroll
        for (int c = 0; c < NR; c++) {
            double2 v = ys[p][c];
            acc[c].x += mr * v.x - mi * v.y;
            acc[c].y += mr * v.y + mi * v.x;
        }
    }
#pragma unroll
    for (int c = 0; c < NR; c++) {
        acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, 1);
        acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, 1);
    }
    if (half == 0)
#pragma unroll
        for (int c = 0; c < NR; c++)
            if (c < nrhs) {
                double2 v = X[(size_t)c * Np + i];
                X[(size_t)c * Np + i] = make_double2(v.x - acc[c].x, v.y - acc[c].y);
            }
    if (blockIdx.x == 0) {
        __syncthreads();
        tri_block_inv<NR>(Df + (size_t)cb * TB * TB, X, Np, nrhs, r0, upper_t, ys);
    }
}

// x += d; per matrix the largest |d| and |x| (for the refinement's stopping test), [F][2].
__global__ void k_ir_update(int Np, int nrhs, double2* __restrict__ x, const double2* __restrict__ d,
                            double* __restrict__ norms) {
    __shared__ double sd[256], sx[256];
    const int f = blockIdx.x;
    const size_t n = (size_t)nrhs * Np;
    double md = 0.0, mx = 0.0;
    for (size_t t = threadIdx.x; t < n; t += blockDim.x) {
        size_t o = (size_t)f * n + t;
        double2 a = x[o], b = d[o];
        a.x += b.x;
        a.y += b.y;
        x[o] = a;
        md = fmax(md, fmax(fabs(b.x), fabs(b.y)));
        mx = fmax(mx, fmax(fabs(a.x), fabs(a.y)));
    }
    sd[threadIdx.x] = md;
    sx[threadIdx.x] = mx;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sd[threadIdx.x] = fmax(sd[threadIdx.x], sd[threadIdx.x + s]);
            sx[threadIdx.x] = fmax(sx[threadIdx.x], sx[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        norms[2 * f] = sd[0];
        norms[2 * f + 1] = sx[0];
    }
}

// The padding rows and columns N..Np of the planar matrices: identity (zero elsewhere).
__global__ void k_pad_identity(float* __restrict__ W, int N, int Np, size_t bstride) {
    const int f = blockIdx.y;
    float* Wr = W + (size_t)f * bstride;
    float* Wi = Wr + (size_t)Np * Np;
    const size_t npad = (size_t)(Np - N);
    const size_t total = 2 * npad * Np;  // the last npad columns and the last npad rows
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        size_t r, c;
        if (t < npad * Np) {
            c = N + t / Np;
            r = t % Np;
        } else {
            size_t u = t - npad * Np;
            r = N + u / Np;
            c = u % Np;
        }
        size_t o = c * Np + r;
        Wr[o] = (r == c) ? 1.f : 0.f;
        Wi[o] = 0.f;
    }
}

}  // namespace hbg
