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
                                                      int* __restrict__ err) {
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
    float* PLf = PL + (size_t)f * NBL * 2 * NBL;
    float* PUf = PU + (size_t)f * 2 * NBL * 2 * NBL;
    const int c = threadIdx.x;
    if (c < NBL) {
        // column c of U11^-1 by back substitution
        float2 x[NBL];
        for (int i = 0; i < NBL; i++) x[i] = make_float2(0.f, 0.f);
        for (int i = c; i >= 0; i--) {
            float sr = (i == c) ? 1.f : 0.f, si = 0.f;
            for (int p = i + 1; p <= c; p++) {
                float2 u = blk[i * LD + p];
                sr -= u.x * x[p].x - u.y * x[p].y;
                si -= u.x * x[p].y + u.y * x[p].x;
            }
            float2 d = blk[i * LD + i];
            float dd = d.x * d.x + d.y * d.y;
            x[i] = make_float2((sr * d.x + si * d.y) / dd, (si * d.x - sr * d.y) / dd);
        }
        // block-real K-major rows: row c: [Ur(:,c); -Ui(:,c)], row NBL + c: [Ui(:,c); Ur(:,c)]
        for (int k = 0; k < NBL; k++) {
            PUf[(size_t)c * 2 * NBL + k] = x[k].x;
            PUf[(size_t)c * 2 * NBL + NBL + k] = -x[k].y;
            PUf[(size_t)(NBL + c) * 2 * NBL + k] = x[k].y;
            PUf[(size_t)(NBL + c) * 2 * NBL + NBL + k] = x[k].x;
        }
    } else if (c < 2 * NBL) {
        // column cc of L11^-1 (unit lower) by forward substitution; written as rows [Lr | Li]
        const int cc = c - NBL;
        float2 x[NBL];
        for (int i = 0; i < NBL; i++) x[i] = make_float2(0.f, 0.f);
        x[cc] = make_float2(1.f, 0.f);
        for (int i = cc + 1; i < NBL; i++) {
            float sr = 0.f, si = 0.f;
            for (int p = cc; p < i; p++) {
                float2 l = blk[i * LD + p];
                sr -= l.x * x[p].x - l.y * x[p].y;
                si -= l.x * x[p].y + l.y * x[p].x;
            }
            x[i] = make_float2(sr, si);
        }
        for (int i = 0; i < NBL; i++) {
            PLf[(size_t)i * 2 * NBL + cc] = x[i].x;
            PLf[(size_t)i * 2 * NBL + NBL + cc] = x[i].y;
        }
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

// out[f][c][k] = bias[f][c][k] - sum_n M(k, n) x[f][c][n], M column-major planar FP32 (entry (k, n)
// at n Np + k), x and out FP64 complex [F][nrhs][ld]; one thread per row, M read once (coalesced
// along k), x staged in shared memory.  bias may be null (zero).
template <int NR>
__global__ void __launch_bounds__(128) k_cgemv_f32(int N, int Np, size_t bstride, int nrhs,
                                                   const float* __restrict__ Mall, const double2* __restrict__ xall,
                                                   int ldx, const double2* __restrict__ bias, int ldb,
                                                   double2* __restrict__ out, int ldo) {
    constexpr int CH = 32;
    __shared__ double2 sx[CH][NR];
    const int f = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const float* Mr = Mall + (size_t)f * bstride;
    const float* Mi = Mr + (size_t)Np * Np;
    const double2* x = xall + (size_t)f * nrhs * ldx;
    double2 acc[NR];
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = make_double2(0.0, 0.0);
    for (int n0 = 0; n0 < N; n0 += CH) {
        __syncthreads();
        for (int t = threadIdx.x; t < CH * NR; t += blockDim.x) {
            int nn = t % CH, c = t / CH;
            sx[nn][c] = (n0 + nn < N && c < nrhs) ? x[(size_t)c * ldx + n0 + nn] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        if (k < N) {
            const int lim = min(CH, N - n0);
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
        for (int c = 0; c < nrhs && c < NR; c++) {
            double2 b = bias ? bias[((size_t)f * nrhs + c) * ldb + k] : make_double2(0.0, 0.0);
            out[((size_t)f * nrhs + c) * ldo + k] = make_double2(b.x - acc[c].x, b.y - acc[c].y);
        }
}

// x = A^-1 r with the factors of M = A^T = L U (FP32 planar, row-major in W): U^T y = r, then
// L^T x = y; FP64 vectors [F][nrhs][Np], in place.  One block per matrix, 32-row blocks: a warp per
// right-hand side solves the triangle, then every thread updates its rows with the block's values
// (row b0 + p of W read along the updated rows: coalesced).
template <int NR>
__global__ void __launch_bounds__(1024) k_trisolve_f32(int Np, size_t bstride, const float* __restrict__ W, int nrhs,
                                                       double2* __restrict__ Xall) {
    __shared__ double2 xs[32][NR];
    const int f = blockIdx.x;
    const float* Mr = W + (size_t)f * bstride;
    const float* Mi = Mr + (size_t)Np * Np;
    double2* X = Xall + (size_t)f * nrhs * Np;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto m = [&](int r, int c) { size_t o = (size_t)r * Np + c; return make_double2(Mr[o], Mi[o]); };
    // forward: U^T y = r  (U^T(i, j) = M(j, i), j <= i)
    for (int b0 = 0; b0 < Np; b0 += 32) {
        if (warp < nrhs) {
            double2 y = X[(size_t)warp * Np + b0 + lane];
            for (int p = 0; p < 32; p++) {
                if (lane == p) {
                    double2 d = m(b0 + p, b0 + p);
                    double dd = d.x * d.x + d.y * d.y;
                    y = make_double2((y.x * d.x + y.y * d.y) / dd, (y.y * d.x - y.x * d.y) / dd);
                }
                double2 yp = make_double2(__shfl_sync(0xffffffffu, y.x, p), __shfl_sync(0xffffffffu, y.y, p));
                if (lane > p) {
                    double2 u = m(b0 + p, b0 + lane);
                    y.x -= u.x * yp.x - u.y * yp.y;
                    y.y -= u.x * yp.y + u.y * yp.x;
                }
            }
            X[(size_t)warp * Np + b0 + lane] = y;
            xs[lane][warp] = y;
        }
        __syncthreads();
        for (int i = b0 + 32 + threadIdx.x; i < Np; i += blockDim.x) {
            double2 acc[NR];
#pragma unroll
            for (int c = 0; c < NR; c++) acc[c] = make_double2(0.0, 0.0);
            for (int p = 0; p < 32; p++) {
                double2 u = m(b0 + p, i);
#pragma unroll
                for (int c = 0; c < NR; c++) {
                    acc[c].x += u.x * xs[p][c].x - u.y * xs[p][c].y;
                    acc[c].y += u.x * xs[p][c].y + u.y * xs[p][c].x;
                }
            }
            for (int c = 0; c < nrhs; c++) {
                double2 v = X[(size_t)c * Np + i];
                X[(size_t)c * Np + i] = make_double2(v.x - acc[c].x, v.y - acc[c].y);
            }
        }
        __syncthreads();
    }
    // backward: L^T x = y  (L^T(i, j) = M(j, i), j > i, unit diagonal)
    for (int b0 = Np - 32; b0 >= 0; b0 -= 32) {
        if (warp < nrhs) {
            double2 x = X[(size_t)warp * Np + b0 + lane];
            for (int p = 31; p >= 0; p--) {
                double2 xp = make_double2(__shfl_sync(0xffffffffu, x.x, p), __shfl_sync(0xffffffffu, x.y, p));
                if (lane < p) {
                    double2 l = m(b0 + p, b0 + lane);
                    x.x -= l.x * xp.x - l.y * xp.y;
                    x.y -= l.x * xp.y + l.y * xp.x;
                }
            }
            X[(size_t)warp * Np + b0 + lane] = x;
            xs[lane][warp] = x;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < b0; i += blockDim.x) {
            double2 acc[NR];
#pragma unroll
            for (int c = 0; c < NR; c++) acc[c] = make_double2(0.0, 0.0);
            for (int p = 0; p < 32; p++) {
                double2 l = m(b0 + p, i);
#pragma unroll
                for (int c = 0; c < NR; c++) {
                    acc[c].x += l.x * xs[p][c].x - l.y * xs[p][c].y;
                    acc[c].y += l.x * xs[p][c].y + l.y * xs[p][c].x;
                }
            }
            for (int c = 0; c < nrhs; c++) {
                double2 v = X[(size_t)c * Np + i];
                X[(size_t)c * Np + i] = make_double2(v.x - acc[c].x, v.y - acc[c].y);
            }
        }
        __syncthreads();
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
