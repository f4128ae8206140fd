// hbg_lu.cu -- the plain FP64 form of the dense complex solve: right-looking blocked LU with partial
// pivoting, batched over the F matrices of a frequency batch (linalg.rs:100-201 restated for the
// GPU: panel factorization, row swaps, unit-lower triangular solve of the block row, trailing
// update), then the substitution for the nrhs right-hand sides (linalg.rs:189-201).
//
// Matrices are column-major complex128 (entry (i, j) at i + j N), matrix f at A + f * stride.
// ipiv[f * N + i] is the 0-based row swapped with row i at step i (LAPACK's layout).
#include "hbg_device.cuh"
#include "hbg_internal.h"

namespace hbg {

constexpr int NB = 32;  // panel width

__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }

// Panel k0..k0+nb-1, rows k0..N-1, one block per matrix: for each column the pivot (largest
// modulus, first index on a tie), the row swap inside the panel, the scaled column and the
// rank-1 update of the panel's remaining columns.
__global__ void __launch_bounds__(1024) k_panel_f64(int N, int k0, int nb, double2* __restrict__ Aall, size_t stride,
                                                    int32_t* __restrict__ ipiv, int32_t* __restrict__ info) {
    __shared__ double sval[32];
    __shared__ int sidx[32];
    __shared__ double2 prow[NB];
    __shared__ int spiv;
    const int f = blockIdx.x;
    double2* A = Aall + (size_t)f * stride;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = 0; j < nb; j++) {
        const int col = k0 + j;
        double best = -1.0;
        int bi = col;
        for (int i = col + threadIdx.x; i < N; i += blockDim.x) {
            double v = cabs2(A[(size_t)i + (size_t)col * N]);
            if (v > best) {
                best = v;
                bi = i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_down_sync(0xffffffffu, best, o);
            int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            sval[warp] = best;
            sidx[warp] = bi;
        }
        __syncthreads();
        if (warp == 0) {
            best = lane < nw ? sval[lane] : -1.0;
            bi = lane < nw ? sidx[lane] : N;
            for (int o = 16; o > 0; o >>= 1) {
                double ov = __shfl_down_sync(0xffffffffu, best, o);
                int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            if (lane == 0) {
                spiv = bi;
                ipiv[(size_t)f * N + col] = bi;
                if (!(best > 0.0) && info[f] == 0) info[f] = col + 1;
            }
        }
        __syncthreads();
        const int p = spiv;
        // swap rows col and p in the panel's columns; keep the pivot row in shared memory
        for (int c = threadIdx.x; c < nb; c += blockDim.x) {
            size_t a = (size_t)col + (size_t)(k0 + c) * N, b = (size_t)p + (size_t)(k0 + c) * N;
            double2 va = A[a], vb = A[b];
            if (p != col) {
                A[a] = vb;
                A[b] = va;
            }
            prow[c] = vb;
        }
        __syncthreads();
        double2 piv = prow[j];
        double d = cabs2(piv);
        double2 inv = d > 0.0 ? make_double2(piv.x / d, -piv.y / d) : make_double2(0.0, 0.0);
        for (int i = col + 1 + threadIdx.x; i < N; i += blockDim.x) {
            double2 l = cmul(A[(size_t)i + (size_t)col * N], inv);
            A[(size_t)i + (size_t)col * N] = l;
            for (int c = j + 1; c < nb; c++) {
                size_t o = (size_t)i + (size_t)(k0 + c) * N;
                A[o] = csub(A[o], cmul(l, prow[c]));
            }
        }
        __syncthreads();
    }
}

// The panel's row swaps on every column outside it (one thread per column).
__global__ void k_laswp_f64(int N, int k0, int nb, double2* __restrict__ Aall, size_t stride,
                            const int32_t* __restrict__ ipiv) {
    const int f = blockIdx.y;
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N - nb) return;
    if (c >= k0) c += nb;
    double2* A = Aall + (size_t)f * stride + (size_t)c * N;
    const int32_t* pv = ipiv + (size_t)f * N;
    for (int j = 0; j < nb; j++) {
        int r = k0 + j, p = pv[r];
        if (p != r) {
            double2 t = A[r];
            A[r] = A[p];
            A[p] = t;
        }
    }
}

// U12 = L11^-1 A12: one warp per column right of the panel, lane i holding row k0 + i.
__global__ void k_trsm_f64(int N, int k0, int nb, double2* __restrict__ Aall, size_t stride) {
    __shared__ double2 L[NB][NB + 1];
    const int f = blockIdx.y;
    double2* A = Aall + (size_t)f * stride;
    for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
        int r = t % nb, c = t / nb;
        L[r][c] = A[(size_t)(k0 + r) + (size_t)(k0 + c) * N];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int col = k0 + nb + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (col >= N) return;
    double2 x = lane < nb ? A[(size_t)(k0 + lane) + (size_t)col * N] : make_double2(0.0, 0.0);
    for (int p = 0; p < nb; p++) {
        double2 xp = make_double2(__shfl_sync(0xffffffffu, x.x, p), __shfl_sync(0xffffffffu, x.y, p));
        if (lane > p && lane < nb) x = csub(x, cmul(L[lane][p], xp));
    }
    if (lane < nb) A[(size_t)(k0 + lane) + (size_t)col * N] = x;
}

// Trailing update C -= L21 U12 (K = nb), 64 x 64 tiles, 256 threads of 4 x 4 complex each, the
// K dimension staged through shared memory in chunks of 16.
__global__ void __launch_bounds__(256) k_gemm_update_f64(int N, int k0, int nb, double2* __restrict__ Aall,
                                                        size_t stride) {
    constexpr int KC = 16;
    __shared__ double2 As[KC][64];
    __shared__ double2 Bs[KC][64 + 1];
    const int f = blockIdx.z;
    double2* A = Aall + (size_t)f * stride;
    const int r0 = k0 + nb + blockIdx.x * 64, c0 = k0 + nb + blockIdx.y * 64;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = make_double2(0.0, 0.0);
    for (int kc = 0; kc < nb; kc += KC) {
        const int kn = min(KC, nb - kc);
        __syncthreads();
        for (int t = threadIdx.x; t < 64 * KC; t += 256) {
            int r = t & 63, kk = t >> 6;
            As[kk][r] = (kk < kn && r0 + r < N) ? A[(size_t)(r0 + r) + (size_t)(k0 + kc + kk) * N] : make_double2(0.0, 0.0);
            int kb = t % KC, cc = t / KC;
            Bs[kb][cc] = (kb < kn && c0 + cc < N) ? A[(size_t)(k0 + kc + kb) + (size_t)(c0 + cc) * N] : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < KC; kk++) {
            double2 av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; a++) av[a] = As[kk][tx + 16 * a];
#pragma unroll
            for (int b = 0; b < 4; b++) bv[b] = Bs[kk][ty + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) {
                    acc[a][b].x += av[a].x * bv[b].x - av[a].y * bv[b].y;
                    acc[a][b].y += av[a].x * bv[b].y + av[a].y * bv[b].x;
                }
        }
    }
#pragma unroll
    for (int b = 0; b < 4; b++) {
        int c = c0 + ty + 16 * b;
        if (c >= N) continue;
#pragma unroll
        for (int a = 0; a < 4; a++) {
            int r = r0 + tx + 16 * a;
            if (r < N) {
                size_t o = (size_t)r + (size_t)c * N;
                A[o] = csub(A[o], acc[a][b]);
            }
        }
    }
}

int lu_factor_f64(int N, int F, double2* A, size_t stride, int32_t* ipiv, int32_t* info, cudaStream_t s,
                  int64_t* launches) {
    KernelProfiler& P = profiler();
    cudaMemsetAsync(info, 0, sizeof(int32_t) * F, s);
    for (int k0 = 0; k0 < N; k0 += NB) {
        int nb = N - k0 < NB ? N - k0 : NB;
        const double m = N - k0;
        P.begin(s);
        k_panel_f64<<<F, 1024, 0, s>>>(N, k0, nb, A, stride, ipiv, info);
        // complex LU of an m x nb panel: 8 (m nb^2 - nb^3 / 3) real flops
        P.end(KF_LU_PANEL, F * 8.0 * (m * nb * nb - nb * (double)nb * nb / 3.0), s);
        (*launches)++;
        if (N - nb > 0) {
            P.begin(s);
            k_laswp_f64<<<dim3((N - nb + 127) / 128, F), 128, 0, s>>>(N, k0, nb, A, stride, ipiv);
            P.end(KF_LU_LASWP, F * 2.0 * nb * (N - nb) * 16.0 * 2.0, s);
            (*launches)++;
        }
        int right = N - k0 - nb;
        if (right > 0) {
            P.begin(s);
            k_trsm_f64<<<dim3((right + 7) / 8, F), 256, 0, s>>>(N, k0, nb, A, stride);
            P.end(KF_LU_TRSM, F * 4.0 * nb * (double)nb * right, s);
            dim3 g((right + 63) / 64, (right + 63) / 64, F);
            P.begin(s);
            k_gemm_update_f64<<<g, 256, 0, s>>>(N, k0, nb, A, stride);
            // complex C -= L U: 8 m n k real flops
            P.end(KF_LU_GEMM, F * 8.0 * (double)right * right * nb, s);
            (*launches) += 2;
        }
    }
    return 0;
}

// ------------------------------------------------------------------ substitution
// One block per matrix: the row permutation from the swaps (in shared memory), the gather of P B
// into X, then forward substitution with the unit lower factor and back substitution with the
// upper factor, in blocks of 32 rows: a warp per right-hand side solves the 32 x 32 triangle,
// then every thread updates its rows of the rest with the block's solution.
// Bin and X are [F][nrhs][N] (one column per right-hand side).
template <int NR>
__global__ void __launch_bounds__(1024) k_lu_solve_f64(int N, const double2* __restrict__ LUall, size_t stride,
                                                       const int32_t* __restrict__ ipiv, int nrhs,
                                                       const double2* __restrict__ Ball, double2* __restrict__ Xall) {
    extern __shared__ int32_t perm[];
    __shared__ double2 xs[32][NR];
    const int f = blockIdx.x;
    const double2* LU = LUall + (size_t)f * stride;
    const double2* B = Ball + (size_t)f * nrhs * N;
    double2* X = Xall + (size_t)f * nrhs * N;
    const int32_t* pv = ipiv + (size_t)f * N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) perm[i] = i;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < N; i++) {
            int p = pv[i];
            if (p != i) {
                int t = perm[i];
                perm[i] = perm[p];
                perm[p] = t;
            }
        }
    __syncthreads();
    for (int c = 0; c < nrhs; c++)
        for (int i = threadIdx.x; i < N; i += blockDim.x) X[(size_t)c * N + i] = B[(size_t)c * N + perm[i]];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // forward: L y = P b
    for (int b0 = 0; b0 < N; b0 += 32) {
        int bn = min(32, N - b0);
        if (warp < nrhs) {
            double2 x = lane < bn ? X[(size_t)warp * N + b0 + lane] : make_double2(0.0, 0.0);
            for (int p = 0; p < bn; p++) {
                double2 xp = make_double2(__shfl_sync(0xffffffffu, x.x, p), __shfl_sync(0xffffffffu, x.y, p));
                if (lane > p && lane < bn) x = csub(x, cmul(LU[(size_t)(b0 + lane) + (size_t)(b0 + p) * N], xp));
            }
            if (lane < bn) {
                X[(size_t)warp * N + b0 + lane] = x;
                xs[lane][warp] = x;
            }
        }
        __syncthreads();
        for (int i = b0 + bn + threadIdx.x; i < N; i += blockDim.x) {
            double2 acc[NR];
#pragma unroll
            for (int c = 0; c < NR; c++) acc[c] = make_double2(0.0, 0.0);
            for (int p = 0; p < bn; p++) {
                double2 l = LU[(size_t)i + (size_t)(b0 + p) * N];
#pragma unroll
                for (int c = 0; c < NR; c++) {
                    acc[c].x += l.x * xs[p][c].x - l.y * xs[p][c].y;
                    acc[c].y += l.x * xs[p][c].y + l.y * xs[p][c].x;
                }
            }
            for (int c = 0; c < nrhs; c++) X[(size_t)c * N + i] = csub(X[(size_t)c * N + i], acc[c]);
        }
        __syncthreads();
    }
    // backward: U x = y, blocks from the bottom
    const int nblk = (N + 31) / 32;
    for (int bb = nblk - 1; bb >= 0; bb--) {
        int b0 = bb * 32, bn = min(32, N - b0);
        if (warp < nrhs) {
            double2 x = lane < bn ? X[(size_t)warp * N + b0 + lane] : make_double2(0.0, 0.0);
            for (int p = bn - 1; p >= 0; p--) {
                if (lane == p) {
                    double2 up = LU[(size_t)(b0 + p) + (size_t)(b0 + p) * N];
                    double d = cabs2(up);
                    x = make_double2((x.x * up.x + x.y * up.y) / d, (x.y * up.x - x.x * up.y) / d);
                }
                double2 xp = make_double2(__shfl_sync(0xffffffffu, x.x, p), __shfl_sync(0xffffffffu, x.y, p));
                if (lane < p) x = csub(x, cmul(LU[(size_t)(b0 + lane) + (size_t)(b0 + p) * N], xp));
            }
            if (lane < bn) {
                X[(size_t)warp * N + b0 + lane] = x;
                xs[lane][warp] = x;
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < b0; i += blockDim.x) {
            double2 acc[NR];
#pragma unroll
            for (int c = 0; c < NR; c++) acc[c] = make_double2(0.0, 0.0);
            for (int p = 0; p < bn; p++) {
                double2 u = LU[(size_t)i + (size_t)(b0 + p) * N];
#pragma unroll
                for (int c = 0; c < NR; c++) {
                    acc[c].x += u.x * xs[p][c].x - u.y * xs[p][c].y;
                    acc[c].y += u.x * xs[p][c].y + u.y * xs[p][c].x;
                }
            }
            for (int c = 0; c < nrhs; c++) X[(size_t)c * N + i] = csub(X[(size_t)c * N + i], acc[c]);
        }
        __syncthreads();
    }
}

int lu_solve_f64(int N, int F, const double2* LU, size_t stride, const int32_t* ipiv, int nrhs, const double2* B,
                 double2* X, cudaStream_t s) {
    size_t smem = sizeof(int32_t) * (size_t)N;
    if (nrhs > 32 || smem > 200 * 1024) return 1;
    if (nrhs <= 8) {
        cudaFuncSetAttribute(k_lu_solve_f64<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_lu_solve_f64<8><<<F, 1024, smem, s>>>(N, LU, stride, ipiv, nrhs, B, X);
    } else if (nrhs <= 16) {
        cudaFuncSetAttribute(k_lu_solve_f64<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_lu_solve_f64<16><<<F, 1024, smem, s>>>(N, LU, stride, ipiv, nrhs, B, X);
    } else {
        cudaFuncSetAttribute(k_lu_solve_f64<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_lu_solve_f64<32><<<F, 1024, smem, s>>>(N, LU, stride, ipiv, nrhs, B, X);
    }
    return 0;
}

}  // namespace hbg
