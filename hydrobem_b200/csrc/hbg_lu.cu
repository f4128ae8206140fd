// hbg_lu.cu -- the plain FP64 form of the dense complex solve: right-looking blocked LU with partial
// pivoting, batched over the F matrices of a frequency batch (linalg.rs:100-201 restated for the
// GPU: panel factorization, row swaps, unit-lower triangular solve of the block row, trailing
// update), then the substitution for the nrhs right-hand sides (linalg.rs:189-201).
//
// Matrices are column-major complex128 (entry (i, j) at i + j N), matrix f at A + f * stride.
// ipiv[f * N + i] is the 0-based row swapped with row i at step i (LAPACK's layout).
#include <atomic>

#include "hbg_device.cuh"
#include "hbg_internal.h"

namespace hbg {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }

// Blocking of the factorization: panels of LU_NB columns, each factored recursively (halves) down to
// strips of at most LU_BASE columns.  The default schedule takes the whole batch as one group (every
// launch covers all its matrices) with look-ahead: the next panel is factored on a high-priority stream
// beside the trailing update of the current one.  Measured on the 40 matrices of order 4096 of the
// benchmark job: 322 ms, against 333 / 345 / 353 ms for 2 / 3 / 4 groups and 340 ms without look-ahead.
constexpr int LU_NB = 128;
constexpr int LU_BASE = 8;
constexpr int LU_F64_GROUPS = 1;      // the default schedule's groups
constexpr int LU_F64_MAX_GROUPS = 8;

// ------------------------------------------------------------------ base strip
// Columns c0 .. c0 + w - 1 (w <= LU_BASE), rows c0 .. N - 1, one CTA per matrix: for each column the
// pivot (largest modulus, first index on a tie: LAPACK's izamax), the swap of the two rows across the
// whole panel (columns pk0 .. pk0 + pnb - 1: the recursion then needs no interchanges of its own), the
// column scaled by the pivot and the rank-1 update of the strip's remaining columns.  The candidates of
// the next column's pivot are taken while its entries are updated (one pass a column); each thread
// updates two rows at a time, their loads in flight together.
__device__ __forceinline__ void lu_base_row(double2* A, int N, int i, int c0, int col, int j, int w, double2 inv,
                                            const double2* prow, double2 a, double2* v, double& best, int& bi,
                                            bool store) {
    if (!store) return;
    const double2 l = cmul(a, inv);
    A[(size_t)i + (size_t)col * N] = l;
#pragma unroll
    for (int c = 0; c < LU_BASE; c++)
        if (c > j && c < w) {
            v[c] = csub(v[c], cmul(l, prow[c]));
            A[(size_t)i + (size_t)(c0 + c) * N] = v[c];
            if (c == j + 1) {
                const double m = cabs2(v[c]);
                if (m > best) best = m, bi = i;
            }
        }
}

__global__ void __launch_bounds__(512) k_lu_base(int N, int c0, int w, int pk0, int pnb, double2* __restrict__ Aall,
                                                 size_t stride, int32_t* __restrict__ ipiv, int32_t* __restrict__ info) {
    __shared__ double sval[32];
    __shared__ int sidx[32];
    __shared__ double2 prow[LU_BASE];
    __shared__ int spiv;
    const int f = blockIdx.x;
    double2* A = Aall + (size_t)f * stride;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double best = -1.0;
    int bi = N;
    for (int i = c0 + threadIdx.x; i < N; i += blockDim.x) {
        const double v = cabs2(A[(size_t)i + (size_t)c0 * N]);
        if (v > best) best = v, bi = i;
    }
    for (int j = 0; j < w; j++) {
        const int col = c0 + j;
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) best = ov, bi = oi;
        }
        if (lane == 0) sval[warp] = best, sidx[warp] = bi;
        __syncthreads();
        if (warp == 0) {
            best = lane < nw ? sval[lane] : -1.0;
            bi = lane < nw ? sidx[lane] : N;
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, best, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) best = ov, bi = oi;
            }
            if (lane == 0) {
                const int p = bi < N ? bi : col;
                spiv = p;
                ipiv[(size_t)f * N + col] = p;
                if (!(best > 0.0) && info[f] == 0) info[f] = col + 1;
            }
        }
        __syncthreads();
        const int p = spiv;
        if (p != col)  // swap rows col and p across the panel
            for (int t = threadIdx.x; t < pnb; t += blockDim.x) {
                const size_t a = (size_t)col + (size_t)(pk0 + t) * N, b = (size_t)p + (size_t)(pk0 + t) * N;
                const double2 va = A[a];
                A[a] = A[b];
                A[b] = va;
            }
        __syncthreads();
        if (threadIdx.x < w) prow[threadIdx.x] = A[(size_t)col + (size_t)(c0 + threadIdx.x) * N];
        __syncthreads();
        const double2 piv = prow[j];
        const double d = cabs2(piv);
        const double2 inv = d > 0.0 ? make_double2(piv.x / d, -piv.y / d) : make_double2(0.0, 0.0);
        best = -1.0;
        bi = N;
        const int step = blockDim.x;
        for (int i = col + 1 + threadIdx.x; i < N; i += 2 * step) {
            const int i2 = i + step;
            const bool two = i2 < N;
            double2 v0[LU_BASE], v1[LU_BASE];
            const double2 a0 = A[(size_t)i + (size_t)col * N];
            const double2 a1 = two ? A[(size_t)i2 + (size_t)col * N] : make_double2(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < LU_BASE; c++) {
                if (c > j && c < w) v0[c] = A[(size_t)i + (size_t)(c0 + c) * N];
                if (two && c > j && c < w) v1[c] = A[(size_t)i2 + (size_t)(c0 + c) * N];
            }
            lu_base_row(A, N, i, c0, col, j, w, inv, prow, a0, v0, best, bi, true);
            lu_base_row(A, N, i2, c0, col, j, w, inv, prow, a1, v1, best, bi, two);
        }
    }
}

// ------------------------------------------------------------------ row interchanges
// The swaps of rows r0 .. r1 - 1 (in order, LAPACK's zlaswp) on the columns [ca, cb) and [cc, cd), one
// thread per column.
__global__ void k_lu_laswp(int N, int r0, int r1, int ca, int cb, int cc, int cd, double2* __restrict__ Aall,
                           size_t stride, const int32_t* __restrict__ ipiv) {
    const int f = blockIdx.y;
    const int t = blockIdx.x * blockDim.x + threadIdx.x, n1 = cb - ca;
    if (t >= n1 + (cd - cc)) return;
    const int col = t < n1 ? ca + t : cc + (t - n1);
    double2* A = Aall + (size_t)f * stride + (size_t)col * N;
    const int32_t* pv = ipiv + (size_t)f * N;
    for (int r = r0; r < r1; r++) {
        const int p = pv[r];
        if (p != r) {
            const double2 x = A[r];
            A[r] = A[p];
            A[p] = x;
        }
    }
}

// ------------------------------------------------------------------ triangular solves of a block row
// B := L^-1 B (lower: L the unit lower n1 x n1 block of the factor at (c0, c0)) or B := U^-1 B (upper: U
// the upper block, diagonal included), B the rows c0 .. c0 + n1 - 1, columns [cb, ce) of the matrix X
// (the factor matrix itself inside the LU, the right-hand sides in the substitution).  The triangle is
// packed by columns in shared memory; a warp takes CPW columns of B at once (independent chains), lane
// l holding rows l, l + 32, ... (NQ of them), each solved entry broadcast by shuffles.
template <int NQ, int CPW, bool UPPER>
__global__ void __launch_bounds__(512) k_lu_trsm(int N, int c0, int n1, int cb, int ce, const double2* __restrict__ Lall,
                                                 size_t lstride, double2* __restrict__ Xall, size_t xstride) {
    extern __shared__ double2 Lc[];
    const int f = blockIdx.y;
    const double2* L = Lall + (size_t)f * lstride;
    double2* X = Xall + (size_t)f * xstride;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // lower: column p holds rows p + 1 .. n1 - 1 at loff(p) + r - p - 1;
    // upper: column p holds rows 0 .. p at uoff(p) + r
    auto loff = [n1](int p) { return p * (2 * n1 - p - 1) / 2; };
    auto uoff = [](int p) { return p * (p + 1) / 2; };
    if (UPPER) {
        for (int p = warp; p < n1; p += nw)
            for (int r = lane; r <= p; r += 32) Lc[uoff(p) + r] = L[(size_t)(c0 + r) + (size_t)(c0 + p) * N];
    } else {
        for (int p = warp; p < n1 - 1; p += nw)
            for (int r = p + 1 + lane; r < n1; r += 32) Lc[loff(p) + r - p - 1] = L[(size_t)(c0 + r) + (size_t)(c0 + p) * N];
    }
    __syncthreads();
    for (int col0 = cb + (blockIdx.x * nw + warp) * CPW; col0 < ce; col0 += gridDim.x * nw * CPW) {
        double2 x[CPW][NQ];
#pragma unroll
        for (int c = 0; c < CPW; c++)
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const int r = lane + 32 * q;
                x[c][q] = (r < n1 && col0 + c < ce) ? X[(size_t)(c0 + r) + (size_t)(col0 + c) * N] : make_double2(0.0, 0.0);
            }
        if (!UPPER) {
#pragma unroll
            for (int sblk = 0; sblk < NQ; sblk++) {
                for (int pp = 0; pp < 32; pp++) {
                    const int p = 32 * sblk + pp;
                    if (p >= n1 - 1) break;
                    double2 xp[CPW];
#pragma unroll
                    for (int c = 0; c < CPW; c++)
                        xp[c] = make_double2(__shfl_sync(0xffffffffu, x[c][sblk].x, pp), __shfl_sync(0xffffffffu, x[c][sblk].y, pp));
                    const int base = loff(p) - p - 1;  // L(r, p) at base + r
#pragma unroll
                    for (int q = sblk; q < NQ; q++) {
                        const int r = lane + 32 * q;
                        if (r > p && r < n1) {
                            const double2 l = Lc[base + r];
#pragma unroll
                            for (int c = 0; c < CPW; c++) x[c][q] = csub(x[c][q], cmul(l, xp[c]));
                        }
                    }
                }
            }
        } else {
#pragma unroll
            for (int sblk = NQ - 1; sblk >= 0; sblk--) {
                for (int pp = 31; pp >= 0; pp--) {
                    const int p = 32 * sblk + pp;
                    if (p >= n1) continue;
                    const double2 d = Lc[uoff(p) + p];
                    const double dd = cabs2(d);
                    const double2 dinv = dd > 0.0 ? make_double2(d.x / dd, -d.y / dd) : make_double2(0.0, 0.0);
                    double2 xp[CPW];
#pragma unroll
                    for (int c = 0; c < CPW; c++) {
                        if (lane == pp) x[c][sblk] = cmul(x[c][sblk], dinv);
                        xp[c] = make_double2(__shfl_sync(0xffffffffu, x[c][sblk].x, pp), __shfl_sync(0xffffffffu, x[c][sblk].y, pp));
                    }
#pragma unroll
                    for (int q = 0; q <= sblk; q++) {
                        const int r = lane + 32 * q;
                        if (r < p) {
                            const double2 u = Lc[uoff(p) + r];
#pragma unroll
                            for (int c = 0; c < CPW; c++) x[c][q] = csub(x[c][q], cmul(u, xp[c]));
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < CPW; c++)
#pragma unroll
            for (int q = 0; q < NQ; q++) {
                const int r = lane + 32 * q;
                if (r < n1 && col0 + c < ce) X[(size_t)(c0 + r) + (size_t)(col0 + c) * N] = x[c][q];
            }
    }
}

template <bool UPPER>
static void launch_lu_trsm(int N, int F, int c0, int n1, int cb, int ce, const double2* L, size_t lstride, double2* X,
                           size_t xstride, cudaStream_t s) {
    constexpr int CPW = 4, threads = 512, nw = threads / 32;
    const int cols = ce - cb;
    const size_t sm = sizeof(double2) * (size_t)n1 * (UPPER ? n1 + 1 : n1 - 1) / 2;
    // each CTA loads the triangle once and walks many columns: a few CTAs per matrix
    const int gx = std::max(1, std::min((cols + nw * CPW - 1) / (nw * CPW), 16));
    const dim3 g(gx, F);
    if (n1 <= 32)
        k_lu_trsm<1, CPW, UPPER><<<g, threads, sm, s>>>(N, c0, n1, cb, ce, L, lstride, X, xstride);
    else if (n1 <= 64)
        k_lu_trsm<2, CPW, UPPER><<<g, threads, sm, s>>>(N, c0, n1, cb, ce, L, lstride, X, xstride);
    else
        k_lu_trsm<4, CPW, UPPER><<<g, threads, sm, s>>>(N, c0, n1, cb, ce, L, lstride, X, xstride);
}

// ------------------------------------------------------------------ trailing update on FP64 warp MMA
// C -= A B for each matrix of the batch (A rows r0 .., columns k0 .. k0 + K of one matrix; B rows k0 ..
// k0 + K, columns c0 .. and C rows r0 .., columns c0 .. of another -- the same one inside the LU, the
// right-hand sides in the substitution), complex128 column-major, leading dimension N.  The complex product as a real
// one on the interleaved (re, im) layout: C_r (2M x n) -= Ahat (2M x 2K) B_r (2K x n), where B_r and C_r
// are the matrices' own memory read as doubles and Ahat(2r + c, 2k + c') is a_r, -a_i, a_i, a_r for
// (c, c') = (0, 0), (0, 1), (1, 0), (1, 1), read on the fly from A's interleaved tile.  Tiles of 64 complex
// rows x 32 WN columns per CTA, 4 x WN warps of 32 real rows x 32 columns (4 x 4 m8n8k4 f64 tiles each), K
// staged by cp.async in chunks of 16 complex (double-buffered, zero-filled beyond the edges).  The sums
// are staged through shared memory (the operand buffers, free by then) so that C is read and written in
// whole columns with all of a thread's loads in flight together: one memory round trip per tile, which
// is what a tall, narrow product of the recursion (K and n of 8 to 64) costs most.  WN = 2 (64 columns,
// two CTAs an SM) for the wide trailing updates, WN = 1 (32 columns, four CTAs an SM) for narrow ones.
template <int WN>
struct ZgTile {
    static constexpr int T = 128 * WN;     // threads: 4 x WN warps
    static constexpr int ZM = 64;          // complex rows of the tile
    static constexpr int ZN = 32 * WN;     // columns of the tile
    static constexpr int ZK = 16;          // complex k of a staged chunk
    static constexpr int AP = 2 * ZM + 8;  // doubles per k-column of the A tile (padded: conflict-free fragments)
    static constexpr int BP = 2 * ZK + 4;  // doubles per column of the B tile
    static constexpr int CP = 2 * ZM + 4;  // doubles per column of the staged sums (4 mod 16: two wavefronts a store)
    static constexpr int SMEM = 2 * (ZK * AP + ZN * BP) * 8;
    static_assert(ZN * CP * 8 <= SMEM, "the staged sums fit in the operand buffers");
};
constexpr int ZG_NARROW = 1024;  // products of at most this many columns take the 32-column tiles

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool ok) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gmem), "r"(ok ? 16 : 0) : "memory");
}

template <int WN>
__global__ void __launch_bounds__(128 * WN, 4 / WN) k_lu_zgemm(int N, const double2* Aall, size_t astride, double2* Call,
                                                             size_t cstride, int r0, int c0, int k0, int M, int n, int K) {
    using G = ZgTile<WN>;
    extern __shared__ double zg_smem[];
    double* As = zg_smem;                      // [2][ZK][AP]
    double* Bs = zg_smem + 2 * G::ZK * G::AP;  // [2][ZN][BP]
    const int f = blockIdx.z;
    const double2* A = Aall + (size_t)f * astride;  // the A operand (rows r0 .., columns k0 ..)
    double2* C = Call + (size_t)f * cstride;        // the B operand (rows k0 .., columns c0 ..) and C
    const int tm = blockIdx.x * G::ZM, tn = blockIdx.y * G::ZN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp & 3, wn = warp >> 2;
    const int nchunk = (K + G::ZK - 1) / G::ZK;
    auto load = [&](int buf, int kc) {
#pragma unroll
        for (int q = 0; q < G::ZK * G::ZM / G::T; q++) {  // A: k-column kk, complex row rr
            const int idx = tid + G::T * q, kk = idx / G::ZM, rr = idx % G::ZM, kg = kc * G::ZK + kk;
            const bool ok = tm + rr < M && kg < K;
            const double2* src = ok ? A + (size_t)(r0 + tm + rr) + (size_t)(k0 + kg) * N : A;
            cp_async16(As + (size_t)(buf * G::ZK + kk) * G::AP + 2 * rr, src, ok);
        }
#pragma unroll
        for (int q = 0; q < G::ZK * G::ZN / G::T; q++) {  // B: column cc, complex row kk
            const int idx = tid + G::T * q, cc = idx / G::ZK, kk = idx % G::ZK, kg = kc * G::ZK + kk;
            const bool ok = tn + cc < n && kg < K;
            const double2* src = ok ? C + (size_t)(k0 + kg) + (size_t)(c0 + tn + cc) * N : C;
            cp_async16(Bs + (size_t)(buf * G::ZN + cc) * G::BP + 2 * kk, src, ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
    load(0, 0);
    for (int kc = 0; kc < nchunk; kc++) {
        if (kc + 1 < nchunk) {
            load((kc + 1) & 1, kc + 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const double* Ab = As + (size_t)(kc & 1) * G::ZK * G::AP;
        const double* Bb = Bs + (size_t)(kc & 1) * G::ZN * G::BP;
#pragma unroll
        for (int ks = 0; ks < 2 * G::ZK / 4; ks++) {
            const int kq = 4 * ks + (lane & 3), k = kq >> 1, cpart = kq & 1;
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int R = wm * 32 + 8 * i + (lane >> 2);
                const double v = Ab[k * G::AP + (R ^ cpart)];
                a[i] = ((R & 1) == 0 && cpart) ? -v : v;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bb[(wn * 32 + 8 * j + (lane >> 2)) * G::BP + kq];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                                 : "+d"(acc[i][j][0]), "+d"(acc[i][j][1])
                                 : "d"(a[i]), "d"(b[j]));
        }
        __syncthreads();  // the buffer is refilled by the next iteration's load (or holds the sums below)
    }
    // the sums, column by column (real row R = 2 r + part), then C -= them a whole column at a time
    double* Cs = zg_smem;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int e = 0; e < 2; e++)
                Cs[(wn * 32 + 8 * j + 2 * (lane & 3) + e) * G::CP + wm * 32 + 8 * i + (lane >> 2)] = acc[i][j][e];
    __syncthreads();
    constexpr int PER = G::ZM * G::ZN / G::T;
    double2 cv[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int idx = tid + G::T * q, r = idx % G::ZM, c = idx / G::ZM;
        if (tm + r < M && tn + c < n) cv[q] = C[(size_t)(r0 + tm + r) + (size_t)(c0 + tn + c) * N];
    }
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int idx = tid + G::T * q, r = idx % G::ZM, c = idx / G::ZM;
        if (tm + r < M && tn + c < n) {
            const double2 sum = *reinterpret_cast<const double2*>(Cs + c * G::CP + 2 * r);
            C[(size_t)(r0 + tm + r) + (size_t)(c0 + tn + c) * N] = make_double2(cv[q].x - sum.x, cv[q].y - sum.y);
        }
    }
}

static void lu_zgemm_attributes() {
    cudaFuncSetAttribute(k_lu_zgemm<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, ZgTile<1>::SMEM);
    cudaFuncSetAttribute(k_lu_zgemm<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ZgTile<2>::SMEM);
}

// The tile width of a product of n columns, autotuned per device: when the device is first used
// (before any solve's work is queued on it) both widths are timed on a product of each width bucket
// n <= 8, 16, ..., 2048 and 4096 (2048 rows, K = min(n, 128), four matrices, the best of three launches
// each, on scratch buffers freed afterwards) and the 64-column tile is taken where it is at least 2 %
// faster.  Until then, or if the timing cannot run, products of at most ZG_NARROW columns take the
// 32-column tile (the choice the measurements on the benchmark's shapes gave).
constexpr int ZG_TUNE_BUCKETS = 10;
struct ZgTune {
    std::atomic<bool> ready{false};
    bool measured = false;
    bool wide[ZG_TUNE_BUCKETS] = {};
    float us[ZG_TUNE_BUCKETS][2] = {};
};
static ZgTune g_zg_tune[16];

static int zg_bucket(int n) {
    int b = 0;
    while (b < ZG_TUNE_BUCKETS - 1 && n > (8 << b)) b++;
    return b;
}

static void launch_lu_zgemm_wn(bool wide, int N, int F, const double2* A, size_t astride, double2* C, size_t cstride,
                               int r0, int c0, int k0, int M, int n, int K, cudaStream_t s) {
    if (!wide) {
        using G = ZgTile<1>;
        k_lu_zgemm<1><<<dim3((M + G::ZM - 1) / G::ZM, (n + G::ZN - 1) / G::ZN, F), G::T, G::SMEM, s>>>(
            N, A, astride, C, cstride, r0, c0, k0, M, n, K);
    } else {
        using G = ZgTile<2>;
        k_lu_zgemm<2><<<dim3((M + G::ZM - 1) / G::ZM, (n + G::ZN - 1) / G::ZN, F), G::T, G::SMEM, s>>>(
            N, A, astride, C, cstride, r0, c0, k0, M, n, K);
    }
}

// C -= A B over the batch of F matrices (the arguments of k_lu_zgemm), the tile width as tuned
static void launch_lu_zgemm(int N, int F, const double2* A, size_t astride, double2* C, size_t cstride, int r0, int c0,
                            int k0, int M, int n, int K, cudaStream_t s) {
    if (M <= 0 || n <= 0 || K <= 0) return;
    int dev = 0;
    cudaGetDevice(&dev);
    const ZgTune& t = g_zg_tune[dev < 0 || dev >= 16 ? 0 : dev];
    const bool wide = t.ready.load(std::memory_order_acquire) ? t.wide[zg_bucket(n)] : n > ZG_NARROW;
    launch_lu_zgemm_wn(wide, N, F, A, astride, C, cstride, r0, c0, k0, M, n, K, s);
}

void lu_tune_device(int dev) {
    if (dev < 0 || dev >= 16) return;
    ZgTune& t = g_zg_tune[dev];
    if (t.ready.load(std::memory_order_acquire)) return;
    for (int b = 0; b < ZG_TUNE_BUCKETS; b++) t.wide[b] = (8 << b) > ZG_NARROW;
    constexpr int M = 2048, F = 4, KMAX = 128, NMAX = 8 << (ZG_TUNE_BUCKETS - 1);
    const int N = M + KMAX;  // leading dimension: B in rows 0 .. K - 1, C in rows KMAX .. N - 1
    const size_t astride = (size_t)N * KMAX, cstride = (size_t)N * NMAX;
    double2 *A = nullptr, *C = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    bool ok = cudaMalloc(&A, sizeof(double2) * astride * F) == cudaSuccess &&
              cudaMalloc(&C, sizeof(double2) * cstride * F) == cudaSuccess &&
              cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
    if (ok) {
        lu_zgemm_attributes();
        ok = cudaMemsetAsync(A, 0, sizeof(double2) * astride * F, s) == cudaSuccess &&
             cudaMemsetAsync(C, 0, sizeof(double2) * cstride * F, s) == cudaSuccess;
        for (int b = 0; ok && b < ZG_TUNE_BUCKETS; b++) {
            const int n = 8 << b, K = std::min(n, KMAX);
            for (int w = 0; w < 2; w++) {
                float best = 1e30f;
                launch_lu_zgemm_wn(w == 1, N, F, A, astride, C, cstride, KMAX, 0, 0, M, n, K, s);
                for (int r = 0; r < 3 && ok; r++) {
                    cudaEventRecord(e0, s);
                    launch_lu_zgemm_wn(w == 1, N, F, A, astride, C, cstride, KMAX, 0, 0, M, n, K, s);
                    cudaEventRecord(e1, s);
                    float ms = 0.f;
                    ok = cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
                    best = std::min(best, ms);
                }
                t.us[b][w] = 1e3f * best;
            }
            t.wide[b] = t.us[b][1] < 0.98f * t.us[b][0];
        }
        t.measured = ok;
        if (!ok)
            for (int b = 0; b < ZG_TUNE_BUCKETS; b++) t.wide[b] = (8 << b) > ZG_NARROW;
    }
    cudaGetLastError();  // a failed timing leaves the heuristic choice, not an error for the solve
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (A) cudaFree(A);
    if (C) cudaFree(C);
    t.ready.store(true, std::memory_order_release);
}

int lu_tuned_tiles(int dev, int32_t* wide, float* us) {
    if (dev < 0 || dev >= 16) return 0;
    const ZgTune& t = g_zg_tune[dev];
    if (!t.ready.load(std::memory_order_acquire)) return 0;
    for (int b = 0; b < ZG_TUNE_BUCKETS; b++) {
        wide[b] = t.wide[b] ? 1 : 0;
        us[2 * b] = t.us[b][0];
        us[2 * b + 1] = t.us[b][1];
    }
    return t.measured ? 2 : 1;
}

// ------------------------------------------------------------------ the factorization
namespace {
// The schedule: the matrices of a batch in `groups` groups, and with look-ahead each group on two streams
// -- the panel stream factors panel b + 1 (after the update of its own columns) while the update stream
// applies panel b to the columns beyond it (linalg.rs:134-185's look-ahead, with streams for threads).
struct LuF64Schedule {
    int groups = LU_F64_GROUPS;
    int lookahead = 1;
};
LuF64Schedule& lu_f64_schedule_ref() {
    static LuF64Schedule s;
    return s;
}

struct LuF64Streams {
    cudaStream_t p[LU_F64_MAX_GROUPS] = {}, u[LU_F64_MAX_GROUPS] = {};
    cudaEvent_t fork = nullptr, ep[LU_F64_MAX_GROUPS] = {}, eu[LU_F64_MAX_GROUPS] = {};
    cudaEvent_t joinp[LU_F64_MAX_GROUPS] = {}, joinu[LU_F64_MAX_GROUPS] = {};
    bool ok = false;
};
LuF64Streams& lu_f64_streams() {
    static thread_local LuF64Streams t[16];
    int d = 0;
    cudaGetDevice(&d);
    if (d < 0 || d >= 16) d = 0;
    LuF64Streams& x = t[d];
    if (!x.ok) {
        bool ok = true;
        auto ev = [&](cudaEvent_t* e) { ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess; };
        // the panel streams at the highest priority: a panel's CTAs take the first SM slots that the
        // update stream's trailing product frees, so the panel chain stays ahead of the products
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        for (int i = 0; i < LU_F64_MAX_GROUPS; i++) {
            ok = ok && cudaStreamCreateWithPriority(&x.p[i], cudaStreamNonBlocking, hi) == cudaSuccess;
            ok = ok && cudaStreamCreateWithFlags(&x.u[i], cudaStreamNonBlocking) == cudaSuccess;
            ev(&x.ep[i]);
            ev(&x.eu[i]);
            ev(&x.joinp[i]);
            ev(&x.joinu[i]);
        }
        ev(&x.fork);
        x.ok = ok;
    }
    return x;
}

struct LuF64 {
    int N, F;  // matrix order, matrices of this group
    double2* A;
    size_t stride;
    int32_t* ipiv;
    int32_t* info;
    cudaStream_t sp, su;  // panel stream, update stream (the same without look-ahead)
    cudaEvent_t ep, eu;   // the panel stream's part of a step done, the update stream's part done
    int64_t* launches;

    void laswp(cudaStream_t s, int r0, int r1, int ca, int cb, int cc, int cd) {
        const int cols = (cb - ca) + (cd - cc);
        if (cols <= 0 || r1 <= r0) return;
        KernelProfiler& P = profiler();
        P.begin(s);
        k_lu_laswp<<<dim3((cols + 127) / 128, F), 128, 0, s>>>(N, r0, r1, ca, cb, cc, cd, A, stride, ipiv);
        P.end(KF_LU_LASWP, (double)F * cols * (r1 - r0) * 64.0, s);
        (*launches)++;
    }
    void trsm(cudaStream_t s, int c0, int n1, int cb, int ce) {
        if (ce <= cb || n1 <= 1) return;
        KernelProfiler& P = profiler();
        P.begin(s);
        launch_lu_trsm<false>(N, F, c0, n1, cb, ce, A, stride, A, stride, s);
        // complex TRSM: 4 n1^2 cols real flops
        P.end(KF_LU_TRSM, (double)F * 4.0 * n1 * (double)n1 * (ce - cb), s);
        (*launches)++;
    }
    void gemm(cudaStream_t s, int r0, int c0, int k0, int M, int n, int K) {
        if (M <= 0 || n <= 0 || K <= 0) return;
        KernelProfiler& P = profiler();
        P.begin(s);
        launch_lu_zgemm(N, F, A, stride, A, stride, r0, c0, k0, M, n, K, s);
        // complex C -= A B: 8 M n K real flops
        P.end(KF_LU_GEMM, (double)F * 8.0 * M * (double)n * K, s);
        (*launches)++;
    }
    // columns c0 .. c0 + w - 1, rows c0 .. N - 1 of the panel pk0 .. pk0 + pnb - 1 (dgetrf2's recursion:
    // the left half, the triangular solve of the right half's block row, the update of the right half,
    // the right half; the strips swap their rows across the whole panel, so no interchanges between)
    int pk0 = 0, pnb = 0;
    void panel(int c0, int w) {
        if (w <= LU_BASE) {
            KernelProfiler& P = profiler();
            const double m = N - c0;
            P.begin(sp);
            k_lu_base<<<F, 512, 0, sp>>>(N, c0, w, pk0, pnb, A, stride, ipiv, info);
            P.end(KF_LU_PANEL, (double)F * 8.0 * (m * w * w - (double)w * w * w / 3.0), sp);
            (*launches)++;
            return;
        }
        const int n1 = w / 2 / LU_BASE * LU_BASE > 0 ? w / 2 / LU_BASE * LU_BASE : w / 2, n2 = w - n1;
        panel(c0, n1);
        trsm(sp, c0, n1, c0 + n1, c0 + w);
        gemm(sp, c0 + n1, c0 + n1, c0, N - c0 - n1, n2, n1);
        panel(c0 + n1, n2);
    }
    // right-looking, one stream: panel, interchanges, block row, trailing update
    void factor() {
        for (int k0 = 0; k0 < N; k0 += LU_NB) {
            const int nb = std::min(LU_NB, N - k0);
            pk0 = k0;
            pnb = nb;
            panel(k0, nb);
            laswp(sp, k0, k0 + nb, 0, k0, k0 + nb, N);
            trsm(sp, k0, nb, k0 + nb, N);
            gemm(sp, k0 + nb, k0 + nb, k0, N - k0 - nb, N - k0 - nb, nb);
        }
    }
    // with look-ahead: step b's panel stream factors panel b (columns k0 .. k1) and signals the update
    // stream, which swaps rows and solves the block row on the columns k2 .. N and applies panel b to
    // them; the panel stream meanwhile waits for the update stream's step b - 1 (which wrote columns k1 ..
    // and read panel b - 1's factor columns that these interchanges reach), then applies panel b to the
    // left columns and to panel b + 1's columns (k1 .. k2) and goes on to panel b + 1 while the update
    // stream's product of step b runs.  Every column range is written by one stream at a time, in the
    // order of the plain schedule, so the factors are the same to the bit.
    void factor_lookahead() {
        for (int k0 = 0, b = 0; k0 < N; k0 += LU_NB, b++) {
            const int nb = std::min(LU_NB, N - k0), k1 = k0 + nb, k2 = std::min(N, k1 + LU_NB);
            pk0 = k0;
            pnb = nb;
            panel(k0, nb);
            if (k2 < N) {
                cudaEventRecord(ep, sp);
                cudaStreamWaitEvent(su, ep, 0);
                laswp(su, k0, k1, k2, N, 0, 0);
                trsm(su, k0, nb, k2, N);
                gemm(su, k1, k2, k0, N - k1, N - k2, nb);
            }
            if (b > 0) cudaStreamWaitEvent(sp, eu, 0);
            if (k2 < N) cudaEventRecord(eu, su);
            laswp(sp, k0, k1, 0, k0, k1, k2);
            trsm(sp, k0, nb, k1, k2);
            gemm(sp, k1, k1, k0, N - k1, k2 - k1, nb);
        }
    }
};
}  // namespace

void lu_f64_schedule(int groups, int lookahead) {
    LuF64Schedule& s = lu_f64_schedule_ref();
    s.groups = std::max(1, std::min(groups, LU_F64_MAX_GROUPS));
    s.lookahead = lookahead ? 1 : 0;
}

static void lu_f64_attributes() {
    lu_zgemm_attributes();
    cudaFuncSetAttribute(k_lu_trsm<4, 4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(double2) * LU_NB * (LU_NB - 1) / 2));
    cudaFuncSetAttribute(k_lu_trsm<4, 4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(double2) * LU_NB * (LU_NB + 1) / 2));
}

int lu_factor_f64(int N, int F, double2* A, size_t stride, int32_t* ipiv, int32_t* info, cudaStream_t s,
                  int64_t* launches) {
    lu_f64_attributes();
    cudaMemsetAsync(info, 0, sizeof(int32_t) * F, s);
    LuF64Streams& side = lu_f64_streams();
    const LuF64Schedule& sched = lu_f64_schedule_ref();
    if (!side.ok) {  // no side streams: one group, no look-ahead, on the caller's stream
        LuF64{N, F, A, stride, ipiv, info, s, s, nullptr, nullptr, launches}.factor();
        return 0;
    }
    const int ng = std::max(1, std::min(sched.groups, F));
    cudaEventRecord(side.fork, s);
    for (int g = 0, f0 = 0; g < ng; g++) {
        const int fg = F / ng + (g < F % ng ? 1 : 0);
        cudaStreamWaitEvent(side.p[g], side.fork, 0);
        cudaStreamWaitEvent(side.u[g], side.fork, 0);
        LuF64 lu{N, fg, A + (size_t)f0 * stride, stride, ipiv + (size_t)f0 * N, info + f0, side.p[g], side.u[g],
                 side.ep[g], side.eu[g], launches};
        if (sched.lookahead)
            lu.factor_lookahead();
        else
            lu.factor();
        cudaEventRecord(side.joinp[g], side.p[g]);
        cudaEventRecord(side.joinu[g], side.u[g]);
        cudaStreamWaitEvent(s, side.joinp[g], 0);
        cudaStreamWaitEvent(s, side.joinu[g], 0);
        f0 += fg;
    }
    return 0;
}

// ------------------------------------------------------------------ substitution
// X = A^-1 B with the factors: the row interchanges gathered into a permutation (one CTA per matrix),
// P B gathered into X, then blocked forward and back substitution over the LU_NB-row blocks: each block
// solved by the triangular kernel (unit lower, then upper with its diagonal), the rest of the right-hand
// sides updated by the warp-MMA product with the block's factor columns -- every factor entry read once
// per direction, all the batch's matrices in each launch.  B and X are [F][nrhs][N].
__global__ void k_lu_permute(int N, const int32_t* __restrict__ ipiv, int nrhs, const double2* __restrict__ Ball,
                             double2* __restrict__ Xall) {
    extern __shared__ int32_t perm[];
    const int f = blockIdx.x;
    const int32_t* pv = ipiv + (size_t)f * N;
    const double2* B = Ball + (size_t)f * nrhs * N;
    double2* X = Xall + (size_t)f * nrhs * N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) perm[i] = i;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < N; i++) {
            const int p = pv[i];
            if (p != i) {
                const int t = perm[i];
                perm[i] = perm[p];
                perm[p] = t;
            }
        }
    __syncthreads();
    for (int c = 0; c < nrhs; c++)
        for (int i = threadIdx.x; i < N; i += blockDim.x) X[(size_t)c * N + i] = B[(size_t)c * N + perm[i]];
}

int lu_solve_f64(int N, int F, const double2* LU, size_t stride, const int32_t* ipiv, int nrhs, const double2* B,
                 double2* X, cudaStream_t s) {
    const size_t smem = sizeof(int32_t) * (size_t)N;
    if (nrhs > 32 || smem > 200 * 1024) return 1;
    lu_f64_attributes();
    cudaFuncSetAttribute(k_lu_permute, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_lu_permute<<<F, 512, smem, s>>>(N, ipiv, nrhs, B, X);
    const size_t xs = (size_t)nrhs * N;
    auto update = [&](int r0, int k0, int M, int K) {
        launch_lu_zgemm(N, F, LU, stride, X, xs, r0, 0, k0, M, nrhs, K, s);
    };
    for (int b0 = 0; b0 < N; b0 += LU_NB) {  // L y = P b
        const int nb = std::min(LU_NB, N - b0);
        if (nb > 1) launch_lu_trsm<false>(N, F, b0, nb, 0, nrhs, LU, stride, X, xs, s);
        update(b0 + nb, b0, N - b0 - nb, nb);
    }
    for (int b0 = (N - 1) / LU_NB * LU_NB; b0 >= 0; b0 -= LU_NB) {  // U x = y, the last block first
        const int nb = std::min(LU_NB, N - b0);
        launch_lu_trsm<true>(N, F, b0, nb, 0, nrhs, LU, stride, X, xs, s);
        update(0, b0, b0, nb);
    }
    return 0;
}

}  // namespace hbg
