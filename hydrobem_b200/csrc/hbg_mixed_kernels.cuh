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
#include <cuda_fp16.h>

#include "hbg_tc.cuh"

namespace hbg {

constexpr int NBL = 128;  // LU block width (complex columns)
constexpr int GBM = 128, GBK = 32, GSTAGES = 4, GBN = 256;
constexpr int GNBOX = 2;  // ring of 32-column output boxes in shared memory

struct GemmArgs {
    int M, Nc, Kp;         // rows, real output columns, real inner dimension
    int a_planar;          // A from the planar matrix (x = a_x0 + kk % a_kc, plane = kk / a_kc) or a packed buffer
    int a_x0, a_kc, a_row0;
    int mode;              // 0 store, 1 store and scatter into the GEMM3 operand, 2 subtract
    int o_row0, o_col0, o_nc;  // output placement in the planar matrix: column j' -> plane j' / o_nc
    int batch;             // matrices in the launch
    int b0;                // index of the launch's first matrix in the tensor maps
    int b_split;           // 0: B coordinates (kk, row); > 0: B viewed as [row][2][.]: (kk % b_split, kk / b_split, row)
    float* p3;             // a later update's B operand [F][2 p3_n][p3_ld] (mode 1)
    size_t p3_bstride;
    int p3_n;
    int p3_ld, p3_kh, p3_koff;  // row length, offset of the second (imaginary-weight) half, first row of this block
    __half* p3h;           // mode 1: an FP16 copy of the p3 scatter (same layout), or null
    // mode 0: an FP16 copy of the output rows from h16_row0 on, [F][rows][h16_ld]: output column j' of
    // plane p at p * (h16_ld / 2) + h16_koff + j' % o_nc, row o_row0 + i at o_row0 + i - h16_row0
    __half* h16;
    size_t h16_bstride;
    int h16_ld, h16_row0, h16_koff;
    int* err;
};

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
    return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

constexpr int GEMM_THREADS = 192;  // warp 0 TMA, warp 1 MMA, warps 2..5 epilogue
constexpr size_t GEMM_STAGE_BYTES = (size_t)(GBM + GBN) * GBK * 4;
constexpr size_t GEMM_BOX_BYTES = (size_t)GBM * 32 * 4;  // one 32-column box of the output tile
constexpr size_t gemm_smem_bytes() { return 1024 + GSTAGES * GEMM_STAGE_BYTES + GNBOX * GEMM_BOX_BYTES + 256; }

// Persistent, warp-specialized TF32 GEMM of the mixed LU: tiles of 128 x 256 (real columns) taken
// round-robin over (row tile, column tile, matrix).  Warp 0 lane 0 streams the A/B k-chunks through a
// 3-stage TMA ring; warp 1 lane 0 issues tcgen05.mma (M 128, N 256) into one of two TMEM
// accumulators; warps 2..5 read the accumulator (tcgen05.ld) in 32-column chunks, place each chunk in
// a ring of four shared-memory boxes (128-byte swizzle, conflict-free 16-byte accesses) and write it
// out by TMA: a store, or for the trailing update a TMA reduction that adds -acc to C in L2 (so C
// never passes through the SM).  The epilogue of one tile overlaps the main loop of the next.
// F16: the same pipeline on FP16 operands (kind::f16, 64 halves per 128-byte k-chunk row, packed A only).
template <bool F16 = false>
__global__ void __launch_bounds__(GEMM_THREADS, 1) k_gemm_tf32(const __grid_constant__ CUtensorMap mapA,
                                                               const __grid_constant__ CUtensorMap mapB,
                                                               const __grid_constant__ CUtensorMap mapC,
                                                               GemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = align1024(smem_raw);
    float* sA = reinterpret_cast<float*>(base);
    float* sB = sA + GSTAGES * GBM * GBK;
    float* sBox = sB + GSTAGES * GBN * GBK;  // [GNBOX][128 rows][32]
    uint64_t* full = reinterpret_cast<uint64_t*>(sBox + GNBOX * GBM * 32);
    uint64_t* empty = full + GSTAGES;
    uint64_t* tfull = empty + GSTAGES;  // [2]
    uint64_t* tempty = tfull + 2;       // [2]
    uint64_t* drain = tempty + 2;       // the MMA warp's last commit (every issued MMA complete)
    uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = (g.M + GBM - 1) / GBM, nt = (g.Nc + GBN - 1) / GBN;
    const int ntiles = mt * nt * g.batch;
    constexpr int KE = F16 ? 2 * GBK : GBK;  // operand elements per k-chunk (128 bytes a row either way)
    const int nk = g.Kp / KE;
    if (threadIdx.x == 0) {
        for (int s = 0; s < GSTAGES; s++) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            tc::mbar_init(&tfull[b], 1);
            tc::mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
        }
        tc::mbar_init(drain, 1);
        tc::fence_barrier_init();
        tc::prefetch_tensormap(&mapA);
        tc::prefetch_tensormap(&mapB);
        tc::prefetch_tensormap(&mapC);
    }
    if (warp == 0) tc::tmem_alloc(tslot, 2 * GBN);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tslot;
    auto tile_coords = [&](int t, int& m0, int& n0, int& f) {
        f = g.b0 + t / (mt * nt);
        int r = t % (mt * nt);
        n0 = (r / mt) * GBN;  // row tiles fastest: consecutive CTAs share the B block
        m0 = (r % mt) * GBM;
    };
    if (warp == 0) {
        if (lane == 0) {
            int kc_global = 0;
            bool bad = false;
            for (int t = blockIdx.x; t < ntiles && !bad; t += gridDim.x) {
                int m0, n0, f;
                tile_coords(t, m0, n0, f);
                for (int kc = 0; kc < nk; kc++, kc_global++) {
                    const int s = kc_global % GSTAGES;
                    if (kc_global >= GSTAGES && !tc::mbar_wait(&empty[s], ((kc_global / GSTAGES) - 1) & 1)) {
                        atomicExch(g.err, 1);
                        bad = true;
                        break;
                    }
                    tc::mbar_arrive_expect_tx(&full[s], (uint32_t)GEMM_STAGE_BYTES);
                    const int kk = kc * KE;
                    int ax = kk, plane = 0;
                    if (!F16 && g.a_planar) {
                        ax = g.a_x0 + kk % g.a_kc;
                        plane = kk / g.a_kc;
                    }
                    tc::tma_load_4d(sA + s * GBM * GBK, &mapA, &full[s], ax, g.a_row0 + m0, plane, f);
                    if (g.b_split)
                        tc::tma_load_4d(sB + s * GBN * GBK, &mapB, &full[s], kk % g.b_split, kk / g.b_split, n0, f);
                    else
                        tc::tma_load_4d(sB + s * GBN * GBK, &mapB, &full[s], kk, n0, 0, f);
                }
            }
            // every load still in flight lands before the CTA leaves (also after an error): the last
            // phase armed on each stage completes (bounded)
            for (int k = kc_global > GSTAGES ? kc_global - GSTAGES : 0; k < kc_global; k++)
                if (!tc::mbar_wait(&full[k % GSTAGES], (k / GSTAGES) & 1)) {
                    atomicExch(g.err, 6);
                    break;
                }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = F16 ? tc::idesc_f16(GBM, GBN) : tc::idesc_tf32(GBM, GBN);
            int kc_global = 0, it = 0;
            for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
                const int b = it & 1;
                // the accumulator buffer must have been drained by the epilogue of tile it - 2
                if (it >= 2 && !tc::mbar_wait(&tempty[b], ((it >> 1) - 1) & 1)) {
                    atomicExch(g.err, 5);
                    break;
                }
                tc::tc_fence_after();
                const uint32_t d = tmem + b * GBN;
                bool bad = false;
                for (int kc = 0; kc < nk; kc++, kc_global++) {
                    const int s = kc_global % GSTAGES;
                    if (!tc::mbar_wait(&full[s], (kc_global / GSTAGES) & 1)) {
                        atomicExch(g.err, 2);
                        bad = true;
                        break;
                    }
                    tc::tc_fence_after();
                    const uint32_t a0 = tc::smem_u32(sA + s * GBM * GBK), b0 = tc::smem_u32(sB + s * GBN * GBK);
                    // four MMAs per 128-byte row: K = 8 (tf32) or 16 (f16), 32 bytes apart
#pragma unroll
                    for (int k8 = 0; k8 < 4; k8++) {
                        if constexpr (F16)
                            tc::mma_f16(d, tc::desc_kmajor_sw128(a0 + 32 * k8), tc::desc_kmajor_sw128(b0 + 32 * k8),
                                        idesc, (kc | k8) != 0);
                        else
                            tc::mma_tf32(d, tc::desc_kmajor_sw128(a0 + 32 * k8), tc::desc_kmajor_sw128(b0 + 32 * k8),
                                         idesc, (kc | k8) != 0);
                    }
                    tc::mma_commit(&empty[s]);
                }
                tc::mma_commit(&tfull[b]);
                if (bad) break;
            }
            // every issued MMA completes before TMEM is freed (also after an error; bounded)
            tc::mma_commit(drain);
            if (!tc::mbar_wait(drain, 0)) atomicExch(g.err, 7);
        }
    } else {
        // epilogue warps 2..5: TMEM lane quadrant (warp % 4), rows 32 (warp % 4) .. + 32 of the tile;
        // thread 64 (warp 2, lane 0) issues the box writes and tracks their bulk groups
        const int quad = warp & 3;
        const int r = quad * 32 + lane;  // row within the tile
        const bool issuer = threadIdx.x == 64;
        int it = 0, bx = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
            int m0, n0, f;
            tile_coords(t, m0, n0, f);
            const int b = it & 1;
            const bool ok = tc::mbar_wait(&tfull[b], (it >> 1) & 1);
            // one decision for the four epilogue warps, so none waits at a barrier the others left
            __syncwarp();
            if (!tc::bar_and(ok, 1, 128)) {
                if (issuer) atomicExch(g.err, 3);
                break;
            }
            tc::tc_fence_after();
            for (int q = 0; q < GBN / 32; q++, bx++) {
                float v[32];
                tc::tmem_ld32(tmem + b * GBN + ((uint32_t)(quad * 32) << 16) + q * 32, v);
                const int jg = n0 + 32 * q;  // real output column of the chunk
                const bool live = jg < g.Nc;
                const int plane = jg >= g.o_nc ? 1 : 0, col = jg - plane * g.o_nc;
                // the box slot is free once the write issued GNBOX boxes ago has read it
                if (issuer && bx >= GNBOX) tc::bulk_wait_read_n<GNBOX - 1>();
                asm volatile("bar.sync 1, 128;" ::: "memory");
                float* row = sBox + (bx % GNBOX) * GBM * 32 + r * 32;  // 128 B, 16-byte chunks swizzled by r % 8
                const float sg = g.mode == 2 ? -1.f : 1.f;  // the trailing update adds -acc to C
#pragma unroll
                for (int j = 0; j < 8; j++)
                    *reinterpret_cast<float4*>(row + 4 * (j ^ (r & 7))) =
                        make_float4(sg * v[4 * j], sg * v[4 * j + 1], sg * v[4 * j + 2], sg * v[4 * j + 3]);
                if (g.mode == 1 && live && m0 + r < g.M) {
                    // U(kk = row, j) into the block-real K-major operand of a later update (rows 2n,
                    // p3_ld wide): row j [Ur(:, j) | -Ui(:, j)], row n + j [Ui(:, j) | Ur(:, j)]
                    float* p3f = g.p3 + (size_t)f * g.p3_bstride;
                    __half* p3hf = g.p3h ? g.p3h + (size_t)f * g.p3_bstride : nullptr;
                    const int n = g.p3_n, kk = g.p3_koff + m0 + r, ld = g.p3_ld, kh = g.p3_kh;
#pragma unroll
                    for (int i = 0; i < 32; i++) {
                        const int j = col + i;
                        size_t o1, o2;
                        float w1;
                        if (plane == 0) {
                            o1 = (size_t)j * ld + kk;
                            o2 = (size_t)(n + j) * ld + kh + kk;
                            w1 = v[i];
                        } else {
                            o1 = (size_t)j * ld + kh + kk;
                            o2 = (size_t)(n + j) * ld + kk;
                            w1 = -v[i];
                        }
                        p3f[o1] = w1;
                        p3f[o2] = v[i];
                        if (p3hf) {
                            p3hf[o1] = __float2half_rn(w1);
                            p3hf[o2] = __float2half_rn(v[i]);
                        }
                    }
                }
                if (g.mode == 0 && g.h16 && live && m0 + r < g.M && g.o_row0 + m0 + r >= g.h16_row0) {
                    __half* h = g.h16 + (size_t)f * g.h16_bstride + (size_t)(g.o_row0 + m0 + r - g.h16_row0) * g.h16_ld +
                                plane * (g.h16_ld / 2) + g.h16_koff + col;
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        __half2 hv[4];
#pragma unroll
                        for (int e = 0; e < 4; e++) hv[e] = __floats2half2_rn(v[8 * j + 2 * e], v[8 * j + 2 * e + 1]);
                        *reinterpret_cast<uint4*>(h + 8 * j) = *reinterpret_cast<const uint4*>(hv);
                    }
                }
                tc::fence_proxy_async_smem();
                asm volatile("bar.sync 1, 128;" ::: "memory");
                if (issuer) {
                    const float* box = sBox + (bx % GNBOX) * GBM * 32;
                    if (live) {
                        if (g.mode == 2)
                            tc::tma_reduce_add_4d(&mapC, box, g.o_col0 + col, g.o_row0 + m0, plane, f);
                        else
                            tc::tma_store_4d(&mapC, box, g.o_col0 + col, g.o_row0 + m0, plane, f);
                    }
                    tc::bulk_commit();  // one group per box (empty for a chunk beyond the output)
                }
            }
            // the accumulator buffer is free for the MMA of tile it + 2
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&tempty[b]);
        }
        if (issuer) tc::bulk_wait_all();
    }
    tc::tc_fence_before();
    __syncthreads();
    // freed even when a drain wait above gave up (err set, the results discarded): a CTA that left
    // holding TMEM would stall every later allocation on its SM
    if (warp == 0) tc::tmem_dealloc(tmem, 2 * GBN);
}

// ---- the diagonal block: M11 = L11 U11 (no pivoting), then L11^-1 and U11^-1.  Two CTAs per matrix
// (blockIdx.x = 2 f + side) factor the same block in their own shared memory; side 0 then forms L^-1
// (and writes the factors back to W), side 1 U^-1.  Outputs: PL ([Lr | Li] rows of L^-1, the A operand
// of GEMM2, [F][NBL][2 NBL]), PU (U^-1 in the block-real K-major form, the B operand of GEMM1,
// [F][2 NBL][2 NBL]) and DINV (U^-1 on and above the diagonal, L^-1 below it, per block, for the
// triangular solves).  A pivot of modulus below 1e-15 sets err (the mixed form then reports the
// frequency; the FP64 form pivots).
constexpr int DF_THREADS = 512, DF_LD = NBL + 1, DF_BLK = 32, DF_NB = NBL / DF_BLK, DF_SLD = DF_BLK + 1;

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// complex multiply-adds as four FMA instructions (no separate product and sum)
__device__ __forceinline__ void cfma_sub(float2& x, float2 a, float2 b) {  // x -= a b
    x.x = fmaf(-a.x, b.x, x.x);
    x.x = fmaf(a.y, b.y, x.x);
    x.y = fmaf(-a.x, b.y, x.y);
    x.y = fmaf(-a.y, b.x, x.y);
}
__device__ __forceinline__ void cfma_add(float2& x, float2 a, float2 b) {  // x += a b
    x.x = fmaf(a.x, b.x, x.x);
    x.x = fmaf(-a.y, b.y, x.x);
    x.y = fmaf(a.x, b.y, x.y);
    x.y = fmaf(a.y, b.x, x.y);
}

// LU by 16-column panels: the 16 x 16 diagonal block by one warp in registers (lane = row, the pivot
// row published through shared memory, no CTA barrier per pivot), then L21 = A21 U11^-1 (a lane per
// row) and U12 = L11^-1 A12 (a lane per column) by independent substitutions, then A22 -= L21 U12 by
// all warps in register tiles.  Inverses: the eight 16 x 16 diagonal blocks inverted in registers and
// put in place, then the off-diagonal blocks by the block recursion inv([[A, 0], [C, B]]) =
// [[A^-1, 0], [-B^-1 C A^-1, B^-1]] (16 -> 32 -> 64 -> 128; for U the transposed pattern), each level
// two products of block-triangular operands through a shared scratch.  (Fully unrolled code run by a
// single warp, and per-pivot shuffles, were measured slower than these short register recursions.)
constexpr int DF3_TLD = 2 * DF_BLK + 1, DF3_P = 16;  // DF3_P: LU panel width
constexpr int DF3_TSZ = DF_NB * DF_BLK * DF_SLD;  // the scratch: 4 blocks of 32 x DF_SLD (>= 64 x DF3_TLD)
static_assert(DF3_TSZ >= 2 * DF_BLK * DF3_TLD, "scratch holds the 64 x 64 product");
constexpr size_t df_smem_bytes() { return (size_t)(NBL * DF_LD + DF3_TSZ + NBL) * sizeof(float2); }

__device__ __forceinline__ float2 crecip(float2 d) {  // 1 / d by one reciprocal of |d|^2
    const float r = __frcp_rn(d.x * d.x + d.y * d.y);
    return make_float2(d.x * r, -d.y * r);
}

// A22 -= L21 U12 over rows and columns b0 .. NBL - 1 (n2 = NBL - b0 = 16 TR = 32 TC), k over the panel
// c0 .. c0 + 31: warp w the rows b0 + 16 a + w, lane the columns b0 + 32 b + lane.
template <int TR, int TC>
__device__ __forceinline__ void df3_trailing(float2* blk, int c0, int b0) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2 acc[TR][TC];
#pragma unroll
    for (int a = 0; a < TR; a++)
#pragma unroll
        for (int b = 0; b < TC; b++) acc[a][b] = make_float2(0.f, 0.f);
#pragma unroll 4
    for (int k = 0; k < DF3_P; k++) {
        float2 l[TR], u[TC];
#pragma unroll
        for (int a = 0; a < TR; a++) l[a] = blk[(b0 + 16 * a + warp) * DF_LD + c0 + k];
#pragma unroll
        for (int b = 0; b < TC; b++) u[b] = blk[(c0 + k) * DF_LD + min(b0 + 32 * b + lane, NBL - 1)];
#pragma unroll
        for (int a = 0; a < TR; a++)
#pragma unroll
            for (int b = 0; b < TC; b++) cfma_add(acc[a][b], l[a], u[b]);
    }
#pragma unroll
    for (int a = 0; a < TR; a++)
#pragma unroll
        for (int b = 0; b < TC; b++)
            if (b0 + 32 * b + lane < NBL) {
                float2& x = blk[(b0 + 16 * a + warp) * DF_LD + b0 + 32 * b + lane];
                x = make_float2(x.x - acc[a][b].x, x.y - acc[a][b].y);
            }
}

// Step J of a 16 x 16 LU by lanes 0..15 of a warp (lane = row, a = the lane's row; lanes 16..31 hold
// zeros): the pivot row published through shared memory (row, 16 entries), rcp[J] = 1 / U(J, J), ok
// false on a pivot of modulus below 1e-15.  Recursion keeps every register index constant; no
// branch around the updates (lanes at or above the pivot subtract zero).
template <int J>
__device__ __forceinline__ void df3_lu16_step(float2 (&a)[DF3_P], int lane, float2* row, float2* rcp, bool& ok) {
    if constexpr (J < DF3_P) {
        if (lane == J)
#pragma unroll
            for (int k = J; k < DF3_P; k++) row[k] = a[k];
        __syncwarp();
        const float2 d = row[J];
        ok = ok && d.x * d.x + d.y * d.y > 1e-30f;
        const float2 inv = crecip(d);
        if (lane == 0) rcp[J] = inv;
        const float2 l = cmulf(a[J], inv);
        const float2 lm = lane > J ? l : make_float2(0.f, 0.f);
#pragma unroll
        for (int k = J + 1; k < DF3_P; k++) cfma_sub(a[k], lm, row[k]);
        if (lane > J) a[J] = l;
        __syncwarp();
        df3_lu16_step<J + 1>(a, lane, row, rcp, ok);
    }
}

// x = x U^-1 for the upper 16 x 16 block at Ub (leading dimension DF_LD; rcp[k] = 1 / U(k, k)): step K
// finishes x[K] and removes it from the later unknowns.
template <int K>
__device__ __forceinline__ void df3_urow16_step(float2 (&x)[DF3_P], const float2* Ub, const float2* rcp) {
    if constexpr (K < DF3_P) {
        x[K] = cmulf(x[K], rcp[K]);
#pragma unroll
        for (int j = K + 1; j < DF3_P; j++) cfma_sub(x[j], x[K], Ub[K * DF_LD + j]);
        df3_urow16_step<K + 1>(x, Ub, rcp);
    }
}

// x = x L^-1 for the unit lower 16 x 16 block at Lb, from the last column: step K (x[K] final) removes
// x[K] from the earlier unknowns.
template <int K>
__device__ __forceinline__ void df3_lrow16_back_step(float2 (&x)[DF3_P], const float2* Lb) {
    if constexpr (K > 0) {
#pragma unroll
        for (int j = 0; j < K; j++) cfma_sub(x[j], x[K], Lb[K * DF_LD + j]);
        df3_lrow16_back_step<K - 1>(x, Lb);
    }
}

// y = L^-1 y for the unit lower 16 x 16 block at Lb, step K removing y[K] from the later unknowns.
template <int K>
__device__ __forceinline__ void df3_lcol16_step(float2 (&y)[DF3_P], const float2* Lb) {
    if constexpr (K < DF3_P - 1) {
#pragma unroll
        for (int j = K + 1; j < DF3_P; j++) cfma_sub(y[j], Lb[j * DF_LD + K], y[K]);
        df3_lcol16_step<K + 1>(y, Lb);
    }
}

// Block-triangular operand patterns of df3_product (block = 32 x 32): which k of the sum are nonzero
// for the output tile in block row ib, block column jb of C.
enum Df3Tri { DF3_B_LOWER, DF3_A_LOWER, DF3_B_UPPER, DF3_A_UPPER };

// C(m x m) = sgn A(m x m) B(m x m), m = 32 or 64, A and B of leading dimensions lda, ldb, C of ldc;
// threads tid0 .. tid0 + nthr - 1, each a 2 x 2 tile: rows 2 ri + {0, 1}, columns cj + {0, 16} of a
// 32 x 32 output block (consecutive lanes read consecutive columns of B).
__device__ __forceinline__ void df3_product(const float2* A, int lda, const float2* B, int ldb, float2* C, int ldc,
                                            int m, Df3Tri tri, float sgn, int tid, int nthr) {
    const int nbk = m / DF_BLK, tiles = nbk * nbk * 256;
    for (int t = tid; t < tiles; t += nthr) {
        const int blkid = t / 256, w = t % 256, ib = blkid / nbk, jb = blkid % nbk;
        const int i0 = ib * DF_BLK + 2 * (w / 16), j0 = jb * DF_BLK + (w % 16);
        int klo = 0, khi = m;
        if (tri == DF3_B_LOWER) klo = jb * DF_BLK;
        if (tri == DF3_A_LOWER) khi = (ib + 1) * DF_BLK;
        if (tri == DF3_B_UPPER) khi = (jb + 1) * DF_BLK;
        if (tri == DF3_A_UPPER) klo = ib * DF_BLK;
        float2 c00 = make_float2(0.f, 0.f), c01 = c00, c10 = c00, c11 = c00;
#pragma unroll 4
        for (int k = klo; k < khi; k++) {
            const float2 a0 = A[i0 * lda + k], a1 = A[(i0 + 1) * lda + k];
            const float2 b0 = B[k * ldb + j0], b1 = B[k * ldb + j0 + 16];
            cfma_add(c00, a0, b0);
            cfma_add(c01, a0, b1);
            cfma_add(c10, a1, b0);
            cfma_add(c11, a1, b1);
        }
        C[i0 * ldc + j0] = make_float2(sgn * c00.x, sgn * c00.y);
        C[i0 * ldc + j0 + 16] = make_float2(sgn * c01.x, sgn * c01.y);
        C[(i0 + 1) * ldc + j0] = make_float2(sgn * c10.x, sgn * c10.y);
        C[(i0 + 1) * ldc + j0 + 16] = make_float2(sgn * c11.x, sgn * c11.y);
    }
}

__global__ void __launch_bounds__(DF_THREADS) k_diag_factor(float* __restrict__ W, int Np, size_t bstride, int k0,
                                                              float* __restrict__ PL, float* __restrict__ PU,
                                                              float2* __restrict__ DINV, int* __restrict__ err) {
    extern __shared__ float2 df_smem[];
    float2* blk = df_smem;                   // [NBL][DF_LD]: the block, then its factors, then the inverse
    float2* T = blk + NBL * DF_LD;  // scratch: the diagonal-block inverses, then the products of the recursion
    float2* rcp = T + DF3_TSZ;      // [NBL]: 1 / U(j, j)
    const int f = blockIdx.x >> 1, side = blockIdx.x & 1;
    const bool upper = side == 1;
    float* Wr = W + (size_t)f * bstride;
    float* Wi = Wr + (size_t)Np * Np;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the block in 16-byte loads (rows of 128 entries, k0 and Np multiples of 128), 16 in flight a thread
#pragma unroll 8
    for (int t = threadIdx.x; t < NBL * NBL / 4; t += DF_THREADS) {
        const int r = t / (NBL / 4), c = 4 * (t % (NBL / 4));
        const size_t o = (size_t)(k0 + r) * Np + k0 + c;
        const float4 re = *reinterpret_cast<const float4*>(Wr + o), im = *reinterpret_cast<const float4*>(Wi + o);
        float2* d = blk + r * DF_LD + c;
        d[0] = make_float2(re.x, im.x);
        d[1] = make_float2(re.y, im.y);
        d[2] = make_float2(re.z, im.z);
        d[3] = make_float2(re.w, im.w);
    }
    __syncthreads();
#pragma unroll 1
    for (int pb = 0; pb < NBL / DF3_P; pb++) {
        const int c0 = pb * DF3_P, b0 = c0 + DF3_P, n2 = NBL - b0;
        if (warp == 0) {  // the 16 x 16 diagonal block: lane = row (lanes 16..31 carry zeros, write nothing)
            float2* P = blk + c0 * DF_LD + c0;
            float2 a[DF3_P];
#pragma unroll
            for (int k = 0; k < DF3_P; k++) a[k] = lane < DF3_P ? P[lane * DF_LD + k] : make_float2(0.f, 0.f);
            bool ok = true;
            df3_lu16_step<0>(a, lane, T, rcp + c0, ok);
            if (lane == 0 && !ok) atomicExch(err, 10);
            if (lane < DF3_P)
#pragma unroll
                for (int k = 0; k < DF3_P; k++) P[lane * DF_LD + k] = a[k];
        }
        __syncthreads();
        if (n2 == 0) break;
        const int nw = (n2 + 31) / 32;  // warps of each substitution
        if (warp >= 1 && warp <= nw) {  // L21 = A21 U11^-1: lane = row
            const int i = b0 + 32 * (warp - 1) + lane;
            if (i < NBL) {
                float2 x[DF3_P];
#pragma unroll
                for (int k = 0; k < DF3_P; k++) x[k] = blk[i * DF_LD + c0 + k];
                df3_urow16_step<0>(x, blk + c0 * DF_LD + c0, rcp + c0);
#pragma unroll
                for (int k = 0; k < DF3_P; k++) blk[i * DF_LD + c0 + k] = x[k];
            }
        } else if (warp >= 5 && warp < 5 + nw) {  // U12 = L11^-1 A12: lane = column
            const int cc = b0 + 32 * (warp - 5) + lane;
            if (cc < NBL) {
                float2 y[DF3_P];
#pragma unroll
                for (int k = 0; k < DF3_P; k++) y[k] = blk[(c0 + k) * DF_LD + cc];
                df3_lcol16_step<0>(y, blk + c0 * DF_LD + c0);
#pragma unroll
                for (int k = 0; k < DF3_P; k++) blk[(c0 + k) * DF_LD + cc] = y[k];
            }
        }
        __syncthreads();
        switch (n2 / DF3_P) {  // A22 -= L21 U12 (k over the 16 panel columns)
            case 7: df3_trailing<7, 4>(blk, c0, b0); break;
            case 6: df3_trailing<6, 3>(blk, c0, b0); break;
            case 5: df3_trailing<5, 3>(blk, c0, b0); break;
            case 4: df3_trailing<4, 2>(blk, c0, b0); break;
            case 3: df3_trailing<3, 2>(blk, c0, b0); break;
            case 2: df3_trailing<2, 1>(blk, c0, b0); break;
            default: df3_trailing<1, 1>(blk, c0, b0); break;
        }
        __syncthreads();
    }
    // ---- the factors back to W (side 0)
    if (side == 0)
#pragma unroll 8
        for (int t = threadIdx.x; t < NBL * NBL / 4; t += DF_THREADS) {
            const int r = t / (NBL / 4), c = 4 * (t % (NBL / 4));
            const size_t o = (size_t)(k0 + r) * Np + k0 + c;
            const float2* d = blk + r * DF_LD + c;
            *reinterpret_cast<float4*>(Wr + o) = make_float4(d[0].x, d[1].x, d[2].x, d[3].x);
            *reinterpret_cast<float4*>(Wi + o) = make_float4(d[0].y, d[1].y, d[2].y, d[3].y);
        }
    __syncthreads();
    // ---- the inverse of this side's factor, in place in blk
    // the eight 16 x 16 diagonal blocks (warp w: block w, lane = row of its inverse, in registers)
    constexpr int P = DF3_P, PL16 = DF3_P + 1;
    if (warp < NBL / P) {
        const float2* Ab = blk + warp * P * DF_LD + warp * P;
        float2 x[P];
#pragma unroll
        for (int k = 0; k < P; k++) x[k] = make_float2(k == lane ? 1.f : 0.f, 0.f);
        if (!upper)
            df3_lrow16_back_step<P - 1>(x, Ab);
        else
            df3_urow16_step<0>(x, Ab, rcp + warp * P);
        if (lane < P)
#pragma unroll
            for (int k = 0; k < P; k++) T[(warp * P + lane) * PL16 + k] = x[k];
    }
    __syncthreads();
    // ... into place, with zeros in the other triangle's 16-block of each 32 x 32 diagonal block
    for (int t = threadIdx.x; t < NBL * P; t += DF_THREADS) {
        const int w = t / (P * P), i = (t / P) % P, k = t % P;
        blk[(w * P + i) * DF_LD + w * P + k] = T[(w * P + i) * PL16 + k];
        const int z = w ^ 1;  // the partner block of the 32-block
        if ((z > w) == !upper) blk[(w * P + i) * DF_LD + z * P + k] = make_float2(0.f, 0.f);
    }
    __syncthreads();
    // 32-level: the four pairs at once (128 threads each); lower X(I, J) = -X(I, I) L(I, J) X(J, J) for
    // (I, J) = (2q + 1, 2q), upper Y(I, J) = -Y(I, I) U(I, J) Y(J, J) for (2q, 2q + 1) (16-blocks)
    {
        const int q = threadIdx.x / 128, tq = threadIdx.x % 128;
        const int I = (upper ? 2 * q : 2 * q + 1) * P, J = (upper ? 2 * q + 1 : 2 * q) * P;
        float2* Tq = T + q * P * PL16;
        // T = L(I, J) X(J, J), then X(I, J) = -X(I, I) T: two 16 x 16 outputs a thread
#pragma unroll
        for (int pass = 0; pass < 2; pass++) {
            const float2* A = pass == 0 ? blk + I * DF_LD + J : blk + I * DF_LD + I;
            const int lda = DF_LD;
            const float2* B = pass == 0 ? blk + J * DF_LD + J : Tq;
            const int ldb = pass == 0 ? DF_LD : PL16;
            const int r = tq / 8, c0 = (tq % 8) * 2;  // rows 0..15, column pairs
            float2 c00 = make_float2(0.f, 0.f), c01 = c00;
#pragma unroll 4
            for (int k = 0; k < P; k++) {
                const float2 a = A[r * lda + k];
                cfma_add(c00, a, B[k * ldb + c0]);
                cfma_add(c01, a, B[k * ldb + c0 + 1]);
            }
            __syncthreads();  // (pass 0) every thread's reads of L(I, J) done; (pass 1) of T
            if (pass == 0) {
                Tq[r * PL16 + c0] = c00;
                Tq[r * PL16 + c0 + 1] = c01;
            } else {
                blk[(I + r) * DF_LD + J + c0] = make_float2(-c00.x, -c00.y);
                blk[(I + r) * DF_LD + J + c0 + 1] = make_float2(-c01.x, -c01.y);
            }
            __syncthreads();
        }
    }
    // 64-level: the two pairs of 32-blocks at once (256 threads each); lower: X(I, J) = -X(I, I) L(I, J)
    // X(J, J) for (I, J) = (1, 0), (3, 2); upper: Y(I, J) = -Y(I, I) U(I, J) Y(J, J) for (0, 1), (2, 3)
    {
        const int q = threadIdx.x / 256, tq = threadIdx.x % 256;
        const int d0 = 2 * q * DF_BLK, d1 = d0 + DF_BLK;  // the pair's two diagonal blocks
        const int I = upper ? d0 : d1, J = upper ? d1 : d0;
        float2* Tq = T + q * DF_BLK * DF3_TLD;  // [32][DF3_TLD] rows of the pair's scratch
        df3_product(blk + I * DF_LD + J, DF_LD, blk + J * DF_LD + J, DF_LD, Tq, DF3_TLD, DF_BLK,
                    upper ? DF3_B_UPPER : DF3_B_LOWER, 1.f, tq, 256);
        __syncthreads();
        df3_product(blk + I * DF_LD + I, DF_LD, Tq, DF3_TLD, blk + I * DF_LD + J, DF_LD, DF_BLK,
                    upper ? DF3_A_UPPER : DF3_A_LOWER, -1.f, tq, 256);
    }
    __syncthreads();
    // 128-level: lower X21 = -X22 (L21 X11), upper Y12 = -Y11 (U12 Y22), 64 x 64 blocks
    {
        const int h = 2 * DF_BLK;
        const int I = upper ? 0 : h, J = upper ? h : 0;
        df3_product(blk + I * DF_LD + J, DF_LD, blk + J * DF_LD + J, DF_LD, T, DF3_TLD, h,
                    upper ? DF3_B_UPPER : DF3_B_LOWER, 1.f, threadIdx.x, DF_THREADS);
        __syncthreads();
        df3_product(blk + I * DF_LD + I, DF_LD, T, DF3_TLD, blk + I * DF_LD + J, DF_LD, h,
                    upper ? DF3_A_UPPER : DF3_A_LOWER, -1.f, threadIdx.x, DF_THREADS);
    }
    __syncthreads();
    // ---- outputs: this side's triangle of the inverse
    {
        float2* D = DINV + ((size_t)f * (Np / NBL) + k0 / NBL) * NBL * NBL;
        for (int t = threadIdx.x; t < NBL * NBL; t += DF_THREADS) {
            const int i = t / NBL, c = t % NBL;
            if ((i > c) == !upper) D[t] = blk[i * DF_LD + c];
        }
    }
    if (!upper) {
        float* PLf = PL + (size_t)f * NBL * 2 * NBL;
        for (int t = threadIdx.x; t < NBL * NBL; t += DF_THREADS) {  // [Lr | Li] rows of L^-1 (c fastest)
            const int i = t / NBL, c = t % NBL;
            const float2 l = i > c ? blk[i * DF_LD + c] : make_float2(i == c ? 1.f : 0.f, 0.f);
            PLf[(size_t)i * 2 * NBL + c] = l.x;
            PLf[(size_t)i * 2 * NBL + NBL + c] = l.y;
        }
    } else {
        float* PUf = PU + (size_t)f * 2 * NBL * 2 * NBL;
        for (int t = threadIdx.x; t < NBL * NBL; t += DF_THREADS) {
            // U^-1 block-real K-major (i fastest): row c: [Ur(:, c); -Ui(:, c)], row NBL + c: [Ui(:, c); Ur(:, c)]
            const int c = t / NBL, i = t % NBL;
            const float2 u = i <= c ? blk[i * DF_LD + c] : make_float2(0.f, 0.f);
            PUf[(size_t)c * 2 * NBL + i] = u.x;
            PUf[(size_t)c * 2 * NBL + NBL + i] = -u.y;
            PUf[(size_t)(NBL + c) * 2 * NBL + i] = u.y;
            PUf[(size_t)(NBL + c) * 2 * NBL + NBL + i] = u.x;
        }
    }
}

// The block row B = rows k0..k0+NBL, columns c0..c0+n in the block-real K-major form
// [F][2n][2 NBL]: row j: [Br(:, j); -Bi(:, j)], row n + j: [Bi(:, j); Br(:, j)] (32 x 32 tiles
// transposed through shared memory).
__global__ void k_prep_block_row(const float* __restrict__ W, int Np, size_t bstride, int k0, int c0, int n,
                                 float* __restrict__ P2, size_t p2_bstride) {
    __shared__ float tr[32][33], ti[32][33];
    const int f = blockIdx.z;
    const int j0 = blockIdx.x * 32, kk0 = blockIdx.y * 32;
    const float* Wr = W + (size_t)f * bstride;
    const float* Wi = Wr + (size_t)Np * Np;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += blockDim.y) {
        size_t o = (size_t)(k0 + kk0 + r) * Np + c0 + j0 + tx;
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
            if (lim == CH) {
                // a full chunk: the matrix entries of 8 columns loaded ahead of their products
#pragma unroll
                for (int q = 0; q < CH; q += 8) {
                    float mr[8], mi[8];
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const size_t o = (size_t)(n0 + q + j) * Np + k;
                        mr[j] = Mr[o];
                        mi[j] = Mi[o];
                    }
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const double dr = mr[j], di = mi[j];
#pragma unroll
                        for (int c = 0; c < NR; c++) {
                            const double2 v = sx[q + j][c];
                            acc[c].x += dr * v.x - di * v.y;
                            acc[c].y += dr * v.y + di * v.x;
                        }
                    }
                }
            } else {
                for (int nn = 0; nn < lim; nn++) {
                    const size_t o = (size_t)(n0 + nn) * Np + k;
                    const double mr = Mr[o], mi = Mi[o];
#pragma unroll
                    for (int c = 0; c < NR; c++) {
                        const double2 v = sx[nn][c];
                        acc[c].x += mr * v.x - mi * v.y;
                        acc[c].y += mr * v.y + mi * v.x;
                    }
                }
            }
        }
    }
    if (k < N)
#pragma unroll
        for (int c = 0; c < NR; c++)
            if (c < nrhs) part[(((size_t)z * F + f) * nrhs + c) * N + k] = acc[c];
}

// The same partial products with the matrix and vector tiles streamed by TMA: CTA of 256 rows k
// (two a thread: t and t + 128, so each vector entry read from shared memory feeds both) over a
// chunk of columns n, 16 columns per stage (both FP32 planes, 32 KB, and the 16 complex entries of
// every right-hand side), GV_STAGES stages in flight from a producer warp, so the bytes in flight do
// not depend on registers; FP64 accumulation as above.
// Packed FP32 pairs (fma.rn.f32x2: two FP32 FMAs per instruction).  A complex multiply-add
// acc += m v is two packed FMAs: acc += (m.re, m.re) (v.re, v.im), then acc += (-m.im, m.im) (v.im, v.re);
// the right-hand sides are kept in shared memory as {re, im, im, re} so one 16-byte load gives both
// orders.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2pack(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 f2unpack(f32x2 r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ f32x2 ffma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ float4 dup_swap(float2 v) { return make_float4(v.x, v.y, v.y, v.x); }

constexpr int GV_ROWS = 256, GV_COLS = 16, GV_STAGES = 3, GV_CHUNK = 1024;
constexpr int GV_WORKERS = GV_ROWS / 2;
constexpr int GV_THREADS = GV_WORKERS + 32;
template <int NR>
__host__ __device__ constexpr size_t gv_tx_bytes() {  // bytes one stage receives
    return (size_t)2 * GV_COLS * GV_ROWS * 4 + (size_t)NR * GV_COLS * 16;
}
template <int NR>
__host__ __device__ constexpr size_t gv_stage_bytes() {  // stage stride in shared memory (1024-byte aligned)
    return (gv_tx_bytes<NR>() + 1023) / 1024 * 1024;
}
template <int NR>
__host__ __device__ constexpr size_t gv_smem_bytes() {
    return 1024 + GV_STAGES * gv_stage_bytes<NR>() + 128;
}

template <int NR>
__global__ void __launch_bounds__(GV_THREADS) k_cgemv_tma(const __grid_constant__ CUtensorMap mapM,
                                                             const __grid_constant__ CUtensorMap mapX, int N,
                                                             int nrhs, int c0, double2* __restrict__ part, int F,
                                                             int* __restrict__ err) {
    extern __shared__ uint8_t gv_raw[];
    uint8_t* base = align1024(gv_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(base + GV_STAGES * gv_stage_bytes<NR>());
    uint64_t* empty = full + GV_STAGES;
    const int f = blockIdx.y, z = blockIdx.z;
    const int k0 = blockIdx.x * GV_ROWS;
    const int nbeg = z * GV_CHUNK, nend = min(N, nbeg + GV_CHUNK);
    const int nst = (nend - nbeg + GV_COLS - 1) / GV_COLS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < GV_STAGES; s++) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], GV_WORKERS / 32);
        }
        tc::fence_barrier_init();
    }
    __syncthreads();
    if (warp == GV_WORKERS / 32) {
        if (lane == 0) {
            tc::prefetch_tensormap(&mapM);
            tc::prefetch_tensormap(&mapX);
            for (int si = 0; si < nst; si++) {
                const int s = si % GV_STAGES;
                if (si >= GV_STAGES && !tc::mbar_wait(&empty[s], ((si / GV_STAGES) - 1) & 1)) {
                    atomicExch(err, 6);
                    break;
                }
                uint8_t* st = base + s * gv_stage_bytes<NR>();
                const int n0 = nbeg + si * GV_COLS;
                tc::mbar_arrive_expect_tx(&full[s], (uint32_t)gv_tx_bytes<NR>());
                tc::tma_load_4d(st, &mapM, &full[s], k0, n0, 0, f);
                tc::tma_load_4d(st + GV_COLS * GV_ROWS * 4, &mapM, &full[s], k0, n0, 1, f);
                tc::tma_load_4d(st + 2 * GV_COLS * GV_ROWS * 4, &mapX, &full[s], 2 * n0, c0, f, 0);
            }
        }
        return;
    }
    double2 acc[NR], acd[NR];  // rows k0 + t and k0 + t + GV_WORKERS
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = acd[c] = make_double2(0.0, 0.0);
    const int t = threadIdx.x;
    for (int si = 0; si < nst; si++) {
        const int s = si % GV_STAGES;
        if (!tc::mbar_wait(&full[s], (si / GV_STAGES) & 1)) {
            atomicExch(err, 7);
            break;
        }
        const uint8_t* st = base + s * gv_stage_bytes<NR>();
        const float* sMr = reinterpret_cast<const float*>(st);
        const float* sMi = sMr + GV_COLS * GV_ROWS;
        const double2* sx = reinterpret_cast<const double2*>(st + 2 * GV_COLS * GV_ROWS * 4);  // [NR][GV_COLS]
        // columns beyond N are never read (the padding may hold anything)
        const int lim = min(GV_COLS, nend - (nbeg + si * GV_COLS));
#pragma unroll 2
        for (int j = 0; j < lim; j++) {
            const double mr = sMr[j * GV_ROWS + t], mi = sMi[j * GV_ROWS + t];
            const double nr = sMr[j * GV_ROWS + t + GV_WORKERS], ni = sMi[j * GV_ROWS + t + GV_WORKERS];
#pragma unroll
            for (int c = 0; c < NR; c++) {  // four fused multiply-adds a row (the pipe's limit)
                const double2 v = sx[c * GV_COLS + j];
                acc[c].x = fma(-mi, v.y, fma(mr, v.x, acc[c].x));
                acc[c].y = fma(mi, v.x, fma(mr, v.y, acc[c].y));
                acd[c].x = fma(-ni, v.y, fma(nr, v.x, acd[c].x));
                acd[c].y = fma(ni, v.x, fma(nr, v.y, acd[c].y));
            }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[s]);
    }
    const int k = k0 + t, kd = k + GV_WORKERS;
#pragma unroll
    for (int c = 0; c < NR; c++)
        if (c0 + c < nrhs) {
            if (k < N) part[(((size_t)z * F + f) * nrhs + c0 + c) * N + k] = acc[c];
            if (kd < N) part[(((size_t)z * F + f) * nrhs + c0 + c) * N + kd] = acd[c];
        }
}

// The same product with a complex64 vector d (a refinement correction): part = M d over column chunks,
// each product and each 16-column sum in FP32, the sums added into FP64.  For a correction d that is
// small against the solution (|d| ~ 1e-3 |x| after the first), FP32 products put errors of ~1e-10 of
// |A x| into the residual r - M d, far below what the refinement converges to.
template <int NR>
__host__ __device__ constexpr size_t gv32_tx_bytes() {
    return (size_t)2 * GV_COLS * GV_ROWS * 4 + (size_t)NR * GV_COLS * 8;
}
template <int NR>
__host__ __device__ constexpr size_t gv32_stage_bytes() {
    return (gv32_tx_bytes<NR>() + 1023) / 1024 * 1024;
}
template <int NR>
__host__ __device__ constexpr size_t gv32_smem_bytes() {
    return 1024 + GV_STAGES * gv32_stage_bytes<NR>() + 128;
}

template <int NR>
__global__ void __launch_bounds__(GV_THREADS) k_cgemv32_tma(const __grid_constant__ CUtensorMap mapM,
                                                               const __grid_constant__ CUtensorMap mapD, int N,
                                                               int nrhs, int c0, double2* __restrict__ part, int F,
                                                               int* __restrict__ err) {
    extern __shared__ uint8_t gv_raw[];
    uint8_t* base = align1024(gv_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(base + GV_STAGES * gv32_stage_bytes<NR>());
    uint64_t* empty = full + GV_STAGES;
    const int f = blockIdx.y, z = blockIdx.z;
    const int k0 = blockIdx.x * GV_ROWS;
    const int nbeg = z * GV_CHUNK, nend = min(N, nbeg + GV_CHUNK);
    const int nst = (nend - nbeg + GV_COLS - 1) / GV_COLS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < GV_STAGES; s++) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], GV_WORKERS / 32);
        }
        tc::fence_barrier_init();
    }
    __syncthreads();
    if (warp == GV_WORKERS / 32) {
        if (lane == 0) {
            tc::prefetch_tensormap(&mapM);
            tc::prefetch_tensormap(&mapD);
            for (int si = 0; si < nst; si++) {
                const int s = si % GV_STAGES;
                if (si >= GV_STAGES && !tc::mbar_wait(&empty[s], ((si / GV_STAGES) - 1) & 1)) {
                    atomicExch(err, 6);
                    break;
                }
                uint8_t* st = base + s * gv32_stage_bytes<NR>();
                const int n0 = nbeg + si * GV_COLS;
                tc::mbar_arrive_expect_tx(&full[s], (uint32_t)gv32_tx_bytes<NR>());
                tc::tma_load_4d(st, &mapM, &full[s], k0, n0, 0, f);
                tc::tma_load_4d(st + GV_COLS * GV_ROWS * 4, &mapM, &full[s], k0, n0, 1, f);
                tc::tma_load_4d(st + 2 * GV_COLS * GV_ROWS * 4, &mapD, &full[s], 2 * n0, c0, f, 0);
            }
        }
        return;
    }
    double2 acc[NR], acd[NR];  // rows k0 + t and k0 + t + GV_WORKERS
#pragma unroll
    for (int c = 0; c < NR; c++) acc[c] = acd[c] = make_double2(0.0, 0.0);
    const int t = threadIdx.x;
    for (int si = 0; si < nst; si++) {
        const int s = si % GV_STAGES;
        if (!tc::mbar_wait(&full[s], (si / GV_STAGES) & 1)) {
            atomicExch(err, 7);
            break;
        }
        const uint8_t* st = base + s * gv32_stage_bytes<NR>();
        const float* sMr = reinterpret_cast<const float*>(st);
        const float* sMi = sMr + GV_COLS * GV_ROWS;
        const float2* sd = reinterpret_cast<const float2*>(st + 2 * GV_COLS * GV_ROWS * 4);  // [NR][GV_COLS]
        const int lim = min(GV_COLS, nend - (nbeg + si * GV_COLS));
        f32x2 a0[NR], a1[NR];
#pragma unroll
        for (int c = 0; c < NR; c++) a0[c] = a1[c] = f2pack(0.f, 0.f);
#pragma unroll 4
        for (int j = 0; j < lim; j++) {
            const float mr = sMr[j * GV_ROWS + t], mi = sMi[j * GV_ROWS + t];
            const float nr = sMr[j * GV_ROWS + t + GV_WORKERS], ni = sMi[j * GV_ROWS + t + GV_WORKERS];
            const f32x2 m0 = f2pack(mr, mr), q0 = f2pack(-mi, mi), m1 = f2pack(nr, nr), q1 = f2pack(-ni, ni);
#pragma unroll
            for (int c = 0; c < NR; c++) {
                const float2 v = sd[c * GV_COLS + j];
                const f32x2 vv = f2pack(v.x, v.y), vs = f2pack(v.y, v.x);
                a0[c] = ffma2(m0, vv, a0[c]);
                a0[c] = ffma2(q0, vs, a0[c]);
                a1[c] = ffma2(m1, vv, a1[c]);
                a1[c] = ffma2(q1, vs, a1[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < NR; c++) {
            const float2 u0 = f2unpack(a0[c]), u1 = f2unpack(a1[c]);
            acc[c].x += (double)u0.x;
            acc[c].y += (double)u0.y;
            acd[c].x += (double)u1.x;
            acd[c].y += (double)u1.y;
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[s]);
    }
    const int k = k0 + t, kd = k + GV_WORKERS;
#pragma unroll
    for (int c = 0; c < NR; c++)
        if (c0 + c < nrhs) {
            if (k < N) part[(((size_t)z * F + f) * nrhs + c0 + c) * N + k] = acc[c];
            if (kd < N) part[(((size_t)z * F + f) * nrhs + c0 + c) * N + kd] = acd[c];
        }
}

template <class T>
__device__ __forceinline__ T make_out(double x, double y);
template <>
__device__ __forceinline__ double2 make_out<double2>(double x, double y) {
    return make_double2(x, y);
}
template <>
__device__ __forceinline__ float2 make_out<float2>(double x, double y) {
    return make_float2((float)x, (float)y);
}

__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2((double)v.x, (double)v.y); }

template <class T, class BT = double2>
__global__ void k_gemv_reduce(int N, int nrhs, int F, int nz, const double2* __restrict__ part,
                              const BT* __restrict__ bias, int ldb, T* __restrict__ out, int ldo) {
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
    double2 b = bias ? to_d2(bias[((size_t)f * nrhs + c) * ldb + k]) : make_double2(0.0, 0.0);
    out[((size_t)f * nrhs + c) * ldo + k] = make_out<T>(b.x - sr, b.y - si);
}

// d = A^-1 r with the factors of M = A^T = L U (FP32 planar, row-major in W): U^T y = r, then
// L^T d = y, in FP32 (the correction only needs the accuracy of the TF32 factors; the residual that
// sets the attainable accuracy is formed in FP64), vectors [F][nrhs][Np] complex64 in place, in
// blocks of TB = 128 rows.  One launch per block step: every CTA of the step owns 128 rows and
// subtracts the contribution of the block solved by the previous step (row s0 + p of W read along
// its rows: coalesced); the CTA that owns the next diagonal block then solves it by the stored
// inverse of that block.
constexpr int TB = 128;
constexpr int TRI_THREADS = 256;


// The diagonal block of U^T (upper_t) or L^T, solved by its stored inverse: y_b = D^T r_b with
// D = U_bb^-1 (upper part of the stored block, with the diagonal) or L_bb^-1 (lower part, unit
// diagonal).  Rows b0..b0+TB of X in place, right-hand sides in chunks of NR.  Thread t < TB owns
// column t for the first half of the block's rows, thread t + TB the same column for the second
// half; each loads the 16 entries of a chunk before using them (one memory latency per chunk).
template <int NR>
__device__ __forceinline__ void tri_diag_f32(const float2* __restrict__ D, float2* X, int Np, int nrhs, int b0,
                                             bool upper_t, float4 (*rs)[NR], float2 (*pt)[NR]) {
    const int i = threadIdx.x % TB, half = threadIdx.x / TB;
    for (int c0 = 0; c0 < nrhs; c0 += NR) {
        const int nc = min(NR, nrhs - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < TB * NR; t += blockDim.x) {
            const int p = t % TB, c = t / TB;
            rs[p][c] = dup_swap(c < nc ? X[(size_t)(c0 + c) * Np + b0 + p] : make_float2(0.f, 0.f));
        }
        __syncthreads();
        f32x2 acc[NR];
#pragma unroll
        for (int c = 0; c < NR; c++)  // the unit diagonal of L^-1
            acc[c] = (!upper_t && half == (i >= TB / 2 ? 1 : 0)) ? f2pack(rs[i][c].x, rs[i][c].y) : f2pack(0.f, 0.f);
        const int pb = half * (TB / 2);
#pragma unroll 1
        for (int pc = 0; pc < TB / 2; pc += 16) {
            // the chunk's rows p = pb + pc .. + 15 that this row uses (p <= i for U^-1, p > i for L^-1):
            // none, and its loads are skipped (half of the triangle's inverse is zero)
            const int p0 = pb + pc;
            if (upper_t ? p0 > i : p0 + 15 <= i) continue;
            float2 dv[16];
#pragma unroll
            for (int q = 0; q < 16; q++) dv[q] = D[(pb + pc + q) * TB + i];
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int p = pb + pc + q;
                if (upper_t ? p <= i : p > i) {
                    const f32x2 m = f2pack(dv[q].x, dv[q].x), mn = f2pack(-dv[q].y, dv[q].y);
#pragma unroll
                    for (int c = 0; c < NR; c++) {
                        const float4 v = rs[p][c];
                        acc[c] = ffma2(m, f2pack(v.x, v.y), acc[c]);
                        acc[c] = ffma2(mn, f2pack(v.z, v.w), acc[c]);
                    }
                }
            }
        }
        if (half == 1)
#pragma unroll
            for (int c = 0; c < NR; c++) pt[i][c] = f2unpack(acc[c]);
        __syncthreads();
        if (half == 0)
#pragma unroll
            for (int c = 0; c < NR; c++)
                if (c < nc) {
                    const float2 q2 = pt[i][c], a = f2unpack(acc[c]);
                    X[(size_t)(c0 + c) * Np + b0 + i] = make_float2(a.x + q2.x, a.y + q2.y);
                }
    }
}

// One block step of the forward (upper_t) or backward solve.  step = index of the block solved by
// the previous launch (-1: none, only the first diagonal block is solved).  Thread layout: warp w
// owns rows 32 (w % 2) + lane and 64 more, and the quarter w / 2 of the solved block's 128
// entries, loaded 16 at a time before use; every lane of a warp reads the same solved entry (a
// shared-memory broadcast).
template <int NR>
__global__ void __launch_bounds__(TRI_THREADS, 2) k_tri_step(int Np, size_t bstride, const float* __restrict__ W,
                                                          const float2* __restrict__ DINV, int nrhs,
                                                          float2* __restrict__ Xall, int step, int upper_t) {
    extern __shared__ float4 tri_smem4[];  // ys [TB][NR] as {re, im, im, re}, partial sums [3][TB][NR]
    float4(*ys)[NR] = reinterpret_cast<float4(*)[NR]>(tri_smem4);
    float2(*pt)[NR] = reinterpret_cast<float2(*)[NR]>(tri_smem4 + TB * NR);
    const int f = blockIdx.y;
    const float* Mr = W + (size_t)f * bstride;
    const float* Mi = Mr + (size_t)Np * Np;
    float2* X = Xall + (size_t)f * nrhs * Np;
    const int nblk = Np / TB;
    const float2* Df = DINV + (size_t)f * nblk * TB * TB;
    if (step < 0) {
        const int first = upper_t ? 0 : nblk - 1;
        tri_diag_f32<NR>(Df + (size_t)first * TB * TB, X, Np, nrhs, first * TB, upper_t, ys, pt);
        return;
    }
    const int s0 = step * TB;
    const int cb = upper_t ? step + 1 + blockIdx.x : step - 1 - blockIdx.x;
    const int r0 = cb * TB;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int li = 32 * (warp & 1) + lane;  // local rows li and li + 64
    const int pq = warp >> 1;               // quarter of the solved block
    const float* pr = Mr + (size_t)(s0 + pq * 32) * Np + r0 + li;
    const float* pi = Mi + (size_t)(s0 + pq * 32) * Np + r0 + li;
    for (int c0 = 0; c0 < nrhs; c0 += NR) {
        const int nc = min(NR, nrhs - c0);
        __syncthreads();
        for (int t = threadIdx.x; t < TB * NR; t += blockDim.x) {
            const int p = t % TB, c = t / TB;
            ys[p][c] = dup_swap(c < nc ? X[(size_t)(c0 + c) * Np + s0 + p] : make_float2(0.f, 0.f));
        }
        __syncthreads();
        f32x2 a0[NR], a1[NR];
#pragma unroll
        for (int c = 0; c < NR; c++) a0[c] = a1[c] = f2pack(0.f, 0.f);
#pragma unroll 1
        for (int pc = 0; pc < 32; pc += 16) {
            float r0v[16], i0v[16], r1v[16], i1v[16];
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const size_t o = (size_t)(pc + q) * Np;
                r0v[q] = pr[o];
                i0v[q] = pi[o];
                r1v[q] = pr[o + 64];
                i1v[q] = pi[o + 64];
            }
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const f32x2 m0 = f2pack(r0v[q], r0v[q]), n0 = f2pack(-i0v[q], i0v[q]);
                const f32x2 m1 = f2pack(r1v[q], r1v[q]), n1 = f2pack(-i1v[q], i1v[q]);
#pragma unroll
                for (int c = 0; c < NR; c++) {
                    const float4 v4 = ys[pq * 32 + pc + q][c];
                    const f32x2 v = f2pack(v4.x, v4.y), vs = f2pack(v4.z, v4.w);
                    a0[c] = ffma2(m0, v, a0[c]);
                    a0[c] = ffma2(n0, vs, a0[c]);
                    a1[c] = ffma2(m1, v, a1[c]);
                    a1[c] = ffma2(n1, vs, a1[c]);
                }
            }
        }
        if (pq > 0)
#pragma unroll
            for (int c = 0; c < NR; c++) {
                pt[(pq - 1) * TB + li][c] = f2unpack(a0[c]);
                pt[(pq - 1) * TB + li + 64][c] = f2unpack(a1[c]);
            }
        __syncthreads();
        if (pq == 0)
#pragma unroll
            for (int c = 0; c < NR; c++)
                if (c < nc) {
                    float2 s0v = f2unpack(a0[c]), s1v = f2unpack(a1[c]);
#pragma unroll
                    for (int h = 0; h < 3; h++) {
                        const float2 q0 = pt[h * TB + li][c], q1 = pt[h * TB + li + 64][c];
                        s0v.x += q0.x;
                        s0v.y += q0.y;
                        s1v.x += q1.x;
                        s1v.y += q1.y;
                    }
                    float2* x0 = X + (size_t)(c0 + c) * Np + r0 + li;
                    const float2 v0 = x0[0], v1 = x0[64];
                    x0[0] = make_float2(v0.x - s0v.x, v0.y - s0v.y);
                    x0[64] = make_float2(v1.x - s1v.x, v1.y - s1v.y);
                }
    }
    if (blockIdx.x == 0) tri_diag_f32<NR>(Df + (size_t)cb * TB * TB, X, Np, nrhs, r0, upper_t, ys, pt);
}

constexpr size_t tri_smem_bytes(int nr) { return (size_t)TB * nr * (sizeof(float4) + 3 * sizeof(float2)); }

// The same solve as one persistent launch per direction (up to NR right-hand sides): the work items
// are (k, f), block k in solve order of matrix f, handed out by a ticket counter in the order
// k nb + f.  An item streams the block row of the factor against the blocks 0 .. k-1 as their
// solutions are published (ctrl[1 + f] = blocks of matrix f done), subtracts the sum, solves its
// diagonal block by the stored inverse and publishes it.  An item waits only on items of smaller
// ticket, which running CTAs hold, so the sweep cannot deadlock; every wait is bounded (error 8).
// ctrl = [ticket, done[nb]], zero at launch.
constexpr uint32_t TRI_WAIT_LIMIT = 1u << 20;

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <int NR>
__global__ void __launch_bounds__(TRI_THREADS, NR > 16 ? 1 : 2) k_tri_sweep(int Np, size_t bstride, const float* __restrict__ W,
                                                           const float2* __restrict__ DINV, int nrhs,
                                                           float2* __restrict__ Xall, int nb, int upper_t,
                                                           int* __restrict__ ctrl, int* __restrict__ err) {
    extern __shared__ float4 tri_smem4[];  // ys [TB][NR] as {re, im, im, re}, partial sums [3][TB][NR]
    float4(*ys)[NR] = reinterpret_cast<float4(*)[NR]>(tri_smem4);
    float2(*pt)[NR] = reinterpret_cast<float2(*)[NR]>(tri_smem4 + TB * NR);
    __shared__ int s_item, s_stop;
    const int nblk = Np / TB, items = nblk * nb;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int li = 32 * (warp & 1) + lane;  // local rows li and li + 64
    const int pq = warp >> 1;               // quarter of each solved block
    for (;;) {
        __syncthreads();  // the previous item's shared data consumed
        if (threadIdx.x == 0) s_item = atomicAdd(ctrl, 1);
        __syncthreads();
        const int t = s_item;
        if (t >= items) return;
        const int k = t / nb, f = t % nb;
        const int r0 = (upper_t ? k : nblk - 1 - k) * TB;
        const float* Mr = W + (size_t)f * bstride;
        const float* Mi = Mr + (size_t)Np * Np;
        float2* X = Xall + (size_t)f * nrhs * Np;
        int* done = ctrl + 1 + f;
        f32x2 a0[NR], a1[NR];
#pragma unroll
        for (int c = 0; c < NR; c++) a0[c] = a1[c] = f2pack(0.f, 0.f);
#pragma unroll 1
        for (int kk = 0; kk < k; kk++) {
            const int s0 = (upper_t ? kk : nblk - 1 - kk) * TB;
            if (threadIdx.x == 0) {
                int stop = 0;
                uint32_t n = 0;
                while (ld_acquire_gpu(done) <= kk) {
                    if (*(volatile int*)err != 0) {
                        stop = 1;
                        break;
                    }
                    if (++n > TRI_WAIT_LIMIT) {
                        atomicExch(err, 8);
                        stop = 1;
                        break;
                    }
                    __nanosleep(64);
                }
                s_stop = stop;
            }
            __syncthreads();
            if (s_stop) return;
            // the solved block (written by another CTA: read through L2)
            for (int tt = threadIdx.x; tt < TB * NR; tt += blockDim.x) {
                const int p = tt % TB, c = tt / TB;
                ys[p][c] = dup_swap(c < nrhs ? __ldcg(X + (size_t)c * Np + s0 + p) : make_float2(0.f, 0.f));
            }
            __syncthreads();
            const float* pr = Mr + (size_t)(s0 + pq * 32) * Np + r0 + li;
            const float* pi = Mi + (size_t)(s0 + pq * 32) * Np + r0 + li;
#pragma unroll 1
            for (int pc = 0; pc < 32; pc += 16) {
                float r0v[16], i0v[16], r1v[16], i1v[16];
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const size_t o = (size_t)(pc + q) * Np;
                    r0v[q] = __ldg(pr + o);
                    i0v[q] = __ldg(pi + o);
                    r1v[q] = __ldg(pr + o + 64);
                    i1v[q] = __ldg(pi + o + 64);
                }
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const f32x2 m0 = f2pack(r0v[q], r0v[q]), n0 = f2pack(-i0v[q], i0v[q]);
                    const f32x2 m1 = f2pack(r1v[q], r1v[q]), n1 = f2pack(-i1v[q], i1v[q]);
#pragma unroll
                    for (int c = 0; c < NR; c++) {
                        const float4 v4 = ys[pq * 32 + pc + q][c];
                        const f32x2 v = f2pack(v4.x, v4.y), vs = f2pack(v4.z, v4.w);
                        a0[c] = ffma2(m0, v, a0[c]);
                        a0[c] = ffma2(n0, vs, a0[c]);
                        a1[c] = ffma2(m1, v, a1[c]);
                        a1[c] = ffma2(n1, vs, a1[c]);
                    }
                }
            }
            __syncthreads();  // ys read by every warp before the next block overwrites it
        }
        if (k > 0) {
            if (pq > 0)
#pragma unroll
                for (int c = 0; c < NR; c++) {
                    pt[(pq - 1) * TB + li][c] = f2unpack(a0[c]);
                    pt[(pq - 1) * TB + li + 64][c] = f2unpack(a1[c]);
                }
            __syncthreads();
            if (pq == 0)
#pragma unroll
                for (int c = 0; c < NR; c++)
                    if (c < nrhs) {
                        float2 s0v = f2unpack(a0[c]), s1v = f2unpack(a1[c]);
#pragma unroll
                        for (int h = 0; h < 3; h++) {
                            const float2 q0 = pt[h * TB + li][c], q1 = pt[h * TB + li + 64][c];
                            s0v.x += q0.x;
                            s0v.y += q0.y;
                            s1v.x += q1.x;
                            s1v.y += q1.y;
                        }
                        float2* x0 = X + (size_t)c * Np + r0 + li;
                        const float2 v0 = x0[0], v1 = x0[64];
                        x0[0] = make_float2(v0.x - s0v.x, v0.y - s0v.y);
                        x0[64] = make_float2(v1.x - s1v.x, v1.y - s1v.y);
                    }
        }
        tri_diag_f32<NR>(DINV + ((size_t)f * nblk + r0 / TB) * TB * TB, X, Np, nrhs, r0, upper_t, ys, pt);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) st_release_gpu(done, k + 1);
    }
}

// FP64 vectors to complex64 (the right-hand sides entering the first correction).
__global__ void k_to_c64(size_t n, const double2* __restrict__ a, float2* __restrict__ b) {
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        b[t] = make_float2((float)a[t].x, (float)a[t].y);
}

// x += d; per matrix the largest |d| and |x| (for the refinement's stopping test), [F][2].
__global__ void k_ir_update(int Np, int nrhs, double2* __restrict__ x, const float2* __restrict__ d,
                            double* __restrict__ norms) {
    __shared__ double sd[256], sx[256];
    const int f = blockIdx.x;
    const size_t n = (size_t)nrhs * Np;
    double md = 0.0, mx = 0.0;
    for (size_t t = threadIdx.x; t < n; t += blockDim.x) {
        size_t o = (size_t)f * n + t;
        double2 a = x[o];
        const float2 b = d[o];
        a.x += (double)b.x;
        a.y += (double)b.y;
        x[o] = a;
        md = fmax(md, fmax(fabs((double)b.x), fabs((double)b.y)));
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
