// hbg_mixed.cu -- the mixed-precision form of the frequency solve: the pair kernels in FP64 as in
// the FP64 form, the matrices stored as complex64 (two FP32 planes), the LU on the tensor cores
// (tcgen05 kind::tf32, FP32 accumulation, no pivoting), the right-hand sides and the residuals
// accumulated in FP64, and iterative refinement until the correction is below 1e-12 of the solution.
// The result is the solution of the complex64-rounded system (the reference's production path
// stores its matrices in complex64 too, lo_frequency.rs:1-6).
#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "hbg_mixed.h"
#include "hbg_mixed_kernels.cuh"

namespace hbg {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static const EncodeTiledFn fn = [] {  // resolved once, thread-safe (the pipelines of a batch share it)
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<EncodeTiledFn>(p);
        return (EncodeTiledFn) nullptr;
    }();
    return fn;
}

// A 4-D FP32 tensor map (x innermost) with a {32, box_rows, 1, 1} box in the 128-byte swizzle.
static bool make_map(CUtensorMap* m, void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t d3, uint64_t s1,
                     uint64_t s2, uint64_t s3, uint32_t box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[4] = {d0, d1, d2, d3};
    cuuint64_t strides[3] = {s1, s2, s3};
    cuuint32_t box[4] = {32, box_rows, 1, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

// The same for FP16 rows: box {64, box_rows} (128 bytes a row, 128-byte swizzle).
static bool make_map16(CUtensorMap* m, void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t d3, uint64_t s1,
                       uint64_t s2, uint64_t s3, uint32_t box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[4] = {d0, d1, d2, d3};
    cuuint64_t strides[3] = {s1, s2, s3};
    cuuint32_t box[4] = {64, box_rows, 1, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 4, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

// Rows of 2 w floats viewed as [rows][2][w]: dims {w, 2, rows, d3}, box {32, 1, box_rows, 1}, the
// 128-byte swizzle (the same shared-memory tile as make_map's).
static bool make_map_split(CUtensorMap* m, void* base, uint64_t w, uint64_t rows, uint64_t d3, uint64_t row_stride,
                           uint64_t s3, uint32_t box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[4] = {w, 2, rows, d3};
    cuuint64_t strides[3] = {w * 4, row_stride, s3};
    cuuint32_t box[4] = {32, 1, box_rows, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

// A 4-D tensor map with an arbitrary box, no swizzle (plain row-major tiles in shared memory).
static bool make_map_box(CUtensorMap* m, CUtensorMapDataType dt, void* base, const uint64_t dims[4],
                         const uint64_t strides[3], const uint32_t box[4]) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t d[4] = {dims[0], dims[1], dims[2], dims[3]};
    cuuint64_t st[3] = {strides[0], strides[1], strides[2]};
    cuuint32_t bx[4] = {box[0], box[1], box[2], box[3]};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(m, dt, 4, base, d, st, bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

struct MixedBuffers {
    void* p[24] = {};
    int n = 0;
    ~MixedBuffers() {
        for (int i = 0; i < n; i++)
            if (p[i]) cudaFree(p[i]);
    }
    template <class T>
    T* get(size_t count) {
        void* q = nullptr;
        if (cudaMalloc(&q, count * sizeof(T)) != cudaSuccess) return nullptr;
        p[n++] = q;
        return reinterpret_cast<T*>(q);
    }
};

// Refinement stops when the error left after the last correction d_k is predicted below IR_TOL of
// the largest solution entry: that error is about rho |d_k|, rho = |d_k| / |d_{k-1}| being the
// observed contraction (about 1e-3 with the TF32 factors), and at most |d_k| itself.  The solution
// is then that of the complex64 system to ~1e-9, far inside its ~1e-7 distance from the FP64
// system's solution (the rounding of the stored matrix).
constexpr double IR_TOL = 1e-9;
constexpr int IR_MAX_IT = 30;

// Corrections run back to back before the host first looks at their norms: the count the previous
// batch of the same problem needed, IR_GUESS_START at a problem's first batch, at least 2.  Every problem
// starts from the same count, so its corrections -- and the frequencies it hands to the FP64 form --
// do not depend on what the host thread solved before (the pipelines of a batch take the problems in
// an order that varies from call to call).
constexpr int IR_GUESS_START = 3;  // the benchmark workload's count
inline int& ir_guess() {
    static thread_local int g = IR_GUESS_START;
    return g;
}

// Side streams for the LU of LU_GROUPS groups of a batch and their fork/join events, per device and
// host thread (kept across solves).
constexpr int LU_GROUPS = 4;  // at most (the streams kept)
static std::atomic<int> g_lu_groups_override{0};
void mixed_lu_groups(int groups) { g_lu_groups_override = std::max(0, std::min(groups, LU_GROUPS)); }
// the groups of a batch of ns systems of order Np: about eight systems a group, at most LU_GROUPS (a group's
// launches cover its systems, so a group of a few small systems leaves its products and factors too
// short to fill the device).  Measured: the 40 systems of order 4096 of the benchmark job 67.0 / 67.5 /
// 68.1 ms a job with 4 / 3 / 2 groups; the 64 uneven bodies (16 systems a batch, orders 896-5632, two
// pipelines) 1.79 s with 2 groups against 1.83 / 1.85-2.08 / 1.85-1.93 s with 1 / 3 / 4.
static int lu_groups_for(int Np, int ns) {
    (void)Np;
    const int o = g_lu_groups_override.load();
    return std::max(1, std::min(o > 0 ? o : std::min(LU_GROUPS, ns / 8), ns));
}
struct SideStreams {
    cudaStream_t s[LU_GROUPS + 1] = {};  // the LU groups, then the right-hand sides
    cudaEvent_t fork = nullptr, join[LU_GROUPS + 1] = {};
    bool ok = false;
};
static SideStreams& side_streams() {
    static thread_local SideStreams t[16];
    int d = 0;
    cudaGetDevice(&d);
    if (d < 0 || d >= 16) d = 0;
    SideStreams& x = t[d];
    if (!x.ok) {
        bool ok = true;
        for (int i = 0; i <= LU_GROUPS; i++) {
            ok = ok && cudaStreamCreateWithFlags(&x.s[i], cudaStreamNonBlocking) == cudaSuccess;
            ok = ok && cudaEventCreateWithFlags(&x.join[i], cudaEventDisableTiming) == cudaSuccess;
        }
        x.ok = ok && cudaEventCreateWithFlags(&x.fork, cudaEventDisableTiming) == cudaSuccess;
    }
    return x;
}

#define MIXED_FAIL(code, text, fq) \
    do {                           \
        *msg = text;               \
        *freq = fq;                \
        return code;               \
    } while (0)

int mixed_solve_frequencies(const PanelsView& pv, const double* st, const HbgProblem& pr, const HbgOptions& opt,
                            bool fin, double depth, cudaStream_t s, double* prof, int64_t* launches, const char** msg,
                            int64_t* freq, const std::function<void()>& start, const double* motion,
                            const FieldArgs& field, std::vector<int64_t>* fallback) {
    KernelProfiler& P = profiler();
    ir_guess() = IR_GUESS_START;
    // N panels; with symmetry sectors G systems of Nm = N / G unknowns per frequency (one of N otherwise)
    const int N = pv.N, G = pv.G, Nm = N / G, F = (int)pr.n_omega, H = (int)pr.n_heading, D = 6 * pv.nbod,
              nrhs = D + H;
    const int Np = (Nm + NBL - 1) / NBL * NBL;
    const size_t NP2 = (size_t)Np * Np, MB = 2 * NP2;  // floats per matrix (two planes)
    if (nrhs > 32) MIXED_FAIL(HB_ERR_UNSUPPORTED, "more than 32 right-hand sides (6 per body and one per heading)", -1);
    if (!encode_fn()) MIXED_FAIL(HB_ERR_UNSUPPORTED, "the driver offers no tensor-map encoder (TMA)", -1);
    // ---- batch size from free memory
    // GEMM operand buffers of the block row (rows 2n <= 2 (Np - NBL), 2 NBL wide), per frequency
    const size_t prep_rows = std::max<size_t>(2 * (size_t)(Np - NBL), GBN);
    const size_t prep = prep_rows * 2 * NBL;
    // per system: the matrices, the LU operands, the diagonal-block inverses, the refinement vectors
    size_t per_sys = 3 * MB * 4 + 3 * prep * 4 + (size_t)(NBL * 2 * NBL + 4 * NBL * NBL) * 4 +
                     4 * (size_t)nrhs * Np * 16 + 64 + (size_t)(Np / NBL) * NBL * NBL * 8;
    // per frequency: G systems, the boundary values and incident wave of every panel (with sectors also
    // the projected right-hand sides and the recombined potentials), the finite-depth tiles
    size_t per = G * per_sys + (size_t)(nrhs + H) * N * 16 + (G > 1 ? (size_t)2 * nrhs * N * 16 : 0) +
                 (fin ? (size_t)(T1_SIZE + T2_SIZE) * 8 + (size_t)(T1F_SIZE + T2F_SIZE) * 4 + (size_t)FP_PLANES * N * 8 + (size_t)6912 * 3 * 8 : 0);
    // The batch size from free memory; cudaMemGetInfo can take milliseconds, so the decision is kept per
    // thread and device for the same problem shape while the workspace still holds its buffers.
    Workspace& ws = workspace();
    int B = 0;
    {
        struct BatchChoice {
            int N = -1, G = -1, nrhs = -1, fin = -1, F = -1, B = 0;
            int64_t max_batch = -2;
            size_t budget = 0;
        };
        static thread_local BatchChoice last[16];
        int dev_b = 0;
        cudaGetDevice(&dev_b);
        BatchChoice& c = last[dev_b < 0 || dev_b >= 16 ? 0 : dev_b];
        const bool same = c.N == N && c.G == G && c.nrhs == nrhs && c.fin == (int)fin && c.F == F &&
                          c.max_batch == opt.max_batch && c.budget == hbm_budget();
        const size_t mats = MB * (size_t)std::max(c.B, 0) * G * 4;
        if (same && c.B > 0 && ws.bytes[WS_S32] >= mats && ws.bytes[WS_W] >= mats) {
            B = c.B;
        } else {
            size_t freeb = 0, totalb = 0;
            if (cudaMemGetInfo(&freeb, &totalb) != cudaSuccess)
                MIXED_FAIL(HB_ERR_INTERNAL, "cudaMemGetInfo failed", -1);
            freeb += ws.bytes[WS_S32] + ws.bytes[WS_A32] + ws.bytes[WS_W] + ws.bytes[WS_DINV];
            size_t avail = (size_t)(0.85 * (double)freeb);
            if (hbm_budget() > 0) avail = std::min(avail, hbm_budget());
            B = (int)std::max<size_t>(1, avail / per);
            if (opt.max_batch > 0) B = std::min(B, (int)opt.max_batch);
            B = std::min(B, F);
            c = BatchChoice{N, G, nrhs, (int)fin, F, B, opt.max_batch, hbm_budget()};
        }
    }
    const size_t nblk = (size_t)Np / NBL;
    const int BS = B * G;  // systems per batch
    bool okb = true;
    auto get = [&](int slot, size_t bytes) -> void* {
        void* q = ws.get(slot, bytes);
        okb = okb && q != nullptr;
        return q;
    };
    float* S32 = (float*)get(WS_S32, MB * BS * 4);
    float* A32 = (float*)get(WS_A32, MB * BS * 4);
    float* W = (float*)get(WS_W, MB * BS * 4);
    float* P2 = (float*)get(WS_P2, prep * BS * 4);
    // a later update's B operand: rows of 4 NBL (two 128-row blocks of U) for the 256-deep trailing update
    const size_t p3size = 2 * prep;
    float* P3 = (float*)get(WS_P3, p3size * BS * 4);
    // FP16 operands of the trailing update: P3's 4 NBL-wide layout, and the L rows of the outer step's
    // two block columns beyond its panel, [rows][Lr (2 NBL) | Li (2 NBL)]
    __half* P3h = (__half*)get(WS_P3H, p3size * BS * 2);
    const size_t l16_rows = std::max<size_t>(Np > 2 * NBL ? Np - 2 * NBL : 0, GBM);
    __half* L16 = (__half*)get(WS_L16, l16_rows * 4 * NBL * BS * 2);
    float* PL = (float*)get(WS_PL, (size_t)NBL * 2 * NBL * BS * 4);
    float* PU = (float*)get(WS_PU, (size_t)4 * NBL * NBL * BS * 4);
    float2* DINV = (float2*)get(WS_DINV, nblk * NBL * NBL * BS * sizeof(float2));
    double2* u = (double2*)get(WS_U, (size_t)nrhs * N * B * 16);
    double2* phiI = (double2*)get(WS_PHII, (size_t)std::max(H, 1) * N * B * 16);
    // symmetry sectors: the right-hand sides projected on the sectors, the potentials of every panel
    double2* up = G > 1 ? (double2*)get(WS_UP, (size_t)nrhs * Nm * BS * 16) : nullptr;
    double2* phi = G > 1 ? (double2*)get(WS_PHI, (size_t)nrhs * N * B * 16) : nullptr;
    double2* b = (double2*)get(WS_B, (size_t)nrhs * Np * BS * 16);
    double2* x = (double2*)get(WS_XM, (size_t)nrhs * Np * BS * 16);
    float2* r = (float2*)get(WS_R, (size_t)nrhs * Np * BS * 8);
    float2* rs = (float2*)get(WS_RS, (size_t)nrhs * Np * BS * 8);  // a residual kept for r - A d
    double* norms = (double*)get(WS_NORMS, IR_MAX_IT * 2 * (size_t)BS * 8);  // [iteration][batch][2]
    int* err = (int*)get(WS_ERR, sizeof(int));
    int* tctrl = (int*)get(WS_TRI_CTRL, sizeof(int) * (1 + (size_t)BS));  // the triangular sweeps' tickets
    FreqInfo* dfi = (FreqInfo*)get(WS_FI, sizeof(FreqInfo) * B);
    FdParams* dfd = (FdParams*)get(WS_FD, sizeof(FdParams) * B);
    double* dheads = (double*)get(WS_HEADS, sizeof(double) * std::max(H, 1));
    double* tiles = fin ? (double*)get(WS_TILES, sizeof(double) * (T1_SIZE + T2_SIZE) * B) : nullptr;
    float* tiles_f = fin ? (float*)get(WS_TILES_F, sizeof(float) * (T1F_SIZE + T2F_SIZE) * B) : nullptr;
    // the wave-term network (optional): its parameters, the packed BF16 image the assembly loads, and
    // the count of pairs it served
    const bool sg = opt.surrogate != nullptr;
    float* sg_params = sg ? (float*)get(WS_SG_PARAMS, sizeof(float) * SURROGATE_FLOATS) : nullptr;
    uint8_t* sg_img = sg ? (uint8_t*)get(WS_SG_IMG, sg_image_bytes()) : nullptr;
    unsigned long long* sg_count = sg ? (unsigned long long*)get(WS_SG_COUNT, sizeof(unsigned long long)) : nullptr;
    double* scr = fin ? (double*)get(WS_SCR, sizeof(double) * 6912 * 3 * B) : nullptr;
    double* fpt = fin ? (double*)get(WS_FPT, sizeof(double) * FP_PLANES * N * B) : nullptr;
    const int nfp = field.P;
    // A, B [D][D], X, FK, SC, motions, Haskind [H][D], field values [P][D] and 3 x [P][H] per frequency
    // the Kochin functions kr, krt [TK][D], kd, kdt [TK][H] and the drift [H][H][3] after them
    const int TK = pr.kochin_angles > 0 && H > 0 ? pr.kochin_angles : 0;
    const size_t kochin_per = ((size_t)TK * 2 * (D + H) + (TK ? (size_t)3 * H * H : 0)) * 2;
    const size_t out_per = 2 * (size_t)D * D + 5 * (size_t)H * 2 * D + (size_t)nfp * 2 * (D + 3 * H) + kochin_per,
                 DD = (size_t)D * D;
    double* dout = (double*)get(WS_OUT, sizeof(double) * out_per * B);
    double* fq = nfp && fin ? (double*)get(WS_FQ, sizeof(double) * FP_PLANES * (size_t)(N + nfp) * B) : nullptr;
    if (!okb) MIXED_FAIL(HB_ERR_INTERNAL, "device memory allocation failed for the mixed form", -1);
    last_surrogate_pairs() = 0;
    // ---- tensor maps (whole batch; the batch index is the 4th coordinate)
    CUtensorMap mapW, mapPL, mapPU, mapP2, mapP3, mapP3h, mapL16, mapP3w16;
    const uint64_t fb = 4;  // bytes per float
    bool okm = make_map(&mapW, W, Np, Np, 2, BS, Np * fb, NP2 * fb, MB * fb, GBM) &&
               make_map(&mapPL, PL, 2 * NBL, NBL, 1, BS, 2 * NBL * fb, (uint64_t)NBL * 2 * NBL * fb,
                        (uint64_t)NBL * 2 * NBL * fb, GBM) &&
               make_map(&mapPU, PU, 2 * NBL, 2 * NBL, 1, BS, 2 * NBL * fb, (uint64_t)4 * NBL * NBL * fb,
                        (uint64_t)4 * NBL * NBL * fb, GBN) &&
               make_map(&mapP2, P2, 2 * NBL, prep_rows, 1, BS, 2 * NBL * fb, prep * fb, prep * fb, GBN) &&
               // P3 as rows of 2 NBL (one 128-row block of U), of 4 NBL (two blocks), and the 4 NBL rows
               // viewed as [2][2 NBL] halves (the first block alone: x = kk % NBL, half = kk / NBL)
               make_map(&mapP3, P3, 2 * NBL, prep_rows, 1, BS, 2 * NBL * fb, p3size * fb, p3size * fb, GBN) &&
               make_map16(&mapP3w16, P3h, 4 * NBL, prep_rows, 1, BS, 4 * NBL * 2, p3size * 2, p3size * 2, GBN) &&
               make_map16(&mapL16, L16, 4 * NBL, l16_rows, 1, BS, 4 * NBL * 2, l16_rows * 4 * NBL * 2,
                          l16_rows * 4 * NBL * 2, GBM) &&
               make_map_split(&mapP3h, P3, 2 * NBL, prep_rows, BS, 4 * NBL * fb, p3size * fb, GBN);
    if (!okm) MIXED_FAIL(HB_ERR_INTERNAL, "tensor-map encoding failed", -1);
    const int smem = (int)gemm_smem_bytes();
    cudaFuncSetAttribute(k_gemm_tf32<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_gemm_tf32<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int dev = 0, n_sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    const int dsmem = (int)df_smem_bytes();
    cudaFuncSetAttribute(k_diag_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, dsmem);
    cudaFuncSetAttribute(k_tri_step<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri_smem_bytes(8));
    cudaFuncSetAttribute(k_tri_step<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri_smem_bytes(10));
    cudaFuncSetAttribute(k_tri_step<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri_smem_bytes(12));
    cudaFuncSetAttribute(k_tri_step<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri_smem_bytes(16));
    // the persistent sweeps: as many CTAs as fit at once
    // (the sweep's products are FP32-FMA bound beyond 16 columns: no more padded columns than needed)
    const int nr_sweep = nrhs <= 8    ? 8
                         : nrhs <= 10 ? 10
                         : nrhs <= 12 ? 12
                         : nrhs <= 16 ? 16
                         : nrhs <= 20 ? 20
                         : nrhs <= 24 ? 24
                                      : 32;
    const void* sweep_fn = nr_sweep == 8    ? (const void*)k_tri_sweep<8>
                           : nr_sweep == 10 ? (const void*)k_tri_sweep<10>
                           : nr_sweep == 12 ? (const void*)k_tri_sweep<12>
                           : nr_sweep == 16 ? (const void*)k_tri_sweep<16>
                           : nr_sweep == 20 ? (const void*)k_tri_sweep<20>
                           : nr_sweep == 24 ? (const void*)k_tri_sweep<24>
                                            : (const void*)k_tri_sweep<32>;
    cudaFuncSetAttribute(sweep_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri_smem_bytes(nr_sweep));
    int sweep_per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sweep_per_sm, sweep_fn, TRI_THREADS, tri_smem_bytes(nr_sweep));
    const int sweep_ctas = n_sm * std::max(sweep_per_sm, 1);
    std::vector<double> heads(std::max(H, 1));
    for (int h = 0; h < H; h++) heads[h] = pr.headings_deg[h] * PI / 180.0;
    std::vector<FreqInfo> fi(B);
    std::vector<FdParams> fdh(B);
    // page-locked: the reads of norms, outputs and the error flag queue behind the work, no host wait
    double* hout = (double*)ws.host(HS_OUT, sizeof(double) * (out_per * B + 1));
    double* hn = (double*)ws.host(HS_NORMS, sizeof(double) * IR_MAX_IT * 2 * (size_t)BS);
    if (!hout || !hn) MIXED_FAIL(HB_ERR_INTERNAL, "page-locked host memory could not be allocated", -1);
    int* herr = reinterpret_cast<int*>(hout + out_per * B);
    // out = bias - M x over the batch (M column-major planar FP32), FP64 accumulation
    const int nz = (Nm + GEMV_CHUNK - 1) / GEMV_CHUNK;
    double2* part = (double2*)ws.get(WS_PART, (size_t)nz * BS * nrhs * Nm * 16);
    if (!part) MIXED_FAIL(HB_ERR_INTERNAL, "device memory allocation failed for the mixed form", -1);
    for (auto fn : {(const void*)k_cgemv_tma<4>, (const void*)k_cgemv_tma<8>, (const void*)k_cgemv_tma<10>,
                    (const void*)k_cgemv_tma<12>, (const void*)k_cgemv_tma<16>})
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gv_smem_bytes<16>());
    // the column width of a chunk of w right-hand sides (the products are FP64-FMA bound: the padded
    // columns of the last chunk cost as much as real ones)
    auto chunk_width = [](int w) { return w <= 4 ? 4 : w <= 8 ? 8 : w <= 10 ? 10 : w <= 12 ? 12 : 16; };
    // the TMA form (its maps cover exactly the matrices and vectors of the batch), beyond 16 right-hand
    // sides in column chunks of 16 (the matrix streamed once a chunk); the register form if a map fails
    auto gemv_tma = [&](const float* Mm, const double2* xv, int ldx, int nb, int nzt, cudaStream_t s) -> bool {
        CUtensorMap mM, mX;
        const uint64_t dm[4] = {(uint64_t)Np, (uint64_t)Np, 2, (uint64_t)nb};
        const uint64_t sm[3] = {(uint64_t)Np * 4, NP2 * 4, MB * 4};
        const uint32_t bm[4] = {GV_ROWS, GV_COLS, 1, 1};
        if (!make_map_box(&mM, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (void*)Mm, dm, sm, bm)) return false;
        dim3 g((Nm + GV_ROWS - 1) / GV_ROWS, nb, nzt);
        for (int c0 = 0; c0 < nrhs; c0 += 16) {
            const int nr = chunk_width(std::min(16, nrhs - c0));
            const uint64_t dx[4] = {2 * (uint64_t)ldx, (uint64_t)nrhs, (uint64_t)nb, 1};
            const uint64_t sx[3] = {(uint64_t)ldx * 16, (uint64_t)nrhs * ldx * 16, (uint64_t)nb * nrhs * ldx * 16};
            const uint32_t bx[4] = {2 * GV_COLS, (uint32_t)nr, 1, 1};
            if (!make_map_box(&mX, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (void*)xv, dx, sx, bx)) return false;
            if (nr == 4)
                k_cgemv_tma<4><<<g, GV_THREADS, gv_smem_bytes<4>(), s>>>(mM, mX, Nm, nrhs, c0, part, nb, err);
            else if (nr == 8)
                k_cgemv_tma<8><<<g, GV_THREADS, gv_smem_bytes<8>(), s>>>(mM, mX, Nm, nrhs, c0, part, nb, err);
            else if (nr == 10)
                k_cgemv_tma<10><<<g, GV_THREADS, gv_smem_bytes<10>(), s>>>(mM, mX, Nm, nrhs, c0, part, nb, err);
            else if (nr == 12)
                k_cgemv_tma<12><<<g, GV_THREADS, gv_smem_bytes<12>(), s>>>(mM, mX, Nm, nrhs, c0, part, nb, err);
            else
                k_cgemv_tma<16><<<g, GV_THREADS, gv_smem_bytes<16>(), s>>>(mM, mX, Nm, nrhs, c0, part, nb, err);
        }
        return true;
    };
    const int nz_tma = (Nm + GV_CHUNK - 1) / GV_CHUNK;
    for (auto fn : {(const void*)k_cgemv32_tma<4>, (const void*)k_cgemv32_tma<8>, (const void*)k_cgemv32_tma<10>,
                    (const void*)k_cgemv32_tma<12>, (const void*)k_cgemv32_tma<16>})
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gv32_smem_bytes<16>());
    // r = rk - M d with the complex64 correction d (FP32 products, FP64 sums; beyond 16 columns in chunks):
    // the residual after a correction that is small against the solution
    auto gemv32 = [&](const float* Mm, const float2* dv, const float2* rk, float2* out, int nb) {
        CUtensorMap mM, mD;
        const uint64_t dm[4] = {(uint64_t)Np, (uint64_t)Np, 2, (uint64_t)nb};
        const uint64_t sm[3] = {(uint64_t)Np * 4, NP2 * 4, MB * 4};
        const uint32_t bm[4] = {GV_ROWS, GV_COLS, 1, 1};
        const uint64_t dd[4] = {2 * (uint64_t)Np, (uint64_t)nrhs, (uint64_t)nb, 1};
        const uint64_t sd[3] = {(uint64_t)Np * 8, (uint64_t)nrhs * Np * 8, (uint64_t)nb * nrhs * Np * 8};
        if (!make_map_box(&mM, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (void*)Mm, dm, sm, bm)) return false;
        CUtensorMap mDc[2];  // the map of each chunk width (a full chunk, the last one)
        const int nrc[2] = {chunk_width(std::min(16, nrhs)), chunk_width(nrhs - (nrhs - 1) / 16 * 16)};
        for (int q = 0; q < 2; q++) {
            const uint32_t bd[4] = {2 * GV_COLS, (uint32_t)nrc[q], 1, 1};
            if (!make_map_box(&mDc[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (void*)dv, dd, sd, bd)) return false;
        }
        P.begin(s);
        dim3 g((Nm + GV_ROWS - 1) / GV_ROWS, nb, nz_tma);
        for (int c0 = 0; c0 < nrhs; c0 += 16) {
            const bool last = c0 + 16 >= nrhs;
            const int nr = nrc[last];
            mD = mDc[last];
            if (nr == 4)
                k_cgemv32_tma<4><<<g, GV_THREADS, gv32_smem_bytes<4>(), s>>>(mM, mD, Nm, nrhs, c0, part, nb, err);
            else if (nr == 8)
                k_cgemv32_tma<8><<<g, GV_THREADS, gv32_smem_bytes<8>(), s>>>(mM, mD, Nm, nrhs, c0, part, nb, err);
            else if (nr == 10)
                k_cgemv32_tma<10><<<g, GV_THREADS, gv32_smem_bytes<10>(), s>>>(mM, mD, Nm, nrhs, c0, part, nb, err);
            else if (nr == 12)
                k_cgemv32_tma<12><<<g, GV_THREADS, gv32_smem_bytes<12>(), s>>>(mM, mD, Nm, nrhs, c0, part, nb, err);
            else
                k_cgemv32_tma<16><<<g, GV_THREADS, gv32_smem_bytes<16>(), s>>>(mM, mD, Nm, nrhs, c0, part, nb, err);
        }
        k_gemv_reduce<float2, float2><<<dim3((unsigned)(((size_t)nrhs * Nm + 255) / 256), nb), 256, 0, s>>>(
            Nm, nrhs, nb, nz_tma, part, rk, Np, out, Np);
        P.end(KF_MIXED_RESIDUAL, 8.0 * (double)Nm * Nm * nb, s);
        *launches += 2;
        return true;
    };
    auto gemv = [&](const float* Mm, const double2* xv, int ldx, const double2* bias, auto* out, int nb, int fam,
                    cudaStream_t s) {
        P.begin(s);
        dim3 g((Nm + 127) / 128, nb, nz);
        int nzr = nz;
        if (gemv_tma(Mm, xv, ldx, nb, nz_tma, s))
            nzr = nz_tma;
        else if (nrhs <= 8)
            k_cgemv_part<8><<<g, 128, 0, s>>>(Nm, Np, MB, nrhs, Mm, xv, ldx, part, nb);
        else if (nrhs <= 10)
            k_cgemv_part<10><<<g, 128, 0, s>>>(Nm, Np, MB, nrhs, Mm, xv, ldx, part, nb);
        else if (nrhs <= 12)
            k_cgemv_part<12><<<g, 128, 0, s>>>(Nm, Np, MB, nrhs, Mm, xv, ldx, part, nb);
        else if (nrhs <= 16)
            k_cgemv_part<16><<<g, 128, 0, s>>>(Nm, Np, MB, nrhs, Mm, xv, ldx, part, nb);
        else
            k_cgemv_part<32><<<g, 128, 0, s>>>(Nm, Np, MB, nrhs, Mm, xv, ldx, part, nb);
        k_gemv_reduce<<<dim3((unsigned)(((size_t)nrhs * Nm + 255) / 256), nb), 256, 0, s>>>(Nm, nrhs, nb, nzr, part,
                                                                                           bias, Np, out, Np);
        P.end(fam, 8.0 * (double)Nm * Nm * nb, s);
        *launches += 2;
    };
    // d = A^-1 d in place (complex64) with the FP32 factors in W: U^T y = d, then L^T d = y, the
    // diagonal blocks by the products with their inverses (stored by the LU)
    auto trisolve = [&](float2* xv, int nb) {
        const int nblk_i = Np / TB;
        P.begin(s);
        if (nrhs <= 32) {  // one persistent sweep per direction
            const int grid = std::min(nblk_i * nb, sweep_ctas);
            const size_t sm = tri_smem_bytes(nr_sweep);
            for (int up = 1; up >= 0; up--) {
                cudaMemsetAsync(tctrl, 0, sizeof(int) * (1 + (size_t)nb), s);
                if (nr_sweep == 8)
                    k_tri_sweep<8><<<grid, TRI_THREADS, sm, s>>>(Np, MB, W, DINV, nrhs, xv, nb, up, tctrl, err);
                else if (nr_sweep == 10)
                    k_tri_sweep<10><<<grid, TRI_THREADS, sm, s>>>(Np, MB, W, DINV, nrhs, xv, nb, up, tctrl, err);
                else if (nr_sweep == 12)
                    k_tri_sweep<12><<<grid, TRI_THREADS, sm, s>>>(Np, MB, W, DINV, nrhs, xv, nb, up, tctrl, err);
                else if (nr_sweep == 16)
                    k_tri_sweep<16><<<grid, TRI_THREADS, sm, s>>>(Np, MB, W, DINV, nrhs, xv, nb, up, tctrl, err);
                else if (nr_sweep == 20)
                    k_tri_sweep<20><<<grid, TRI_THREADS, sm, s>>>(Np, MB, W, DINV, nrhs, xv, nb, up, tctrl, err);
                else if (nr_sweep == 24)
                    k_tri_sweep<24><<<grid, TRI_THREADS, sm, s>>>(Np, MB, W, DINV, nrhs, xv, nb, up, tctrl, err);
                else
                    k_tri_sweep<32><<<grid, TRI_THREADS, sm, s>>>(Np, MB, W, DINV, nrhs, xv, nb, up, tctrl, err);
                (*launches)++;
            }
            P.end(KF_LU_SOLVE, 8.0 * (double)NP2 * nb, s);
            return;
        }
        for (int dir = 0; dir < 2; dir++) {
            const int up = dir == 0;
            for (int st = -1; st < nblk_i - 1; st++) {
                const int cnt = st < 0 ? 1 : nblk_i - 1 - st;
                const int stepi = st < 0 ? -1 : (up ? st : nblk_i - 1 - st);
                dim3 g(cnt, nb);
                if (nrhs <= 8)
                    k_tri_step<8><<<g, TRI_THREADS, tri_smem_bytes(8), s>>>(Np, MB, W, DINV, nrhs, xv, stepi, up);
                else if (nrhs <= 10)
                    k_tri_step<10><<<g, TRI_THREADS, tri_smem_bytes(10), s>>>(Np, MB, W, DINV, nrhs, xv, stepi, up);
                else if (nrhs <= 12)
                    k_tri_step<12><<<g, TRI_THREADS, tri_smem_bytes(12), s>>>(Np, MB, W, DINV, nrhs, xv, stepi, up);
                else
                    k_tri_step<16><<<g, TRI_THREADS, tri_smem_bytes(16), s>>>(Np, MB, W, DINV, nrhs, xv, stepi, up);
                (*launches)++;
            }
        }
        // the factors read once per direction (8 B per entry)
        P.end(KF_LU_SOLVE, 8.0 * (double)NP2 * nb, s);
    };
    // matrices f0 .. f0 + nb of the batch on stream st, at most cap persistent CTAs
    auto gemm = [&](const CUtensorMap& mA, const CUtensorMap& mB, GemmArgs g, int f0, int nb, cudaStream_t st,
                    int cap, bool f16) {
        g.batch = nb;
        g.b0 = f0;
        const int tiles = ((g.M + GBM - 1) / GBM) * ((g.Nc + GBN - 1) / GBN) * nb;
        P.begin(st);
        if (f16)
            k_gemm_tf32<true><<<std::min(tiles, cap), GEMM_THREADS, smem, st>>>(mA, mB, mapW, g);
        else
            k_gemm_tf32<false><<<std::min(tiles, cap), GEMM_THREADS, smem, st>>>(mA, mB, mapW, g);
        P.end(KF_MIXED_GEMM, 2.0 * g.M * (double)g.Nc * g.Kp * nb, st);
        (*launches)++;
    };
    SideStreams& side = side_streams();
    if (!side.ok) MIXED_FAIL(HB_ERR_INTERNAL, "CUDA streams for the LU could not be created", -1);
    // ---- the device work: statics, then per batch assembly, LU, refinement, forces
    start();
    cudaMemcpyAsync(dheads, heads.data(), sizeof(double) * heads.size(), cudaMemcpyHostToDevice, s);
    if (sg) {
        cudaMemcpyAsync(sg_params, opt.surrogate, sizeof(float) * SURROGATE_FLOATS, cudaMemcpyHostToDevice, s);
        launch_sg_pack(sg_params, sg_img, s);
        cudaMemsetAsync(sg_count, 0, sizeof(unsigned long long), s);
        (*launches)++;
    }
    for (int f0 = 0; f0 < F; f0 += B) {
        if (opt.cancel && *opt.cancel) MIXED_FAIL(HB_ERR_CANCELLED, "the solve was cancelled", f0);
        const int nb = std::min(B, F - f0), ns = nb * G;  // frequencies, systems
        for (int i = 0; i < nb; i++) {
            double w = pr.omegas[f0 + i], K = w * w / opt.gravity;
            fi[i].omega = w;
            fi[i].K = K;
            fi[i].k = fin ? dispersion_x0(K * depth) / depth : K;
            fi[i].logc = opt.logarithmic ? 1.0 : 0.0;
            if (fin) make_fd_params(depth, K, fdh[i]);
        }
        cudaMemcpyAsync(dfi, fi.data(), sizeof(FreqInfo) * nb, cudaMemcpyHostToDevice, s);
        if (fin) cudaMemcpyAsync(dfd, fdh.data(), sizeof(FdParams) * nb, cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(err, 0, sizeof(int), s);
        // ---- assembly, boundary values, right-hand sides
        {
            EventTimer t(s, &prof[1]);
            if (fin) {
                P.begin(s);
                launch_fd_tiles(nb, dfd, tiles, scr, s);
                launch_tiles_f32(nb, tiles, tiles_f, s);
                launch_fin_points(pv, nb, dfd, fpt, s);
                if (nfp) launch_field_fin(pv, field.pts, nfp, nb, dfd, fq, s);
                P.end(KF_FD_TILES, 0.0, s);
                *launches += 4 + (nfp > 0);
            }
            P.begin(s);
            if (sg)
                launch_assemble_f32_sg(pv, st, nb, dfi, dfd, tiles_f, fpt, fin, S32, A32, Np, sg_img, sg_count, err, s);
            else
                launch_assemble_f32(pv, st, nb, dfi, dfd, tiles_f, fpt, fin, S32, A32, Np, s);
            if (G > 1) {
                launch_sectors_f32(S32, A32, nb, G, Nm, Np, s);
                (*launches)++;
            }
            // algorithmic bytes per pair: 4 FP64 statics read (32 B), S and A written as complex64 (16 B)
            P.end(KF_ASSEMBLE, 48.0 * (double)Nm * N * nb, s);
            if (Np > Nm) k_pad_identity<<<dim3(64, ns), 256, 0, s>>>(A32, Nm, Np, MB);
            cudaMemcpyAsync(W, A32, MB * ns * 4, cudaMemcpyDeviceToDevice, s);
            P.begin(s);
            launch_boundary(pv, nb, dfi, H, dheads, depth, opt.gravity, u, phiI, s);
            P.end(KF_BOUNDARY, 0.0, s);
            *launches += 2 + (Np > Nm);  // the assembly, the boundary values, the identity padding
            t.stop();
        }
        // ---- LU of M = A^T without pivoting, blocked by NBL, the products on the tensor cores
        {
            EventTimer t(s, &prof[2]);
            // Two 128-column blocks per outer step: the second block is updated by the first alone, the
            // block row of both is solved, and the trailing matrix is updated once per 256 columns
            // (K' = 512: half the passes over it of a 128-column step).
            // The LU of LU_GROUPS groups of the batch on side streams: the diagonal-block factors (one
            // CTA per matrix, barrier-bound) of one group run beside the tensor-core products of the
            // others, whose persistent grids leave that many SMs free.
            struct Half {
                cudaStream_t st;
                int f0, nb, cap;
            };
            auto diag = [&](const Half& h, int k0) {
                P.begin(h.st);
                k_diag_factor<<<2 * h.nb, DF_THREADS, dsmem, h.st>>>(W + (size_t)h.f0 * MB, Np, MB, k0,
                                                                  PL + (size_t)h.f0 * NBL * 2 * NBL,
                                                                  PU + (size_t)h.f0 * 4 * NBL * NBL,
                                                                  DINV + (size_t)h.f0 * nblk * NBL * NBL, err);
                P.end(KF_LU_PANEL, 8.0 * NBL * (double)NBL * NBL * h.nb, h.st);
                (*launches)++;
            };
            auto prep_row = [&](const Half& h, int k0, int c0, int ncols) {  // rows k0..k0+NBL, columns c0..c0+ncols
                P.begin(h.st);
                k_prep_block_row<<<dim3(ncols / 32, NBL / 32, h.nb), dim3(32, 8), 0, h.st>>>(
                    W + (size_t)h.f0 * MB, Np, MB, k0, c0, ncols, P2 + (size_t)h.f0 * prep, prep);
                P.end(KF_MIXED_CONVERT, 2.0 * NBL * (double)ncols * 4 * 3 * h.nb, h.st);
                (*launches)++;
            };
            GemmArgs g0{};
            g0.err = err;
            // L(rows below the block) = M(., block k0) U_kk^-1; the rows from h16_row0 on also into L16 at
            // column offset h16_koff (0: the outer step's first block, NBL: its second)
            auto gemm_l = [&](const Half& h, int k0, int rows, int h16_row0, int h16_koff) {
                GemmArgs g = g0;
                g.h16 = L16;
                g.h16_bstride = l16_rows * 4 * NBL;
                g.h16_ld = 4 * NBL;
                g.h16_row0 = h16_row0;
                g.h16_koff = h16_koff;
                g.M = rows;
                g.Nc = 2 * NBL;
                g.Kp = 2 * NBL;
                g.a_planar = 1;
                g.a_x0 = k0;
                g.a_kc = NBL;
                g.a_row0 = k0 + NBL;
                g.mode = 0;
                g.o_row0 = k0 + NBL;
                g.o_col0 = k0;
                g.o_nc = NBL;
                gemm(mapW, mapPU, g, h.f0, h.nb, h.st, h.cap, false);
            };
            // U(rows k0..k0+NBL, columns c0..c0+ncols) = L_kk^-1 B (prepared in P2), and its block-real
            // copy into P3 (rows of ld floats, this block's rows from koff, second half at kh)
            auto gemm_u = [&](const Half& h, int k0, int c0, int ncols, int ld, int kh, int koff) {
                GemmArgs g = g0;
                g.M = NBL;
                g.Nc = 2 * ncols;
                g.Kp = 2 * NBL;
                g.a_planar = 0;
                g.mode = 1;
                g.o_row0 = k0;
                g.o_col0 = c0;
                g.o_nc = ncols;
                g.p3 = P3;
                g.p3_bstride = p3size;
                g.p3_n = ncols;
                g.p3_ld = ld;
                g.p3_kh = kh;
                g.p3_koff = koff;
                g.p3h = ld == 4 * NBL ? P3h : nullptr;  // the trailing update's FP16 copy
                gemm(mapPL, mapP2, g, h.f0, h.nb, h.st, h.cap, false);
            };
            // M(rows row0.., columns c0..c0+ncols) -= L(rows, columns a_x0..a_x0+a_kc) U (B operand)
            auto update = [&](const Half& h, int rows, int row0, int c0, int ncols, int a_x0, int a_kc,
                              const CUtensorMap& mB, int b_split) {
                GemmArgs g = g0;
                g.M = rows;
                g.Nc = 2 * ncols;
                g.Kp = 2 * a_kc;
                g.a_planar = 1;
                g.a_x0 = a_x0;
                g.a_kc = a_kc;
                g.a_row0 = row0;
                g.mode = 2;
                g.o_row0 = row0;
                g.o_col0 = c0;
                g.o_nc = ncols;
                g.b_split = b_split;
                gemm(mapW, mB, g, h.f0, h.nb, h.st, h.cap, false);
            };
            // the trailing matrix (rows and columns c2.., n of each) -= [L of the step's two blocks] U13,
            // K' = 512, FP16 operands (L16, P3h), FP32 accumulation and reduction into W
            auto trailing = [&](const Half& h, int c2, int n) {
                GemmArgs g = g0;
                g.M = n;
                g.Nc = 2 * n;
                g.Kp = 4 * NBL;
                g.a_planar = 0;
                g.a_row0 = 0;
                g.mode = 2;
                g.o_row0 = c2;
                g.o_col0 = c2;
                g.o_nc = n;
                gemm(mapL16, mapP3w16, g, h.f0, h.nb, h.st, h.cap, true);
            };
            // one outer step (columns K0 .. K0 + 2 NBL) of one half
            auto outer_step = [&](const Half& h, int K0) {
                const int k1 = K0 + NBL, c2 = K0 + 2 * NBL, n = Np - c2;
                // first block: factor, L below it, U of the second block's columns, update of the second block
                diag(h, K0);
                prep_row(h, K0, k1, NBL);
                gemm_l(h, K0, Np - k1, c2, 0);
                gemm_u(h, K0, k1, NBL, 2 * NBL, NBL, 0);
                update(h, Np - k1, k1, k1, NBL, K0, NBL, mapP3, 0);
                // U of the first block's rows beyond the panel (while L_KK^-1 is at hand)
                if (n > 0) {
                    prep_row(h, K0, c2, n);
                    gemm_u(h, K0, c2, n, 4 * NBL, 2 * NBL, 0);
                }
                // second block
                diag(h, k1);
                if (n > 0) {
                    gemm_l(h, k1, n, c2, NBL);
                    update(h, NBL, k1, c2, n, K0, NBL, mapP3h, NBL);  // its rows beyond the panel: -= L21 U13
                    prep_row(h, k1, c2, n);
                    gemm_u(h, k1, c2, n, 4 * NBL, 2 * NBL, NBL);
                    trailing(h, c2, n);  // the trailing matrix, K' = 512
                }
            };
            const int nh = lu_groups_for(Np, ns);
            Half hs[LU_GROUPS];
            for (int i = 0, f0 = 0; i < nh; i++) {
                const int ni = ns / nh + (i < ns % nh ? 1 : 0);
                hs[i] = Half{side.s[i], f0, ni, std::max(n_sm - 2 * (ns - ni), 1)};  // diagonal factors: two CTAs a matrix
                f0 += ni;
            }
            cudaEventRecord(side.fork, s);
            for (int i = 0; i < nh; i++) cudaStreamWaitEvent(hs[i].st, side.fork, 0);
            // the right-hand sides b = -S u on their own stream, beside the LU (the refinement needs them)
            cudaStream_t srhs = side.s[LU_GROUPS];
            cudaStreamWaitEvent(srhs, side.fork, 0);
            cudaMemsetAsync(b, 0, sizeof(double2) * nrhs * Np * ns, srhs);
            if (G > 1) {  // projected on the sectors first
                launch_project(u, up, nb, G, Nm, nrhs, Nm, srhs);
                (*launches)++;
            }
            gemv(S32, G > 1 ? up : u, Nm, nullptr, b, ns, KF_RHS, srhs);
            cudaEventRecord(side.join[LU_GROUPS], srhs);
            int K0 = 0;
            for (; K0 + 2 * NBL <= Np; K0 += 2 * NBL)
                for (int i = 0; i < nh; i++) outer_step(hs[i], K0);
            if (K0 < Np)  // an odd last block
                for (int i = 0; i < nh; i++) diag(hs[i], K0);
            for (int i = 0; i < nh; i++) {
                cudaEventRecord(side.join[i], hs[i].st);
                cudaStreamWaitEvent(s, side.join[i], 0);
            }
            cudaStreamWaitEvent(s, side.join[LU_GROUPS], 0);
            t.stop();
        }
        // ---- refinement: x_{i+1} = x_i + A^-1 (b - A x_i), A^-1 by the TF32 factors, residuals in FP64
        int it = 0;
        bool converged = false;
        {
            EventTimer t(s, &prof[3]);
            cudaMemsetAsync(x, 0, sizeof(double2) * nrhs * Np * ns, s);
            k_to_c64<<<592, 256, 0, s>>>((size_t)nrhs * Np * ns, b, r);
            (*launches)++;
            IrHistory& hist = last_ir_history();
            hist.n = 0;
            // the largest relative correction over the batch at iteration i (norms of slot i)
            auto worst_at = [&](int i) {
                double worst = 0.0;
                for (int f = 0; f < ns; f++) {
                    double ratio = hn[(size_t)i * 2 * ns + 2 * f] / std::max(hn[(size_t)i * 2 * ns + 2 * f + 1], 1e-300);
                    if (!std::isfinite(ratio)) ratio = INFINITY;
                    worst = std::max(worst, ratio);
                }
                return worst;
            };
            auto correction = [&](int i) {  // d = A^-1 r (FP32), x += d, norms into slot i
                trisolve(r, ns);
                k_ir_update<<<ns, 256, 0, s>>>(Np, nrhs, x, r, norms + (size_t)i * 2 * ns);
                *launches += 1;
            };
            // the forces and the readback of outputs, norms and the error flag (one wait for all)
            auto forces = [&]() {
                EventTimer tf(s, &prof[4]);
                double* dA = dout;
                double* dB = dout + DD * nb;
                double2* dX = reinterpret_cast<double2*>(dout + 2 * DD * nb);
                double2* dFK = dX + (size_t)H * D * nb;
                double2* dSC = dFK + (size_t)H * D * nb;
                if (G > 1) {  // the potentials of every panel from the sector solutions
                    launch_recombine(x, phi, nb, G, Nm, nrhs, Np, s);
                    (*launches)++;
                }
                P.begin(s);
                launch_forces(pv, nb, dfi, H, G > 1 ? phi : x, G > 1 ? N : Np, phiI, opt.density, dA, dB, dX, dFK, dSC, s);
                P.end(KF_FORCES, 16.0 * (double)N * (nrhs + H) * nb, s);
                launch_haskind(pv, nb, dfi, H, G > 1 ? phi : x, G > 1 ? N : Np, u, phiI, opt.density,
                               dSC + 2 * (size_t)H * D * nb + (size_t)nfp * (D + 3 * H) * nb, s);
                *launches += 1 + (H > 0);
                if (motion && H > 0) {  // the motion equation of every frequency (motion.rs:121-158)
                    launch_motions(nb, D, H, dfi, dA, dB, dX, motion, motion + DD, motion + 2 * DD,
                                   dSC + (size_t)H * D * nb, err, s);
                    (*launches)++;
                }
                if (nfp) {  // the field points from the potentials of every panel
                    double2* fr = dSC + 2 * (size_t)H * D * nb;
                    double2* fi_ = fr + (size_t)nfp * D * nb;
                    launch_field(pv, field.pts, nfp, field.stp, nb, dfi, dfd, tiles, fq, fin, H, dheads, depth,
                                 opt.gravity, G > 1 ? phi : x, G > 1 ? N : Np, u, phiI, fr, fi_, fi_ + (size_t)nfp * H * nb,
                                 fi_ + 2 * (size_t)nfp * H * nb, s);
                    (*launches)++;
                }
                if (TK) {  // the Kochin functions, then the momentum drift (with the motions when computed)
                    double2* kr = dSC + 3 * (size_t)H * D * nb + (size_t)nfp * (D + 3 * H) * nb;
                    double2* krt = kr + (size_t)TK * D * nb;
                    double2* kd = krt + (size_t)TK * D * nb;
                    double2* kdt = kd + (size_t)TK * H * nb;
                    launch_kochin(pv, nb, dfi, TK, H, depth, G > 1 ? phi : x, G > 1 ? N : Np, u, phiI, kr, krt, kd, kdt, s);
                    launch_drift(nb, D, H, TK, dfi, depth, opt.gravity, opt.density, dheads, kr, krt, kd, kdt,
                                 motion ? dSC + (size_t)H * D * nb : nullptr, kdt + (size_t)TK * H * nb, s);
                    *launches += 2;
                }
                cudaMemcpyAsync(hout, dout, sizeof(double) * out_per * nb, cudaMemcpyDeviceToHost, s);
                cudaMemcpyAsync(herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
                tf.stop();
                solve_end().record(s);
            };
            // the first `guess` corrections and the forces without waiting on the host, then one look
            // at all the norms; further corrections (and the forces again) only when they fall short.
            // The residual after the first correction is b - A x with FP64 products; after a later one
            // (|d| ~ 1e-3 |x| and smaller) it is r - A d with FP32 products (the r before the
            // correction kept in rs); the host-driven corrections beyond `guess` use b - A x again.
            const int guess = std::min(std::max(ir_guess(), 2), IR_MAX_IT);
            for (int i = 0; i < guess; i++) {
                const bool more = i + 1 < guess, inc = more && i >= 1 && rs;
                if (inc) cudaMemcpyAsync(rs, r, sizeof(float2) * nrhs * Np * ns, cudaMemcpyDeviceToDevice, s);
                correction(i);
                if (more && !(inc && gemv32(A32, r, rs, r, ns))) gemv(A32, x, Np, b, r, ns, KF_MIXED_RESIDUAL, s);
            }
            cudaMemcpyAsync(hn, norms, sizeof(double) * 2 * ns * guess, cudaMemcpyDeviceToHost, s);
            t.stop();
            forces();
            cudaStreamSynchronize(s);
            double prev = INFINITY;
            bool stalled = false;
            for (it = 0; it < guess; it++) {
                const double worst = worst_at(it);
                hist.ratio[hist.n++] = worst;
                const double rho = it > 0 ? std::min(1.0, worst / prev) : 1.0;
                if (worst * rho <= IR_TOL) {  // the error left is negligible
                    converged = true;
                    break;
                }
                if (it >= 3 && !(worst < 0.5 * prev)) stalled = true;  // stalled or diverging
                prev = worst;
            }
            if (converged) {
                ir_guess() = it + 1;
                it = guess;  // the corrections that ran (a later one only refines further)
            } else if (!stalled && *herr == 0) {
                // further corrections, one host look each: no residual after the one that meets the test
                EventTimer t2(s, &prof[3]);
                for (it = guess; it < IR_MAX_IT; it++) {
                    gemv(A32, x, Np, b, r, ns, KF_MIXED_RESIDUAL, s);
                    correction(it);
                    cudaMemcpyAsync(hn + (size_t)it * 2 * ns, norms + (size_t)it * 2 * ns, sizeof(double) * 2 * ns,
                                    cudaMemcpyDeviceToHost, s);
                    cudaStreamSynchronize(s);
                    const double worst = worst_at(it);
                    hist.ratio[hist.n++] = worst;
                    const double rho = std::min(1.0, worst / prev);
                    if (worst * rho <= IR_TOL) {
                        converged = true;
                        ir_guess() = it + 1;
                        it++;
                        break;
                    }
                    if (it >= 3 && !(worst < 0.5 * prev)) break;
                    prev = worst;
                }
                t2.stop();
                // the outputs read back so far are those of the iterate after `guess` corrections; the
                // keep-or-redo test below looks at the last correction, so the outputs must be its
                // iterate's, converged or not
                if (hist.n > guess) {
                    forces();
                    cudaStreamSynchronize(s);
                }
            }
        }
        P.flush();
        {
            const cudaError_t ce = cudaGetLastError();
            if (ce != cudaSuccess) {
                static thread_local std::string why;
                why = std::string("CUDA error in the mixed-precision solve: ") + cudaGetErrorString(ce);
                MIXED_FAIL(HB_ERR_INTERNAL, why.c_str(), f0);
            }
        }
        if (*herr == 8) MIXED_FAIL(HB_ERR_INTERNAL, "a triangular sweep wait timed out", f0);
        if (*herr == 11) MIXED_FAIL(HB_ERR_NUMERICAL, "singular motion equation", f0);
        if (*herr != 0 && *herr != 10) MIXED_FAIL(HB_ERR_INTERNAL, "a tensor-core pipeline wait timed out", f0);
        // Frequencies the reduced-precision factors cannot solve (a zero pivot of the unpivoted LU: the whole
        // batch; a system whose corrections do not contract, as near an irregular frequency) go to the FP64
        // form; a system counts as solved when its own predicted error, as the batch test, is below IR_TOL.
        std::vector<char> redo(nb, 0);
        if (*herr == 10) {
            std::fill(redo.begin(), redo.end(), 1);
        } else if (!converged) {
            const int last = last_ir_history().n - 1;
            for (int q = 0; q < ns; q++) {
                auto ratio = [&](int i) {
                    const double r = hn[(size_t)i * 2 * ns + 2 * q] / std::max(hn[(size_t)i * 2 * ns + 2 * q + 1], 1e-300);
                    return std::isfinite(r) ? r : INFINITY;
                };
                const double rl = last >= 0 ? ratio(last) : INFINITY;
                const double rho = last >= 1 ? std::min(1.0, rl / std::max(ratio(last - 1), 1e-300)) : 1.0;
                if (!(rl * rho <= IR_TOL)) redo[q / G] = 1;
            }
        }
        if (!fallback) {
            for (int i = 0; i < nb; i++)
                if (redo[i])
                    MIXED_FAIL(HB_ERR_NUMERICAL, "iterative refinement of the mixed-precision solve did not converge", f0 + i);
        }
        const double* hA = hout;
        const double* hB = hA + DD * nb;
        const double* hX = hA + 2 * DD * nb;
        const double* hFK = hX + (size_t)H * 2 * D * nb;
        const double* hSC = hFK + (size_t)H * 2 * D * nb;
        const double* hMo = hSC + (size_t)H * 2 * D * nb;
        const double* hFr = hMo + (size_t)H * 2 * D * nb;
        const double* hFi = hFr + (size_t)nfp * 2 * D * nb;
        const double* hHK = hFi + (size_t)nfp * 2 * 3 * H * nb;
        const double* hKr = hHK + (size_t)H * 2 * D * nb;
        for (int i = 0; i < nb; i++) {
            const size_t fo = (size_t)(f0 + i), hx = (size_t)H * 2 * D;
            if (redo[i]) {
                fallback->push_back((int64_t)fo);
                continue;
            }
            for (size_t q = 0; q < DD; q++)
                if (!std::isfinite(hA[DD * i + q]) || !std::isfinite(hB[DD * i + q]))
                    MIXED_FAIL(HB_ERR_NUMERICAL, "non-finite solution", f0 + i);
            if (pr.out.added_mass) memcpy(pr.out.added_mass + fo * DD, hA + DD * i, DD * sizeof(double));
            if (pr.out.radiation_damping) memcpy(pr.out.radiation_damping + fo * DD, hB + DD * i, DD * sizeof(double));
            if (pr.out.excitation) memcpy(pr.out.excitation + fo * hx, hX + hx * i, hx * sizeof(double));
            if (pr.out.froude_krylov) memcpy(pr.out.froude_krylov + fo * hx, hFK + hx * i, hx * sizeof(double));
            if (pr.out.scattering) memcpy(pr.out.scattering + fo * hx, hSC + hx * i, hx * sizeof(double));
            if (motion && pr.out.motions) memcpy(pr.out.motions + fo * hx, hMo + hx * i, hx * sizeof(double));
            if (pr.out.haskind) memcpy(pr.out.haskind + fo * hx, hHK + hx * i, hx * sizeof(double));
            if (TK) copy_kochin(pr.out, hKr, TK, D, H, nb, i, fo);
            if (nfp) {
                const size_t pd = (size_t)nfp * 2 * D, ph = (size_t)nfp * 2 * H;
                if (pr.out.field_radiation) memcpy(pr.out.field_radiation + fo * pd, hFr + pd * i, pd * sizeof(double));
                double* dst3[3] = {pr.out.field_incident, pr.out.field_scattering, pr.out.field_diffraction};
                for (int q = 0; q < 3; q++)
                    if (dst3[q]) memcpy(dst3[q] + fo * ph, hFi + ph * ((size_t)q * nb + i), ph * sizeof(double));
            }
        }
        last_ir_iterations() = it;
    }
    if (sg) {
        unsigned long long used = 0;
        cudaMemcpyAsync(&used, sg_count, sizeof used, cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        last_surrogate_pairs() = (long long)used;
    }
    return 0;
}

// Test support: C (M x N, row-major FP32) = A (M x K, row-major) B^T where B is given N x K
// (K-major), or C -= A B^T, on the tcgen05 TF32 path of the mixed LU.  M, N, K multiples of 128,
// 128, 32.
int debug_gemm_tf32(int M, int N, int K, const float* A, const float* B, float* C, bool subtract, const char** msg) {
    if (M % GBM || N % 128 || K % GBK || M <= 0 || N <= 0 || K <= 0) {
        *msg = "debug GEMM shape: M % 128, N % 128, K % 32";
        return HB_ERR_VALUE;
    }
    if (!encode_fn()) {
        *msg = "no tensor-map encoder";
        return HB_ERR_UNSUPPORTED;
    }
    MixedBuffers mb;
    float* dA = mb.get<float>((size_t)M * K);
    float* dB = mb.get<float>((size_t)N * K);
    float* dC = mb.get<float>((size_t)M * N);
    int* err = mb.get<int>(1);
    if (!dA || !dB || !dC || !err) {
        *msg = "allocation failed";
        return HB_ERR_INTERNAL;
    }
    cudaMemcpy(dA, A, sizeof(float) * M * K, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B, sizeof(float) * N * K, cudaMemcpyHostToDevice);
    if (subtract) cudaMemcpy(dC, C, sizeof(float) * M * N, cudaMemcpyHostToDevice);
    cudaMemset(err, 0, sizeof(int));
    CUtensorMap mA, mB, mC;
    if (!make_map(&mA, dA, K, M, 1, 1, (uint64_t)K * 4, (uint64_t)M * K * 4, (uint64_t)M * K * 4, GBM) ||
        !make_map(&mB, dB, K, N, 1, 1, (uint64_t)K * 4, (uint64_t)N * K * 4, (uint64_t)N * K * 4, GBN) ||
        !make_map(&mC, dC, N, M, 1, 1, (uint64_t)N * 4, (uint64_t)M * N * 4, (uint64_t)M * N * 4, GBM)) {
        *msg = "tensor-map encoding failed";
        return HB_ERR_INTERNAL;
    }
    GemmArgs g{};
    g.M = M;
    g.Nc = N;
    g.Kp = K;
    g.a_planar = 0;
    g.mode = subtract ? 2 : 0;
    g.o_nc = N;
    g.batch = 1;
    g.err = err;
    const int smem = (int)gemm_smem_bytes();
    cudaFuncSetAttribute(k_gemm_tf32<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_gemm_tf32<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int dev = 0, n_sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    // fewer CTAs than tiles, so that the persistent loop and both accumulator buffers are exercised
    const int tiles = (M / GBM) * ((N + GBN - 1) / GBN);
    k_gemm_tf32<false><<<std::max(1, std::min(tiles / 3, n_sm)), GEMM_THREADS, smem>>>(mA, mB, mC, g);
    int herr = 0;
    cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(C, dC, sizeof(float) * M * N, cudaMemcpyDeviceToHost);
    if (cudaGetLastError() != cudaSuccess) {
        *msg = "CUDA error";
        return HB_ERR_INTERNAL;
    }
    if (herr) {
        *msg = "pipeline wait timed out";
        return HB_ERR_INTERNAL;
    }
    return 0;
}

}  // namespace hbg
