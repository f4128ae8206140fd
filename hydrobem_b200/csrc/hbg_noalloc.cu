// hbg_noalloc.cu -- the statics of a panel set (Rankine source and dipole integrals with the
// logarithmic-singularity corrections, the frequency-independent part of every influence matrix)
// computed into caller-owned device memory without allocating anything on the device.
//
// The scratch of the statics kernels (the panel planes, the worklist of pairs that need adaptive
// integration, the flags) lives in one file-scope __device__ array of fixed size, so a caller that
// owns all device memory itself -- a pool allocator, a host process that must not grow its device
// footprint after start-up -- can compute statics without the library calling cudaMalloc.  The
// panel count is bounded by that array: at most NOALLOC_MAX_PANELS panels.
#include <mutex>

namespace hbg {

constexpr int NOALLOC_MAX_PANELS = 2048;
constexpr int NOALLOC_WORK_CAP = 1 << 16;  // adaptive pairs; the allocating path's cap at N <= 4096
constexpr size_t NA_PLANES_BYTES = (size_t)P_PLANES * NOALLOC_MAX_PANELS * sizeof(double);
constexpr size_t NA_WORK_BYTES = (size_t)2 * NOALLOC_WORK_CAP * sizeof(int32_t);
constexpr size_t NA_KIND_BYTES = (size_t)NOALLOC_MAX_PANELS * sizeof(int32_t);
constexpr size_t NA_FLAG_BYTES = 256;
constexpr size_t NA_BYTES = NA_PLANES_BYTES + NA_WORK_BYTES + NA_KIND_BYTES + NA_FLAG_BYTES;
static_assert(NA_PLANES_BYTES % 256 == 0 && NA_WORK_BYTES % 256 == 0 && NA_KIND_BYTES % 256 == 0,
              "every part of the scratch starts at a 256-byte boundary");

// 1,196,032 B of panel planes + 524,288 B of worklist + 8,192 B of panel kinds + 256 B of flags
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

enum NaFlag { NA_BAD_PANEL = 0, NA_NWORK = 1, NA_BAD_KIND = 2, NA_BELOW_BOTTOM = 3 };

// Per call, before the geometry: the flags reset (the worklist count must start at zero, the
// first-bad-index flags at INT_MAX), the panel kinds copied (zero when the caller gives none) and
// checked, and the vertices checked against the sea bottom.
__global__ void k_noalloc_prepare(int N, const double* __restrict__ verts, const int32_t* __restrict__ kinds_in,
                                  int32_t* __restrict__ kinds, int32_t* __restrict__ flags, double depth) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < N) {
        const int32_t k = kinds_in ? kinds_in[j] : 0;
        kinds[j] = k;
        if (k != HBG_WET && k != HBG_INTERIOR) atomicMin(&flags[NA_BAD_KIND], j);
        if (depth > 0.0)
            for (int v = 0; v < 4; v++)
                if (verts[12 * j + 3 * v + 2] < -depth * (1.0 + 1e-12)) atomicMin(&flags[NA_BELOW_BOTTOM], j);
    }
}

__global__ void k_noalloc_flags(int32_t* flags) {
    if (threadIdx.x == 0) {
        flags[NA_BAD_PANEL] = 0x7fffffff;
        flags[NA_NWORK] = 0;
        flags[NA_BAD_KIND] = 0x7fffffff;
        flags[NA_BELOW_BOTTOM] = 0x7fffffff;
    }
}

struct NoallocDevice {
    unsigned char* scratch = nullptr;
};
static std::mutex g_noalloc_mutex;
static NoallocDevice g_noalloc_dev[16];

// The scratch address on the current device and the quadrature constants of the statics kernels,
// resolved once per device (cudaGetSymbolAddress with that device current; cudaMemcpyToSymbol).
static unsigned char* noalloc_scratch(int dev) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (dev < 0 || dev >= 16) throw Failure{HB_ERR_ARGUMENT, "device ordinal out of range"};
    NoallocDevice& d = g_noalloc_dev[dev];
    if (d.scratch) return d.scratch;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        throw Failure{HB_ERR_INTERNAL, std::string("cudaGetSymbolAddress of the fixed scratch failed: ") +
                                           cudaGetErrorString(e)};
    static double glx[17][16], glw[17][16];
    memset(glx, 0, sizeof glx);
    memset(glw, 0, sizeof glw);
    for (int n = 1; n <= 16; n++) gauss_legendre(n, glx[n], glw[n]);
    set_constants_statics(glx, glw);
    CUDA_OK(cudaGetLastError());
    d.scratch = static_cast<unsigned char*>(p);
    return d.scratch;
}

}  // namespace hbg

using namespace hbg;

extern "C" HbStatus hbg_statics_noalloc(const double* d_vertices, const int32_t* d_kinds, int64_t n_panels,
                                        double depth, int32_t logarithmic, double log_tolerance, double* d_statics,
                                        void* stream) {
    try {
        if (!d_vertices || !d_statics) return fail({HB_ERR_ARGUMENT, "null argument"});
        if (n_panels <= 0) return fail({HB_ERR_VALUE, "n_panels must be positive"});
        if (n_panels > NOALLOC_MAX_PANELS)
            return fail({HB_ERR_VALUE, "n_panels " + std::to_string(n_panels) +
                                           " exceeds the 2048 panels of the fixed scratch of hbg_statics_noalloc"});
        if (logarithmic && !(log_tolerance > 0.0)) return fail({HB_ERR_VALUE, "log_tolerance must be positive"});
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            return fail({HB_ERR_UNSUPPORTED, "no CUDA device: this library runs the path on the GPU only"});
        int dev = 0;
        CUDA_OK(cudaGetDevice(&dev));
        unsigned char* base = noalloc_scratch(dev);
        double* planes = reinterpret_cast<double*>(base);
        int32_t* work = reinterpret_cast<int32_t*>(base + NA_PLANES_BYTES);
        int32_t* kinds = reinterpret_cast<int32_t*>(base + NA_PLANES_BYTES + NA_WORK_BYTES);
        int32_t* flags = reinterpret_cast<int32_t*>(base + NA_PLANES_BYTES + NA_WORK_BYTES + NA_KIND_BYTES);
        const int N = (int)n_panels;
        const bool fin = finite_depth(depth);
        const double d = fin ? depth : 0.0;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        k_noalloc_flags<<<1, 32, 0, s>>>(flags);
        k_noalloc_prepare<<<(N + 127) / 128, 128, 0, s>>>(N, d_vertices, d_kinds, kinds, flags, d);
        launch_panel_geometry(N, d_vertices, kinds, planes, &flags[NA_BAD_PANEL], s);
        int32_t hf[4] = {0, 0, 0, 0};
        CUDA_OK(cudaMemcpyAsync(hf, flags, sizeof hf, cudaMemcpyDeviceToHost, s));
        CUDA_OK(cudaStreamSynchronize(s));
        CUDA_OK(cudaGetLastError());
        if (hf[NA_BAD_KIND] != 0x7fffffff) return fail({HB_ERR_UNSUPPORTED, "panel kind not on this route"});
        if (hf[NA_BELOW_BOTTOM] != 0x7fffffff) return fail({HB_ERR_VALUE, "a vertex lies below the sea bottom"});
        if (hf[NA_BAD_PANEL] != 0x7fffffff)
            return fail({HB_ERR_VALUE, "invalid panel " + std::to_string(hf[NA_BAD_PANEL] + 1) +
                                           " (degenerate, non-convex or non-finite)"});
        PanelsView pv{N, planes, kinds};
        launch_statics(pv, d, logarithmic, log_tolerance, d_statics, work, &flags[NA_NWORK], NOALLOC_WORK_CAP, s);
        int32_t nwork = 0;
        CUDA_OK(cudaMemcpyAsync(&nwork, &flags[NA_NWORK], sizeof nwork, cudaMemcpyDeviceToHost, s));
        CUDA_OK(cudaStreamSynchronize(s));
        if (nwork > NOALLOC_WORK_CAP)
            return fail({HB_ERR_INTERNAL, "adaptive log-integral worklist overflow in the fixed scratch"});
        launch_statics_adaptive(pv, work, nwork, d_statics, s);
        CUDA_OK(cudaStreamSynchronize(s));
        CUDA_OK(cudaGetLastError());
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    } catch (...) {
        return fail({HB_ERR_INTERNAL, "internal error"});
    }
}
