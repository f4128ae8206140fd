// hbg_internal.h -- host-side declarations shared by the translation units of libhydrobem_gpu.
#pragma once
#include <vector>
#include <cstdint>
#include <cuda_runtime.h>

#include "hbg_device.cuh"

namespace hbg {

// Kernel-family timing (off by default): CUDA events around each launch on its stream, resolved at
// the next host synchronization, with the algorithmic work of the launch (bytes or flops).
enum KernelFamily {
    KF_GEOMETRY = 0, KF_STATICS, KF_STATICS_ADAPTIVE, KF_FD_TILES, KF_ASSEMBLE, KF_BOUNDARY, KF_RHS,
    KF_LU_PANEL, KF_LU_LASWP, KF_LU_TRSM, KF_LU_GEMM, KF_LU_SOLVE, KF_FORCES, KF_MIXED_CONVERT,
    KF_MIXED_GEMM, KF_MIXED_RESIDUAL, KF_COUNT
};

struct KernelProfiler {
    bool on = false;
    double ms[KF_COUNT] = {};
    double work[KF_COUNT] = {};
    int64_t launches[KF_COUNT] = {};
    struct Pending {
        int fam;
        cudaEvent_t a, b;
    };
    Pending pend[4096];
    int npend = 0;
    void reset() {
        for (int i = 0; i < KF_COUNT; i++) ms[i] = work[i] = 0.0, launches[i] = 0;
    }
    // record around a launch; call begin() before and end() after the launch on stream s
    cudaEvent_t begin(cudaStream_t s) {
        if (!on) return nullptr;
        if (npend == 4096) flush();
        cudaEventCreate(&pend[npend].a);
        cudaEventRecord(pend[npend].a, s);
        return pend[npend].a;
    }
    void end(int fam, double w, cudaStream_t s) {
        launches[fam]++;
        work[fam] += w;
        if (!on) return;
        cudaEventCreate(&pend[npend].b);
        cudaEventRecord(pend[npend].b, s);
        pend[npend].fam = fam;
        npend++;
    }
    void flush() {
        for (int i = 0; i < npend; i++) {
            cudaEventSynchronize(pend[i].b);
            float t = 0.f;
            cudaEventElapsedTime(&t, pend[i].a, pend[i].b);
            ms[pend[i].fam] += t;
            cudaEventDestroy(pend[i].a);
            cudaEventDestroy(pend[i].b);
        }
        npend = 0;
    }
};

KernelProfiler& profiler();

// Device buffers kept across calls (per host thread and device), by role: a solve reuses the
// buffers of the previous one when they are large enough, so repeated solves allocate nothing.
// hbg_release_workspace frees them.
enum WsSlot {
    WS_VERTS = 0, WS_KIND, WS_PLANES, WS_BAD, WS_ST, WS_WORK, WS_NWORK, WS_S, WS_A, WS_U, WS_RHS, WS_X, WS_PHII,
    WS_IPIV, WS_INFO, WS_FI, WS_FD, WS_TILES, WS_SCR, WS_FPT, WS_HEADS, WS_OUT, WS_S32, WS_A32, WS_W, WS_P2,
    WS_P3, WS_PL, WS_PU, WS_B, WS_XM, WS_R, WS_NORMS, WS_ERR, WS_PART, WS_DINV, WS_TILES_F, WS_SG_PARAMS,
    WS_SG_IMG, WS_SG_COUNT, WS_TRI_CTRL, WS_RS, WS_L16, WS_P3H, WS_PBODY, WS_RCEN, WS_UP, WS_PHI, WS_RIGID, WS_HYD, WS_FPTS, WS_FST, WS_FQ, WS_TIERS, WS_ORIG, WS_COUNT
};

// Page-locked host buffers of a solve: a device-to-host copy into pageable memory waits for the
// stream, one into these does not.
enum HostSlot { HS_FLAGS = 0, HS_NORMS, HS_OUT, HS_COUNT };

struct Workspace {
    void* p[WS_COUNT] = {};
    size_t bytes[WS_COUNT] = {};
    void* hp[HS_COUNT] = {};
    size_t hbytes[HS_COUNT] = {};
    // a page-locked host buffer of at least b bytes for the slot (nullptr when the allocation fails)
    void* host(int slot, size_t b) {
        if (b == 0) b = 16;
        if (hbytes[slot] >= b) return hp[slot];
        if (hp[slot]) cudaFreeHost(hp[slot]);
        hp[slot] = nullptr;
        hbytes[slot] = 0;
        if (cudaMallocHost(&hp[slot], b) != cudaSuccess) return nullptr;
        hbytes[slot] = b;
        return hp[slot];
    }
    // a buffer of at least b bytes for the slot (nullptr when the allocation fails)
    void* get(int slot, size_t b) {
        if (b == 0) b = 16;
        if (bytes[slot] >= b) return p[slot];
        if (p[slot]) cudaFree(p[slot]);
        p[slot] = nullptr;
        bytes[slot] = 0;
        if (cudaMalloc(&p[slot], b) != cudaSuccess) return nullptr;
        bytes[slot] = b;
        return p[slot];
    }
    size_t held() const {
        size_t t = 0;
        for (int i = 0; i < WS_COUNT; i++) t += bytes[i];
        return t;
    }
    void release() {
        for (int i = 0; i < WS_COUNT; i++) {
            if (p[i]) cudaFree(p[i]);
            p[i] = nullptr;
            bytes[i] = 0;
        }
        for (int i = 0; i < HS_COUNT; i++) {
            if (hp[i]) cudaFreeHost(hp[i]);
            hp[i] = nullptr;
            hbytes[i] = 0;
        }
    }
};

Workspace& workspace();  // of the current device, this host thread

// Refinement iterations of the last mixed-precision batch of this thread.
inline int& last_ir_iterations() {
    static thread_local int n = 0;
    return n;
}

// The largest relative correction max|d| / max|x| over the batch, per refinement iteration, of
// the last mixed-precision batch of this thread.
struct IrHistory {
    double ratio[32];
    int n = 0;
};
inline IrHistory& last_ir_history() {
    static thread_local IrHistory h;
    return h;
}

// Phase timings recorded without waiting: the event pairs are kept until flush(), which the solve
// calls once its stream has finished, so a phase boundary never stalls the host.  The events come
// from a per-device pool kept across solves (creating events can take a driver lock, and a host
// thread held there while the device runs short of queued work would idle the device).
struct PhaseTimers {
    struct Pending {
        cudaEvent_t a, b;
        double* acc;
        int dev;
    };
    std::vector<Pending> pend;
    std::vector<cudaEvent_t> pool[16];
    static int device() {
        int d = 0;
        cudaGetDevice(&d);
        return d < 0 || d >= 16 ? 0 : d;
    }
    cudaEvent_t take(int dev) {
        if (pool[dev].empty()) {
            cudaEvent_t e = nullptr;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = pool[dev].back();
        pool[dev].pop_back();
        return e;
    }
    void give(int dev, cudaEvent_t e) { pool[dev].push_back(e); }
    void flush() {
        for (auto& p : pend) {
            cudaEventSynchronize(p.b);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, p.a, p.b);
            *p.acc += ms;
            give(p.dev, p.a);
            give(p.dev, p.b);
        }
        pend.clear();
    }
};
// The device memory the solves of this host thread may hold in their workspace (0: no limit beyond 85 %
// of the free memory): a pipeline's share when several problems are solved at once.
inline size_t& hbm_budget() {
    static thread_local size_t b = 0;
    return b;
}

inline PhaseTimers& phase_timers() {
    static thread_local PhaseTimers t;
    return t;
}

// The device span of a solve: `begin` recorded with its first device operation, `end` after the last
// device operation of each batch is queued (its output readback), before the host waits.  The
// solve's time runs from one to the other: host work before the first operation (argument checks,
// sizing, allocation) and the host's wake-up and output handling after the wait are not device time.
struct SolveMark {
    cudaEvent_t e[16] = {};
    int dev = 0;
    bool recorded = false;
    void record(cudaStream_t s) {
        dev = PhaseTimers::device();
        if (!e[dev]) cudaEventCreate(&e[dev]);
        cudaEventRecord(e[dev], s);
        recorded = true;
    }
    cudaEvent_t event() const { return e[dev]; }
};
inline SolveMark& solve_begin() {
    static thread_local SolveMark t;
    return t;
}
inline SolveMark& solve_end() {
    static thread_local SolveMark t;
    return t;
}

// Device time of a phase: events on the stream, added to *acc at the next PhaseTimers::flush().
struct EventTimer {
    cudaEvent_t a{}, b{};
    cudaStream_t s;
    double* acc;
    int dev;
    bool stopped = false;
    EventTimer(cudaStream_t st, double* target) : s(st), acc(target), dev(PhaseTimers::device()) {
        a = phase_timers().take(dev);
        b = phase_timers().take(dev);
        cudaEventRecord(a, s);
    }
    void stop() {
        cudaEventRecord(b, s);
        phase_timers().pend.push_back({a, b, acc, dev});
        stopped = true;
    }
    ~EventTimer() {
        if (!stopped) {
            phase_timers().give(dev, a);
            phase_timers().give(dev, b);
        }
    }
};

// Per-frequency data of one batch entry (one body, one omega).
struct FreqInfo {
    double omega, K, k;   // radian frequency, K = omega^2 / g, incident wave number
    double logc;          // weight of the analytic log-singularity integral (0 or 1)
};

void set_constants(const double glx[17][16], const double glw[17][16], const Tables& tab);
void set_constants_statics(const double glx[17][16], const double glw[17][16]);
// tiers (optional, [N][TIER_FLOATS_HOST]): the float32 Gauss tiers of the production Rankine rule
constexpr int TIER_FLOATS_HOST = 416;
// orig: the index of each panel in the caller's order (the invalid panel reported is the first in that
// order), or null when the panels are in it
void launch_panel_geometry(int N, const double* verts, const int32_t* kind, double* planes, int32_t* bad,
                           cudaStream_t s, float* tiers = nullptr, const int32_t* orig = nullptr);
// mixed: the mixed form's variant (far Rankine points and the order-4 log rule in FP32)
void launch_statics(const PanelsView& pv, double depth, int logint, double tol, double* st, int32_t* work,
                    int32_t* nwork, int work_cap, cudaStream_t s, bool mixed = false);
void launch_statics_adaptive(const PanelsView& pv, const int32_t* work, int nwork, double* st, cudaStream_t s);
// q: [entry count, queue cursor (zero)] in device memory; nothing runs when *bad != clean
void launch_statics_adaptive_q(const PanelsView& pv, const int32_t* work, int32_t* q, int work_cap,
                               const int32_t* bad, int32_t clean, double* st, cudaStream_t s);

// finite depth: per-frequency tiles [F][T1 | T2] and fin-point planes [F][FP_PLANES][N]
void launch_fd_tiles(int F, const FdParams* fd, double* tiles, double* scratch, cudaStream_t s);
void launch_fin_points(const PanelsView& pv, int F, const FdParams* fd, double* fpt, cudaStream_t s);

// assembly of S and A (complex128, column-major Nm x Nm per matrix, stride mat_stride elements; Nm =
// pv.N / pv.G, and with symmetry sectors the G image blocks of each frequency, matrices f G + g)
void launch_assemble_f64(const PanelsView& pv, const double* st, int F, const FreqInfo* fi, const FdParams* fd,
                         const double* tiles, const double* fpt, bool finite, double2* S, double2* A,
                         size_t mat_stride, cudaStream_t s);
void launch_assemble_f32(const PanelsView& pv, const double* st, int F, const FreqInfo* fi, const FdParams* fd,
                         const float* tiles, const double* fpt, bool finite, float* S, float* A, int Np,
                         cudaStream_t s);
void launch_tiles_f32(int F, const double* tiles, float* tiles_f, cudaStream_t s);
// symmetry sectors: the image blocks of F frequencies into their sector matrices (in place), the
// right-hand sides projected on the sectors up[F G][nrhs][ldp], the potentials of every panel
// phi[F][nrhs][G Nm] from the sector solutions x[F G][nrhs][ldx]
void launch_sectors_f64(double2* S, double2* A, int F, int G, int Nm, size_t mat_stride, cudaStream_t s);
void launch_sectors_f32(float* S, float* A, int F, int G, int Nm, int Np, cudaStream_t s);
void launch_project(const double2* u, double2* up, int F, int G, int Nm, int nrhs, int ldp, cudaStream_t s);
void launch_recombine(const double2* x, double2* phi, int F, int G, int Nm, int nrhs, int ldx, cudaStream_t s);
// the wave-term network inside the mixed assembly: its parameters followed by the outputs' means and
// spreads
constexpr int SURROGATE_FLOATS = 50822 + 12;
void launch_sg_pack(const float* params_norm, uint8_t* img, cudaStream_t s);
size_t sg_image_bytes();
void launch_assemble_f32_sg(const PanelsView& pv, const double* st, int F, const FreqInfo* fi, const FdParams* fd,
                            const float* tiles, const double* fpt, bool finite, float* S, float* A, int Np,
                            const uint8_t* img, unsigned long long* counts, int* err, cudaStream_t s);
// pairs (unordered, over all frequencies) whose wave term came from the network in the last mixed solve
inline long long& last_surrogate_pairs() {
    static thread_local long long n = 0;
    return n;
}
// boundary values u [F][nrhs][N] and incident wave phiI [F][H][N]
void launch_boundary(const PanelsView& pv, int F, const FreqInfo* fi, int H, const double* heads, double depth,
                     double grav, double2* u, double2* phiI, cudaStream_t s);
// rhs[F][nrhs][N] = -S u
void launch_rhs_f64(int N, int F, int nrhs, const double2* S, size_t mat_stride, const double2* u, double2* rhs,
                    cudaStream_t s);
// field points: the fin-point planes of the panels then the P points ([F][FP_PLANES][N + P]); the elevation
// or p / (rho g) at each point, radiation [F][P][D], incident, scattered and total [F][P][H]
void launch_field_fin(const PanelsView& pv, const double* pts, int P, int F, const FdParams* fd, double* fq,
                      cudaStream_t s);
void launch_field(const PanelsView& pv, const double* pts, int P, const double* stp, int F, const FreqInfo* fi,
                  const FdParams* fd, const double* tiles, const double* fq, bool finite, int H, const double* heads,
                  double depth, double grav, const double2* phi, int ldphi, const double2* u, const double2* phiI,
                  double2* frad, double2* finc, double2* fsca, double2* fdif, cudaStream_t s);
// frequencies of the last hbg_solve_batch of this thread that the mixed form handed to the FP64 form
inline int64_t& last_fallback_count() {
    static thread_local int64_t n = 0;
    return n;
}
// the device time (ms) of those frequencies' FP64 solves (statics included: the whole FP64 route)
inline double& last_fallback_ms() {
    static thread_local double ms = 0.0;
    return ms;
}
// the rigid data of the motions as uploaded, per body: mass (NaN: displaced), centre of gravity (3),
// inertia kind, inertia (9), inertia origin (3)
constexpr int RIGID_PER_BODY = 17;
// hydrostatics of each body (records of HBG_HS doubles) and the block-diagonal motion matrices M, C and
// the additional damping B_ext (D x D row-major); the motions xi[F][H][D] of F frequencies
void launch_hydrostatics(const PanelsView& pv, const double* rig, const double* cext, const double* bext, double rho,
                         double grav, double* hs, double* MM, double* CC, double* BB, cudaStream_t s);
void launch_motions(int F, int D, int H, const FreqInfo* fi, const double* A, const double* B, const double2* X,
                    const double* MM, const double* CC, const double* BB, double2* xi, int* err, cudaStream_t s);
// forces: out[F][...] A, B [6][6], X, FK, SC [H][6] complex, all f64
void launch_forces(const PanelsView& pv, int F, const FreqInfo* fi, int H, const double2* phi, int ldphi,
                   const double2* phiI, double rho, double* A, double* B, double2* X, double2* FK, double2* SC,
                   cudaStream_t s);
// Haskind exciting force HK [F][H][D] from the radiation potentials, the incident wave and the diffraction
// columns' boundary values u (lo_frequency.rs:1118-1171)
void launch_haskind(const PanelsView& pv, int F, const FreqInfo* fi, int H, const double2* phi, int ldphi,
                    const double2* u, const double2* phiI, double rho, double2* HK, cudaStream_t s);
// Kochin functions kr, krt [F][T][D], kd, kdt [F][T][H] of the solved potentials on T global angles, and the
// momentum drift [F][H][H][3] from them and the motions xi [F][H][D] (null: a fixed body)
void launch_kochin(const PanelsView& pv, int F, const FreqInfo* fi, int T, int H, double depth, const double2* phi,
                   int ldphi, const double2* u, const double2* phiI, double2* kr, double2* krt, double2* kd,
                   double2* kdt, cudaStream_t s);
void launch_drift(int F, int D, int H, int T, const FreqInfo* fi, double depth, double grav, double rho,
                  const double* heads, const double2* kr, const double2* krt, const double2* kd, const double2* kdt,
                  const double2* xi, double2* drift, cudaStream_t s);
constexpr int KOCHIN_MAX_HT = 4096;  // headings x Kochin angles of one problem (the drift's shared memory)

// host-side finite-depth scalars of one ordinary frequency (green_fin.rs:874-934)
void make_fd_params(double h, double K, FdParams& fd);
double dispersion_x0(double H);

// plain FP64 LU with partial pivoting, batched over F matrices (in place), and the solve
int lu_factor_f64(int N, int F, double2* A, size_t mat_stride, int32_t* ipiv, int32_t* info, cudaStream_t s,
                  int64_t* launches);
int lu_solve_f64(int N, int F, const double2* LU, size_t mat_stride, const int32_t* ipiv, int nrhs, const double2* B,
                 double2* X, cudaStream_t s);
// the factorization's schedule for the calls that follow (process-wide): the batch in `groups` groups of
// matrices on side streams (1 to 8), and look-ahead (panel b + 1 factored beside panel b's update) on or off
void lu_f64_schedule(int groups, int lookahead);
// the FP64 products' tile widths of a device, timed once when the device is first used; and the table
// (per width bucket n <= 8, 16, ..., 2048, 4096: 64-column tile or not, and the two timings in
// microseconds): 0 before the tuning, 1 heuristic (the timing could not run), 2 measured
void lu_tune_device(int dev);
int lu_tuned_tiles(int dev, int32_t* wide, float* us);

}  // namespace hbg
