/*
 * hydrobem_gpu.h -- C ABI of libhydrobem_gpu.so, the B200 implementation of HydroBEM's low-order
 * frequency-domain hot path: per-frequency assembly of the source and dipole influence matrices,
 * the dense complex solve for the radiation and diffraction potentials, and the pressure
 * integration to added mass, radiation damping and exciting force.
 *
 * Two layers:
 *  1. The model/solve/results subset of the reference's ABI (crates/hydrobem-c/include/hydrobem.h),
 *     same names, status codes and conventions, for the items of the low-order open-sea route.
 *  2. The batched entry hbg_solve_batch, which the model layer calls and which a caller with many
 *     bodies and frequencies can use directly (it mirrors solve_frequency,
 *     crates/hydrobem/src/lo_frequency.rs:1565-1576, run over whole frequency batches).
 *
 * Conventions (as docs/reference/c-api.md:49-146): every call returns an HbStatus; a failed call
 * sets a per-thread message (hb_last_error_message); out-pointers are checked first, so a refused
 * call changes nothing; arrays are C order, complex values (re, im) pairs; exceptions never cross
 * the boundary.  No torch types anywhere: plain pointers and sizes.
 */
#ifndef HYDROBEM_GPU_H
#define HYDROBEM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status: the codes of hydrobem.h:42-98 */
typedef int32_t HbStatus;
#define HB_OK 0
#define HB_ERR_VALUE 1
#define HB_ERR_TYPE 2
#define HB_ERR_UNSUPPORTED 3
#define HB_ERR_STATE 4
#define HB_ERR_CANCELLED 5
#define HB_ERR_INTERNAL 6
#define HB_ERR_ARGUMENT 7
#define HB_ERR_NUMERICAL 8
#define HB_ERR_IO 9
#define HB_ERR_EXISTS 10

/* ---- element types of HbColumn (hydrobem.h:116-151) */
#define HB_F64 1
#define HB_F32 2
#define HB_I32 3
#define HB_I64 4
#define HB_U64 5
#define HB_C64 6
#define HB_C128 7

/* The version of the reference's ABI that the hb_* subset of this header mirrors
 * (crates/hydrobem-c/src/info.rs:15, capi/include/hydrobem.h:208): hb_abi_version() returns it, so a
 * caller built against hydrobem.h and comparing with its HB_ABI_VERSION accepts this library. */
#define HB_ABI_VERSION 8
/* The revision of this library's own hbg_* entry points and structs (hbg_library_version()). */
#define HBG_ABI_VERSION 9

/* ==================================================================== batched entry */

/* precision forms of the solve */
#define HBG_FP64 0  /* FP64 assembly, FP64 LU: the correctness oracle form */
#define HBG_MIXED 1 /* complex64 matrices, reduced-precision tensor-core LU, FP64 refinement */
/* HbgOptions.statics_rule, the mixed form's Rankine rule */
#define HBG_STATICS_ACCURATE 0   /* closed forms within 20 panel radii, float32 3 x 3 rule beyond (default) */
#define HBG_STATICS_PRODUCTION 1 /* the reference's production rule: float32 Gauss tiers from 2 radii,
                                  * float32 rows (panel_integrals.rs:190-216, 288-363) */

/* panel kinds (crates/hydrobem/src/low_order.rs:224-238; only these reach this route) */
#define HBG_WET 0      /* wetted body surface */
#define HBG_INTERIOR 1 /* interior free surface z = 0 (irregular-frequency removal) */

/* One problem's panels: n_panels quadrilaterals, vertices [n_panels][4][3] (a triangle repeats its
 * last vertex, the right-hand-rule normal into the fluid: docs/reference/inputs-meshes.md §1);
 * kinds [n_panels] or NULL (all wet).  Global frame.  Interacting bodies (the reference's several
 * bodies of one model, crates/hydrobem/src/lo_frequency.rs:236-251, low_order.rs:313): n_bodies > 1
 * with panel_body [n_panels] the body of each panel (0 .. n_bodies - 1) and rotation_centers
 * [n_bodies][3] the point each body's rotations are about (NULL: the origin); n_bodies 0 or 1 and
 * panel_body NULL: one rigid body.  The rigid modes are 6 per body (surge, sway, heave, roll, pitch,
 * yaw), D = 6 n_bodies in all.
 * Symmetry planes (the reference's mesh symmetry, crates/hydrobem/src/lo_geometry.rs:25-36): with
 * symmetry != HBG_SYM_NONE the n_panels panels are one sector of the body (x >= 0 for the yz plane,
 * y >= 0 for the xz plane), kinds and panel_body are given for them, and the library adds their mirror
 * images (orientation restored); the solve then runs one system of n_panels unknowns per sector (2 or
 * 4 per frequency) instead of one of 2 or 4 n_panels: 4 or 16 times less LU work.  Each body keeps
 * its rotation centre; the results are those of the whole mirrored body. */
#define HBG_SYM_NONE 0
#define HBG_SYM_YZ 1   /* mirror x -> -x */
#define HBG_SYM_XZ 2   /* mirror y -> -y */
#define HBG_SYM_BOTH 3 /* both planes: 4 sectors */
typedef struct HbgBody {
    int64_t n_panels;
    const double *vertices;
    const int32_t *kinds;
    const int32_t *panel_body;
    int32_t n_bodies;
    const double *rotation_centers;
    int32_t symmetry;
} HbgBody;

/* The rigid-body data of the motions (crates/hydrobem/src/motion.rs, hydrostatics.rs:315-356), per body
 * in the global frame of the panels:
 *   mass [n_bodies]             kg; NaN: the displaced mass rho V (V the x estimate of the volume)
 *   center_of_gravity [n_bodies][3]
 *   inertia_kind [n_bodies]     HBG_INERTIA_COMPONENTS: inertia [3][3] in kg m^2; HBG_INERTIA_GYRATION:
 *                               radii of gyration r [3][3] in m, I_ij = m r_ij |r_ij| with the mass in use
 *   inertia [n_bodies][3][3]    about inertia_origin, body axes
 *   inertia_origin [n_bodies][3]  the point the inertia is about
 *   stiffness, damping [D][D]   additional matrices about the rotation centres, or NULL
 * The motion equation of each frequency: (C - w^2 (M + A) + i w (B + B_ext)) xi = X (motion.rs:121-158),
 * C the hydrostatic stiffness with the weight terms plus the additional stiffness, M the rigid inertia
 * about the rotation centres. */
#define HBG_INERTIA_COMPONENTS 0
#define HBG_INERTIA_GYRATION 1
typedef struct HbgRigid {
    const double *mass;
    const double *center_of_gravity;
    const int32_t *inertia_kind;
    const double *inertia;
    const double *inertia_origin;
    const double *stiffness;
    const double *damping;
} HbgRigid;

/* The hydrostatics record of one body (hydrostatics.rs:143-313), HBG_HS doubles, global frame:
 *   [0..3) the three volume estimates (x n_x, y n_y, z n_z), [3..6) the centre of buoyancy,
 *   [6] the waterplane area, [7..9) its centroid (x, y), [9..45) the stiffness of the rho g terms,
 *   [45..81) the stiffness with the weight terms, [81] the mass in use (NaN without one), [82] the
 *   displaced mass rho V_x; stiffness matrices 6 x 6 row-major about the rotation centre. */
#define HBG_HS 83

/* Outputs of one problem, caller-allocated host arrays (NULL: not wanted), float64, D = 6 n_bodies:
 *   added_mass, radiation_damping  [n_omega][D][D]   (coordinate i, radiation mode j)
 *   excitation, froude_krylov, scattering, motions, haskind  [n_omega][n_heading][D][2]  (re, im)
 *   hydrostatics  [n_bodies][HBG_HS]
 *   field_radiation  [n_omega][n_field_points][D][2]: the elevation (z = 0) or p / (rho g) per unit
 *                    displacement of each radiation mode
 *   field_incident, field_scattering, field_diffraction  [n_omega][n_field_points][n_heading][2]: the
 *                    incident, scattered and total waves there, per unit wave amplitude
 *                    (lo_frequency.rs:1392-1470)
 * motions needs the problem's rigid data, the field outputs its field points. */
typedef struct HbgOutputs {
    double *added_mass;
    double *radiation_damping;
    double *excitation;
    double *froude_krylov;
    double *scattering;
    double *motions;
    double *hydrostatics;
    double *field_radiation;
    double *field_incident;
    double *field_scattering;
    double *field_diffraction;
    double *haskind; /* [F][H][D] complex: the exciting force by the Haskind relation from the radiation
                      * potentials (lo_frequency.rs:1118-1171; the reference's excitation_haskind) */
    /* with HbgProblem.kochin_angles = T > 0 (lo_frequency.rs:1277-1374, response.rs:183-300):
     *   kochin_radiation, kochin_radiation_derivative  [F][T][D][2]: the Kochin functions of the radiation
     *       potentials on the angles 2 pi t / T and their angular derivatives, per unit velocity
     *   kochin_diffraction, kochin_diffraction_derivative  [F][T][H][2]: those of the scattered wave
     *   drift  [F][H][H][3][2]: the mean drift by momentum conservation (surge, sway force, yaw moment
     *       about the global z axis) of every heading pair, the motions included when they are asked for
     *       (`motions` not NULL; a fixed body otherwise); the equal pairs are real */
    double *kochin_radiation;
    double *kochin_radiation_derivative;
    double *kochin_diffraction;
    double *kochin_diffraction_derivative;
    double *drift;
} HbgOutputs;

typedef struct HbgProblem {
    HbgBody body;
    const double *omegas; /* rad/s, > 0 and finite */
    int64_t n_omega;
    const double *headings_deg;
    int64_t n_heading;
    HbgOutputs out;
    const HbgRigid *rigid;       /* NULL: no motions */
    const double *field_points;  /* [n_field_points][3], global, in the fluid at z <= 0; NULL: none */
    int64_t n_field_points;
    int32_t kochin_angles;       /* T > 0: the Kochin functions on T angles and the momentum drift (needs
                                  * headings; T * n_heading <= 4096); 0: none */
} HbgProblem;

typedef struct HbgOptions {
    int32_t precision;            /* HBG_FP64 or HBG_MIXED */
    int32_t logarithmic;          /* analytic log-singularity integral (default 1) */
    double log_tolerance;         /* default 1e-4 */
    double gravity;               /* default 9.80665 */
    double density;               /* default 1000 */
    double depth;                 /* <= 0 or inf: infinite depth */
    int32_t max_batch;            /* frequencies per device batch; 0: from free memory */
    int32_t device;               /* CUDA device ordinal */
    const volatile int32_t *cancel; /* optional: nonzero cancels between batches (HB_ERR_CANCELLED) */
    const float *surrogate;       /* optional, mixed form only: a trained wave-term network (50822
                                   * parameters then 12 output means/spreads, as hbg_surrogate_train
                                   * returns them) used in the assembly inside its domain; NULL: tables */
    int32_t statics_rule;         /* mixed form only: HBG_STATICS_ACCURATE (default) or HBG_STATICS_PRODUCTION */
    int32_t concurrency;          /* problems of one call solved at once on the device, each on its own
                                   * stream and share of the free memory, the next problem to the next free
                                   * pipeline, the costliest first (the reference's worker pool,
                                   * parallel.rs:31-109): 0 (default) chosen by the tuner from the problems'
                                   * sizes, 1 one after another, 2..8 that many */
} HbgOptions;

/* Defaults of the reference's schema (document_schema.rs:202-232). */
void hbg_default_options(HbgOptions *opt);

/* Solve every frequency and heading of every problem on the GPU.
 * Replaces: SolveJob::run -> solver::solve -> run_frequencies -> solve_frequency
 * (crates/hydrobem/src/model_solve.rs:310-370, solver.rs:265-345, lo_frequency.rs:1565-1635). */
HbStatus hbg_solve_batch(const HbgProblem *problems, int64_t n_problems, const HbgOptions *opt);

/* Timing of the phases of the last hbg_solve_batch of this thread, in milliseconds of device time
 * (the phase times of HB_PROFILE, low_order.rs:184-208): [statics, assembly, lu, substitution,
 * forces, total]. */
HbStatus hbg_last_profile(double *ms6);

/* Kernel-family timing of this thread's solves (the kernel-level counterpart of HB_PROFILE,
 * low_order.rs:184-208): on != 0 records CUDA events around every launch on the solve's stream.
 * hbg_kernel_profile: for family 0..15 (geometry, statics, statics_adaptive, fd_tiles, assemble,
 * boundary, rhs, lu_panel, lu_laswp, lu_trsm, lu_gemm, lu_solve, forces, mixed_convert, mixed_gemm,
 * mixed_residual) the summed device milliseconds of the last hbg_solve_batch (0 when timing is
 * off), its launches, and its algorithmic work (bytes for the memory-bound families, real flops for
 * lu_panel, lu_trsm, lu_gemm and mixed_gemm). */
HbStatus hbg_profile_kernels(int32_t on);
HbStatus hbg_kernel_profile(int32_t family, double *ms, int64_t *launches, double *work);

/* Device buffers are kept across solves of the same host thread (a repeated solve allocates
 * nothing); this frees them.  No counterpart in the reference (its buffers are per solve). */
HbStatus hbg_release_workspace(void);

/* The frequencies of the last hbg_solve_batch of this thread that the mixed form solved with the FP64 form
 * instead: those whose iterative refinement did not converge (its reduced-precision factors do not
 * contract the error, as next to an irregular frequency of a body without an interior lid) or whose
 * unpivoted LU met a zero pivot. */
HbStatus hbg_last_fallback_count(int64_t *count);
/* The device time in milliseconds of those frequencies' FP64 solves in the last hbg_solve_batch of this
 * thread (summed over the pipelines of a concurrent call; each fallback solve repeats the statics). */
HbStatus hbg_last_fallback_time(double *ms);

/* The kernels launched by the last hbg_solve_batch of this thread. */
HbStatus hbg_last_launch_count(int64_t *count);

/* ---- mesh files */

/* A low-order GDF file as read (crates/hydrobem/src/gdf.rs:511-535): the label line, ULEN, GRAV, the symmetry
 * flags ISX (x = 0 a plane of symmetry) and ISY (y = 0), and n_panels panels of 4 vertices, vertices
 * [n_panels][4][3] owned by the library until hbg_gdf_free. */
typedef struct HbgGdf {
    char label[256];
    double ulen;
    double gravity;
    int32_t isx;
    int32_t isy;
    int64_t n_panels;
    double *vertices;
} HbgGdf;

/* Reads a low-order GDF file: Fortran list-directed records (free format, commas as spaces, D exponents,
 * text after a line's numbers a comment); a trailing record of zeros only with zero_trailer.  HB_ERR_IO
 * when the file cannot be read, HB_ERR_VALUE with the reason for a malformed one. */
HbStatus hbg_read_gdf(const char *path, int32_t zero_trailer, HbgGdf *out);
HbStatus hbg_gdf_free(HbgGdf *gdf);

/* The reference's options of hb_model_load_mesh (hydrobem.h:835-852); on this route only zero_trailer is
 * read, a higher-order file is HB_ERR_UNSUPPORTED. */
typedef struct HbMeshOptions {
    int32_t higher_order;
    int32_t zero_trailer;
    const char *spl_path;
    const int32_t *discretization;
    size_t discretization_rows;
    double panel_size;
    int32_t spline_order;
    int32_t outer_quadrature;
    int32_t inner_quadrature;
} HbMeshOptions;

/* Test support: the static influence data (planes rs, rd, dl, dd; entry (k, j) at k + j N of each
 * plane, N*N doubles per plane) and the matrices S and A = 2 pi I - D (column-major complex128,
 * N*N (re, im) pairs) of one body at one frequency, FP64 form.  Any output pointer may be NULL.
 * With body->symmetry (G = 2 or 4 sectors of n = n_panels): the statics of the sector rows against
 * all G n panels (entry (k, j) at k + j n, n G n doubles per plane), and the G sector matrices S_c,
 * A_c one after the other (n*n pairs each).  With opt->statics_rule HBG_STATICS_PRODUCTION the statics
 * follow the reference's production rule (float32 Gauss tiers, float32 rows); the matrices are FP64
 * either way.
 * Replaces no reference interface (it exposes compute_static, lo_static.rs:254-308, and
 * Frequency::matrices, lo_frequency.rs:276-312, for the parity tests). */
HbStatus hbg_debug_matrices(const HbgBody *body, double omega, const HbgOptions *opt, double *statics, double *S,
                            double *A);

/* Test support: C = A B^T (subtract == 0) or C -= A B^T (subtract != 0, C read first) on the
 * tensor-core path of the mixed LU (tcgen05 kind::tf32, FP32 accumulation): A [M][K], B [N][K],
 * C [M][N], row-major FP32 host arrays; M % 128 == 0, N % 128 == 0, K % 32 == 0.  Replaces no
 * reference interface (the product kernel of the trailing update, linalg.rs:114-125, exposed for
 * its numerics test). */
HbStatus hbg_debug_gemm_tf32(int32_t M, int32_t N, int32_t K, const float *A, const float *B, float *C,
                             int32_t subtract);

/* Test support: X = A^-1 B for `batch` complex128 systems of order n by the FP64 form's LU (partial
 * pivoting, the FP64 warp-MMA trailing update) and substitution: A [batch][n][n] column-major (entry
 * (i, j) at 2 (i + j n)), B and X [batch][nrhs][n], interleaved (re, im) host arrays; nrhs <= 32.
 * HB_ERR_NUMERICAL on an exactly singular matrix.  Replaces no reference interface (the dense solve
 * of Real::lu_solve, linalg.rs:100-201 and 321-354, exposed for its numerics test). */
HbStatus hbg_debug_lu_f64(int32_t n, int32_t batch, const double *A, int32_t nrhs, const double *B, double *X);

/* Measured compute peaks of the current device, for the benchmark's rooflines: out3[0] FP64 FMA,
 * out3[1] FP64 warp MMA (mma.sync m8n8k4), out3[2] TF32 tcgen05 MMA, all dense TFLOP/s, each from
 * a kernel that keeps its pipe busy from registers or shared memory.  Replaces no reference
 * interface. */
HbStatus hbg_measure_peaks(double *out3);

/* ---- the learned part: an MLP surrogate of the regular part of the infinite-depth wave term
 * (inputs X = K R in [0, 100), Y = -K (z + zeta) in [0, 50), log-scaled, and a third input 0; outputs
 * g, g_X, g_Y with g = F + 2 e^-Y J0(X) (log(Y + R0) + gamma - log 2), and I, I_X, I_Y),
 * 3 -> 128 x 4 -> 6, SiLU, BF16 weights, FP32 accumulation, evaluated by tcgen05.mma (TMEM
 * accumulators).  No counterpart in the reference (it replaces the table
 * evaluation of green_inf.rs:316-368 inside its domain, the table remaining the fallback and the
 * judge of its error).  params: 50822 floats; norm: 12 floats (means, spreads of the outputs). */

/* Train on the current device: n_train samples of the library's own table evaluation (2-D Halton,
 * log-spaced), `steps` Adam steps of `batch` samples (cosine learning-rate decay from lr), then
 * validate on n_val further samples through the tensor-core inference kernel.  report[15]: loss of
 * the first and last step, training device ms, validation rms error / spread per output [3..8],
 * max |error| / max |target| per output [9..14]. */
HbStatus hbg_surrogate_train(int64_t n_train, int32_t batch, int32_t steps, double lr, uint64_t seed, int64_t n_val,
                             float *params, float *norm, double *report);

/* Test support: the gradient of the mean squared error over n standardized samples (inputs [n][3],
 * targets [n][6]) at params, computed by the training kernels; grads [50822]. */
HbStatus hbg_surrogate_grad(const float *params, int32_t n, const float *inputs, const float *targets, float *grads,
                            double *loss);

/* The network (tensor cores) and the table evaluation at the same n points xy [n][2] = (X, Y) in
 * [0, 100) x [0, 50): out_net, out_table [n][6] (either may be NULL); ms2 = device milliseconds of each over
 * the n points (points resident on the device). */
HbStatus hbg_surrogate_eval(const float *params, const float *norm, int32_t n, const double *xy, double *out_net,
                            double *out_table, double *ms2);

/* Pairs (unordered, summed over frequencies) whose wave term came from the network in the last
 * mixed solve of this thread with HbgOptions.surrogate set (0 otherwise). */
HbStatus hbg_last_surrogate_pairs(int64_t *n);

/* Refinement iterations of the last mixed-precision frequency batch of this thread. */
HbStatus hbg_last_ir_iterations(int32_t *n);

/* The refinement history of that batch: per iteration the largest relative correction
 * max|d| / max|x| over its frequencies (*n <= 32 values into ratios32[32]). */
HbStatus hbg_last_ir_history(double *ratios32, int32_t *n);

/* The statics of one panel set -- the frequency-independent Rankine source and dipole integrals
 * with their logarithmic-singularity corrections, FP64 [4][N][N] with entry (k, j) of plane q at
 * q N^2 + k + j N -- written into caller-owned device memory, with NO device allocation by the
 * library.  No counterpart in the reference (its statics are allocated inside the solve).
 *
 * For callers that own all device memory themselves (a pool allocator, a process that must not
 * grow its device footprint once running): the kernels' scratch (panel planes, adaptive-pair
 * worklist, flags) is one fixed __device__ array of 1.73 MB inside the library, so n_panels is at
 * most 2048; larger sets are rejected with HB_ERR_VALUE.  Every argument pointer is device memory
 * of the CURRENT device: d_vertices [N][4][3] (normals into the fluid), d_kinds [N] (HBG_WET /
 * HBG_INTERIOR, or NULL for all wetted), d_statics [4 N^2].  depth <= 0 or non-finite = infinite
 * depth.  The call runs on `stream` (a cudaStream_t; NULL = the legacy default stream), resets the
 * scratch's flags and worklist count itself, and synchronizes that stream before it returns, so
 * it cannot be captured into a CUDA graph.  The first call on each device resolves the scratch
 * address (cudaGetSymbolAddress) and writes the quadrature constants: make it before any stream
 * capture on that device begins.  All calls on one device share the one scratch array: calls
 * that overlap in time (from several host threads, or on several streams) race on it and must be
 * serialized by the caller. */
HbStatus hbg_statics_noalloc(const double *d_vertices, const int32_t *d_kinds, int64_t n_panels, double depth,
                             int32_t logarithmic, double log_tolerance, double *d_statics, void *stream);

/* ==================================================================== reference ABI subset */

typedef struct HbModel HbModel;

/* A mesh of the model read from a low-order GDF file (hydrobem.h:879-886): its panels and the symmetry
 * planes of ISX / ISY; `out` the new mesh object. */
HbStatus hb_model_load_mesh(HbModel *model, const char *name, const char *path, const HbMeshOptions *options,
                            uint64_t *out);
typedef struct HbResults HbResults;

typedef struct HbLocation {
    int64_t body;
    int64_t mesh;
    int64_t element;
    int64_t field_point;
    int64_t lid;
    int64_t frequency;
} HbLocation;

typedef struct HbColumn {
    const char *name;
    int32_t dtype;
    size_t ndim;
    const size_t *shape;
    size_t count;
    const void *data;
} HbColumn;

typedef struct HbProgress {
    int32_t stage;
    int64_t frequency;
    uint64_t stage_done;
    uint64_t stage_total;
    uint64_t frequencies_done;
    uint64_t frequencies_total;
    double seconds;
    int32_t worker;
    int32_t phase;
    int32_t step;
    int64_t item;
} HbProgress;

typedef int32_t (*HbProgressFn)(const HbProgress *progress, void *user);

#define HB_NO_OBJECT UINT64_MAX

/* hydrobem.h:233: returns HB_ABI_VERSION (8), the ABI of the reference header this subset mirrors */
uint32_t hb_abi_version(void);
/* No counterpart in the reference: the tile widths the library's tuner chose for the FP64 form's complex
 * products on a device, timed once when the device is first used (before any solve's work is queued):
 * per width bucket b = 0..9 (products of n <= 8, 16, ..., 2048 columns, then 4096), wide[b] = 1 for the
 * 64-column tile, 0 for the 32-column one, us[2b], us[2b + 1] the two timings (microseconds, 2048 rows,
 * K = min(n, 128), four matrices).  state: 0 not tuned yet, 1 the default choice (the timing could not
 * run), 2 measured. */
HbStatus hbg_tuned_tiles(int32_t device, int32_t *state, int32_t *wide, float *us);

/* No counterpart in the reference: the revision of the hbg_* entry points (HBG_ABI_VERSION). */
uint32_t hbg_library_version(void);
/* hydrobem.h:247, 256 */
const char *hb_last_error_message(void);
HbStatus hb_last_error_location(HbLocation *location);
/* hydrobem.h:507, 557 */
HbStatus hb_model_new(HbModel **out);
HbStatus hb_model_free(HbModel *model);
/* hydrobem.h:574 */
HbStatus hb_model_cancel(HbModel *model);
/* hydrobem.h:670: "" the model, "environment", "options", "bodies/<name>" */
HbStatus hb_object(HbModel *model, const char *path, uint64_t *object);
/* hydrobem.h:698: a body in the list "bodies" of the model */
HbStatus hb_add(HbModel *model, uint64_t parent, const char *list, const char *type_name, const char *name,
                int64_t index, uint64_t *out);
/* hydrobem.h:764-814: the items of the route (environment: omegas, periods, headings, depth,
 * gravity, density; body: vertices [P][4][3] (its mesh), kinds; options: logarithmic_integration,
 * log_tolerance, precision ("fp64" | "mixed"), device) */
HbStatus hb_set_bool(HbModel *model, uint64_t object, const char *item, int32_t value);
HbStatus hb_set_int(HbModel *model, uint64_t object, const char *item, int64_t value);
HbStatus hb_set_real(HbModel *model, uint64_t object, const char *item, double value);
HbStatus hb_set_text(HbModel *model, uint64_t object, const char *item, const char *value);
HbStatus hb_set_reals(HbModel *model, uint64_t object, const char *item, const double *data, const size_t *shape,
                      size_t ndim);
HbStatus hb_set_ints(HbModel *model, uint64_t object, const char *item, const int64_t *data, const size_t *shape,
                     size_t ndim);
/* hydrobem.h:646 */
HbStatus hb_model_solve(HbModel *model, HbProgressFn progress, void *user, HbResults **out);
/* hydrobem.h:1146, 1154, 1164: quantities omegas, headings, added_mass and radiation_damping
 * (HB_F32 [F][D][K]), excitation_diffraction, excitation_froude_krylov, excitation_scattering
 * (HB_C64 [F][H][D]), excitation_haskind (HB_C64 [F][H][K], K = D radiation columns); the extension
 * quantities <name>_f64 (HB_F64 / HB_C128) keep double precision. */
/* hydrobem.h:975-987 (a results object in place of the reference's HbTable): the panels as the solve uses
 * them, host work only; role "wetted", "lid" or both comma separated (null: both); the stored form of a
 * symmetric mesh unless include_reflections.  Quantities vertices (HB_F64 [P][4][3], global), body
 * (HB_I32 [P]) and kind (HB_I32 [P], HBG_WET / HBG_INTERIOR). */
HbStatus hb_model_panels(HbModel *model, const char *role, int32_t include_reflections, HbResults **out);
void hb_results_free(HbResults *results);
HbStatus hb_results_has(HbResults *results, const char *name, int32_t *has);
HbStatus hb_results_quantity(HbResults *results, const char *name, HbColumn *column);

#ifdef __cplusplus
}
#endif
#endif
