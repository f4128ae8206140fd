/*
 * hb_oracle.h -- CPU oracle of the low-order frequency-domain BEM path (TEST INFRASTRUCTURE).
 *
 * A plain-C FP64 restatement of HydroBEM's diagnostic double-precision path (HB_DIAG_DOUBLE,
 * crates/hydrobem/src/env_hooks.rs:2-5): closed-form Rankine integrals to 1000 panel radii,
 * the log-singularity corrections, the identity form of the infinite-depth wave kernel, the
 * finite-depth kernel from per-frequency tiles, assembly of S and A = 2 pi I - D.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only as the checker.
 */
#ifndef HB_ORACLE_H
#define HB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Panel geometry (crates/hydrobem/src/panel_integrals.rs:22-39 PanelGeom, without the f32 tiers). */
typedef struct hbo_panel {
    int32_t nv;          /* distinct vertices (3 or 4) */
    int32_t pad;
    double v[4][3];      /* distinct projected vertices */
    double c[3];         /* area centroid */
    double n[3];         /* unit normal into the fluid */
    double area;
    double radius;       /* max |v - c| */
    double elen[4];      /* edge lengths */
    double em[4][3];     /* outward in-plane unit normals of the edges */
    double gx[9][3];     /* 3 x 3 Gauss points of the bilinear map of the projected vertices */
    double gw[9];
    double q[4][3];      /* the projected vertices as given (a repeated vertex kept): the bilinear map */
} hbo_panel;

/* surface kinds (low_order.rs:224-238): only these two reach the configs' route */
enum { HBO_WET = 0, HBO_INTERIOR = 1 };

int hbo_load_tables(const char *path);                      /* 0 ok, else error */

/* Arithmetic of the reference's default (production) path instead of its diagnostic double path
 * (HB_DIAG_DOUBLE off, crates/hydrobem/src/env_hooks.rs:51-56), process-wide until switched back:
 * Rankine integrals by float32 Gauss tiers of orders 6, 5, 4, 3 from 2 to 3, 4, 8 and beyond 8 panel
 * radii (panel_integrals.rs:288-363) and by the 3 x 3 FP64 rule beyond 12 radii where the closed forms
 * are called directly (229-240); the log-singularity integral by the 3 x 3 rule beyond 12 radii
 * (380-392); the wave kernel from the direct 2-D tables outside [0, 2)^2 (green_inf.rs:316-330,
 * 661-667); static rows rounded to float32 (lo_static.rs:59-119 with R = f32).  0: diagnostic. */
void hbo_set_production(int on);

/* geometry.rs:120-199 make_panel + panel_integrals.rs:145-217 make_panel_geom.
 * Returns 0, or 1 + index of the first invalid panel. */
int hbo_make_panels(int np, const double *verts, hbo_panel *out);
/* Interior (z = 0 lid) panels: placed exactly in z = 0 with normal +z (lo_geometry.rs:706-716). */
int hbo_make_panels_kinds(int np, const double *verts, const int32_t *kind, hbo_panel *out);

/* Kernels exposed for the golden-vector tests. */
void hbo_wave_kernel(double X, double Y, double out[7]);   /* F, FX, FY, I, IX, IY, c */
double hbo_dispersion_x0(double H);
double hbo_dispersion_xn(double H, int n);
/* mode: 0 ordinary, 1 omega = 0, 2 omega = inf.  out: Wr WrR WrZ Wrz Wi WiR WiZ Wiz */
void hbo_finite_kernel(double h, double K, int mode, double R, double z, double zeta, double out[8]);
void hbo_rankine(const hbo_panel *p, const double x[3], double out[2]);
/* the rule the static rows use at x: the float32 Gauss tier by distance in the production mode
 * (panel_integrals.rs:359-363 rankine_any), the closed forms otherwise */
void hbo_rankine_any(const hbo_panel *p, const double x[3], double out[2]);
void hbo_log_singularity(const hbo_panel *p, const double image[3], double out[2]);
double hbo_log_in_plane(const hbo_panel *p, const double x[3]);

/* Static influence rows at the panel centroids (lo_static.rs:59-119): out[(k*N + j)*4 + {rs,rd,dl,dd}] */
int hbo_statics(int N, const hbo_panel *pg, const int32_t *kind, double depth, int logint, double tol,
                double *out);

/* One ordinary frequency: S and A (column-major N x N complex128, entry (k,n) at k + n N)
 * (lo_frequency.rs:276-537 with G = 1). depth <= 0 or inf: infinite depth. */
int hbo_assemble(int N, const hbo_panel *pg, const int32_t *kind, const double *statics, double depth,
                 double omega, double grav, int logint, double *S, double *A);

/* the same with S and A stored as complex64 (the production path's matrices, lo_frequency.rs:1-6: f64
 * kernels, f32 storage) */
int hbo_assemble_c64(int N, const hbo_panel *pg, const int32_t *kind, const double *statics, double depth,
                     double omega, double grav, int logint, float *S, float *A);

/* the influence rows of P field points: (S, D column) of every panel at every point, [P][N] complex */
int hbo_field_influence(int N, const hbo_panel *pg, const int32_t *kind, int P, const double *pts, double depth,
                        double omega, double grav, int logint, double tol, double *S, double *D);

/* wave number of the incident wave: K for infinite depth, dispersion_x0(K h)/h otherwise */
double hbo_wavenumber(double omega, double depth, double grav);

#ifdef __cplusplus
}
#endif
#endif
