/*
 * hb_oracle.c -- CPU oracle (TEST INFRASTRUCTURE, never the product) of HydroBEM's low-order
 * frequency-domain path in its diagnostic double-precision form (HB_DIAG_DOUBLE,
 * crates/hydrobem/src/env_hooks.rs:2-5).  Each function cites the reference file:line it restates.
 * Paths are relative to crates/hydrobem/src/ of the reference.
 */
#include "hb_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PI 3.14159265358979323846
#define GAMMA 0.5772156649015329          /* constants.rs:4 */
#define LOG2 0.6931471805599453           /* constants.rs:5 */

/* ------------------------------------------------------------------ tables */
/* tables/green_inf_tables.rs:5-11, tables/green_fin_tables.rs:5-11 */
#define XT 30
#define YT 30
#define N1 16
#define N2 7
#define N3 6
#define HANKEL_TERMS 14
#define STRUVE_TERMS 14
#define FM 9
#define NW 12
#define REGIONS 13
#define NK 17
#define H_MIN 1.0e-12
#define HC 50.0
#define K_LO 0.5
#define NC (NW + 1)

static double *T1D, *T2D, *T2DD, *TASY, *TMETA, *TQ, *TL0, *TBK;
static double *tables_blob;
static int g_prod; /* the reference's production arithmetic (hbo_set_production) */

void hbo_set_production(int on) { g_prod = on != 0; }

int hbo_load_tables(const char *path) {
    if (tables_blob) return 0;
    FILE *f = fopen(path, "rb");
    if (!f) return 1;
    char magic[8];
    uint64_t cnt;
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "HBGTBL01", 8) != 0 || fread(&cnt, 8, 1, f) != 1 || cnt != 8) {
        fclose(f);
        return 2;
    }
    uint64_t len[8], total = 0;
    for (int i = 0; i < 8; i++) {
        char name[16];
        if (fread(name, 1, 16, f) != 16 || fread(&len[i], 8, 1, f) != 1) { fclose(f); return 3; }
        total += len[i];
    }
    static const uint64_t want[8] = {2040, 115200, 176400, 56, 65, 24570, 130, 1728};
    for (int i = 0; i < 8; i++)
        if (len[i] != want[i]) { fclose(f); return 4; }
    double *b = (double *)malloc(total * sizeof(double));
    if (fread(b, sizeof(double), total, f) != total) { fclose(f); free(b); return 5; }
    fclose(f);
    double *p = b;
    T1D = p; p += len[0];
    T2D = p; p += len[1];
    T2DD = p; p += len[2];
    TASY = p; p += len[3];
    TMETA = p; p += len[4];
    TQ = p; p += len[5];
    TL0 = p; p += len[6];
    TBK = p;
    tables_blob = b;
    return 0;
}

/* ------------------------------------------------------------------ small vector helpers */
static inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void cross3(const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double norm3(const double *a) { return sqrt(dot3(a, a)); }
static inline void sub3(const double *a, const double *b, double *o) {
    o[0] = a[0] - b[0];
    o[1] = a[1] - b[1];
    o[2] = a[2] - b[2];
}

/* ------------------------------------------------------------------ Gauss-Legendre (quadrature.rs:17-62) */
static double GL_X[17][16], GL_W[17][16];
static int gl_ready;

static void gauss_legendre(int n, double *x, double *w) {
    double nf = n;
    for (int i = 0; i < (n + 1) / 2; i++) {
        double z = cos(PI * (i + 0.75) / (nf + 0.5)), dp;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; k++) {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = nf * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (fabs(dz) <= 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; k++) {
            double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = nf * (z * p1 - p0) / (z * z - 1.0);
        x[i] = -z;
        x[n - 1 - i] = z;
        double wi = 2.0 / ((1.0 - z * z) * dp * dp);
        w[i] = wi;
        w[n - 1 - i] = wi;
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

static void gl_init(void) {
    if (gl_ready) return;
    for (int n = 1; n <= 16; n++) gauss_legendre(n, GL_X[n], GL_W[n]);
    gl_ready = 1;
}

/* patch_geometry.rs:14-22: the bilinear map, corners (-1,-1), (1,-1), (1,1), (-1,1) */
static void bilinear(const double vt[4][3], double u, double v, double *x, double *jac) {
    double n0 = 0.25 * (1.0 - u) * (1.0 - v), n1 = 0.25 * (1.0 + u) * (1.0 - v);
    double n2 = 0.25 * (1.0 + u) * (1.0 + v), n3 = 0.25 * (1.0 - u) * (1.0 + v);
    double xu[3], xv[3], cr[3];
    for (int d = 0; d < 3; d++) {
        x[d] = n0 * vt[0][d] + n1 * vt[1][d] + n2 * vt[2][d] + n3 * vt[3][d];
        xu[d] = (0.25 * (1.0 - v)) * (vt[1][d] - vt[0][d]) + (0.25 * (1.0 + v)) * (vt[2][d] - vt[3][d]);
        xv[d] = (0.25 * (1.0 - u)) * (vt[3][d] - vt[0][d]) + (0.25 * (1.0 + u)) * (vt[2][d] - vt[1][d]);
    }
    cross3(xu, xv, cr);
    *jac = norm3(cr);
}

/* ------------------------------------------------------------------ panels */
#define COINCIDENCE_TOL 1e-6
#define CONVEXITY_TOL 1e-6

/* geometry.rs:120-199 (make_panel): projection onto the midpoint plane, then
 * panel_integrals.rs:145-217 (make_panel_geom) without the f32 tier rules. */
static int make_one(const double *v12, int kind, hbo_panel *g) {
    double raw[4][3];
    for (int i = 0; i < 12; i++)
        if (!isfinite(v12[i])) return 1;
    for (int i = 0; i < 4; i++)
        for (int d = 0; d < 3; d++) raw[i][d] = v12[3 * i + d];
    double diameter = 0.0, t[3];
    for (int i = 0; i < 4; i++)
        for (int j = i + 1; j < 4; j++) {
            sub3(raw[i], raw[j], t);
            double nn = norm3(t);
            if (nn > diameter) diameter = nn;
        }
    if (diameter == 0.0) return 1;
    double tol = COINCIDENCE_TOL * diameter;
    int keep[4], m = 0;
    for (int i = 0; i < 4; i++) {
        sub3(raw[i], raw[(i + 1) % 4], t);
        if (norm3(t) > tol) keep[m++] = i;
    }
    if (m < 3) return 1;
    for (int a = 0; a < m; a++)
        for (int b = a + 1; b < m; b++) {
            sub3(raw[keep[a]], raw[keep[b]], t);
            if (norm3(t) <= tol) return 1;
        }
    double c[3], d1[3], d2[3], n[3];
    for (int d = 0; d < 3; d++) c[d] = 0.25 * (raw[0][d] + raw[1][d] + raw[2][d] + raw[3][d]);
    sub3(raw[2], raw[0], d1);
    sub3(raw[3], raw[1], d2);
    cross3(d1, d2, n);
    double nn = norm3(n);
    if (0.5 * nn <= COINCIDENCE_TOL * diameter * diameter) return 1;
    double nh[3] = {n[0] / nn, n[1] / nn, n[2] / nn};
    /* (1/nn) * n is a multiply of each component by the reciprocal in the reference */
    double inv = 1.0 / nn;
    nh[0] = inv * n[0];
    nh[1] = inv * n[1];
    nh[2] = inv * n[2];
    double proj[4][3];
    for (int i = 0; i < 4; i++) {
        sub3(raw[i], c, t);
        double s = dot3(t, nh);
        for (int d = 0; d < 3; d++) proj[i][d] = raw[i][d] - s * nh[d];
    }
    double poly[4][3];
    for (int a = 0; a < m; a++)
        for (int d = 0; d < 3; d++) poly[a][d] = proj[keep[a]][d];
    for (int a = 0; a < m; a++) {
        double e1[3], e2[3], cr[3];
        sub3(poly[(a + 1) % m], poly[a], e1);
        sub3(poly[(a + 2) % m], poly[(a + 1) % m], e2);
        cross3(e1, e2, cr);
        double s = dot3(cr, nh) / (norm3(e1) * norm3(e2));
        if (!(s > CONVEXITY_TOL)) return 1;
    }
    double area = 0.0, mom[3] = {0, 0, 0};
    for (int a = 1; a < m - 1; a++) {
        double e1[3], e2[3], cr[3];
        sub3(poly[a], poly[0], e1);
        sub3(poly[a + 1], poly[0], e2);
        cross3(e1, e2, cr);
        double tt = 0.5 * dot3(cr, nh);
        area += tt;
        for (int d = 0; d < 3; d++) mom[d] += (tt / 3.0) * (poly[0][d] + poly[a][d] + poly[a + 1][d]);
    }
    double cent[3];
    for (int d = 0; d < 3; d++) cent[d] = (1.0 / area) * mom[d];
    double normal[3] = {nh[0], nh[1], nh[2]};
    double q[4][3];
    memcpy(q, proj, sizeof q);
    if (kind == HBO_INTERIOR) {
        /* lo_geometry.rs:706-716: interior surfaces lie exactly in z = 0, normal +z, a downward
         * element taken counter-clockwise from above */
        if (nh[2] < 0.0) {
            double s[3];
            memcpy(s, q[1], sizeof s);
            memcpy(q[1], q[3], sizeof s);
            memcpy(q[3], s, sizeof s);
        }
        for (int i = 0; i < 4; i++) q[i][2] = 0.0;
        cent[2] = 0.0;
        normal[0] = 0.0;
        normal[1] = 0.0;
        normal[2] = 1.0;
    }
    /* make_panel_geom */
    memset(g, 0, sizeof *g);
    memcpy(g->n, normal, sizeof normal);
    memcpy(g->c, cent, sizeof cent);
    g->area = area;
    double diam = 0.0;
    for (int i = 0; i < 4; i++)
        for (int j = i + 1; j < 4; j++) {
            sub3(q[i], q[j], t);
            double nn2 = norm3(t);
            if (nn2 > diam) diam = nn2;
        }
    for (int i = 0; i < 4; i++) {
        sub3(q[i], q[(i + 1) % 4], t);
        if (norm3(t) > COINCIDENCE_TOL * diam) {
            memcpy(g->v[g->nv], q[i], sizeof t);
            g->nv++;
        }
    }
    int nv = g->nv;
    for (int i = 0; i < nv; i++) {
        sub3(g->v[i], cent, t);
        double r = norm3(t);
        if (r > g->radius) g->radius = r;
    }
    for (int e = 0; e < nv; e++) {
        double edge[3], cr[3];
        sub3(g->v[(e + 1) % nv], g->v[e], edge);
        g->elen[e] = norm3(edge);
        cross3(edge, normal, cr);
        for (int d = 0; d < 3; d++) g->em[e][d] = (1.0 / g->elen[e]) * cr[d];
    }
    gl_init();
    double sum = 0.0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double jac;
            bilinear((const double(*)[3])q, GL_X[3][i], GL_X[3][j], g->gx[3 * i + j], &jac);
            g->gw[3 * i + j] = GL_W[3][i] * GL_W[3][j] * jac;
            sum += g->gw[3 * i + j];
        }
    for (int k = 0; k < 9; k++) g->gw[k] *= area / sum;
    memcpy(g->q, q, sizeof q);
    return 0;
}

int hbo_make_panels_kinds(int np, const double *verts, const int32_t *kind, hbo_panel *out) {
    for (int i = 0; i < np; i++)
        if (make_one(verts + 12 * i, kind ? kind[i] : HBO_WET, out + i)) return 1 + i;
    return 0;
}

int hbo_make_panels(int np, const double *verts, hbo_panel *out) {
    return hbo_make_panels_kinds(np, verts, NULL, out);
}

/* ------------------------------------------------------------------ Rankine integrals */
/* panel_integrals.rs:226-275 rankine(): closed forms within 1000 radii (diagnostic mode) or FAR_RATIO =
 * 12 radii (production), the 3 x 3 FP64 rule beyond */
#define FAR_RATIO 12.0
#define EXACT_RATIO 2.0
static void rankine(const hbo_panel *p, const double *x, double *S, double *D) {
    double rc[3];
    sub3(x, p->c, rc);
    double dist = norm3(rc);
    if (dist > (g_prod ? FAR_RATIO : 1000.0) * p->radius) {
        double s = 0.0, dd = 0.0;
        for (int k = 0; k < 9; k++) {
            double r[3];
            sub3(x, p->gx[k], r);
            double ir = 1.0 / norm3(r);
            s += p->gw[k] * ir;
            dd += p->gw[k] * dot3(p->n, r) * ir * ir * ir;
        }
        *S = s;
        *D = dd;
        return;
    }
    double w = dot3(rc, p->n);
    int nv = p->nv;
    double av[4][3], r[4];
    for (int i = 0; i < nv; i++) {
        sub3(p->v[i], x, av[i]);
        r[i] = norm3(av[i]);
    }
    double omega = 0.0;
    if (fabs(w) > 1e-12 * p->radius) {
        for (int i = 1; i < nv - 1; i++) {
            double bc[3];
            cross3(av[i], av[i + 1], bc);
            double num = dot3(av[0], bc);
            double den = r[0] * r[i] * r[i + 1] + dot3(av[0], av[i]) * r[i + 1] + dot3(av[0], av[i + 1]) * r[i] +
                         dot3(av[i], av[i + 1]) * r[0];
            omega -= 2.0 * atan2(num, den);
        }
    }
    double s = 0.0;
    for (int e = 0; e < nv; e++) {
        int f = (e + 1) % nv;
        double d = dot3(av[e], p->em[e]);
        if (fabs(d) <= 1e-14 * p->radius) continue;
        double q = r[e] * r[f] + dot3(av[e], av[f]);
        if (!(q > 0.0)) continue;
        double sum = r[e] + r[f] + p->elen[e];
        s += d * log(sum * sum / (2.0 * q));
    }
    *S = s - w * omega;
    *D = omega;
}

void hbo_rankine(const hbo_panel *p, const double x[3], double out[2]) { rankine(p, x, &out[0], &out[1]); }

/* The float32 Gauss tiers of the production path (panel_integrals.rs:190-216): for orders 3, 4, 5, 6 the
 * n x n points of the bilinear map relative to the centroid and the weights scaled to the exact area,
 * each block padded with zero weights to a multiple of 8 (lengths 16, 16, 32, 40). */
#define TIER_FLOATS 416
static const int TIER_OFF[4] = {0, 64, 128, 256}, TIER_LEN[4] = {16, 16, 32, 40};
static void panel_tiers(const hbo_panel *p, float *tq) {
    memset(tq, 0, sizeof(float) * TIER_FLOATS);
    for (int t = 0; t < 4; t++) {
        const int n = 3 + t, cnt = n * n, len = TIER_LEN[t];
        float *b = tq + TIER_OFF[t];
        double pts[36][3], ww[36], wsum = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double jac;
                bilinear((const double(*)[3])p->q, GL_X[n][i], GL_X[n][j], pts[i * n + j], &jac);
                ww[i * n + j] = GL_W[n][i] * GL_W[n][j] * jac;
                wsum += ww[i * n + j];
            }
        for (int k = 0; k < cnt; k++) {
            b[k] = (float)(pts[k][0] - p->c[0]);
            b[len + k] = (float)(pts[k][1] - p->c[1]);
            b[2 * len + k] = (float)(pts[k][2] - p->c[2]);
            b[3 * len + k] = (float)(ww[k] * p->area / wsum);
        }
    }
}

/* panel_integrals.rs:288-300 rankine_tier: 0 (order 3) beyond 8 radii, 1 (4) from 4, 2 (5) from 3,
 * 3 (6) from 2, -1 (closed forms) within 2 */
static inline int rankine_tier(double r) {
    return r >= 8.0 ? 0 : r >= 4.0 ? 1 : r >= 3.0 ? 2 : r >= EXACT_RATIO ? 3 : -1;
}

/* panel_integrals.rs:305-357 rankine_gauss: the tier's rule in float32 on the point taken relative to the
 * centroid in double, eight accumulator lanes summed in double */
static void rankine_gauss(const hbo_panel *p, const float *tq, const double *x, int t, double *S, double *D) {
    const int len = TIER_LEN[t];
    const float *b = tq + TIER_OFF[t];
    const float px = (float)(x[0] - p->c[0]), py = (float)(x[1] - p->c[1]), pz = (float)(x[2] - p->c[2]);
    const float nx = (float)p->n[0], ny = (float)p->n[1], nz = (float)p->n[2];
    float sacc[8] = {0}, dacc[8] = {0};
    for (int k = 0; k < len; k += 8)
        for (int l = 0; l < 8; l++) {
            const float rx = px - b[k + l], ry = py - b[len + k + l], rz = pz - b[2 * len + k + l];
            const float w = b[3 * len + k + l];
            const float r2 = fmaf(rz, rz, fmaf(rx, rx, ry * ry));
            const float ir = 1.0f / sqrtf(r2);
            const float nr = fmaf(nz, rz, fmaf(nx, rx, ny * ry));
            sacc[l] = fmaf(w, ir, sacc[l]);
            dacc[l] = fmaf(w * nr, ir * (ir * ir), dacc[l]);
        }
    double s = 0.0, d = 0.0;
    for (int l = 0; l < 8; l++) {
        s += (double)sacc[l];
        d += (double)dacc[l];
    }
    *S = s;
    *D = d;
}

/* panel_integrals.rs:359-363 rankine_any: the tier rule, or the closed forms within 2 radii (the
 * diagnostic mode: always the closed forms) */
static void rankine_any(const hbo_panel *p, const float *tq, const double *x, double *S, double *D) {
    double rc[3];
    sub3(x, p->c, rc);
    const int t = (g_prod && tq) ? rankine_tier(norm3(rc) / p->radius) : -1;
    if (t < 0)
        rankine(p, x, S, D);
    else
        rankine_gauss(p, tq, x, t, S, D);
}

void hbo_rankine_any(const hbo_panel *p, const double x[3], double out[2]) {
    gl_init();
    float tq[TIER_FLOATS];
    panel_tiers(p, tq);
    rankine_any(p, tq, x, &out[0], &out[1]);
}

/* panel_integrals.rs:281-286 psi_terms */
static inline void psi_terms(const double *xi, const double *pp, const double *n, double *psi, double *dpsi) {
    double d[3];
    sub3(xi, pp, d);
    double R = norm3(d);
    double den = R - d[2];
    *psi = log(den);
    *dpsi = (dot3(d, n) / R - n[2]) / den;
}

/* the panel map of the log integrals: distinct vertices, a triangle's last one repeated
 * (panel_integrals.rs:50-54) */
static void panel_map(const hbo_panel *p, double m[4][3]) {
    memcpy(m[0], p->v[0], 3 * sizeof(double));
    memcpy(m[1], p->v[1], 3 * sizeof(double));
    memcpy(m[2], p->v[2], 3 * sizeof(double));
    memcpy(m[3], p->nv == 4 ? p->v[3] : p->v[2], 3 * sizeof(double));
}

typedef struct {
    double map[4][3];
    const hbo_panel *p;
    const double *image;
    double tol_l, tol_d;
} log_ctx;

/* the 4 x 4 Gauss rule of a cell (panel_integrals.rs:80-98) */
static void log_cell(const log_ctx *c, double u0, double u1, double v0, double v1, double *s) {
    s[0] = s[1] = 0.0;
    double hu = 0.5 * (u1 - u0), hv = 0.5 * (v1 - v0);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            double xi[3], jac, psi, dpsi;
            bilinear((const double(*)[3])c->map, u0 + hu * (GL_X[4][i] + 1.0), v0 + hv * (GL_X[4][j] + 1.0), xi, &jac);
            double ww = GL_W[4][i] * GL_W[4][j] * hu * hv * jac;
            psi_terms(xi, c->image, c->p->n, &psi, &dpsi);
            s[0] += ww * psi;
            s[1] += ww * dpsi;
        }
}

/* adaptive quadrisection, at most 14 levels (panel_integrals.rs:100-120) */
static void log_adapt(const log_ctx *c, double u0, double u1, double v0, double v1, const double *prev, int depth,
                      double *acc) {
    double um = 0.5 * (u0 + u1), vm = 0.5 * (v0 + v1);
    double cc[4][2];
    log_cell(c, u0, um, v0, vm, cc[0]);
    log_cell(c, um, u1, v0, vm, cc[1]);
    log_cell(c, um, u1, vm, v1, cc[2]);
    log_cell(c, u0, um, vm, v1, cc[3]);
    double sum[2];
    for (int k = 0; k < 2; k++) sum[k] = cc[0][k] + cc[1][k] + cc[2][k] + cc[3][k];
    if (depth >= 14 || (fabs(sum[0] - prev[0]) <= c->tol_l && fabs(sum[1] - prev[1]) <= c->tol_d)) {
        acc[0] += sum[0];
        acc[1] += sum[1];
        return;
    }
    double us[4][2] = {{u0, um}, {um, u1}, {um, u1}, {u0, um}};
    double vs[4][2] = {{v0, vm}, {v0, vm}, {vm, v1}, {vm, v1}};
    for (int q = 0; q < 4; q++) log_adapt(c, us[q][0], us[q][1], vs[q][0], vs[q][1], cc[q], depth + 1, acc);
}

/* panel_integrals.rs:380-450 log_singularity, diagnostic mode (no 3 x 3 far rule) */
static void log_singularity(const hbo_panel *p, const double *image, double *L, double *Ld) {
    double t[3];
    sub3(image, p->c, t);
    double dist = norm3(t);
    if (g_prod && dist > FAR_RATIO * p->radius) {  /* production: the 3 x 3 rule far away (380-392) */
        double l = 0.0, ld = 0.0;
        for (int k = 0; k < 9; k++) {
            double psi, dpsi;
            psi_terms(p->gx[k], image, p->n, &psi, &dpsi);
            l += p->gw[k] * psi;
            ld += p->gw[k] * dpsi;
        }
        *L = l;
        *Ld = ld;
        return;
    }
    log_ctx c;
    panel_map(p, c.map);
    c.p = p;
    c.image = image;
    double top = p->v[0][2];
    for (int i = 1; i < p->nv; i++)
        if (p->v[i][2] > top) top = p->v[i][2];
    double r = dist / p->radius;
    double clearance = (image[2] - top) / p->radius;
    int order = 0;
    if (clearance >= 0.5 || r >= 2.0)
        order = r >= 6.0 ? 4 : r >= 3.0 ? 5 : r >= 2.0 ? 6 : r >= 1.5 ? 8 : r >= 1.0 ? 10 : 0;
    if (order > 0) {
        double l = 0.0, ld = 0.0;
        for (int i = 0; i < order; i++)
            for (int j = 0; j < order; j++) {
                double xi[3], jac, psi, dpsi;
                bilinear((const double(*)[3])c.map, GL_X[order][i], GL_X[order][j], xi, &jac);
                psi_terms(xi, image, p->n, &psi, &dpsi);
                double ww = GL_W[order][i] * GL_W[order][j] * jac;
                l += ww * psi;
                ld += ww * dpsi;
            }
        *L = l;
        *Ld = ld;
        return;
    }
    double dmin = dist - p->radius;
    if (dmin < 1e-3 * p->radius) dmin = 1e-3 * p->radius;
    double scale = fabs(log(dist + p->radius)) + 1.0;
    c.tol_l = 1e-13 * p->area * scale;
    c.tol_d = 1e-13 * p->area / dmin;
    double whole[2], acc[2] = {0.0, 0.0};
    log_cell(&c, -1.0, 1.0, -1.0, 1.0, whole);
    log_adapt(&c, -1.0, 1.0, -1.0, 1.0, whole, 0, acc);
    *L = acc[0];
    *Ld = acc[1];
}

void hbo_log_singularity(const hbo_panel *p, const double image[3], double out[2]) {
    gl_init();
    log_singularity(p, image, &out[0], &out[1]);
}

/* panel_integrals.rs:625-648 log_in_plane */
double hbo_log_in_plane(const hbo_panel *p, const double *x) {
    int nv = p->nv;
    double sum = 0.0;
    for (int i = 0; i < nv; i++) {
        const double *a = p->v[i], *b = p->v[(i + 1) % nv];
        double ax[3], bx[3], e[3];
        sub3(a, x, ax);
        double h = dot3(ax, p->em[i]);
        if (h == 0.0) continue;
        for (int d = 0; d < 3; d++) e[d] = (1.0 / p->elen[i]) * (b[d] - a[d]);
        sub3(b, x, bx);
        double t1 = dot3(ax, e), t2 = dot3(bx, e);
        double q1 = h * h + t1 * t1, q2 = h * h + t2 * t2;
        double F1 = 0.5 * (t1 * log(q1) - 2.0 * t1 + 2.0 * h * atan(t1 / h)) - 0.5 * t1;
        double F2 = 0.5 * (t2 * log(q2) - 2.0 * t2 + 2.0 * h * atan(t2 / h)) - 0.5 * t2;
        sum += 0.5 * h * (F2 - F1);
    }
    return sum;
}

/* ------------------------------------------------------------------ statics (lo_static.rs) */
/* lo_static.rs:47-55 log_pair */
static inline int log_pair(const hbo_panel *p, const double *x, double tol) {
    double dx = x[0] - p->c[0], dy = x[1] - p->c[1], zz = fabs(x[2] + p->c[2]);
    double d = sqrt(dx * dx + dy * dy + zz * zz) + zz;
    return d * d * tol < 0.6 * p->radius * p->radius;
}

/* lo_static.rs:59-119 static_row (field point x against every panel); tiers: the panels' float32 Gauss
 * tiers in the production mode (rankine_pair = rankine_any at the point and its free-surface image),
 * NULL in the diagnostic mode */
static void static_row(int N, const hbo_panel *pg, const int32_t *kind, const double *x, int logint, double tol,
                       double depth, const float *tiers, double *row) {
    int finite = isfinite(depth) && depth > 0.0;
    double xb[3] = {x[0], x[1], -x[2]};
    double xp[6][3];
    if (finite) {
        double h = depth;
        double pts[6][3] = {{x[0], x[1], x[2]},           {x[0], x[1], -x[2] - 2.0 * h}, {x[0], x[1], -x[2]},
                            {x[0], x[1], x[2] + 2.0 * h}, {x[0], x[1], x[2] - 2.0 * h},  {x[0], x[1], -x[2] - 4.0 * h}};
        memcpy(xp, pts, sizeof pts);
    }
    for (int j = 0; j < N; j++) {
        const hbo_panel *p = pg + j;
        const float *tq = tiers ? tiers + (size_t)j * TIER_FLOATS : NULL;
        double s0, d0, sb, db;
        rankine_any(p, tq, x, &s0, &d0);
        rankine_any(p, tq, xb, &sb, &db);
        double sr = s0 + sb, dr = d0 + db;
        if (finite) {
            double s2, d2, s4, d4, s5, d5, s6, d6;
            rankine_any(p, tq, xp[1], &s2, &d2);
            rankine_any(p, tq, xp[3], &s4, &d4);
            rankine(p, xp[4], &s5, &d5);
            rankine(p, xp[5], &s6, &d6);
            sr += (s2 + s4) + s5 + s6;
            dr += (d2 + d4) + d5 + d6;
        }
        double *e = row + 4 * j;
        e[0] = sr;
        e[1] = dr;
        int use_log = logint && log_pair(p, x, tol);
        if (use_log && kind && kind[j] == HBO_INTERIOR && x[2] == 0.0) {
            double L = hbo_log_in_plane(p, x);
            double t[3];
            sub3(p->c, x, t);
            double Rr = norm3(t);
            e[2] = Rr > 0.0 ? L - p->area * log(Rr) : L;
            e[3] = 0.0;
        } else if (use_log) {
            double L, Ld, psi, dpsi;
            log_singularity(p, xb, &L, &Ld);
            psi_terms(p->c, xb, p->n, &psi, &dpsi);
            e[2] = L - p->area * psi;
            e[3] = Ld - p->area * dpsi;
        } else {
            e[2] = 0.0;
            e[3] = 0.0;
        }
        if (tiers)  /* production: the static rows are stored in float32 */
            for (int q = 0; q < 4; q++) e[q] = (double)(float)e[q];
    }
}

int hbo_statics(int N, const hbo_panel *pg, const int32_t *kind, double depth, int logint, double tol, double *out) {
    gl_init();
    float *tiers = NULL;
    if (g_prod) {
        tiers = (float *)malloc(sizeof(float) * TIER_FLOATS * (size_t)(N > 0 ? N : 1));
        if (!tiers) return 1;
#pragma omp parallel for schedule(static)
        for (int j = 0; j < N; j++) panel_tiers(pg + j, tiers + (size_t)j * TIER_FLOATS);
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < N; k++) static_row(N, pg, kind, pg[k].c, logint, tol, depth, tiers, out + (size_t)k * N * 4);
    free(tiers);
    return 0;
}

/* ------------------------------------------------------------------ infinite-depth wave kernel (green_inf.rs) */
/* green_inf.rs:58-73 table1d */
static void table1d(double X, double *r) {
    int i = (int)X;
    if (i >= XT) i = XT - 1;
    double t = 2.0 * (X - i) - 1.0;
    const double *c = T1D + (size_t)i * (N1 + 1) * 4;
    r[0] = r[1] = r[2] = r[3] = 0.0;
    for (int j = N1; j >= 0; j--)
        for (int f = 0; f < 4; f++) r[f] = r[f] * t + c[4 * j + f];
}

/* green_inf.rs:78-107 table2d: (V, V_X) */
static void table2d(double X, double Y, double *v, double *vx) {
    int ix = (int)X, iy = (int)Y;
    if (ix >= XT) ix = XT - 1;
    if (iy >= YT) iy = YT - 1;
    double tx = 2.0 * (X - ix) - 1.0, ty = 2.0 * (Y - iy) - 1.0;
    enum { M = N2 + 1 };
    const double *c = T2D + ((size_t)iy * XT + ix) * 2 * M * M;
    double s[2] = {0.0, 0.0};
    for (int q = 0; q < 2; q++) {
        const double *cq = c + q * M * M;
        double r[M];
        for (int a = 0; a < M; a++) r[a] = 0.0;
        for (int j = M - 1; j >= 0; j--)
            for (int a = 0; a < M; a++) r[a] = r[a] * tx + cq[j * M + a];
        for (int a = M - 1; a >= 0; a--) s[q] = s[q] * ty + r[a];
    }
    *v = s[0];
    *vx = s[1];
}

/* green_inf.rs:114-139 table2d_direct: the first nq of (F, F_X, c, c_X) (c = e^-Y J0) from the direct
 * tables of the production path, X < XT, Y < YT */
static void table2d_direct(double X, double Y, int nq, double *f) {
    int ix = (int)X, iy = (int)Y;
    double tx = 2.0 * (X - ix) - 1.0, ty = 2.0 * (Y - iy) - 1.0;
    enum { M = N3 + 1 };
    const double *c = T2DD + ((size_t)iy * XT + ix) * 4 * M * M;
    for (int q = 0; q < nq; q++) {
        const double *cq = c + q * M * M;
        double r[M];
        for (int a = 0; a < M; a++) r[a] = 0.0;
        for (int j = M - 1; j >= 0; j--)
            for (int a = 0; a < M; a++) r[a] = r[a] * tx + cq[j * M + a];
        double sq = 0.0;
        for (int a = M - 1; a >= 0; a--) sq = sq * ty + r[a];
        f[q] = sq;
    }
}

/* green_inf.rs:145-172 hankel01: (J0, Y0, J1, Y1) for x >= XT */
static void hankel01(double x, double *j0, double *y0, double *j1, double *y1) {
    double inv = 1.0 / x, inv2 = inv * inv;
    double P[2] = {0, 0}, Q[2] = {0, 0};
    for (int nu = 0; nu < 2; nu++) {
        const double *a = TASY + nu * HANKEL_TERMS;
        double pw = 1.0;
        for (int k = 0; 2 * k + 1 < HANKEL_TERMS; k++) {
            double s = (k % 2 != 0) ? -1.0 : 1.0;
            P[nu] += s * a[2 * k] * pw;
            Q[nu] += s * a[2 * k + 1] * pw * inv;
            pw *= inv2;
        }
    }
    double chi = x - 0.25 * PI;
    double sq = sqrt(2.0 / (PI * x));
    double c = cos(chi), sn = sin(chi);
    *j0 = sq * (P[0] * c - Q[0] * sn);
    *y0 = sq * (P[0] * sn + Q[0] * c);
    *j1 = sq * (P[1] * sn + Q[1] * c);
    *y1 = sq * (-P[1] * c + Q[1] * sn);
}

/* green_inf.rs:175-187 struve_minus_y */
static double struve_minus_y(int nu, double x) {
    const double *c = TASY + 2 * HANKEL_TERMS + nu * STRUVE_TERMS;
    double inv2 = 1.0 / (x * x), s = 0.0, pw = nu == 0 ? 1.0 / x : 1.0;
    for (int k = 0; k < STRUVE_TERMS; k++) {
        s += c[k] * pw;
        pw *= inv2;
    }
    return s;
}

/* green_inf.rs:189-266 partial integration of Havelock's integral */
#define FAR_TERMS 15
#define FAR_TOL 1e-14
static void taylor_sum(double X, double t0, double *P, double *PX) {
    double A = X * X + t0 * t0, ia = 1.0 / A, ir = sqrt(ia);
    double a = ir, b = -X * ir * ia, am1 = 0.0, bm1 = 0.0, fact = 1.0, size = ir;
    double p = a, px = b;
    for (int n = 0; n + 1 < FAR_TERMS; n++) {
        double an = a, bn = b, nf = n, k = 2 * n + 1;
        double invn = 1.0 / (double)(n + 1);
        a = -(k * t0 * an + nf * am1) * ia * invn;
        b = -(k * t0 * bn + nf * bm1) * ia * invn - a * 2.0 * X * ia;
        am1 = an;
        bm1 = bn;
        fact *= (n + 1);
        size *= (n + 1) * ir;
        double s = (n % 2 != 0) ? fact : -fact;
        p += s * a;
        px += s * b;
        if (size < FAR_TOL) break;
    }
    *P = p;
    *PX = px;
}

static void far_series(double X, double Y, double w, double *P, double *PX) {
    taylor_sum(X, Y, P, PX);
    if (w > 1e-17) {
        double P0, PX0;
        taylor_sum(X, 0.0, &P0, &PX0);
        *P -= w * P0;
        *PX -= w * PX0;
    }
}

/* green_inf.rs:287-296 bessel_j01 */
static void bessel_j01(double X, double *j0, double *j1) {
    if (X < XT) {
        double f[4];
        table1d(X, f);
        *j0 = f[0];
        *j1 = f[1];
    } else {
        double y0, y1;
        hankel01(X, j0, &y0, j1, &y1);
    }
}

/* green_inf.rs:298-312 bessel_jy01 */
static void bessel_jy01(double X, double *j0, double *y0, double *j1, double *y1) {
    if (X >= XT) {
        hankel01(X, j0, y0, j1, y1);
        return;
    }
    double f[4];
    table1d(X, f);
    *j0 = f[0];
    *j1 = f[1];
    double L = log(0.5 * X) + GAMMA;
    *y0 = f[2] + 2.0 / PI * L * f[0];
    *y1 = -f[3] - 2.0 / PI * (f[0] / X - L * f[1]);
}

/* green_inf.rs:316-368 wave_kernel, diagnostic mode (no direct 2D tables):
 * out = F, FX, FY, I, IX, IY, c */
void hbo_wave_kernel(double X, double Y, double *out) {
    double R0 = sqrt(X * X + Y * Y);
    if (g_prod && X < XT && Y < YT && (X >= 2.0 || Y >= 2.0)) {  /* green_inf.rs:319-330 */
        double f[4];
        table2d_direct(X, Y, 4, f);
        out[0] = f[0];
        out[1] = f[1];
        out[2] = -f[0] - 2.0 / R0;
        out[6] = f[2];
        out[3] = -2.0 * PI * f[2];
        out[4] = 2.0 * PI * f[3];
        out[5] = -out[3];
        return;
    }
    double eY = exp(-Y), j0, j1, F, FX;
    if (X < XT && Y < YT) {
        double f[4], v, vx;
        table1d(X, f);
        j0 = f[0];
        j1 = f[1];
        table2d(X, Y, &v, &vx);
        double lg = log(Y + R0) + (GAMMA - LOG2);
        F = -2.0 * eY * j0 * lg - PI * eY * f[2] - 2.0 * R0 * v;
        FX = 2.0 * eY * j1 * lg - 2.0 * eY * j0 * X / (R0 * (Y + R0)) - PI * eY * f[3] - 2.0 * (X / R0) * v -
             2.0 * R0 * vx;
    } else if (Y >= YT) {
        bessel_j01(X, &j0, &j1);
        double P, PX;
        far_series(X, Y, 0.0, &P, &PX);
        F = -2.0 * P;
        FX = -2.0 * PX;
    } else {
        double y0, y1;
        hankel01(X, &j0, &y0, &j1, &y1);
        double h0py0 = struve_minus_y(0, X) + 2.0 * y0;
        double dh0py0 = 2.0 / PI - struve_minus_y(1, X) - 2.0 * y1;
        double P, PX;
        far_series(X, Y, eY, &P, &PX);
        F = -PI * eY * h0py0 - 2.0 * P;
        FX = -PI * eY * dh0py0 - 2.0 * PX;
    }
    out[0] = F;
    out[1] = FX;
    out[2] = -F - 2.0 / R0;
    out[6] = eY * j0;
    out[3] = -2.0 * PI * eY * j0;
    out[4] = 2.0 * PI * eY * j1;
    out[5] = -out[3];
}

/* green_inf.rs:657-675 wave_real (the direct tables first in the production mode) */
static void wave_real(double X, double Y, double *F, double *FX, double *FY) {
    double R0 = sqrt(X * X + Y * Y);
    if (g_prod && X < XT && Y < YT && (X >= 2.0 || Y >= 2.0)) {
        double f[2];
        table2d_direct(X, Y, 2, f);
        *F = f[0];
        *FX = f[1];
    } else if (Y >= YT) {
        double P, PX;
        far_series(X, Y, 0.0, &P, &PX);
        *F = -2.0 * P;
        *FX = -2.0 * PX;
    } else {
        double w[7];
        hbo_wave_kernel(X, Y, w);
        *F = w[0];
        *FX = w[1];
    }
    *FY = -*F - 2.0 / R0;
}

/* ------------------------------------------------------------------ dispersion (dispersion.rs) */
/* dispersion.rs:19-52 */
double hbo_dispersion_x0(double H) {
    if (!(H > 0.0)) return 0.0;
    if (H >= 40.0) return H;
    double lo = H > sqrt(H) ? H : sqrt(H);
    double hi = 0.5 * (H + sqrt(H * H + 4.0 * H));
    double x = H < 1.0 ? sqrt(H) * (1.0 + H / 6.0) : H;
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    double prev = -1.0;
    for (int it = 0; it < 200; it++) {
        double t = tanh(x), f = x * t - H;
        if (f < 0.0) lo = x;
        else hi = x;
        double fp = t + x * (1.0 - t * t);
        double xn = x - f / fp;
        if (!(xn >= lo && xn <= hi)) xn = 0.5 * (lo + hi);
        if (xn == x || xn == prev) break;
        prev = x;
        x = xn;
    }
    return x;
}

/* dispersion.rs:62-95 */
double hbo_dispersion_xn(double H, int n) {
    double npi = n * PI;
    if (!(H > 0.0)) return npi;
    if (isinf(H)) return npi - 0.5 * PI;
    double lo = 0.0, hi = 0.5 * PI;
    double d = atan(H / (npi - 0.25 * PI)), prev = -1.0;
    for (int it = 0; it < 200; it++) {
        double s = sin(d), c = cos(d);
        double g = (npi - d) * s - H * c;
        if (g < 0.0) lo = d;
        else hi = d;
        double gp = (npi - d) * c + (H - 1.0) * s;
        double dn = d - g / gp;
        if (!(dn > lo && dn < hi)) dn = 0.5 * (lo + hi);
        if (dn == d || dn == prev) break;
        prev = d;
        d = dn;
    }
    return npi - d;
}

/* ------------------------------------------------------------------ finite depth (green_fin.rs) */
#define FIN_ROOTS 24
#define SERIES_STOP 18.0
#define TS 8
#define TW 8
#define TV 16
#define TD 5
#define TN (TD + 1)
#define XMAX 0.5

typedef struct {
    int mode; /* 0 ordinary, 1 zero, 2 infinite */
    double h, K, H, k0, A0;
    double sign[6];
    double kn[FIN_ROOTS], cn[FIN_ROOTS];
    double P[(FM + 1) * NC];
    double T1[TS * TW * 3 * TN * TN];
    double T2[TS * TV * 3 * TN * TN];
} fdepth;

typedef struct {
    double d, a, b, c;
    double cs[2 * FIN_ROOTS];
} finpoint;

/* quadrature.rs:120-160: Chebyshev power basis T_j(t) = sum_k a[j][k] t^k */
static void cheb_power_basis(int n, double *a) {
    memset(a, 0, sizeof(double) * n * n);
    a[0] = 1.0;
    a[1 * n + 1] = 1.0;
    for (int j = 2; j < n; j++)
        for (int k = 0; k < n; k++) a[j * n + k] = (k > 0 ? 2.0 * a[(j - 1) * n + k - 1] : 0.0) - a[(j - 2) * n + k];
}

/* green_fin.rs:361-382 region_coefficients */
static void region_coefficients(int r, double x, double *cw) {
    const double *meta = TMETA + 5 * r;
    double a = meta[1], b = meta[2];
    int n = (int)meta[3];
    const double *c = TQ + (size_t)meta[4];
    double y = 2.0 * (x - a) / (b - a) - 1.0;
    double Tx[64];
    Tx[0] = 1.0;
    Tx[1] = y;
    for (int j = 2; j <= n; j++) Tx[j] = 2.0 * y * Tx[j - 1] - Tx[j - 2];
    for (int m = 0; m <= FM; m++)
        for (int jw = 0; jw < NC; jw++) {
            double s = 0.0;
            for (int jx = 0; jx <= n; jx++) s += c[(m * (n + 1) + jx) * NC + jw] * Tx[jx];
            cw[m * NC + jw] = s;
        }
}

/* green_fin.rs:345-358, 385-392 cheb_to_power / power_table */
static void power_table(const double *cw, double *P) {
    double a[NC * NC];
    cheb_power_basis(NC, a);
    for (int m = 0; m <= FM; m++) {
        const double *c = cw + m * NC;
        double *p = P + m * NC;
        for (int k = 0; k < NC; k++) p[k] = c[0] * a[0 * NC + k] + c[1] * a[1 * NC + k];
        for (int j = 2; j < NC; j++)
            for (int k = 0; k < NC; k++) p[k] += c[j] * a[j * NC + k];
    }
}

/* green_fin.rs:394-421 q_eval2: (Q, dQ/ds, dQ/dw) at w1 and w2 */
static void q_eval2(const double *P, double s, double w1, double w2, double *v, double *vs, double *qw) {
    double y[2] = {0.5 * w1 - 1.0, 0.5 * w2 - 1.0};
    double vy[2] = {0, 0};
    v[0] = v[1] = vs[0] = vs[1] = 0.0;
    for (int m = FM; m >= 0; m--) {
        const double *c = P + m * NC;
        double p[2] = {c[NC - 1], c[NC - 1]}, dp[2] = {0, 0};
        for (int k = NC - 2; k >= 0; k--)
            for (int i = 0; i < 2; i++) {
                dp[i] = dp[i] * y[i] + p[i];
                p[i] = p[i] * y[i] + c[k];
            }
        for (int i = 0; i < 2; i++) {
            vs[i] = vs[i] * s + v[i];
            v[i] = v[i] * s + p[i];
            vy[i] = vy[i] * s + dp[i];
        }
    }
    qw[0] = 0.5 * vy[0];
    qw[1] = 0.5 * vy[1];
}

/* green_fin.rs:425-446 scaled_k01: (e^x sqrt(x) K0, e^x sqrt(x) K1) */
static void scaled_k01(double x, double *g0, double *g1) {
    int i;
    double t;
    if (x < 1.0) {
        i = 0;
        t = 2.0 * (x - K_LO) / (1.0 - K_LO) - 1.0;
    } else {
        i = (int)x;
        t = 2.0 * (x - i) - 1.0;
    }
    const double *c = TBK + (size_t)i * (NK + 1) * 2;
    double a0 = 0.0, a1 = 0.0;
    for (int j = NK; j >= 0; j--) {
        a0 = a0 * t + c[2 * j];
        a1 = a1 * t + c[2 * j + 1];
    }
    *g0 = a0;
    *g1 = a1;
}

/* green_fin.rs:461-491 phi_direct */
static void phi_direct(const fdepth *fd, int which, double xb, double vb, double *out) {
    double q[2], qs[2], qw[2];
    q_eval2(fd->P, xb * xb, vb * vb, vb * vb, q, qs, qw);
    out[0] = q[0];
    out[1] = 2.0 * xb * qs[0];
    out[2] = 2.0 * vb * qw[0];
    if (fd->mode != 0) return;
    double H = fd->H, X = H * xb, H2 = H * H, F, FX, FY;
    if (which == 1) {
        wave_real(X, H * (2.0 - vb), &F, &FX, &FY);
        out[0] += H * F;
        out[1] += H2 * FX;
        out[2] -= H2 * FY;
        wave_real(X, H * (2.0 + vb), &F, &FX, &FY);
        out[0] += H * F;
        out[1] += H2 * FX;
        out[2] += H2 * FY;
    } else {
        wave_real(X, H * (2.0 + vb), &F, &FX, &FY);
        out[0] += H * F;
        out[1] += H2 * FX;
        out[2] += H2 * FY;
    }
}

/* green_fin.rs:493-564 build_tiles */
static void build_tiles(fdepth *fd) {
    enum { N = TN };
    double t[N], a[N * N], cs[N][N];
    for (int i = 0; i < N; i++) t[i] = cos(PI * (i + 0.5) / N);
    cheb_power_basis(N, a);
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) cs[j][i] = cos(PI * j * (i + 0.5) / N);
    for (int which = 1; which <= 2; which++) {
        int ny = which == 1 ? TW : TV;
        double ymax = which == 1 ? 1.0 : 2.0;
        double *out = which == 1 ? fd->T1 : fd->T2;
        memset(out, 0, sizeof(double) * TS * ny * 3 * N * N);
        double dx = XMAX / TS, dy = ymax / ny;
        for (int ix = 0; ix < TS; ix++)
            for (int iy = 0; iy < ny; iy++) {
                double f[3][N][N];
                for (int i = 0; i < N; i++)
                    for (int j = 0; j < N; j++) {
                        double v[3];
                        phi_direct(fd, which, dx * (ix + 0.5 * (t[i] + 1.0)), dy * (iy + 0.5 * (t[j] + 1.0)), v);
                        for (int q = 0; q < 3; q++) f[q][i][j] = v[q];
                    }
                for (int q = 0; q < 3; q++) {
                    double c[N][N];
                    for (int ji = 0; ji < N; ji++)
                        for (int jj = 0; jj < N; jj++) {
                            double acc = 0.0;
                            for (int i = 0; i < N; i++)
                                for (int j = 0; j < N; j++) acc += f[q][i][j] * cs[ji][i] * cs[jj][j];
                            c[ji][jj] = acc * (ji != 0 ? 2.0 : 1.0) * (jj != 0 ? 2.0 : 1.0) / (double)(N * N);
                        }
                    double *pw = out + ((size_t)(ix * ny + iy) * 3 + q) * N * N;
                    for (int ji = 0; ji < N; ji++)
                        for (int jj = 0; jj < N; jj++)
                            for (int ki = 0; ki <= ji; ki++)
                                for (int kj = 0; kj <= jj; kj++) pw[ki * N + kj] += c[ji][jj] * a[ji * N + ki] * a[jj * N + kj];
                }
            }
    }
}

/* green_fin.rs:566-600 tile_of / phi_tiles */
static void phi_tiles(const fdepth *fd, int which, double xb, double vb, double *v) {
    enum { N = TN };
    int ny = which == 1 ? TW : TV;
    double ymax = which == 1 ? 1.0 : 2.0;
    double ux = xb * (TS / XMAX), uy = vb * (ny / ymax);
    int ix = (int)ux, iy = (int)uy;
    if (ix > TS - 1) ix = TS - 1;
    if (iy > ny - 1) iy = ny - 1;
    double tx = 2.0 * (ux - ix) - 1.0, ty = 2.0 * (uy - iy) - 1.0;
    const double *c = (which == 1 ? fd->T1 : fd->T2) + (size_t)(ix * ny + iy) * 3 * N * N;
    v[0] = v[1] = v[2] = 0.0;
    for (int i = N - 1; i >= 0; i--)
        for (int q = 0; q < 3; q++) {
            const double *r = c + q * N * N + i * N;
            double p = r[N - 1];
            for (int j = N - 2; j >= 0; j--) p = p * ty + r[j];
            v[q] = v[q] * tx + p;
        }
}

/* green_fin.rs:874-934 make_finite_depth (tiles on) */
static void make_finite_depth(fdepth *fd, double h, double K, int mode) {
    memset(fd, 0, sizeof *fd);
    fd->mode = mode;
    fd->h = h;
    for (int p = 0; p < 6; p++) fd->sign[p] = 1.0;
    double cw[(FM + 1) * NC];
    if (mode == 1) {
        for (int n = 1; n <= FIN_ROOTS; n++) {
            fd->kn[n - 1] = n * PI / h;
            fd->cn[n - 1] = 4.0 / h;
        }
        memcpy(cw, TL0, sizeof cw);
        power_table(cw, fd->P);
        build_tiles(fd);
        return;
    }
    if (mode == 2) {
        double sg[6] = {1, 1, -1, -1, -1, -1};
        memcpy(fd->sign, sg, sizeof sg);
        for (int n = 1; n <= FIN_ROOTS; n++) {
            fd->kn[n - 1] = (n - 0.5) * PI / h;
            fd->cn[n - 1] = 4.0 / h;
        }
        region_coefficients(REGIONS - 1, 0.0, cw);
        power_table(cw, fd->P);
        build_tiles(fd);
        return;
    }
    fd->K = K;
    fd->H = K * h;
    double x0 = hbo_dispersion_x0(fd->H);
    fd->k0 = x0 / h;
    fd->A0 = 2.0 * PI * fd->k0 / (-expm1(-4.0 * x0) + 4.0 * x0 * exp(-2.0 * x0));
    for (int n = 1; n <= FIN_ROOTS; n++) {
        double k = hbo_dispersion_xn(fd->H, n) / h;
        fd->kn[n - 1] = k;
        fd->cn[n - 1] = 4.0 * (k * k + K * K) / (k * k * h + K * K * h - K);
    }
    if (fd->H < H_MIN) {
        memcpy(cw, TL0, sizeof cw);
        cw[0] -= 0.5 * log(fd->H);
    } else if (fd->H >= HC) {
        region_coefficients(REGIONS - 1, 1.0 / fd->H, cw);
    } else {
        double tau = log(fd->H);
        int r = 0;
        while (r + 2 < REGIONS && tau > TMETA[5 * r + 2]) r++;
        region_coefficients(r, tau, cw);
    }
    power_table(cw, fd->P);
    build_tiles(fd);
}

/* green_fin.rs:937-952 fin_point */
static void fin_point(const fdepth *fd, double z, finpoint *p) {
    double h = fd->h, k0 = fd->k0;
    p->d = p->a = p->b = p->c = 0.0;
    if (fd->mode == 0) {
        p->d = exp(k0 * z);
        p->a = exp(-k0 * (z + h));
        p->b = exp(-k0 * (h - z));
        p->c = exp(-k0 * (z + 2.0 * h));
    }
    for (int n = 0; n < FIN_ROOTS; n++) {
        p->cs[2 * n] = cos(fd->kn[n] * (z + h));
        p->cs[2 * n + 1] = sin(fd->kn[n] * (z + h));
    }
}

/* green_fin.rs:803-808 wave_real_or_limit */
static void wave_real_or_limit(double K, double R, double v3, double *F, double *FX, double *FY) {
    if (R == 0.0 && v3 == 0.0) {
        *F = -2.0 * (GAMMA - LOG2 + log(K));
        *FX = 0.0;
        *FY = 0.0;
    } else
        wave_real(K * R, K * v3, F, FX, FY);
}

/* green_fin.rs:1007-1095 finite_kernel (tiled integral form or series form) with optional fin points */
static void finite_kernel(const fdepth *fd, double R, double z, double zeta, const finpoint *pz, const finpoint *pzeta,
                          double *o) {
    double h = fd->h;
    double d1 = z - zeta;
    double sg = d1 > 0.0 ? 1.0 : d1 < 0.0 ? -1.0 : 0.0;
    double v[6] = {fabs(d1), z + zeta + 2.0 * h, -(z + zeta), d1 + 2.0 * h, -d1 + 2.0 * h, z + zeta + 4.0 * h};
    int ordinary = fd->mode == 0;
    double e[4] = {0, 0, 0, 0};
    if (ordinary) {
        double e3, e4, e5, e6;
        if (pz && pzeta) {
            e3 = pz->d * pzeta->d;
            e4 = pz->a * pzeta->b;
            e5 = pz->b * pzeta->a;
            e6 = pz->c * pzeta->c;
        } else {
            e3 = exp(-fd->k0 * v[2]);
            e4 = exp(-fd->k0 * v[3]);
            e5 = exp(-fd->k0 * v[4]);
            e6 = exp(-fd->k0 * v[5]);
        }
        e[0] = e3 + e4 + e5 + e6;
        e[1] = fd->k0 * (e3 + e4 - e5 - e6);
        e[2] = fd->k0 * (e3 - e4 + e5 - e6);
        e[3] = fd->k0 * fd->k0 * (e3 - e4 - e5 + e6);
    }
    memset(o, 0, 8 * sizeof(double));
    if (R >= 0.5 * h) {
        /* series_form (green_fin.rs:247-322) */
        double re = 0, reR = 0, reZ = 0, rez = 0;
        for (int n = 0; n < FIN_ROOTS; n++) {
            double k = fd->kn[n], x = k * R;
            if (x >= SERIES_STOP) break;
            double g0, g1;
            scaled_k01(x, &g0, &g1);
            double ex = exp(-x) / sqrt(x);
            double K0 = g0 * ex, K1 = g1 * ex;
            double cz, sz, cs, ss;
            if (pz && pzeta) {
                cz = pz->cs[2 * n];
                sz = pz->cs[2 * n + 1];
                cs = pzeta->cs[2 * n];
                ss = pzeta->cs[2 * n + 1];
            } else {
                cz = cos(k * (z + h));
                sz = sin(k * (z + h));
                cs = cos(k * (zeta + h));
                ss = sin(k * (zeta + h));
            }
            double c = fd->cn[n];
            re += c * cz * cs * K0;
            reR -= c * cz * cs * k * K1;
            reZ -= c * cz * k * ss * K0;
            rez -= c * k * sz * cs * K0;
        }
        if (ordinary) {
            double j0, y0, j1, y1;
            bessel_jy01(fd->k0 * R, &j0, &y0, &j1, &y1);
            re += -fd->A0 * e[0] * y0;
            reR += fd->A0 * e[0] * fd->k0 * y1;
            reZ += -fd->A0 * e[1] * y0;
            rez += -fd->A0 * e[2] * y0;
            o[4] = -fd->A0 * e[0] * j0;
            o[5] = fd->A0 * e[0] * fd->k0 * j1;
            o[6] = -fd->A0 * e[1] * j0;
            o[7] = -fd->A0 * e[2] * j0;
        } else if (fd->mode == 1) {
            re += -2.0 / h * (log(R / (2.0 * h)) + GAMMA);
            reR += -2.0 / (h * R);
        }
        double dvz[6] = {-sg, 1.0, -1.0, -1.0, 1.0, 1.0};
        double dvf[6] = {sg, 1.0, -1.0, 1.0, -1.0, 1.0};
        for (int p = 0; p < 6; p++) {
            double r2 = R * R + v[p] * v[p], r = sqrt(r2);
            double ir3 = fd->sign[p] / (r2 * r);
            re -= fd->sign[p] / r;
            reR += R * ir3;
            reZ += v[p] * dvz[p] * ir3;
            rez += v[p] * dvf[p] * ir3;
        }
        o[0] = re;
        o[1] = reR;
        o[2] = reZ;
        o[3] = rez;
        return;
    }
    double ih = 1.0 / h, ih2 = ih * ih, f1[3], f2[3];
    phi_tiles(fd, 1, R * ih, v[0] * ih, f1);
    phi_tiles(fd, 2, R * ih, v[1] * ih, f2);
    o[0] = ih * (f1[0] + f2[0]);
    o[1] = ih2 * (f1[1] + f2[1]);
    double A1z = -sg * ih2 * f1[2], Bz = ih2 * f2[2];
    if (ordinary) {
        double K = fd->K, F3, F3X, F3Y;
        wave_real_or_limit(K, R, v[2], &F3, &F3X, &F3Y);
        o[0] += K * F3;
        o[1] += K * K * F3X;
        Bz -= K * K * F3Y;
        double j0, j1;
        bessel_j01(fd->k0 * R, &j0, &j1);
        o[4] = -fd->A0 * e[0] * j0;
        o[5] = fd->A0 * e[0] * fd->k0 * j1;
        o[6] = -fd->A0 * e[1] * j0;
        o[7] = -fd->A0 * e[2] * j0;
    }
    o[2] = A1z + Bz;
    o[3] = -A1z + Bz;
}

void hbo_finite_kernel(double h, double K, int mode, double R, double z, double zeta, double *out) {
    fdepth *fd = (fdepth *)malloc(sizeof(fdepth));
    make_finite_depth(fd, h, K, mode);
    finite_kernel(fd, R, z, zeta, NULL, NULL, out);
    free(fd);
}

/* ------------------------------------------------------------------ assembly (lo_frequency.rs, low_order.rs) */
double hbo_wavenumber(double omega, double depth, double grav) {
    double K = omega * omega / grav;
    if (isfinite(depth) && depth > 0.0) return hbo_dispersion_x0(K * depth) / depth;
    return K;
}

/* low_order.rs:627-648 pair_kernel and 717-730 wave_kern (infinite depth):
 * kern = Wr WrR WrZ Wrz Wi WiR WiZ Wiz */
static void pair_kernel_inf(double K, const double *x, const double *xi, double *k, double *Rout) {
    double dx = x[0] - xi[0], dy = x[1] - xi[1];
    double R = sqrt(dx * dx + dy * dy);
    *Rout = R;
    memset(k, 0, 8 * sizeof(double));
    if (R == 0.0 && x[2] == 0.0 && xi[2] == 0.0) {
        k[0] = -2.0 * K * (GAMMA - LOG2 + log(K));
        k[4] = -2.0 * PI * K;
        return;
    }
    double w[7];
    hbo_wave_kernel(K * R, -K * (x[2] + xi[2]), w);
    double K2 = K * K;
    k[0] = K * w[0];
    k[1] = K2 * w[1];
    k[2] = -K2 * w[2];
    k[3] = k[2];
    k[4] = K * w[3];
    k[5] = K2 * w[4];
    k[6] = -K2 * w[5];
    k[7] = k[6];
}

/* low_order.rs:738-769 apply_kernel + 781-790 kind_column: (S, D column) of panel j at x */
static void apply_kernel(const hbo_panel *p, int kindj, const double *st, const double *x, double K, double logc,
                         const double *k, double R, int swapped, double *S, double *D) {
    double a = R > 0.0 ? ((x[0] - p->c[0]) * p->n[0] + (x[1] - p->c[1]) * p->n[1]) / R : 0.0;
    double A = p->area;
    double rz = swapped ? k[3] : k[2];
    double iz = swapped ? k[7] : k[6];
    S[0] = st[0] + A * k[0] - 2.0 * K * logc * st[2];
    S[1] = A * k[4];
    D[0] = st[1] + A * (-k[1] * a + rz * p->n[2]) - 2.0 * K * logc * st[3];
    D[1] = A * (-k[5] * a + iz * p->n[2]);
    if (kindj == HBO_INTERIOR) {
        D[0] = K * S[0];
        D[1] = K * S[1];
    }
}

/* lo_frequency.rs:74-84 free_term */
static double free_term(int kind) { return kind == HBO_INTERIOR ? -4.0 * PI : 2.0 * PI; }

static void put_entry(double *M, float *M32, size_t o, double re, double im) {
    if (M32) {
        M32[2 * o] = (float)re;
        M32[2 * o + 1] = (float)im;
    } else {
        M[2 * o] = re;
        M[2 * o + 1] = im;
    }
}

static int assemble_into(int N, const hbo_panel *pg, const int32_t *kind, const double *statics, double depth,
                         double omega, double grav, int logint, double *S, double *A, float *S32, float *A32);

int hbo_assemble(int N, const hbo_panel *pg, const int32_t *kind, const double *statics, double depth, double omega,
                 double grav, int logint, double *S, double *A) {
    return assemble_into(N, pg, kind, statics, depth, omega, grav, logint, S, A, NULL, NULL);
}

int hbo_assemble_c64(int N, const hbo_panel *pg, const int32_t *kind, const double *statics, double depth,
                     double omega, double grav, int logint, float *S, float *A) {
    return assemble_into(N, pg, kind, statics, depth, omega, grav, logint, NULL, NULL, S, A);
}

static int assemble_into(int N, const hbo_panel *pg, const int32_t *kind, const double *statics, double depth,
                         double omega, double grav, int logint, double *S, double *A, float *S32, float *A32) {
    double K = omega * omega / grav;
    double logc = logint ? 1.0 : 0.0;
    int finite = isfinite(depth) && depth > 0.0;
    fdepth *fd = NULL;
    finpoint *fpt = NULL;
    if (finite) {
        fd = (fdepth *)malloc(sizeof(fdepth));
        make_finite_depth(fd, depth, K, 0);
        fpt = (finpoint *)malloc(sizeof(finpoint) * N);
        for (int j = 0; j < N; j++) fin_point(fd, pg[j].c[2], fpt + j);
    }
    /* every unordered pair once: G(x, xi) = G(xi, x), the swapped source derivative for (n, k)
     * (lo_frequency.rs:399-537, G = 1) */
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < N; k++) {
        const double *xk = pg[k].c;
        int kk = kind ? kind[k] : HBO_WET;
        for (int n = k; n < N; n++) {
            const double *xn = pg[n].c;
            int kn = kind ? kind[n] : HBO_WET;
            double w[8], R;
            if (finite) {
                double dx = xk[0] - xn[0], dy = xk[1] - xn[1];
                R = sqrt(dx * dx + dy * dy);
                finite_kernel(fd, R, xk[2], xn[2], fpt + k, fpt + n, w);
            } else {
                pair_kernel_inf(K, xk, xn, w, &R);
            }
            double s1[2], d1[2];
            apply_kernel(pg + n, kn, statics + ((size_t)k * N + n) * 4, xk, K, logc, w, R, 0, s1, d1);
            size_t o = (size_t)k + (size_t)n * N;
            put_entry(S, S32, o, s1[0], s1[1]);
            put_entry(A, A32, o, (k == n ? free_term(kk) : 0.0) - d1[0], -d1[1]);
            if (n != k) {
                double s2[2], d2[2];
                apply_kernel(pg + k, kk, statics + ((size_t)n * N + k) * 4, xn, K, logc, w, R, 1, s2, d2);
                size_t o2 = (size_t)n + (size_t)k * N;
                put_entry(S, S32, o2, s2[0], s2[1]);
                put_entry(A, A32, o2, -d2[0], -d2[1]);
            }
        }
    }
    free(fd);
    free(fpt);
    return 0;
}

/* lo_frequency.rs:1392-1470 field_values, the influence rows of the field points: (S, D column) of every
 * panel j at every point x_p (the static row of the point, lo_static.rs:59-119, then the pair kernel and
 * apply_kernel as for a collocation point); S, D [P][N] complex as (re, im) pairs. */
int hbo_field_influence(int N, const hbo_panel *pg, const int32_t *kind, int P, const double *pts, double depth,
                        double omega, double grav, int logint, double tol, double *S, double *D) {
    gl_init();
    double K = omega * omega / grav;
    double logc = logint ? 1.0 : 0.0;
    int finite = isfinite(depth) && depth > 0.0;
    fdepth *fd = NULL;
    finpoint *fpt = NULL;
    if (finite) {
        fd = (fdepth *)malloc(sizeof(fdepth));
        make_finite_depth(fd, depth, K, 0);
        fpt = (finpoint *)malloc(sizeof(finpoint) * N);
        for (int j = 0; j < N; j++) fin_point(fd, pg[j].c[2], fpt + j);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int p = 0; p < P; p++) {
        const double *x = pts + 3 * p;
        double *row = (double *)malloc(sizeof(double) * 4 * N);
        static_row(N, pg, kind, x, logint, tol, depth, NULL, row);
        finpoint fx;
        if (finite) fin_point(fd, x[2], &fx);
        for (int j = 0; j < N; j++) {
            double w[8], R;
            if (finite) {
                double dx = x[0] - pg[j].c[0], dy = x[1] - pg[j].c[1];
                R = sqrt(dx * dx + dy * dy);
                finite_kernel(fd, R, x[2], pg[j].c[2], &fx, fpt + j, w);
            } else {
                pair_kernel_inf(K, x, pg[j].c, w, &R);
            }
            double s[2], d[2];
            apply_kernel(pg + j, kind ? kind[j] : HBO_WET, row + 4 * (size_t)j, x, K, logc, w, R, 0, s, d);
            size_t o = (size_t)p * N + j;
            S[2 * o] = s[0];
            S[2 * o + 1] = s[1];
            D[2 * o] = d[0];
            D[2 * o + 1] = d[1];
        }
        free(row);
    }
    free(fd);
    free(fpt);
    return 0;
}
