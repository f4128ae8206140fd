// hbg_statics.cu -- panel geometry and the frequency-independent influence data (FP64).
//
// Geometry: one thread per panel (geometry.rs:120-199 make_panel, panel_integrals.rs:145-217
// make_panel_geom).  Statics: one thread per (row k, panel j) pair computes the Rankine source and
// dipole of 1/r + 1/r' (finite depth: the six image terms) by the closed forms of
// panel_integrals.rs:226-275 and the log-singularity corrections dl, dd of lo_static.rs:99-117.
// Pairs whose log integral needs the adaptive rule (image within 2 radii and less than half a
// radius above the panel, panel_integrals.rs:407-449) are appended to a worklist and integrated by
// a second kernel with an explicit depth-first stack, in the reference's cell order.
//
// Layout: statics planes [4][N*N] (rs, rd, dl, dd), entry (k, j) at k + j*N (column-major, the
// layout of the matrices the assembly writes), so a warp of consecutive rows k writes coalesced.
//
// This file is its own translation unit, compiled without floating-point contraction (-fmad=false):
// the reference picks closed forms, Gauss orders and the adaptive rule by thresholds on geometric
// ratios (distance over panel radius, clearance, log_pair), which regular meshes put exactly on
// the thresholds; with the same IEEE operations in the same order as the reference, every such
// decision (and every geometric quantity) is the reference's to the bit.
#include "hbg_device.cuh"
#include "hbg_internal.h"

namespace hbg {

constexpr double COINCIDENCE_TOL = 1e-6;
constexpr double CONVEXITY_TOL = 1e-6;

__device__ __forceinline__ void bilinear(const double vt[4][3], double u, double v, double* x, double& jac) {
    double n0 = 0.25 * (1.0 - u) * (1.0 - v), n1 = 0.25 * (1.0 + u) * (1.0 - v);
    double n2 = 0.25 * (1.0 + u) * (1.0 + v), n3 = 0.25 * (1.0 - u) * (1.0 + v);
    double xu[3], xv[3], cr[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        x[d] = n0 * vt[0][d] + n1 * vt[1][d] + n2 * vt[2][d] + n3 * vt[3][d];
        xu[d] = (0.25 * (1.0 - v)) * (vt[1][d] - vt[0][d]) + (0.25 * (1.0 + v)) * (vt[2][d] - vt[3][d]);
        xv[d] = (0.25 * (1.0 - u)) * (vt[3][d] - vt[0][d]) + (0.25 * (1.0 + u)) * (vt[2][d] - vt[1][d]);
    }
    cross3(xu, xv, cr);
    jac = norm3(cr);
}

// ------------------------------------------------------------------ geometry
// The reference's production rule of the Rankine integrals (panel_integrals.rs:190-216, 288-363): per
// panel the float32 Gauss tiers of orders 3, 4, 5, 6 (points of the bilinear map relative to the
// centroid, weights scaled to the exact area), each block padded with zero weights to a multiple of 8:
// tier_len(t) points at tier_off(t), planes x, y, z, w of tier_len(t) floats each.
constexpr int TIER_FLOATS = 416;
static_assert(TIER_FLOATS == TIER_FLOATS_HOST, "the host's tier buffer size");
__device__ __forceinline__ int tier_off(int t) { return t == 0 ? 0 : t == 1 ? 64 : t == 2 ? 128 : 256; }
__device__ __forceinline__ int tier_len(int t) { return t <= 1 ? 16 : t == 2 ? 32 : 40; }

__global__ void k_panel_geometry(int N, const double* __restrict__ verts, const int32_t* __restrict__ kind,
                                 double* __restrict__ P, int32_t* __restrict__ bad, float* __restrict__ tiers,
                                 const int32_t* __restrict__ orig) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    double raw[4][3];
    bool ok = true;
    for (int i = 0; i < 4; i++)
        for (int d = 0; d < 3; d++) {
            raw[i][d] = verts[(size_t)j * 12 + 3 * i + d];
            ok = ok && isfinite(raw[i][d]);
        }
    auto fail = [&]() { atomicMin(bad, orig ? orig[j] : j); };  // the panel's index in the caller's order
    if (!ok) { fail(); return; }
    double t[3];
    double diameter = 0.0;
    for (int i = 0; i < 4; i++)
        for (int k = i + 1; k < 4; k++) {
            for (int d = 0; d < 3; d++) t[d] = raw[i][d] - raw[k][d];
            diameter = fmax(diameter, norm3(t));
        }
    if (diameter == 0.0) { fail(); return; }
    double tol = COINCIDENCE_TOL * diameter;
    int keep[4], m = 0;
    for (int i = 0; i < 4; i++) {
        for (int d = 0; d < 3; d++) t[d] = raw[i][d] - raw[(i + 1) % 4][d];
        if (norm3(t) > tol) keep[m++] = i;
    }
    if (m < 3) { fail(); return; }
    for (int a = 0; a < m; a++)
        for (int b = a + 1; b < m; b++) {
            for (int d = 0; d < 3; d++) t[d] = raw[keep[a]][d] - raw[keep[b]][d];
            if (norm3(t) <= tol) { fail(); return; }
        }
    double c[3], d1[3], d2[3], n[3];
    for (int d = 0; d < 3; d++) {
        c[d] = 0.25 * (raw[0][d] + raw[1][d] + raw[2][d] + raw[3][d]);
        d1[d] = raw[2][d] - raw[0][d];
        d2[d] = raw[3][d] - raw[1][d];
    }
    cross3(d1, d2, n);
    double nn = norm3(n);
    if (0.5 * nn <= COINCIDENCE_TOL * diameter * diameter) { fail(); return; }
    double inv = 1.0 / nn, nh[3] = {inv * n[0], inv * n[1], inv * n[2]};
    double q[4][3];
    for (int i = 0; i < 4; i++) {
        for (int d = 0; d < 3; d++) t[d] = raw[i][d] - c[d];
        double s = dot3(t, nh);
        for (int d = 0; d < 3; d++) q[i][d] = raw[i][d] - s * nh[d];
    }
    double poly[4][3];
    for (int a = 0; a < m; a++)
        for (int d = 0; d < 3; d++) poly[a][d] = q[keep[a]][d];
    for (int a = 0; a < m; a++) {
        double e1[3], e2[3], cr[3];
        for (int d = 0; d < 3; d++) {
            e1[d] = poly[(a + 1) % m][d] - poly[a][d];
            e2[d] = poly[(a + 2) % m][d] - poly[(a + 1) % m][d];
        }
        cross3(e1, e2, cr);
        double s = dot3(cr, nh) / (norm3(e1) * norm3(e2));
        if (!(s > CONVEXITY_TOL)) { fail(); return; }
    }
    double area = 0.0, mom[3] = {0, 0, 0};
    for (int a = 1; a < m - 1; a++) {
        double e1[3], e2[3], cr[3];
        for (int d = 0; d < 3; d++) {
            e1[d] = poly[a][d] - poly[0][d];
            e2[d] = poly[a + 1][d] - poly[0][d];
        }
        cross3(e1, e2, cr);
        double tt = 0.5 * dot3(cr, nh);
        area += tt;
        for (int d = 0; d < 3; d++) mom[d] += (tt / 3.0) * (poly[0][d] + poly[a][d] + poly[a + 1][d]);
    }
    double cent[3], normal[3] = {nh[0], nh[1], nh[2]};
    for (int d = 0; d < 3; d++) cent[d] = (1.0 / area) * mom[d];
    if (kind && kind[j] == 1) {
        // interior free surface: exactly in z = 0, normal +z (lo_geometry.rs:706-716)
        if (nh[2] < 0.0)
            for (int d = 0; d < 3; d++) {
                double s = q[1][d];
                q[1][d] = q[3][d];
                q[3][d] = s;
            }
        for (int i = 0; i < 4; i++) q[i][2] = 0.0;
        cent[2] = 0.0;
        normal[0] = 0.0;
        normal[1] = 0.0;
        normal[2] = 1.0;
    }
    auto W = [&](int plane, double val) { P[(size_t)plane * N + j] = val; };
    for (int d = 0; d < 3; d++) {
        W(P_C + d, cent[d]);
        W(P_N + d, normal[d]);
    }
    W(P_AREA, area);
    double diam = 0.0;
    for (int i = 0; i < 4; i++)
        for (int k = i + 1; k < 4; k++) {
            for (int d = 0; d < 3; d++) t[d] = q[i][d] - q[k][d];
            diam = fmax(diam, norm3(t));
        }
    double v[4][3] = {};
    int nv = 0;
    for (int i = 0; i < 4; i++) {
        for (int d = 0; d < 3; d++) t[d] = q[i][d] - q[(i + 1) % 4][d];
        if (norm3(t) > COINCIDENCE_TOL * diam) {
            for (int d = 0; d < 3; d++) v[nv][d] = q[i][d];
            nv++;
        }
    }
    double radius = 0.0;
    for (int i = 0; i < nv; i++) {
        for (int d = 0; d < 3; d++) t[d] = v[i][d] - cent[d];
        radius = fmax(radius, norm3(t));
    }
    W(P_RADIUS, radius);
    W(P_NV, (double)nv);
    for (int i = 0; i < 4; i++)
        for (int d = 0; d < 3; d++) W(P_V + 3 * i + d, v[i][d]);
    for (int e = 0; e < 4; e++) {
        double edge[3] = {0, 0, 0}, cr[3] = {0, 0, 0}, len = 0.0;
        if (e < nv) {
            for (int d = 0; d < 3; d++) edge[d] = v[(e + 1) % nv][d] - v[e][d];
            len = norm3(edge);
            cross3(edge, normal, cr);
            for (int d = 0; d < 3; d++) cr[d] *= 1.0 / len;
        }
        W(P_ELEN + e, len);
        for (int d = 0; d < 3; d++) W(P_EM + 3 * e + d, cr[d]);
    }
    double gw[9], sum = 0.0;
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            double x[3], jac;
            bilinear(q, c_glx[3][i], c_glx[3][k], x, jac);
            for (int d = 0; d < 3; d++) W(P_GX + 3 * (3 * i + k) + d, x[d]);
            gw[3 * i + k] = c_glw[3][i] * c_glw[3][k] * jac;
            sum += gw[3 * i + k];
        }
    for (int k = 0; k < 9; k++) W(P_GW + k, gw[k] * (area / sum));
    if (tiers) {
        float* tb = tiers + (size_t)j * TIER_FLOATS;
        for (int t = 0; t < 4; t++) {
            const int n = 3 + t, len = tier_len(t);
            float* b = tb + tier_off(t);
            double wsum = 0.0;
            for (int i = 0; i < n; i++)
                for (int k = 0; k < n; k++) {
                    double x[3], jac;
                    bilinear(q, c_glx[n][i], c_glx[n][k], x, jac);
                    wsum += c_glw[n][i] * c_glw[n][k] * jac;
                }
            for (int i = 0; i < n; i++)
                for (int k = 0; k < n; k++) {
                    double x[3], jac;
                    bilinear(q, c_glx[n][i], c_glx[n][k], x, jac);
                    const int e = i * n + k;
                    b[e] = (float)(x[0] - cent[0]);
                    b[len + e] = (float)(x[1] - cent[1]);
                    b[2 * len + e] = (float)(x[2] - cent[2]);
                    b[3 * len + e] = (float)(c_glw[n][i] * c_glw[n][k] * jac * area / wsum);
                }
            for (int e = n * n; e < len; e++) b[e] = b[len + e] = b[2 * len + e] = b[3 * len + e] = 0.f;
        }
    }
}

// ------------------------------------------------------------------ Rankine closed forms
struct PanelRegs {
    int nv;
    double c[3], n[3], area, radius;
    double v[4][3], em[4][3], elen[4];
};

__device__ __forceinline__ void load_panel(const PanelsView& pv, int j, PanelRegs& p) {
    p.nv = (int)pv.at(P_NV, j);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        p.c[d] = pv.at(P_C + d, j);
        p.n[d] = pv.at(P_N + d, j);
    }
    p.area = pv.at(P_AREA, j);
    p.radius = pv.at(P_RADIUS, j);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        p.elen[i] = pv.at(P_ELEN + i, j);
#pragma unroll
        for (int d = 0; d < 3; d++) {
            p.v[i][d] = pv.at(P_V + 3 * i + d, j);
            p.em[i][d] = pv.at(P_EM + 3 * i + d, j);
        }
    }
}

// panel_integrals.rs:226-275 (closed forms; beyond `far` radii the 3 x 3 rule: 1000 in the reference's
// double-precision mode, 12 in its production mode)
__device__ inline void rankine(const PanelsView& pv, int j, const PanelRegs& p, const double* x, double& S, double& D,
                               double far = 1000.0) {
    double rc[3] = {x[0] - p.c[0], x[1] - p.c[1], x[2] - p.c[2]};
    double dist = norm3(rc);
    if (dist > far * p.radius) {
        double s = 0.0, dd = 0.0;
        for (int k = 0; k < 9; k++) {
            double r[3];
            for (int d = 0; d < 3; d++) r[d] = x[d] - pv.at(P_GX + 3 * k + d, j);
            double ir = 1.0 / norm3(r), w = pv.at(P_GW + k, j);
            s += w * ir;
            dd += w * dot3(p.n, r) * ir * ir * ir;
        }
        S = s;
        D = dd;
        return;
    }
    double w = dot3(rc, p.n);
    int nv = p.nv;
    double av[4][3], r[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        for (int d = 0; d < 3; d++) av[i][d] = p.v[i][d] - x[d];
        r[i] = norm3(av[i]);
    }
    double omega = 0.0;
    if (fabs(w) > 1e-12 * p.radius) {
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
        int f = (e + 1) == nv ? 0 : e + 1;
        double d = dot3(av[e], p.em[e]);
        if (fabs(d) <= 1e-14 * p.radius) continue;
        double q = r[e] * r[f] + dot3(av[e], av[f]);
        if (!(q > 0.0)) continue;
        double sum = r[e] + r[f] + p.elen[e];
        s += d * log(sum * sum / (2.0 * q));
    }
    S = s - w * omega;
    D = omega;
}

__device__ __forceinline__ void psi_terms(const double* xi, const double* pp, const double* n, double& psi, double& dpsi) {
    double d[3] = {xi[0] - pp[0], xi[1] - pp[1], xi[2] - pp[2]};
    double R = norm3(d);
    double den = R - d[2];
    psi = log(den);
    dpsi = (dot3(d, n) / R - n[2]) / den;
}

__device__ __forceinline__ void panel_map(const PanelRegs& p, double m[4][3]) {
    for (int d = 0; d < 3; d++) {
        m[0][d] = p.v[0][d];
        m[1][d] = p.v[1][d];
        m[2][d] = p.v[2][d];
        m[3][d] = p.nv == 4 ? p.v[3][d] : p.v[2][d];
    }
}

// the Gauss order of the log integral by distance, 0 for the adaptive rule (panel_integrals.rs:407-432)
__device__ __forceinline__ int log_order(const PanelRegs& p, const double* image) {
    double t[3] = {image[0] - p.c[0], image[1] - p.c[1], image[2] - p.c[2]};
    double dist = norm3(t);
    double top = p.v[0][2];
    for (int i = 1; i < p.nv; i++) top = fmax(top, p.v[i][2]);
    double r = dist / p.radius;
    double clearance = (image[2] - top) / p.radius;
    if (clearance >= 0.5 || r >= 2.0) return r >= 6.0 ? 4 : r >= 3.0 ? 5 : r >= 2.0 ? 6 : r >= 1.5 ? 8 : r >= 1.0 ? 10 : 0;
    return 0;
}

__device__ inline void log_gauss(const PanelRegs& p, const double* image, int order, double& L, double& Ld) {
    double m[4][3];
    panel_map(p, m);
    double l = 0.0, ld = 0.0;
    for (int i = 0; i < order; i++)
        for (int j = 0; j < order; j++) {
            double xi[3], jac, psi, dpsi;
            bilinear(m, c_glx[order][i], c_glx[order][j], xi, jac);
            psi_terms(xi, image, p.n, psi, dpsi);
            double ww = c_glw[order][i] * c_glw[order][j] * jac;
            l += ww * psi;
            ld += ww * dpsi;
        }
    L = l;
    Ld = ld;
}

// ---- the mixed form's far-field shortcuts (its matrices are rounded to FP32 afterwards)
// A point farther than MIX_FAR panel radii from the panel: the Rankine integrals by the panel's 3 x 3
// Gauss rule (the rule the closed forms give way to beyond 1000 radii), in FP32 on FP64 differences.
// The rule's error falls as (radius / distance)^6, below FP32 rounding at 20 radii.
constexpr double MIX_FAR = 20.0;

__device__ __forceinline__ void rankine_gauss_f32(const PanelsView& pv, int j, const PanelRegs& p, const double* x,
                                                  double& S, double& D) {
    const float n0 = (float)p.n[0], n1 = (float)p.n[1], n2 = (float)p.n[2];
    float s = 0.f, dd = 0.f;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const float r0 = (float)(x[0] - pv.at(P_GX + 3 * k, j));
        const float r1 = (float)(x[1] - pv.at(P_GX + 3 * k + 1, j));
        const float r2 = (float)(x[2] - pv.at(P_GX + 3 * k + 2, j));
        const float w = (float)pv.at(P_GW + k, j);
        const float ir = rsqrtf(__fmaf_rn(r0, r0, __fmaf_rn(r1, r1, r2 * r2)));
        const float wi = w * ir;
        s += wi;
        dd = __fmaf_rn(wi * ir * ir, __fmaf_rn(n0, r0, __fmaf_rn(n1, r1, n2 * r2)), dd);
    }
    S = s;
    D = dd;
}

// log_gauss with the integrand log(R - dz) and its normal derivative in FP32 (positions, weights and
// sums in FP64): R - dz = R + |dz| for an image above the panel, so no cancellation.
__device__ inline void log_gauss_f32(const PanelRegs& p, const double* image, int order, double& L, double& Ld) {
    double m[4][3];
    panel_map(p, m);
    const float n0 = (float)p.n[0], n1 = (float)p.n[1], n2 = (float)p.n[2];
    double l = 0.0, ld = 0.0;
    for (int i = 0; i < order; i++)
        for (int j = 0; j < order; j++) {
            double xi[3], jac;
            bilinear(m, c_glx[order][i], c_glx[order][j], xi, jac);
            const float d0 = (float)(xi[0] - image[0]), d1 = (float)(xi[1] - image[1]), d2 = (float)(xi[2] - image[2]);
            const float R = sqrtf(__fmaf_rn(d0, d0, __fmaf_rn(d1, d1, d2 * d2)));
            const float den = R - d2;
            const float psi = logf(den);
            const float dpsi = (__fmaf_rn(d0, n0, __fmaf_rn(d1, n1, d2 * n2)) / R - n2) / den;
            const double ww = c_glw[order][i] * c_glw[order][j] * jac;
            l += ww * (double)psi;
            ld += ww * (double)dpsi;
        }
    L = l;
    Ld = ld;
}

// ---- the reference's production rule (the mixed form)
// panel_integrals.rs:288-300 rankine_tier: 0 (order 3) beyond 8 radii, 1 (order 4) from 4, 2 (order 5)
// from 3, 3 (order 6) from 2; -1 (the closed forms) within 2
__device__ __forceinline__ int rankine_tier(double r) {
    return r >= 8.0 ? 0 : r >= 4.0 ? 1 : r >= 3.0 ? 2 : r >= 2.0 ? 3 : -1;
}

// panel_integrals.rs:305-357 rankine_gauss: the tier's rule in float32 on the point taken relative to the
// centroid in double, eight accumulator lanes summed in double (the reference's lane order)
__device__ inline void rankine_gauss_tier(const PanelRegs& p, const float* __restrict__ tq, const double* x, int t,
                                          double& S, double& D) {
    const int len = tier_len(t);
    const float* b = tq + tier_off(t);
    const float px = (float)(x[0] - p.c[0]), py = (float)(x[1] - p.c[1]), pz = (float)(x[2] - p.c[2]);
    const float nx = (float)p.n[0], ny = (float)p.n[1], nz = (float)p.n[2];
    float sacc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, dacc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < len; k += 8)
#pragma unroll
        for (int l = 0; l < 8; l++) {
            const float rx = px - b[k + l], ry = py - b[len + k + l], rz = pz - b[2 * len + k + l];
            const float w = b[3 * len + k + l];
            const float r2 = __fmaf_rn(rz, rz, __fmaf_rn(rx, rx, ry * ry));
            const float ir = 1.0f / sqrtf(r2);
            const float nr = __fmaf_rn(nz, rz, __fmaf_rn(nx, rx, ny * ry));
            sacc[l] = __fmaf_rn(w, ir, sacc[l]);
            dacc[l] = __fmaf_rn(w * nr, ir * (ir * ir), dacc[l]);
        }
    double s = 0.0, d = 0.0;
#pragma unroll
    for (int l = 0; l < 8; l++) {
        s += (double)sacc[l];
        d += (double)dacc[l];
    }
    S = s;
    D = d;
}

// Rankine integrals at x: with the tiers, panel_integrals.rs:359-363 rankine_any of the production mode
// (the tiers, or the closed forms within 2 radii); the mixed form's own rule otherwise (the closed
// forms, the FP32 3 x 3 rule beyond MIX_FAR radii); the FP64 form the closed forms.
template <bool MIXED>
__device__ __forceinline__ void rankine_at(const PanelsView& pv, int j, const PanelRegs& p, const double* x, double& S,
                                           double& D) {
    if constexpr (MIXED) {
        const double t0 = x[0] - p.c[0], t1 = x[1] - p.c[1], t2 = x[2] - p.c[2];
        if (pv.tiers) {  // the production rule
            const double rc[3] = {t0, t1, t2};
            const int t = rankine_tier(norm3(rc) / p.radius);
            if (t >= 0) {
                rankine_gauss_tier(p, pv.tiers + (size_t)j * TIER_FLOATS, x, t, S, D);
                return;
            }
        } else {  // the mixed form's own rule: the closed forms within MIX_FAR radii
            const double far = MIX_FAR * p.radius;
            if (t0 * t0 + t1 * t1 + t2 * t2 > far * far) {
                rankine_gauss_f32(pv, j, p, x, S, D);
                return;
            }
        }
    }
    rankine(pv, j, p, x, S, D);
}

// panel_integrals.rs:380-392: in the production mode the log integral of an image farther than 12 radii
// by the panel's 3 x 3 rule in double
__device__ inline void log_far_3x3(const PanelsView& pv, int j, const PanelRegs& p, const double* image, double& L,
                                   double& Ld) {
    double l = 0.0, ld = 0.0;
    for (int k = 0; k < 9; k++) {
        const double xi[3] = {pv.at(P_GX + 3 * k, j), pv.at(P_GX + 3 * k + 1, j), pv.at(P_GX + 3 * k + 2, j)};
        double psi, dpsi;
        psi_terms(xi, image, p.n, psi, dpsi);
        const double w = pv.at(P_GW + k, j);
        l += w * psi;
        ld += w * dpsi;
    }
    L = l;
    Ld = ld;
}

__device__ __forceinline__ double to_f32(double v) { return (double)(float)v; }

// lo_static.rs:47-55 log_pair
__device__ __forceinline__ bool log_pair(const PanelRegs& p, const double* x, double tol) {
    double dx = x[0] - p.c[0], dy = x[1] - p.c[1], zz = fabs(x[2] + p.c[2]);
    double d = sqrt(dx * dx + dy * dy + zz * zz) + zz;
    return d * d * tol < 0.6 * p.radius * p.radius;
}

// panel_integrals.rs:625-648 log_in_plane
__device__ inline double log_in_plane(const PanelRegs& p, const double* x) {
    double sum = 0.0;
    for (int i = 0; i < p.nv; i++) {
        int i1 = (i + 1) == p.nv ? 0 : i + 1;
        double ax[3], bx[3], e[3];
        for (int d = 0; d < 3; d++) {
            ax[d] = p.v[i][d] - x[d];
            bx[d] = p.v[i1][d] - x[d];
        }
        double h = dot3(ax, p.em[i]);
        if (h == 0.0) continue;
        for (int d = 0; d < 3; d++) e[d] = (1.0 / p.elen[i]) * (p.v[i1][d] - p.v[i][d]);
        double t1 = dot3(ax, e), t2 = dot3(bx, e);
        double q1 = h * h + t1 * t1, q2 = h * h + t2 * t2;
        double F1 = 0.5 * (t1 * log(q1) - 2.0 * t1 + 2.0 * h * atan(t1 / h)) - 0.5 * t1;
        double F2 = 0.5 * (t2 * log(q2) - 2.0 * t2 + 2.0 * h * atan(t2 / h)) - 0.5 * t2;
        sum += 0.5 * h * (F2 - F1);
    }
    return sum;
}

// One (row k, panel j) pair: rs, rd and (unless adaptive) dl, dd.  lo_static.rs:59-119
// Four planes of Nr x N (rows k < Nr = N / G, the sector's points, or the Nr field points; every panel
// j), entry at k + j Nr.
// MIXED: the mixed form's variant (far Rankine points and the order-4 log rule in FP32, above; with
// pv.tiers the reference's production rule instead, rows in float32); the FP64 form runs the reference's
// double-precision arithmetic to the bit.
template <bool MIXED>
__global__ void __launch_bounds__(256, 2) k_statics(PanelsView pv, double depth, int logint, double tol,
                                                 double* __restrict__ st, int32_t* __restrict__ work,
                                                 int32_t* __restrict__ nwork, int work_cap) {
    // rows: the sector's panels (or the field points); columns: all panels
    const int N = pv.N, Nr = pv.rows ? pv.nrows : N / pv.G;
    int k = blockIdx.x * 32 + threadIdx.x;
    int j = blockIdx.y * 8 + threadIdx.y;
    // the panel of each warp (36 values every lane of the warp reads) in shared memory rather than in
    // 72 registers of every lane
    __shared__ PanelRegs sp[8];
    if (threadIdx.x == 0 && j < N) load_panel(pv, j, sp[threadIdx.y]);
    __syncthreads();
    if (k >= Nr || j >= N) return;
    const PanelRegs& p = sp[threadIdx.y];
    double x[3];
    for (int d = 0; d < 3; d++) x[d] = pv.rows ? pv.rows[3 * k + d] : pv.at(P_C + d, k);
    double xb[3] = {x[0], x[1], -x[2]};
    double s0, d0, sb, db;
    rankine_at<MIXED>(pv, j, p, x, s0, d0);
    rankine_at<MIXED>(pv, j, p, xb, sb, db);
    double sr = s0 + sb, dr = d0 + db;
    if (depth > 0.0) {
        double h = depth;
        double p1[3] = {x[0], x[1], -x[2] - 2.0 * h}, p3[3] = {x[0], x[1], x[2] + 2.0 * h};
        double p4[3] = {x[0], x[1], x[2] - 2.0 * h}, p5[3] = {x[0], x[1], -x[2] - 4.0 * h};
        double s2, d2, s4, d4, s5, d5, s6, d6;
        rankine_at<MIXED>(pv, j, p, p1, s2, d2);
        rankine_at<MIXED>(pv, j, p, p3, s4, d4);
        if (MIXED && pv.tiers) {  // production: the two deep images by the 3 x 3 rule beyond 12 radii
            rankine(pv, j, p, p4, s5, d5, 12.0);  // (lo_static.rs:82-88)
            rankine(pv, j, p, p5, s6, d6, 12.0);
        } else {
            rankine_at<MIXED>(pv, j, p, p4, s5, d5);
            rankine_at<MIXED>(pv, j, p, p5, s6, d6);
        }
        sr += (s2 + s4) + s5 + s6;
        dr += (d2 + d4) + d5 + d6;
    }
    const bool prod = MIXED && pv.tiers;  // the production rows are stored in float32
    size_t NN = (size_t)Nr * N, o = (size_t)k + (size_t)j * Nr;
    st[o] = prod ? to_f32(sr) : sr;
    st[NN + o] = prod ? to_f32(dr) : dr;
    double dl = 0.0, dd = 0.0;
    bool use_log = logint && log_pair(p, x, tol);
    if (use_log && pv.kind[j] == 1 && x[2] == 0.0) {
        double L = log_in_plane(p, x);
        double t[3] = {p.c[0] - x[0], p.c[1] - x[1], p.c[2] - x[2]};
        double Rr = norm3(t);
        dl = Rr > 0.0 ? L - p.area * log(Rr) : L;
    } else if (use_log) {
        const double tb[3] = {xb[0] - p.c[0], xb[1] - p.c[1], xb[2] - p.c[2]};
        const bool far3 = prod && norm3(tb) > 12.0 * p.radius;
        int order = far3 ? 3 : log_order(p, xb);
        if (order > 0) {
            double L, Ld, psi, dpsi;
            if (far3)
                log_far_3x3(pv, j, p, xb, L, Ld);
            else if (MIXED && !prod && order == 4)
                log_gauss_f32(p, xb, order, L, Ld);
            else
                log_gauss(p, xb, order, L, Ld);
            psi_terms(p.c, xb, p.n, psi, dpsi);
            dl = L - p.area * psi;
            dd = Ld - p.area * dpsi;
        } else {
            int slot = atomicAdd(nwork, 1);
            if (slot < work_cap) {
                work[2 * slot] = k;
                work[2 * slot + 1] = j;
            }
        }
    }
    st[2 * NN + o] = prod ? to_f32(dl) : dl;
    st[3 * NN + o] = prod ? to_f32(dd) : dd;
}

// 4 x 4 Gauss rule of a cell of the parameter square (panel_integrals.rs:80-98)
__device__ inline void log_cell(const double m[4][3], const double* image, const double* n, double u0, double u1,
                                double v0, double v1, double* s) {
    s[0] = s[1] = 0.0;
    double hu = 0.5 * (u1 - u0), hv = 0.5 * (v1 - v0);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            double xi[3], jac, psi, dpsi;
            bilinear(m, u0 + hu * (c_glx[4][i] + 1.0), v0 + hv * (c_glx[4][j] + 1.0), xi, jac);
            double ww = c_glw[4][i] * c_glw[4][j] * hu * hv * jac;
            psi_terms(xi, image, n, psi, dpsi);
            s[0] += ww * psi;
            s[1] += ww * dpsi;
        }
}

// The adaptive pairs: quadrisection to 1e-13 of the integrals' scale, at most 14 levels, cells
// taken in the depth-first order of panel_integrals.rs:100-120.  One warp per pair: at each level
// the 32 lanes evaluate the 4 sub-cells x 16 Gauss points (two points a lane), reduce them per
// sub-cell by shuffles, and lane 0 keeps the depth-first stack in shared memory.
constexpr int AD_WARPS = 4, AD_STACK = 48;

struct AdCell {
    double u0, u1, v0, v1, p0, p1;
    int depth;
};

__device__ __forceinline__ void log_point(const double m[4][3], const double* image, const double* n, double u0,
                                          double u1, double v0, double v1, int i, int j, double& a, double& b) {
    double hu = 0.5 * (u1 - u0), hv = 0.5 * (v1 - v0);
    double xi[3], jac, psi, dpsi;
    bilinear(m, u0 + hu * (c_glx[4][i] + 1.0), v0 + hv * (c_glx[4][j] + 1.0), xi, jac);
    double ww = c_glw[4][i] * c_glw[4][j] * hu * hv * jac;
    psi_terms(xi, image, n, psi, dpsi);
    a = ww * psi;
    b = ww * dpsi;
}

// One adaptive pair (worklist entry t) by the calling warp; stk: the warp's stack in shared memory.
__device__ void adaptive_pair(const PanelsView& pv, const int32_t* __restrict__ work, int t, double* __restrict__ st,
                              AdCell* stk, int lane) {
    const int N = pv.N;
    const int k = work[2 * t], j = work[2 * t + 1];
    PanelRegs p;
    load_panel(pv, j, p);
    double xb[3];
    for (int d = 0; d < 3; d++) xb[d] = pv.rows ? pv.rows[3 * k + d] : pv.at(P_C + d, k);
    xb[2] = -xb[2];
    double m[4][3];
    panel_map(p, m);
    double tt[3] = {xb[0] - p.c[0], xb[1] - p.c[1], xb[2] - p.c[2]};
    double dist = norm3(tt);
    double dmin = fmax(dist - p.radius, 1e-3 * p.radius);
    double scale = fabs(log(dist + p.radius)) + 1.0;
    double tol_l = 1e-13 * p.area * scale, tol_d = 1e-13 * p.area / dmin;
    // the whole square by one 4 x 4 cell (lanes 0..15 one point each)
    double wa = 0.0, wb = 0.0;
    if (lane < 16) log_point(m, xb, p.n, -1.0, 1.0, -1.0, 1.0, lane / 4, lane % 4, wa, wb);
    for (int o = 16; o > 0; o >>= 1) {
        wa += __shfl_xor_sync(0xffffffffu, wa, o);
        wb += __shfl_xor_sync(0xffffffffu, wb, o);
    }
    int sp = 0;
    if (lane == 0) stk[0] = AdCell{-1.0, 1.0, -1.0, 1.0, wa, wb, 0};
    sp = 1;
    __syncwarp();
    double acc0 = 0.0, acc1 = 0.0;
    while (sp > 0) {
        AdCell c = stk[sp - 1];
        sp--;
        __syncwarp();
        const double um = 0.5 * (c.u0 + c.u1), vm = 0.5 * (c.v0 + c.v1);
        const double us0[4] = {c.u0, um, um, c.u0}, us1[4] = {um, c.u1, c.u1, um};
        const double vs0[4] = {c.v0, c.v0, vm, vm}, vs1[4] = {vm, vm, c.v1, c.v1};
        // lane l: point l of sub-cells (l / 16) and (l / 16) + 2
        const int sa = lane >> 4, q = lane & 15;
        double a0, b0, a1, b1;
        log_point(m, xb, p.n, us0[sa], us1[sa], vs0[sa], vs1[sa], q / 4, q % 4, a0, b0);
        log_point(m, xb, p.n, us0[sa + 2], us1[sa + 2], vs0[sa + 2], vs1[sa + 2], q / 4, q % 4, a1, b1);
        for (int o = 8; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            b0 += __shfl_xor_sync(0xffffffffu, b0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            b1 += __shfl_xor_sync(0xffffffffu, b1, o);
        }
        double cc[4][2];
        cc[0][0] = __shfl_sync(0xffffffffu, a0, 0);
        cc[0][1] = __shfl_sync(0xffffffffu, b0, 0);
        cc[1][0] = __shfl_sync(0xffffffffu, a0, 16);
        cc[1][1] = __shfl_sync(0xffffffffu, b0, 16);
        cc[2][0] = __shfl_sync(0xffffffffu, a1, 0);
        cc[2][1] = __shfl_sync(0xffffffffu, b1, 0);
        cc[3][0] = __shfl_sync(0xffffffffu, a1, 16);
        cc[3][1] = __shfl_sync(0xffffffffu, b1, 16);
        const double s0 = cc[0][0] + cc[1][0] + cc[2][0] + cc[3][0];
        const double s1 = cc[0][1] + cc[1][1] + cc[2][1] + cc[3][1];
        if (c.depth >= 14 || (fabs(s0 - c.p0) <= tol_l && fabs(s1 - c.p1) <= tol_d) || sp + 4 > AD_STACK) {
            acc0 += s0;
            acc1 += s1;
            continue;
        }
        if (lane == 0)
            for (int qq = 3; qq >= 0; qq--)
                stk[sp + 3 - qq] = AdCell{us0[qq], us1[qq], vs0[qq], vs1[qq], cc[qq][0], cc[qq][1], c.depth + 1};
        sp += 4;
        __syncwarp();
    }
    if (lane == 0) {
        double psi, dpsi;
        psi_terms(p.c, xb, p.n, psi, dpsi);
        const int Nr = pv.rows ? pv.nrows : N / pv.G;
        size_t NN = (size_t)Nr * N, o = (size_t)k + (size_t)j * Nr;
        const double vl = acc0 - p.area * psi, vd = acc1 - p.area * dpsi;
        st[2 * NN + o] = pv.tiers ? to_f32(vl) : vl;  // the production rows in float32
        st[3 * NN + o] = pv.tiers ? to_f32(vd) : vd;
    }
}

// One warp per worklist entry, the entry count given by the host.
__global__ void __launch_bounds__(AD_WARPS * 32) k_statics_adaptive(PanelsView pv, const int32_t* __restrict__ work,
                                                                    int nwork, double* __restrict__ st) {
    __shared__ AdCell stack[AD_WARPS][AD_STACK];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * AD_WARPS + warp;
    if (t >= nwork) return;
    adaptive_pair(pv, work, t, st, stack[warp], lane);
}

// The same with the entry count in device memory (q[0], capped at work_cap) and the entries taken
// from a queue (cursor q[1], zero at launch), so that the host need not wait for the count.  No
// work when the geometry flagged an invalid panel (*bad != clean): the solve reports it.
__global__ void __launch_bounds__(AD_WARPS * 32) k_statics_adaptive_q(PanelsView pv, const int32_t* __restrict__ work,
                                                                      int32_t* q, int work_cap,
                                                                      const int32_t* __restrict__ bad, int32_t clean,
                                                                      double* __restrict__ st) {
    __shared__ AdCell stack[AD_WARPS][AD_STACK];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (*bad != clean) return;
    const int nwork = min(*(volatile int32_t*)q, work_cap);
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(q + 1, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= nwork) return;
        adaptive_pair(pv, work, t, st, stack[warp], lane);
        __syncwarp();
    }
}

// ------------------------------------------------------------------ host launchers
void launch_panel_geometry(int N, const double* verts, const int32_t* kind, double* planes, int32_t* bad,
                           cudaStream_t s, float* tiers, const int32_t* orig) {
    k_panel_geometry<<<(N + 127) / 128, 128, 0, s>>>(N, verts, kind, planes, bad, tiers, orig);
}

void launch_statics(const PanelsView& pv, double depth, int logint, double tol, double* st, int32_t* work,
                    int32_t* nwork, int work_cap, cudaStream_t s, bool mixed) {
    dim3 grid(((pv.rows ? pv.nrows : pv.N / pv.G) + 31) / 32, (pv.N + 7) / 8);
    if (mixed)
        k_statics<true><<<grid, dim3(32, 8), 0, s>>>(pv, depth, logint, tol, st, work, nwork, work_cap);
    else
        k_statics<false><<<grid, dim3(32, 8), 0, s>>>(pv, depth, logint, tol, st, work, nwork, work_cap);
}

void launch_statics_adaptive(const PanelsView& pv, const int32_t* work, int nwork, double* st, cudaStream_t s) {
    if (nwork > 0) k_statics_adaptive<<<(nwork + AD_WARPS - 1) / AD_WARPS, AD_WARPS * 32, 0, s>>>(pv, work, nwork, st);
}

void launch_statics_adaptive_q(const PanelsView& pv, const int32_t* work, int32_t* q, int work_cap,
                               const int32_t* bad, int32_t clean, double* st, cudaStream_t s) {
    static int grid[16] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 16) dev = 0;
    if (grid[dev] == 0) {
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_statics_adaptive_q, AD_WARPS * 32, 0);
        grid[dev] = std::max(1, sms * std::max(per, 1));
    }
    k_statics_adaptive_q<<<grid[dev], AD_WARPS * 32, 0, s>>>(pv, work, q, work_cap, bad, clean, st);
}

void set_constants_statics(const double glx[17][16], const double glw[17][16]) {
    cudaMemcpyToSymbol(c_glx, glx, sizeof(double) * 17 * 16);
    cudaMemcpyToSymbol(c_glw, glw, sizeof(double) * 17 * 16);
}

}  // namespace hbg
