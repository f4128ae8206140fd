// hbg_device.cuh -- device-side data layout and FP64 kernel functions of the low-order BEM path.
//
// The Green-function tables (generated data of the reference, checksum-verified at load) live in
// global memory; the hot kernels read them through the read-only path (L2-resident: 2.3 MB).
// Panels are stored as structure-of-arrays planes of N doubles each, so a warp that walks 32
// consecutive panels issues coalesced loads, and a warp that holds one panel gets a broadcast.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hbg {

constexpr double PI = 3.14159265358979323846;
constexpr double GAMMA = 0.5772156649015329;   // Euler's constant (constants.rs:4)
constexpr double LOG2 = 0.6931471805599453;
// table layout (tables/green_inf_tables.rs:5-11, green_fin_tables.rs:5-11)
constexpr int XT = 30, YT = 30, N1 = 16, N2 = 7, N3 = 6, HANKEL_TERMS = 14, STRUVE_TERMS = 14;
constexpr int FM = 9, NW = 12, REGIONS = 13, NK = 17;
constexpr int NC = NW + 1;
constexpr double K_LO = 0.5;
constexpr int FIN_ROOTS = 24;
constexpr double SERIES_STOP = 18.0;
constexpr int TS = 8, TW = 8, TV = 16, TD = 5, TN = TD + 1;
constexpr double XMAX = 0.5;
constexpr int T1_SIZE = TS * TW * 3 * TN * TN;
constexpr int T2_SIZE = TS * TV * 3 * TN * TN;
// The mixed form's FP32 tiles: the same Chebyshev interpolants truncated to degree TFD in each
// variable, each block of (TFD + 1)^2 power-basis coefficients padded to whole float4 loads.
constexpr int TFD = 3, TFN = TFD + 1, TFB = (TFN * TFN + 3) / 4 * 4;
constexpr int T1F_SIZE = TS * TW * 3 * TFB, T2F_SIZE = TS * TV * 3 * TFB;
// The mixed form's FP32 copies of TABLE_1D and TABLE_2D, their Chebyshev series cut the same way:
// TABLE_1D to T1D_FN terms per cell (degree 16 stored; the dropped terms sum below 3e-10), TABLE_2D
// to T2D_FX x T2D_FY terms in (X, Y) per quantity (8 x 8 stored; dropped below 5e-8), each block of
// T2D_FX T2D_FY coefficients padded to T2D_FB floats (whole float4 loads).
constexpr int T1D_FN = 8;
constexpr int T2D_FX = 6, T2D_FY = 7, T2D_FB = (T2D_FX * T2D_FY + 3) / 4 * 4;

struct Tables {
    const double* t1d;   // [30][17][4]     J0, J1, Yt, Yt'
    const double* t2d;   // [30][30][2][8][8] V, V_X
    const double* t2dd;  // direct tiles (production branch; unused by the FP64 form)
    const double* asy;   // Hankel / Struve asymptotics
    const double* meta;  // finite depth: region meta
    const double* q;     // Q_m Chebyshev coefficients
    const double* l0;
    const double* bk;    // scaled K0, K1 tiles
    const float* t2d_f;  // t2d rounded to FP32 (the mixed form's coefficient reads)
    const float* t1d_f;  // t1d rounded to FP32
};

// Panels in structure-of-arrays planes (each plane N doubles, plane p at base + p N).
enum PanelPlane {
    P_C = 0,       // centroid x y z            (3)
    P_N = 3,       // unit normal               (3)
    P_AREA = 6,
    P_RADIUS = 7,
    P_V = 8,       // 4 vertices x 3            (12) distinct projected vertices
    P_EM = 20,     // edge in-plane normals     (12)
    P_ELEN = 32,   // edge lengths              (4)
    P_GX = 36,     // 3x3 Gauss points          (27)
    P_GW = 63,     // weights                   (9)
    P_NV = 72,     // distinct vertex count (as double)
    P_PLANES = 73
};

// The geometry kernel's invalid-panel flag: the lowest invalid panel index, this value when none.
constexpr int32_t PANELS_VALID = 0x7fffffff;

struct PanelsView {
    int N;
    const double* p;     // P_PLANES planes of N
    const int32_t* kind; // 0 wet, 1 interior
    // optional: the invalid-panel flag; kernels that see it set (!= PANELS_VALID) skip their work
    const int32_t* bad = nullptr;
    // the bodies of a multi-body problem: body index of each panel (null: all body 0), the rotation
    // centre of each body (3 per body; null: the origin), the body count
    const int32_t* body = nullptr;
    const double* rcen = nullptr;
    int nbod = 1;
    // symmetry sectors (lo_geometry.rs:25-36): the N panels are the Ns = N / G panels of one sector
    // followed by their images under each reflection of the group (image g of panel n at g Ns + n,
    // order e, then x, y, xy reflections); the statics and the system matrices have the Ns sector rows
    int G = 1;
    // field points as the statics' rows instead of the sector's centroids: nrows points (x, y, z)
    const double* rows = nullptr;
    int nrows = 0;
    // the mixed form: each panel's float32 Gauss tiers ([N][TIER_FLOATS]); the statics then follow the
    // reference's production rule (null: its double-precision rule)
    const float* tiers = nullptr;
    __device__ __forceinline__ bool invalid() const { return bad && *(volatile const int32_t*)bad != PANELS_VALID; }
    // generalized normal of rigid mode `mode` (body mode / 6: surge, sway, heave, roll, pitch, yaw about
    // its rotation centre) on panel j: zero on the panels of the other bodies
    __device__ __forceinline__ double gen_normal(int j, int mode) const {
        const int b = mode / 6, m = mode - 6 * (mode / 6);
        if ((body ? body[j] : 0) != b) return 0.0;
        const double nx = at(P_N, j), ny = at(P_N + 1, j), nz = at(P_N + 2, j);
        if (m < 3) return m == 0 ? nx : m == 1 ? ny : nz;
        const double cx = at(P_C, j) - (rcen ? rcen[3 * b] : 0.0), cy = at(P_C + 1, j) - (rcen ? rcen[3 * b + 1] : 0.0),
                     cz = at(P_C + 2, j) - (rcen ? rcen[3 * b + 2] : 0.0);
        return m == 3 ? cy * nz - cz * ny : m == 4 ? cz * nx - cx * nz : cx * ny - cy * nx;
    }
    __device__ __forceinline__ double at(int plane, int j) const { return p[(size_t)plane * N + j]; }
};

// Per-frequency scalars of the finite-depth kernel (green_fin.rs:83-110 FiniteDepth).
struct FdParams {
    int mode;   // 0 ordinary, 1 omega = 0, 2 omega = inf
    int pad;
    double h, K, H, k0, A0;
    double sign[6];
    double kn[FIN_ROOTS];
    double cn[FIN_ROOTS];
    double P[(FM + 1) * NC];
};

// the fin_point data of one panel depth (green_fin.rs:119-130), stored as planes per frequency
constexpr int FP_PLANES = 4 + 2 * FIN_ROOTS;

// Gauss-Legendre rules of orders 1..16 and the table pointers: one copy per translation unit
// (hbg_statics.cu and hbg_all.cu), each set by its own set_constants function.
static __constant__ double c_glx[17][16];
static __constant__ double c_glw[17][16];
static __constant__ Tables c_tab;

// ------------------------------------------------------------------ small helpers
__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void cross3(const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double norm3(const double* a) { return sqrt(dot3(a, a)); }

// ------------------------------------------------------------------ infinite depth (green_inf.rs)
// 1D tiles: J0, J1, Yt, Yt' (green_inf.rs:58-73)
__device__ __forceinline__ void table1d(double X, double* r) {
    int i = (int)X;
    if (i >= XT) i = XT - 1;
    double t = 2.0 * (X - i) - 1.0;
    const double* c = c_tab.t1d + i * (N1 + 1) * 4;
    double r0 = 0, r1 = 0, r2 = 0, r3 = 0;
#pragma unroll
    for (int j = N1; j >= 0; j--) {
        double2 ca = __ldg(reinterpret_cast<const double2*>(c + 4 * j));
        double2 cb = __ldg(reinterpret_cast<const double2*>(c + 4 * j + 2));
        r0 = r0 * t + ca.x;
        r1 = r1 * t + ca.y;
        r2 = r2 * t + cb.x;
        r3 = r3 * t + cb.y;
    }
    r[0] = r0; r[1] = r1; r[2] = r2; r[3] = r3;
}

// table1d from the FP32 copy (the mixed form): one float4 per Chebyshev term, FP32 Horner chains.
__device__ __forceinline__ void table1d_f32(double X, double* r) {
    int i = (int)X;
    if (i >= XT) i = XT - 1;
    const float t = (float)(2.0 * (X - i) - 1.0);
    const float4* c = reinterpret_cast<const float4*>(c_tab.t1d_f + i * T1D_FN * 4);
    float r0 = 0.f, r1 = 0.f, r2 = 0.f, r3 = 0.f;
#pragma unroll
    for (int j = T1D_FN - 1; j >= 0; j--) {
        const float4 cc = __ldg(c + j);
        r0 = r0 * t + cc.x;
        r1 = r1 * t + cc.y;
        r2 = r2 * t + cc.z;
        r3 = r3 * t + cc.w;
    }
    r[0] = r0; r[1] = r1; r[2] = r2; r[3] = r3;
}

template <bool F32>
__device__ __forceinline__ void table1d_t(double X, double* r) {
    if constexpr (F32)
        table1d_f32(X, r);
    else
        table1d(X, r);
}

// 2D tiles of V and V_X (green_inf.rs:78-107): Horner in tx per y power, then in ty
__device__ __forceinline__ void table2d(double X, double Y, double& v, double& vx) {
    int ix = (int)X, iy = (int)Y;
    if (ix >= XT) ix = XT - 1;
    if (iy >= YT) iy = YT - 1;
    double tx = 2.0 * (X - ix) - 1.0, ty = 2.0 * (Y - iy) - 1.0;
    constexpr int M = N2 + 1;
    const double* c = c_tab.t2d + ((size_t)iy * XT + ix) * 2 * M * M;
    double s[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const double* cq = c + q * M * M;
        double r[M];
#pragma unroll
        for (int a = 0; a < M; a++) r[a] = 0.0;
#pragma unroll
        for (int j = M - 1; j >= 0; j--) {
#pragma unroll
            for (int a = 0; a < M; a += 2) {
                double2 cc = __ldg(reinterpret_cast<const double2*>(cq + j * M + a));
                r[a] = r[a] * tx + cc.x;
                r[a + 1] = r[a + 1] * tx + cc.y;
            }
        }
        double acc = 0.0;
#pragma unroll
        for (int a = M - 1; a >= 0; a--) acc = acc * ty + r[a];
        s[q] = acc;
    }
    v = s[0];
    vx = s[1];
}

// table2d from the FP32 copy of the coefficients (the mixed form): per cell and quantity a block of
// T2D_FX x T2D_FY power-basis coefficients (row j: the tx^j terms over the powers of ty), FP32 Horner
// chains.
__device__ __forceinline__ void table2d_f32(double X, double Y, double& v, double& vx) {
    int ix = (int)X, iy = (int)Y;
    if (ix >= XT) ix = XT - 1;
    if (iy >= YT) iy = YT - 1;
    const float tx = (float)(2.0 * (X - ix) - 1.0), ty = (float)(2.0 * (Y - iy) - 1.0);
    const float4* c = reinterpret_cast<const float4*>(c_tab.t2d_f + ((size_t)iy * XT + ix) * 2 * T2D_FB);
    float s[2];
#pragma unroll
    for (int q = 0; q < 2; q++) {
        float cf[T2D_FB];
#pragma unroll
        for (int u = 0; u < T2D_FB / 4; u++) {
            const float4 a = __ldg(c + q * (T2D_FB / 4) + u);
            cf[4 * u] = a.x;
            cf[4 * u + 1] = a.y;
            cf[4 * u + 2] = a.z;
            cf[4 * u + 3] = a.w;
        }
        float r[T2D_FY];
#pragma unroll
        for (int a = 0; a < T2D_FY; a++) r[a] = cf[(T2D_FX - 1) * T2D_FY + a];
#pragma unroll
        for (int j = T2D_FX - 2; j >= 0; j--)
#pragma unroll
            for (int a = 0; a < T2D_FY; a++) r[a] = r[a] * tx + cf[j * T2D_FY + a];
        float acc = r[T2D_FY - 1];
#pragma unroll
        for (int a = T2D_FY - 2; a >= 0; a--) acc = acc * ty + r[a];
        s[q] = acc;
    }
    v = s[0];
    vx = s[1];
}

// Hankel asymptotics J0 Y0 J1 Y1 for x >= XT (green_inf.rs:145-172)
__device__ inline void hankel01(double x, double& j0, double& y0, double& j1, double& y1) {
    double inv = 1.0 / x, inv2 = inv * inv;
    double P[2] = {0, 0}, Q[2] = {0, 0};
#pragma unroll
    for (int nu = 0; nu < 2; nu++) {
        const double* a = c_tab.asy + nu * HANKEL_TERMS;
        double pw = 1.0;
#pragma unroll
        for (int k = 0; 2 * k + 1 < HANKEL_TERMS; k++) {
            double s = (k % 2 != 0) ? -1.0 : 1.0;
            P[nu] += s * __ldg(a + 2 * k) * pw;
            Q[nu] += s * __ldg(a + 2 * k + 1) * pw * inv;
            pw *= inv2;
        }
    }
    double chi = x - 0.25 * PI;
    double sq = sqrt(2.0 / (PI * x));
    double sn, c;
    sincos(chi, &sn, &c);
    j0 = sq * (P[0] * c - Q[0] * sn);
    y0 = sq * (P[0] * sn + Q[0] * c);
    j1 = sq * (P[1] * sn + Q[1] * c);
    y1 = sq * (-P[1] * c + Q[1] * sn);
}

__device__ inline double struve_minus_y(int nu, double x) {
    const double* c = c_tab.asy + 2 * HANKEL_TERMS + nu * STRUVE_TERMS;
    double inv2 = 1.0 / (x * x), s = 0.0, pw = nu == 0 ? 1.0 / x : 1.0;
    for (int k = 0; k < STRUVE_TERMS; k++) {
        s += __ldg(c + k) * pw;
        pw *= inv2;
    }
    return s;
}

// Partial integration of Havelock's integral, adaptive stop (green_inf.rs:189-266)
__device__ inline void taylor_sum(double X, double t0, double& P, double& PX) {
    constexpr int FAR_TERMS = 15;
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
        if (size < 1e-14) break;
    }
    P = p;
    PX = px;
}

__device__ inline void far_series(double X, double Y, double w, double& P, double& PX) {
    taylor_sum(X, Y, P, PX);
    if (w > 1e-17) {
        double P0, PX0;
        taylor_sum(X, 0.0, P0, PX0);
        P -= w * P0;
        PX -= w * PX0;
    }
}

template <bool F32 = false>
__device__ inline void bessel_j01(double X, double& j0, double& j1) {
    if (X < XT) {
        double f[4];
        table1d_t<F32>(X, f);
        j0 = f[0];
        j1 = f[1];
    } else {
        double y0, y1;
        hankel01(X, j0, y0, j1, y1);
    }
}

template <bool F32 = false>
__device__ inline void bessel_jy01(double X, double& j0, double& y0, double& j1, double& y1) {
    if (X >= XT) {
        hankel01(X, j0, y0, j1, y1);
        return;
    }
    double f[4];
    table1d_t<F32>(X, f);
    j0 = f[0];
    j1 = f[1];
    double L = log(0.5 * X) + GAMMA;
    y0 = f[2] + 2.0 / PI * L * f[0];
    y1 = -f[3] - 2.0 / PI * (f[0] / X - L * f[1]);
}

// The wave part Ft, Gi and their derivatives (green_inf.rs:316-368, identity form everywhere in
// [0, XT) x [0, YT): the double-precision rule). w = F, FX, FY, I, IX, IY, c
struct Wave {
    double F, FX, FY, I, IX, IY, c;
};

template <bool F32 = false>
__device__ inline Wave wave_kernel(double X, double Y) {
    Wave o;
    double R0 = sqrt(X * X + Y * Y);
    double eY = exp(-Y), j0, j1, F, FX;
    if (X < XT && Y < YT) {
        double f[4], v, vx;
        table1d_t<F32>(X, f);
        j0 = f[0];
        j1 = f[1];
        if constexpr (F32)
            table2d_f32(X, Y, v, vx);
        else
            table2d(X, Y, v, vx);
        double lg = log(Y + R0) + (GAMMA - LOG2);
        F = -2.0 * eY * j0 * lg - PI * eY * f[2] - 2.0 * R0 * v;
        FX = 2.0 * eY * j1 * lg - 2.0 * eY * j0 * X / (R0 * (Y + R0)) - PI * eY * f[3] - 2.0 * (X / R0) * v -
             2.0 * R0 * vx;
    } else if (Y >= YT) {
        bessel_j01<F32>(X, j0, j1);
        double P, PX;
        far_series(X, Y, 0.0, P, PX);
        F = -2.0 * P;
        FX = -2.0 * PX;
    } else {
        double y0, y1;
        hankel01(X, j0, y0, j1, y1);
        double h0py0 = struve_minus_y(0, X) + 2.0 * y0;
        double dh0py0 = 2.0 / PI - struve_minus_y(1, X) - 2.0 * y1;
        double P, PX;
        far_series(X, Y, eY, P, PX);
        F = -PI * eY * h0py0 - 2.0 * P;
        FX = -PI * eY * dh0py0 - 2.0 * PX;
    }
    o.F = F;
    o.FX = FX;
    o.FY = -F - 2.0 / R0;
    o.c = eY * j0;
    o.I = -2.0 * PI * eY * j0;
    o.IX = 2.0 * PI * eY * j1;
    o.IY = -o.I;
    return o;
}

// real part only (green_inf.rs:647-675)
template <bool F32 = false>
__device__ inline void wave_real(double X, double Y, double& F, double& FX, double& FY) {
    double R0 = sqrt(X * X + Y * Y);
    if (Y >= YT) {
        double P, PX;
        far_series(X, Y, 0.0, P, PX);
        F = -2.0 * P;
        FX = -2.0 * PX;
    } else {
        Wave w = wave_kernel<F32>(X, Y);
        F = w.F;
        FX = w.FX;
    }
    FY = -F - 2.0 / R0;
}

// ------------------------------------------------------------------ finite depth (green_fin.rs)
__device__ inline void scaled_k01(double x, double& g0, double& g1) {
    int i;
    double t;
    if (x < 1.0) {
        i = 0;
        t = 2.0 * (x - K_LO) / (1.0 - K_LO) - 1.0;
    } else {
        i = (int)x;
        t = 2.0 * (x - i) - 1.0;
    }
    const double* c = c_tab.bk + i * (NK + 1) * 2;
    double a0 = 0.0, a1 = 0.0;
    for (int j = NK; j >= 0; j--) {
        double2 cc = __ldg(reinterpret_cast<const double2*>(c + 2 * j));
        a0 = a0 * t + cc.x;
        a1 = a1 * t + cc.y;
    }
    g0 = a0;
    g1 = a1;
}

// Q(s, w) and its derivatives at w1, w2 (green_fin.rs:394-421)
__device__ inline void q_eval2(const double* P, double s, double w1, double w2, double* v, double* vs, double* qw) {
    double y0 = 0.5 * w1 - 1.0, y1 = 0.5 * w2 - 1.0;
    double v0 = 0, v1 = 0, s0 = 0, s1 = 0, d0 = 0, d1 = 0;
    for (int m = FM; m >= 0; m--) {
        const double* c = P + m * NC;
        double p0 = c[NC - 1], p1 = c[NC - 1], dp0 = 0, dp1 = 0;
        for (int k = NC - 2; k >= 0; k--) {
            dp0 = dp0 * y0 + p0;
            p0 = p0 * y0 + c[k];
            dp1 = dp1 * y1 + p1;
            p1 = p1 * y1 + c[k];
        }
        s0 = s0 * s + v0;
        v0 = v0 * s + p0;
        d0 = d0 * s + dp0;
        s1 = s1 * s + v1;
        v1 = v1 * s + p1;
        d1 = d1 * s + dp1;
    }
    v[0] = v0; v[1] = v1;
    vs[0] = s0; vs[1] = s1;
    qw[0] = 0.5 * d0; qw[1] = 0.5 * d1;
}

// Phi, dPhi/dxb, dPhi/dvb directly (green_fin.rs:461-491)
__device__ inline void phi_direct(const FdParams& fd, int which, double xb, double vb, double* out) {
    double q[2], qs[2], qw[2];
    q_eval2(fd.P, xb * xb, vb * vb, vb * vb, q, qs, qw);
    out[0] = q[0];
    out[1] = 2.0 * xb * qs[0];
    out[2] = 2.0 * vb * qw[0];
    if (fd.mode != 0) return;
    double H = fd.H, X = H * xb, H2 = H * H, F, FX, FY;
    if (which == 1) {
        wave_real(X, H * (2.0 - vb), F, FX, FY);
        out[0] += H * F;
        out[1] += H2 * FX;
        out[2] -= H2 * FY;
    }
    wave_real(X, H * (2.0 + vb), F, FX, FY);
    out[0] += H * F;
    out[1] += H2 * FX;
    out[2] += H2 * FY;
}

// Phi and its two derivatives from the per-frequency tiles (green_fin.rs:566-600)
__device__ __forceinline__ void phi_tiles(const double* T, int which, double xb, double vb, double* v) {
    constexpr int N = TN;
    static_assert(TN == 6, "the vectorized Horner chain below is written for degree-5 tiles");
    int ny = which == 1 ? TW : TV;
    double ymax = which == 1 ? 1.0 : 2.0;
    double ux = xb * (TS / XMAX), uy = vb * (ny / ymax);
    int ix = (int)ux, iy = (int)uy;
    if (ix > TS - 1) ix = TS - 1;
    if (iy > ny - 1) iy = ny - 1;
    double tx = 2.0 * (ux - ix) - 1.0, ty = 2.0 * (uy - iy) - 1.0;
    const double* c = T + (size_t)(ix * ny + iy) * 3 * N * N;
    double v0 = 0, v1 = 0, v2 = 0;
    // rows of N = 6 coefficients, 16-byte aligned: three double2 loads a row
#pragma unroll
    for (int i = N - 1; i >= 0; i--) {
        double pq[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const double2* r = reinterpret_cast<const double2*>(c + q * N * N + i * N);
            double2 a = __ldg(r), b = __ldg(r + 1), d = __ldg(r + 2);
            double p = d.y;
            p = p * ty + d.x;
            p = p * ty + b.y;
            p = p * ty + b.x;
            p = p * ty + a.y;
            p = p * ty + a.x;
            pq[q] = p;
        }
        v0 = v0 * tx + pq[0];
        v1 = v1 * tx + pq[1];
        v2 = v2 * tx + pq[2];
    }
    v[0] = v0; v[1] = v1; v[2] = v2;
}

// phi_tiles from the FP32 tiles of the mixed form: per tile 3 blocks of TFB coefficients of degree
// TFD in each variable, FP32 Horner chains.
__device__ __forceinline__ void phi_tiles_f32(const float* T, int which, double xb, double vb, double* v) {
    constexpr int N = TFN;
    int ny = which == 1 ? TW : TV;
    double ymax = which == 1 ? 1.0 : 2.0;
    double ux = xb * (TS / XMAX), uy = vb * (ny / ymax);
    int ix = (int)ux, iy = (int)uy;
    if (ix > TS - 1) ix = TS - 1;
    if (iy > ny - 1) iy = ny - 1;
    const float tx = (float)(2.0 * (ux - ix) - 1.0), ty = (float)(2.0 * (uy - iy) - 1.0);
    const float4* c = reinterpret_cast<const float4*>(T + (size_t)(ix * ny + iy) * 3 * TFB);
#pragma unroll
    for (int q = 0; q < 3; q++) {
        float cf[TFB];
#pragma unroll
        for (int u = 0; u < TFB / 4; u++) {
            const float4 a = __ldg(c + q * (TFB / 4) + u);
            cf[4 * u] = a.x;
            cf[4 * u + 1] = a.y;
            cf[4 * u + 2] = a.z;
            cf[4 * u + 3] = a.w;
        }
        float vq = 0.f;
#pragma unroll
        for (int i = N - 1; i >= 0; i--) {
            float p = cf[i * N + N - 1];
#pragma unroll
            for (int j = N - 2; j >= 0; j--) p = p * ty + cf[i * N + j];
            vq = vq * tx + p;
        }
        v[q] = vq;
    }
}

// Regular part of the kernel: Wr WrR WrZ Wrz Wi WiR WiZ Wiz (green_fin.rs:48-60 Kern)
struct Kern {
    double Wr, WrR, WrZ, Wrz, Wi, WiR, WiZ, Wiz;
};

// low_order.rs:717-730 wave_kern: infinite depth, ordinary frequency
__device__ __forceinline__ Kern wave_kern(double K, const Wave& w) {
    double K2 = K * K;
    Kern k;
    k.Wr = K * w.F;
    k.WrR = K2 * w.FX;
    k.WrZ = -K2 * w.FY;
    k.Wrz = k.WrZ;
    k.Wi = K * w.I;
    k.WiR = K2 * w.IX;
    k.WiZ = -K2 * w.IY;
    k.Wiz = k.WiZ;
    return k;
}

// low_order.rs:627-648 pair_kernel, infinite depth
template <bool F32 = false>
__device__ inline Kern pair_kernel_inf(double K, double R, double z, double zeta) {
    if (R == 0.0 && z == 0.0 && zeta == 0.0) {
        Kern k = {};
        k.Wr = -2.0 * K * (GAMMA - LOG2 + log(K));
        k.Wi = -2.0 * PI * K;
        return k;
    }
    return wave_kern(K, wave_kernel<F32>(K * R, -K * (z + zeta)));
}

// green_fin.rs:1007-1095 finite_kernel with the fin_point data of both points.
// fz / fzeta: pointers to the plane-0 entry of the point in the fin_point planes (stride N).
// SW: the infinite-depth wave term F3 at (K R, K v3) is supplied by the caller (*sw, when not null).
template <bool F32 = false, class TT = double, bool SW = false>
__device__ inline Kern finite_kernel(const FdParams& fd, const TT* T1, const TT* T2, double R, double z,
                                     double zeta, const double* fz, const double* fzeta, int stride,
                                     const Wave* sw = nullptr) {
    double h = fd.h;
    double d1 = z - zeta;
    double sg = d1 > 0.0 ? 1.0 : d1 < 0.0 ? -1.0 : 0.0;
    double v[6] = {fabs(d1), z + zeta + 2.0 * h, -(z + zeta), d1 + 2.0 * h, -d1 + 2.0 * h, z + zeta + 4.0 * h};
    bool ordinary = fd.mode == 0;
    double e0 = 0, e1 = 0, e2 = 0;
    if (ordinary) {
        double e3 = fz[0] * fzeta[0];
        double e4 = fz[stride] * fzeta[2 * stride];
        double e5 = fz[2 * stride] * fzeta[stride];
        double e6 = fz[3 * stride] * fzeta[3 * stride];
        e0 = e3 + e4 + e5 + e6;
        e1 = fd.k0 * (e3 + e4 - e5 - e6);
        e2 = fd.k0 * (e3 - e4 + e5 - e6);
    }
    Kern o = {};
    if (R >= 0.5 * h) {
        double re = 0, reR = 0, reZ = 0, rez = 0;
        for (int n = 0; n < FIN_ROOTS; n++) {
            double k = fd.kn[n], x = k * R;
            if (x >= SERIES_STOP) break;
            double g0, g1;
            scaled_k01(x, g0, g1);
            double ex = exp(-x) / sqrt(x);
            double K0 = g0 * ex, K1 = g1 * ex;
            double cz = fz[(4 + 2 * n) * stride], sz = fz[(5 + 2 * n) * stride];
            double cs = fzeta[(4 + 2 * n) * stride], ss = fzeta[(5 + 2 * n) * stride];
            double c = fd.cn[n];
            re += c * cz * cs * K0;
            reR -= c * cz * cs * k * K1;
            reZ -= c * cz * k * ss * K0;
            rez -= c * k * sz * cs * K0;
        }
        if (ordinary) {
            double j0, y0, j1, y1;
            bessel_jy01<F32>(fd.k0 * R, j0, y0, j1, y1);
            re += -fd.A0 * e0 * y0;
            reR += fd.A0 * e0 * fd.k0 * y1;
            reZ += -fd.A0 * e1 * y0;
            rez += -fd.A0 * e2 * y0;
            o.Wi = -fd.A0 * e0 * j0;
            o.WiR = fd.A0 * e0 * fd.k0 * j1;
            o.WiZ = -fd.A0 * e1 * j0;
            o.Wiz = -fd.A0 * e2 * j0;
        } else if (fd.mode == 1) {
            re += -2.0 / h * (log(R / (2.0 * h)) + GAMMA);
            reR += -2.0 / (h * R);
        }
        const double dvz[6] = {-sg, 1.0, -1.0, -1.0, 1.0, 1.0};
        const double dvf[6] = {sg, 1.0, -1.0, 1.0, -1.0, 1.0};
#pragma unroll
        for (int p = 0; p < 6; p++) {
            double r2 = R * R + v[p] * v[p], r = sqrt(r2);
            double ir3 = fd.sign[p] / (r2 * r);
            re -= fd.sign[p] / r;
            reR += R * ir3;
            reZ += v[p] * dvz[p] * ir3;
            rez += v[p] * dvf[p] * ir3;
        }
        o.Wr = re;
        o.WrR = reR;
        o.WrZ = reZ;
        o.Wrz = rez;
        return o;
    }
    double ih = 1.0 / h, ih2 = ih * ih, f1[3], f2[3];
    if constexpr (F32) {
        phi_tiles_f32(T1, 1, R * ih, v[0] * ih, f1);
        phi_tiles_f32(T2, 2, R * ih, v[1] * ih, f2);
    } else {
        phi_tiles(T1, 1, R * ih, v[0] * ih, f1);
        phi_tiles(T2, 2, R * ih, v[1] * ih, f2);
    }
    o.Wr = ih * (f1[0] + f2[0]);
    o.WrR = ih2 * (f1[1] + f2[1]);
    double A1z = -sg * ih2 * f1[2], Bz = ih2 * f2[2];
    if (ordinary) {
        double K = fd.K, F3, F3X, F3Y;
        if (R == 0.0 && v[2] == 0.0) {  // wave_real_or_limit (green_fin.rs:803-808)
            F3 = -2.0 * (GAMMA - LOG2 + log(K));
            F3X = 0.0;
            F3Y = 0.0;
        } else {
            if constexpr (SW) {
                if (sw) {
                    F3 = sw->F;
                    F3X = sw->FX;
                    F3Y = sw->FY;
                } else {
                    wave_real<F32>(K * R, K * v[2], F3, F3X, F3Y);
                }
            } else {
                wave_real<F32>(K * R, K * v[2], F3, F3X, F3Y);
            }
        }
        o.Wr += K * F3;
        o.WrR += K * K * F3X;
        Bz -= K * K * F3Y;
        double j0, j1;
        bessel_j01<F32>(fd.k0 * R, j0, j1);
        o.Wi = -fd.A0 * e0 * j0;
        o.WiR = fd.A0 * e0 * fd.k0 * j1;
        o.WiZ = -fd.A0 * e1 * j0;
        o.Wiz = -fd.A0 * e2 * j0;
    }
    o.WrZ = A1z + Bz;
    o.Wrz = -A1z + Bz;
    return o;
}

}  // namespace hbg
