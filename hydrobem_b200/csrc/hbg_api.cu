// hbg_api.cu -- host orchestration and the C ABI of libhydrobem_gpu.so.
//
// The solve of one body: panel geometry and the static influence data once (device), then the
// frequencies in batches sized to the free device memory: per batch the finite-depth tiles, the
// assembly of S and A, boundary values, right-hand sides, LU, substitution and forces, all on one
// stream, results copied back once per batch.  The host only computes per-frequency scalars
// (dispersion roots and the finite-depth power table, solve_common.rs:44-71) and checks statuses.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hydrobem_gpu.h"
#include "hbg_internal.h"
#include "hbg_mixed.h"

extern "C" const unsigned char hbg_tables_blob[];
extern "C" const unsigned char hbg_tables_blob_end[];

namespace hbg {

// ------------------------------------------------------------------ errors (per thread)
static thread_local std::string g_error;
static thread_local HbLocation g_location = {-1, -1, -1, -1, -1, -1};
static thread_local double g_profile[6];
static thread_local int64_t g_launches;

static thread_local KernelProfiler* g_prof = nullptr;
static thread_local Workspace* g_ws[16] = {};

Workspace& workspace() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 16) dev = 0;
    if (!g_ws[dev]) g_ws[dev] = new Workspace();
    return *g_ws[dev];
}
KernelProfiler& profiler() {
    if (!g_prof) g_prof = new KernelProfiler();
    return *g_prof;
}

struct Failure {
    HbStatus code;
    std::string msg;
    int64_t body = -1, frequency = -1;
};

static HbStatus fail(const Failure& f) {
    g_error = f.msg;
    g_location = HbLocation{f.body, -1, -1, -1, -1, f.frequency};
    return f.code;
}

#define CUDA_OK(expr)                                                                                   \
    do {                                                                                                \
        cudaError_t _e = (expr);                                                                        \
        if (_e != cudaSuccess) throw Failure{HB_ERR_INTERNAL, std::string("CUDA: ") + cudaGetErrorString(_e)}; \
    } while (0)

// ------------------------------------------------------------------ tables
struct HostTables {
    const double* arr[8] = {};
    size_t len[8] = {};
    bool ok = false;
    std::string why;
};

static uint64_t fnv1a(const double* v, size_t n, uint64_t h) {
    const unsigned char* b = reinterpret_cast<const unsigned char*>(v);
    for (size_t i = 0; i < n * 8; i++) {
        h ^= b[i];
        h *= 0x100000001B3ull;
    }
    return h;
}

// The embedded blob (tables/green_tables.bin): header, then eight float64 arrays; the checksums of
// the reference (green_inf.rs:268-283, green_fin.rs:853-868).
static const HostTables& host_tables() {
    static HostTables t;
    static std::once_flag once;
    std::call_once(once, [] {
        const unsigned char* p = hbg_tables_blob;
        size_t size = (size_t)(hbg_tables_blob_end - hbg_tables_blob);
        if (size < 16 || memcmp(p, "HBGTBL01", 8) != 0) {
            t.why = "Green-function tables: bad header";
            return;
        }
        uint64_t cnt;
        memcpy(&cnt, p + 8, 8);
        if (cnt != 8) {
            t.why = "Green-function tables: unexpected array count";
            return;
        }
        static const size_t want[8] = {2040, 115200, 176400, 56, 65, 24570, 130, 1728};
        size_t off = 16 + 8 * 24;
        for (int i = 0; i < 8; i++) {
            uint64_t n;
            memcpy(&n, p + 16 + i * 24 + 16, 8);
            if (n != want[i]) {
                t.why = "Green-function tables: unexpected array length";
                return;
            }
            t.arr[i] = reinterpret_cast<const double*>(p + off);
            t.len[i] = n;
            off += n * 8;
        }
        if (off != size) {
            t.why = "Green-function tables: size mismatch";
            return;
        }
        uint64_t hi = 0xCBF29CE484222325ull, hf = 0xCBF29CE484222325ull;
        for (int i = 0; i < 4; i++) hi = fnv1a(t.arr[i], t.len[i], hi);
        for (int i = 4; i < 8; i++) hf = fnv1a(t.arr[i], t.len[i], hf);
        if (hi != 0xCAC816A5E6E5C8F2ull || hf != 0x4982F563A8976372ull) {
            t.why = "Green-function tables fail their checksum";
            return;
        }
        t.ok = true;
    });
    return t;
}

// Gauss-Legendre nodes and weights of orders 1..16 (quadrature.rs:17-62: Newton on P_n)
static void gauss_legendre(int n, double* x, double* w) {
    double nf = n;
    for (int i = 0; i < (n + 1) / 2; i++) {
        double z = std::cos(PI * (i + 0.75) / (nf + 0.5)), dp = 1.0;
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
            if (std::fabs(dz) <= 1e-16) break;
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

// Chebyshev truncation of a power-basis block on [-1, 1]^2: p[i * ps + j] (n1 x n2) the coefficient
// of t1^i t2^j, re-expanded in Chebyshev polynomials T_a(t1) T_b(t2), the series cut to a < m1,
// b < m2 and returned to the power basis in o[i * m2 + j] (m1 x m2).
static void cheb_truncate(const double* p, int ps, int n1, int n2, int m1, int m2, double* o) {
    constexpr int NMAX = 17;
    double cp[NMAX][NMAX] = {};  // cp[j][k]: coefficient of t^k in T_j
    cp[0][0] = 1.0;
    cp[1][1] = 1.0;
    for (int j = 2; j < NMAX; j++)
        for (int k = 0; k < NMAX; k++) cp[j][k] = (k > 0 ? 2.0 * cp[j - 1][k - 1] : 0.0) - cp[j - 2][k];
    std::vector<double> c((size_t)n1 * n2);
    for (int i = 0; i < n1; i++)
        for (int j = 0; j < n2; j++) c[(size_t)i * n2 + j] = p[(size_t)i * ps + j];
    // power -> Chebyshev along t2 (rows), then t1 (columns): p_k = sum_j c_j cp[j][k], top degree first
    for (int i = 0; i < n1; i++)
        for (int j = n2 - 1; j >= 0; j--) {
            double cj = c[(size_t)i * n2 + j] / cp[j][j];
            for (int k = 0; k < j; k++) c[(size_t)i * n2 + k] -= cj * cp[j][k];
            c[(size_t)i * n2 + j] = cj;
        }
    for (int j = 0; j < n2; j++)
        for (int i = n1 - 1; i >= 0; i--) {
            double ci = c[(size_t)i * n2 + j] / cp[i][i];
            for (int k = 0; k < i; k++) c[(size_t)k * n2 + j] -= ci * cp[i][k];
            c[(size_t)i * n2 + j] = ci;
        }
    for (int ki = 0; ki < m1; ki++)
        for (int kj = 0; kj < m2; kj++) {
            double acc = 0.0;
            for (int a = ki; a < m1; a++)
                for (int b = kj; b < m2; b++) acc += c[(size_t)a * n2 + b] * cp[a][ki] * cp[b][kj];
            o[ki * m2 + kj] = acc;
        }
}

struct DeviceCtx {
    bool ready = false;
    double* tables = nullptr;
    float* t2d_f = nullptr;
    float* t1d_f = nullptr;
    Tables tab{};
};

static std::mutex g_dev_mutex;
static DeviceCtx g_dev[16];

static DeviceCtx& device_ctx(int dev) {
    std::lock_guard<std::mutex> lock(g_dev_mutex);
    if (dev < 0 || dev >= 16) throw Failure{HB_ERR_ARGUMENT, "device ordinal out of range"};
    DeviceCtx& d = g_dev[dev];
    if (d.ready) return d;
    const HostTables& ht = host_tables();
    if (!ht.ok) throw Failure{HB_ERR_INTERNAL, ht.why};
    // every array at a 256-byte boundary (the kernels read the tables as double2)
    auto padded = [](size_t n) { return (n + 31) / 32 * 32; };
    size_t total = 0;
    for (int i = 0; i < 8; i++) total += padded(ht.len[i]);
    CUDA_OK(cudaMalloc(&d.tables, total * sizeof(double)));
    size_t off = 0;
    const double* dp[8];
    for (int i = 0; i < 8; i++) {
        CUDA_OK(cudaMemcpy(d.tables + off, ht.arr[i], ht.len[i] * sizeof(double), cudaMemcpyHostToDevice));
        dp[i] = d.tables + off;
        off += padded(ht.len[i]);
    }
    // The mixed form's FP32 copies of TABLE_2D (cells [YT][XT], per quantity 8 x 8 coefficients, row
    // j the tx^j terms) and TABLE_1D (cells [XT], N1 + 1 terms of 4 quantities), their Chebyshev
    // series cut to T2D_FX x T2D_FY and T1D_FN terms
    constexpr int M2 = N2 + 1;
    std::vector<float> t2f((size_t)XT * YT * 2 * T2D_FB, 0.f);
    double blk[M2 * M2];
    for (int cell = 0; cell < XT * YT; cell++)
        for (int q = 0; q < 2; q++) {
            cheb_truncate(ht.arr[1] + ((size_t)cell * 2 + q) * M2 * M2, M2, M2, M2, T2D_FX, T2D_FY, blk);
            for (int k = 0; k < T2D_FX * T2D_FY; k++) t2f[((size_t)cell * 2 + q) * T2D_FB + k] = (float)blk[k];
        }
    CUDA_OK(cudaMalloc(&d.t2d_f, t2f.size() * sizeof(float)));
    CUDA_OK(cudaMemcpy(d.t2d_f, t2f.data(), t2f.size() * sizeof(float), cudaMemcpyHostToDevice));
    std::vector<float> t1f((size_t)XT * T1D_FN * 4);
    for (int cell = 0; cell < XT; cell++)
        for (int q = 0; q < 4; q++) {
            // the terms of quantity q sit at stride 4: a 17 x 1 block with row stride 4
            cheb_truncate(ht.arr[0] + (size_t)cell * (N1 + 1) * 4 + q, 4, N1 + 1, 1, T1D_FN, 1, blk);
            for (int k = 0; k < T1D_FN; k++) t1f[((size_t)cell * T1D_FN + k) * 4 + q] = (float)blk[k];
        }
    CUDA_OK(cudaMalloc(&d.t1d_f, t1f.size() * sizeof(float)));
    CUDA_OK(cudaMemcpy(d.t1d_f, t1f.data(), t1f.size() * sizeof(float), cudaMemcpyHostToDevice));
    d.tab = Tables{dp[0], dp[1], dp[2], dp[3], dp[4], dp[5], dp[6], dp[7], d.t2d_f, d.t1d_f};
    static double glx[17][16], glw[17][16];
    memset(glx, 0, sizeof glx);
    memset(glw, 0, sizeof glw);
    for (int n = 1; n <= 16; n++) gauss_legendre(n, glx[n], glw[n]);
    set_constants(glx, glw, d.tab);
    set_constants_statics(glx, glw);
    CUDA_OK(cudaGetLastError());
    lu_tune_device(dev);  // before any solve's work is queued on the device
    d.ready = true;
    return d;
}

// ------------------------------------------------------------------ finite-depth scalars (host)
// dispersion.rs:19-95
double dispersion_x0(double H) {
    if (!(H > 0.0)) return 0.0;
    if (H >= 40.0) return H;
    double lo = std::max(H, std::sqrt(H)), hi = 0.5 * (H + std::sqrt(H * H + 4.0 * H));
    double x = H < 1.0 ? std::sqrt(H) * (1.0 + H / 6.0) : H;
    x = std::min(std::max(x, lo), hi);
    double prev = -1.0;
    for (int it = 0; it < 200; it++) {
        double t = std::tanh(x), f = x * t - H;
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

static double dispersion_xn(double H, int n) {
    double npi = n * PI;
    if (!(H > 0.0)) return npi;
    if (std::isinf(H)) return npi - 0.5 * PI;
    double lo = 0.0, hi = 0.5 * PI, d = std::atan(H / (npi - 0.25 * PI)), prev = -1.0;
    for (int it = 0; it < 200; it++) {
        double s = std::sin(d), c = std::cos(d);
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

// green_fin.rs:345-392 region coefficients and power table, 874-934 make_finite_depth (ordinary)
void make_fd_params(double h, double K, FdParams& fd) {
    const HostTables& ht = host_tables();
    const double *meta = ht.arr[4], *Q = ht.arr[5], *L0 = ht.arr[6];
    memset(&fd, 0, sizeof fd);
    fd.mode = 0;
    fd.h = h;
    for (int p = 0; p < 6; p++) fd.sign[p] = 1.0;
    fd.K = K;
    fd.H = K * h;
    double x0 = dispersion_x0(fd.H);
    fd.k0 = x0 / h;
    fd.A0 = 2.0 * PI * fd.k0 / (-std::expm1(-4.0 * x0) + 4.0 * x0 * std::exp(-2.0 * x0));
    for (int n = 1; n <= FIN_ROOTS; n++) {
        double k = dispersion_xn(fd.H, n) / h;
        fd.kn[n - 1] = k;
        fd.cn[n - 1] = 4.0 * (k * k + K * K) / (k * k * h + K * K * h - K);
    }
    double cw[(FM + 1) * NC];
    auto region = [&](int r, double x) {
        const double* m = meta + 5 * r;
        double a = m[1], b = m[2];
        int n = (int)m[3];
        const double* c = Q + (size_t)m[4];
        double y = 2.0 * (x - a) / (b - a) - 1.0, Tx[64];
        Tx[0] = 1.0;
        Tx[1] = y;
        for (int j = 2; j <= n; j++) Tx[j] = 2.0 * y * Tx[j - 1] - Tx[j - 2];
        for (int mm = 0; mm <= FM; mm++)
            for (int jw = 0; jw < NC; jw++) {
                double s = 0.0;
                for (int jx = 0; jx <= n; jx++) s += c[(mm * (n + 1) + jx) * NC + jw] * Tx[jx];
                cw[mm * NC + jw] = s;
            }
    };
    if (fd.H < 1e-12) {
        memcpy(cw, L0, sizeof cw);
        cw[0] -= 0.5 * std::log(fd.H);
    } else if (fd.H >= 50.0) {
        region(REGIONS - 1, 1.0 / fd.H);
    } else {
        double tau = std::log(fd.H);
        int r = 0;
        while (r + 2 < REGIONS && tau > meta[5 * r + 2]) r++;
        region(r, tau);
    }
    double a[NC][NC] = {};
    a[0][0] = 1.0;
    a[1][1] = 1.0;
    for (int j = 2; j < NC; j++)
        for (int k = 0; k < NC; k++) a[j][k] = (k > 0 ? 2.0 * a[j - 1][k - 1] : 0.0) - a[j - 2][k];
    for (int m = 0; m <= FM; m++) {
        const double* c = cw + m * NC;
        double* p = fd.P + m * NC;
        for (int k = 0; k < NC; k++) p[k] = c[0] * a[0][k] + c[1] * a[1][k];
        for (int j = 2; j < NC; j++)
            for (int k = 0; k < NC; k++) p[k] += c[j] * a[j][k];
    }
}

// ------------------------------------------------------------------ device buffers
// A slot of the per-thread workspace (kept across calls).
struct WsBuf {
    Workspace& ws;
    int slot;
    void* p = nullptr;
    size_t bytes = 0;
    WsBuf(Workspace& w, int s) : ws(w), slot(s) {}
    void alloc(size_t b) {
        p = ws.get(slot, b);
        if (!p) throw Failure{HB_ERR_INTERNAL, "device memory allocation failed"};
        bytes = b;
    }
    template <class T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    void alloc(size_t b) {
        if (b <= bytes) return;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        CUDA_OK(cudaMalloc(&p, b));
        bytes = b;
    }
    template <class T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

static bool finite_depth(double d) { return std::isfinite(d) && d > 0.0; }

// One body through the whole path; outputs to the caller's host arrays.
// The panels of a body given as one symmetry sector followed by their mirror images (image g of panel n
// at g Ns + n; reflections in the order e, x, y, xy of the character table; a mirrored quadrilateral
// has its vertex order reversed so that its normal still points into the fluid), with the kinds and
// the bodies of the images those of their sector panels.
static void mirror_sector(const HbgBody& b, int G, std::vector<double>& v, std::vector<int32_t>& kind,
                          std::vector<int32_t>& body) {
    const size_t Ns = (size_t)b.n_panels;
    std::vector<std::pair<double, double>> refl = {{1.0, 1.0}};
    if (b.symmetry == HBG_SYM_YZ || b.symmetry == HBG_SYM_BOTH) refl.push_back({-1.0, 1.0});
    if (b.symmetry == HBG_SYM_XZ || b.symmetry == HBG_SYM_BOTH) refl.push_back({1.0, -1.0});
    if (b.symmetry == HBG_SYM_BOTH) refl.push_back({-1.0, -1.0});
    v.resize(12 * Ns * G);
    kind.resize(Ns * G);
    body.resize(b.panel_body ? Ns * G : 0);
    for (int g = 0; g < G; g++) {
        const double sx = refl[g].first, sy = refl[g].second;
        const bool flip = sx * sy < 0.0;
        for (size_t p = 0; p < Ns; p++) {
            double* o = &v[12 * (g * Ns + p)];
            for (int i = 0; i < 4; i++) {
                const double* q = b.vertices + 12 * p + 3 * (flip && (i & 1) ? 4 - i : i);
                o[3 * i] = sx * q[0];
                o[3 * i + 1] = sy * q[1];
                o[3 * i + 2] = q[2];
            }
            kind[g * Ns + p] = b.kinds ? b.kinds[p] : HBG_WET;
            if (b.panel_body) body[g * Ns + p] = b.panel_body[p];
        }
    }
}

// The panels (n of them, vertices [n][4][3]) in the Morton order of their centroids (10 bits an axis over
// the bounding box; ties in the given order): a[j] the given index of the j-th panel.  Empty for fewer than
// 64 panels or non-finite coordinates (the given order; the geometry reports the latter).
static std::vector<int32_t> spatial_order(const double* v, int64_t n) {
    if (n < 64) return {};
    std::vector<double> c(3 * (size_t)n);
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t j = 0; j < n; j++)
        for (int d = 0; d < 3; d++) {
            const double* q = v + 12 * (size_t)j + d;
            const double x = 0.25 * (q[0] + q[3] + q[6] + q[9]);
            if (!std::isfinite(x)) return {};
            c[3 * (size_t)j + d] = x;
            lo[d] = std::min(lo[d], x);
            hi[d] = std::max(hi[d], x);
        }
    auto spread = [](uint64_t x) {  // the 10 bits of x at every third position
        x &= 0x3ff;
        x = (x | (x << 16)) & 0x030000FFull;
        x = (x | (x << 8)) & 0x0300F00Full;
        x = (x | (x << 4)) & 0x030C30C3ull;
        x = (x | (x << 2)) & 0x09249249ull;
        return x;
    };
    std::vector<std::pair<uint64_t, int32_t>> key((size_t)n);
    for (int64_t j = 0; j < n; j++) {
        uint64_t code = 0;
        for (int d = 0; d < 3; d++) {
            const double span = hi[d] - lo[d];
            const uint64_t q = span > 0.0 ? (uint64_t)std::min(1023.0, std::floor((c[3 * (size_t)j + d] - lo[d]) / span * 1023.0)) : 0;
            code |= spread(q) << d;
        }
        key[(size_t)j] = {code, (int32_t)j};
    }
    std::stable_sort(key.begin(), key.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::vector<int32_t> a((size_t)n);
    for (int64_t j = 0; j < n; j++) a[(size_t)j] = key[(size_t)j].second;
    return a;
}

static void solve_problem(const HbgProblem& pr_in, const HbgOptions& opt, int64_t body_index, cudaStream_t s) {
    const int64_t N64 = pr_in.body.n_panels;
    if (N64 < 1 || N64 > 60000) throw Failure{HB_ERR_VALUE, "panel count outside 1..60000", body_index};
    // symmetry sectors: G systems of Nm = n_panels unknowns per frequency over the N = G Nm panels
    const int sym = pr_in.body.symmetry;
    if (sym < HBG_SYM_NONE || sym > HBG_SYM_BOTH) throw Failure{HB_ERR_VALUE, "symmetry outside 0..3", body_index};
    const int G = sym == HBG_SYM_BOTH ? 4 : sym != HBG_SYM_NONE ? 2 : 1;
    if (G > 1 && opt.precision == HBG_MIXED && opt.surrogate)
        throw Failure{HB_ERR_UNSUPPORTED, "symmetry sectors with the wave-term network are not on this route", body_index};
    // The stored panels in the Morton order of their centroids: the 32 x 32 panel pairs of an assembly tile
    // then lie close together, so the table cells of their wave kernels differ less across a warp (fewer
    // L1 wavefronts per coefficient gather).  The outputs are sums over the panels: the order changes only
    // their rounding; an invalid panel is still reported by its index in the caller's order.
    std::vector<int32_t> perm = spatial_order(pr_in.body.vertices, N64);
    std::vector<double> pverts;
    std::vector<int32_t> pkinds, pbody;
    HbgProblem pin = pr_in;
    if (!perm.empty()) {
        const size_t n = perm.size();
        pverts.resize(12 * n);
        for (size_t a = 0; a < n; a++)
            memcpy(&pverts[12 * a], pr_in.body.vertices + 12 * (size_t)perm[a], 12 * sizeof(double));
        pin.body.vertices = pverts.data();
        if (pr_in.body.kinds) {
            pkinds.resize(n);
            for (size_t a = 0; a < n; a++) pkinds[a] = pr_in.body.kinds[perm[a]];
            pin.body.kinds = pkinds.data();
        }
        if (pr_in.body.panel_body) {
            pbody.resize(n);
            for (size_t a = 0; a < n; a++) pbody[a] = pr_in.body.panel_body[perm[a]];
            pin.body.panel_body = pbody.data();
        }
    }
    HbgProblem pr = pin;
    std::vector<double> mverts;
    std::vector<int32_t> mkinds, mbody;
    if (G > 1) {
        mirror_sector(pin.body, G, mverts, mkinds, mbody);
        pr.body.n_panels = N64 * G;
        pr.body.vertices = mverts.data();
        pr.body.kinds = mkinds.data();
        pr.body.panel_body = pin.body.panel_body ? mbody.data() : nullptr;
    }
    const int N = (int)(N64 * G), Nm = (int)N64;
    // the caller's index of every panel (the images of a sector after it, sector by sector)
    std::vector<int32_t> orig;
    if (!perm.empty()) {
        orig.resize(N);
        for (int j = 0; j < N; j++) orig[j] = (j / Nm) * Nm + perm[j % Nm];
    }
    const int F = (int)pr.n_omega, H = (int)pr.n_heading;
    for (int i = 0; i < F; i++)
        if (!(pr.omegas[i] > 0.0) || !std::isfinite(pr.omegas[i]))
            throw Failure{HB_ERR_VALUE, "an omega is not positive and finite (the limits are not on this route)",
                          body_index, i};
    // interacting bodies: 6 rigid modes each
    const int nbod = pr.body.n_bodies > 1 ? (int)pr.body.n_bodies : 1;
    if (pr.body.n_bodies < 0 || nbod > 64) throw Failure{HB_ERR_VALUE, "n_bodies outside 0..64", body_index};
    if (nbod > 1 && !pr.body.panel_body) throw Failure{HB_ERR_ARGUMENT, "several bodies without panel_body", body_index};
    if (pr.body.panel_body)
        for (int j = 0; j < N; j++)
            if (pr.body.panel_body[j] < 0 || pr.body.panel_body[j] >= nbod)
                throw Failure{HB_ERR_VALUE, "a panel_body entry outside 0 .. n_bodies - 1", body_index};
    if (pr.body.rotation_centers)
        for (int i = 0; i < 3 * nbod; i++)
            if (!std::isfinite(pr.body.rotation_centers[i]))
                throw Failure{HB_ERR_VALUE, "a rotation centre is not finite", body_index};
    const int D = 6 * nbod;
    if (D + H > 32) throw Failure{HB_ERR_UNSUPPORTED, "more than 32 right-hand sides (6 per body and one per heading)", body_index};
    // motions (motion.rs) need the rigid-body data; the hydrostatics records need only the panels
    const HbgRigid* rigid = pr.rigid;
    // the Kochin functions and the momentum drift (the motions enter when the rigid data are given)
    const int TK = pr.kochin_angles > 0 && H > 0 ? pr.kochin_angles : 0;
    if (pr.kochin_angles < 0) throw Failure{HB_ERR_VALUE, "negative Kochin angle count", body_index};
    if ((size_t)TK * H > (size_t)KOCHIN_MAX_HT)
        throw Failure{HB_ERR_UNSUPPORTED, "Kochin angles x headings above 4096", body_index};
    const bool motions = pr.out.motions != nullptr && H > 0;
    if (pr.out.motions && !rigid)
        throw Failure{HB_ERR_VALUE, "motions need the rigid-body data (mass, centre of gravity, inertia)", body_index};
    if (rigid) {
        if (!rigid->mass || !rigid->center_of_gravity || !rigid->inertia || !rigid->inertia_origin)
            throw Failure{HB_ERR_ARGUMENT, "rigid data without mass, centre of gravity, inertia or its origin", body_index};
        for (int b = 0; b < nbod; b++) {
            const double m = rigid->mass[b];
            if (!(std::isnan(m) || (m >= 0.0 && std::isfinite(m))))
                throw Failure{HB_ERR_VALUE, "a mass is negative or infinite", body_index};
            const int k = rigid->inertia_kind ? rigid->inertia_kind[b] : HBG_INERTIA_COMPONENTS;
            if (k != HBG_INERTIA_COMPONENTS && k != HBG_INERTIA_GYRATION)
                throw Failure{HB_ERR_VALUE, "inertia_kind is neither components nor radii of gyration", body_index};
            for (int i = 0; i < 3; i++)
                if (!std::isfinite(rigid->center_of_gravity[3 * b + i]) || !std::isfinite(rigid->inertia_origin[3 * b + i]))
                    throw Failure{HB_ERR_VALUE, "a centre of gravity or inertia origin is not finite", body_index};
            for (int i = 0; i < 9; i++)
                if (!std::isfinite(rigid->inertia[9 * b + i]))
                    throw Failure{HB_ERR_VALUE, "an inertia entry is not finite", body_index};
        }
        for (int i = 0; i < D * D; i++)
            if ((rigid->stiffness && !std::isfinite(rigid->stiffness[i])) ||
                (rigid->damping && !std::isfinite(rigid->damping[i])))
                throw Failure{HB_ERR_VALUE, "an additional stiffness or damping entry is not finite", body_index};
    }
    const bool hydro = rigid || pr.out.hydrostatics;
    // field points (lo_frequency.rs:1392-1470): in the fluid at z <= 0, above the sea bed
    const int nfp = pr.field_points && pr.n_field_points > 0 ? (int)pr.n_field_points : 0;
    if (pr.n_field_points < 0 || pr.n_field_points > 100000)
        throw Failure{HB_ERR_VALUE, "n_field_points outside 0..100000", body_index};
    for (int p = 0; p < nfp; p++) {
        const double* q = pr.field_points + 3 * p;
        if (!std::isfinite(q[0]) || !std::isfinite(q[1]) || !std::isfinite(q[2]) || q[2] > 0.0)
            throw Failure{HB_ERR_VALUE, "a field point is not finite or lies above the free surface", body_index};
        if (finite_depth(opt.depth) && q[2] < -opt.depth)
            throw Failure{HB_ERR_VALUE, "a field point lies below the sea bed", body_index};
    }
    const bool field = nfp > 0 && (pr.out.field_radiation || pr.out.field_incident || pr.out.field_scattering ||
                                 pr.out.field_diffraction);
    if (H > 26) throw Failure{HB_ERR_UNSUPPORTED, "more than 26 headings per solve", body_index};
    const bool fin = finite_depth(opt.depth);
    const double depth = fin ? opt.depth : 0.0;
    if (fin && !(opt.depth > 0.0)) throw Failure{HB_ERR_VALUE, "depth must be positive", body_index};
    if (fin) {
        for (int64_t j = 0; j < N64 * 4; j++)
            if (pr.body.vertices[3 * j + 2] < -opt.depth * (1.0 + 1e-12))
                throw Failure{HB_ERR_VALUE, "a vertex lies below the sea bottom", body_index};
    }
    // ---- geometry and statics: buffers here, the device work in run_statics (which the mixed form
    // calls once its own host-side setup is done, so that no driver call of that setup stands between
    // the statics and the assembly in the device's queue)
    Workspace& ws = workspace();
    WsBuf dverts(ws, WS_VERTS), dkind(ws, WS_KIND), dplanes(ws, WS_PLANES), dbad(ws, WS_BAD), dst(ws, WS_ST),
        dwork(ws, WS_WORK), dnwork(ws, WS_NWORK), dpbody(ws, WS_PBODY), drcen(ws, WS_RCEN), drig(ws, WS_RIGID),
        dhyd(ws, WS_HYD), dtiers(ws, WS_TIERS), dorig(ws, WS_ORIG);
    if (!orig.empty()) dorig.alloc(sizeof(int32_t) * N);
    const bool multi = nbod > 1 && pr.body.panel_body;
    // the mixed form with the reference's production statics rule: the panels' float32 Gauss tiers
    const bool prod_statics = opt.precision == HBG_MIXED && opt.statics_rule == HBG_STATICS_PRODUCTION;
    if (prod_statics) dtiers.alloc(sizeof(float) * TIER_FLOATS_HOST * (size_t)N);
    if (multi) dpbody.alloc(sizeof(int32_t) * N);
    if (pr.body.rotation_centers) drcen.alloc(sizeof(double) * 3 * nbod);
    // the rigid data [n_bodies][RIGID_PER_BODY] then the additional stiffness and damping (D x D each); the
    // hydrostatics records [n_bodies][HBG_HS] then the motion matrices M, C, B_ext (D x D each)
    const size_t DD2 = (size_t)D * D;
    std::vector<double> rigid_host;
    if (rigid) {
        rigid_host.assign((size_t)nbod * RIGID_PER_BODY + 2 * DD2, 0.0);
        for (int b = 0; b < nbod; b++) {
            double* r = &rigid_host[(size_t)b * RIGID_PER_BODY];
            r[0] = rigid->mass[b];
            for (int i = 0; i < 3; i++) r[1 + i] = rigid->center_of_gravity[3 * b + i];
            r[4] = rigid->inertia_kind ? rigid->inertia_kind[b] : HBG_INERTIA_COMPONENTS;
            for (int i = 0; i < 9; i++) r[5 + i] = rigid->inertia[9 * b + i];
            for (int i = 0; i < 3; i++) r[14 + i] = rigid->inertia_origin[3 * b + i];
        }
        double* ext = &rigid_host[(size_t)nbod * RIGID_PER_BODY];
        if (rigid->stiffness) memcpy(ext, rigid->stiffness, sizeof(double) * DD2);
        if (rigid->damping) memcpy(ext + DD2, rigid->damping, sizeof(double) * DD2);
        drig.alloc(sizeof(double) * rigid_host.size());
    }
    if (hydro) dhyd.alloc(sizeof(double) * ((size_t)nbod * HBG_HS + 3 * DD2));
    // the field points and their statics rows [4][P][N] (entry (p, j) at p + j P)
    WsBuf dpts(ws, WS_FPTS), dfst(ws, WS_FST);
    if (field) {
        dpts.alloc(sizeof(double) * 3 * nfp);
        dfst.alloc(sizeof(double) * 4 * (size_t)nfp * N);
    }
    const double* mot_mats = hydro ? dhyd.as<double>() + (size_t)nbod * HBG_HS : nullptr;
    std::vector<int32_t> kinds(N, 0);
    if (pr.body.kinds)
        for (int j = 0; j < N; j++) {
            int k = pr.body.kinds[j];
            if (k != HBG_WET && k != HBG_INTERIOR) throw Failure{HB_ERR_UNSUPPORTED, "panel kind not on this route", body_index};
            kinds[j] = k;
        }
    const size_t NS = (size_t)Nm * N, NN = (size_t)Nm * Nm;  // a statics plane (sector rows), a system matrix
    const int work_cap = std::max(1 << 16, 16 * N);
    dverts.alloc(sizeof(double) * 12 * N);
    dkind.alloc(sizeof(int32_t) * N);
    dplanes.alloc(sizeof(double) * P_PLANES * N);
    dbad.alloc(sizeof(int32_t));
    dst.alloc(sizeof(double) * 4 * NS);
    dwork.alloc(sizeof(int32_t) * 2 * work_cap);
    dnwork.alloc(2 * sizeof(int32_t));  // [adaptive worklist size, queue cursor]
    const int32_t big = PANELS_VALID;
    // page-locked: [first invalid panel, adaptive worklist size]
    // [first invalid panel, adaptive worklist size, that of the field points]
    int32_t* hflags = static_cast<int32_t*>(ws.host(HS_FLAGS, 3 * sizeof(int32_t)));
    if (!hflags) throw Failure{HB_ERR_INTERNAL, "page-locked host memory could not be allocated", body_index};
    double* prof = g_profile;
    bool statics_ran = false;
    auto run_statics = [&]() {
        if (!solve_begin().recorded) solve_begin().record(s);
        CUDA_OK(cudaMemcpyAsync(dverts.p, pr.body.vertices, sizeof(double) * 12 * N, cudaMemcpyHostToDevice, s));
        CUDA_OK(cudaMemcpyAsync(dkind.p, kinds.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice, s));
        CUDA_OK(cudaMemcpyAsync(dbad.p, &big, sizeof big, cudaMemcpyHostToDevice, s));
        if (!orig.empty())
            CUDA_OK(cudaMemcpyAsync(dorig.p, orig.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice, s));
        if (multi)
            CUDA_OK(cudaMemcpyAsync(dpbody.p, pr.body.panel_body, sizeof(int32_t) * N, cudaMemcpyHostToDevice, s));
        if (pr.body.rotation_centers)
            CUDA_OK(cudaMemcpyAsync(drcen.p, pr.body.rotation_centers, sizeof(double) * 3 * nbod,
                                    cudaMemcpyHostToDevice, s));
        EventTimer t(s, &prof[0]);
        KernelProfiler& P = profiler();
        P.begin(s);
        launch_panel_geometry(N, dverts.as<double>(), dkind.as<int32_t>(), dplanes.as<double>(), dbad.as<int32_t>(), s,
                              prod_statics ? dtiers.as<float>() : nullptr, orig.empty() ? nullptr : dorig.as<int32_t>());
        P.end(KF_GEOMETRY, 0.0, s);
        g_launches++;
        PanelsView pv{N, dplanes.as<double>(), dkind.as<int32_t>()};
        pv.G = G;
        if (prod_statics) pv.tiers = dtiers.as<float>();
        if (hydro) {  // the hydrostatics and motion matrices of every body, once per problem
            if (rigid)
                CUDA_OK(cudaMemcpyAsync(drig.p, rigid_host.data(), sizeof(double) * rigid_host.size(),
                                        cudaMemcpyHostToDevice, s));
            PanelsView pb{N, dplanes.as<double>(), dkind.as<int32_t>(), nullptr, multi ? dpbody.as<int32_t>() : nullptr,
                          pr.body.rotation_centers ? drcen.as<double>() : nullptr, nbod, G};
            const double* rg = rigid ? drig.as<double>() : nullptr;
            const double* ext = rigid ? rg + (size_t)nbod * RIGID_PER_BODY : nullptr;
            double* hs = dhyd.as<double>();
            double* mm = hs + (size_t)nbod * HBG_HS;
            launch_hydrostatics(pb, rg, rigid && rigid->stiffness ? ext : nullptr,
                                rigid && rigid->damping ? ext + DD2 : nullptr, opt.density, opt.gravity, hs, mm,
                                mm + DD2, mm + 2 * DD2, s);
            g_launches++;
        }
        CUDA_OK(cudaMemsetAsync(dnwork.p, 0, 2 * sizeof(int32_t), s));
        P.begin(s);
        launch_statics(pv, depth, opt.logarithmic, opt.log_tolerance, dst.as<double>(), dwork.as<int32_t>(),
                       dnwork.as<int32_t>(), work_cap, s, opt.precision == HBG_MIXED);
        // algorithmic bytes: the four FP64 planes written
        P.end(KF_STATICS, 32.0 * (double)NS, s);
        // the first invalid panel (geometry) and the adaptive worklist size, read at the next wait of the
        // solve; the adaptive kernel takes the size from device memory and does nothing on invalid panels
        CUDA_OK(cudaMemcpyAsync(hflags, dbad.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CUDA_OK(cudaMemcpyAsync(hflags + 1, dnwork.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        P.begin(s);
        launch_statics_adaptive_q(pv, dwork.as<int32_t>(), dnwork.as<int32_t>(), work_cap, dbad.as<int32_t>(), big,
                                  dst.as<double>(), s);
        P.end(KF_STATICS_ADAPTIVE, 0.0, s);
        g_launches += 2;
        hflags[2] = 0;
        if (field) {  // the statics rows of the field points (FP64 rules), the worklist reused after the above
            CUDA_OK(cudaMemcpyAsync(dpts.p, pr.field_points, sizeof(double) * 3 * nfp, cudaMemcpyHostToDevice, s));
            PanelsView pq{N, dplanes.as<double>(), dkind.as<int32_t>()};
            pq.rows = dpts.as<double>();
            pq.nrows = nfp;
            CUDA_OK(cudaMemsetAsync(dnwork.p, 0, 2 * sizeof(int32_t), s));
            launch_statics(pq, depth, opt.logarithmic, opt.log_tolerance, dfst.as<double>(), dwork.as<int32_t>(),
                           dnwork.as<int32_t>(), work_cap, s, false);
            CUDA_OK(cudaMemcpyAsync(hflags + 2, dnwork.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            launch_statics_adaptive_q(pq, dwork.as<int32_t>(), dnwork.as<int32_t>(), work_cap, dbad.as<int32_t>(), big,
                                      dfst.as<double>(), s);
            g_launches += 2;
        }
        t.stop();
        statics_ran = true;
    };
    // once the stream has passed the statics: invalid panels come first among the failures
    auto statics_check = [&]() {
        if (!statics_ran) return;
        if (hflags[0] != big)
            throw Failure{HB_ERR_VALUE,
                          "invalid panel " + std::to_string(hflags[0] + 1) + " (degenerate, non-convex or non-finite)",
                          body_index};
        if (hflags[1] > work_cap || hflags[2] > work_cap)
            throw Failure{HB_ERR_INTERNAL, "adaptive log-integral worklist overflow", body_index};
    };
    // the mixed form's assembly kernels skip their work on invalid panels (the flag in device memory),
    // so that its solve runs without a host wait until the end; the FP64 form waits here
    PanelsView pv{N, dplanes.as<double>(), dkind.as<int32_t>(), dbad.as<int32_t>(),
                  multi ? dpbody.as<int32_t>() : nullptr, pr.body.rotation_centers ? drcen.as<double>() : nullptr, nbod, G};
    if (F == 0 || opt.precision != HBG_MIXED) {
        run_statics();
        CUDA_OK(cudaStreamSynchronize(s));
        profiler().flush();
        statics_check();
        if (pr.out.hydrostatics)
            CUDA_OK(cudaMemcpy(pr.out.hydrostatics, dhyd.p, sizeof(double) * nbod * HBG_HS, cudaMemcpyDeviceToHost));
        if (F == 0) return;
    }
    const int nrhs = D + H;
    if (opt.precision == HBG_MIXED) {
        const char* msg = "";
        int64_t fq = -1;
        std::vector<int64_t> fallback;  // frequencies the mixed form hands to the FP64 form
        int rc = mixed_solve_frequencies(pv, dst.as<double>(), pr, opt, fin, depth, s, prof, &g_launches, &msg, &fq,
                                         run_statics, motions ? mot_mats : nullptr,
                                         FieldArgs{field ? dpts.as<double>() : nullptr, field ? nfp : 0, dfst.as<double>()},
                                         &fallback);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e == cudaSuccess) statics_check();
        if (rc != 0) throw Failure{rc, msg, body_index, fq};
        CUDA_OK(e);
        if (pr.out.hydrostatics)
            CUDA_OK(cudaMemcpy(pr.out.hydrostatics, dhyd.p, sizeof(double) * nbod * HBG_HS, cudaMemcpyDeviceToHost));
        if (!fallback.empty()) {
            // the frequencies whose refinement did not converge, solved again by the FP64 form (pivoted LU)
            const size_t nf = fallback.size(), DDo = (size_t)D * D, HD = (size_t)H * 2 * D;
            const size_t PD = (size_t)(field ? nfp : 0) * 2 * D, PH = (size_t)(field ? nfp : 0) * 2 * H;
            const size_t RD = (size_t)TK * 2 * D, RH = (size_t)TK * 2 * H, RR = TK ? (size_t)H * H * 6 : 0;
            std::vector<double> om(nf), a(nf * DDo), b(nf * DDo), x(nf * HD), fk(nf * HD), sc(nf * HD), mo(nf * HD),
                hk(nf * HD), fr(nf * PD), fi(nf * PH), fs(nf * PH), fdf(nf * PH), kr(nf * RD), krt(nf * RD),
                kd(nf * RH), kdt(nf * RH), dr(nf * RR);
            for (size_t i = 0; i < nf; i++) om[i] = pr.omegas[fallback[i]];
            HbgProblem sub = pr_in;
            sub.omegas = om.data();
            sub.n_omega = (int64_t)nf;
            sub.out = HbgOutputs{a.data(), b.data(), x.data(), fk.data(), sc.data(), motions ? mo.data() : nullptr,
                                 nullptr, PD ? fr.data() : nullptr, PH ? fi.data() : nullptr, PH ? fs.data() : nullptr,
                                 PH ? fdf.data() : nullptr, hk.data(), RD ? kr.data() : nullptr,
                                 RD ? krt.data() : nullptr, RH ? kd.data() : nullptr, RH ? kdt.data() : nullptr,
                                 RR ? dr.data() : nullptr};
            HbgOptions o64 = opt;
            o64.precision = HBG_FP64;
            o64.surrogate = nullptr;
            cudaEvent_t fb0 = nullptr, fb1 = nullptr;
            cudaEventCreate(&fb0);
            cudaEventCreate(&fb1);
            cudaEventRecord(fb0, s);
            solve_problem(sub, o64, body_index, s);
            cudaEventRecord(fb1, s);
            float fb_ms = 0.f;
            if (cudaEventSynchronize(fb1) == cudaSuccess && cudaEventElapsedTime(&fb_ms, fb0, fb1) == cudaSuccess)
                last_fallback_ms() += fb_ms;
            cudaEventDestroy(fb0);
            cudaEventDestroy(fb1);
            for (size_t i = 0; i < nf; i++) {
                const size_t fo = (size_t)fallback[i];
                auto put = [&](double* dst, const std::vector<double>& src, size_t per) {
                    if (dst && per) memcpy(dst + fo * per, src.data() + i * per, per * sizeof(double));
                };
                put(pr.out.added_mass, a, DDo);
                put(pr.out.radiation_damping, b, DDo);
                put(pr.out.excitation, x, HD);
                put(pr.out.froude_krylov, fk, HD);
                put(pr.out.scattering, sc, HD);
                if (motions) put(pr.out.motions, mo, HD);
                put(pr.out.haskind, hk, HD);
                put(pr.out.kochin_radiation, kr, RD);
                put(pr.out.kochin_radiation_derivative, krt, RD);
                put(pr.out.kochin_diffraction, kd, RH);
                put(pr.out.kochin_diffraction_derivative, kdt, RH);
                put(pr.out.drift, dr, RR);
                if (field) {
                    put(pr.out.field_radiation, fr, PD);
                    put(pr.out.field_incident, fi, PH);
                    put(pr.out.field_scattering, fs, PH);
                    put(pr.out.field_diffraction, fdf, PH);
                }
            }
            last_fallback_count() += (int64_t)nf;
        }
        return;
    }
    // ---- frequency batches
    // per frequency: G systems (S, A, right-hand sides, solutions, pivots), the boundary values and incident
    // wave of every panel, with sectors the projected right-hand sides and the recombined potentials
    size_t per_freq = G * (2 * NN * sizeof(double2) + (size_t)2 * nrhs * Nm * sizeof(double2) + (size_t)Nm * 4 + 4) +
                      (size_t)(nrhs + H) * N * sizeof(double2) + (G > 1 ? (size_t)2 * nrhs * N * sizeof(double2) : 0) +
                      (fin ? (size_t)(T1_SIZE + T2_SIZE) * 8 + (size_t)FP_PLANES * N * 8 +
                                                              (size_t)6912 * 3 * 8
                                                        : 0);
    // the batch size from free memory, kept per thread and device for the same problem shape while the
    // workspace holds its buffers (cudaMemGetInfo can take milliseconds)
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
        const size_t mats = NN * G * (size_t)std::max(c.B, 0);
        if (same && c.B > 0 && ws.bytes[WS_S] >= sizeof(double2) * mats && ws.bytes[WS_A] >= sizeof(double2) * mats) {
            B = c.B;
        } else {
            size_t freeb = 0, totalb = 0;
            CUDA_OK(cudaMemGetInfo(&freeb, &totalb));
            const size_t reusable = ws.bytes[WS_S] + ws.bytes[WS_A];
            size_t avail = (size_t)(0.85 * (double)(freeb + reusable));
            if (hbm_budget() > 0) avail = std::min(avail, hbm_budget());
            B = (int)std::max<size_t>(1, avail / per_freq);
            if (opt.max_batch > 0) B = std::min(B, (int)opt.max_batch);
            B = std::min(B, F);
            c = BatchChoice{N, G, nrhs, (int)fin, F, B, opt.max_batch, hbm_budget()};
        }
    }
    const size_t BS = (size_t)B * G;  // systems per batch
    WsBuf dS(ws, WS_S), dA(ws, WS_A), du(ws, WS_U), drhs(ws, WS_RHS), dX(ws, WS_X), dphiI(ws, WS_PHII),
        dipiv(ws, WS_IPIV), dinfo(ws, WS_INFO), dfi(ws, WS_FI), dfd(ws, WS_FD), dtiles(ws, WS_TILES),
        dscr(ws, WS_SCR), dfpt(ws, WS_FPT), dheads(ws, WS_HEADS), dout(ws, WS_OUT), dup(ws, WS_UP), dphi(ws, WS_PHI);
    dS.alloc(sizeof(double2) * NN * BS);
    dA.alloc(sizeof(double2) * NN * BS);
    du.alloc(sizeof(double2) * (size_t)nrhs * N * B);
    drhs.alloc(sizeof(double2) * (size_t)nrhs * Nm * BS);
    dX.alloc(sizeof(double2) * (size_t)nrhs * Nm * BS);
    if (G > 1) {
        dup.alloc(sizeof(double2) * (size_t)nrhs * Nm * BS);
        dphi.alloc(sizeof(double2) * (size_t)nrhs * N * B);
    }
    dphiI.alloc(sizeof(double2) * (size_t)std::max(H, 1) * N * B);
    dipiv.alloc(sizeof(int32_t) * (size_t)Nm * BS);
    dinfo.alloc(sizeof(int32_t) * BS);
    dfi.alloc(sizeof(FreqInfo) * B);
    dfd.alloc(sizeof(FdParams) * B);
    if (fin) {
        dtiles.alloc(sizeof(double) * (size_t)(T1_SIZE + T2_SIZE) * B);
        dscr.alloc(sizeof(double) * (size_t)6912 * 3 * B);
        dfpt.alloc(sizeof(double) * (size_t)FP_PLANES * N * B);
    }
    std::vector<double> heads(std::max(H, 1));
    for (int h = 0; h < H; h++) heads[h] = pr.headings_deg[h] * PI / 180.0;
    dheads.alloc(sizeof(double) * heads.size());
    CUDA_OK(cudaMemcpyAsync(dheads.p, heads.data(), sizeof(double) * heads.size(), cudaMemcpyHostToDevice, s));
    // outputs per batch: A, B [D][D], X, FK, SC, motions [H][D], field values [P][D] and 3 x [P][H]
    const int Pf = field ? nfp : 0;
    // outputs per batch: ..., then the Haskind exciting force [H][D], then (TK > 0) the Kochin functions
    // kr, krt [TK][D], kd, kdt [TK][H] and the drift [H][H][3]
    const size_t kochin_per = (size_t)TK * 2 * (D + H) + (TK ? (size_t)3 * H * H : 0);
    const size_t out_per = 2 * (size_t)D * D * sizeof(double) + 5 * (size_t)H * D * sizeof(double2) +
                           (size_t)Pf * (D + 3 * H) * sizeof(double2) + kochin_per * sizeof(double2);
    WsBuf dfq(ws, WS_FQ);
    if (field && fin) dfq.alloc(sizeof(double) * FP_PLANES * (size_t)(N + nfp) * B);
    WsBuf derr(ws, WS_ERR);
    derr.alloc(sizeof(int32_t));
    dout.alloc(out_per * B);
    // page-locked outputs and pivot flags: their reads queue behind the work
    unsigned char* hout = static_cast<unsigned char*>(ws.host(HS_OUT, out_per * B + sizeof(int32_t) * (BS + 1)));
    if (!hout) throw Failure{HB_ERR_INTERNAL, "page-locked host memory could not be allocated", body_index};
    int32_t* info = reinterpret_cast<int32_t*>(hout + out_per * B);
    int32_t* herr = info + BS;
    std::vector<FreqInfo> fi(B);
    std::vector<FdParams> fdh(B);
    for (int f0 = 0; f0 < F; f0 += B) {
        if (opt.cancel && *opt.cancel) throw Failure{HB_ERR_CANCELLED, "the solve was cancelled", body_index, f0};
        const int nb = std::min(B, F - f0), ns = nb * G;
        for (int i = 0; i < nb; i++) {
            double w = pr.omegas[f0 + i], K = w * w / opt.gravity;
            fi[i].omega = w;
            fi[i].K = K;
            fi[i].k = fin ? dispersion_x0(K * depth) / depth : K;
            fi[i].logc = opt.logarithmic ? 1.0 : 0.0;
            if (fin) make_fd_params(depth, K, fdh[i]);
        }
        CUDA_OK(cudaMemcpyAsync(dfi.p, fi.data(), sizeof(FreqInfo) * nb, cudaMemcpyHostToDevice, s));
        if (fin) {
            CUDA_OK(cudaMemcpyAsync(dfd.p, fdh.data(), sizeof(FdParams) * nb, cudaMemcpyHostToDevice, s));
        }
        {
            EventTimer t(s, &prof[1]);
            KernelProfiler& P = profiler();
            if (fin) {
                P.begin(s);
                launch_fd_tiles(nb, dfd.as<FdParams>(), dtiles.as<double>(), dscr.as<double>(), s);
                launch_fin_points(pv, nb, dfd.as<FdParams>(), dfpt.as<double>(), s);
                if (field) launch_field_fin(pv, dpts.as<double>(), nfp, nb, dfd.as<FdParams>(), dfq.as<double>(), s);
                P.end(KF_FD_TILES, 0.0, s);
                g_launches += 3 + field;
            }
            P.begin(s);
            launch_assemble_f64(pv, dst.as<double>(), nb, dfi.as<FreqInfo>(), dfd.as<FdParams>(), dtiles.as<double>(),
                                dfpt.as<double>(), fin, dS.as<double2>(), dA.as<double2>(), NN, s);
            if (G > 1) launch_sectors_f64(dS.as<double2>(), dA.as<double2>(), nb, G, Nm, NN, s);
            // algorithmic bytes per pair: 4 statics read (32 B), S and A written (32 B)
            P.end(KF_ASSEMBLE, 64.0 * (double)NN * ns, s);
            P.begin(s);
            launch_boundary(pv, nb, dfi.as<FreqInfo>(), H, dheads.as<double>(), depth, opt.gravity, du.as<double2>(),
                            dphiI.as<double2>(), s);
            P.end(KF_BOUNDARY, 0.0, s);
            const double2* urhs = du.as<double2>();
            if (G > 1) {
                launch_project(du.as<double2>(), dup.as<double2>(), nb, G, Nm, nrhs, Nm, s);
                urhs = dup.as<double2>();
            }
            P.begin(s);
            launch_rhs_f64(Nm, ns, nrhs, dS.as<double2>(), NN, urhs, drhs.as<double2>(), s);
            // S read once (16 B per entry)
            P.end(KF_RHS, 16.0 * (double)NN * ns, s);
            g_launches += 3 + 2 * (G > 1);
            t.stop();
        }
        {
            EventTimer t(s, &prof[2]);
            lu_factor_f64(Nm, ns, dA.as<double2>(), NN, dipiv.as<int32_t>(), dinfo.as<int32_t>(), s, &g_launches);
            t.stop();
        }
        {
            EventTimer t(s, &prof[3]);
            KernelProfiler& P = profiler();
            P.begin(s);
            if (lu_solve_f64(Nm, ns, dA.as<double2>(), NN, dipiv.as<int32_t>(), nrhs, drhs.as<double2>(),
                             dX.as<double2>(), s))
                throw Failure{HB_ERR_UNSUPPORTED, "too many right-hand sides or panels for the substitution kernel", body_index};
            // the factors read once (16 B per entry)
            P.end(KF_LU_SOLVE, 16.0 * (double)NN * ns, s);
            g_launches += 1;
            t.stop();
        }
        {
            EventTimer t(s, &prof[4]);
            double* base = dout.as<double>();
            double* dAo = base;
            double* dBo = base + (size_t)D * D * nb;
            double2* dXo = reinterpret_cast<double2*>(base + 2 * (size_t)D * D * nb);
            double2* dFK = dXo + (size_t)H * D * nb;
            double2* dSC = dFK + (size_t)H * D * nb;
            KernelProfiler& P = profiler();
            // the potentials of every panel: the sector solutions recombined (one system: as solved)
            const double2* phi = dX.as<double2>();
            if (G > 1) {
                launch_recombine(dX.as<double2>(), dphi.as<double2>(), nb, G, Nm, nrhs, Nm, s);
                phi = dphi.as<double2>();
                g_launches++;
            }
            P.begin(s);
            launch_forces(pv, nb, dfi.as<FreqInfo>(), H, phi, N, dphiI.as<double2>(), opt.density, dAo, dBo, dXo, dFK,
                          dSC, s);
            P.end(KF_FORCES, 16.0 * (double)N * (nrhs + H) * nb, s);
            launch_haskind(pv, nb, dfi.as<FreqInfo>(), H, phi, N, du.as<double2>(), dphiI.as<double2>(), opt.density,
                           dSC + 2 * (size_t)H * D * nb + (size_t)Pf * (D + 3 * H) * nb, s);
            g_launches += 1 + (H > 0);
            CUDA_OK(cudaMemsetAsync(derr.p, 0, sizeof(int32_t), s));
            if (motions) {
                launch_motions(nb, D, H, dfi.as<FreqInfo>(), dAo, dBo, dXo, mot_mats, mot_mats + DD2, mot_mats + 2 * DD2,
                               dSC + (size_t)H * D * nb, derr.as<int32_t>(), s);
                g_launches++;
            }
            if (field) {  // the field points from the potentials of every panel
                double2* fr = dSC + 2 * (size_t)H * D * nb;
                double2* fi_ = fr + (size_t)nfp * D * nb;
                launch_field(pv, dpts.as<double>(), nfp, dfst.as<double>(), nb, dfi.as<FreqInfo>(), dfd.as<FdParams>(),
                             dtiles.as<double>(), dfq.as<double>(), fin, H, dheads.as<double>(), depth, opt.gravity,
                             phi, N, du.as<double2>(), dphiI.as<double2>(), fr, fi_, fi_ + (size_t)nfp * H * nb,
                             fi_ + 2 * (size_t)nfp * H * nb, s);
                g_launches++;
            }
            if (TK) {  // the Kochin functions, then the momentum drift (with the motions when computed)
                double2* kr = dSC + 3 * (size_t)H * D * nb + (size_t)Pf * (D + 3 * H) * nb;
                double2* krt = kr + (size_t)TK * D * nb;
                double2* kd = krt + (size_t)TK * D * nb;
                double2* kdt = kd + (size_t)TK * H * nb;
                double2* dr = kdt + (size_t)TK * H * nb;
                launch_kochin(pv, nb, dfi.as<FreqInfo>(), TK, H, depth, phi, N, du.as<double2>(), dphiI.as<double2>(),
                              kr, krt, kd, kdt, s);
                launch_drift(nb, D, H, TK, dfi.as<FreqInfo>(), depth, opt.gravity, opt.density, dheads.as<double>(), kr,
                             krt, kd, kdt, motions ? dSC + (size_t)H * D * nb : nullptr, dr, s);
                g_launches += 2;
            }
            CUDA_OK(cudaMemcpyAsync(hout, dout.p, out_per * nb, cudaMemcpyDeviceToHost, s));
            CUDA_OK(cudaMemcpyAsync(info, dinfo.p, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost, s));
            CUDA_OK(cudaMemcpyAsync(herr, derr.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            t.stop();
            solve_end().record(s);
        }
        CUDA_OK(cudaStreamSynchronize(s));
        CUDA_OK(cudaGetLastError());
        profiler().flush();
        const double* hb = reinterpret_cast<const double*>(hout);
        const double* hA = hb;
        const size_t DD = (size_t)D * D;
        const double* hB = hb + DD * nb;
        const double* hX = hb + 2 * DD * nb;
        const double* hFK = hX + (size_t)H * 2 * D * nb;
        const double* hSC = hFK + (size_t)H * 2 * D * nb;
        const double* hMo = hSC + (size_t)H * 2 * D * nb;
        const double* hFr = hMo + (size_t)H * 2 * D * nb;
        const double* hFi = hFr + (size_t)Pf * 2 * D * nb;
        const double* hHK = hFi + (size_t)Pf * 2 * 3 * H * nb;
        const double* hKr = hHK + (size_t)H * 2 * D * nb;
        if (*herr != 0) throw Failure{HB_ERR_NUMERICAL, "singular motion equation", body_index, f0};
        for (int i = 0; i < nb; i++) {
            for (int c = 0; c < G; c++)
                if (info[i * G + c] != 0)
                    throw Failure{HB_ERR_NUMERICAL,
                                  "singular system matrix (zero pivot " + std::to_string(info[i * G + c]) + ")",
                                  body_index, f0 + i};
            for (size_t q = 0; q < DD; q++)
                if (!std::isfinite(hA[DD * i + q]) || !std::isfinite(hB[DD * i + q]))
                    throw Failure{HB_ERR_NUMERICAL, "non-finite solution", body_index, f0 + i};
            const size_t fo = (size_t)(f0 + i);
            if (pr.out.added_mass) memcpy(pr.out.added_mass + fo * DD, hA + DD * i, DD * sizeof(double));
            if (pr.out.radiation_damping) memcpy(pr.out.radiation_damping + fo * DD, hB + DD * i, DD * sizeof(double));
            const size_t hx = (size_t)H * 2 * D;
            if (pr.out.excitation) memcpy(pr.out.excitation + fo * hx, hX + hx * i, hx * sizeof(double));
            if (pr.out.froude_krylov) memcpy(pr.out.froude_krylov + fo * hx, hFK + hx * i, hx * sizeof(double));
            if (pr.out.scattering) memcpy(pr.out.scattering + fo * hx, hSC + hx * i, hx * sizeof(double));
            if (motions && pr.out.motions) memcpy(pr.out.motions + fo * hx, hMo + hx * i, hx * sizeof(double));
            if (pr.out.haskind) memcpy(pr.out.haskind + fo * hx, hHK + hx * i, hx * sizeof(double));
            if (field) {
                const size_t pd = (size_t)nfp * 2 * D, ph = (size_t)nfp * 2 * H;
                if (pr.out.field_radiation) memcpy(pr.out.field_radiation + fo * pd, hFr + pd * i, pd * sizeof(double));
                double* dst3[3] = {pr.out.field_incident, pr.out.field_scattering, pr.out.field_diffraction};
                for (int q = 0; q < 3; q++)
                    if (dst3[q]) memcpy(dst3[q] + fo * ph, hFi + ph * ((size_t)q * nb + i), ph * sizeof(double));
            }
            if (TK) copy_kochin(pr.out, hKr, TK, D, H, nb, i, fo);
        }
    }
}

}  // namespace hbg

using namespace hbg;

// ==================================================================== C ABI: batched entry
extern "C" void hbg_default_options(HbgOptions* opt) {
    if (!opt) return;
    opt->precision = HBG_FP64;
    opt->logarithmic = 1;
    opt->log_tolerance = 1e-4;
    opt->gravity = 9.80665;
    opt->density = 1000.0;
    opt->depth = INFINITY;
    opt->max_batch = 0;
    opt->concurrency = 0;
    opt->device = 0;
    opt->cancel = nullptr;
    opt->surrogate = nullptr;
    opt->statics_rule = HBG_STATICS_ACCURATE;
}

// ------------------------------------------------------------------ the cross-body work queue
// Several problems of one call solved at once: K pipelines, each a host thread of a pool kept per device
// for the life of the process (so that its thread-local workspace, streams and side streams persist
// across calls like the calling thread's own), with its own stream and 1/K of the free device memory.
// The problems go costliest first to the next free pipeline: the reference's worker pool over
// independent units (parallel.rs:31-109), with the device's streams for threads.
namespace {
class PipelinePool {
public:
    explicit PipelinePool(int dev) : dev_(dev) {}
    // job(w) on pipelines w = 0 .. k - 1; returns when all have finished (calls are serialised)
    void run(int k, const std::function<void(int)>& job) {
        std::lock_guard<std::mutex> one(run_m_);
        std::unique_lock<std::mutex> lk(m_);
        while ((int)threads_ < k) {
            const int w = threads_++;
            std::thread([this, w] { loop(w); }).detach();
        }
        job_ = &job;
        k_ = k;
        left_ = k;
        gen_++;
        cv_.notify_all();
        done_.wait(lk, [this] { return left_ == 0; });
        job_ = nullptr;
    }
    int threads() {
        std::lock_guard<std::mutex> lk(m_);
        return threads_;
    }

private:
    void loop(int w) {
        cudaSetDevice(dev_);
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(int)>* job = nullptr;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (w >= k_) continue;
                job = job_;
            }
            (*job)(w);
            std::lock_guard<std::mutex> lk(m_);
            if (--left_ == 0) done_.notify_all();
        }
    }
    int dev_;
    std::mutex run_m_, m_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* job_ = nullptr;
    int threads_ = 0, k_ = 0, left_ = 0;
    uint64_t gen_ = 0;
};

// the pool of a device (created on first use when `create`; kept for the process: its threads never exit)
PipelinePool* pipeline_pool_ptr(int dev, bool create) {
    static std::mutex m;
    static PipelinePool* pools[16] = {};
    std::lock_guard<std::mutex> lk(m);
    if (!pools[dev] && create) pools[dev] = new PipelinePool(dev);
    return pools[dev];
}
PipelinePool& pipeline_pool(int dev) { return *pipeline_pool_ptr(dev, true); }

cudaStream_t& pipeline_stream() {
    static thread_local cudaStream_t s = nullptr;
    return s;
}

// What a pipeline hands back: its phase times, counters and kernel-family records, and the workspace
// it holds afterwards (part of the memory the next call shares out).
struct PipelineStats {
    double phase[5] = {};
    int64_t launches = 0, fallbacks = 0;
    double fallback_ms = 0.0;
    long long sg_pairs = 0;
    int ir_iterations = 0;
    double kms[KF_COUNT] = {}, kwork[KF_COUNT] = {};
    int64_t klaunches[KF_COUNT] = {};
    size_t held = 0;
};
// per device and pipeline: the workspace bytes it held after its last call (what it can reuse)
std::atomic<size_t> g_pool_held[16][8];

// The modelled cost of a problem (the LU of each system against its assembly, per frequency): the order
// in which the pipelines take the problems.
double problem_cost(const HbgProblem& p) {
    const int G = p.body.symmetry == HBG_SYM_BOTH ? 4 : p.body.symmetry != HBG_SYM_NONE ? 2 : 1;
    const double n = (double)p.body.n_panels;
    return (double)std::max<int64_t>(p.n_omega, 1) * G * (n * n * n + 1.0e3 * G * n * n);
}
}  // namespace

// The pipelines for a call that leaves the choice to the library: two when the call has several problems
// none of which is large (the 64 uneven bodies of 840-5928 panels, 16 frequencies each, mixed form:
// 450 / 545 / 538 / 513 frequency solves/s with 1 / 2 / 3 / 4 pipelines; the small bodies' triangular
// sweeps and refinement are latency-bound chains that another body's products fill in), else one (a large
// problem keeps the whole memory for its frequency batches).
static int tuned_concurrency(const HbgProblem* problems, int64_t n, const HbgOptions& opt) {
    (void)opt;
    if (n < 2) return 1;
    for (int64_t p = 0; p < n; p++) {
        const int G = problems[p].body.symmetry == HBG_SYM_BOTH ? 4 : problems[p].body.symmetry != HBG_SYM_NONE ? 2 : 1;
        if (problems[p].body.n_panels * G > 8192) return 1;
    }
    return 2;
}

// The problems of a call on K pipelines (K >= 2): the device time from the first queued operation to
// the last, the phases summed over the pipelines, the counters added up; on failure the failure of the
// lowest problem index is returned (problems after it may have been solved, as with one pipeline those
// before it).
static void solve_concurrent(const HbgProblem* problems, int64_t n, const HbgOptions& opt, int K) {
    const int dev = opt.device;
    PipelinePool& pool = pipeline_pool(dev);
    std::vector<int64_t> order((size_t)n);
    for (int64_t i = 0; i < n; i++) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t a, int64_t b) { return problem_cost(problems[a]) > problem_cost(problems[b]); });
    // the calling thread's own buffers (from earlier one-after-another solves) are freed: the pipelines
    // share the device memory, and a solve on this thread allocates again what it needs
    workspace().release();
    size_t freeb = 0, totalb = 0;
    CUDA_OK(cudaMemGetInfo(&freeb, &totalb));
    size_t reusable = 0;  // the buffers of the pipelines this call uses (the others keep theirs)
    for (int w = 0; w < K; w++) reusable += g_pool_held[dev][w].load();
    const size_t budget = (size_t)(0.85 * (double)(freeb + reusable) / K);
    std::vector<PipelineStats> stats((size_t)K);
    std::vector<cudaEvent_t> ends((size_t)K, nullptr);
    cudaStream_t s0;
    CUDA_OK(cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (auto& e : ends) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    cudaEventRecord(e0, s0);
    const bool prof_on = profiler().on;
    std::atomic<int64_t> next{0};
    std::atomic<bool> failed{false};
    std::mutex fm;
    Failure first{HB_OK, ""};
    int64_t first_at = -1;
    auto record = [&](const Failure& f, int64_t p) {
        std::lock_guard<std::mutex> lk(fm);
        if (first_at < 0 || p < first_at) first = f, first_at = p;
        failed = true;
    };
    std::function<void(int)> job = [&](int w) {
        PipelineStats& st = stats[(size_t)w];
        hbm_budget() = budget;
        for (int i = 0; i < 6; i++) g_profile[i] = 0.0;
        g_launches = 0;
        last_fallback_count() = 0;
        last_fallback_ms() = 0.0;
        last_surrogate_pairs() = 0;
        KernelProfiler& P = profiler();
        P.reset();
        P.on = prof_on;
        phase_timers().flush();
        solve_begin().recorded = false;
        solve_end().recorded = false;
        cudaStream_t& s = pipeline_stream();
        if (!s && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
            s = nullptr;
            record(Failure{HB_ERR_INTERNAL, "CUDA: a pipeline stream could not be created"}, -1);
        }
        if (s) {
            cudaStreamWaitEvent(s, e0, 0);
            int64_t p = -1;
            try {
                for (;;) {
                    if (failed.load()) break;
                    const int64_t i = next.fetch_add(1);
                    if (i >= n) break;
                    p = order[(size_t)i];
                    solve_problem(problems[p], opt, p, s);
                }
            } catch (const Failure& f) {
                record(f, p);
            } catch (const std::exception& e) {
                record(Failure{HB_ERR_INTERNAL, std::string("internal error: ") + e.what(), p}, p);
            } catch (...) {
                record(Failure{HB_ERR_INTERNAL, "internal error", p}, p);
            }
            cudaEventRecord(ends[(size_t)w], s);
            cudaStreamSynchronize(s);
        }
        phase_timers().flush();
        P.flush();
        for (int i = 0; i < 5; i++) st.phase[i] = g_profile[i];
        st.launches = g_launches;
        st.fallbacks = last_fallback_count();
        st.fallback_ms = last_fallback_ms();
        st.sg_pairs = last_surrogate_pairs();
        st.ir_iterations = last_ir_iterations();
        for (int i = 0; i < KF_COUNT; i++) st.kms[i] = P.ms[i], st.kwork[i] = P.work[i], st.klaunches[i] = P.launches[i];
        st.held = workspace().held();
        g_pool_held[dev][w].store(st.held);
        hbm_budget() = 0;
    };
    pool.run(K, job);
    for (auto& e : ends) cudaStreamWaitEvent(s0, e, 0);
    cudaEventRecord(e1, s0);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    KernelProfiler& P = profiler();
    int ir = 0;
    for (const PipelineStats& st : stats) {
        for (int i = 0; i < 5; i++) g_profile[i] += st.phase[i];
        g_launches += st.launches;
        last_fallback_count() += st.fallbacks;
        last_fallback_ms() += st.fallback_ms;
        last_surrogate_pairs() += st.sg_pairs;
        ir = std::max(ir, st.ir_iterations);
        for (int i = 0; i < KF_COUNT; i++) P.ms[i] += st.kms[i], P.work[i] += st.kwork[i], P.launches[i] += st.klaunches[i];
    }
    last_ir_iterations() = ir;
    last_ir_history().n = 0;
    g_profile[5] = ms;
    for (auto& e : ends) cudaEventDestroy(e);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s0);
    if (failed.load()) throw first;
}

extern "C" HbStatus hbg_solve_batch(const HbgProblem* problems, int64_t n_problems, const HbgOptions* opt) {
    try {
        if (!problems || !opt || n_problems < 0) return fail({HB_ERR_ARGUMENT, "null argument"});
        for (int i = 0; i < 6; i++) g_profile[i] = 0.0;
        g_launches = 0;
        last_fallback_count() = 0;
        last_fallback_ms() = 0.0;
        profiler().reset();
        for (int64_t p = 0; p < n_problems; p++) {
            const HbgProblem& pr = problems[p];
            if (!pr.body.vertices || pr.n_omega < 0 || pr.n_heading < 0 || (pr.n_omega > 0 && !pr.omegas) ||
                (pr.n_heading > 0 && !pr.headings_deg))
                return fail({HB_ERR_ARGUMENT, "problem with a null array", p});
        }
        if (opt->precision != HBG_FP64 && opt->precision != HBG_MIXED)
            return fail({HB_ERR_VALUE, "unknown precision form"});
        if (opt->surrogate && opt->precision != HBG_MIXED)
            return fail({HB_ERR_VALUE, "the wave-term network is an option of the mixed form only"});
        if (opt->statics_rule != HBG_STATICS_ACCURATE && opt->statics_rule != HBG_STATICS_PRODUCTION)
            return fail({HB_ERR_VALUE, "unknown statics rule"});
        if (opt->statics_rule == HBG_STATICS_PRODUCTION && opt->precision != HBG_MIXED)
            return fail({HB_ERR_UNSUPPORTED, "the production statics rule is an option of the mixed form (the FP64 "
                                             "form is the reference's double-precision path)"});
        if (!(opt->gravity > 0.0) || !(opt->density > 0.0) || opt->log_tolerance < 0.0)
            return fail({HB_ERR_VALUE, "gravity and density must be positive, log_tolerance nonnegative"});
        if (opt->concurrency < 0 || opt->concurrency > 8) return fail({HB_ERR_VALUE, "concurrency outside 0..8"});
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            return fail({HB_ERR_UNSUPPORTED, "no CUDA device: this library runs the path on the GPU only"});
        if (opt->device < 0 || opt->device >= ndev) return fail({HB_ERR_ARGUMENT, "device ordinal out of range"});
        CUDA_OK(cudaSetDevice(opt->device));
        device_ctx(opt->device);
        const int K = (int)std::min<int64_t>(opt->concurrency > 0 ? opt->concurrency
                                                                  : tuned_concurrency(problems, n_problems, *opt),
                                             n_problems);
        if (K >= 2) {
            phase_timers().flush();
            solve_concurrent(problems, n_problems, *opt, K);
            return HB_OK;
        }
        // one after another on this thread: the pipelines' buffers (from an earlier concurrent call) are
        // freed, so that this thread's batches may use the device memory
        if (PipelinePool* pool = pipeline_pool_ptr(opt->device, false)) {
            bool held = false;
            for (int w = 0; w < 8; w++) held = held || g_pool_held[opt->device][w].load() > 0;
            if (held) {
                pool->run(pool->threads(), [](int) { workspace().release(); });
                for (int w = 0; w < 8; w++) g_pool_held[opt->device][w].store(0);
            }
        }
        cudaStream_t s;
        CUDA_OK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
        phase_timers().flush();
        solve_begin().recorded = false;
        solve_end().recorded = false;
        try {
            for (int64_t p = 0; p < n_problems; p++) solve_problem(problems[p], *opt, p, s);
        } catch (...) {
            cudaStreamSynchronize(s);
            phase_timers().flush();
            cudaStreamDestroy(s);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        phase_timers().flush();
        float ms = 0.f;
        cudaEventElapsedTime(&ms, solve_begin().recorded ? solve_begin().event() : e0,
                             solve_end().recorded ? solve_end().event() : e1);
        g_profile[5] = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaStreamDestroy(s);
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    } catch (const std::exception& e) {
        return fail({HB_ERR_INTERNAL, std::string("internal error: ") + e.what()});
    } catch (...) {
        return fail({HB_ERR_INTERNAL, "internal error"});
    }
}

extern "C" HbStatus hbg_last_profile(double* ms6) {
    if (!ms6) return fail({HB_ERR_ARGUMENT, "null argument"});
    for (int i = 0; i < 6; i++) ms6[i] = g_profile[i];
    return HB_OK;
}

extern "C" HbStatus hbg_profile_kernels(int32_t on) {
    profiler().on = on != 0;
    return HB_OK;
}

extern "C" HbStatus hbg_kernel_profile(int32_t family, double* ms, int64_t* launches, double* work) {
    if (!ms || !launches || !work) return fail({HB_ERR_ARGUMENT, "null argument"});
    if (family < 0 || family >= KF_COUNT) return fail({HB_ERR_ARGUMENT, "kernel family out of range"});
    KernelProfiler& P = profiler();
    *ms = P.ms[family];
    *launches = P.launches[family];
    *work = P.work[family];
    return HB_OK;
}

extern "C" HbStatus hbg_release_workspace(void) {
    for (int d = 0; d < 16; d++)
        if (g_ws[d]) {
            int cur = 0;
            cudaGetDevice(&cur);
            cudaSetDevice(d);
            g_ws[d]->release();
            cudaSetDevice(cur);
        }
    // and the buffers of the device's pipelines (concurrent solves)
    for (int d = 0; d < 16; d++)
        if (PipelinePool* pool = pipeline_pool_ptr(d, false)) {
            const int k = pool->threads();
            if (k > 0) pool->run(k, [](int) { workspace().release(); });
            for (int w = 0; w < 8; w++) g_pool_held[d][w].store(0);
        }
    return HB_OK;
}

extern "C" HbStatus hbg_last_fallback_count(int64_t* count) {
    if (!count) return fail({HB_ERR_ARGUMENT, "null argument"});
    *count = last_fallback_count();
    return HB_OK;
}

extern "C" HbStatus hbg_last_fallback_time(double* ms) {
    if (!ms) return fail({HB_ERR_ARGUMENT, "null argument"});
    *ms = last_fallback_ms();
    return HB_OK;
}

extern "C" HbStatus hbg_last_launch_count(int64_t* count) {
    if (!count) return fail({HB_ERR_ARGUMENT, "null argument"});
    *count = g_launches;
    return HB_OK;
}

// Test support: the statics and the matrices S, A of one body at one frequency, FP64.
extern "C" HbStatus hbg_debug_matrices(const HbgBody* body, double omega, const HbgOptions* opt, double* statics,
                                       double* S, double* A) {
    try {
        if (!body || !opt || !body->vertices) return fail({HB_ERR_ARGUMENT, "null argument"});
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            return fail({HB_ERR_UNSUPPORTED, "no CUDA device: this library runs the path on the GPU only"});
        CUDA_OK(cudaSetDevice(opt->device));
        device_ctx(opt->device);
        // with symmetry planes: the sector's panels mirrored, statics of the sector rows, G sector matrices
        const int sym = body->symmetry;
        if (sym < HBG_SYM_NONE || sym > HBG_SYM_BOTH) return fail({HB_ERR_VALUE, "symmetry outside 0..3"});
        const int G = sym == HBG_SYM_BOTH ? 4 : sym != HBG_SYM_NONE ? 2 : 1;
        const int Nm = (int)body->n_panels, N = Nm * G;
        std::vector<double> mverts;
        std::vector<int32_t> kinds, mbody;
        if (G > 1) {
            mirror_sector(*body, G, mverts, kinds, mbody);
        } else {
            kinds.assign(N, 0);
            if (body->kinds)
                for (int j = 0; j < N; j++) kinds[j] = body->kinds[j];
        }
        const double* verts = G > 1 ? mverts.data() : body->vertices;
        const bool fin = finite_depth(opt->depth);
        const double depth = fin ? opt->depth : 0.0;
        cudaStream_t s = 0;
        DevBuf dverts, dkind, dplanes, dbad, dst, dwork, dnwork, dS, dA, dfi, dfd, dtiles, dscr, dfpt;
        dverts.alloc(sizeof(double) * 12 * N);
        dkind.alloc(sizeof(int32_t) * N);
        dplanes.alloc(sizeof(double) * P_PLANES * N);
        dbad.alloc(sizeof(int32_t));
        CUDA_OK(cudaMemcpy(dverts.p, verts, sizeof(double) * 12 * N, cudaMemcpyHostToDevice));
        CUDA_OK(cudaMemcpy(dkind.p, kinds.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
        int32_t big = 0x7fffffff;
        CUDA_OK(cudaMemcpy(dbad.p, &big, sizeof big, cudaMemcpyHostToDevice));
        // the statics by the reference's production rule on request; the matrices FP64 either way
        const bool prod = opt->statics_rule == HBG_STATICS_PRODUCTION;
        DevBuf dtiers;
        if (prod) dtiers.alloc(sizeof(float) * TIER_FLOATS_HOST * (size_t)N);
        launch_panel_geometry(N, dverts.as<double>(), dkind.as<int32_t>(), dplanes.as<double>(), dbad.as<int32_t>(), s,
                              prod ? dtiers.as<float>() : nullptr);
        PanelsView pv{N, dplanes.as<double>(), dkind.as<int32_t>()};
        pv.G = G;
        if (prod) pv.tiers = dtiers.as<float>();
        const size_t NS = (size_t)Nm * N, NN = (size_t)Nm * Nm;
        dst.alloc(sizeof(double) * 4 * NS);
        const int cap = std::max(1 << 16, 16 * N);
        dwork.alloc(sizeof(int32_t) * 2 * cap);
        dnwork.alloc(sizeof(int32_t));
        CUDA_OK(cudaMemset(dnwork.p, 0, sizeof(int32_t)));
        launch_statics(pv, depth, opt->logarithmic, opt->log_tolerance, dst.as<double>(), dwork.as<int32_t>(),
                       dnwork.as<int32_t>(), cap, s, prod);
        int32_t nwork = 0;
        CUDA_OK(cudaMemcpy(&nwork, dnwork.p, sizeof nwork, cudaMemcpyDeviceToHost));
        if (nwork > cap) return fail({HB_ERR_INTERNAL, "worklist overflow"});
        launch_statics_adaptive(pv, dwork.as<int32_t>(), nwork, dst.as<double>(), s);
        FreqInfo fi{omega, omega * omega / opt->gravity, 0.0, opt->logarithmic ? 1.0 : 0.0};
        FdParams fdh;
        dfi.alloc(sizeof fi);
        dfd.alloc(sizeof fdh);
        CUDA_OK(cudaMemcpy(dfi.p, &fi, sizeof fi, cudaMemcpyHostToDevice));
        if (fin) {
            make_fd_params(depth, fi.K, fdh);
            CUDA_OK(cudaMemcpy(dfd.p, &fdh, sizeof fdh, cudaMemcpyHostToDevice));
            dtiles.alloc(sizeof(double) * (T1_SIZE + T2_SIZE));
            dscr.alloc(sizeof(double) * 6912 * 3);
            dfpt.alloc(sizeof(double) * FP_PLANES * N);
            launch_fd_tiles(1, dfd.as<FdParams>(), dtiles.as<double>(), dscr.as<double>(), s);
            launch_fin_points(pv, 1, dfd.as<FdParams>(), dfpt.as<double>(), s);
        }
        dS.alloc(sizeof(double2) * NN * G);
        dA.alloc(sizeof(double2) * NN * G);
        launch_assemble_f64(pv, dst.as<double>(), 1, dfi.as<FreqInfo>(), dfd.as<FdParams>(), dtiles.as<double>(),
                            dfpt.as<double>(), fin, dS.as<double2>(), dA.as<double2>(), NN, s);
        if (G > 1) launch_sectors_f64(dS.as<double2>(), dA.as<double2>(), 1, G, Nm, NN, s);
        CUDA_OK(cudaDeviceSynchronize());
        CUDA_OK(cudaGetLastError());
        if (statics) CUDA_OK(cudaMemcpy(statics, dst.p, sizeof(double) * 4 * NS, cudaMemcpyDeviceToHost));
        if (S) CUDA_OK(cudaMemcpy(S, dS.p, sizeof(double2) * NN * G, cudaMemcpyDeviceToHost));
        if (A) CUDA_OK(cudaMemcpy(A, dA.p, sizeof(double2) * NN * G, cudaMemcpyDeviceToHost));
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    } catch (...) {
        return fail({HB_ERR_INTERNAL, "internal error"});
    }
}

extern "C" HbStatus hbg_debug_gemm_tf32(int32_t M, int32_t N, int32_t K, const float* A, const float* B, float* C,
                                        int32_t subtract) {
    try {
        if (!A || !B || !C) return fail({HB_ERR_ARGUMENT, "null argument"});
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            return fail({HB_ERR_UNSUPPORTED, "no CUDA device: this library runs the path on the GPU only"});
        device_ctx(0);
        const char* msg = "";
        int rc = debug_gemm_tf32(M, N, K, A, B, C, subtract != 0, &msg);
        if (rc) return fail({rc, msg});
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    }
}

extern "C" HbStatus hbg_debug_lu_f64(int32_t n, int32_t batch, const double* A, int32_t nrhs, const double* B,
                                     double* X) {
    try {
        if (!A || !B || !X) return fail({HB_ERR_ARGUMENT, "null argument"});
        if (n <= 0 || batch <= 0 || nrhs <= 0 || nrhs > 32) return fail({HB_ERR_VALUE, "debug LU: n, batch > 0, 0 < nrhs <= 32"});
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            return fail({HB_ERR_UNSUPPORTED, "no CUDA device: this library runs the path on the GPU only"});
        device_ctx(0);
        const size_t NN = (size_t)n * n, nb = (size_t)nrhs * n;
        double2 *dA = nullptr, *dB = nullptr, *dX = nullptr;
        int32_t *dp = nullptr, *di = nullptr;
        auto release = [&]() {
            cudaFree(dA);
            cudaFree(dB);
            cudaFree(dX);
            cudaFree(dp);
            cudaFree(di);
        };
        if (cudaMalloc(&dA, sizeof(double2) * NN * batch) != cudaSuccess ||
            cudaMalloc(&dB, sizeof(double2) * nb * batch) != cudaSuccess ||
            cudaMalloc(&dX, sizeof(double2) * nb * batch) != cudaSuccess ||
            cudaMalloc(&dp, sizeof(int32_t) * (size_t)n * batch) != cudaSuccess ||
            cudaMalloc(&di, sizeof(int32_t) * batch) != cudaSuccess) {
            release();
            return fail({HB_ERR_INTERNAL, "device memory allocation failed"});
        }
        cudaStream_t s = nullptr;
        cudaMemcpy(dA, A, sizeof(double2) * NN * batch, cudaMemcpyHostToDevice);
        cudaMemcpy(dB, B, sizeof(double2) * nb * batch, cudaMemcpyHostToDevice);
        int64_t launches = 0;
        lu_factor_f64(n, batch, dA, NN, dp, di, s, &launches);
        lu_solve_f64(n, batch, dA, NN, dp, nrhs, dB, dX, s);
        std::vector<int32_t> info(batch);
        cudaMemcpy(info.data(), di, sizeof(int32_t) * batch, cudaMemcpyDeviceToHost);
        cudaMemcpy(X, dX, sizeof(double2) * nb * batch, cudaMemcpyDeviceToHost);
        const cudaError_t e = cudaGetLastError();
        release();
        if (e != cudaSuccess) return fail({HB_ERR_INTERNAL, std::string("CUDA: ") + cudaGetErrorString(e)});
        for (int f = 0; f < batch; f++)
            if (info[f]) return fail({HB_ERR_NUMERICAL, "singular matrix (zero pivot " + std::to_string(info[f]) + ")"});
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    }
}

static int current_device_ready() {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        throw Failure{HB_ERR_UNSUPPORTED, "no CUDA device: this library runs the path on the GPU only"};
    int dev = 0;
    CUDA_OK(cudaGetDevice(&dev));
    device_ctx(dev);
    return dev;
}

extern "C" HbStatus hbg_surrogate_train(int64_t n_train, int32_t batch, int32_t steps, double lr, uint64_t seed,
                                        int64_t n_val, float* params, float* norm, double* report) {
    try {
        if (!params || !norm || !report) return fail({HB_ERR_ARGUMENT, "null argument"});
        current_device_ready();
        const char* msg = "";
        int rc = surrogate_train(n_train, batch, steps, lr, seed, n_val, params, norm, report, &msg);
        if (rc) return fail({rc, msg});
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    }
}

extern "C" HbStatus hbg_surrogate_grad(const float* params, int32_t n, const float* inputs, const float* targets,
                                       float* grads, double* loss) {
    try {
        if (!params || !inputs || !targets || !grads || !loss) return fail({HB_ERR_ARGUMENT, "null argument"});
        current_device_ready();
        const char* msg = "";
        int rc = surrogate_grad(params, n, inputs, targets, grads, loss, &msg);
        if (rc) return fail({rc, msg});
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    }
}

extern "C" HbStatus hbg_surrogate_eval(const float* params, const float* norm, int32_t n, const double* xy,
                                       double* out_net, double* out_table, double* ms2) {
    try {
        if (!params || !norm || !xy || !ms2) return fail({HB_ERR_ARGUMENT, "null argument"});
        if (n < 1) return fail({HB_ERR_VALUE, "n must be positive"});
        for (int32_t i = 0; i < n; i++)
            if (!(xy[2 * i] >= 0.0 && xy[2 * i] < 100.0 && xy[2 * i + 1] >= 0.0 && xy[2 * i + 1] < 50.0))
                return fail({HB_ERR_VALUE, "points must lie in the trained domain [0, 100) x [0, 50)"});
        current_device_ready();
        const char* msg = "";
        int rc = surrogate_eval(params, norm, n, xy, out_net, out_table, ms2, &msg);
        if (rc) return fail({rc, msg});
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    }
}

extern "C" HbStatus hbg_last_surrogate_pairs(int64_t* n) {
    if (!n) return fail({HB_ERR_ARGUMENT, "null argument"});
    *n = last_surrogate_pairs();
    return HB_OK;
}

extern "C" HbStatus hbg_measure_peaks(double* out3) {
    try {
        if (!out3) return fail({HB_ERR_ARGUMENT, "null argument"});
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            return fail({HB_ERR_UNSUPPORTED, "no CUDA device: this library runs the path on the GPU only"});
        const char* msg = "";
        int rc = measure_peaks(out3, &msg);
        if (rc) return fail({rc, msg});
        return HB_OK;
    } catch (const Failure& f) {
        return fail(f);
    }
}

extern "C" HbStatus hbg_last_ir_history(double* ratios32, int32_t* n) {
    if (!ratios32 || !n) return fail({HB_ERR_ARGUMENT, "null argument"});
    const IrHistory& h = last_ir_history();
    for (int i = 0; i < h.n; i++) ratios32[i] = h.ratio[i];
    *n = h.n;
    return HB_OK;
}

extern "C" HbStatus hbg_last_ir_iterations(int32_t* n) {
    if (!n) return fail({HB_ERR_ARGUMENT, "null argument"});
    *n = last_ir_iterations();
    return HB_OK;
}

extern "C" HbStatus hbg_tuned_tiles(int32_t device, int32_t* state, int32_t* wide, float* us) {
    if (!state || !wide || !us) return fail({HB_ERR_ARGUMENT, "null argument"});
    if (device < 0 || device >= 16) return fail({HB_ERR_ARGUMENT, "device ordinal out of range"});
    *state = lu_tuned_tiles(device, wide, us);
    return HB_OK;
}

extern "C" const char* hb_last_error_message(void) { return g_error.c_str(); }

extern "C" HbStatus hb_last_error_location(HbLocation* location) {
    if (!location) return HB_ERR_ARGUMENT;
    *location = g_location;
    return HB_OK;
}

extern "C" uint32_t hb_abi_version(void) { return HB_ABI_VERSION; }
extern "C" uint32_t hbg_library_version(void) { return HBG_ABI_VERSION; }
