// hbg_model.cu -- the model/solve/results subset of the reference's C ABI (hydrobem.h), for the
// items of the low-order open-sea route of rigid bodies.  Objects: the model (""),
// "environment", "options", "meshes/<name>" (kind panels: vertices [P,4,3], symmetry) and
// "bodies/<name>" (mesh, interior_surface, interior_surface_mesh, position, rotation_center; yaw 0).
// Several bodies interact in one solve, 6 rigid modes each in the order the bodies were added, each
// mesh moved to the body's position and the modes about its rotation centre (body-local, as the
// reference's document_schema.rs:281-285 items).  A mesh with symmetry planes
// is expanded to the full mesh (the stored elements, then their x, y and xy reflections,
// geometry.rs:208-235), which solves the same discrete equations as the reference's character
// decomposition.  Items and routes outside this subset are refused with HB_ERR_UNSUPPORTED, as the
// reference refuses routes it lacks.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace hbg {

struct MeshObj {
    std::string name;
    std::vector<double> vertices;  // [P][4][3]
    std::string symmetry = "none";
};

struct BodyObj {
    std::string name;
    std::string mesh;
    std::string interior = "detect";
    std::string interior_mesh;
    double position[3] = {0.0, 0.0, 0.0};         // the global position of the body origin
    double rotation_center[3] = {0.0, 0.0, 0.0};  // body-local
    // mass properties (document_schema.rs:287-297): centre of gravity (body-local), mass given or
    // "displaced", inertia as components or radii of gyration about inertia_origin
    bool has_cg = false;
    double cg[3] = {0.0, 0.0, 0.0};
    int mass_kind = 0;  // 0 none, 1 given, 2 displaced
    double mass = 0.0;
    std::string inertia_input = "radii_of_gyration";
    double I[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // Ixx, Ixy, Ixz, Iyy, Iyz, Izz
    double gyration[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    std::string inertia_origin = "center_of_gravity";  // or rotation_center, or point
    double inertia_point[3] = {0.0, 0.0, 0.0};          // body-local
};

struct Quantity {
    std::string name;
    int32_t dtype;
    std::vector<size_t> shape;
    std::vector<unsigned char> data;
};

}  // namespace hbg

struct HbResults {
    std::vector<hbg::Quantity> q;
};

struct HbModel {
    std::mutex lock;
    std::atomic<int32_t> cancel{0};
    std::atomic<bool> solving{false};
    // environment
    std::vector<double> omegas, periods, headings;
    std::string frequency_input = "omegas";
    double depth = INFINITY, gravity = 9.80665, density = 1000.0;
    // options
    bool logarithmic = true;
    double log_tolerance = 1e-4;
    std::string precision = "fp64";
    std::string statics_rule = "accurate";  // gpu_statics_rule: accurate or production (mixed form)
    int64_t device = 0;
    bool motion = false;
    bool field_pressure = false;
    // the mean drift by momentum conservation (Kochin functions on kochin_angles angles, 0: automatic)
    bool drift_momentum = false, drift_bidirectional = false;
    int64_t kochin_angles = 0;
    std::vector<double> field_points;  // [P][3] global
    std::vector<hbg::MeshObj> meshes;
    std::vector<hbg::BodyObj> bodies;
    std::unique_ptr<HbResults> results;
};

namespace hbg {

constexpr uint64_t OBJ_MODEL = 0, OBJ_ENV = 1, OBJ_OPTIONS = 2, OBJ_MESH0 = 1000, OBJ_BODY0 = 2000000;

static HbStatus refuse(HbStatus code, const std::string& msg) { return fail(Failure{code, msg}); }

template <class F>
static HbStatus guard(F&& f) {
    try {
        return f();
    } catch (const Failure& e) {
        return fail(e);
    } catch (const std::exception& e) {
        return fail(Failure{HB_ERR_INTERNAL, std::string("internal error: ") + e.what()});
    } catch (...) {
        return fail(Failure{HB_ERR_INTERNAL, "internal error"});
    }
}

static bool is_mesh(const HbModel* m, uint64_t o) { return o >= OBJ_MESH0 && o < OBJ_MESH0 + m->meshes.size(); }
static bool is_body(const HbModel* m, uint64_t o) { return o >= OBJ_BODY0 && o < OBJ_BODY0 + m->bodies.size(); }

static std::vector<double> reals(const double* data, const size_t* shape, size_t ndim, size_t& count) {
    count = 1;
    for (size_t i = 0; i < ndim; i++) count *= shape[i];
    return std::vector<double>(data, data + count);
}

static void add_quantity(HbResults* r, const std::string& name, int32_t dtype, std::vector<size_t> shape,
                         const void* src, size_t bytes) {
    Quantity q{name, dtype, std::move(shape), std::vector<unsigned char>(bytes)};
    if (bytes) memcpy(q.data.data(), src, bytes);
    r->q.push_back(std::move(q));
}

// The full panels of stored panels with symmetry planes (the reflected copies, orientation restored).
static std::vector<double> reflect(const std::vector<double>& vertices, const std::string& symmetry) {
    std::vector<std::pair<double, double>> refl = {{1.0, 1.0}};
    if (symmetry == "yz" || symmetry == "xz_and_yz") refl.push_back({-1.0, 1.0});
    if (symmetry == "xz" || symmetry == "xz_and_yz") refl.push_back({1.0, -1.0});
    if (symmetry == "xz_and_yz") refl.push_back({-1.0, -1.0});
    size_t P = vertices.size() / 12;
    std::vector<double> out;
    out.reserve(refl.size() * vertices.size());
    for (auto [sx, sy] : refl)
        for (size_t p = 0; p < P; p++) {
            const double* v = &vertices[12 * p];
            int order[4] = {0, 1, 2, 3};
            if (sx * sy < 0) {
                order[1] = 3;
                order[3] = 1;
            }
            for (int i = 0; i < 4; i++) {
                const double* q = v + 3 * order[i];
                out.push_back(sx * q[0]);
                out.push_back(sy * q[1]);
                out.push_back(q[2]);
            }
        }
    return out;
}

static std::vector<double> expand(const MeshObj& m) { return reflect(m.vertices, m.symmetry); }

// interior.rs:79-138 projected: the interior free surface as the vertical projection onto z = z0 (the free
// surface in body coordinates) of the downward-facing wetted panels, vertex order reversed so that the
// projected panels face up; panels lying in z0 (a zero-draft part) and vertical ones (|n_z| <= 1e-6) are
// skipped; an upward-facing panel makes the projection multi-valued.  The normal is the panel's: the unit
// cross product of its diagonals (geometry.rs:160-165).  why: the reason when the surface cannot be made.
static std::vector<double> projected_lid(const std::vector<double>& v, double z0, std::string& why) {
    constexpr double SLOPE = 1e-6, PLANE_TOL = 1e-6;
    const size_t P = v.size() / 12;
    double ext = 1.0;
    for (double x : v) ext = std::max(ext, std::fabs(x));
    const double tol = PLANE_TOL * ext;
    std::vector<double> out;
    for (size_t p = 0; p < P; p++) {
        const double* q = &v[12 * p];
        bool flat = true;
        for (int i = 0; i < 4; i++) flat = flat && std::fabs(q[3 * i + 2] - z0) <= tol;
        if (flat) continue;
        const double d1[3] = {q[6] - q[0], q[7] - q[1], q[8] - q[2]}, d2[3] = {q[9] - q[3], q[10] - q[4], q[11] - q[5]};
        const double n[3] = {d1[1] * d2[2] - d1[2] * d2[1], d1[2] * d2[0] - d1[0] * d2[2], d1[0] * d2[1] - d1[1] * d2[0]};
        const double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        const double nz = nn > 0.0 ? n[2] / nn : 0.0;
        if (nz > SLOPE) {
            why = "wetted element " + std::to_string(p + 1) +
                  " faces upward, so the vertical projection of the wetted surface is multi-valued";
            return {};
        }
        if (nz >= -SLOPE) continue;  // vertical
        for (int i = 0; i < 4; i++) {
            out.push_back(q[3 * (3 - i)]);
            out.push_back(q[3 * (3 - i) + 1]);
            out.push_back(z0);
        }
    }
    if (out.empty()) why = "no wetted element faces downward";
    return out;
}

// ------------------------------------------------------------------ graded interior surface
// interior.rs:139-515 graded, on the stored panels of a mesh whose symmetry flags isx / isy declare the
// planes x = 0 / y = 0.  The waterline is rebuilt as closed contours in the quadrant x, y >= 0, each
// region fanned from its area centroid to every waterline segment, the rays cut at
// t_k = sin(pi k / (2N)), N = ceil(mean ray / mean segment); the innermost cell a triangle, the others
// quadrilaterals.  The output is stored-form panels (reflected like the mesh), facing up.
namespace graded {

struct P2 {
    double x, y;
};
using Loop = std::vector<P2>;

static double dist(P2 a, P2 b) { return std::hypot(a.x - b.x, a.y - b.y); }
static double orient(P2 o, P2 a, P2 b) { return (a.x - o.x) * (b.y - o.y) - (a.y - o.y) * (b.x - o.x); }

// polygon.rs:94-99
static double seg_dist(P2 x, P2 a, P2 b) {
    const double ex = b.x - a.x, ey = b.y - a.y, ee = ex * ex + ey * ey;
    const double t = ee > 0.0 ? std::min(1.0, std::max(0.0, ((x.x - a.x) * ex + (x.y - a.y) * ey) / ee)) : 0.0;
    return dist(x, P2{a.x + t * ex, a.y + t * ey});
}

// polygon.rs:81-90: the segments pq and ab cross, or an end lies exactly on the other
static bool meet(P2 p, P2 q, P2 a, P2 b) {
    const double d1 = orient(a, b, p), d2 = orient(a, b, q), d3 = orient(p, q, a), d4 = orient(p, q, b);
    if (((d1 > 0 && d2 < 0) || (d1 < 0 && d2 > 0)) && ((d3 > 0 && d4 < 0) || (d3 < 0 && d4 > 0))) return true;
    auto on = [](P2 o, P2 e, P2 x, double d) {
        return d == 0.0 && x.x >= std::min(o.x, e.x) && x.x <= std::max(o.x, e.x) && x.y >= std::min(o.y, e.y) &&
               x.y <= std::max(o.y, e.y);
    };
    return on(a, b, p, d1) || on(a, b, q, d2) || on(p, q, a, d3) || on(p, q, b, d4);
}

// polygon.rs:111-149: two loops, or two edges of one loop that do not follow each other, cross or
// come within tol
static bool loops_meet(const std::vector<Loop>& loops, double tol) {
    struct E {
        size_t l, k;
        P2 a, b;
    };
    std::vector<E> e;
    for (size_t l = 0; l < loops.size(); l++)
        for (size_t k = 0; k < loops[l].size(); k++) e.push_back({l, k, loops[l][k], loops[l][(k + 1) % loops[l].size()]});
    auto lo = [&](const E& s, int c) { return (c ? std::min(s.a.y, s.b.y) : std::min(s.a.x, s.b.x)) - tol; };
    auto hi = [&](const E& s, int c) { return (c ? std::max(s.a.y, s.b.y) : std::max(s.a.x, s.b.x)) + tol; };
    for (size_t i = 0; i < e.size(); i++)
        for (size_t j = i + 1; j < e.size(); j++) {
            const E &f = e[i], &g = e[j];
            if (lo(f, 0) > hi(g, 0) || lo(g, 0) > hi(f, 0) || lo(f, 1) > hi(g, 1) || lo(g, 1) > hi(f, 1)) continue;
            if (f.l == g.l) {
                const size_t n = loops[f.l].size();
                if (n <= 3 || (f.k + 1) % n == g.k || (g.k + 1) % n == f.k) continue;
            }
            if (meet(f.a, f.b, g.a, g.b) || seg_dist(f.a, g.a, g.b) <= tol || seg_dist(f.b, g.a, g.b) <= tol ||
                seg_dist(g.a, f.a, f.b) <= tol || seg_dist(g.b, f.a, f.b) <= tol)
                return true;
        }
    return false;
}

static double signed_area(const Loop& l) {
    double a = 0.0;
    for (size_t k = 0; k < l.size(); k++) a += l[k].x * l[(k + 1) % l.size()].y - l[(k + 1) % l.size()].x * l[k].y;
    return 0.5 * a;
}

static bool inside(const Loop& l, P2 x) {
    bool c = false;
    for (size_t k = 0; k < l.size(); k++) {
        const P2 p = l[k], q = l[(k + 1) % l.size()];
        if ((p.y > x.y) != (q.y > x.y) && x.x < p.x + (x.y - p.y) / (q.y - p.y) * (q.x - p.x)) c = !c;
    }
    return c;
}

// The waterplane regions of the stored panels in the quadrant x, y >= 0 (interior.rs:139-153, 358-391):
// counter-clockwise outer contours, each with its clockwise holes (a hole belongs to the smallest outer
// contour around it); (sx, sy) maps back to the stored side; target the mean waterline segment length;
// merge: collinear points merged (the waterline generator; the fan keeps them).  False with the reason.
struct Regions {
    std::vector<Loop> outers;
    std::vector<std::vector<Loop>> holes;
    double sx = 1.0, sy = 1.0, target = 0.0, tol = 0.0, z0 = 0.0;
    bool ax_x = false, ax_y = false;
};

static Loop merge_collinear(const Loop& l, double tol);

static bool regions(const std::vector<double>& v, bool isx, bool isy, double z0, bool merge, Regions& g,
                    std::string& why) {
    constexpr double SLOPE = 1e-6, PLANE_TOL = 1e-6;
    const size_t P = v.size() / 12;
    double ext = 1.0;  // the mesh reference length
    for (double x : v) ext = std::max(ext, std::fabs(x));
    const double tol = PLANE_TOL * ext;
    // interior.rs:158-214 waterline segments, the body section on their left
    std::vector<std::pair<P2, P2>> segs;
    for (size_t p = 0; p < P; p++) {
        const double* q = &v[12 * p];
        const double d1[3] = {q[6] - q[0], q[7] - q[1], q[8] - q[2]}, d2[3] = {q[9] - q[3], q[10] - q[4], q[11] - q[5]};
        double n[3] = {d1[1] * d2[2] - d1[2] * d2[1], d1[2] * d2[0] - d1[0] * d2[2], d1[0] * d2[1] - d1[1] * d2[0]};
        const double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nn > 0.0)
            for (double& c : n) c /= nn;
        if (std::hypot(n[0], n[1]) < SLOPE) continue;
        for (int i = 0; i < 4; i++) {
            const double *u = q + 3 * i, *w = q + 3 * ((i + 1) % 4);
            if (std::fabs(u[2] - z0) > tol || std::fabs(w[2] - z0) > tol) continue;
            P2 a{u[0], u[1]}, b{w[0], w[1]};
            if (dist(a, b) <= tol) continue;
            if ((b.x - a.x) * -n[1] + (b.y - a.y) * n[0] < 0.0) std::swap(a, b);
            segs.push_back({a, b});
        }
    }
    if (segs.empty()) return why = "the wetted surface has no waterline", false;
    double total = 0.0;
    for (auto& s : segs) total += dist(s.first, s.second);
    g.target = total / (double)segs.size();
    double mx = 0.0, my = 0.0;
    for (auto& s : segs) mx += s.first.x + s.second.x, my += s.first.y + s.second.y;
    const double sx = isx && mx < 0.0 ? -1.0 : 1.0, sy = isy && my < 0.0 ? -1.0 : 1.0;
    for (auto& s : segs) {
        s.first = {sx * s.first.x, sy * s.first.y};
        s.second = {sx * s.second.x, sy * s.second.y};
        if (sx * sy < 0.0) std::swap(s.first, s.second);
    }
    // interior.rs:217-272 open chains and closed loops
    const size_t n = segs.size();
    std::vector<long> nxt(n, -1), prv(n, -1);
    for (size_t i = 0; i < n; i++)
        for (size_t j = 0; j < n; j++) {
            if (i == j || dist(segs[i].second, segs[j].first) > tol) continue;
            if (nxt[i] >= 0 || prv[j] >= 0) return why = "waterline contours touch or cross", false;
            nxt[i] = (long)j;
            prv[j] = (long)i;
        }
    std::vector<bool> used(n, false);
    std::vector<Loop> chains, loops;
    for (size_t s = 0; s < n; s++) {
        if (prv[s] >= 0) continue;
        Loop c{segs[s].first};
        for (long k = (long)s; k >= 0; k = nxt[k]) {
            used[k] = true;
            c.push_back(segs[k].second);
        }
        chains.push_back(c);
    }
    for (size_t s = 0; s < n; s++) {
        if (used[s]) continue;
        Loop c;
        for (long k = (long)s; !used[k];) {
            used[k] = true;
            c.push_back(segs[k].first);
            k = nxt[k];
            if (k < 0) return why = "broken waterline loop", false;
        }
        loops.push_back(c);
    }
    // interior.rs:274-340 the open chains closed along the symmetry axes: the quadrant boundary
    // traversed +x along y = 0, then -y along x = 0, wrapping through the corner
    const bool ax_x = isy, ax_y = isx;
    auto on_x = [&](P2 p) { return ax_x && std::fabs(p.y) <= tol && (p.x >= -tol || !ax_y); };
    auto on_y = [&](P2 p) { return ax_y && std::fabs(p.x) <= tol && (p.y >= -tol || !ax_x); };
    auto key_start = [&](P2 p) { return on_x(p) ? std::make_pair(0, p.x) : std::make_pair(1, -p.y); };
    auto key_end = [&](P2 p) { return on_y(p) ? std::make_pair(1, -p.y) : std::make_pair(0, p.x); };
    const std::string open = "the waterline does not close";
    for (auto& c : chains)
        if (!(on_x(c.front()) || on_y(c.front())) || !(on_x(c.back()) || on_y(c.back()))) return why = open, false;
    std::vector<bool> cused(chains.size(), false);
    for (size_t c0 = 0; c0 < chains.size(); c0++) {
        if (cused[c0]) continue;
        Loop l;
        for (size_t c = c0;;) {
            cused[c] = true;
            l.insert(l.end(), chains[c].begin(), chains[c].end());
            const auto ke = key_end(chains[c].back());
            long best = -1;
            bool wrap = false;
            for (int pass = 0; pass < 2 && best < 0; pass++) {
                for (size_t d = 0; d < chains.size(); d++) {
                    if (cused[d] && d != c0) continue;
                    const auto ks = key_start(chains[d].front());
                    if (pass == 0 && ks < ke) continue;
                    if (best < 0 || ks < key_start(chains[best].front())) best = (long)d;
                }
                wrap = pass == 1;
            }
            if (best < 0) return why = open, false;
            if (ke.first == 0 && key_start(chains[best].front()).first == 1 && !wrap) return why = open, false;
            if (wrap) {
                if (!(ax_x && ax_y)) return why = open, false;
                l.push_back(P2{0.0, 0.0});
            }
            if ((size_t)best == c0) break;
            c = (size_t)best;
        }
        loops.push_back(l);
    }
    // interior.rs:343-357 repeated points (and the closing repetition) dropped
    for (auto& l : loops) {
        Loop c;
        for (P2 p : l)
            if (c.empty() || dist(c.back(), p) > tol) c.push_back(p);
        while (c.size() > 1 && dist(c.front(), c.back()) <= tol) c.pop_back();
        l = merge ? merge_collinear(c, tol) : c;
    }
    if (loops_meet(loops, tol)) return why = "waterline contours cross or touch", false;
    // interior.rs:360-391 outer loops (counter-clockwise) and the holes of each
    std::vector<Loop> holes;
    for (auto& l : loops)
        if (l.size() >= 3) (signed_area(l) > 0.0 ? g.outers : holes).push_back(l);
    if (g.outers.empty()) return why = "no enclosed region", false;
    g.holes.assign(g.outers.size(), {});
    for (auto& h : holes) {
        long owner = -1;
        for (size_t o = 0; o < g.outers.size(); o++)
            if (inside(g.outers[o], h[0]) &&
                (owner < 0 || std::fabs(signed_area(g.outers[o])) < std::fabs(signed_area(g.outers[owner]))))
                owner = (long)o;
        if (owner < 0) return why = "a waterline contour lies outside the body", false;
        g.holes[owner].push_back(h);
    }
    g.sx = sx;
    g.sy = sy;
    g.tol = tol;
    g.z0 = z0;
    g.ax_x = ax_x;
    g.ax_y = ax_y;
    return true;
}

// interior.rs:394-409 a polygon (3 or 4 corners, counter-clockwise in the quadrant) as a stored panel
static void emit_panel(const Regions& g, const P2* cs, int k, std::vector<double>& out) {
    double w[4][3];
    for (int i = 0; i < k; i++) w[i][0] = g.sx * cs[i].x, w[i][1] = g.sy * cs[i].y, w[i][2] = g.z0;
    if (g.sx * g.sy < 0.0) std::reverse(&w[0], &w[k]);
    if (k == 3)
        for (int d = 0; d < 3; d++) w[3][d] = w[2][d];
    for (int i = 0; i < 4; i++)
        for (int d = 0; d < 3; d++) out.push_back(w[i][d]);
}

static std::vector<double> lid(const std::vector<double>& v, bool isx, bool isy, double z0, std::string& why) {
    Regions g;
    if (!regions(v, isx, isy, z0, false, g, why)) return {};
    const double tol = g.tol;
    const bool ax_x = g.ax_x, ax_y = g.ax_y;
    const std::vector<Loop>& outers = g.outers;
    for (const auto& hs : g.holes)
        if (!hs.empty()) return why = "a waterplane region has an opening (a moonpool); use 'waterline'", std::vector<double>{};
    std::vector<double> out;
    auto emit = [&](std::initializer_list<P2> cs) { emit_panel(g, cs.begin(), (int)cs.size(), out); };
    // interior.rs:447-517 the fan of each region
    for (const Loop& l : outers) {
        double a = 0.0, cx = 0.0, cy = 0.0;
        bool on_y0 = false, on_x0 = false;
        for (size_t i = 0; i < l.size(); i++) {
            const P2 p = l[i], q = l[(i + 1) % l.size()];
            const double c = p.x * q.y - p.y * q.x;
            a += 0.5 * c;
            cx += (p.x + q.x) * c / 6.0;
            cy += (p.y + q.y) * c / 6.0;
            on_y0 = on_y0 || (ax_x && std::fabs(p.y) <= tol && std::fabs(q.y) <= tol);
            on_x0 = on_x0 || (ax_y && std::fabs(p.x) <= tol && std::fabs(q.x) <= tol);
        }
        P2 c{cx / a, cy / a};
        if (on_x0) c.x = 0.0;
        if (on_y0) c.y = 0.0;
        std::vector<std::pair<P2, P2>> fan;
        double ray = 0.0, seg = 0.0;
        for (size_t i = 0; i < l.size(); i++) {
            const P2 p = l[i], q = l[(i + 1) % l.size()];
            const double s = orient(c, p, q);
            if (std::fabs(s) <= tol * dist(p, q)) continue;  // an edge through the centroid bounds no area
            if (s < 0.0)
                return why = "a ray from the centroid of a waterplane region meets its waterline more than once; use 'waterline'",
                       std::vector<double>{};
            fan.push_back({p, q});
            ray += 0.5 * (dist(c, p) + dist(c, q));
            seg += dist(p, q);
        }
        if (fan.empty()) return why = "no enclosed region", std::vector<double>{};
        const int N = std::max(1, (int)std::ceil(ray / seg - 1e-9));
        std::vector<double> t(N + 1);
        for (int k = 0; k <= N; k++) t[k] = k == N ? 1.0 : std::sin(0.5 * PI * k / N);
        auto at = [&](P2 p, double s) { return P2{c.x + s * (p.x - c.x), c.y + s * (p.y - c.y)}; };
        for (auto& [p, q] : fan) {
            emit({c, at(p, t[1]), at(q, t[1])});
            for (int k = 1; k < N; k++) emit({at(p, t[k]), at(p, t[k + 1]), at(q, t[k + 1]), at(q, t[k])});
        }
    }
    return out;
}

// ------------------------------------------------------------------ waterline generator
// polygon.rs:154-700 and interior.rs:408-434: the regions (collinear points merged, holes kept)
// triangulated -- every hole bridged to the outer loop, the bridged polygon cut into ears, Lawson flips
// to the constrained Delaunay triangulation -- then refined (Ruppert's circumcentre insertion with
// Shewchuk's rules) to edges of at most twice the mean waterline segment and angles of at least 25
// degrees, in one fixed order of insertions, so the same triangles on every run.

// polygon.rs:154-170 the loop without the vertices within tol of the line through their neighbours
static Loop merge_collinear(const Loop& l, double tol) {
    Loop c = l;
    bool changed = true;
    while (changed && c.size() > 3) {
        changed = false;
        for (size_t i = 0; i < c.size(); i++) {
            const size_t n = c.size();
            const P2 a = c[(i + n - 1) % n], b = c[i], d = c[(i + 1) % n];
            if (std::fabs(orient(a, b, d)) <= tol * dist(a, d)) {
                c.erase(c.begin() + (long)i);
                changed = true;
                break;
            }
        }
    }
    return c;
}

// polygon.rs:220-258 the holes merged into the outer loop (the rightmost hole first), each by a bridge
// from its rightmost vertex (the last of equal ones) to the nearest vertex visible from it (the first
// of equal ones), preferably to its right
static bool bridge(const Loop& outer, std::vector<Loop> holes, double eps, Loop& poly) {
    poly = outer;
    auto right = [](const Loop& l) {
        double r = -INFINITY;
        for (const P2& p : l) r = std::max(r, p.x);
        return r;
    };
    std::stable_sort(holes.begin(), holes.end(), [&](const Loop& a, const Loop& b) { return right(b) < right(a); });
    for (size_t hi = 0; hi < holes.size(); hi++) {
        const Loop& h = holes[hi];
        size_t mi = 0;
        for (size_t i = 0; i < h.size(); i++)
            if (h[i].x >= h[mi].x) mi = i;
        const P2 m = h[mi];
        const size_t n = poly.size();
        auto visible = [&](size_t k) {
            const P2 p = poly[k];
            for (size_t e = 0; e < n; e++)
                if (!(e == k || (e + 1) % n == k) && meet(m, p, poly[e], poly[(e + 1) % n])) return false;
            for (size_t e = 0; e < h.size(); e++)
                if (!(e == mi || (e + 1) % h.size() == mi) && meet(m, p, h[e], h[(e + 1) % h.size()])) return false;
            for (size_t l = hi + 1; l < holes.size(); l++)
                for (size_t e = 0; e < holes[l].size(); e++)
                    if (meet(m, p, holes[l][e], holes[l][(e + 1) % holes[l].size()])) return false;
            return true;
        };
        long best = -1;
        for (int pass = 0; pass < 2 && best < 0; pass++)
            for (size_t k = 0; k < n; k++)
                if ((pass == 1 || poly[k].x >= m.x - eps) && visible(k) &&
                    (best < 0 || dist(poly[k], m) < dist(poly[best], m)))
                    best = (long)k;
        if (best < 0) return false;
        Loop next(poly.begin(), poly.begin() + best + 1);
        for (size_t k = 0; k <= h.size(); k++) next.push_back(h[(mi + k) % h.size()]);
        next.insert(next.end(), poly.begin() + best, poly.end());
        poly = next;
    }
    return true;
}

using Tri = std::array<long, 3>;

// polygon.rs:262-306 ear clipping of the counter-clockwise bridged polygon; straight corners dropped
static bool ears(const Loop& poly, double eps, std::vector<Tri>& out) {
    auto straight = [](P2 a, P2 b, P2 c) { return std::fabs(orient(a, b, c)) <= 1e-12 * dist(a, b) * dist(b, c); };
    std::vector<long> idx(poly.size());
    for (size_t i = 0; i < idx.size(); i++) idx[i] = (long)i;
    while (idx.size() > 3) {
        const size_t n = idx.size();
        bool clipped = false;
        for (size_t i = 0; i < n; i++) {
            const long ia = idx[(i + n - 1) % n], ib = idx[i], ic = idx[(i + 1) % n];
            const P2 a = poly[ia], b = poly[ib], c = poly[ic];
            if (straight(a, b, c)) {
                idx.erase(idx.begin() + (long)i);
                clipped = true;
                break;
            }
            if (orient(a, b, c) < 0.0) continue;  // reflex
            auto at = [&](P2 x, P2 y) { return std::fabs(x.x - y.x) <= eps && std::fabs(x.y - y.y) <= eps; };
            bool ear = true;
            for (long k : idx) {
                const P2 x = poly[k];
                if (!(at(x, a) || at(x, b) || at(x, c) ||
                      !(orient(a, b, x) > 0.0 && orient(b, c, x) > 0.0 && orient(c, a, x) > 0.0))) {
                    ear = false;
                    break;
                }
            }
            if (ear) {
                out.push_back({ia, ib, ic});
                idx.erase(idx.begin() + (long)i);
                clipped = true;
                break;
            }
        }
        if (!clipped) return false;
    }
    if (idx.size() == 3 && !straight(poly[idx[0]], poly[idx[1]], poly[idx[2]])) out.push_back({idx[0], idx[1], idx[2]});
    return true;
}

static double incircle(P2 pa, P2 pb, P2 pc, P2 pd) {
    const double adx = pa.x - pd.x, ady = pa.y - pd.y, bdx = pb.x - pd.x, bdy = pb.y - pd.y;
    const double cdx = pc.x - pd.x, cdy = pc.y - pd.y;
    return (adx * adx + ady * ady) * (bdx * cdy - cdx * bdy) - (bdx * bdx + bdy * bdy) * (adx * cdy - cdx * ady) +
           (cdx * cdx + cdy * cdy) * (adx * bdy - bdx * ady);
}

using EdgeKey = std::pair<long, long>;
static EdgeKey ekey(long a, long b) { return {std::min(a, b), std::max(a, b)}; }
constexpr long NONE = -1;

// polygon.rs:310-388 Lawson flips to the constrained Delaunay triangulation, in place
static bool delaunay_flips(const Loop& p, std::vector<Tri>& tris) {
    std::map<EdgeKey, std::array<long, 2>> owners;
    std::vector<EdgeKey> fixed;
    for (size_t t = 0; t < tris.size(); t++)
        for (int e = 0; e < 3; e++) {
            const EdgeKey k = ekey(tris[t][e], tris[t][(e + 1) % 3]);
            auto it = owners.try_emplace(k, std::array<long, 2>{NONE, NONE}).first;
            if (it->second[0] == NONE)
                it->second[0] = (long)t;
            else if (it->second[1] == NONE)
                it->second[1] = (long)t;
            else
                fixed.push_back(k);
        }
    for (auto& k : fixed) owners[k] = {NONE, NONE};
    const size_t limit = std::max<size_t>(tris.size() * tris.size(), 16);
    size_t flips = 0;
    for (;;) {
        bool flipped = false;
        for (size_t t = 0; t < tris.size(); t++)
            for (int e = 0; e < 3; e++) {
                const long a = tris[t][e], b = tris[t][(e + 1) % 3], c = tris[t][(e + 2) % 3];
                const auto o = owners.at(ekey(a, b));
                const long u = o[0] == (long)t ? o[1] : o[0];
                if (u == NONE || u > (long)t) continue;
                int f = -1;
                for (int g = 0; g < 3 && f < 0; g++)
                    if (tris[u][g] == b && tris[u][(g + 1) % 3] == a) f = g;
                if (f < 0) return false;
                const long d = tris[u][(f + 2) % 3];
                const double ob = orient(p[a], p[b], p[c]);
                if (incircle(p[a], p[b], p[c], p[d]) > 1e-12 * ob * ob && orient(p[c], p[d], p[b]) > 0.0 &&
                    orient(p[d], p[c], p[a]) > 0.0) {
                    tris[t] = {c, d, b};
                    tris[u] = {d, c, a};
                    owners.erase(ekey(a, b));
                    owners[ekey(c, d)] = {(long)t, u};
                    const std::array<std::tuple<EdgeKey, long, long>, 2> fix = {
                        std::make_tuple(ekey(d, b), u, (long)t), std::make_tuple(ekey(c, a), (long)t, u)};
                    for (auto& [edge, from, to] : fix)
                        for (long& x : owners.at(edge))
                            if (x == from) x = to;
                    flipped = true;
                    if (++flips > limit) return false;
                    break;  // the triangle t is new: its edges at the next pass
                }
            }
        if (!flipped) return true;
    }
}

static P2 circumcentre(P2 a, P2 b, P2 c) {
    const double bx = b.x - a.x, by = b.y - a.y, cx = c.x - a.x, cy = c.y - a.y;
    const double d = 2.0 * (bx * cy - by * cx);
    const double b2 = bx * bx + by * by, c2 = cx * cx + cy * cy;
    return P2{a.x + (cy * b2 - by * c2) / d, a.y + (bx * c2 - cx * b2) / d};
}

// polygon.rs:428-576 a triangulation under refinement
struct Mesh2 {
    std::vector<P2> p;
    std::vector<Tri> t;
    std::vector<bool> alive;
    std::map<EdgeKey, std::array<long, 2>> owners;
    std::map<EdgeKey, double> segs;  // boundary edges, with the length of the boundary edge each was split from

    long add_tri(Tri q) {
        const long id = (long)t.size();
        t.push_back(q);
        alive.push_back(true);
        for (int e = 0; e < 3; e++) {
            auto& o = owners.try_emplace(ekey(q[e], q[(e + 1) % 3]), std::array<long, 2>{NONE, NONE}).first->second;
            if (o[0] == NONE)
                o[0] = id;
            else
                o[1] = id;
        }
        return id;
    }
    void kill(long id) {
        alive[id] = false;
        const Tri q = t[id];
        for (int e = 0; e < 3; e++) {
            auto it = owners.find(ekey(q[e], q[(e + 1) % 3]));
            if (it == owners.end()) continue;
            for (long& x : it->second)
                if (x == id) x = NONE;
            if (it->second[0] == NONE && it->second[1] == NONE) owners.erase(it);
        }
    }
    long across(long tt, long a, long b) const {
        auto it = owners.find(ekey(a, b));
        if (it == owners.end()) return NONE;
        return it->second[0] == tt ? it->second[1] : it->second[0];
    }
    bool is_seg(long a, long b) const { return segs.count(ekey(a, b)) != 0; }
    // the triangle holding c, walked from tt along the line from its centroid (kind 0), the first boundary
    // edge the line meets (kind 1, in u, v), or lost (kind 2)
    int locate(long tt, P2 c, long& out, long& u_out, long& v_out) const {
        Tri q = t[tt];
        const P2 g{(p[q[0]].x + p[q[1]].x + p[q[2]].x) / 3.0, (p[q[0]].y + p[q[1]].y + p[q[2]].y) / 3.0};
        long cur = tt, from = NONE;
        for (size_t step = 0; step < t.size() + 3; step++) {
            q = t[cur];
            long ex_u = NONE, ex_v = NONE, ex_n = NONE, f_u = NONE, f_v = NONE, f_n = NONE;
            bool any = false, found = false;
            for (int e = 0; e < 3; e++) {
                const long u = q[e], v = q[(e + 1) % 3];
                const double su = orient(g, c, p[u]), sv = orient(g, c, p[v]);
                if (orient(p[u], p[v], c) < 0.0 && ((su <= 0.0 && sv >= 0.0) || (su >= 0.0 && sv <= 0.0))) {
                    const long n = across(cur, u, v);
                    if (!any) f_u = u, f_v = v, f_n = n, any = true;
                    if (!found && n != from) ex_u = u, ex_v = v, ex_n = n, found = true;
                }
            }
            if (!found && any) ex_u = f_u, ex_v = f_v, ex_n = f_n, found = true;
            if (!found) {
                bool in = true;
                for (int e = 0; e < 3; e++) in = in && orient(p[q[e]], p[q[(e + 1) % 3]], c) >= 0.0;
                if (!in) return 2;
                out = cur;
                return 0;
            }
            if (is_seg(ex_u, ex_v) || ex_n == NONE) {
                u_out = ex_u;
                v_out = ex_v;
                return 1;
            }
            from = cur;
            cur = ex_n;
        }
        return 2;
    }
    // the cavity of x from tt (triangles reachable across non-boundary edges whose circumcircles hold x)
    // and its boundary edges in the sense of their triangles
    void cavity(long tt, P2 x, std::vector<long>& cav, std::vector<std::pair<long, long>>& bnd) const {
        cav.assign(1, tt);
        auto has = [&](long n) { return std::find(cav.begin(), cav.end(), n) != cav.end(); };
        for (size_t k = 0; k < cav.size(); k++) {
            const Tri q = t[cav[k]];
            for (int e = 0; e < 3; e++) {
                const long u = q[e], v = q[(e + 1) % 3];
                if (is_seg(u, v)) continue;
                const long n = across(cav[k], u, v);
                if (n == NONE || has(n)) continue;
                const Tri r = t[n];
                if (incircle(p[r[0]], p[r[1]], p[r[2]], x) > 0.0) cav.push_back(n);
            }
        }
        bnd.clear();
        for (long c : cav) {
            const Tri q = t[c];
            for (int e = 0; e < 3; e++) {
                const long u = q[e], v = q[(e + 1) % 3];
                const long n = across(c, u, v);
                if (n == NONE || !has(n) || is_seg(u, v)) bnd.push_back({u, v});
            }
        }
    }
    // the cavity replaced by the fan from the new vertex x to its boundary edges but skip; false (nothing
    // changed) when a fan triangle would not turn counter-clockwise by more than the rounding
    bool insert(const std::vector<long>& cav, const std::vector<std::pair<long, long>>& bnd, P2 x,
                std::pair<long, long> skip, std::vector<long>& fresh) {
        std::vector<std::pair<long, long>> fan;
        for (auto& uv : bnd)
            if (uv != skip) fan.push_back(uv);
        for (auto& [u, v] : fan) {
            const P2 pu = p[u], pv = p[v];
            const double l2 = (pu.x - pv.x) * (pu.x - pv.x) + (pu.y - pv.y) * (pu.y - pv.y);
            if (orient(pu, pv, x) <= 1e-9 * l2) return false;
        }
        const long id = (long)p.size();
        p.push_back(x);
        for (long c : cav) kill(c);
        fresh.clear();
        for (auto& [u, v] : fan) fresh.push_back(add_tri({u, v, id}));
        return true;
    }
};

// polygon.rs:593-700 the triangles (counter-clockwise) of a region refined to `size` and the smallest
// angle of 25 degrees; at most cap live triangles
static bool triangulate_refined(const Loop& outer, const std::vector<Loop>& holes, double eps, double size, size_t cap,
                                std::vector<std::array<P2, 3>>& out, std::string& why) {
    Loop poly;
    if (!bridge(outer, holes, eps, poly)) return why = "polygon triangulation: a hole without a bridge", false;
    std::vector<Tri> tris;
    if (!ears(poly, eps, tris)) return why = "polygon triangulation: the ear clipping failed", false;
    Mesh2 m;
    std::map<std::pair<uint64_t, uint64_t>, long> id_of;  // the two ends of a bridge are exact copies: one vertex
    std::vector<long> ids;
    for (const P2& x : poly) {
        uint64_t bx, by;
        std::memcpy(&bx, &x.x, 8);
        std::memcpy(&by, &x.y, 8);
        auto it = id_of.try_emplace({bx, by}, (long)m.p.size());
        if (it.second) m.p.push_back(x);
        ids.push_back(it.first->second);
    }
    std::vector<Tri> t;
    for (const Tri& q : tris) t.push_back({ids[q[0]], ids[q[1]], ids[q[2]]});
    if (!delaunay_flips(m.p, t)) return why = "polygon triangulation: the Delaunay flips do not end", false;
    for (const Tri& q : t) m.add_tri(q);
    double shortest = INFINITY;
    for (size_t i = 0; i < m.t.size(); i++) {
        const Tri q = m.t[i];
        for (int e = 0; e < 3; e++) {
            const long u = q[e], v = q[(e + 1) % 3];
            if (m.across((long)i, u, v) == NONE) {
                const double l = dist(m.p[u], m.p[v]);
                m.segs[ekey(u, v)] = l;
                shortest = std::min(shortest, l);
            }
        }
    }
    const double ratio = 0.5 / std::sin(25.0 * PI / 180.0);  // circumradius over the shortest edge
    std::deque<long> queue;
    for (size_t i = 0; i < m.t.size(); i++) queue.push_back((long)i);
    size_t live = m.t.size();
    std::vector<long> cav, fresh;
    std::vector<std::pair<long, long>> bnd;
    while (!queue.empty()) {
        const long i = queue.front();
        queue.pop_front();
        if (!m.alive[i] || live > cap) continue;
        const Tri q = m.t[i];
        const P2 a = m.p[q[0]], b = m.p[q[1]], c = m.p[q[2]];
        const double l0 = dist(b, c), l1 = dist(c, a), l2 = dist(a, b);
        const double lo = std::min(std::min(l0, l1), l2), hi = std::max(std::max(l0, l1), l2);
        const P2 cc = circumcentre(a, b, c);
        const bool big = hi > size;
        const bool skinny = dist(cc, a) > ratio * lo && lo >= 0.25 * shortest;
        if (!big && !skinny) continue;
        long t0 = NONE, su = NONE, sv = NONE;
        const int kind = m.locate(i, cc, t0, su, sv);
        if (kind == 2) continue;
        bool split = kind == 1, fan = false;
        size_t removed = 0;
        if (kind == 0) {
            m.cavity(t0, cc, cav, bnd);
            for (auto& [u, v] : bnd)
                if (m.is_seg(u, v)) {
                    const P2 pu = m.p[u], pv = m.p[v];
                    if ((pu.x - cc.x) * (pv.x - cc.x) + (pu.y - cc.y) * (pv.y - cc.y) < 0.0) {
                        split = true, su = u, sv = v;
                        break;
                    }
                }
            if (!split) {
                removed = cav.size();
                fan = m.insert(cav, bnd, cc, {NONE, NONE}, fresh);
            }
        }
        if (split) {
            const double l = dist(m.p[su], m.p[sv]);
            if (!(l > size || l >= 0.75 * std::min(0.5 * size, m.segs.at(ekey(su, sv))))) continue;
            const auto s = m.owners.at(ekey(su, sv));
            const long ts = s[0] != NONE ? s[0] : s[1];
            const Tri qs = m.t[ts];
            long u = NONE, v = NONE;
            for (int e = 0; e < 3 && u == NONE; e++)
                if (ekey(qs[e], qs[(e + 1) % 3]) == ekey(su, sv)) u = qs[e], v = qs[(e + 1) % 3];
            const P2 mid{0.5 * (m.p[u].x + m.p[v].x), 0.5 * (m.p[u].y + m.p[v].y)};
            m.cavity(ts, mid, cav, bnd);
            const double from = m.segs.at(ekey(u, v));
            if (m.insert(cav, bnd, mid, {u, v}, fresh)) {
                const long x = (long)m.p.size() - 1;
                m.segs.erase(ekey(u, v));
                m.segs[ekey(u, x)] = from;
                m.segs[ekey(x, v)] = from;
                live += fresh.size() - cav.size();
                for (long f : fresh) queue.push_back(f);
                if (m.alive[i]) queue.push_back(i);
            }
        } else if (fan) {
            live += fresh.size() - removed;
            for (long f : fresh) queue.push_back(f);
        }
    }
    for (size_t i = 0; i < m.t.size(); i++)
        if (m.alive[i]) out.push_back({m.p[m.t[i][0]], m.p[m.t[i][1]], m.p[m.t[i][2]]});
    return true;
}

// interior.rs:408-434 the waterline generator on the stored panels
static std::vector<double> waterline_lid(const std::vector<double>& v, bool isx, bool isy, double z0, std::string& why) {
    constexpr size_t MAX_GENERATED = 200000;  // more would make the dense system impractical
    Regions g;
    if (!regions(v, isx, isy, z0, true, g, why)) return {};
    std::vector<std::array<P2, 3>> done;
    for (size_t o = 0; o < g.outers.size(); o++) {
        if (!triangulate_refined(g.outers[o], g.holes[o], g.tol, 2.0 * g.target, MAX_GENERATED - done.size(), done, why))
            return {};
        if (done.size() > MAX_GENERATED)
            return why = "the waterplane needs more than 200000 panels of twice the mean waterline segment length; use "
                         "'graded' or a mesh of its own",
                   std::vector<double>{};
    }
    std::vector<double> out;
    for (auto& tri : done) emit_panel(g, tri.data(), 3, out);
    return out;
}

}  // namespace graded

// The panels of body b in body coordinates (bv [P][4][3]) with their kinds (bk), the interior surface
// appended.  form -1: a lone body whose mesh (and interior mesh) declare the same symmetry planes,
// placed on them, keeps the stored panels (solved by symmetry sectors, one system per sector; sym set
// to its planes), any other arrangement takes its whole mirrored mesh; 0: always the mirrored mesh;
// 1: always the stored panels (sym the mesh's planes).
static HbStatus body_panels(const HbModel* model, const BodyObj& b, int form, std::vector<double>& bv,
                            std::vector<int32_t>& bk, int32_t& sym) {
    const MeshObj* mesh = nullptr;
    const MeshObj* lid = nullptr;
    for (auto& m : model->meshes) {
        if (m.name == b.mesh) mesh = &m;
        if (m.name == b.interior_mesh) lid = &m;
    }
    if (!mesh || mesh->vertices.empty()) return refuse(HB_ERR_VALUE, "the body has no panels mesh");
    const int msym = mesh->symmetry == "yz" ? HBG_SYM_YZ : mesh->symmetry == "xz" ? HBG_SYM_XZ
                     : mesh->symmetry == "xz_and_yz"                         ? HBG_SYM_BOTH
                                                                             : HBG_SYM_NONE;
    const bool on_planes = (!(msym & HBG_SYM_YZ) || b.position[0] == 0.0) &&
                           (!(msym & HBG_SYM_XZ) || b.position[1] == 0.0);
    const bool sectors = form == 1 || (form == -1 && msym != HBG_SYM_NONE && on_planes &&
                                       (b.interior != "mesh" || (lid && lid->symmetry == mesh->symmetry)));
    bv = sectors ? mesh->vertices : expand(*mesh);
    sym = sectors ? msym : HBG_SYM_NONE;
    size_t P = bv.size() / 12;
    bk.assign(P, HBG_WET);
    if (b.interior == "detect")
        for (size_t p = 0; p < P; p++) {
            bool z0 = true;
            for (int i = 0; i < 4; i++) z0 = z0 && bv[12 * p + 3 * i + 2] == 0.0;
            if (z0) bk[p] = HBG_INTERIOR;
        }
    if (b.interior == "projected") {
        std::string why;
        std::vector<double> lv = projected_lid(bv, -b.position[2], why);
        if (!why.empty()) return refuse(HB_ERR_VALUE, "body '" + b.name + "': interior surface 'projected': " + why);
        bv.insert(bv.end(), lv.begin(), lv.end());
        bk.resize(bv.size() / 12, HBG_INTERIOR);
    }
    if (b.interior == "graded" || b.interior == "waterline") {
        // generated on the stored panels and reflected like them (interior.rs:521-575)
        std::string why;
        const bool isx = (msym & HBG_SYM_YZ) != 0, isy = (msym & HBG_SYM_XZ) != 0;
        std::vector<double> lv = b.interior == "graded" ? graded::lid(mesh->vertices, isx, isy, -b.position[2], why)
                                                        : graded::waterline_lid(mesh->vertices, isx, isy, -b.position[2], why);
        if (!why.empty())
            return refuse(HB_ERR_VALUE, "body '" + b.name + "': interior surface '" + b.interior + "': " + why);
        if (!sectors) lv = reflect(lv, mesh->symmetry);
        bv.insert(bv.end(), lv.begin(), lv.end());
        bk.resize(bv.size() / 12, HBG_INTERIOR);
    }
    if (b.interior == "mesh") {
        if (!lid) return refuse(HB_ERR_VALUE, "interior_surface_mesh names no mesh");
        std::vector<double> lv = sectors ? lid->vertices : expand(*lid);
        bv.insert(bv.end(), lv.begin(), lv.end());
        bk.resize(bv.size() / 12, HBG_INTERIOR);
    }
    return HB_OK;
}

}  // namespace hbg

using namespace hbg;

extern "C" HbStatus hb_model_new(HbModel** out) {
    return guard([&]() -> HbStatus {
        if (!out) return refuse(HB_ERR_ARGUMENT, "null out-pointer");
        *out = new HbModel();
        return HB_OK;
    });
}

extern "C" HbStatus hb_model_free(HbModel* model) {
    if (!model) return HB_OK;
    if (model->solving) return refuse(HB_ERR_STATE, "the model is solving");
    delete model;
    return HB_OK;
}

extern "C" HbStatus hb_model_cancel(HbModel* model) {
    if (!model) return refuse(HB_ERR_ARGUMENT, "null model");
    model->cancel = 1;
    return HB_OK;
}

extern "C" HbStatus hb_object(HbModel* model, const char* path, uint64_t* object) {
    return guard([&]() -> HbStatus {
        if (!model || !path || !object) return refuse(HB_ERR_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> g(model->lock);
        std::string p(path);
        if (p.empty()) return *object = OBJ_MODEL, HB_OK;
        if (p == "environment") return *object = OBJ_ENV, HB_OK;
        if (p == "options" || p == "first_order") return *object = OBJ_OPTIONS, HB_OK;
        for (size_t i = 0; i < model->meshes.size(); i++)
            if (p == "meshes/" + model->meshes[i].name) return *object = OBJ_MESH0 + i, HB_OK;
        for (size_t i = 0; i < model->bodies.size(); i++)
            if (p == "bodies/" + model->bodies[i].name) return *object = OBJ_BODY0 + i, HB_OK;
        return refuse(HB_ERR_VALUE, "no object at the path \"" + p + "\"");
    });
}

extern "C" HbStatus hb_add(HbModel* model, uint64_t parent, const char* list, const char* type_name,
                           const char* name, int64_t index, uint64_t* out) {
    return guard([&]() -> HbStatus {
        if (!model || !list || !out) return refuse(HB_ERR_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> g(model->lock);
        if (parent != OBJ_MODEL) return refuse(HB_ERR_UNSUPPORTED, "only the lists of the model are on this route");
        if (index != -1) return refuse(HB_ERR_UNSUPPORTED, "objects are added at the end of their list (index -1)");
        std::string l(list), t(type_name ? type_name : ""), n(name ? name : "");
        if (n.empty()) return refuse(HB_ERR_VALUE, "a mesh or body needs a name");
        if (l == "meshes" && (t.empty() || t == "Mesh")) {
            for (auto& m : model->meshes)
                if (m.name == n) return refuse(HB_ERR_VALUE, "a mesh of that name exists");
            model->meshes.push_back(MeshObj{n});
            *out = OBJ_MESH0 + model->meshes.size() - 1;
            return HB_OK;
        }
        if (l == "bodies" && (t.empty() || t == "Body")) {
            for (auto& b : model->bodies)
                if (b.name == n) return refuse(HB_ERR_VALUE, "a body of that name exists");
            model->bodies.push_back(BodyObj{n});
            *out = OBJ_BODY0 + model->bodies.size() - 1;
            return HB_OK;
        }
        return refuse(HB_ERR_UNSUPPORTED, "the list \"" + l + "\" is not on this route");
    });
}

// hydrobem.h:879-886 hb_model_load_mesh for a low-order GDF file: a new mesh of the model with its panels
// and the symmetry planes of its ISX / ISY flags (x = 0: yz, y = 0: xz); ULEN and GRAV stay in the file
// (the environment keeps its own gravity).  Higher-order files and the SPL / discretization options of the
// reference are not on this route.
extern "C" HbStatus hb_model_load_mesh(HbModel* model, const char* name, const char* path, const HbMeshOptions* options,
                                       uint64_t* out) {
    return guard([&]() -> HbStatus {
        if (!model || !name || !path || !out) return refuse(HB_ERR_ARGUMENT, "null argument");
        if (options && (options->higher_order || options->spl_path || options->discretization ||
                        options->panel_size > 0.0))
            return refuse(HB_ERR_UNSUPPORTED, "higher-order meshes are not on this route");
        std::string label;
        double ulen = 0.0, grav = 0.0;
        int isx = 0, isy = 0;
        std::vector<double> v;
        read_gdf(path, options && options->zero_trailer, label, ulen, grav, isx, isy, v);
        for (double x : v)
            if (!std::isfinite(x)) return refuse(HB_ERR_VALUE, std::string(path) + ": non-finite vertex coordinate");
        std::lock_guard<std::mutex> g(model->lock);
        const std::string n(name);
        if (n.empty()) return refuse(HB_ERR_VALUE, "a mesh needs a name");
        for (auto& m : model->meshes)
            if (m.name == n) return refuse(HB_ERR_VALUE, "a mesh of that name exists");
        MeshObj m{n};
        m.vertices.swap(v);
        m.symmetry = isx && isy ? "xz_and_yz" : isx ? "yz" : isy ? "xz" : "none";
        model->meshes.push_back(std::move(m));
        *out = OBJ_MESH0 + model->meshes.size() - 1;
        return HB_OK;
    });
}

extern "C" HbStatus hb_set_reals(HbModel* model, uint64_t object, const char* item, const double* data,
                                 const size_t* shape, size_t ndim) {
    return guard([&]() -> HbStatus {
        if (!model || !item || (!data && ndim > 0) || (!shape && ndim > 0)) return refuse(HB_ERR_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> g(model->lock);
        std::string it(item);
        size_t count = 0;
        std::vector<double> v = reals(data, shape, ndim, count);
        for (double x : v)
            if (std::isnan(x)) return refuse(HB_ERR_VALUE, "NaN in " + it);
        if (object == OBJ_ENV) {
            if (ndim != 1) return refuse(HB_ERR_VALUE, it + " is a 1-D array");
            if (it == "omegas" || it == "periods") {
                for (double x : v)
                    if (x < 0.0) return refuse(HB_ERR_VALUE, it + " must be >= 0");
                (it == "omegas" ? model->omegas : model->periods) = v;
                return HB_OK;
            }
            if (it == "headings") {
                for (double x : v)
                    if (!std::isfinite(x)) return refuse(HB_ERR_VALUE, "headings must be finite");
                model->headings = v;
                return HB_OK;
            }
        }
        if (is_body(model, object) && (it == "position" || it == "rotation_center" || it == "center_of_gravity" ||
                                       it == "inertia_origin")) {
            if (ndim != 1 || shape[0] != 3) return refuse(HB_ERR_VALUE, it + " has 3 values");
            for (double x : v)
                if (!std::isfinite(x)) return refuse(HB_ERR_VALUE, it + " must be finite");
            BodyObj& b = model->bodies[object - OBJ_BODY0];
            double* dst = it == "position" ? b.position : it == "rotation_center" ? b.rotation_center
                          : it == "center_of_gravity"                          ? b.cg
                                                                               : b.inertia_point;
            for (int d = 0; d < 3; d++) dst[d] = v[d];
            if (it == "center_of_gravity") b.has_cg = true;
            if (it == "inertia_origin") b.inertia_origin = "point";
            return HB_OK;
        }
        if (object == OBJ_OPTIONS && it == "field_points") {
            if (ndim != 2 || shape[1] != 3) return refuse(HB_ERR_VALUE, "field_points have the shape (N, 3)");
            for (size_t i = 0; i < v.size(); i++)
                if (!std::isfinite(v[i]) || (i % 3 == 2 && v[i] > 0.0))
                    return refuse(HB_ERR_VALUE, "field_points are finite, at z <= 0");
            model->field_points = v;
            return HB_OK;
        }
        if (is_body(model, object) && it == "radii_of_gyration") {
            const bool diag = ndim == 1 && shape[0] == 3, full = ndim == 2 && shape[0] == 3 && shape[1] == 3;
            if (!diag && !full) return refuse(HB_ERR_VALUE, "radii_of_gyration has 3 values or 3 x 3");
            for (double x : v)
                if (!std::isfinite(x)) return refuse(HB_ERR_VALUE, "radii_of_gyration must be finite");
            if (full)
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < i; j++)
                        if (v[3 * i + j] != v[3 * j + i]) return refuse(HB_ERR_VALUE, "radii_of_gyration is symmetric");
            BodyObj& b = model->bodies[object - OBJ_BODY0];
            for (int k = 0; k < 9; k++) b.gyration[k] = full ? v[k] : (k % 4 == 0 ? v[k / 4] : 0.0);
            return HB_OK;
        }
        if (is_mesh(model, object) && it == "vertices") {
            if (ndim != 3 || shape[1] != 4 || shape[2] != 3) return refuse(HB_ERR_VALUE, "vertices have the shape (P, 4, 3)");
            for (double x : v)
                if (!std::isfinite(x)) return refuse(HB_ERR_VALUE, "non-finite vertex coordinate");
            model->meshes[object - OBJ_MESH0].vertices = v;
            return HB_OK;
        }
        return refuse(HB_ERR_UNSUPPORTED, "the item \"" + it + "\" of this object is not on this route");
    });
}

extern "C" HbStatus hb_set_real(HbModel* model, uint64_t object, const char* item, double value) {
    return guard([&]() -> HbStatus {
        if (!model || !item) return refuse(HB_ERR_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> g(model->lock);
        std::string it(item);
        if (std::isnan(value)) return refuse(HB_ERR_VALUE, "NaN");
        if (is_body(model, object) && it == "yaw")
            return value == 0.0 ? HB_OK : refuse(HB_ERR_UNSUPPORTED, "a body rotated about z (yaw != 0) is not on this route");
        if (is_body(model, object)) {
            BodyObj& b = model->bodies[object - OBJ_BODY0];
            if (it == "mass") {
                if (!(value >= 0.0) || !std::isfinite(value)) return refuse(HB_ERR_VALUE, "mass >= 0 and finite");
                b.mass = value;
                b.mass_kind = 1;
                return HB_OK;
            }
            static const char* comp[6] = {"Ixx", "Ixy", "Ixz", "Iyy", "Iyz", "Izz"};
            for (int k = 0; k < 6; k++)
                if (it == comp[k]) {
                    if (!std::isfinite(value)) return refuse(HB_ERR_VALUE, it + " must be finite");
                    b.I[k] = value;
                    return HB_OK;
                }
        }
        if (object == OBJ_ENV) {
            if (it == "depth") {
                if (!(value > 0.0)) return refuse(HB_ERR_VALUE, "depth > 0 (inf for infinite depth)");
                model->depth = value;
                return HB_OK;
            }
            if (it == "gravity" || it == "density") {
                if (!(value > 0.0) || !std::isfinite(value)) return refuse(HB_ERR_VALUE, it + " must be positive");
                (it == "gravity" ? model->gravity : model->density) = value;
                return HB_OK;
            }
        }
        if (object == OBJ_OPTIONS && it == "log_tolerance") {
            if (!(value >= 0.0)) return refuse(HB_ERR_VALUE, "log_tolerance >= 0");
            model->log_tolerance = value;
            return HB_OK;
        }
        return refuse(HB_ERR_UNSUPPORTED, "the item \"" + it + "\" of this object is not on this route");
    });
}

extern "C" HbStatus hb_set_bool(HbModel* model, uint64_t object, const char* item, int32_t value) {
    return guard([&]() -> HbStatus {
        if (!model || !item) return refuse(HB_ERR_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> g(model->lock);
        std::string it(item);
        if (object == OBJ_OPTIONS && it == "logarithmic_integration") {
            model->logarithmic = value != 0;
            return HB_OK;
        }
        if (object == OBJ_OPTIONS && it == "motion") {
            model->motion = value != 0;
            return HB_OK;
        }
        if (object == OBJ_OPTIONS && it == "field_pressure") {
            model->field_pressure = value != 0;
            return HB_OK;
        }
        if (object == OBJ_OPTIONS && it == "drift_momentum_conservation") {
            model->drift_momentum = value != 0;
            return HB_OK;
        }
        if (object == OBJ_OPTIONS && it == "drift_bidirectional") {
            model->drift_bidirectional = value != 0;
            return HB_OK;
        }
        return refuse(HB_ERR_UNSUPPORTED, "the item \"" + it + "\" of this object is not on this route");
    });
}

extern "C" HbStatus hb_set_int(HbModel* model, uint64_t object, const char* item, int64_t value) {
    return guard([&]() -> HbStatus {
        if (!model || !item) return refuse(HB_ERR_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> g(model->lock);
        std::string it(item);
        if (object == OBJ_OPTIONS && it == "gpu_device") {
            if (value < 0) return refuse(HB_ERR_VALUE, "gpu_device >= 0");
            model->device = value;
            return HB_OK;
        }
        if (object == OBJ_OPTIONS && it == "drift_momentum_conservation_angles") {  // document_schema.rs:249
            if (value < 1 || value > 65536) return refuse(HB_ERR_VALUE, "drift_momentum_conservation_angles 1..65536 or auto");
            model->kochin_angles = value;
            return HB_OK;
        }
        return refuse(HB_ERR_UNSUPPORTED, "the item \"" + it + "\" of this object is not on this route");
    });
}

extern "C" HbStatus hb_set_ints(HbModel* model, uint64_t object, const char* item, const int64_t*, const size_t*,
                                size_t) {
    if (!model || !item) return refuse(HB_ERR_ARGUMENT, "null argument");
    return refuse(HB_ERR_UNSUPPORTED, std::string("the item \"") + item + "\" of this object is not on this route");
}

extern "C" HbStatus hb_set_text(HbModel* model, uint64_t object, const char* item, const char* value) {
    return guard([&]() -> HbStatus {
        if (!model || !item || !value) return refuse(HB_ERR_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> g(model->lock);
        std::string it(item), v(value);
        if (object == OBJ_ENV && it == "frequency_input") {
            if (v != "omegas" && v != "periods") return refuse(HB_ERR_VALUE, "frequency_input is omegas or periods");
            model->frequency_input = v;
            return HB_OK;
        }
        if (object == OBJ_OPTIONS && it == "gpu_statics_rule") {
            if (v != "accurate" && v != "production")
                return refuse(HB_ERR_VALUE, "gpu_statics_rule is accurate or production");
            model->statics_rule = v;
            return HB_OK;
        }
        if (object == OBJ_OPTIONS && it == "gpu_precision") {
            if (v != "fp64" && v != "mixed") return refuse(HB_ERR_VALUE, "gpu_precision is fp64 or mixed");
            model->precision = v;
            return HB_OK;
        }
        if (object == OBJ_OPTIONS && it == "drift_momentum_conservation_angles") {
            if (v != "auto") return refuse(HB_ERR_VALUE, "drift_momentum_conservation_angles 1..65536 or auto");
            model->kochin_angles = 0;
            return HB_OK;
        }
        if (is_mesh(model, object)) {
            MeshObj& m = model->meshes[object - OBJ_MESH0];
            if (it == "kind") return v == "panels" ? HB_OK : refuse(HB_ERR_UNSUPPORTED, "only panels meshes are on this route");
            if (it == "symmetry") {
                if (v != "none" && v != "yz" && v != "xz" && v != "xz_and_yz")
                    return refuse(HB_ERR_VALUE, "symmetry is none, yz, xz or xz_and_yz");
                m.symmetry = v;
                return HB_OK;
            }
        }
        if (is_body(model, object)) {
            BodyObj& b = model->bodies[object - OBJ_BODY0];
            if (it == "mesh") return b.mesh = v, HB_OK;
            if (it == "interior_surface") {
                if (v != "none" && v != "detect" && v != "mesh" && v != "projected" && v != "graded" && v != "waterline")
                    return refuse(HB_ERR_UNSUPPORTED,
                                  "interior_surface none, detect, projected, graded, waterline or mesh on this route");
                return b.interior = v, HB_OK;
            }
            if (it == "interior_surface_mesh") return b.interior_mesh = v, HB_OK;
            if (it == "mass") {
                if (v != "displaced") return refuse(HB_ERR_VALUE, "mass is a number or \"displaced\"");
                b.mass_kind = 2;
                return HB_OK;
            }
            if (it == "inertia_input") {
                if (v != "components" && v != "radii_of_gyration")
                    return refuse(HB_ERR_VALUE, "inertia_input is components or radii_of_gyration");
                return b.inertia_input = v, HB_OK;
            }
            if (it == "inertia_origin") {
                if (v != "center_of_gravity" && v != "rotation_center")
                    return refuse(HB_ERR_VALUE, "inertia_origin is center_of_gravity, rotation_center or a point");
                return b.inertia_origin = v, HB_OK;
            }
        }
        return refuse(HB_ERR_UNSUPPORTED, "the item \"" + it + "\" of this object is not on this route");
    });
}

extern "C" HbStatus hb_model_solve(HbModel* model, HbProgressFn progress, void* user, HbResults** out) {
    return guard([&]() -> HbStatus {
        if (!model) return refuse(HB_ERR_ARGUMENT, "null model");
        if (model->solving.exchange(true)) return refuse(HB_ERR_STATE, "the model is solving");
        struct Done {
            HbModel* m;
            ~Done() { m->solving = false; }
        } done{model};
        std::vector<double> verts, omegas, heads, centers;
        std::vector<int32_t> kinds, panel_body;
        int32_t symmetry = HBG_SYM_NONE;
        // mass properties in the global frame (all bodies or none: the weight terms and the motions)
        std::vector<double> rmass, rcg, rinertia, rorigin;
        std::vector<int32_t> rkind;
        bool all_rigid = true;
        HbgOptions opt;
        hbg_default_options(&opt);
        {
            std::lock_guard<std::mutex> g(model->lock);
            if (model->bodies.empty()) return refuse(HB_ERR_VALUE, "the model has no body");
            for (size_t bi = 0; bi < model->bodies.size(); bi++) {
                const BodyObj& b = model->bodies[bi];
                std::vector<double> bv;
                std::vector<int32_t> bk;
                int32_t bsym = HBG_SYM_NONE;
                if (HbStatus st = body_panels(model, b, model->bodies.size() == 1 ? -1 : 0, bv, bk, bsym)) return st;
                if (bsym != HBG_SYM_NONE) symmetry = bsym;
                for (size_t q = 0; q < bv.size(); q++) bv[q] += b.position[q % 3];  // body to global
                verts.insert(verts.end(), bv.begin(), bv.end());
                kinds.insert(kinds.end(), bk.begin(), bk.end());
                panel_body.insert(panel_body.end(), bk.size(), (int32_t)bi);
                for (int d = 0; d < 3; d++) centers.push_back(b.position[d] + b.rotation_center[d]);
                all_rigid = all_rigid && b.has_cg && b.mass_kind != 0;
                rmass.push_back(b.mass_kind == 2 ? NAN : b.mass);
                for (int d = 0; d < 3; d++) rcg.push_back(b.position[d] + b.cg[d]);
                const bool comps = b.inertia_input == "components";
                rkind.push_back(comps ? HBG_INERTIA_COMPONENTS : HBG_INERTIA_GYRATION);
                const double J[9] = {b.I[0], b.I[1], b.I[2], b.I[1], b.I[3], b.I[4], b.I[2], b.I[4], b.I[5]};
                for (int k = 0; k < 9; k++) rinertia.push_back(comps ? J[k] : b.gyration[k]);
                const double* o = b.inertia_origin == "center_of_gravity" ? b.cg
                                  : b.inertia_origin == "rotation_center" ? b.rotation_center
                                                                          : b.inertia_point;
                for (int d = 0; d < 3; d++) rorigin.push_back(b.position[d] + o[d]);
            }
            if (model->motion && !all_rigid)
                return refuse(HB_ERR_VALUE, "the motions need the mass and center_of_gravity of every body");
            const std::vector<double>& f = model->frequency_input == "omegas" ? model->omegas : model->periods;
            for (double x : f) {
                double w = model->frequency_input == "omegas" ? x : (x > 0.0 ? 2.0 * PI / x : INFINITY);
                if (!(w > 0.0) || !std::isfinite(w))
                    return refuse(HB_ERR_UNSUPPORTED, "the zero- and infinite-frequency limits are not on this route");
                omegas.push_back(w);
            }
            heads = model->headings;
            opt.precision = model->precision == "mixed" ? HBG_MIXED : HBG_FP64;
            opt.statics_rule = model->statics_rule == "production" ? HBG_STATICS_PRODUCTION : HBG_STATICS_ACCURATE;
            opt.logarithmic = model->logarithmic;
            opt.log_tolerance = model->log_tolerance;
            opt.gravity = model->gravity;
            opt.density = model->density;
            opt.depth = model->depth;
            opt.device = (int32_t)model->device;
        }
        opt.cancel = reinterpret_cast<const volatile int32_t*>(&model->cancel);
        if (model->cancel.exchange(0) != 0) return refuse(HB_ERR_CANCELLED, "the solve was cancelled");
        const size_t F = omegas.size(), H = heads.size(), NB = centers.size() / 3, D = 6 * NB;
        std::vector<double> A(F * D * D), B(F * D * D), X(F * H * D * 2), FK(F * H * D * 2), SC(F * H * D * 2),
            MO(F * H * D * 2), HK(F * H * D * 2), HS(NB * HBG_HS);
        std::vector<double> fpts;
        {
            std::lock_guard<std::mutex> g(model->lock);
            if (model->field_pressure) fpts = model->field_points;
        }
        const size_t NP = fpts.size() / 3;
        std::vector<double> FR(F * NP * D * 2), FI(F * NP * H * 2), FS(F * NP * H * 2), FDF(F * NP * H * 2);
        const bool want_motion = model->motion && H > 0;
        // the Kochin angles of the momentum drift: given, or the reference's automatic count
        // (response.rs:109-176): 8 ceil((2 ceil(k R) + 96) / 8), k the largest wave number, R the largest
        // horizontal distance of a vertex from the origin
        size_t T = 0;
        if (model->drift_momentum && H > 0) {
            if (model->kochin_angles > 0) {
                T = (size_t)model->kochin_angles;
            } else {
                double kmax = 0.0, R = 0.0;
                const bool fin = std::isfinite(opt.depth) && opt.depth > 0.0;
                for (double w : omegas) {
                    const double K = w * w / opt.gravity;
                    kmax = std::max(kmax, fin ? dispersion_x0(K * opt.depth) / opt.depth : K);
                }
                for (size_t q = 0; q + 2 < verts.size(); q += 3) R = std::max(R, std::hypot(verts[q], verts[q + 1]));
                const size_t n = 2 * (size_t)std::ceil(kmax * R) + 96;
                T = 8 * ((n + 7) / 8);
            }
        }
        std::vector<double> KR(F * T * D * 2), KRT(F * T * D * 2), KD(F * T * H * 2), KDT(F * T * H * 2),
            DR(T ? F * H * H * 3 * 2 : 0);
        HbgRigid rig{rmass.data(), rcg.data(), rkind.data(), rinertia.data(), rorigin.data(), nullptr, nullptr};
        HbgProblem pr{};
        pr.rigid = all_rigid ? &rig : nullptr;
        pr.body.n_panels = (int64_t)(verts.size() / 12);
        pr.body.vertices = verts.data();
        pr.body.kinds = kinds.data();
        pr.body.panel_body = panel_body.data();
        pr.body.n_bodies = (int32_t)NB;
        pr.body.rotation_centers = centers.data();
        pr.body.symmetry = symmetry;
        pr.omegas = omegas.data();
        pr.n_omega = (int64_t)F;
        pr.headings_deg = heads.data();
        pr.n_heading = (int64_t)H;
        pr.out = HbgOutputs{A.data(), B.data(), X.data(), FK.data(), SC.data(), want_motion ? MO.data() : nullptr,
                            HS.data(), NP ? FR.data() : nullptr, NP ? FI.data() : nullptr, NP ? FS.data() : nullptr,
                            NP ? FDF.data() : nullptr, HK.data(), T ? KR.data() : nullptr, T ? KRT.data() : nullptr,
                            T ? KD.data() : nullptr, T ? KDT.data() : nullptr, T ? DR.data() : nullptr};
        pr.kochin_angles = (int32_t)T;
        pr.field_points = NP ? fpts.data() : nullptr;
        pr.n_field_points = (int64_t)NP;
        if (progress) {
            HbProgress pg{};
            pg.stage = 0;
            pg.frequency = -2;
            pg.frequencies_total = F;
            if (progress(&pg, user) == 0) return refuse(HB_ERR_CANCELLED, "the solve was cancelled");
        }
        HbStatus st = hbg_solve_batch(&pr, 1, &opt);
        if (st != HB_OK) return st;
        if (progress) {
            HbProgress pg{};
            pg.stage = 0;
            pg.frequency = -4;
            pg.frequencies_done = F;
            pg.frequencies_total = F;
            pg.seconds = g_profile[5] * 1e-3;
            progress(&pg, user);
        }
        auto r = std::make_unique<HbResults>();
        add_quantity(r.get(), "omegas", HB_F64, {F}, omegas.data(), F * 8);
        add_quantity(r.get(), "headings", HB_F64, {H}, heads.data(), H * 8);
        std::vector<float> a32(F * D * D), b32(F * D * D), x32(F * H * D * 2), fk32(F * H * D * 2), sc32(F * H * D * 2);
        for (size_t i = 0; i < F * D * D; i++) {
            a32[i] = (float)A[i];
            b32[i] = (float)B[i];
        }
        for (size_t i = 0; i < F * H * D * 2; i++) {
            x32[i] = (float)X[i];
            fk32[i] = (float)FK[i];
            sc32[i] = (float)SC[i];
        }
        // [F][D][D] and [F][H][D]: coordinate i and mode j of every body, bodies in the order added
        add_quantity(r.get(), "added_mass", HB_F32, {F, D, D}, a32.data(), a32.size() * 4);
        add_quantity(r.get(), "radiation_damping", HB_F32, {F, D, D}, b32.data(), b32.size() * 4);
        add_quantity(r.get(), "excitation_diffraction", HB_C64, {F, H, D}, x32.data(), x32.size() * 4);
        add_quantity(r.get(), "excitation_froude_krylov", HB_C64, {F, H, D}, fk32.data(), fk32.size() * 4);
        add_quantity(r.get(), "excitation_scattering", HB_C64, {F, H, D}, sc32.data(), sc32.size() * 4);
        add_quantity(r.get(), "added_mass_f64", HB_F64, {F, D, D}, A.data(), A.size() * 8);
        add_quantity(r.get(), "radiation_damping_f64", HB_F64, {F, D, D}, B.data(), B.size() * 8);
        add_quantity(r.get(), "excitation_diffraction_f64", HB_C128, {F, H, D}, X.data(), X.size() * 8);
        add_quantity(r.get(), "excitation_froude_krylov_f64", HB_C128, {F, H, D}, FK.data(), FK.size() * 8);
        add_quantity(r.get(), "excitation_scattering_f64", HB_C128, {F, H, D}, SC.data(), SC.size() * 8);
        if (H) {  // solve_driver.rs:370-384: [F][H][K], K = D radiation columns (rigid modes) on this route
            std::vector<float> hk32(HK.size());
            for (size_t i = 0; i < HK.size(); i++) hk32[i] = (float)HK[i];
            add_quantity(r.get(), "excitation_haskind", HB_C64, {F, H, D}, hk32.data(), hk32.size() * 4);
            add_quantity(r.get(), "excitation_haskind_f64", HB_C128, {F, H, D}, HK.data(), HK.size() * 8);
        }
        if (NP) {  // quantities.rs:58-62: the points, then the elevation or p / (rho g) per column and heading
            add_quantity(r.get(), "field_points", HB_F64, {NP, 3}, fpts.data(), fpts.size() * 8);
            const std::pair<const char*, std::vector<double>*> fq[4] = {{"field_points_pressure_radiation", &FR},
                                                                        {"field_points_pressure_incident", &FI},
                                                                        {"field_points_pressure_scattering", &FS},
                                                                        {"field_points_pressure_diffraction", &FDF}};
            for (int q = 0; q < 4; q++) {
                std::vector<double>& v = *fq[q].second;
                std::vector<float> v32(v.size());
                for (size_t i = 0; i < v.size(); i++) v32[i] = (float)v[i];
                const size_t cols = q == 0 ? D : H;
                add_quantity(r.get(), fq[q].first, HB_C64, {F, NP, cols}, v32.data(), v32.size() * 4);
                add_quantity(r.get(), std::string(fq[q].first) + "_f64", HB_C128, {F, NP, cols}, v.data(), v.size() * 8);
            }
        }
        if (T) {  // quantities.rs:79-88: the Kochin functions, the drift of the heading pairs
            std::vector<double> ang(T);
            for (size_t t = 0; t < T; t++) ang[t] = 2.0 * PI * (double)t / (double)T;
            add_quantity(r.get(), "kochin_angles", HB_F64, {T}, ang.data(), T * 8);
            const std::pair<const char*, std::vector<double>*> kq[4] = {{"kochin_radiation", &KR},
                                                                        {"kochin_radiation_derivative", &KRT},
                                                                        {"kochin_diffraction", &KD},
                                                                        {"kochin_diffraction_derivative", &KDT}};
            for (int q = 0; q < 4; q++) {
                std::vector<double>& v = *kq[q].second;
                std::vector<float> v32(v.size());
                for (size_t i = 0; i < v.size(); i++) v32[i] = (float)v[i];
                const size_t cols = q < 2 ? D : H;
                add_quantity(r.get(), kq[q].first, HB_C64, {F, T, cols}, v32.data(), v32.size() * 4);
                add_quantity(r.get(), std::string(kq[q].first) + "_f64", HB_C128, {F, T, cols}, v.data(), v.size() * 8);
            }
            // heading_pairs.rs:12-25: (h, h) unidirectional, every h_a <= h_b bidirectional
            std::vector<std::pair<size_t, size_t>> hp;
            for (size_t a = 0; a < H; a++)
                for (size_t b = a; b < (model->drift_bidirectional ? H : a + 1); b++) hp.emplace_back(a, b);
            std::vector<double> dv, pairs;
            for (size_t fq = 0; fq < F; fq++)
                for (auto& p : hp)
                    for (int c = 0; c < 3; c++) {
                        const double* z = &DR[((((fq * H + p.first) * H + p.second) * 3) + c) * 2];
                        dv.push_back(z[0]);
                        dv.push_back(z[1]);
                    }
            for (auto& p : hp) {
                pairs.push_back(heads[p.first]);
                pairs.push_back(heads[p.second]);
            }
            add_quantity(r.get(), "drift_momentum_conservation", HB_C128, {F, hp.size(), 3}, dv.data(), dv.size() * 8);
            add_quantity(r.get(), "drift_heading_pairs", HB_F64, {hp.size(), 2}, pairs.data(), pairs.size() * 8);
        }
        if (want_motion) {
            std::vector<float> m32(F * H * D * 2);
            for (size_t i = 0; i < m32.size(); i++) m32[i] = (float)MO[i];
            add_quantity(r.get(), "motion", HB_C64, {F, H, D}, m32.data(), m32.size() * 4);
            add_quantity(r.get(), "motion_f64", HB_C128, {F, H, D}, MO.data(), MO.size() * 8);
        }
        {
            // the hydrostatics of every body (quantities.rs:102-112), body coordinates as the reference's
            std::vector<double> vols(NB * 3), vol(NB), disp(NB), cb(NB * 3), aw(NB), wc(NB * 2), crg(NB * 36), cw(NB * 36),
                mass(NB), cgo(NB * 3), gm(NB * 2);
            const double rg = model->density * model->gravity;
            for (size_t b = 0; b < NB; b++) {
                const double* h = &HS[b * HBG_HS];
                const BodyObj& bo = model->bodies[b];
                for (int k = 0; k < 3; k++) vols[3 * b + k] = h[k];
                vol[b] = (h[0] + h[1] + h[2]) / 3.0;
                disp[b] = h[82];
                for (int k = 0; k < 3; k++) cb[3 * b + k] = h[3 + k] - bo.position[k];
                aw[b] = h[6];
                for (int k = 0; k < 2; k++) wc[2 * b + k] = h[7 + k] - bo.position[k];
                for (int k = 0; k < 36; k++) {
                    crg[36 * b + k] = h[9 + k];
                    cw[36 * b + k] = h[45 + k];
                }
                mass[b] = h[81];
                for (int k = 0; k < 3; k++) cgo[3 * b + k] = bo.has_cg ? bo.cg[k] : NAN;
                const bool weight = all_rigid && h[0] != 0.0;
                gm[2 * b] = weight ? h[45 + 3 * 6 + 3] / (rg * h[0]) : NAN;
                gm[2 * b + 1] = weight ? h[45 + 4 * 6 + 4] / (rg * h[0]) : NAN;
            }
            add_quantity(r.get(), "hydrostatics_volumes", HB_F64, {NB, 3}, vols.data(), vols.size() * 8);
            add_quantity(r.get(), "hydrostatics_volume", HB_F64, {NB}, vol.data(), vol.size() * 8);
            add_quantity(r.get(), "hydrostatics_displaced_mass", HB_F64, {NB}, disp.data(), disp.size() * 8);
            add_quantity(r.get(), "hydrostatics_center_of_buoyancy", HB_F64, {NB, 3}, cb.data(), cb.size() * 8);
            add_quantity(r.get(), "hydrostatics_waterplane_area", HB_F64, {NB}, aw.data(), aw.size() * 8);
            add_quantity(r.get(), "hydrostatics_waterplane_centroid", HB_F64, {NB, 2}, wc.data(), wc.size() * 8);
            add_quantity(r.get(), "hydrostatics_stiffness_rho_g", HB_F64, {NB, 6, 6}, crg.data(), crg.size() * 8);
            add_quantity(r.get(), "hydrostatics_stiffness", HB_F64, {NB, 6, 6}, cw.data(), cw.size() * 8);
            add_quantity(r.get(), "hydrostatics_mass", HB_F64, {NB}, mass.data(), mass.size() * 8);
            add_quantity(r.get(), "hydrostatics_center_of_gravity", HB_F64, {NB, 3}, cgo.data(), cgo.size() * 8);
            add_quantity(r.get(), "hydrostatics_metacentric_height", HB_F64, {NB, 2}, gm.data(), gm.size() * 8);
        }
        {
            std::lock_guard<std::mutex> g(model->lock);
            model->results = std::make_unique<HbResults>(*r);
        }
        if (out) *out = r.release();
        return HB_OK;
    });
}

// hydrobem.h:975-987 hb_model_panels: the panels as the solve uses them, host work only (a results
// object in place of the reference's table).  Roles
// "wetted" and "lid" (the interior free surface), comma separated, null for both; the stored form of
// each body's symmetric mesh unless include_reflections.  Quantities: vertices (HB_F64 [P][4][3],
// global), body (HB_I32 [P], zero-based in the order added), kind (HB_I32 [P], HBG_WET / HBG_INTERIOR).
extern "C" HbStatus hb_model_panels(HbModel* model, const char* role, int32_t include_reflections, HbResults** out) {
    return guard([&]() -> HbStatus {
        if (!model || !out) return refuse(HB_ERR_ARGUMENT, "null model or out-pointer");
        *out = nullptr;
        bool want[2] = {role == nullptr, role == nullptr};
        if (role) {
            std::string r(role);
            size_t a = 0;
            while (a <= r.size()) {
                size_t e = r.find(',', a);
                if (e == std::string::npos) e = r.size();
                const std::string w = r.substr(a, e - a);
                if (w == "wetted") want[HBG_WET] = true;
                else if (w == "lid") want[HBG_INTERIOR] = true;
                else return refuse(HB_ERR_UNSUPPORTED, "panel role '" + w + "' is not on this route (wetted, lid)");
                a = e + 1;
            }
        }
        std::vector<double> verts;
        std::vector<int32_t> body, kind;
        {
            std::lock_guard<std::mutex> g(model->lock);
            for (size_t bi = 0; bi < model->bodies.size(); bi++) {
                const BodyObj& b = model->bodies[bi];
                std::vector<double> bv;
                std::vector<int32_t> bk;
                int32_t sym = HBG_SYM_NONE;
                if (HbStatus st = body_panels(model, b, include_reflections ? 0 : 1, bv, bk, sym)) return st;
                for (size_t p = 0; p < bk.size(); p++) {
                    if (!want[bk[p]]) continue;
                    for (int q = 0; q < 12; q++) verts.push_back(bv[12 * p + q] + b.position[q % 3]);
                    body.push_back((int32_t)bi);
                    kind.push_back(bk[p]);
                }
            }
        }
        auto r = std::make_unique<HbResults>();
        const size_t P = kind.size();
        add_quantity(r.get(), "vertices", HB_F64, {P, 4, 3}, verts.data(), verts.size() * sizeof(double));
        add_quantity(r.get(), "body", HB_I32, {P}, body.data(), P * sizeof(int32_t));
        add_quantity(r.get(), "kind", HB_I32, {P}, kind.data(), P * sizeof(int32_t));
        *out = r.release();
        return HB_OK;
    });
}

extern "C" void hb_results_free(HbResults* results) { delete results; }

extern "C" HbStatus hb_results_has(HbResults* results, const char* name, int32_t* has) {
    if (!results || !name || !has) return refuse(HB_ERR_ARGUMENT, "null argument");
    *has = 0;
    for (auto& q : results->q)
        if (q.name == name) *has = 1;
    return HB_OK;
}

extern "C" HbStatus hb_results_quantity(HbResults* results, const char* name, HbColumn* column) {
    if (!results || !name || !column) return refuse(HB_ERR_ARGUMENT, "null argument");
    for (auto& q : results->q)
        if (q.name == name) {
            size_t count = 1;
            for (size_t d : q.shape) count *= d;
            *column = HbColumn{q.name.c_str(), q.dtype, q.shape.size(), q.shape.data(), count, q.data.data()};
            return HB_OK;
        }
    return refuse(HB_ERR_VALUE, std::string("no quantity \"") + name + "\" in these results");
}
