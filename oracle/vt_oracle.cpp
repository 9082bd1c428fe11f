// vt_oracle.cpp -- CPU oracle: f64 restatement of voronota-ltr's tessellation hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the B200 kernels and the
// timed CPU baseline; the product library never links it.
//
// Every function names the reference function it restates (paths relative to the
// voronota-ltr project).  Arithmetic follows the reference's evaluation order:
//   * Rust `mul_add` -> std::fma; nothing else is contracted (build with
//     -ffp-contract=off, no fast-math);
//   * nalgebra 0.34.2 fixed-size Vector3 arithmetic (third-party, not vendored in the
//     reference): dot = (x*x' + y*y') + z*z', norm = sqrt(dot(v,v)), normalize = v / norm
//     (component division), cross = (ay*bz - az*by, az*bx - ax*bz, ax*by - ay*bx),
//     UnitQuaternion::from_axis_angle(u, t) = (cos(t/2), u*sin(t/2)) and
//     q * v = (t*w + q.v x t) + v with t = 2 (q.v x v).
// Bit-level parity with the Rust build is therefore unpinned at the nalgebra and libm
// boundary; result-level parity is pinned by the reference's golden values
// (tests/test_oracle_goldens.py).
//
// Parallelism mirrors the reference's Rayon sites: per-ball neighbour search
// (tessellation.rs:70-73) and per-pair contact construction (tessellation.rs:141-159,
// 211-236) run on a std::thread pool with dynamic chunks; every output element is computed independently, so the
// results do not depend on the thread count.

#include "vt_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <unordered_map>
#include <vector>

#include <atomic>
#include <functional>
#include <thread>

namespace {

bool g_faithful_grid_update = true;

constexpr double EPSILON = 1e-10;  // geometry.rs:17
constexpr double PI = 3.14159265358979323846;
constexpr double TAU = 6.28318530717958647692;
constexpr double FRAC_PI_3 = 1.04719755119659774615;
constexpr double HEXAGON_SCALE = 1.19;  // contact.rs:448
constexpr uint64_t NULL_ID = UINT64_MAX;

// ---- float_cmp (geometry.rs:22-54) ----
inline bool feq(double a, double b) { return std::fabs(a - b) <= EPSILON; }
inline bool flt(double a, double b) { return a + EPSILON < b; }
inline bool fgt(double a, double b) { return a - EPSILON > b; }
inline bool fle(double a, double b) { return a < b + EPSILON; }
inline bool fge(double a, double b) { return a + EPSILON > b; }

// Rust f64::max / min: the non-NaN operand wins.
inline double rmax(double a, double b) { return std::fmax(a, b); }
inline double rmin(double a, double b) { return std::fmin(a, b); }
inline double rclamp(double v, double lo, double hi) {
    if (std::isnan(v)) return v;
    return v < lo ? lo : (v > hi ? hi : v);
}

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double norm2(V3 a) { return dot(a, a); }
inline double norm(V3 a) { return std::sqrt(norm2(a)); }
inline V3 normalize(V3 a) { return a / norm(a); }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct Sphere {  // types.rs:33-64
    V3 c;
    double r;
};

// ---- geometry.rs ----
inline bool point_equals(V3 a, V3 b) { return feq(a.x, b.x) && feq(a.y, b.y) && feq(a.z, b.z); }
inline bool sphere_intersects_sphere(const Sphere& a, const Sphere& b) {  // :66-69
    double sum_r = a.r + b.r;
    return flt(norm2(b.c - a.c), sum_r * sum_r);
}
inline bool sphere_equals_sphere(const Sphere& a, const Sphere& b) {  // :73-75
    return feq(a.r, b.r) && point_equals(a.c, b.c);
}
inline bool sphere_contains_sphere(const Sphere& a, const Sphere& b) {  // :79-82
    double diff_r = a.r - b.r;
    return fge(a.r, b.r) && fle(norm2(b.c - a.c), diff_r * diff_r);
}
inline double signed_distance_to_plane_unit(V3 pp, V3 n, V3 x) { return dot(n, x - pp); }  // :96-102
inline double signed_distance_to_plane(V3 pp, V3 n, V3 x) {  // :86-92
    return signed_distance_to_plane_unit(pp, normalize(n), x);
}
inline int halfspace_of_point_unit(V3 pp, V3 n, V3 x) {  // :118-131
    double sd = signed_distance_to_plane_unit(pp, n, x);
    if (fgt(sd, 0.0)) return 1;
    if (flt(sd, 0.0)) return -1;
    return 0;
}
inline V3 intersection_of_plane_and_segment(V3 pp, V3 n, V3 a, V3 b) {  // :134-148
    double da = signed_distance_to_plane(pp, n, a);
    double db = signed_distance_to_plane(pp, n, b);
    if (std::fabs(da - db) < EPSILON) return a;
    double t = da / (da - db);
    return a + (b - a) * t;
}
inline double triangle_area(V3 a, V3 b, V3 c) { return norm(cross(b - a, c - a)) / 2.0; }  // :152-154
inline double min_angle(V3 o, V3 a, V3 b) {  // :157-161
    V3 v1 = normalize(a - o), v2 = normalize(b - o);
    return std::acos(rclamp(dot(v1, v2), -1.0, 1.0));
}
inline double directed_angle(V3 o, V3 a, V3 b, V3 c) {  // :165-176
    double angle = min_angle(o, a, b);
    V3 v1 = normalize(a - o), v2 = normalize(b - o);
    V3 n = cross(v1, v2);
    if (dot(c - o, n) >= 0.0) return angle;
    return TAU - angle;
}
inline V3 any_normal_of_vector(V3 a) {  // :179-193
    V3 b = a;
    if (!feq(b.x, 0.0) && (!feq(b.y, 0.0) || !feq(b.z, 0.0))) {
        b.x = -b.x;
        return normalize(cross(a, b));
    } else if (!feq(b.y, 0.0) && (!feq(b.x, 0.0) || !feq(b.z, 0.0))) {
        b.y = -b.y;
        return normalize(cross(a, b));
    } else if (!feq(b.x, 0.0)) {
        return {0.0, 1.0, 0.0};
    }
    return {1.0, 0.0, 0.0};
}
inline V3 rotate_point_around_axis(V3 axis, double angle, V3 p) {  // :196-203
    if (norm2(axis) <= 0.0) return p;
    V3 u = normalize(axis);  // Unit::new_normalize
    double half = angle / 2.0;
    double s = std::sin(half), c = std::cos(half);
    V3 qv = u * s;
    V3 t = cross(qv, p) * 2.0;
    V3 cr = cross(qv, t);
    return (t * c + cr) + p;
}
inline double distance_to_intersection_circle_center(const Sphere& a, const Sphere& b) {  // :208-215
    double cm = norm(b.c - a.c);
    if (cm < EPSILON) return 0.0;
    double cos_g = std::fma(b.r, -b.r, std::fma(a.r, a.r, cm * cm)) / (2.0 * a.r * cm);
    return a.r * cos_g;
}
inline V3 center_of_intersection_circle(const Sphere& a, const Sphere& b) {  // :218-226
    V3 cv = b.c - a.c;
    double cm = norm(cv);
    if (cm < EPSILON) return a.c;
    double cos_g = std::fma(b.r, -b.r, std::fma(a.r, a.r, cm * cm)) / (2.0 * a.r * cm);
    return a.c + cv * (a.r * cos_g / cm);
}
inline Sphere intersection_circle_of_two_spheres(const Sphere& a, const Sphere& b) {  // :229-239
    V3 cv = b.c - a.c;
    double cm = norm(cv);
    if (cm < EPSILON) return {a.c, 0.0};
    double cos_g = std::fma(b.r, -b.r, std::fma(a.r, a.r, cm * cm)) / (2.0 * a.r * cm);
    double sin_g = std::sqrt(rmax(1.0 - cos_g * cos_g, 0.0));
    V3 center = a.c + cv * (a.r * cos_g / cm);
    return {center, a.r * sin_g};
}
inline bool project_point_inside_line(V3 o, V3 a, V3 b, V3* out) {  // :243-255
    V3 v = normalize(b - a);
    double l = dot(v, o - a);
    if (l > 0.0 && l * l <= norm2(b - a)) {
        *out = a + v * l;
        return true;
    }
    return false;
}
inline bool intersect_segment_with_circle(const Sphere& circle, V3 p_in, V3 p_out, V3* out) {  // :258-280
    double dist = norm(p_in - p_out);
    if (dist <= 0.0) return false;
    V3 v = (p_in - p_out) / dist;
    V3 u = circle.c - p_out;
    V3 s = p_out + v * dot(v, u);
    double ll = std::fma(circle.r, circle.r, -norm2(circle.c - s));
    if (ll >= 0.0) {
        *out = s - v * std::sqrt(ll);
        return true;
    }
    return false;
}
inline double min_dihedral_angle(V3 o, V3 a, V3 b1, V3 b2) {  // :283-293
    V3 oa = normalize(a - o);
    V3 d1 = b1 - (o + oa * dot(oa, b1 - o));
    V3 d2 = b2 - (o + oa * dot(oa, b2 - o));
    return std::acos(rclamp(dot(normalize(d1), normalize(d2)), -1.0, 1.0));
}

// ---- types.rs ----
struct ValuedId {  // types.rs:148-184
    double value;
    uint64_t index;
};
inline bool valued_less(const ValuedId& a, const ValuedId& b) {
    // partial_cmp on value; Equal or unordered (NaN) falls back to the index.
    if (a.value < b.value) return true;
    if (a.value > b.value) return false;
    return a.index < b.index;
}

struct PBox {  // types.rs:292-376
    V3 a, b, c;
    Sphere shift(const Sphere& s, double wa, double wb, double wc) const {  // :323-347
        return {{std::fma(c.x, wc, std::fma(b.x, wb, std::fma(a.x, wa, s.c.x))),
                 std::fma(c.y, wc, std::fma(b.y, wb, std::fma(a.y, wa, s.c.y))),
                 std::fma(c.z, wc, std::fma(b.z, wb, std::fma(a.z, wa, s.c.z)))},
                s.r};
    }
};
// NEIGHBOR_SHIFTS (types.rs:351-361): lexicographic (sx, sy, sz) over {-1,0,1}^3 minus origin.
struct Shift {
    int x, y, z;
};
static std::vector<Shift> neighbor_shifts() {
    std::vector<Shift> s;
    for (int x = -1; x <= 1; ++x)
        for (int y = -1; y <= 1; ++y)
            for (int z = -1; z <= 1; ++z)
                if (x != 0 || y != 0 || z != 0) s.push_back({x, y, z});
    return s;
}
static std::vector<Sphere> populate_periodic_spheres(const PBox& pb, const std::vector<Sphere>& sp) {  // :364-375
    std::vector<Sphere> out;
    out.reserve(sp.size() * 27);
    out.insert(out.end(), sp.begin(), sp.end());
    for (const Shift& s : neighbor_shifts())
        for (const Sphere& x : sp) out.push_back(pb.shift(x, s.x, s.y, s.z));
    return out;
}

struct ContactSummary {  // ContactDescriptorSummary, types.rs:380-415
    double area = 0, arc_length = 0, solid_angle_a = 0, solid_angle_b = 0;
    double pyramid_volume_a = 0, pyramid_volume_b = 0, distance = 0;
    uint64_t id_a = 0, id_b = 0;
    bool central = false;
    void ensure_ids_ordered() {  // :408-414
        if (id_a > id_b) {
            std::swap(id_a, id_b);
            std::swap(solid_angle_a, solid_angle_b);
            std::swap(pyramid_volume_a, pyramid_volume_b);
        }
    }
};

enum class Stage { Init, ContactsAdded, SasComputed };
struct CellSummary {  // CellContactSummary, types.rs:431-454, 587-675
    uint64_t id = 0;
    double area = 0, arc_length = 0, sa_pos = 0, sa_neg = 0, pv_pos = 0, pv_neg = 0;
    double sas_area = 0, sas_inside_volume = 0;
    uint64_t count = 0;
    Stage stage = Stage::Init;
    void add(const ContactSummary& cds) {  // :589-609
        if (cds.area > 0.0 && (cds.id_a == id || cds.id_b == id)) {
            count += 1;
            area += cds.area;
            arc_length += cds.arc_length;
            double sa, pv;
            if (cds.id_a == id) {
                sa = cds.solid_angle_a;
                pv = cds.pyramid_volume_a;
            } else {
                sa = cds.solid_angle_b;
                pv = cds.pyramid_volume_b;
            }
            sa_pos += rmax(sa, 0.0);
            sa_neg -= rmin(sa, 0.0);
            pv_pos += rmax(pv, 0.0);
            pv_neg -= rmin(pv, 0.0);
            stage = Stage::ContactsAdded;
        }
    }
    void compute_sas(double r) {  // :623-663
        if (stage != Stage::ContactsAdded) return;
        sas_area = 0.0;
        sas_inside_volume = 0.0;
        double diff = std::fabs(sa_pos - sa_neg);
        if (arc_length > 0.0 && diff > 1e-10) {
            if (sa_pos > sa_neg) {
                double angle_diff = sa_pos - sa_neg;
                sas_area = std::fma(4.0, PI, -rmax(angle_diff, 0.0)) * r * r;
            } else {
                double angle_diff = sa_neg - sa_pos;
                sas_area = rmax(angle_diff, 0.0) * r * r;
            }
            sas_inside_volume = (sas_area * r / 3.0) + pv_pos - pv_neg;
            double full_sphere_vol = 4.0 / 3.0 * PI * r * r * r;
            if (sas_inside_volume > full_sphere_vol) {
                sas_area = 0.0;
                sas_inside_volume = pv_pos - pv_neg;
            }
        } else {
            sas_inside_volume = pv_pos - pv_neg;
        }
        stage = Stage::SasComputed;
    }
    void compute_sas_detached(uint64_t new_id, double r) {  // :666-675
        if (stage == Stage::Init) {
            id = new_id;
            sas_area = 4.0 * PI * r * r;
            sas_inside_volume = sas_area * r / 3.0;
            stage = Stage::SasComputed;
        }
    }
};

// ---- spheres_searcher.rs ----
inline int32_t sat_i32(double v) {  // Rust `as i32`: saturating, NaN -> 0
    if (std::isnan(v)) return 0;
    if (v >= 2147483647.0) return INT32_MAX;
    if (v <= -2147483648.0) return INT32_MIN;
    return (int32_t)v;
}
struct GridPoint {
    int32_t x = 0, y = 0, z = 0;
};
inline GridPoint grid_point(const Sphere& s, double box, GridPoint off = {}) {  // :21-36
    return {sat_i32(std::floor(s.c.x / box)) - off.x, sat_i32(std::floor(s.c.y / box)) - off.y,
            sat_i32(std::floor(s.c.z / box)) - off.z};
}
inline int64_t grid_index(GridPoint p, GridPoint size) {  // :39-51
    if (p.x >= 0 && p.y >= 0 && p.z >= 0 && p.x < size.x && p.y < size.y && p.z < size.z)
        return (int64_t)p.z * size.x * size.y + (int64_t)p.y * size.x + p.x;
    return -1;
}
struct GridParams {  // :56-102
    GridPoint offset, size{1, 1, 1};
    double box_size = 1.0;
    static GridParams make(const std::vector<Sphere>& sp) {
        GridParams g;
        if (sp.empty()) return g;
        for (const Sphere& s : sp) g.box_size = rmax(g.box_size, std::fma(s.r, 2.0, 0.25));
        const int pad = 1;
        for (size_t i = 0; i < sp.size(); ++i) {
            GridPoint gp = grid_point(sp[i], g.box_size);
            if (i == 0) {
                g.offset = gp;
                g.size = gp;
            } else {
                g.offset.x = std::min(g.offset.x, gp.x - pad);
                g.offset.y = std::min(g.offset.y, gp.y - pad);
                g.offset.z = std::min(g.offset.z, gp.z - pad);
                g.size.x = std::max(g.size.x, gp.x + pad);
                g.size.y = std::max(g.size.y, gp.y + pad);
                g.size.z = std::max(g.size.z, gp.z + pad);
            }
        }
        g.size.x = g.size.x - g.offset.x + 1;
        g.size.y = g.size.y - g.offset.y + 1;
        g.size.z = g.size.z - g.offset.z + 1;
        return g;
    }
};

struct CollisionResult {
    std::vector<ValuedId> ids;
    bool excluded = false;
};

class Searcher {  // SpheresSearcher, spheres_searcher.rs:115-327
   public:
    std::vector<Sphere> spheres;
    GridParams gp;
    std::vector<int32_t> map_of_boxes;
    std::vector<std::vector<uint64_t>> boxes;

    explicit Searcher(std::vector<Sphere> s) : spheres(std::move(s)) {
        gp = GridParams::make(spheres);
        init_boxes();
    }
    void init_boxes() {  // :224-248
        int64_t total = (int64_t)gp.size.x * gp.size.y * gp.size.z;
        map_of_boxes.assign((size_t)total, -1);
        boxes.clear();
        for (size_t i = 0; i < spheres.size(); ++i) add_to_grid(i);
    }
    void add_to_grid(uint64_t id) {  // :201-217
        int64_t idx = grid_index(grid_point(spheres[id], gp.box_size, gp.offset), gp.size);
        if (idx < 0) return;
        int32_t b = map_of_boxes[idx];
        if (b < 0) {
            map_of_boxes[idx] = (int32_t)boxes.size();
            boxes.push_back({id});
        } else {
            boxes[b].push_back(id);
        }
    }
    void remove_from_grid(uint64_t id) {  // :178-194
        int64_t idx = grid_index(grid_point(spheres[id], gp.box_size, gp.offset), gp.size);
        if (idx < 0) return;
        int32_t b = map_of_boxes[idx];
        if (b < 0) return;
        auto& v = boxes[b];
        auto it = std::find(v.begin(), v.end(), id);
        if (it != v.end()) {  // swap_remove
            *it = v.back();
            v.pop_back();
        }
    }
    void update(const std::vector<Sphere>& s, const std::vector<uint64_t>& changed) {  // :144-175
        std::vector<Sphere> old_spheres = spheres;
        for (uint64_t id : changed)
            if (id < spheres.size() && id < s.size()) spheres[id] = s[id];
        GridParams np = GridParams::make(spheres);
        if (std::fabs(np.box_size - gp.box_size) > 0.01 || np.size.x != gp.size.x ||
            np.size.y != gp.size.y || np.size.z != gp.size.z) {
            gp = np;
            init_boxes();
        } else {
            // The reference removes after the positions were already overwritten
            // (spheres_searcher.rs:146-149 then :164-173), so a sphere that moved to
            // another cell is looked up in its NEW cell and stays registered in the old
            // one.  `g_faithful_grid_update` keeps that behaviour; when it is off the
            // removal uses the old position (the documented incremental == full contract).
            std::vector<uint64_t> uniq = changed;
            if (!g_faithful_grid_update) {  // duplicates would register a sphere twice
                std::sort(uniq.begin(), uniq.end());
                uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
            }
            for (uint64_t id : uniq)
                if (id < spheres.size()) {
                    if (g_faithful_grid_update) {
                        remove_from_grid(id);
                    } else if (id < old_spheres.size()) {
                        std::swap(spheres[id], old_spheres[id]);
                        remove_from_grid(id);
                        std::swap(spheres[id], old_spheres[id]);
                    }
                }
            for (uint64_t id : uniq)
                if (id < spheres.size()) add_to_grid(id);
        }
    }
    CollisionResult find_colliding_ids(uint64_t central, bool discard_hidden) const {  // :253-326
        CollisionResult res;
        if (central >= spheres.size()) return res;
        const Sphere& cs = spheres[central];
        GridPoint g = grid_point(cs, gp.box_size, gp.offset);
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    int64_t idx = grid_index({g.x + dx, g.y + dy, g.z + dz}, gp.size);
                    if (idx < 0) continue;
                    int32_t b = map_of_boxes[idx];
                    if (b < 0) continue;
                    for (uint64_t id : boxes[b]) {
                        if (id == central) continue;
                        const Sphere& cand = spheres[id];
                        if (!sphere_intersects_sphere(cs, cand)) continue;
                        if (discard_hidden && sphere_contains_sphere(cand, cs) &&
                            (!sphere_equals_sphere(cand, cs) || central > id)) {
                            res.ids.clear();
                            res.excluded = true;
                            return res;
                        }
                        if (discard_hidden && sphere_contains_sphere(cs, cand)) continue;
                        res.ids.push_back({distance_to_intersection_circle_center(cs, cand), id});
                    }
                }
        std::sort(res.ids.begin(), res.ids.end(), valued_less);
        return res;
    }
};

// ---- contact.rs ----
struct ContourPoint {  // contact.rs:36-59
    V3 p;
    double angle = 0.0;
    uint64_t left_id, right_id;
    int state = 0;  // 0 Inside, 1 Outside, 2 ArcStart, 3 ArcContinue
    ContourPoint(V3 p_, uint64_t l, uint64_t r) : p(p_), left_id(l), right_id(r) {}
};
using Contour = std::vector<ContourPoint>;

static void init_contour(Contour& c, uint64_t a_id, const Sphere& base, V3 axis) {  // :455-469
    c.clear();
    V3 first = any_normal_of_vector(axis) * base.r * HEXAGON_SCALE;
    double step = FRAC_PI_3;
    c.emplace_back(base.c + first, a_id, a_id);
    double ang = step;
    while (ang < TAU) {
        V3 rot = rotate_point_around_axis(axis, ang, first);
        c.emplace_back(base.c + rot, a_id, a_id);
        ang += step;
    }
}
static bool test_contour_cuttable(V3 a_center, V3 closest, const Contour& c) {  // :472-481
    double thr = norm2(closest - a_center);
    for (const auto& cp : c)
        if (norm2(cp.p - a_center) >= thr) return true;
    return false;
}
static size_t mark_contour(Contour& c, V3 pc, V3 pn, uint64_t cid) {  // :506-521
    size_t count = 0;
    for (auto& cp : c)
        if (halfspace_of_point_unit(pc, pn, cp.p) >= 0) {
            cp.left_id = cid;
            cp.right_id = cid;
            ++count;
        }
    return count;
}
static void cut_contour(Contour& c, V3 pc, V3 pn, uint64_t cid) {  // :524-627
    if (c.size() < 3) return;
    auto is_out = [&](size_t i) { return c[i].left_id == cid && c[i].right_id == cid; };
    long s = -1, e = -1;
    for (size_t i = 0; i < c.size(); ++i)
        if (is_out(i)) {
            s = (long)i;
            break;
        }
    for (size_t i = c.size(); i-- > 0;)
        if (is_out(i)) {
            e = (long)i;
            break;
        }
    if (s < 0 || e < 0) return;
    size_t start = (size_t)s, end = (size_t)e;
    if (start == 0 && end == c.size() - 1) {
        end = 0;
        while (end + 1 < c.size() && is_out(end + 1)) ++end;
        start = c.size() - 1;
        while (start > 0 && is_out(start - 1)) --start;
    }
    if (start == end) {
        ContourPoint cp = c[start];
        c.insert(c.begin() + start, cp);
        end = start + 1;
    } else if (start < end) {
        if (start + 1 < end) c.erase(c.begin() + start + 1, c.begin() + end);
        end = start + 1;
    } else {
        if (start + 1 < c.size()) c.erase(c.begin() + start + 1, c.end());
        if (end > 0) c.erase(c.begin(), c.begin() + end);
        start = c.size() - 1;
        end = 0;
    }
    size_t n = c.size();
    size_t il = start > 0 ? start - 1 : n - 1;
    V3 lip = intersection_of_plane_and_segment(pc, pn, c[start].p, c[il].p);
    ContourPoint ns(lip, c[il].right_id, c[start].left_id);
    c[start] = ns;
    size_t ir = end + 1 < n ? end + 1 : 0;
    V3 rip = intersection_of_plane_and_segment(pc, pn, c[end].p, c[ir].p);
    ContourPoint ne(rip, c[end].right_id, c[ir].left_id);
    c[end] = ne;
    if (!fgt(norm2(c[end].p - c[start].p), 0.0)) {
        c[start].right_id = c[end].right_id;
        c.erase(c.begin() + end);
    }
}
static bool mark_and_cut_contour(Contour& c, V3 pc, V3 pn, uint64_t cid) {  // :484-503
    size_t out = mark_contour(c, pc, pn, cid);
    if (out == 0) return false;
    if (out >= c.size()) {
        c.clear();
        return true;
    }
    cut_contour(c, pc, pn, cid);
    return true;
}
static void restrict_contour_to_circle(Contour& c, const Sphere& ic, V3 axis, uint64_t a_id,
                                       double& sum_angles) {  // :631-769
    sum_angles = 0.0;
    size_t outsiders = 0;
    for (auto& cp : c) {
        if (norm2(cp.p - ic.c) <= ic.r * ic.r) {
            cp.state = 0;
        } else {
            cp.state = 1;
            ++outsiders;
        }
    }
    if (outsiders == 0) return;
    size_t insertions = 0;
    size_t i = 0;
    while (i < c.size()) {
        size_t ni = (i + 1) % c.size();
        int s1 = c[i].state, s2 = c[ni].state;
        if (s1 == 1 || s2 == 1) {
            if (s1 == 1 && s2 == 1) {
                V3 mp, ip1, ip2;
                if (project_point_inside_line(ic.c, c[i].p, c[ni].p, &mp) &&
                    norm2(mp - ic.c) <= ic.r * ic.r) {
                    bool ok1 = intersect_segment_with_circle(ic, mp, c[i].p, &ip1);
                    bool ok2 = intersect_segment_with_circle(ic, mp, c[ni].p, &ip2);
                    if (ok1 && ok2) {
                        uint64_t rid = c[i].right_id, lid = c[ni].left_id;
                        size_t pos = i + 1;
                        c.insert(c.begin() + pos, ContourPoint(ip1, a_id, rid));
                        c.insert(c.begin() + pos + 1, ContourPoint(ip2, lid, a_id));
                        insertions += 2;
                        i += 2;
                    }
                }
            } else if (s1 == 1) {
                V3 ip;
                if (intersect_segment_with_circle(ic, c[ni].p, c[i].p, &ip)) {
                    uint64_t rid = c[i].right_id;
                    c.insert(c.begin() + i + 1, ContourPoint(ip, a_id, rid));
                    insertions += 1;
                    i += 1;
                } else {
                    c[ni].left_id = a_id;
                    c[ni].right_id = c[i].right_id;
                }
            } else {
                V3 ip;
                if (intersect_segment_with_circle(ic, c[i].p, c[ni].p, &ip)) {
                    uint64_t lid = c[ni].left_id;
                    c.insert(c.begin() + i + 1, ContourPoint(ip, lid, a_id));
                    insertions += 1;
                    i += 1;
                } else {
                    c[i].left_id = c[ni].left_id;
                    c[i].right_id = a_id;
                }
            }
        }
        i += 1;
    }
    if (insertions == 0) {
        c.clear();
        return;
    }
    c.erase(std::remove_if(c.begin(), c.end(), [](const ContourPoint& cp) { return cp.state == 1; }),
            c.end());
    if (c.size() < 2) {
        c.clear();
        return;
    }
    for (size_t k = 0; k < c.size(); ++k) {
        size_t nk = (k + 1) % c.size();
        if (c[k].right_id == a_id && c[nk].left_id == a_id) {
            double ang = directed_angle(ic.c, c[k].p, c[nk].p, ic.c + axis);
            c[k].angle = ang;
            sum_angles += ang;
            c[k].state = 2;
        }
    }
    for (size_t k = 0; k < c.size(); ++k) {
        size_t pk = k > 0 ? k - 1 : c.size() - 1;
        if (c[pk].state == 2) c[k].state = 3;
    }
    if (fge(sum_angles, TAU) || (c.size() > 2 && feq(sum_angles, TAU))) {
        sum_angles = TAU;
        c.clear();
    }
}
static double calculate_contour_area(const Contour& c, const Sphere& ic, V3& bary) {  // :773-793
    V3 sum{0.0, 0.0, 0.0};
    for (const auto& cp : c) sum = sum + cp.p;
    bary = sum / (double)c.size();
    double area = 0.0;
    for (size_t i = 0; i < c.size(); ++i) {
        size_t ni = (i + 1) % c.size();
        area += triangle_area(bary, c[i].p, c[ni].p);
        if (c[i].angle > 0.0) area += ic.r * ic.r * (c[i].angle - std::sin(c[i].angle)) * 0.5;
    }
    return area;
}
static double calculate_solid_angle(const Sphere& a, const Sphere& b, const Sphere& ic,
                                    const Contour& c) {  // :797-848
    double turn = 0.0;
    if (c.empty()) {
        turn = TAU * norm(ic.c - a.c) / a.r;
    } else {
        size_t n = c.size();
        for (size_t i = 0; i < n; ++i) {
            size_t pi = i > 0 ? i - 1 : n - 1;
            size_t ni = (i + 1) % n;
            const ContourPoint& p0 = c[pi];
            const ContourPoint& p1 = c[i];
            const ContourPoint& p2 = c[ni];
            if (p0.angle > 0.0) {
                V3 d = cross(b.c - a.c, p1.p - ic.c);
                bool flip = (p0.angle < PI && dot(d, p0.p - p1.p) < 0.0) ||
                            (p0.angle > PI && dot(d, p0.p - p1.p) > 0.0);
                if (flip) d = -d;
                turn += PI - min_dihedral_angle(a.c, p1.p, p1.p + d, p2.p);
            } else if (p1.angle > 0.0) {
                V3 d = cross(b.c - a.c, p1.p - ic.c);
                bool flip = (p1.angle < PI && dot(d, p2.p - p1.p) < 0.0) ||
                            (p1.angle > PI && dot(d, p2.p - p1.p) > 0.0);
                if (flip) d = -d;
                turn += PI - min_dihedral_angle(a.c, p1.p, p0.p, p1.p + d);
                turn += p1.angle * (norm(ic.c - a.c) / a.r);
            } else {
                turn += PI - min_dihedral_angle(a.c, p1.p, p0.p, p2.p);
            }
        }
    }
    double sa = TAU - turn;
    V3 ic_to_a = ic.c - a.c, ic_to_b = ic.c - b.c;
    if (dot(ic_to_a, ic_to_b) > 0.0 && norm2(a.c - ic.c) < norm2(b.c - ic.c)) sa = -sa;
    return sa;
}
static bool contour_is_central(V3 center, const Contour& c, V3 bary) {  // :411-444
    const double FE = 1e-10;
    for (const auto& cp : c)
        if ((cp.angle - FE) > PI) return true;
    size_t n = c.size();
    for (size_t i = 0; i < n; ++i) {
        V3 pi = c[i].p, pj = c[(i + 1) % n].p;
        V3 edge = pj - pi;
        double len = norm(edge);
        if (len < FE) continue;
        V3 u = edge / len;
        V3 foot = pi + u * dot(u, bary - pi);
        V3 nb = bary - foot;
        if (dot(nb, center - pi) < 0.0) return false;
    }
    return true;
}

struct Clipped {  // ClippedContact, contact.rs:181-188
    Contour contour;
    Sphere ic;
    V3 axis;
    V3 bary;
    double sum_arc = 0, area = 0;
};

static bool clip_contact(const std::vector<Sphere>& sp, uint64_t a_id, uint64_t b_id,
                         const std::vector<ValuedId>& nbrs, Clipped& out) {  // :196-341
    if (a_id >= sp.size() || b_id >= sp.size()) return false;
    const Sphere& a = sp[a_id];
    const Sphere& b = sp[b_id];
    if (!sphere_intersects_sphere(a, b) || sphere_contains_sphere(a, b) || sphere_contains_sphere(b, a))
        return false;
    Sphere ic = intersection_circle_of_two_spheres(a, b);
    V3 axis = normalize(b.c - a.c);
    if (ic.r <= 0.0) return false;
    Contour contour;
    bool discarded = false, init = false;
    for (const ValuedId& nb : nbrs) {
        if (discarded) break;
        uint64_t nid = nb.index;
        if (nid == b_id) continue;
        const Sphere& c = sp[nid];
        if (!sphere_intersects_sphere(ic, c) || !sphere_intersects_sphere(b, c)) continue;
        if (sphere_contains_sphere(c, a) || sphere_contains_sphere(c, b)) {
            discarded = true;
            continue;
        }
        V3 pc = center_of_intersection_circle(a, c);
        V3 pn = normalize(c.c - a.c);
        double cos_val = dot(normalize(ic.c - a.c), normalize(pc - a.c));
        if (std::fabs(cos_val) >= 1.0) {
            if (halfspace_of_point_unit(pc, pn, ic.c) > 0) discarded = true;
            continue;
        }
        double l = std::fabs(signed_distance_to_plane_unit(pc, pn, ic.c));
        double xl = l / std::sqrt(std::fma(cos_val, -cos_val, 1.0));
        if (xl >= ic.r) {
            if (halfspace_of_point_unit(pc, pn, ic.c) >= 0) discarded = true;
            continue;
        }
        if (!init) {
            init_contour(contour, a_id, ic, axis);
            init = true;
        } else if (!test_contour_cuttable(a.c, pc, contour)) {
            continue;
        }
        mark_and_cut_contour(contour, pc, pn, nid);
        if (contour.empty()) discarded = true;
    }
    if (discarded) return false;
    V3 bary{0.0, 0.0, 0.0};
    double sum_arc = 0.0, area = 0.0;
    if (!init) {
        bary = ic.c;
        sum_arc = TAU;
        area = ic.r * ic.r * PI;
    } else if (!contour.empty()) {
        restrict_contour_to_circle(contour, ic, axis, a_id, sum_arc);
        if (!contour.empty()) area = calculate_contour_area(contour, ic, bary);
    }
    if (area <= 0.0) return false;
    out.contour = std::move(contour);
    out.ic = ic;
    out.axis = axis;
    out.bary = bary;
    out.sum_arc = sum_arc;
    out.area = area;
    return true;
}

// construct_contact_descriptor (:347-382) + to_summary (:97-114); contacts_only skips the
// solid angles and pyramid volumes exactly as construct_contact_area (:387-404).
static bool contact_summary(const std::vector<Sphere>& sp, uint64_t a_id, uint64_t b_id,
                            const std::vector<ValuedId>& nbrs, bool contacts_only,
                            ContactSummary& s) {
    Clipped cl;
    if (!clip_contact(sp, a_id, b_id, nbrs, cl)) return false;
    s = ContactSummary();
    s.area = cl.area;
    s.arc_length = cl.sum_arc * cl.ic.r;
    s.central = contour_is_central(cl.ic.c, cl.contour, cl.bary);
    s.id_a = a_id;
    s.id_b = b_id;
    if (!contacts_only) {
        const Sphere& a = sp[a_id];
        const Sphere& b = sp[b_id];
        s.solid_angle_a = calculate_solid_angle(a, b, cl.ic, cl.contour);
        s.solid_angle_b = calculate_solid_angle(b, a, cl.ic, cl.contour);
        double sign_a = s.solid_angle_a < 0.0 ? -1.0 : 1.0;
        double sign_b = s.solid_angle_b < 0.0 ? -1.0 : 1.0;
        s.pyramid_volume_a = norm(cl.ic.c - a.c) * cl.area / 3.0 * sign_a;
        s.pyramid_volume_b = norm(cl.ic.c - b.c) * cl.area / 3.0 * sign_b;
        s.distance = norm(b.c - a.c);
    }
    return true;
}

// Tessellation network elements (TessellationVertex / TessellationEdge, types.rs:456-570);
// ids sorted, the NULL id (types.rs:98) is UINT64_MAX.
struct NetVertex {
    uint64_t ids[4];
    double p[3];
};
struct NetEdge {
    uint64_t ids[3];
    double length;
};

constexpr uint64_t NET_NULL = UINT64_MAX;  // NULL_ID (types.rs:98)

void sort_ids4(uint64_t* v) {  // TessellationVertex::sort_ids (types.rs:476-494), a sorting network
    auto cs = [&](int i, int j) {
        if (v[i] > v[j]) std::swap(v[i], v[j]);
    };
    cs(0, 1);
    cs(2, 3);
    cs(0, 2);
    cs(1, 3);
    cs(1, 2);
}
void sort_ids3(uint64_t* v) {  // TessellationEdge::sort_ids (types.rs:543-556)
    auto cs = [&](int i, int j) {
        if (v[i] > v[j]) std::swap(v[i], v[j]);
    };
    cs(0, 1);
    cs(1, 2);
    cs(0, 1);
}

// to_tessellation_elements (contact.rs:119-177) for a valid clipped contact of (a, b).
void tessellation_elements(const Clipped& cl, uint64_t a_id, uint64_t b_id, std::vector<NetEdge>& E,
                           std::vector<NetVertex>& Vs) {
    if (cl.contour.empty()) {  // an uncut contact: one SAS edge, no vertices
        NetEdge e{{a_id, b_id, NET_NULL}, cl.sum_arc * cl.ic.r};
        sort_ids3(e.ids);
        E.push_back(e);
        return;
    }
    const size_t m = cl.contour.size();
    for (size_t i = 0; i < m; ++i) {
        const ContourPoint& cp = cl.contour[i];
        const ContourPoint& nx = cl.contour[(i + 1) % m];
        const bool arc = cp.right_id == a_id;
        NetEdge e{{a_id, b_id, arc ? NET_NULL : cp.right_id}, arc ? cp.angle * cl.ic.r : norm(cp.p - nx.p)};
        sort_ids3(e.ids);
        E.push_back(e);
        NetVertex v{{a_id, b_id, cp.left_id == a_id ? NET_NULL : cp.left_id, arc ? NET_NULL : cp.right_id},
                    {cp.p.x, cp.p.y, cp.p.z}};
        sort_ids4(v.ids);
        Vs.push_back(v);
    }
}

// assemble_tessellation_network (tessellation.rs:334-401): ids mod n for periodic images
// (NULL kept), ids re-sorted, then elements sorted by ids and deduplicated.  The
// reference sorts unstably, so which of several equal-id elements survives is
// unspecified; here it is the first in pair and contour order (a stable sort).
void assemble_network(std::vector<NetEdge>& E, std::vector<NetVertex>& Vs, bool periodic, uint64_t n) {
    auto canon = [&](uint64_t id) { return (periodic && id != NET_NULL) ? id % n : id; };
    for (auto& e : E) {
        for (auto& id : e.ids) id = canon(id);
        sort_ids3(e.ids);
    }
    for (auto& v : Vs) {
        for (auto& id : v.ids) id = canon(id);
        sort_ids4(v.ids);
    }
    std::stable_sort(E.begin(), E.end(), [](const NetEdge& x, const NetEdge& y) {
        return std::lexicographical_compare(x.ids, x.ids + 3, y.ids, y.ids + 3);
    });
    std::stable_sort(Vs.begin(), Vs.end(), [](const NetVertex& x, const NetVertex& y) {
        return std::lexicographical_compare(x.ids, x.ids + 4, y.ids, y.ids + 4);
    });
    E.erase(std::unique(E.begin(), E.end(),
                        [](const NetEdge& x, const NetEdge& y) { return std::equal(x.ids, x.ids + 3, y.ids); }),
            E.end());
    Vs.erase(std::unique(Vs.begin(), Vs.end(),
                         [](const NetVertex& x, const NetVertex& y) { return std::equal(x.ids, x.ids + 4, y.ids); }),
             Vs.end());
}

bool g_network = false;  // vto_compute also builds the tessellation network

inline bool same_group(const int32_t* g, uint64_t ng, uint64_t a, uint64_t b) {  // tessellation.rs:323-328
    return g && a < ng && b < ng && g[a] == g[b];
}

}  // namespace

// ---------------------------------------------------------------------------------------
struct vto_result {
    uint64_t num_balls = 0;
    std::vector<NetVertex> net_v;
    std::vector<NetEdge> net_e;
    std::vector<uint64_t> c_a, c_b;
    std::vector<double> c_area, c_arc;
    std::vector<uint8_t> c_central;
    std::vector<uint64_t> cell_index;
    std::vector<double> cell_sas, cell_vol;
    // internals
    std::vector<uint64_t> nb_off, nb_ids;
    std::vector<double> nb_vals;
    std::vector<uint64_t> p_a, p_b;
    std::vector<uint8_t> p_valid, p_central;
    std::vector<double> p_area, p_arc, p_sa, p_sb, p_pa, p_pb;
};

namespace {

int g_threads = 0;

int thread_count() {
    if (g_threads > 0) return g_threads;
    unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)hc : 1;
}

// Dynamic-schedule parallel loop over [0, n) in chunks (std::thread; the per-element
// work is independent, so results do not depend on the thread count).
void parallel_for(int64_t n, int64_t chunk, const std::function<void(int64_t)>& body) {
    int nt = thread_count();
    if (nt <= 1 || n <= chunk) {
        for (int64_t i = 0; i < n; ++i) body(i);
        return;
    }
    std::atomic<int64_t> next(0);
    auto worker = [&]() {
        for (;;) {
            int64_t b = next.fetch_add(chunk);
            if (b >= n) break;
            int64_t e = std::min(n, b + chunk);
            for (int64_t i = b; i < e; ++i) body(i);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
}

struct CollisionContext {  // tessellation.rs:51-111
    std::vector<Sphere> input;
    std::unique_ptr<Searcher> searcher;
    std::vector<std::vector<ValuedId>> all;
    std::vector<std::pair<uint64_t, uint64_t>> pairs;
    uint64_t n = 0;
    bool periodic = false;
};

static void run_parallel_neighbors(const Searcher& s, uint64_t n, std::vector<std::vector<ValuedId>>& all,
                                   std::vector<uint8_t>* excluded) {
    all.assign(n, {});
    if (excluded) excluded->assign(n, 0);
    parallel_for((int64_t)n, 64, [&](int64_t i) {
        CollisionResult r = s.find_colliding_ids((uint64_t)i, true);
        all[i] = std::move(r.ids);
        if (excluded) (*excluded)[i] = r.excluded;
    });
}

static std::vector<std::pair<uint64_t, uint64_t>> collect_collision_pairs(
    const std::vector<std::vector<ValuedId>>& all, const int32_t* g, uint64_t ng, uint64_t pn,
    bool periodic) {  // tessellation.rs:298-319
    std::vector<std::pair<uint64_t, uint64_t>> out;
    for (uint64_t a = 0; a < all.size(); ++a)
        for (const ValuedId& v : all[a]) {
            uint64_t b = v.index;
            uint64_t bc = periodic ? b % pn : b;
            if (same_group(g, ng, a, bc)) continue;
            if ((periodic && b >= pn) || a < b) out.emplace_back(a, b);
        }
    return out;
}

static void build_context(const double* xyzr, uint64_t n, double probe, const double* pbox9,
                          const int32_t* g, uint64_t ng, CollisionContext& ctx) {
    ctx.n = n;
    ctx.input.resize(n);
    for (uint64_t i = 0; i < n; ++i)
        ctx.input[i] = {{xyzr[4 * i], xyzr[4 * i + 1], xyzr[4 * i + 2]}, xyzr[4 * i + 3] + probe};
    if (pbox9) {  // new_periodic (tessellation.rs:85-110)
        PBox pb{{pbox9[0], pbox9[1], pbox9[2]}, {pbox9[3], pbox9[4], pbox9[5]}, {pbox9[6], pbox9[7], pbox9[8]}};
        ctx.periodic = true;
        ctx.searcher.reset(new Searcher(populate_periodic_spheres(pb, ctx.input)));
    } else {  // new_standard (:63-83)
        ctx.searcher.reset(new Searcher(ctx.input));
    }
    run_parallel_neighbors(*ctx.searcher, n, ctx.all, nullptr);
    ctx.pairs = collect_collision_pairs(ctx.all, g, ng, n, ctx.periodic);
}

// compute_canonical_ids (tessellation.rs:556-601)
static std::vector<uint64_t> canonical_ids(const std::vector<ContactSummary>& s, uint64_t n) {
    std::vector<std::vector<uint64_t>> b2c(n);
    for (uint64_t i = 0; i < s.size(); ++i)
        if (s[i].id_a >= n || s[i].id_b >= n) {
            b2c[s[i].id_a % n].push_back(i);
            b2c[s[i].id_b % n].push_back(i);
        }
    std::vector<uint64_t> can(s.size());
    for (uint64_t i = 0; i < s.size(); ++i) can[i] = i;
    for (uint64_t i = 0; i < s.size(); ++i) {
        if (!(s[i].id_a >= n || s[i].id_b >= n)) continue;
        uint64_t sa = s[i].id_a % n, sb = s[i].id_b % n;
        const auto& cands = b2c[sa].size() <= b2c[sb].size() ? b2c[sa] : b2c[sb];
        for (uint64_t ci : cands) {
            uint64_t ca = s[ci].id_a % n, cb = s[ci].id_b % n;
            if ((ca == sa && cb == sb) || (ca == sb && cb == sa)) {
                can[i] = ci;
                break;
            }
        }
    }
    return can;
}

// compute_cells (tessellation.rs:607-658)
static void compute_cells(const std::vector<ContactSummary>& sums, const std::vector<Sphere>& sp,
                          const std::vector<std::vector<ValuedId>>& all, bool periodic, uint64_t n,
                          vto_result* r) {
    std::vector<CellSummary> cs(n);
    for (uint64_t i = 0; i < n; ++i) cs[i].id = i;
    for (const ContactSummary& c : sums) {
        if (!(c.area > 0.0)) continue;
        if (periodic) {
            if (c.id_a < n) cs[c.id_a].add(c);
            if (c.id_b < n && c.id_b != c.id_a) cs[c.id_b].add(c);
        } else {
            cs[c.id_a].add(c);
            cs[c.id_b].add(c);
        }
    }
    for (uint64_t i = 0; i < n; ++i) {
        if (cs[i].stage == Stage::ContactsAdded)
            cs[i].compute_sas(sp[i].r);
        else if (cs[i].stage == Stage::Init && all[i].empty())
            cs[i].compute_sas_detached(i, sp[i].r);
    }
    for (uint64_t i = 0; i < n; ++i)
        if (cs[i].stage == Stage::SasComputed) {
            r->cell_index.push_back(cs[i].id);
            r->cell_sas.push_back(cs[i].sas_area);
            r->cell_vol.push_back(cs[i].sas_inside_volume);
        }
}

static void push_contact(vto_result* r, uint64_t a, uint64_t b, double area, double arc, bool central) {
    r->c_a.push_back(a);
    r->c_b.push_back(b);
    r->c_area.push_back(area);
    r->c_arc.push_back(arc);
    r->c_central.push_back(central ? 1 : 0);
}

}  // namespace

extern "C" {

void vto_set_threads(int n) { g_threads = n; }
void vto_set_faithful_grid_update(int on) { g_faithful_grid_update = on != 0; }
int vto_get_threads(void) { return thread_count(); }

int vto_compute(const double* xyzr, uint64_t n, double probe, const double* pbox9, const int32_t* groups,
                uint64_t n_groups, int contacts_only, vto_result** out) {
    vto_result* r = new vto_result();
    *out = r;
    r->num_balls = n;
    r->nb_off.assign(n + 1, 0);
    if (n == 0) {  // tessellation.rs:131-133, 205-207
        r->num_balls = 0;
        return 0;
    }
    CollisionContext ctx;
    build_context(xyzr, n, probe, pbox9, groups, n_groups, ctx);
    for (uint64_t i = 0; i < n; ++i) {
        r->nb_off[i + 1] = r->nb_off[i] + ctx.all[i].size();
        for (const ValuedId& v : ctx.all[i]) {
            r->nb_ids.push_back(v.index);
            r->nb_vals.push_back(v.value);
        }
    }
    const auto& sp = ctx.searcher->spheres;
    size_t np = ctx.pairs.size();
    std::vector<ContactSummary> sums(np);
    std::vector<uint8_t> ok(np, 0);
    const bool network = g_network && !contacts_only;
    std::vector<std::vector<NetEdge>> pe(network ? np : 0);
    std::vector<std::vector<NetVertex>> pv(network ? np : 0);
    parallel_for((int64_t)np, 256, [&](int64_t k) {
        uint64_t a = ctx.pairs[k].first, b = ctx.pairs[k].second;
        ContactSummary s;
        if (contact_summary(sp, a, b, ctx.all[a], contacts_only != 0, s)) {
            sums[k] = s;
            ok[k] = 1;
            if (network) {
                Clipped cl;
                if (clip_contact(sp, a, b, ctx.all[a], cl)) tessellation_elements(cl, a, b, pe[k], pv[k]);
            }
        }
    });
    if (network) {
        for (size_t k = 0; k < np; ++k)
            if (ok[k] && sums[k].area > 0.0) {
                r->net_e.insert(r->net_e.end(), pe[k].begin(), pe[k].end());
                r->net_v.insert(r->net_v.end(), pv[k].begin(), pv[k].end());
            }
        assemble_network(r->net_e, r->net_v, ctx.periodic, n);
    }
    r->p_a.resize(np);
    r->p_b.resize(np);
    r->p_valid = ok;
    r->p_area.assign(np, 0);
    r->p_arc.assign(np, 0);
    r->p_central.assign(np, 0);
    r->p_sa.assign(np, 0);
    r->p_sb.assign(np, 0);
    r->p_pa.assign(np, 0);
    r->p_pb.assign(np, 0);
    for (size_t k = 0; k < np; ++k) {
        r->p_a[k] = ctx.pairs[k].first;
        r->p_b[k] = ctx.pairs[k].second;
        if (ok[k]) {
            const ContactSummary& s = sums[k];
            r->p_area[k] = s.area;
            r->p_arc[k] = s.arc_length;
            r->p_central[k] = s.central;
            r->p_sa[k] = s.solid_angle_a;
            r->p_sb[k] = s.solid_angle_b;
            r->p_pa[k] = s.pyramid_volume_a;
            r->p_pb[k] = s.pyramid_volume_b;
        }
    }
    std::vector<ContactSummary> valid;
    valid.reserve(np);
    for (size_t k = 0; k < np; ++k)
        if (ok[k] && sums[k].area > 0.0) {
            ContactSummary s = sums[k];
            s.ensure_ids_ordered();
            valid.push_back(s);
        }
    if (contacts_only) {
        if (!ctx.periodic) {
            for (const auto& s : valid) push_contact(r, s.id_a, s.id_b, s.area, s.arc_length, s.central);
        } else {
            // deduplicate_and_canonicalize_contacts (tessellation.rs:172-188): first occurrence
            // per canonical (min, max) pair in pair order; reference output order is
            // unspecified (HashMap) -- here it is the order of first occurrence.
            std::unordered_map<uint64_t, uint8_t> seen;
            std::map<std::pair<uint64_t, uint64_t>, int> seen2;
            for (const auto& s : valid) {
                uint64_t ca = s.id_a % n, cb = s.id_b % n;
                std::pair<uint64_t, uint64_t> key = ca <= cb ? std::make_pair(ca, cb) : std::make_pair(cb, ca);
                if (seen2.emplace(key, 1).second)
                    push_contact(r, key.first, key.second, s.area, s.arc_length, s.central);
            }
        }
        return 0;
    }
    compute_cells(valid, ctx.input, ctx.all, ctx.periodic, n, r);
    if (!ctx.periodic) {
        for (const auto& s : valid) push_contact(r, s.id_a, s.id_b, s.area, s.arc_length, s.central);
    } else {
        std::vector<uint64_t> can = canonical_ids(valid, n);  // deduplicate_periodic_contacts
        for (size_t i = 0; i < valid.size(); ++i)
            if (can[i] == i)
                push_contact(r, valid[i].id_a % n, valid[i].id_b % n, valid[i].area, valid[i].arc_length,
                             valid[i].central);
    }
    return 0;
}

void vto_set_network(int on) { g_network = on != 0; }
uint64_t vto_num_vertices(const vto_result* r) { return r->net_v.size(); }
uint64_t vto_num_edges(const vto_result* r) { return r->net_e.size(); }
void vto_get_vertices(const vto_result* r, uint64_t* ids4, double* xyz3) {
    for (size_t i = 0; i < r->net_v.size(); ++i) {
        for (int k = 0; k < 4; ++k) ids4[4 * i + k] = r->net_v[i].ids[k];
        for (int k = 0; k < 3; ++k) xyz3[3 * i + k] = r->net_v[i].p[k];
    }
}
void vto_get_edges(const vto_result* r, uint64_t* ids3, double* length) {
    for (size_t i = 0; i < r->net_e.size(); ++i) {
        for (int k = 0; k < 3; ++k) ids3[3 * i + k] = r->net_e[i].ids[k];
        length[i] = r->net_e[i].length;
    }
}
uint64_t vto_num_balls(const vto_result* r) { return r->num_balls; }
uint64_t vto_num_contacts(const vto_result* r) { return r->c_a.size(); }
uint64_t vto_num_cells(const vto_result* r) { return r->cell_index.size(); }
void vto_get_contacts(const vto_result* r, uint64_t* a, uint64_t* b, double* area, double* arc, uint8_t* central) {
    size_t m = r->c_a.size();
    if (m == 0) return;
    std::memcpy(a, r->c_a.data(), m * 8);
    std::memcpy(b, r->c_b.data(), m * 8);
    std::memcpy(area, r->c_area.data(), m * 8);
    std::memcpy(arc, r->c_arc.data(), m * 8);
    std::memcpy(central, r->c_central.data(), m);
}
void vto_get_cells(const vto_result* r, uint64_t* index, double* sas, double* vol) {
    size_t m = r->cell_index.size();
    if (m == 0) return;
    std::memcpy(index, r->cell_index.data(), m * 8);
    std::memcpy(sas, r->cell_sas.data(), m * 8);
    std::memcpy(vol, r->cell_vol.data(), m * 8);
}
uint64_t vto_num_neighbor_entries(const vto_result* r) { return r->nb_ids.size(); }
void vto_get_neighbors(const vto_result* r, uint64_t* off, uint64_t* ids, double* vals) {
    std::memcpy(off, r->nb_off.data(), r->nb_off.size() * 8);
    if (!r->nb_ids.empty()) {
        std::memcpy(ids, r->nb_ids.data(), r->nb_ids.size() * 8);
        std::memcpy(vals, r->nb_vals.data(), r->nb_vals.size() * 8);
    }
}
uint64_t vto_num_pairs(const vto_result* r) { return r->p_a.size(); }
void vto_get_pairs(const vto_result* r, uint64_t* a, uint64_t* b, uint8_t* valid, double* area, double* arc,
                   uint8_t* central, double* sa, double* sb, double* pa, double* pb) {
    size_t m = r->p_a.size();
    if (m == 0) return;
    std::memcpy(a, r->p_a.data(), m * 8);
    std::memcpy(b, r->p_b.data(), m * 8);
    std::memcpy(valid, r->p_valid.data(), m);
    std::memcpy(area, r->p_area.data(), m * 8);
    std::memcpy(arc, r->p_arc.data(), m * 8);
    std::memcpy(central, r->p_central.data(), m);
    std::memcpy(sa, r->p_sa.data(), m * 8);
    std::memcpy(sb, r->p_sb.data(), m * 8);
    std::memcpy(pa, r->p_pa.data(), m * 8);
    std::memcpy(pb, r->p_pb.data(), m * 8);
}
void vto_free(vto_result* r) { delete r; }

}  // extern "C"

// ---------------------------------------------------------------------------------------
// UpdateableTessellation (updateable.rs) over SpheresContainer (spheres_container.rs).
namespace {

struct UpdateResult {
    std::vector<uint64_t> changed, affected;
    bool full = false;
};

struct Container {  // SpheresContainer, spheres_container.rs:28-405
    std::vector<Sphere> spheres;
    bool has_pbox = false;
    PBox pbox{};
    std::vector<Sphere> populated;
    std::vector<uint8_t> excl;
    std::vector<std::vector<ValuedId>> coll;
    uint64_t total_collisions = 0;
    std::shared_ptr<Searcher> searcher;  // copied on backup (value semantics below)

    Container() = default;
    Container(const Container& o)
        : spheres(o.spheres), has_pbox(o.has_pbox), pbox(o.pbox), populated(o.populated), excl(o.excl),
          coll(o.coll), total_collisions(o.total_collisions),
          searcher(o.searcher ? std::make_shared<Searcher>(*o.searcher) : nullptr) {}
    Container& operator=(const Container& o) {
        if (this == &o) return *this;
        spheres = o.spheres;
        has_pbox = o.has_pbox;
        pbox = o.pbox;
        populated = o.populated;
        excl = o.excl;
        coll = o.coll;
        total_collisions = o.total_collisions;
        searcher = o.searcher ? std::make_shared<Searcher>(*o.searcher) : nullptr;
        return *this;
    }

    uint64_t threshold() const { return std::max<uint64_t>(spheres.size() / 2, 10); }  // :288-291
    void populate() {  // :294-300
        populated = has_pbox ? populate_periodic_spheres(pbox, spheres) : spheres;
    }
    void init(const std::vector<Sphere>& s, bool hp, PBox pb) {  // :55-64
        spheres = s;
        has_pbox = hp;
        pbox = pb;
        populate();
        excl.assign(populated.size(), 0);
        searcher = std::make_shared<Searcher>(populated);
        detect_all_collisions();
    }
    void set_excl_periodic(uint64_t id) {  // :327-341
        if (!has_pbox) return;
        uint64_t n = spheres.size();
        if (excl.size() != n * 27) return;
        uint8_t st = excl[id];
        for (uint64_t m = 1; m < 27; ++m) excl[m * n + id] = st;
    }
    void detect_all_collisions() {  // :344-370
        uint64_t n = spheres.size();
        std::vector<uint8_t> ex;
        run_parallel_neighbors(*searcher, n, coll, &ex);
        for (uint64_t i = 0; i < n; ++i) excl[i] = ex[i];
        if (has_pbox)
            for (uint64_t i = 0; i < n; ++i) set_excl_periodic(i);
        recount();
    }
    void update_collisions_for(const std::vector<uint64_t>& ids) {  // :373-394
        std::vector<CollisionResult> res(ids.size());
        parallel_for((int64_t)ids.size(), 16,
                     [&](int64_t k) { res[k] = searcher->find_colliding_ids(ids[k], true); });
        for (size_t k = 0; k < ids.size(); ++k) {
            coll[ids[k]] = std::move(res[k].ids);
            excl[ids[k]] = res[k].excluded;
        }
        if (has_pbox)
            for (uint64_t id : ids) set_excl_periodic(id);
    }
    void recount() {  // :397-404
        uint64_t t = 0;
        for (auto& v : coll) t += v.size();
        total_collisions = t / 2;
    }
    void update_periodic_instances(uint64_t id, std::vector<uint64_t>& changed) {  // :303-324
        if (id >= spheres.size()) return;
        uint64_t n = spheres.size();
        populated[id] = spheres[id];
        changed.push_back(id);
        if (has_pbox) {
            auto shifts = neighbor_shifts();
            for (size_t g = 0; g < shifts.size(); ++g) {
                uint64_t sid = (g + 1) * n + id;
                populated[sid] = pbox.shift(spheres[id], shifts[g].x, shifts[g].y, shifts[g].z);
                changed.push_back(sid);
            }
        }
    }
    // update (:71-182); returns false for "None" (no change).
    bool update(const std::vector<Sphere>& ns, const uint64_t* changed_ids, uint64_t k, bool have_ids,
                UpdateResult& out) {
        out = UpdateResult();
        if (ns.size() != spheres.size()) {
            init(ns, has_pbox, pbox);
            out.full = true;
            return true;
        }
        uint64_t thr = threshold();
        std::vector<uint64_t> changed;
        if (have_ids) {
            for (uint64_t t = 0; t < k; ++t) {
                uint64_t id = changed_ids[t];
                if (id < spheres.size() && !sphere_equals_sphere(ns[id], spheres[id])) changed.push_back(id);
            }
        } else {
            for (uint64_t i = 0; i < ns.size() && changed.size() < thr + 1; ++i)
                if (!sphere_equals_sphere(ns[i], spheres[i])) changed.push_back(i);
        }
        if (changed.empty()) return false;
        if (changed.size() > thr) {
            init(ns, has_pbox, pbox);
            out.full = true;
            return true;
        }
        std::vector<uint64_t> affected = changed;
        std::sort(affected.begin(), affected.end());
        uint64_t n = spheres.size();
        for (uint64_t sid : changed)
            for (const ValuedId& v : coll[sid]) {
                uint64_t cid = v.index % n;
                auto it = std::lower_bound(affected.begin(), affected.end(), cid);
                if (it == affected.end() || *it != cid) {
                    if (affected.size() < thr) {
                        affected.insert(it, cid);
                    } else {
                        init(ns, has_pbox, pbox);
                        out.full = true;
                        return true;
                    }
                }
            }
        std::vector<uint64_t> changed_pop;
        for (uint64_t sid : changed) {
            spheres[sid] = ns[sid];
            update_periodic_instances(sid, changed_pop);
        }
        if (searcher) searcher->update(populated, changed_pop);
        update_collisions_for(affected);
        std::vector<uint64_t> more;
        for (uint64_t sid : changed)
            for (const ValuedId& v : coll[sid]) {
                uint64_t cid = v.index % n;
                if (!std::binary_search(affected.begin(), affected.end(), cid)) {
                    auto it = std::lower_bound(more.begin(), more.end(), cid);
                    if (it == more.end() || *it != cid) more.insert(it, cid);
                }
            }
        if (!more.empty()) {
            update_collisions_for(more);
            affected.insert(affected.end(), more.begin(), more.end());
            std::sort(affected.begin(), affected.end());
            affected.erase(std::unique(affected.begin(), affected.end()), affected.end());
        }
        recount();
        out.changed = changed;
        out.affected = affected;
        out.full = false;
        return true;
    }
    bool set_exclusion(uint64_t id, bool ex, std::vector<uint64_t>& affected) {  // :186-208
        if (id >= spheres.size() || id >= excl.size()) return false;
        if ((excl[id] != 0) == ex) return false;
        excl[id] = ex;
        set_excl_periodic(id);
        affected.assign(1, id);
        uint64_t n = spheres.size();
        for (const ValuedId& v : coll[id]) {
            uint64_t cid = v.index % n;
            auto it = std::lower_bound(affected.begin(), affected.end(), cid);
            if (it == affected.end() || *it != cid) affected.insert(it, cid);
        }
        return true;
    }
    bool is_excluded(uint64_t id) const { return id < excl.size() && excl[id]; }
    void restore_from(const Container& b, const std::vector<uint64_t>& aff) {  // :246-286
        if (aff.empty() || spheres.size() != b.spheres.size() || aff.size() > threshold()) {
            *this = b;
            return;
        }
        uint64_t n = spheres.size();
        for (uint64_t id : aff)
            if (id >= n) {
                *this = b;
                return;
            }
        for (uint64_t id : aff) {
            spheres[id] = b.spheres[id];
            coll[id] = b.coll[id];
            excl[id] = b.excl[id];
            if (has_pbox)
                for (uint64_t m = 1; m < 27; ++m) {
                    uint64_t sid = m * n + id;
                    if (sid < populated.size()) {
                        populated[sid] = b.populated[sid];
                        excl[sid] = b.excl[sid];
                    }
                }
            populated[id] = b.populated[id];
        }
        total_collisions = b.total_collisions;
        if (b.searcher) searcher = std::make_shared<Searcher>(*b.searcher);
    }
};

struct UState {  // State, updateable.rs:104-124
    Container container;
    uint64_t num_balls = 0;
    std::vector<std::vector<ContactSummary>> cbs;  // contacts_by_sphere
    std::vector<CellSummary> cells;
    std::vector<uint64_t> changed, affected;
    bool full = true;
    bool result_empty() const {  // UpdateableResult::is_empty (:35-37)
        bool any_cell = false;
        for (const auto& c : cells)
            if (c.stage == Stage::SasComputed) {
                any_cell = true;
                break;
            }
        return !any_cell || cbs.empty();
    }
};

}  // namespace

struct vto_upd {
    UState st;
    std::unique_ptr<UState> backup;
    bool backup_enabled = false;
    double probe = 0.0;

    void prepare_for_update() {  // :404-420
        if (backup_enabled && !st.result_empty()) backup.reset(new UState(st));
        st.changed.clear();
        st.affected.clear();
        st.full = false;
    }
    std::vector<std::pair<uint64_t, uint64_t>> collect_pairs(const std::vector<uint8_t>* inv) const {  // :516-561
        uint64_t n = st.container.spheres.size();
        const auto& all = st.container.coll;
        const auto& ex = st.container.excl;
        bool periodic = st.container.has_pbox;
        std::vector<std::pair<uint64_t, uint64_t>> out;
        for (uint64_t a = 0; a < all.size() && a < n; ++a) {
            bool ai = !inv || (a < inv->size() && (*inv)[a]);
            if (!ai || (a < ex.size() && ex[a])) continue;
            for (const ValuedId& v : all[a]) {
                uint64_t b = v.index, bc = b % n;
                bool bi = !inv || (bc < inv->size() && (*inv)[bc]);
                if (!bi || (bc < ex.size() && ex[bc])) continue;
                bool inc = (periodic && b >= n) ? true : a < b;
                if (inc) out.emplace_back(a, b);
            }
        }
        return out;
    }
    // compute_contact_summaries_with_dedup (:565-601)
    void summaries_with_dedup(const std::vector<std::pair<uint64_t, uint64_t>>& pairs, bool periodic, uint64_t n,
                              std::vector<ContactSummary>& all_s, std::vector<ContactSummary>& dedup) const {
        const auto& sp = st.container.populated;
        const auto& coll = st.container.coll;
        std::vector<ContactSummary> tmp(pairs.size());
        std::vector<uint8_t> ok(pairs.size(), 0);
        parallel_for((int64_t)pairs.size(), 64, [&](int64_t k) {
            ContactSummary s;
            uint64_t a = pairs[k].first, b = pairs[k].second;
            if (contact_summary(sp, a, b, coll[a], false, s)) {
                s.id_a = a;
                s.id_b = b;
                s.ensure_ids_ordered();
                if (s.area > 0.0) {
                    tmp[k] = s;
                    ok[k] = 1;
                }
            }
        });
        all_s.clear();
        for (size_t k = 0; k < pairs.size(); ++k)
            if (ok[k]) all_s.push_back(tmp[k]);
        if (periodic) {
            std::vector<uint64_t> can = canonical_ids(all_s, n);
            dedup.clear();
            for (size_t i = 0; i < all_s.size(); ++i)
                if (can[i] == i) {
                    ContactSummary s = all_s[i];
                    s.id_a %= n;
                    s.id_b %= n;
                    s.ensure_ids_ordered();
                    dedup.push_back(s);
                }
        } else {
            dedup = all_s;
        }
    }
    void compute_full() {  // :449-474
        uint64_t n = st.container.spheres.size();
        bool periodic = st.container.has_pbox;
        auto pairs = collect_pairs(nullptr);
        std::vector<ContactSummary> all_s, dd;
        summaries_with_dedup(pairs, periodic, n, all_s, dd);
        st.num_balls = n;
        st.cbs.assign(n, {});
        for (const auto& c : dd)
            if (c.area > 0.0) {
                st.cbs[c.id_a].push_back(c);
                if (c.id_b != c.id_a) st.cbs[c.id_b].push_back(c);
            }
        // compute_cells_from_all_summaries (:633-689)
        const auto& sp = st.container.spheres;
        st.cells.assign(n, CellSummary());
        for (uint64_t i = 0; i < n; ++i) st.cells[i].id = i;
        if (periodic) {
            for (const auto& c : all_s)
                if (c.area > 0.0) {
                    if (c.id_a < n) st.cells[c.id_a].add(c);
                    if (c.id_b < n && c.id_b != c.id_a) st.cells[c.id_b].add(c);
                }
        } else {
            for (uint64_t i = 0; i < n; ++i)
                for (const auto& c : st.cbs[i]) st.cells[i].add(c);
        }
        for (uint64_t i = 0; i < n && i < sp.size(); ++i) {
            auto& cs = st.cells[i];
            if (cs.stage == Stage::ContactsAdded)
                cs.compute_sas(sp[i].r);
            else if (cs.stage == Stage::Init && !st.container.is_excluded(i) && st.container.coll[i].empty())
                cs.compute_sas_detached(i, sp[i].r);
        }
    }
    void update_using_affected() {  // :476-514
        uint64_t n = st.container.spheres.size();
        bool periodic = st.container.has_pbox;
        std::vector<uint8_t> inv(n, 0);
        for (uint64_t id : st.affected)
            if (id < n) inv[id] = 1;
        auto pairs = collect_pairs(&inv);
        std::vector<ContactSummary> all_s, dd;
        summaries_with_dedup(pairs, periodic, n, all_s, dd);
        for (uint64_t sid : st.affected)
            if (sid < n) {
                auto& v = st.cbs[sid];
                v.erase(std::remove_if(v.begin(), v.end(),
                                       [&](const ContactSummary& c) { return inv[c.id_a % n] && inv[c.id_b % n]; }),
                        v.end());
            }
        for (const auto& c : dd)
            if (c.area > 0.0) {
                st.cbs[c.id_a].push_back(c);
                if (c.id_b != c.id_a) st.cbs[c.id_b].push_back(c);
            }
        recompute_cells_for_affected();
    }
    void recompute_cells_for_affected() {  // :691-727
        const auto& sp = st.container.spheres;
        for (uint64_t sid : st.affected) {
            if (sid >= sp.size()) continue;
            CellSummary cs;
            cs.id = sid;
            for (const auto& c : st.cbs[sid]) cs.add(c);
            if (cs.stage == Stage::ContactsAdded) {
                cs.compute_sas(sp[sid].r);
            } else if (cs.stage == Stage::Init && !st.container.is_excluded(sid)) {
                if (st.cbs[sid].empty()) cs.compute_sas_detached(sid, sp[sid].r);
            }
            st.cells[sid] = cs;
        }
    }
    std::vector<Sphere> to_spheres(const double* xyzr, uint64_t n) const {
        std::vector<Sphere> s(n);
        for (uint64_t i = 0; i < n; ++i)
            s[i] = {{xyzr[4 * i], xyzr[4 * i + 1], xyzr[4 * i + 2]}, xyzr[4 * i + 3] + probe};
        return s;
    }
    bool update_internal(const double* xyzr, uint64_t n, const uint64_t* ids, uint64_t k, bool have) {  // :422-447
        prepare_for_update();
        std::vector<Sphere> ns = to_spheres(xyzr, n);
        UpdateResult ur;
        if (!st.container.update(ns, ids, k, have, ur)) return false;
        if (ur.full) {
            st.full = true;
            compute_full();
            return true;
        }
        st.changed = ur.changed;
        st.affected = ur.affected;
        st.full = false;
        update_using_affected();
        return true;
    }
};

extern "C" {

vto_upd* vto_upd_create(int with_backup) {
    vto_upd* h = new vto_upd();
    h->backup_enabled = with_backup != 0;
    return h;
}
void vto_upd_destroy(vto_upd* h) { delete h; }
int vto_upd_init(vto_upd* h, const double* xyzr, uint64_t n, double probe, const double* pbox9) {  // :187-201
    h->probe = probe;
    h->prepare_for_update();
    std::vector<Sphere> s = h->to_spheres(xyzr, n);
    PBox pb{};
    if (pbox9) pb = {{pbox9[0], pbox9[1], pbox9[2]}, {pbox9[3], pbox9[4], pbox9[5]}, {pbox9[6], pbox9[7], pbox9[8]}};
    h->st.container.init(s, pbox9 != nullptr, pb);
    h->st.full = true;
    h->st.changed.clear();
    h->st.affected.clear();
    h->compute_full();
    return !h->st.result_empty();
}
int vto_upd_update(vto_upd* h, const double* xyzr, uint64_t n) { return h->update_internal(xyzr, n, nullptr, 0, false); }
int vto_upd_update_with_changed(vto_upd* h, const double* xyzr, uint64_t n, const uint64_t* ids, uint64_t k) {
    if (k == 0) return 0;  // :216-218
    return h->update_internal(xyzr, n, ids, k, true);
}
int vto_upd_set_exclusion(vto_upd* h, uint64_t id, int excluded) {  // :226-271
    if (h->st.result_empty() || id >= h->st.cbs.size() || id >= h->st.container.excl.size()) return 0;
    bool cur = h->st.container.is_excluded(id);
    if (cur == (excluded != 0)) return 0;
    h->prepare_for_update();
    std::vector<uint64_t> affected;
    if (excluded) {
        affected.push_back(id);
        for (const auto& c : h->st.cbs[id]) {
            uint64_t nid = c.id_a == id ? c.id_b : c.id_a;
            auto it = std::lower_bound(affected.begin(), affected.end(), nid);
            if (it == affected.end() || *it != nid) affected.insert(it, nid);
        }
        std::vector<uint64_t> dummy;
        h->st.container.set_exclusion(id, true, dummy);
    } else {
        if (!h->st.container.set_exclusion(id, false, affected)) return 0;
    }
    h->st.changed.assign(1, id);
    h->st.affected = affected;
    h->st.full = false;
    h->update_using_affected();
    return 1;
}
int vto_upd_restore(vto_upd* h) {  // :277-322
    if (!h->backup_enabled || !h->backup) return 0;
    std::unique_ptr<UState> b = std::move(h->backup);
    std::vector<uint64_t> aff = h->st.affected;
    h->st.container.restore_from(b->container, aff);
    uint64_t n = h->st.cbs.size();
    bool rebuild;
    if (h->st.full || b->cbs.size() != n || b->cells.size() != n) {
        h->st.num_balls = b->num_balls;
        h->st.cbs = b->cbs;
        h->st.cells = b->cells;
        rebuild = false;
    } else {
        for (uint64_t id : aff)
            if (id < n) {
                h->st.cbs[id] = b->cbs[id];
                h->st.cells[id] = b->cells[id];
            }
        rebuild = true;
    }
    h->st.changed = b->changed;
    h->st.affected = b->affected;
    h->st.full = b->full;
    (void)rebuild;  // cells are derived from `cells` on demand (rebuild_cells_from_summaries)
    return 1;
}
int vto_upd_last_full_reinit(const vto_upd* h) { return h->st.full ? 1 : 0; }
uint64_t vto_upd_num_changed(const vto_upd* h) { return h->st.changed.size(); }
void vto_upd_get_changed(const vto_upd* h, uint64_t* ids) {
    if (!h->st.changed.empty()) std::memcpy(ids, h->st.changed.data(), h->st.changed.size() * 8);
}
uint64_t vto_upd_num_affected(const vto_upd* h) { return h->st.affected.size(); }
void vto_upd_get_affected(const vto_upd* h, uint64_t* ids) {
    if (!h->st.affected.empty()) std::memcpy(ids, h->st.affected.data(), h->st.affected.size() * 8);
}
vto_result* vto_upd_summary(const vto_upd* h) {  // summary (:332-378)
    vto_result* r = new vto_result();
    uint64_t n = h->st.cbs.size();
    r->num_balls = n;
    r->nb_off.assign(n + 1, 0);
    for (uint64_t i = 0; i < n; ++i)
        for (const auto& c : h->st.cbs[i])
            if (c.id_a == i) push_contact(r, c.id_a, c.id_b, c.area, c.arc_length, c.central);
    for (uint64_t i = 0; i < n && i < h->st.cells.size(); ++i) {
        const auto& cs = h->st.cells[i];
        if (cs.stage == Stage::SasComputed) {
            r->cell_index.push_back(cs.id);
            r->cell_sas.push_back(cs.sas_area);
            r->cell_vol.push_back(cs.sas_inside_volume);
        }
    }
    return r;
}

}  // extern "C"

// ---- compute_solvent_spheres (solvent_spheres.rs:131-330) ----------------------------
// SubdividedIcosahedron::new (subdivided_icosahedron.rs:53-125): the 12 normalised
// icosahedron vertices, then `depth` rounds that split every face in four; the midpoint
// of an edge is appended (normalised) the first time the edge is met, visiting faces in
// order and each face's edges as (v1,v2), (v0,v2), (v0,v1).
static std::vector<V3> icosahedron_directions(int depth) {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    const double base[12][3] = {{t, 1.0, 0.0},  {-t, 1.0, 0.0},  {t, -1.0, 0.0}, {-t, -1.0, 0.0},
                                {1.0, 0.0, t},  {1.0, 0.0, -t},  {-1.0, 0.0, t}, {-1.0, 0.0, -t},
                                {0.0, t, 1.0},  {0.0, -t, 1.0},  {0.0, t, -1.0}, {0.0, -t, -1.0}};
    std::vector<V3> v;
    for (const auto& b : base) v.push_back(normalize(V3{b[0], b[1], b[2]}));
    std::vector<std::array<size_t, 3>> faces = {
        {0, 8, 4},  {1, 10, 7}, {2, 9, 11}, {7, 3, 1},  {0, 5, 10}, {3, 9, 6},  {3, 11, 9},
        {8, 6, 4},  {2, 4, 9},  {3, 7, 11}, {4, 2, 0},  {9, 4, 6},  {2, 11, 5}, {0, 10, 8},
        {5, 0, 2},  {10, 5, 7}, {1, 6, 8},  {1, 8, 10}, {6, 1, 3},  {11, 7, 5}};
    for (int d = 0; d < depth; ++d) {
        std::map<std::pair<size_t, size_t>, size_t> mids;
        std::vector<std::array<size_t, 3>> next;
        next.reserve(faces.size() * 4);
        for (const auto& f : faces) {
            const std::pair<size_t, size_t> edges[3] = {{f[1], f[2]}, {f[0], f[2]}, {f[0], f[1]}};
            size_t m[3];
            for (int k = 0; k < 3; ++k) {
                auto key = edges[k].first < edges[k].second ? edges[k]
                                                            : std::make_pair(edges[k].second, edges[k].first);
                auto it = mids.find(key);
                if (it == mids.end()) {
                    v.push_back(normalize((v[edges[k].first] + v[edges[k].second]) * 0.5));
                    it = mids.emplace(key, v.size() - 1).first;
                }
                m[k] = it->second;
            }
            next.push_back({f[0], m[1], m[2]});
            next.push_back({f[1], m[0], m[2]});
            next.push_back({f[2], m[0], m[1]});
            next.push_back({m[0], m[1], m[2]});
        }
        faces.swap(next);
    }
    return v;
}

struct vto_solvent {
    std::vector<double> x, y, z, radius, weight;
    std::vector<uint64_t> parent;
};

extern "C" {

int vto_icosahedron(int depth, double* xyz3) {
    const auto v = icosahedron_directions(depth < 0 ? 0 : (depth > 4 ? 4 : depth));
    if (xyz3)
        for (size_t i = 0; i < v.size(); ++i) {
            xyz3[3 * i] = v[i].x;
            xyz3[3 * i + 1] = v[i].y;
            xyz3[3 * i + 2] = v[i].z;
        }
    return (int)v.size();
}

int vto_solvent_spheres(const double* xyzr, uint64_t n, double probe, double volume_probe, int depth,
                        const double* pbox9, vto_solvent** out) {
    *out = nullptr;
    // validate_params / validate_balls (:164-194)
    if (!std::isfinite(probe) || probe < 0.0) return 1;
    if (!std::isfinite(volume_probe) || volume_probe < 0.0) return 2;
    for (uint64_t i = 0; i < n; ++i) {
        const double* b = xyzr + 4 * i;
        if (!std::isfinite(b[0]) || !std::isfinite(b[1]) || !std::isfinite(b[2])) return 3;
        if (!std::isfinite(b[3]) || b[3] <= 0.0) return 3;
    }
    vto_solvent* res = new vto_solvent();
    *out = res;
    if (n == 0) return 0;
    const bool net = g_network;
    g_network = false;
    // stage 1 (:149-150)
    vto_result* r1 = nullptr;
    vto_compute(xyzr, n, probe, pbox9, nullptr, 0, 0, &r1);
    // build_neighbor_graph (:201-233): partners of each exposed ball (sas_area > 0); the
    // reference sorts them by distance only to stop early, which does not change results
    std::vector<char> exposed(n, 0);
    for (size_t k = 0; k < r1->cell_index.size(); ++k)
        if (r1->cell_sas[k] > 0.0) exposed[r1->cell_index[k]] = 1;
    std::vector<std::vector<uint64_t>> nb(n);
    for (size_t k = 0; k < r1->c_a.size(); ++k) {
        const uint64_t a = r1->c_a[k], b = r1->c_b[k];
        if (exposed[a]) nb[a].push_back(b);
        if (exposed[b]) nb[b].push_back(a);
    }
    auto center = [&](uint64_t i) { return V3{xyzr[4 * i], xyzr[4 * i + 1], xyzr[4 * i + 2]}; };
    // generate_solvent_spheres / is_valid_solvent_position (:236-289)
    const auto dirs = icosahedron_directions(depth < 0 ? 0 : (depth > 4 ? 4 : depth));
    for (size_t k = 0; k < r1->cell_index.size(); ++k) {
        if (!(r1->cell_sas[k] > 0.0)) continue;
        const uint64_t i = r1->cell_index[k];
        const V3 c = center(i);
        const double ri = xyzr[4 * i + 3], R = ri + probe;
        for (const V3& v : dirs) {
            const V3 p = c + v * R;
            const double da = norm(p - c) - ri;
            bool ok = true;
            for (uint64_t j : nb[i])
                if (norm(p - center(j)) - xyzr[4 * j + 3] <= da) {
                    ok = false;
                    break;
                }
            if (!ok) continue;
            res->x.push_back(p.x);
            res->y.push_back(p.y);
            res->z.push_back(p.z);
            res->radius.push_back(probe);
            res->weight.push_back(0.0);
            res->parent.push_back(i);
        }
    }
    vto_free(r1);
    const size_t S = res->x.size();
    if (S > 0) {
        // compute_solvent_weights (:292-345): adjusted atoms, then the solvent spheres,
        // tessellated with probe 0; a solvent sphere's weight is its cell volume
        std::vector<double> comb(4 * (n + S));
        for (uint64_t i = 0; i < n; ++i) {
            comb[4 * i] = xyzr[4 * i];
            comb[4 * i + 1] = xyzr[4 * i + 1];
            comb[4 * i + 2] = xyzr[4 * i + 2];
            comb[4 * i + 3] = rmax(xyzr[4 * i + 3] - probe + volume_probe, 0.01);
        }
        for (size_t s = 0; s < S; ++s) {
            double* c = comb.data() + 4 * (n + s);
            c[0] = res->x[s];
            c[1] = res->y[s];
            c[2] = res->z[s];
            c[3] = probe + volume_probe;
        }
        vto_result* r2 = nullptr;
        vto_compute(comb.data(), n + S, 0.0, pbox9, nullptr, 0, 0, &r2);
        for (size_t k = 0; k < r2->cell_index.size(); ++k)
            if (r2->cell_index[k] >= n) res->weight[r2->cell_index[k] - n] = r2->cell_vol[k];
        vto_free(r2);
    }
    g_network = net;
    return 0;
}
uint64_t vto_solvent_count(const vto_solvent* s) { return s ? s->x.size() : 0; }
void vto_solvent_get(const vto_solvent* s, double* xyzrw5, uint64_t* parent) {
    for (size_t i = 0; i < s->x.size(); ++i) {
        xyzrw5[5 * i] = s->x[i];
        xyzrw5[5 * i + 1] = s->y[i];
        xyzrw5[5 * i + 2] = s->z[i];
        xyzrw5[5 * i + 3] = s->radius[i];
        xyzrw5[5 * i + 4] = s->weight[i];
        parent[i] = s->parent[i];
    }
}
void vto_solvent_free(vto_solvent* s) { delete s; }

}  // extern "C"
