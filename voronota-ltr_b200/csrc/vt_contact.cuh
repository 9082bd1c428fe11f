// vt_contact.cuh -- one warp per candidate pair (a, b): the contact contour clip.
//
// Restates clip_contact / construct_contact_descriptor / construct_contact_area
// (src/contact.rs:196-404) for a warp.  The contour lives in registers, one point per
// lane (capacity 32); the reference's Vec insert/drain/retain become ballot + shuffle
// gathers:
//   * neighbour pre-tests (contact.rs:236-282) run lane-parallel over a's sorted
//     neighbour list, 32 neighbours at a time; a discard anywhere ends the pair (the
//     reference's result is None whichever neighbour discards first);
//   * the cuts are applied sequentially in list order (contact.rs:284-300), each one a
//     lane-parallel mark (ballot) and a gather that restructures the contour;
//   * restrict_contour_to_circle (contact.rs:631-769) is a per-segment insertion count,
//     a warp prefix sum and a gather;
//   * area, arc angles, solid angles and centrality are warp reductions.
// Contours that would exceed 32 points set the overflow status; such pairs are
// recomputed by the serial fallback kernel.
//
// FP32 (F = true): contour points are assumed accurate to a budget E (a runtime
// band, in float ulps of the pair's length scale S).  Every decision whose margin is
// within its E-derived band is "unsure", and so is every ill-conditioned construction
// that could exceed the budget (a cut grazing an edge, a segment nearly tangent to the
// circle); such pairs are recomputed in FP64.  Decisions that cannot change the outcome
// carry no band: the cuttable pre-filter is skipped (a mark with no outsider is a
// no-op), and the |cos| >= 1 branch only flags when its two branches would classify the
// neighbour differently.  The FP64 instantiation (F = false) is the reference's
// arithmetic operation by operation.
#pragma once
#include "vt_geom.cuh"

namespace vt {

constexpr unsigned kFull = 0xffffffffu;
constexpr float kF32Eps = 1.1920929e-7f;

template <typename T>
__device__ __forceinline__ T wsum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}
__device__ __forceinline__ float wmax(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// Sum over the first `len` lanes.  FP64 adds in lane order starting from 0.0, exactly as
// the reference's sequential loops (contact.rs:776-790, 804-833, 741-751): some of its
// decisions (the centrality test of near-degenerate contours) compare rounding-noise
// sized quantities with zero, so the FP64 path must reproduce the summation order.  FP32
// uses a butterfly; its decisions near zero are inside the band and go to FP64.
__device__ __forceinline__ double lsum(double v, int len) {
    double acc = 0.0;
#pragma unroll 1  // code size: the FP64 kernel is bound by instruction fetch
    for (int k = 0; k < len; ++k) acc += __shfl_sync(kFull, v, k);
    return acc;
}
__device__ __forceinline__ float lsum(float v, int) { return wsum(v); }
// acc = (acc + u_k) + w_k for k in lane order (two additions per element)
__device__ __forceinline__ double lsum2(double u, double w, int len) {
    double acc = 0.0;
#pragma unroll 1
    for (int k = 0; k < len; ++k) {
        acc += __shfl_sync(kFull, u, k);
        acc += __shfl_sync(kFull, w, k);
    }
    return acc;
}
__device__ __forceinline__ float lsum2(float u, float w, int) { return wsum(u + w); }

template <typename T>
struct Pt {  // one contour point (contact.rs:36-47), held by one lane
    V3<T> p;
    uint32_t lid, rid;
    T ang;
};

__device__ __forceinline__ V3<double> wide3(V3<double> v) { return v; }
__device__ __forceinline__ V3<double> wide3(V3<float> v) { return {(double)v.x, (double)v.y, (double)v.z}; }

template <typename T>
__device__ __forceinline__ Pt<T> shfl_pt(const Pt<T>& q, int src) {
    Pt<T> r;
    r.p.x = __shfl_sync(kFull, q.p.x, src);
    r.p.y = __shfl_sync(kFull, q.p.y, src);
    r.p.z = __shfl_sync(kFull, q.p.z, src);
    r.lid = __shfl_sync(kFull, q.lid, src);
    r.rid = __shfl_sync(kFull, q.rid, src);
    r.ang = __shfl_sync(kFull, q.ang, src);
    return r;
}
template <typename T>
__device__ __forceinline__ V3<T> shfl_v3(V3<T> v, int src) {
    return {__shfl_sync(kFull, v.x, src), __shfl_sync(kFull, v.y, src), __shfl_sync(kFull, v.z, src)};
}
// The same for the cut loop and the restriction to the circle, where no point carries an
// arc angle yet (all 0).
template <typename T>
__device__ __forceinline__ Pt<T> shfl_pt_flat(const Pt<T>& q, int src) {
    Pt<T> r;
    r.p = shfl_v3(q.p, src);
    r.lid = __shfl_sync(kFull, q.lid, src);
    r.rid = __shfl_sync(kFull, q.rid, src);
    r.ang = 0;
    return r;
}
// Gathers of only the fields a site reads (the others zero): position and left id (the
// next point in the restriction and the arc angles), position and arc angle (the solid
// angle's turn terms).
template <typename T>
__device__ __forceinline__ Pt<T> shfl_pt_pl(const Pt<T>& q, int src) {
    Pt<T> r;
    r.p = shfl_v3(q.p, src);
    r.lid = __shfl_sync(kFull, q.lid, src);
    r.rid = 0;
    r.ang = 0;
    return r;
}
template <typename T>
__device__ __forceinline__ Pt<T> shfl_pt_pa(const Pt<T>& q, int src) {
    Pt<T> r;
    r.p = shfl_v3(q.p, src);
    r.lid = r.rid = 0;
    r.ang = __shfl_sync(kFull, q.ang, src);
    return r;
}

// sin and cos of the half rotation angles of init_contour (contact.rs:463-468): the
// angles k pi/3 accumulate by repeated addition exactly as in the reference, and the
// rotation needs sin/cos of angle/2.  The angles do not depend on the data, so the host
// evaluates them once with the C library the CPU oracle uses (set_hex_table) and every
// FP64 contour starts from bit-identical hexagon points.
static __constant__ double c_hex_sin[8];
static __constant__ double c_hex_cos[8];
static __constant__ int c_hex_n[1];

// Hexagon of init_contour (contact.rs:455-469).  FP64: quaternion rotations (the
// accumulated angles give 7 points, the 7th 8.9e-16 rad short of a full turn).  FP32:
// the same 7 points from a cos/sin table.
__device__ __forceinline__ int init_contour(Pt<double>& q, int lane, uint32_t a_id, const Sph<double>& ic,
                                            V3<double> axis, float) {
    V3<double> first = any_normal(axis) * ic.r * kHexScale;
    const int npts = c_hex_n[0];
    if (lane < npts) {
        V3<double> rot = lane == 0 ? first : rotate_around_axis(axis, c_hex_sin[lane], c_hex_cos[lane], first);
        q.p = ic.c + rot;
    }
    q.lid = q.rid = a_id;
    q.ang = 0.0;
    return npts;
}
__device__ __forceinline__ int init_contour(Pt<float>& q, int lane, uint32_t a_id, const Sph<float>& ic,
                                            V3<float> axis, float e0) {
    V3<float> first = any_normal(axis) * ic.r * (float)kHexScale;
    V3<float> perp = cross(axis, first);
    const float h = 0.8660254037844386f;
    float c = 1.f, s = 0.f;
    switch (lane) {
        case 1: c = 0.5f; s = h; break;
        case 2: c = -0.5f; s = h; break;
        case 3: c = -1.f; s = 0.f; break;
        case 4: c = -0.5f; s = -h; break;
        case 5: c = 0.5f; s = -h; break;
        case 6: c = 1.f; s = -8.881784197001252e-16f; break;
        default: break;
    }
    q.p = ic.c + first * c + perp * s;
    q.lid = q.rid = a_id;
    q.ang = 0.f;
    return 7;
}

// Neighbour record for the pre-tests.
template <typename T>
struct Nb {
    Sph<T> s;
    uint32_t id;
};

template <typename T>
struct PairGeom {
    Sph<T> A, B, ic;
    V3<T> axis;
    uint32_t a_id, b_id;
    T e0;  // FP32: error budget E of a contour point coordinate (A); 0 in FP64
    T S;   // length scale of the pair (R_a + R_b)
    // FULL and XM: lane 0 writes the contact's first moments here (6 doubles: the arcs'
    // and the area's about a's centre, for the SAS and volume adjoints); null: not wanted
    double* xm_out = nullptr;
};

// ---- FP32 constructions: decisions banded by the point error budget E ----
// Ratio of an intersection's sensitivity to its inputs beyond which the construction is
// treated as ill-conditioned (the point could be off by more than E).
constexpr float kCondMax = 64.f;
// The FP32 cut loop's planes of one pass of 32 neighbours (unit normal, offset), per warp
// in shared memory, for blocks of at most PW warps.
constexpr int kPlaneWarps = 8;
template <int PW>
__device__ __forceinline__ float4* warp_planes() {
    __shared__ float4 s_planes[PW][32];
    return s_planes[threadIdx.x >> 5];
}

// FP32 forms with the plane given by its unit normal n and offset h = n . p: the side of
// x (halfspace_of_point_unit, geometry.rs:118-131, with the same kEps margin and band)
// and the cut point of segment a-b (intersection_of_plane_and_segment, geometry.rs:
// 134-148).  The pre-tests' normal is already unit, so no re-normalisation.  Written with
// explicit roundings, which the compiler neither contracts nor reorders, so that every
// instantiation of the kernel (with or without the arc moments) gives the same values.
__device__ __forceinline__ float plane_offset(V3<float> p, V3<float> n) {
    return __fmaf_rn(p.z, n.z, __fmaf_rn(p.y, n.y, __fmul_rn(p.x, n.x)));
}
__device__ __forceinline__ float plane_side(V3<float> n, float h, V3<float> x) {  // n . x - h
    return __fmaf_rn(n.z, x.z, __fmaf_rn(n.y, x.y, __fmaf_rn(n.x, x.x, -h)));
}
// mark_contour's test halfspace >= 0 (on the plane or outside): its one decision is
// sd + kEps < 0, so only that margin is banded (halfspace's 0 / 1 boundary at sd = kEps
// cannot change the mark).
__device__ __forceinline__ bool outside_or_on_h(Dec<float, true>& d, V3<float> n, float h, V3<float> x, float tol) {
    const float m = plane_side(n, h, x) + (float)kEps;
    d.band(m, tol);
    return !(m < 0.f);
}
__device__ __forceinline__ V3<float> plane_segment_h(Dec<float, true>& d, V3<float> n, float h, V3<float> a,
                                                     V3<float> b, float E) {
    const float da = plane_side(n, h, a);
    const float db = plane_side(n, h, b);
    const float den = __fsub_rn(da, db);
    const float dd = fabsf(den);
    d.band(dd - (float)kEps, 2.f * E);
    if (dd < (float)kEps) return a;
    const V3<float> ab = {__fsub_rn(b.x, a.x), __fsub_rn(b.y, a.y), __fsub_rn(b.z, a.z)};
    if (norm(ab) > kCondMax * dd) d.unsure = true;  // cut grazing the edge
    // a cut point is an output vertex: a correctly rounded division (the kernel's
    // approximate one is biased, moving every cut point the same way along its edge)
    const float t = __fdiv_rn(da, den);
    return {__fmaf_rn(ab.x, t, a.x), __fmaf_rn(ab.y, t, a.y), __fmaf_rn(ab.z, t, a.z)};
}
// intersect_segment_with_circle (geometry.rs:258-280)
__device__ __forceinline__ bool segment_circle_e(Dec<float, true>& d, const Sph<float>& c, V3<float> p_in,
                                                 V3<float> p_out, float E, V3<float>* out) {
    float dist = norm(p_in - p_out);
    d.band(dist, 2.f * E);
    if (dist <= 0.f) return false;
    V3<float> v = (p_in - p_out) / dist;
    V3<float> u = c.c - p_out;
    V3<float> s = p_out + v * dot(v, u);
    V3<float> cs = c.c - s;
    float ll = fmaf(c.r, c.r, -norm2(cs));
    d.band(ll, 4.f * E * (c.r + norm(cs)));
    if (ll >= 0.f) {
        float sq = sqrtf(ll);
        if (kCondMax * sq < c.r) d.unsure = true;  // nearly tangent
        *out = s - v * sq;
        return true;
    }
    return false;
}
// project_point_inside_line (geometry.rs:243-255)
__device__ __forceinline__ bool project_inside_line_e(Dec<float, true>& d, V3<float> o, V3<float> a, V3<float> b,
                                                      float E, V3<float>* out) {
    V3<float> ba = b - a;
    float lb = norm(ba);
    V3<float> v = ba / lb;
    float l = dot(v, o - a);
    Dec<float, true> d1, d2;
    bool p = d1.greater(l, 0.f, 2.f * E);
    bool q = d2.less_eq(l * l, lb * lb, 4.f * E * (fabsf(l) + lb));
    if ((d1.unsure || d2.unsure) && !((!p && !d1.unsure) || (!q && !d2.unsure))) d.unsure = true;
    if (p && q) {
        *out = a + v * l;
        return true;
    }
    return false;
}

// Pre-test classes
enum { kSkip = 0, kDiscard = 1, kCut = 2 };

// contact.rs:236-282 for neighbour c.
__device__ __forceinline__ int pretest(Dec<double, false>& d, const PairGeom<double>& g, const Sph<double>& c,
                                       V3<double>& pc, V3<double>& pn) {
    if (!sphere_intersects(d, g.ic, c, 0.0) || !sphere_intersects(d, g.B, c, 0.0)) return kSkip;
    if (sphere_contains(d, c, g.A, 0.0, 0.0) || sphere_contains(d, c, g.B, 0.0, 0.0)) return kDiscard;
    pc = ic_center(g.A, c);
    pn = normalize(c.c - g.A.c);
    double cos_val = dot(normalize(g.ic.c - g.A.c), normalize(pc - g.A.c));
    if (fabs(cos_val) >= 1.0) return halfspace(d, pc, pn, g.ic.c, 0.0) > 0 ? kDiscard : kSkip;
    double l = fabs(sd_plane_unit(pc, pn, g.ic.c));
    double xl = l / sqrt(fma(cos_val, -cos_val, 1.0));
    if (xl >= g.ic.r) return halfspace(d, pc, pn, g.ic.c, 0.0) >= 0 ? kDiscard : kSkip;
    return kCut;
}
__device__ __forceinline__ int pretest(Dec<float, true>& d, const PairGeom<float>& g, const Sph<float>& c,
                                       V3<float>& pc, V3<float>& pn) {
    const float e0 = 0.25f * g.e0, S = g.S;
    if (!sphere_intersects(d, g.ic, c, 2.f * S * e0) || !sphere_intersects(d, g.B, c, 2.f * S * e0)) return kSkip;
    if (sphere_contains(d, c, g.A, e0, 2.f * S * e0) || sphere_contains(d, c, g.B, e0, 2.f * S * e0))
        return kDiscard;
    pc = ic_center(g.A, c);
    pn = normalize(c.c - g.A.c);
    // normalize(pc - a) is +-pn (a is the origin): the sign of the plane's offset
    float h = dot(pc, pn);
    d.band(h, e0);
    float cos_val = dot(normalize(g.ic.c - g.A.c), h >= 0.f ? pn : -pn);
    float sd = sd_plane_unit(pc, pn, g.ic.c);  // shared by both branches
    Dec<float, true> dh;
    int hs = halfspace(dh, pc, pn, g.ic.c, 2.f * e0);
    float one_m = fmaf(cos_val, -cos_val, 1.f);
    Dec<float, true> dc;
    bool big = dc.greater_eq(fabsf(cos_val), 1.f, 4.f * kF32Eps);
    int cls_a = hs > 0 ? kDiscard : kSkip;  // branch |cos| >= 1
    float xl = fabsf(sd) / sqrtf(fmaxf(one_m, 0.f));
    Dec<float, true> dx;
    int cls_b;  // branch |cos| < 1
    if (dx.greater_eq(xl, g.ic.r, e0 * (2.f + 2.f / fmaxf(one_m, 1e-12f))))
        cls_b = hs >= 0 ? kDiscard : kSkip;
    else
        cls_b = kCut;
    int cls = big ? cls_a : cls_b;
    if (dc.unsure) {
        if (cls_a != cls_b || dh.unsure || dx.unsure) d.unsure = true;
    } else if (big) {
        if (dh.unsure) d.unsure = true;
    } else {
        if (dx.unsure || (cls_b != kCut && dh.unsure)) d.unsure = true;
    }
    return cls;
}

// Result of the warp computation (uniform across lanes).
struct WarpContact {
    bool valid;
    bool unsure;
    bool overflow;
    double area, arc, sa_a, sa_b, pv_a, pv_b;
    // serial kernel: xm[0..2] first moment of the contact's arcs about a's centre (the SAS
    // adjoint), xm[3..5] first moment of the contact's area about a's centre (the volume
    // adjoint); the warp kernel writes them to PairGeom::xm_out instead
    double xm[6];
    bool central;
    bool merged;  // two close points were merged (the kept point takes the other's id)
};

// Solid angle (contact.rs:797-848) summed over the warp's contour.  ea0 / ea1 bound the
// arc-angle errors of the previous and the own point (FP32).  FP64 follows the reference
// term by term (half = 0: lanes hold the points).  FP32 with half != 0: each half-warp holds
// the points of one side (contours of at most 16 points), summed within the half.  FP32
// computes each turn term pi - dihedral as the supplement directly
// (no float rounding of pi, which would bias every solid angle and so every SAS area)
// and sums the terms in double.
template <typename T, bool F>
__device__ __forceinline__ double solid_angle(Dec<T, F>& d, const Sph<T>& a, const Sph<T>& b, const Sph<T>& ic,
                                              const Pt<T>& p0, const Pt<T>& p1, const Pt<T>& p2, bool on, int len,
                                              T e0, T ea0, T ea1, int half = 0) {
    double sa;
    if (len == 0) {
        if constexpr (F)
            sa = kTau - kTau * ((double)norm_rn(ic.c - a.c) / (double)a.r);
        else
            sa = kTau - (double)((T)kTau * norm(ic.c - a.c) / a.r);
    } else {
        double t = 0;
        T t2 = 0;
        if (on) {
            const T pi = (T)kPi;
            // turn term at point p1: pi - dihedral (FP32: the supplement, in double)
            // the two directions of the turn at p1: along the arc's tangent where an arc
            // ends or starts at p1, else towards the neighbouring points
            V3<T> x1 = p0.p, x2 = p2.p;
            const bool arc_in = p0.ang > (T)0, arc_out = !arc_in && p1.ang > (T)0;
            if (arc_in || arc_out) {
                const T ang = arc_in ? p0.ang : p1.ang;
                V3<T> dd = cross(b.c - a.c, p1.p - ic.c);
                V3<T> w = (arc_in ? p0.p : p2.p) - p1.p;
                T dv = dot(dd, w);
                if constexpr (F) {
                    d.band(ang - pi, arc_in ? ea0 : ea1);
                    d.band(dv, (T)2 * e0 * (norm(b.c - a.c) * norm(w) + (T)2 * norm(dd)));
                }
                bool flip = (ang < pi && dv < (T)0) || (ang > pi && dv > (T)0);
                if (flip) dd = -dd;
                if (arc_in)
                    x1 = p1.p + dd;
                else
                    x2 = p1.p + dd;
            }
            if constexpr (F)
                t = dihedral_supplement(a.c, p1.p, x1, x2);
            else
                t = pi - min_dihedral(a.c, p1.p, x1, x2);
            if (arc_out) {
                if constexpr (F)
                    t2 = (T)((double)p1.ang * ((double)norm_rn(ic.c - a.c) / (double)a.r));
                else
                    t2 = p1.ang * (norm(ic.c - a.c) / a.r);
            }
        }
        if constexpr (F) {
            // the sum over the lanes of this side: all 32, or 16 when each half-warp holds
            // one side (half != 0)
            double v = t + (double)t2;
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
            if (!half) v += __shfl_xor_sync(kFull, v, 16);
            sa = kTau - v;
        } else {
            sa = kTau - lsum2(t, t2, len);
        }
    }
    V3<T> ic_to_a = ic.c - a.c, ic_to_b = ic.c - b.c;
    Dec<T, F> d1, d2;
    bool c1 = d1.greater(dot(ic_to_a, ic_to_b), (T)0, (T)4 * e0 * (a.r + b.r));
    bool c2 = d2.less(norm2(a.c - ic.c), norm2(b.c - ic.c), (T)4 * e0 * (a.r + b.r));
    if (F && (d1.unsure || d2.unsure) && !((!c1 && !d1.unsure) || (!c2 && !d2.unsure))) d.unsure = true;
    if (c1 && c2) sa = -sa;
    return sa;
}

// The warp-wide contact computation.  `nb(e)` returns neighbour record e of a's sorted
// list (0 <= e < cnt); entry `kb` is b itself.
// The final contour of a valid contact, for the adjoint: this lane's point (its segment to
// the next point is an arc of angle q.ang when q.rid and the next point's lid are a's id,
// otherwise a straight edge on the radical plane of a and neighbour q.rid), the point
// count (0 with full = true: the whole circle), the circle and the axis a -> b.
template <typename T>
struct ContourOut {
    Pt<T> q;
    int len;
    bool full;
    bool unsure;  // a decision of the contour (not of the descriptor) fell in the band
    Sph<T> ic;
    V3<T> axis;
};

// XM: compile in the first moments (computed and written when g.xm_out is set).  PW: the
// warps per block of the calling kernel (FP32).
// rec(q, len, full, unsure, res), when given, is called by the whole warp once the contour
// of a valid contact and its area, arc length and centrality (in res) are final, before
// the descriptor: a caller stores there what it keeps of them, so that none of it stays
// live through the descriptor code.
struct NoContourRecord {
    template <typename P, typename R>
    __device__ __forceinline__ void operator()(const P&, int, bool, bool, const R&) const {}
};
template <typename T, bool F, bool FULL, bool XM = false, int PW = kPlaneWarps, typename NbFn,
          typename RecFn = NoContourRecord>
__device__ WarpContact contact_warp(const PairGeom<T>& g0, int cnt, int kb, NbFn nb, ContourOut<T>* co = nullptr,
                                    RecFn rec = RecFn()) {
    const int lane = threadIdx.x & 31;
    PairGeom<T> g = g0;
    const T e0 = g.e0;
    Dec<T, F> d;
    WarpContact res;
    res.valid = false;
    res.unsure = false;
    res.overflow = false;
    res.area = res.arc = res.sa_a = res.sa_b = res.pv_a = res.pv_b = 0.0;
    for (int k = 0; k < 6; ++k) res.xm[k] = 0.0;
    res.central = false;
    res.merged = false;

    // contact.rs:206-218
    if (!sphere_intersects(d, g.A, g.B, (T)2 * g.S * e0) || sphere_contains(d, g.A, g.B, e0, (T)2 * g.S * e0) ||
        sphere_contains(d, g.B, g.A, e0, (T)2 * g.S * e0)) {
        res.unsure = __any_sync(kFull, d.unsure);
        return res;
    }
    g.ic = intersection_circle(g.A, g.B);
    g.axis = normalize(g.B.c - g.A.c);
    if (d.less_eq(g.ic.r, (T)0, e0)) {
        res.unsure = __any_sync(kFull, d.unsure);
        return res;
    }

    Pt<T> q;
    q.p = mk<T>(0, 0, 0);
    q.lid = q.rid = g.a_id;
    q.ang = 0;
    int len = 0;
    bool init = false;
    bool discarded = false;

    for (int base = 0; base < cnt && !discarded; base += 32) {
        int e = base + lane;
        int cls = kSkip;
        V3<T> pc = mk<T>(0, 0, 0), pn = mk<T>(0, 0, 0);
        uint32_t cid = 0;
        if (e < cnt && e != kb) {
            Nb<T> c = nb(e);
            cid = c.id;
            cls = pretest(d, g, c.s, pc, pn);
        }
        if constexpr (F) pc.x = plane_offset(pc, pn);  // FP32: the cut loop takes the plane as (pn, pn . pc)
        if (__any_sync(kFull, cls == kDiscard)) {
            discarded = true;
            break;
        }
        unsigned cutmask = __ballot_sync(kFull, cls == kCut);
        // FP32: the pass's cutting planes go to shared memory once, and each cut candidate
        // reads its plane as one broadcast 16-byte load instead of four shuffles (the
        // previous pass's reads end at the first __syncwarp)
        if constexpr (F) {
            __syncwarp();
            if (cls == kCut) warp_planes<PW>()[lane] = make_float4(pn.x, pn.y, pn.z, pc.x);
            __syncwarp();
        }
        while (cutmask) {
            int j = __ffs(cutmask) - 1;
            cutmask &= cutmask - 1;
            V3<T> PC, PN;
            if constexpr (F) {
                const float4 pl = warp_planes<PW>()[j];
                PN = {pl.x, pl.y, pl.z};
                PC.x = pl.w;  // the plane offset
            } else {
                PN = shfl_v3(pn, j);
                PC = shfl_v3(pc, j);
            }
            if (!init) {
                len = init_contour(q, lane, g.a_id, g.ic, g.axis, (float)e0);
                init = true;
            } else if constexpr (!F) {
                // test_contour_cuttable (contact.rs:472-481).  A pure pre-filter: a mark that
                // finds no outsider changes nothing, so the FP32 path goes straight to the mark.
                T thr = norm2(PC - g.A.c);
                bool cut = lane < len && norm2(q.p - g.A.c) >= thr;
                if (!__any_sync(kFull, cut)) continue;
            }
            // mark_contour (contact.rs:506-521)
            bool out;
            if constexpr (F)
                out = lane < len && outside_or_on_h(d, PN, PC.x, q.p, e0);
            else
                out = lane < len && halfspace(d, PC, PN, q.p, e0) >= 0;
            unsigned om = __ballot_sync(kFull, out);
            if (om == 0) continue;
            int nout = __popc(om);
            if (nout >= len) {  // mark_and_cut_contour clears (contact.rs:496-499)
                len = 0;
                discarded = true;
                break;
            }
            const uint32_t CID = __shfl_sync(kFull, cid, j);  // needed only when the mark cuts
            if (out) q.lid = q.rid = CID;
            if (len < 3) continue;  // cut_contour returns early (contact.rs:530-532)
            // cut_contour (contact.rs:534-626)
            int start = __ffs(om) - 1;
            int end = 31 - __clz(om);
            if (start == 0 && end == len - 1) {
                end = __ffs(~om) - 2;
                unsigned top = om << (32 - len);
                start = len - __clz(~top);
            }
            int n2, src, ns, ne;
            if (start == end) {
                n2 = len + 1;
                src = lane <= start ? lane : lane - 1;
                ns = start;
                ne = start + 1;
            } else if (start < end) {
                int drop = end - start - 1;
                n2 = len - drop;
                src = lane <= start ? lane : lane + drop;
                ns = start;
                ne = start + 1;
            } else {
                n2 = start - end + 1;
                src = end + lane;
                ns = n2 - 1;
                ne = 0;
            }
            if (n2 > 32) {
                res.overflow = true;
                res.unsure = __any_sync(kFull, d.unsure);
                return res;
            }
            src = src < 0 ? 0 : (src > 31 ? 31 : src);
            Pt<T> r = shfl_pt_flat(q, src);
            if (lane < n2) q = r;
            int il = ns > 0 ? ns - 1 : n2 - 1;
            int ir = ne + 1 < n2 ? ne + 1 : 0;
            Pt<T> nbp = shfl_pt_flat(q, lane == ns ? il : ir);
            if (lane == ns || lane == ne) {
                V3<T> ip;
                if constexpr (F)
                    ip = plane_segment_h(d, PN, PC.x, q.p, nbp.p, e0);
                else
                    ip = plane_segment(d, PC, PN, q.p, nbp.p, 0.0);
                if (lane == ns) {
                    uint32_t old_l = q.lid;
                    q.lid = nbp.rid;
                    q.rid = old_l;
                } else {
                    uint32_t old_r = q.rid;
                    q.lid = old_r;
                    q.rid = nbp.lid;
                }
                q.p = ip;
                q.ang = 0;
            }
            // merge very close points (contact.rs:622-626): lane ns holds the new point ps
            // and takes pe from lane ne
            const V3<T> pe = shfl_v3(q.p, ne);
            bool close = false;
            if (lane == ns) {
                const T dse = norm2(pe - q.p);
                if constexpr (F) {  // merge threshold: d^2 <= 1e-10, i.e. d <= 1e-5
                    if (fabsf(sqrtf(dse) - 1e-5f) <= 4.f * e0) d.unsure = true;
                }
                close = !(dse - (T)kEps > (T)0);
            }
            if (__any_sync(kFull, close)) {
                res.merged = true;
                const uint32_t erid = __shfl_sync(kFull, q.rid, ne);
                if (lane == ns) q.rid = erid;
                int s2 = lane < ne ? lane : lane + 1;
                s2 = s2 > 31 ? 31 : s2;
                Pt<T> r2 = shfl_pt_flat(q, s2);
                if (lane < n2 - 1) q = r2;
                n2 -= 1;
            }
            len = n2;
        }
    }
    if (discarded) {
        res.unsure = __any_sync(kFull, d.unsure);
        return res;
    }

    T sum_arc = 0, area = 0;
    T area_tol = 0;  // FP32: band of the area <= 0 test (an uncut circle is far from it)
    V3<T> bary = mk<T>(0, 0, 0);
    T tri = 0;                     // this lane's triangle (bary, point, next point) area
    V3<T> vnext = mk<T>(0, 0, 0);  // the next point's position
    bool on = false;
    T ang_err = 0;  // FP32: bound on this lane's arc-angle error
    if (!init) {  // contact.rs:311-314
        bary = g.ic.c;
        sum_arc = (T)kTau;
        area = g.ic.r * g.ic.r * (T)kPi;
        len = 0;
    } else {
        // restrict_contour_to_circle (contact.rs:631-769)
        const T r2 = g.ic.r * g.ic.r;
        bool in = true;
        if (lane < len) {
            T dc2 = norm2(q.p - g.ic.c);
            T tol = 0;
            if constexpr (F) tol = 4.f * (sqrtf(dc2) + g.ic.r) * e0;
            in = d.less_eq(dc2, r2, tol);
        }
        unsigned outm = __ballot_sync(kFull, lane < len && !in);
        if (outm != 0) {
            int nx = lane + 1 < len ? lane + 1 : 0;
            Pt<T> v = shfl_pt_pl(q, nx);  // its position and left id are read
            bool v_in = __shfl_sync(kFull, in, nx);
            int k = 0;
            Pt<T> i1, i2;
            i1 = q;
            i2 = q;
            bool mutV = false, mutU = false;
            if (lane < len) {
                if (!in && !v_in) {
                    V3<T> mp, ip1, ip2;
                    bool ok1, ok2, proj;
                    if constexpr (F) {
                        proj = project_inside_line_e(d, g.ic.c, q.p, v.p, e0, &mp);
                        if (proj) {
                            float dm = norm2(mp - g.ic.c);
                            proj = d.less_eq(dm, r2, 4.f * (sqrtf(dm) + g.ic.r) * e0);
                        }
                    } else {
                        proj = project_inside_line(d, g.ic.c, q.p, v.p, &mp, 0.0, 0.0) && norm2(mp - g.ic.c) <= r2;
                    }
                    if (proj) {
                        if constexpr (F) {
                            ok1 = segment_circle_e(d, g.ic, mp, q.p, e0, &ip1);
                            ok2 = segment_circle_e(d, g.ic, mp, v.p, e0, &ip2);
                        } else {
                            ok1 = segment_circle(d, g.ic, mp, q.p, &ip1, 0.0, 0.0);
                            ok2 = segment_circle(d, g.ic, mp, v.p, &ip2, 0.0, 0.0);
                        }
                        if (ok1 && ok2) {
                            k = 2;
                            i1.p = ip1;
                            i1.lid = g.a_id;
                            i1.rid = q.rid;
                            i1.ang = 0;
                            i2.p = ip2;
                            i2.lid = v.lid;
                            i2.rid = g.a_id;
                            i2.ang = 0;
                        }
                    }
                } else if (!in) {
                    V3<T> ip;
                    bool ok;
                    if constexpr (F)
                        ok = segment_circle_e(d, g.ic, v.p, q.p, e0, &ip);
                    else
                        ok = segment_circle(d, g.ic, v.p, q.p, &ip, 0.0, 0.0);
                    if (ok) {
                        k = 1;
                        i1.p = ip;
                        i1.lid = g.a_id;
                        i1.rid = q.rid;
                        i1.ang = 0;
                    } else {
                        mutV = true;  // contour[next].{left,right} = (a, contour[i].right)
                    }
                } else if (!v_in) {
                    V3<T> ip;
                    bool ok;
                    if constexpr (F)
                        ok = segment_circle_e(d, g.ic, q.p, v.p, e0, &ip);
                    else
                        ok = segment_circle(d, g.ic, q.p, v.p, &ip, 0.0, 0.0);
                    if (ok) {
                        k = 1;
                        i1.p = ip;
                        i1.lid = v.lid;
                        i1.rid = g.a_id;
                        i1.ang = 0;
                    } else {
                        mutU = true;  // contour[i].{left,right} = (contour[next].left, a)
                    }
                }
            }
            int insertions = __reduce_add_sync(kFull, (unsigned)k);
            if (insertions == 0) {
                res.unsure = __any_sync(kFull, d.unsure);
                return res;  // contour cleared -> area 0 -> None
            }
            // id mutations of inside points: W1 from the previous segment, W2 from own.
            int pv = lane > 0 ? lane - 1 : len - 1;
            bool w1 = __shfl_sync(kFull, mutV, pv);
            uint32_t w1_rid = __shfl_sync(kFull, q.rid, pv);
            uint32_t w2_lid = v.lid;
            if (lane < len && in) {
                if (lane == 0) {  // for point 0 the wrap segment writes last
                    if (w1) {
                        q.lid = g.a_id;
                        q.rid = w1_rid;
                    } else if (mutU) {
                        q.lid = w2_lid;
                        q.rid = g.a_id;
                    }
                } else {
                    if (mutU) {
                        q.lid = w2_lid;
                        q.rid = g.a_id;
                    } else if (w1) {
                        q.lid = g.a_id;
                        q.rid = w1_rid;
                    }
                }
            }
            int c = lane < len ? (in ? 1 : 0) + k : 0;
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += t;
            }
            int L = __shfl_sync(kFull, incl, 31);
            int pos = incl - c;
            if (L < 2) {
                res.unsure = __any_sync(kFull, d.unsure);
                return res;
            }
            if (L > 32) {
                res.overflow = true;
                res.unsure = __any_sync(kFull, d.unsure);
                return res;
            }
            // output slot `lane` comes from the first segment j with incl[j] > lane
            int j = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                int t = __shfl_sync(kFull, incl, j + step - 1);
                if (t <= lane) j += step;
            }
            j = j > 31 ? 31 : j;
            int s = __shfl_sync(kFull, pos, j);
            int off = lane - s;
            Pt<T> sp = shfl_pt_flat(q, j);
            Pt<T> s1 = shfl_pt_flat(i1, j);
            Pt<T> s2 = shfl_pt_flat(i2, j);
            bool sin_ = __shfl_sync(kFull, in, j);
            Pt<T> outp = off == 0 ? (sin_ ? sp : s1) : (off == 1 ? (sin_ ? s1 : s2) : s2);
            if (lane < L) q = outp;
            len = L;
            // arc angles (contact.rs:741-754)
            int nx2 = lane + 1 < len ? lane + 1 : 0;
            Pt<T> v2 = shfl_pt_pl(q, nx2);
            T a = 0;
            if (lane < len && q.rid == g.a_id && v2.lid == g.a_id) {
                T tol_dir = 0;
                if constexpr (F) {
                    tol_dir = 4.f * e0 / fmaxf(g.ic.r, 1e-12f) + 8.f * kF32Eps;
                    ang_err = tol_dir;
                }
                a = directed_angle(d, g.ic.c, q.p, v2.p, g.ic.c + g.axis, tol_dir);
            }
            q.ang = a;
            sum_arc = lsum(a, len);
            // full circle after all (contact.rs:765-768): contour cleared, area stays 0
            T sum_err = 0;
            if constexpr (F) sum_err = wsum(ang_err) + 1e-5f;
            if (d.ge(sum_arc, (T)kTau, sum_err) || (len > 2 && d.eq(sum_arc, (T)kTau, sum_err))) {
                res.unsure = __any_sync(kFull, d.unsure);
                return res;
            }
        }
        int nx = lane + 1 < len ? lane + 1 : 0;
        Pt<T> v;
        v.p = shfl_v3(q.p, nx);  // the next point's position only
        // calculate_contour_area (contact.rs:773-793)
        on = lane < len;
        V3<T> pp = on ? q.p : mk<T>(0, 0, 0);
        bary = mk<T>(lsum(pp.x, len), lsum(pp.y, len), lsum(pp.z, len)) / (T)len;
        T t = 0, t2 = 0;
        if (on) {
            t = triangle_area(bary, q.p, v.p);
            if (q.ang > (T)0) t2 = g.ic.r * g.ic.r * (q.ang - sin(q.ang)) * (T)0.5;
        }
        area = lsum2(t, t2, len);
        tri = t;
        vnext = v.p;
        if constexpr (F) {
            // moving each vertex by at most |d| changes the polygon area by at most |d| times
            // the perimeter and an arc segment by at most 2 r |d|: the band of area <= 0
            // is 4 E (perimeter + 2 r per arc), E the point error budget
            T side = on ? norm(v.p - q.p) + (q.ang > (T)0 ? (T)2 * g.ic.r : (T)0) : (T)0;
            area_tol = 4.f * e0 * wsum(side);
        }
    }
    // area <= 0 -> None (contact.rs:329-331)
    bool area_none = d.less_eq(area, (T)0, area_tol);
    if (area_none) {
        res.unsure = __any_sync(kFull, d.unsure);
        return res;
    }

    // contour_is_central (contact.rs:411-444)
    bool central;
    {
        const T fe = (T)1e-10;
        bool reflex = on && d.greater(q.ang - fe, (T)kPi, ang_err);
        if (__any_sync(kFull, reflex)) {
            central = true;
        } else {
            bool bad = false;
            int nx = lane + 1 < len ? lane + 1 : 0;
            V3<T> pj = shfl_v3(q.p, nx);
            if (on) {
                V3<T> edge = pj - q.p;
                T el = norm(edge);
                T eerr = 0;
                if constexpr (F) {
                    eerr = 4.f * e0;
                }
                if (!d.less(el, fe, eerr)) {
                    V3<T> u = edge / el;
                    V3<T> foot = q.p + u * dot(u, bary - q.p);
                    V3<T> nbv = bary - foot;
                    V3<T> cp = g.ic.c - q.p;
                    T tol = 0;
                    if constexpr (F)
                        tol = 4.f * e0 * (norm(nbv) + norm(cp)) * (1.f + 2.f * norm(bary - q.p) / fmaxf(el, 1e-12f));
                    bad = d.less(dot(nbv, cp), (T)0, tol);
                }
            }
            central = !__any_sync(kFull, bad);
        }
    }

    res.valid = true;
    res.area = (double)area;
    res.arc = (double)(sum_arc * g.ic.r);
    res.central = central;
    if (co) {
        co->q = q;
        co->len = len;
        co->full = !init;
        co->unsure = __any_sync(kFull, d.unsure);
        co->ic = g.ic;
        co->axis = g.axis;
    }
    rec(q, len, !init, __any_sync(kFull, d.unsure), res);
    if (FULL) {
        // the moments first: they need the contour, its area and its triangles but not
        // the solid angles, whose code then runs without them in registers
        if (XM && g.xm_out) {
            // integral of (x - a) over the arcs: an arc of angle t from e1 (unit, from the
            // circle centre) around the axis contributes (q - a) rho t + rho^2 (sin t e1 +
            // (1 - cos t) axis x e1), with cos t = e1.e2, sin t = e2.(axis x e1).
            // integral of (x - a) over the area: the triangles (bary, p_k, p_k+1) of the
            // area sum contribute their area times their centroid; the circular segment of
            // an arc its area rho^2 (t - sin t) / 2 at q plus rho^3 (1 - cos t) / 6 (sin t e1
            // + (1 - cos t) axis x e1) (the segment's centroid lies 4 rho sin^3(t/2) /
            // (3 (t - sin t)) from q along the arc's bisector); sin t and cos t come from the
            // arc's end points, as for the arcs' moment
            // Formed in the contour's own precision (the FP32 kernel's coordinates are
            // relative to a, so the moments carry no large offsets), one lane per contour
            // point, then summed over the warp and widened.
            const T rho = g.ic.r;
            const V3<T> qa = g.ic.c - g.A.c;
            V3<T> xk = mk<T>(0, 0, 0), ak = mk<T>(0, 0, 0);
            if (!init) {
                if (lane == 0) {
                    xk = qa * ((T)kTau * rho);
                    ak = qa * area;
                }
            } else if (on) {
                // the triangle's area is the one the contour area summed
                const V3<T> bw = bary - g.A.c, pk = q.p - g.A.c, pn = vnext - g.A.c;
                ak = (bw + pk + pn) * (tri / (T)3);
                if (q.ang > (T)0 && rho > (T)0) {
                    const T ir = (T)1 / rho;
                    const V3<T> e1 = (q.p - g.ic.c) * ir, e2 = (vnext - g.ic.c) * ir;
                    const V3<T> f = cross(g.axis, e1);
                    const T ct = dot(e2, e1), st = dot(e2, f);
                    const V3<T> m = e1 * st + f * ((T)1 - ct);
                    xk = qa * (rho * q.ang) + m * (rho * rho);
                    ak = ak + qa * ((T)0.5 * rho * rho * (q.ang - st)) + m * (rho * rho * rho * ((T)1 - ct) / (T)6);
                }
            }
            const T s0 = wsum(xk.x), s1 = wsum(xk.y), s2 = wsum(xk.z);
            const T s3 = wsum(ak.x), s4 = wsum(ak.y), s5 = wsum(ak.z);
            if (lane == 0) {
                g.xm_out[0] = (double)s0;
                g.xm_out[1] = (double)s1;
                g.xm_out[2] = (double)s2;
                g.xm_out[3] = (double)s3;
                g.xm_out[4] = (double)s4;
                g.xm_out[5] = (double)s5;
            }
        }
        // construct_contact_descriptor (contact.rs:357-381)
        int pvl = lane > 0 ? lane - 1 : (len > 0 ? len - 1 : 0);
        int nxl = len > 0 ? (lane + 1 < len ? lane + 1 : 0) : 0;
        // the neighbouring points of the FP64 solid angles (position and arc angle of the
        // previous, position of the next)
        Pt<T> p0 = q, p2 = q;
        if constexpr (!F) p0 = shfl_pt_pa(q, pvl);
        if constexpr (!F) p2.p = shfl_v3(q.p, nxl);
        const T ea0 = 0;
        // one inlined copy of the solid angle for both sides.  FP64: side a, then side b.
        // FP32: a contour of at most 16 points (almost all) computes both sides at once,
        // lanes 0-15 side a and lanes 16-31 side b on the same points; longer ones take two
        // passes with a lane per point.
        double sab[2];
        if constexpr (F) {
            const int split = len <= 16 ? 1 : 0;
#pragma unroll 1
            for (int pass = 0; pass < 2 - split; ++pass) {
                const int side = split ? (lane >> 4) : pass;
                const int L = split ? (lane & 15) : lane;
                const int pv = L > 0 ? L - 1 : (len > 0 ? len - 1 : 0);
                const int nx = len > 0 ? (L + 1 < len ? L + 1 : 0) : 0;
                const Pt<T> m1 = shfl_pt_pa(q, L), m0 = shfl_pt_pa(q, pv);
                Pt<T> m2 = m1;
                m2.p = shfl_v3(q.p, nx);
                const T e1 = __shfl_sync(kFull, ang_err, L), em = __shfl_sync(kFull, ang_err, pv);
                const Sph<T> s0 = side ? g.B : g.A, s1 = side ? g.A : g.B;
                const double v = solid_angle(d, s0, s1, g.ic, m0, m1, m2, L < len, len, e0, em, e1, split);
                if (split) {
                    sab[0] = __shfl_sync(kFull, v, 0);
                    sab[1] = __shfl_sync(kFull, v, 16);
                } else {
                    sab[pass] = v;
                }
            }
        } else {
#pragma unroll 1
            for (int side = 0; side < 2; ++side) {
                const Sph<T> s0 = side ? g.B : g.A, s1 = side ? g.A : g.B;
                sab[side] = solid_angle(d, s0, s1, g.ic, p0, q, p2, on, len, e0, ea0, ang_err);
            }
        }
        const double sa = sab[0], sb = sab[1];
        T sign_a = sa < 0.0 ? (T)-1 : (T)1;
        T sign_b = sb < 0.0 ? (T)-1 : (T)1;
        res.sa_a = sa;
        res.sa_b = sb;
        if constexpr (F) {
            res.pv_a = (double)norm_rn(g.ic.c - g.A.c) * (double)area / 3.0 * (double)sign_a;
            res.pv_b = (double)norm_rn(g.ic.c - g.B.c) * (double)area / 3.0 * (double)sign_b;
        } else {
            res.pv_a = (double)(norm(g.ic.c - g.A.c) * area / (T)3 * sign_a);
            res.pv_b = (double)(norm(g.ic.c - g.B.c) * area / (T)3 * sign_b);
        }
    }
    res.unsure = __any_sync(kFull, d.unsure);
    return res;
}

}  // namespace vt
