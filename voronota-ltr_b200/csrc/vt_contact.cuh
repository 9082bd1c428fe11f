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
#pragma once
#include "vt_geom.cuh"

namespace vt {

constexpr unsigned kFull = 0xffffffffu;

template <typename T>
__device__ __forceinline__ T wsum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Sum over the first `len` lanes.  FP64 adds in lane order starting from 0.0, exactly as
// the reference's sequential loops (contact.rs:776-790, 804-833, 741-751): some of its
// decisions (the centrality test of near-degenerate contours) compare rounding-noise
// sized quantities with zero, so the FP64 path must reproduce the summation order.  FP32
// uses a butterfly; its decisions near zero are inside the band and go to FP64.
__device__ __forceinline__ double lsum(double v, int len) {
    double acc = 0.0;
    for (int k = 0; k < len; ++k) acc += __shfl_sync(kFull, v, k);
    return acc;
}
__device__ __forceinline__ float lsum(float v, int) { return wsum(v); }
// acc = (acc + u_k) + w_k for k in lane order (two additions per element)
__device__ __forceinline__ double lsum2(double u, double w, int len) {
    double acc = 0.0;
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

// sin and cos of the half rotation angles of init_contour (contact.rs:463-468): the
// angles k pi/3 accumulate by repeated addition exactly as in the reference, and the
// rotation needs sin/cos of angle/2.  The angles do not depend on the data, so the host
// evaluates them once with the C library the CPU oracle uses (set_hex_table) and every
// FP64 contour starts from bit-identical hexagon points.  Entry 0 holds the count.
static __constant__ double c_hex_sin[8];
static __constant__ double c_hex_cos[8];
static __constant__ int c_hex_n[1];

// Hexagon of init_contour (contact.rs:455-469).  FP64: quaternion rotations (the
// accumulated angles give 7 points, the 7th 8.9e-16 rad short of a full turn).  FP32:
// the same 7 points from a cos/sin table.
__device__ __forceinline__ int init_contour(Pt<double>& q, int lane, uint32_t a_id, const Sph<double>& ic,
                                            V3<double> axis) {
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
                                            V3<float> axis) {
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
    // FP32 band widths: lengths (k S), squared lengths (k S^2), cubed lengths (k S^3)
    // and dimensionless quantities (k), with S the pair's length scale.
    T tol, tolsq, tol3, tola;
};

// Pre-test classes
enum { kSkip = 0, kDiscard = 1, kCut = 2 };

template <typename T, bool F>
__device__ __forceinline__ int pretest(Dec<T, F>& d, const PairGeom<T>& g, const Sph<T>& c, V3<T>& pc, V3<T>& pn) {
    // contact.rs:236-282
    if (!sphere_intersects(d, g.ic, c, g.tolsq) || !sphere_intersects(d, g.B, c, g.tolsq)) return kSkip;
    if (sphere_contains(d, c, g.A, g.tol, g.tolsq) || sphere_contains(d, c, g.B, g.tol, g.tolsq)) return kDiscard;
    pc = ic_center(g.A, c);
    pn = normalize(c.c - g.A.c);
    T cos_val = dot(normalize(g.ic.c - g.A.c), normalize(pc - g.A.c));
    if (d.greater_eq(fabs(cos_val), (T)1, g.tola)) {
        return halfspace(d, pc, pn, g.ic.c, g.tol) > 0 ? kDiscard : kSkip;
    }
    T l = fabs(sd_plane_unit(pc, pn, g.ic.c));
    T xl = l / sqrt(fma(cos_val, -cos_val, (T)1));
    if (d.greater_eq(xl, g.ic.r, g.tol)) {
        return halfspace(d, pc, pn, g.ic.c, g.tol) >= 0 ? kDiscard : kSkip;
    }
    return kCut;
}

// Result of the warp computation (uniform across lanes).
struct WarpContact {
    bool valid;
    bool unsure;
    bool overflow;
    double area, arc, sa_a, sa_b, pv_a, pv_b;
    bool central;
};

// Solid angle (contact.rs:797-848) summed over the warp's contour.
template <typename T, bool F>
__device__ __forceinline__ T solid_angle(Dec<T, F>& d, const Sph<T>& a, const Sph<T>& b, const Sph<T>& ic,
                                         const Pt<T>& p0, const Pt<T>& p1, const Pt<T>& p2, bool on, int len,
                                         T tolsq, T tol3, T tola) {
    T turn = 0;
    if (len == 0) {
        turn = (T)kTau * norm(ic.c - a.c) / a.r;
    } else {
        T t = 0, t2 = 0;
        if (on) {
            const T pi = (T)kPi;
            if (p0.ang > (T)0) {
                V3<T> dd = cross(b.c - a.c, p1.p - ic.c);
                T dv = dot(dd, p0.p - p1.p);
                d.band(p0.ang - pi, tola);
                d.band(dv, tol3);
                bool flip = (p0.ang < pi && dv < (T)0) || (p0.ang > pi && dv > (T)0);
                if (flip) dd = -dd;
                t = pi - min_dihedral(a.c, p1.p, p1.p + dd, p2.p);
            } else if (p1.ang > (T)0) {
                V3<T> dd = cross(b.c - a.c, p1.p - ic.c);
                T dv = dot(dd, p2.p - p1.p);
                d.band(p1.ang - pi, tola);
                d.band(dv, tol3);
                bool flip = (p1.ang < pi && dv < (T)0) || (p1.ang > pi && dv > (T)0);
                if (flip) dd = -dd;
                t = pi - min_dihedral(a.c, p1.p, p0.p, p1.p + dd);
                t2 = p1.ang * (norm(ic.c - a.c) / a.r);
            } else {
                t = pi - min_dihedral(a.c, p1.p, p0.p, p2.p);
            }
        }
        turn = lsum2(t, t2, len);
    }
    T sa = (T)kTau - turn;
    V3<T> ic_to_a = ic.c - a.c, ic_to_b = ic.c - b.c;
    Dec<T, F> d1, d2;
    bool c1 = d1.greater(dot(ic_to_a, ic_to_b), (T)0, tolsq);
    bool c2 = d2.less(norm2(a.c - ic.c), norm2(b.c - ic.c), tolsq);
    if (F && (d1.unsure || d2.unsure) && !((!c1 && !d1.unsure) || (!c2 && !d2.unsure))) d.unsure = true;
    if (c1 && c2) sa = -sa;
    return sa;
}

// The warp-wide contact computation.  `nb(e)` returns neighbour record e of a's sorted
// list (0 <= e < cnt); entry `kb` is b itself.
template <typename T, bool F, bool FULL, typename NbFn>
__device__ WarpContact contact_warp(const PairGeom<T>& g0, int cnt, int kb, NbFn nb) {
    const int lane = threadIdx.x & 31;
    PairGeom<T> g = g0;
    Dec<T, F> d;
    WarpContact res;
    res.valid = false;
    res.unsure = false;
    res.overflow = false;
    res.area = res.arc = res.sa_a = res.sa_b = res.pv_a = res.pv_b = 0.0;
    res.central = false;

    // contact.rs:206-218
    if (!sphere_intersects(d, g.A, g.B, g.tolsq) || sphere_contains(d, g.A, g.B, g.tol, g.tolsq) ||
        sphere_contains(d, g.B, g.A, g.tol, g.tolsq)) {
        res.unsure = __any_sync(kFull, d.unsure);
        return res;
    }
    g.ic = intersection_circle(g.A, g.B);
    g.axis = normalize(g.B.c - g.A.c);
    if (d.less_eq(g.ic.r, (T)0, g.tol)) {
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
        if (__any_sync(kFull, cls == kDiscard)) {
            discarded = true;
            break;
        }
        unsigned cutmask = __ballot_sync(kFull, cls == kCut);
        while (cutmask) {
            int j = __ffs(cutmask) - 1;
            cutmask &= cutmask - 1;
            V3<T> PC = shfl_v3(pc, j), PN = shfl_v3(pn, j);
            uint32_t CID = __shfl_sync(kFull, cid, j);
            if (!init) {
                len = init_contour(q, lane, g.a_id, g.ic, g.axis);
                init = true;
            } else {
                // test_contour_cuttable (contact.rs:472-481)
                T thr = norm2(PC - g.A.c);
                bool cut = lane < len && d.greater_eq(norm2(q.p - g.A.c), thr, g.tolsq);
                if (!__any_sync(kFull, cut)) continue;
            }
            // mark_contour (contact.rs:506-521)
            bool out = lane < len && halfspace(d, PC, PN, q.p, g.tol) >= 0;
            unsigned om = __ballot_sync(kFull, out);
            if (om == 0) continue;
            int nout = __popc(om);
            if (nout >= len) {  // mark_and_cut_contour clears (contact.rs:496-499)
                len = 0;
                discarded = true;
                break;
            }
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
            Pt<T> r = shfl_pt(q, src);
            if (lane < n2) q = r;
            int il = ns > 0 ? ns - 1 : n2 - 1;
            int ir = ne + 1 < n2 ? ne + 1 : 0;
            Pt<T> nbp = shfl_pt(q, lane == ns ? il : ir);
            if (lane == ns) {
                V3<T> ip = plane_segment(d, PC, PN, q.p, nbp.p, g.tol);
                uint32_t old_l = q.lid;
                q.p = ip;
                q.lid = nbp.rid;
                q.rid = old_l;
                q.ang = 0;
            } else if (lane == ne) {
                V3<T> ip = plane_segment(d, PC, PN, q.p, nbp.p, g.tol);
                uint32_t old_r = q.rid;
                q.p = ip;
                q.lid = old_r;
                q.rid = nbp.lid;
                q.ang = 0;
            }
            // merge very close points (contact.rs:622-626)
            V3<T> ps = shfl_v3(q.p, ns), pe = shfl_v3(q.p, ne);
            uint32_t erid = __shfl_sync(kFull, q.rid, ne);
            if (!d.gt(norm2(pe - ps), (T)0, g.tolsq)) {
                if (lane == ns) q.rid = erid;
                int s2 = lane < ne ? lane : lane + 1;
                s2 = s2 > 31 ? 31 : s2;
                Pt<T> r2 = shfl_pt(q, s2);
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
    V3<T> bary = mk<T>(0, 0, 0);
    bool on = false;
    if (!init) {  // contact.rs:311-314
        bary = g.ic.c;
        sum_arc = (T)kTau;
        area = g.ic.r * g.ic.r * (T)kPi;
        len = 0;
    } else {
        // restrict_contour_to_circle (contact.rs:631-769)
        const T r2 = g.ic.r * g.ic.r;
        bool in = true;
        if (lane < len) in = d.less_eq(norm2(q.p - g.ic.c), r2, g.tolsq);
        unsigned outm = __ballot_sync(kFull, lane < len && !in);
        if (outm != 0) {
            int nx = lane + 1 < len ? lane + 1 : 0;
            Pt<T> v = shfl_pt(q, nx);
            bool v_in = __shfl_sync(kFull, in, nx);
            int k = 0;
            Pt<T> i1, i2;
            i1 = q;
            i2 = q;
            bool mutV = false, mutU = false;
            if (lane < len) {
                if (!in && !v_in) {
                    V3<T> mp, ip1, ip2;
                    if (project_inside_line(d, g.ic.c, q.p, v.p, &mp, g.tol, g.tolsq) &&
                        d.less_eq(norm2(mp - g.ic.c), r2, g.tolsq)) {
                        bool ok1 = segment_circle(d, g.ic, mp, q.p, &ip1, g.tol, g.tolsq);
                        bool ok2 = segment_circle(d, g.ic, mp, v.p, &ip2, g.tol, g.tolsq);
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
                    if (segment_circle(d, g.ic, v.p, q.p, &ip, g.tol, g.tolsq)) {
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
                    if (segment_circle(d, g.ic, q.p, v.p, &ip, g.tol, g.tolsq)) {
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
                bool w1_last = (lane == 0);  // for point 0 the wrap segment writes last
                if (w1_last) {
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
            // inclusive warp scan of c
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
            Pt<T> sp = shfl_pt(q, j);
            Pt<T> s1 = shfl_pt(i1, j);
            Pt<T> s2 = shfl_pt(i2, j);
            bool sin_ = __shfl_sync(kFull, in, j);
            Pt<T> outp = off == 0 ? (sin_ ? sp : s1) : (off == 1 ? (sin_ ? s1 : s2) : s2);
            if (lane < L) q = outp;
            len = L;
            // arc angles (contact.rs:741-754)
            int nx2 = lane + 1 < len ? lane + 1 : 0;
            Pt<T> v2 = shfl_pt(q, nx2);
            T a = 0;
            if (lane < len && q.rid == g.a_id && v2.lid == g.a_id)
                a = directed_angle(d, g.ic.c, q.p, v2.p, g.ic.c + g.axis, g.tola);
            q.ang = a;
            sum_arc = lsum(a, len);
            // full circle after all (contact.rs:765-768): contour cleared, area stays 0
            if (d.ge(sum_arc, (T)kTau, g.tola) || (len > 2 && d.eq(sum_arc, (T)kTau, g.tola))) {
                res.unsure = __any_sync(kFull, d.unsure);
                return res;
            }
        }
        int nx = lane + 1 < len ? lane + 1 : 0;
        Pt<T> v = shfl_pt(q, nx);
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
    }
    // area <= 0 -> None (contact.rs:329-331)
    if (d.less_eq(area, (T)0, g.tolsq)) {
        res.unsure = __any_sync(kFull, d.unsure);
        return res;
    }

    // contour_is_central (contact.rs:411-444)
    bool central;
    {
        const T fe = (T)1e-10;
        bool reflex = on && d.greater(q.ang - fe, (T)kPi, g.tola);
        if (__any_sync(kFull, reflex)) {
            central = true;
        } else {
            bool bad = false;
            int nx = lane + 1 < len ? lane + 1 : 0;
            V3<T> pj = shfl_v3(q.p, nx);
            if (on) {
                V3<T> edge = pj - q.p;
                T el = norm(edge);
                if (!d.less(el, fe, g.tol)) {
                    V3<T> u = edge / el;
                    V3<T> foot = q.p + u * dot(u, bary - q.p);
                    V3<T> nbv = bary - foot;
                    bad = d.less(dot(nbv, g.ic.c - q.p), (T)0, g.tolsq);
                }
            }
            central = !__any_sync(kFull, bad);
        }
    }

    res.valid = true;
    res.area = (double)area;
    res.arc = (double)(sum_arc * g.ic.r);
    res.central = central;
    if (FULL) {
        // construct_contact_descriptor (contact.rs:357-381)
        int pvl = lane > 0 ? lane - 1 : (len > 0 ? len - 1 : 0);
        int nxl = len > 0 ? (lane + 1 < len ? lane + 1 : 0) : 0;
        Pt<T> p0 = shfl_pt(q, pvl);
        Pt<T> p2 = shfl_pt(q, nxl);
        T sa = solid_angle(d, g.A, g.B, g.ic, p0, q, p2, on, len, g.tolsq, g.tol3, g.tola);
        T sb = solid_angle(d, g.B, g.A, g.ic, p0, q, p2, on, len, g.tolsq, g.tol3, g.tola);
        d.band(sa, g.tola);
        d.band(sb, g.tola);
        T sign_a = sa < (T)0 ? (T)-1 : (T)1;
        T sign_b = sb < (T)0 ? (T)-1 : (T)1;
        res.sa_a = (double)sa;
        res.sa_b = (double)sb;
        res.pv_a = (double)(norm(g.ic.c - g.A.c) * area / (T)3 * sign_a);
        res.pv_b = (double)(norm(g.ic.c - g.B.c) * area / (T)3 * sign_b);
    }
    res.unsure = __any_sync(kFull, d.unsure);
    return res;
}

}  // namespace vt
