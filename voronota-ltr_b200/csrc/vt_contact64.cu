// vt_contact64.cu -- FP64 contact kernels (compiled with --fmad=false).
//   k_contact64      one warp per pair, exact reference arithmetic; over all pairs (plain
//                    FP64 path) or over the pairs the FP32 kernel flagged as unsure.
//   k_contact_serial one thread per pair whose contour outgrew a warp (32 points); the
//                    contour lives in a per-thread slice of a global scratch buffer.
#include <cmath>

#include "vt_adjoint.cuh"
#include "vt_contact.cuh"
#include "vt_pipeline.cuh"

namespace vt {

namespace {

constexpr int kWarps = 4;

__device__ __forceinline__ Sph<double> sph_of(double4 v) { return {{v.x, v.y, v.z}, v.w}; }

__device__ __forceinline__ void write_pair(const DevBufs& b, uint32_t p, const WarpContact& r, uint8_t extra) {
    b.p_status[p] = (r.valid ? kValid : 0) | extra;
    b.p_area[p] = r.valid ? r.area : 0.0;
    b.p_arc[p] = r.valid ? r.arc : 0.0;
    b.p_central[p] = r.valid && r.central ? 1 : 0;
    b.p_sa_a[p] = r.valid ? r.sa_a : 0.0;
    b.p_sa_b[p] = r.valid ? r.sa_b : 0.0;
    b.p_pv_a[p] = r.valid ? r.pv_a : 0.0;
    b.p_pv_b[p] = r.valid ? r.pv_b : 0.0;
}

// 4 resident blocks per SM: at most 128 registers a thread (a few bytes of spill) for 16
// warps per SM, against 12 at the 150 registers the kernel would take.  XM: compile in the
// arc first moments (only when the caller records them).
template <bool FULL, bool XM>
__global__ void __launch_bounds__(kWarps * 32, 4) k_contact64(DevBufs b, uint32_t P, int from_list) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t count = from_list ? *b.d_redo_count : P;
    for (uint32_t it = blockIdx.x * kWarps + w; it < count; it += gridDim.x * kWarps) {
        const uint32_t p = from_list ? b.redo_list[it] : it;
        const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
        const uint32_t off = b.nb_off[a], cnt = b.nb_cnt[a];
        PairGeom<double> g;
        g.A = sph_of(b.sph[a]);
        g.B = sph_of(b.sph[b.nb_slot[eb]]);
        g.a_id = a;
        g.b_id = b.nb_id[eb];
        g.e0 = 0.0;
        g.S = g.A.r + g.B.r;
        if (XM && b.p_arcm) g.xm_out = b.p_arcm + 6 * (size_t)p;
        const double4* sph = b.sph;
        const uint32_t* nslot = b.nb_slot + off;
        const uint32_t* nid = b.nb_id + off;
        auto nbf = [&](int e) {
            Nb<double> r;
            r.s = sph_of(sph[nslot[e]]);
            r.id = nid[e];
            return r;
        };
        WarpContact r = contact_warp<double, false, FULL, XM>(g, (int)cnt, (int)(eb - off), nbf);
        if (lane == 0) write_pair(b, p, r, r.overflow ? kOverflow : 0);
    }
}

// ---------------------------------------------------------------------------------------
// Serial fallback: clip_contact and the descriptor for one pair per thread, with the
// contour in global scratch (kSerialCap points).  Same arithmetic as the warp kernel.
struct SP {
    double x, y, z, ang;
    uint32_t lid, rid;
    int state;  // 0 inside, 1 outside, 2 arc start
};

struct Contour {
    SP* v;
    int n;
    int cap;
    bool overflow;
    __device__ void insert(int at, const SP& s) {
        if (n >= cap) {
            overflow = true;
            return;
        }
        for (int k = n; k > at; --k) v[k] = v[k - 1];
        v[at] = s;
        ++n;
    }
    __device__ void erase(int from, int to) {  // [from, to)
        int d = to - from;
        if (d <= 0) return;
        for (int k = from; k + d < n; ++k) v[k] = v[k + d];
        n -= d;
    }
};
__device__ __forceinline__ V3<double> P3(const SP& s) { return {s.x, s.y, s.z}; }
__device__ __forceinline__ SP mkp(V3<double> p, uint32_t l, uint32_t r) {
    SP s;
    s.x = p.x;
    s.y = p.y;
    s.z = p.z;
    s.ang = 0.0;
    s.lid = l;
    s.rid = r;
    s.state = 0;
    return s;
}

__device__ bool serial_clip(const DevBufs& b, uint32_t p, Contour& c, Sph<double>& ic_out, V3<double>& axis_out,
                            V3<double>& bary, double& sum_arc, double& area) {
    Dec<double, false> d;
    const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
    const uint32_t off = b.nb_off[a], cnt = b.nb_cnt[a];
    const Sph<double> A = sph_of(b.sph[a]);
    const Sph<double> B = sph_of(b.sph[b.nb_slot[eb]]);
    const uint32_t a_id = a, b_id = b.nb_id[eb];
    if (!sphere_intersects(d, A, B, 0.0) || sphere_contains(d, A, B, 0.0, 0.0) || sphere_contains(d, B, A, 0.0, 0.0))
        return false;
    Sph<double> ic = intersection_circle(A, B);
    V3<double> axis = normalize(B.c - A.c);
    ic_out = ic;
    axis_out = axis;
    if (ic.r <= 0.0) return false;
    c.n = 0;
    bool init = false;
    for (uint32_t e = 0; e < cnt; ++e) {
        uint32_t nid = b.nb_id[off + e];
        if (nid == b_id) continue;
        Sph<double> C = sph_of(b.sph[b.nb_slot[off + e]]);
        if (!sphere_intersects(d, ic, C, 0.0) || !sphere_intersects(d, B, C, 0.0)) continue;
        if (sphere_contains(d, C, A, 0.0, 0.0) || sphere_contains(d, C, B, 0.0, 0.0)) return false;
        V3<double> pc = ic_center(A, C);
        V3<double> pn = normalize(C.c - A.c);
        double cos_val = dot(normalize(ic.c - A.c), normalize(pc - A.c));
        if (fabs(cos_val) >= 1.0) {
            if (halfspace(d, pc, pn, ic.c, 0.0) > 0) return false;
            continue;
        }
        double l = fabs(sd_plane_unit(pc, pn, ic.c));
        double xl = l / sqrt(fma(cos_val, -cos_val, 1.0));
        if (xl >= ic.r) {
            if (halfspace(d, pc, pn, ic.c, 0.0) >= 0) return false;
            continue;
        }
        if (!init) {  // init_contour
            V3<double> first = any_normal(axis) * ic.r * kHexScale;
            c.n = 0;
            c.v[c.n++] = mkp(ic.c + first, a_id, a_id);
            for (int k = 1; k < c_hex_n[0]; ++k)
                c.insert(c.n, mkp(ic.c + rotate_around_axis(axis, c_hex_sin[k], c_hex_cos[k], first), a_id, a_id));
            init = true;
        } else {  // test_contour_cuttable
            double thr = norm2(pc - A.c);
            bool any = false;
            for (int k = 0; k < c.n; ++k)
                if (norm2(P3(c.v[k]) - A.c) >= thr) {
                    any = true;
                    break;
                }
            if (!any) continue;
        }
        // mark_contour
        int outs = 0;
        for (int k = 0; k < c.n; ++k)
            if (halfspace(d, pc, pn, P3(c.v[k]), 0.0) >= 0) {
                c.v[k].lid = c.v[k].rid = nid;
                ++outs;
            }
        if (outs == 0) continue;
        if (outs >= c.n) return false;  // cleared -> discarded
        if (c.n < 3) continue;
        auto is_out = [&](int k) { return c.v[k].lid == nid && c.v[k].rid == nid; };
        int start = -1, end = -1;
        for (int k = 0; k < c.n; ++k)
            if (is_out(k)) {
                start = k;
                break;
            }
        for (int k = c.n - 1; k >= 0; --k)
            if (is_out(k)) {
                end = k;
                break;
            }
        if (start == 0 && end == c.n - 1) {
            end = 0;
            while (end + 1 < c.n && is_out(end + 1)) ++end;
            start = c.n - 1;
            while (start > 0 && is_out(start - 1)) --start;
        }
        if (start == end) {
            SP cp = c.v[start];
            c.insert(start, cp);
            end = start + 1;
        } else if (start < end) {
            if (start + 1 < end) c.erase(start + 1, end);
            end = start + 1;
        } else {
            if (start + 1 < c.n) c.erase(start + 1, c.n);
            if (end > 0) c.erase(0, end);
            start = c.n - 1;
            end = 0;
        }
        if (c.overflow) return false;
        int nn = c.n;
        int il = start > 0 ? start - 1 : nn - 1;
        V3<double> lip = plane_segment(d, pc, pn, P3(c.v[start]), P3(c.v[il]), 0.0);
        SP ns = mkp(lip, c.v[il].rid, c.v[start].lid);
        c.v[start] = ns;
        int ir = end + 1 < nn ? end + 1 : 0;
        V3<double> rip = plane_segment(d, pc, pn, P3(c.v[end]), P3(c.v[ir]), 0.0);
        SP ne = mkp(rip, c.v[end].rid, c.v[ir].lid);
        c.v[end] = ne;
        if (!(norm2(P3(c.v[end]) - P3(c.v[start])) - kEps > 0.0)) {
            c.v[start].rid = c.v[end].rid;
            c.erase(end, end + 1);
        }
    }
    sum_arc = 0.0;
    area = 0.0;
    bary = mk<double>(0, 0, 0);
    if (!init) {
        bary = ic.c;
        sum_arc = kTau;
        area = ic.r * ic.r * kPi;
        c.n = 0;
        return area > 0.0;
    }
    // restrict_contour_to_circle
    int outsiders = 0;
    for (int k = 0; k < c.n; ++k) {
        if (norm2(P3(c.v[k]) - ic.c) <= ic.r * ic.r) {
            c.v[k].state = 0;
        } else {
            c.v[k].state = 1;
            ++outsiders;
        }
    }
    if (outsiders > 0) {
        int insertions = 0;
        int i = 0;
        while (i < c.n) {
            int ni = (i + 1) % c.n;
            int s1 = c.v[i].state, s2 = c.v[ni].state;
            if (s1 == 1 || s2 == 1) {
                if (s1 == 1 && s2 == 1) {
                    V3<double> mp, ip1, ip2;
                    if (project_inside_line(d, ic.c, P3(c.v[i]), P3(c.v[ni]), &mp, 0.0, 0.0) &&
                        norm2(mp - ic.c) <= ic.r * ic.r) {
                        bool ok1 = segment_circle(d, ic, mp, P3(c.v[i]), &ip1, 0.0, 0.0);
                        bool ok2 = segment_circle(d, ic, mp, P3(c.v[ni]), &ip2, 0.0, 0.0);
                        if (ok1 && ok2) {
                            uint32_t rid = c.v[i].rid, lid = c.v[ni].lid;
                            c.insert(i + 1, mkp(ip1, a_id, rid));
                            c.insert(i + 2, mkp(ip2, lid, a_id));
                            insertions += 2;
                            i += 2;
                        }
                    }
                } else if (s1 == 1) {
                    V3<double> ip;
                    if (segment_circle(d, ic, P3(c.v[ni]), P3(c.v[i]), &ip, 0.0, 0.0)) {
                        uint32_t rid = c.v[i].rid;
                        c.insert(i + 1, mkp(ip, a_id, rid));
                        insertions += 1;
                        i += 1;
                    } else {
                        c.v[ni].lid = a_id;
                        c.v[ni].rid = c.v[i].rid;
                    }
                } else {
                    V3<double> ip;
                    if (segment_circle(d, ic, P3(c.v[i]), P3(c.v[ni]), &ip, 0.0, 0.0)) {
                        uint32_t lid = c.v[ni].lid;
                        c.insert(i + 1, mkp(ip, lid, a_id));
                        insertions += 1;
                        i += 1;
                    } else {
                        c.v[i].lid = c.v[ni].lid;
                        c.v[i].rid = a_id;
                    }
                }
                if (c.overflow) return false;
            }
            i += 1;
        }
        if (insertions == 0) return false;
        int m = 0;
        for (int k = 0; k < c.n; ++k)
            if (c.v[k].state != 1) c.v[m++] = c.v[k];
        c.n = m;
        if (c.n < 2) return false;
        for (int k = 0; k < c.n; ++k) {
            int nk = (k + 1) % c.n;
            if (c.v[k].rid == a_id && c.v[nk].lid == a_id) {
                double ang = directed_angle(d, ic.c, P3(c.v[k]), P3(c.v[nk]), ic.c + axis, 0.0);
                c.v[k].ang = ang;
                sum_arc += ang;
            }
        }
        if (sum_arc + kEps > kTau || (c.n > 2 && fabs(sum_arc - kTau) <= kEps)) return false;
    }
    // calculate_contour_area
    V3<double> s = mk<double>(0, 0, 0);
    for (int k = 0; k < c.n; ++k) s = s + P3(c.v[k]);
    bary = s / (double)c.n;
    for (int k = 0; k < c.n; ++k) {
        int nk = (k + 1) % c.n;
        area += triangle_area(bary, P3(c.v[k]), P3(c.v[nk]));
        if (c.v[k].ang > 0.0) area += ic.r * ic.r * (c.v[k].ang - sin(c.v[k].ang)) * 0.5;
    }
    return area > 0.0;
}

__device__ double serial_solid_angle(const Sph<double>& a, const Sph<double>& b, const Sph<double>& ic,
                                     const Contour& c) {
    double turn = 0.0;
    if (c.n == 0) {
        turn = kTau * norm(ic.c - a.c) / a.r;
    } else {
        for (int i = 0; i < c.n; ++i) {
            const SP& p0 = c.v[i > 0 ? i - 1 : c.n - 1];
            const SP& p1 = c.v[i];
            const SP& p2 = c.v[(i + 1) % c.n];
            if (p0.ang > 0.0) {
                V3<double> dd = cross(b.c - a.c, P3(p1) - ic.c);
                double dv = dot(dd, P3(p0) - P3(p1));
                if ((p0.ang < kPi && dv < 0.0) || (p0.ang > kPi && dv > 0.0)) dd = -dd;
                turn += kPi - min_dihedral(a.c, P3(p1), P3(p1) + dd, P3(p2));
            } else if (p1.ang > 0.0) {
                V3<double> dd = cross(b.c - a.c, P3(p1) - ic.c);
                double dv = dot(dd, P3(p2) - P3(p1));
                if ((p1.ang < kPi && dv < 0.0) || (p1.ang > kPi && dv > 0.0)) dd = -dd;
                turn += kPi - min_dihedral(a.c, P3(p1), P3(p0), P3(p1) + dd);
                turn += p1.ang * (norm(ic.c - a.c) / a.r);
            } else {
                turn += kPi - min_dihedral(a.c, P3(p1), P3(p0), P3(p2));
            }
        }
    }
    double sa = kTau - turn;
    V3<double> ta = ic.c - a.c, tb = ic.c - b.c;
    if (dot(ta, tb) > 0.0 && norm2(a.c - ic.c) < norm2(b.c - ic.c)) sa = -sa;
    return sa;
}

__device__ bool serial_central(V3<double> center, const Contour& c, V3<double> bary) {
    for (int k = 0; k < c.n; ++k)
        if (c.v[k].ang - 1e-10 > kPi) return true;
    for (int i = 0; i < c.n; ++i) {
        V3<double> pi = P3(c.v[i]), pj = P3(c.v[(i + 1) % c.n]);
        V3<double> edge = pj - pi;
        double len = norm(edge);
        if (len < 1e-10) continue;
        V3<double> u = edge / len;
        V3<double> foot = pi + u * dot(u, bary - pi);
        if (dot(bary - foot, center - pi) < 0.0) return false;
    }
    return true;
}

__global__ void k_contact_serial(DevBufs b, int full) {
    const uint32_t count = *b.d_serial_count;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
        if (slot >= b.serial_slots) break;
        const uint32_t p = b.serial_list[t];
        Contour c;
        c.v = reinterpret_cast<SP*>(b.serial_scratch) + (size_t)slot * kSerialCap;
        c.n = 0;
        c.cap = kSerialCap;
        c.overflow = false;
        Sph<double> ic;
        V3<double> axis, bary;
        double sum_arc, area;
        bool ok = serial_clip(b, p, c, ic, axis, bary, sum_arc, area);
        WarpContact r;
        r.valid = ok && !c.overflow;
        r.unsure = false;
        r.overflow = c.overflow;
        r.area = area;
        r.arc = sum_arc * ic.r;
        r.central = r.valid ? serial_central(ic.c, c, bary) : false;
        r.sa_a = r.sa_b = r.pv_a = r.pv_b = 0.0;
        for (int k = 0; k < 6; ++k) r.xm[k] = 0.0;
        if (r.valid && full && b.p_arcm) {  // first moments of the arcs and of the area about a
            const V3<double> pa = sph_of(b.sph[b.pair_a[p]]).c;
            const V3<double> qa = ic.c - pa;
            V3<double> X = mk<double>(0, 0, 0), M = mk<double>(0, 0, 0);
            if (c.n == 0) {
                X = qa * (kTau * ic.r);
                M = qa * area;
            } else {
                const double rho = ic.r;
                for (int k = 0; k < c.n; ++k) {
                    const V3<double> pk = P3(c.v[k]) - pa, pn = P3(c.v[(k + 1) % c.n]) - pa, bw = bary - pa;
                    M = M + (bw + pk + pn) * (0.5 * norm(cross(pk - bw, pn - bw)) / 3.0);
                    if (!(c.v[k].ang > 0.0)) continue;
                    const V3<double> e1 = (P3(c.v[k]) - ic.c) / rho, e2 = (P3(c.v[(k + 1) % c.n]) - ic.c) / rho;
                    const V3<double> f = cross(axis, e1);
                    const double ct = dot(e2, e1), st = dot(e2, f), th = c.v[k].ang;
                    const V3<double> m = e1 * st + f * (1.0 - ct);
                    X = X + qa * (rho * th) + m * (rho * rho);
                    M = M + qa * (0.5 * rho * rho * (th - st)) + m * (rho * rho * rho * (1.0 - ct) / 6.0);
                }
            }
            r.xm[0] = X.x;
            r.xm[1] = X.y;
            r.xm[2] = X.z;
            r.xm[3] = M.x;
            r.xm[4] = M.y;
            r.xm[5] = M.z;
        }
        if (r.valid && full) {
            const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
            const Sph<double> A = sph_of(b.sph[a]);
            const Sph<double> B = sph_of(b.sph[b.nb_slot[eb]]);
            r.sa_a = serial_solid_angle(A, B, ic, c);
            r.sa_b = serial_solid_angle(B, A, ic, c);
            double sign_a = r.sa_a < 0.0 ? -1.0 : 1.0, sign_b = r.sa_b < 0.0 ? -1.0 : 1.0;
            r.pv_a = norm(ic.c - A.c) * area / 3.0 * sign_a;
            r.pv_b = norm(ic.c - B.c) * area / 3.0 * sign_b;
        }
        if (c.overflow) atomicOr(b.err, (uint32_t)kErrOverflow);
        write_pair(b, p, r, 0);
        if (full && b.p_arcm)
            for (int k = 0; k < 6; ++k) b.p_arcm[6 * (size_t)p + k] = r.xm[k];
    }
}

// Tessellation network of the pairs whose contour outgrew a warp: the serial contour, then
// the elements k_net_elements writes for a warp contour (contact.rs:119-177), into the
// overflow area of the element storage (kSerialCap elements per listed pair).
__global__ void k_net_serial(DevBufs b, const uint32_t* __restrict__ voff, NetSlots sl) {
    const uint32_t listed = *sl.ov_count;
    const uint32_t count = listed < sl.ov_cap ? listed : sl.ov_cap;
    const int periodic = b.periodic;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
        if (slot >= b.serial_slots) break;
        const uint32_t p = sl.ov_list[t];
        const uint32_t v = voff[p];
        Contour c;
        c.v = reinterpret_cast<SP*>(b.serial_scratch) + (size_t)slot * kSerialCap;
        c.n = 0;
        c.cap = kSerialCap;
        c.overflow = false;
        Sph<double> ic;
        V3<double> axis, bary;
        double sum_arc, area;
        const bool ok = serial_clip(b, p, c, ic, axis, bary, sum_arc, area);
        const uint32_t o = t * (uint32_t)kSerialCap;  // in the overflow area
        sl.base[v] = sl.split + o;
        if (!ok || c.overflow) {  // counts stay 0
            atomicOr(b.err, (uint32_t)kErrNetwork);
            continue;
        }
        const uint32_t a = b.pair_a[p], bid = b.nb_id[b.pair_e[p]];
        if (c.n == 0) {  // an uncut contact: one SAS edge
            sl.ov_e_ids[o] = net_edge_ids(a, bid, kNetNull, periodic, b.n);
            sl.ov_e_len[o] = sum_arc * ic.r;
            sl.e_cnt[v] = 1;
            continue;
        }
        for (int k = 0; k < c.n; ++k) {
            const SP& cp = c.v[k];
            const SP& nx = c.v[k + 1 < c.n ? k + 1 : 0];
            const bool arc = cp.rid == a;
            sl.ov_e_ids[o + k] = net_edge_ids(a, bid, arc ? kNetNull : cp.rid, periodic, b.n);
            sl.ov_e_len[o + k] = arc ? cp.ang * ic.r : norm(P3(cp) - P3(nx));
            sl.ov_v_ids[o + k] =
                net_vertex_ids(a, bid, cp.lid == a ? kNetNull : cp.lid, arc ? kNetNull : cp.rid, periodic, b.n);
            sl.ov_v_xyz[3 * (size_t)(o + k)] = cp.x;
            sl.ov_v_xyz[3 * (size_t)(o + k) + 1] = cp.y;
            sl.ov_v_xyz[3 * (size_t)(o + k) + 2] = cp.z;
        }
        sl.v_cnt[v] = (uint32_t)c.n;
        sl.e_cnt[v] = (uint32_t)c.n;
    }
}

// Adjoint of the pairs whose contour outgrew a warp (listed by the FP64 adjoint in
// serial_list): the serial contour, then the same per-point and per-pair terms as the warp
// adjoint (vt_adjoint.cuh), summed in contour order by one thread.
template <bool VOL>
__global__ void k_adjoint_serial(DevBufs b, const double* __restrict__ u_contact, const double* __restrict__ w_eff,
                                 const double* __restrict__ v_eff, double* __restrict__ grad) {
    const uint32_t count = *b.d_serial_count;
    const uint32_t n = b.n;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
        if (slot >= b.serial_slots) break;
        const uint32_t p = b.serial_list[t];
        const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
        const uint32_t bid = b.nb_id[eb];
        AdjPair G;
        if (!adjoint_weights(b, p, a, bid, u_contact, w_eff, v_eff, G)) continue;
        Contour c;
        c.v = reinterpret_cast<SP*>(b.serial_scratch) + (size_t)slot * kSerialCap;
        c.n = 0;
        c.cap = kSerialCap;
        c.overflow = false;
        Sph<double> ic;
        V3<double> axis, bary;
        double sum_arc, area;
        const bool ok = serial_clip(b, p, c, ic, axis, bary, sum_arc, area);
        if (!ok || c.overflow) {
            if (c.overflow) atomicOr(b.err, kErrAdjoint);
            continue;
        }
        const Sph<double> A = sph_of(b.sph[a]), B = sph_of(b.sph[b.nb_slot[eb]]);
        G.pa = A.c;
        G.pb = B.c;
        G.Ra = A.r;
        G.Rb = B.r;
        G.q = ic.c;
        G.rho = ic.r;
        G.axis = axis;
        G.a = a;
        G.bid = bid;
        const uint32_t off = b.nb_off[a], cnt = b.nb_cnt[a];
        const uint32_t* nid = b.nb_id + off;
        const uint32_t* nslot = b.nb_slot + off;
        const double4* sph = b.sph;
        auto sphere_of = [&](uint32_t cid) {
            for (uint32_t e = 0; e < cnt; ++e)
                if (nid[e] == cid) return sph[nslot[e]];
            return make_double4(0.0, 0.0, 0.0, 0.0);
        };
        const double u = adj_area_weight<VOL>(G);
        V3<double> ga = mk<double>(0, 0, 0), gb = mk<double>(0, 0, 0), X = mk<double>(0, 0, 0);
        double gra = 0.0, grb = 0.0, L = 0.0;
        if (c.n == 0) {
            L = 2.0 * kPi * G.rho;
            X = G.q * L;
        } else {
            for (int k = 0; k < c.n; ++k) {
                const SP& cp = c.v[k];
                const SP& nx = c.v[k + 1 < c.n ? k + 1 : 0];
                adj_point(G, u, P3(cp), P3(nx), cp.ang, cp.rid, nx.lid, sphere_of, grad, n, ga, gra, gb, grb, L, X);
            }
        }
        adj_finish<VOL>(G, u, L, X, ga, gra, gb, grb, grad, n);
    }
}

}  // namespace

void launch_adjoint_serial(const DevBufs& b, const double* u_contact, const double* w_eff, const double* v_eff,
                           double* grad, cudaStream_t s) {
    const unsigned threads = 128;
    const unsigned blocks = (b.serial_slots + threads - 1) / threads;
    if (v_eff)
        k_adjoint_serial<true><<<blocks, threads, 0, s>>>(b, u_contact, w_eff, v_eff, grad);
    else
        k_adjoint_serial<false><<<blocks, threads, 0, s>>>(b, u_contact, w_eff, v_eff, grad);
    count_launch();
}

void launch_net_serial(const DevBufs& b, const uint32_t* voff, NetSlots sl, cudaStream_t s) {
    unsigned threads = 128;
    unsigned blocks = (b.serial_slots + threads - 1) / threads;
    k_net_serial<<<blocks, threads, 0, s>>>(b, voff, sl); count_launch();
}

void hex_table_values(double* hs, double* hc, int* n) {
    // the reference's accumulation: rotation_angle = pi/3, += pi/3 while < 2 pi
    for (int j = 0; j < 8; ++j) hs[j] = hc[j] = 0.0;
    int k = 1;
    for (double ang = kFracPi3; ang < kTau && k < 8; ang += kFracPi3, ++k) {
        double half = ang / 2.0;
        hs[k] = std::sin(half);
        hc[k] = std::cos(half);
    }
    *n = k;
}

void set_hex_table() {
    double hs[8], hc[8];
    int n = 0;
    hex_table_values(hs, hc, &n);
    cudaMemcpyToSymbol(c_hex_sin, hs, sizeof(hs));
    cudaMemcpyToSymbol(c_hex_cos, hc, sizeof(hc));
    cudaMemcpyToSymbol(c_hex_n, &n, sizeof(int));
    set_hex_table_adjoint();  // the adjoint's and the network's translation units hold
    set_hex_table_network();  // their own copies
}

void launch_contact_f64(const DevBufs& b, uint32_t P, int full, int from_list, cudaStream_t s) {
    size_t work = from_list ? P : P;  // upper bound of the list length is P
    size_t g = (work + kWarps - 1) / kWarps;
    if (g < 1) g = 1;
    if (g > 148 * 64) g = 148 * 64;
    if (full && b.p_arcm)
        k_contact64<true, true><<<(unsigned)g, kWarps * 32, 0, s>>>(b, P, from_list);
    else if (full)
        k_contact64<true, false><<<(unsigned)g, kWarps * 32, 0, s>>>(b, P, from_list);
    else
        k_contact64<false, false><<<(unsigned)g, kWarps * 32, 0, s>>>(b, P, from_list);
    count_launch();
}

void launch_contact_serial(const DevBufs& b, uint32_t, int full, cudaStream_t s) {
    unsigned threads = 128;
    unsigned blocks = (b.serial_slots + threads - 1) / threads;
    k_contact_serial<<<blocks, threads, 0, s>>>(b, full); count_launch();
}

}  // namespace vt
