// vt_contact32.cu -- FP32 bulk contact kernel (one warp per pair).
//
// Works in coordinates relative to ball a (the CSR holds each neighbour's centre minus
// a's centre, rounded once to float, and its radius), so contour geometry keeps ~7
// significant digits of a's neighbourhood rather than of the absolute coordinates.
// Every fuzzy decision is evaluated with an uncertainty band (vt_geom.cuh, Dec<float,
// true>); a pair with any decision inside its band is marked unsure and recomputed by
// the FP64 kernel, as is a pair whose contour outgrew the warp.
// the FP32 kernels' double helpers stay inline (vt_geom.cuh)
#define VT_FP32_UNIT 1
#include "vt_adjoint.cuh"
#include "vt_contact.cuh"
#include "vt_pipeline.cuh"

namespace vt {

namespace {

#ifndef VT_C32_WARPS
#define VT_C32_WARPS 4
#endif
#ifndef VT_C32_MINB
#define VT_C32_MINB 1
#endif
constexpr int kWarps = VT_C32_WARPS;

// One pair: the FP32 contour and the descriptor, written to the pair's outputs.
// REC: also record the pair's contour for the network (DevBufs::rec_*).
template <bool FULL, bool XM, bool REC, int W>
__device__ __forceinline__ void contact_pair32(const DevBufs& b, uint32_t p, float band) {
    const int lane = threadIdx.x & 31;
    const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
    const uint32_t off = b.nb_off[a], cnt = b.nb_cnt[a];
    PairGeom<float> g;
    const float Ra = (float)b.sph[a].w;
    const float4 rb = b.nb_rel[eb];
    g.A = {{0.f, 0.f, 0.f}, Ra};
    g.B = {{rb.x, rb.y, rb.z}, rb.w};
    g.a_id = a;
    g.b_id = b.nb_id[eb];
    g.S = Ra + rb.w;
    g.e0 = band * g.S;
    if (XM && b.p_arcm) g.xm_out = b.p_arcm + 6 * (size_t)p;
    const float4* rel = b.nb_rel + off;
    const uint32_t* nid = b.nb_id + off;
    auto nbf = [&](int e) {
        Nb<float> r;
        float4 v = rel[e];
        r.s = {{v.x, v.y, v.z}, v.w};
        r.id = nid[e];
        return r;
    };
    // the contact's area, arc length and centrality (and with REC its contour, into the
    // pool) are stored as soon as they are final, so that they are not kept in registers
    // through the descriptor code
    auto on_final = [&](const Pt<float>& q, int len, bool full, bool unsure, const WarpContact& rr) {
        if (lane == 0) {
            b.p_area[p] = rr.area;
            b.p_arc[p] = rr.arc;
            b.p_central[p] = rr.central ? 1 : 0;
        }
        if constexpr (REC) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(b.rec_count, (uint32_t)len);
            base = __shfl_sync(0xffffffffu, base, 0);
            if ((uint64_t)base + (uint64_t)len > (uint64_t)b.rec_cap) base = kRecNone;  // pool full: recompute
            if (base != kRecNone && lane < len) {
                b.rec_pts[base + lane] = make_float4(q.p.x, q.p.y, q.p.z, q.ang);
                b.rec_ids[base + lane] = make_uint2(q.lid, q.rid);
            }
            if (lane == 0) {
                b.rec_off[p] = base;
                b.rec_meta[p] =
                    ((uint32_t)len << 8) | (full ? 1u : 0u) | (rr.merged ? 2u : 0u) | (unsure ? 4u : 0u);
            }
        }
    };
    const WarpContact r = contact_warp<float, true, FULL, XM, W>(g, (int)cnt, (int)(eb - off), nbf, nullptr, on_final);
    if (!r.valid && lane == 0) {  // no contact: zero outputs, nothing recorded
        b.p_area[p] = 0.0;
        b.p_arc[p] = 0.0;
        b.p_central[p] = 0;
        if constexpr (REC) {
            b.rec_off[p] = kRecNone;
            b.rec_meta[p] = 0u;
        }
    }
    if (lane == 0) {
        uint8_t st = (r.valid ? kValid : 0) | (r.unsure ? kUnsure : 0) | (r.overflow ? kOverflow : 0);
        b.p_status[p] = st;
        b.p_sa_a[p] = r.valid ? r.sa_a : 0.0;
        b.p_sa_b[p] = r.valid ? r.sa_b : 0.0;
        b.p_pv_a[p] = r.valid ? r.pv_a : 0.0;
        b.p_pv_b[p] = r.valid ? r.pv_b : 0.0;
    }
}

// W warps per block (chosen by the engine's autotuner); the minimum resident blocks keep
// the register budget of a thread at 64 for every W (the arc-moment variant spills a few
// bytes there, which costs less than the occupancy 80 registers would take).
// queue == null: a grid-stride loop over the pairs.  Otherwise a persistent launch (one
// wave of resident blocks) whose warps take chunks of `chunk` consecutive pairs from the
// work counter *queue (zero at launch), so that costly pairs do not leave a tail of idle
// SMs.
template <bool FULL, bool XM, bool REC, int W>
__global__ void __launch_bounds__(W * 32, VT_C32_MINB * 4 / W)
    k_contact32(DevBufs b, uint32_t P, float band, uint32_t* queue, uint32_t chunk) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // one loop (and one inlined copy of the contour code) for both launch forms
    uint32_t p = queue ? 0u : blockIdx.x * W + w, end = queue ? 0u : P;
    const uint32_t step = queue ? 1u : gridDim.x * W;
    for (;;) {
        if (p >= end) {
            if (!queue) break;
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(queue, chunk);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= P) break;
            p = base;
            end = base + chunk < P ? base + chunk : P;
        }
        contact_pair32<FULL, XM, REC, W>(b, p, band);
        p += step;
    }
}

// The FP32 contour the contact kernel of the same call recorded for pair p
// (DevBufs::rec_*), filled in as the warp computation returns it (one point per lane);
// false when none was recorded (the caller recomputes it).
__device__ __forceinline__ bool recorded_contour(const DevBufs& b, uint32_t p, uint32_t a, ContourOut<float>& co,
                                                 WarpContact& r) {
    const uint32_t ro = b.rec_off ? b.rec_off[p] : kRecNone;
    if (ro == kRecNone) return false;
    const int lane = threadIdx.x & 31;
    const uint32_t meta = b.rec_meta[p];
    co.len = (int)(meta >> 8);
    co.full = (meta & 1u) != 0;
    if (lane < co.len) {
        const float4 q = b.rec_pts[ro + lane];
        const uint2 ids = b.rec_ids[ro + lane];
        co.q.p = {q.x, q.y, q.z};
        co.q.ang = q.w;
        co.q.lid = ids.x;
        co.q.rid = ids.y;
    } else {
        co.q.p = {0.f, 0.f, 0.f};
        co.q.ang = 0.f;
        co.q.lid = co.q.rid = a;
    }
    r.valid = true;
    r.overflow = false;
    r.merged = (meta & 2u) != 0;
    r.unsure = (meta & 4u) != 0;
    return true;
}

// Double spheres of a's neighbours by id, for the vertex placement and the adjoint (up to
// three lookups per contour point).  A per-warp open-addressing table in shared memory
// (id -> sphere slot, multiplicative hashing with linear probing, filled once per ball a:
// a warp's consecutive pairs mostly share a) answers a lookup in a probe or two, where a
// scan of the list costs about one iteration per list entry on the slowest lane; lists
// longer than kIdTabMax are scanned.  Ids are distinct within a list and below
// 0xffffffff (the host bounds them by 27 n), the table's empty key.
constexpr int kIdTabBits = 7, kIdTabSize = 1 << kIdTabBits;
constexpr uint32_t kIdTabMax = 96, kIdTabEmpty = 0xffffffffu;
struct IdTab {
    uint32_t key[kIdTabSize];
    uint32_t slot[kIdTabSize];
};
__device__ __forceinline__ uint32_t idtab_hash(uint32_t id) { return (id * 0x9E3779B1u) >> (32 - kIdTabBits); }

struct NbSpheres {
    IdTab* t;
    const double4* sph;
    const uint32_t* nid;
    const uint32_t* nslot;
    uint32_t cnt;
    uint32_t tab_a;  // the ball whose list the table holds (kIdTabEmpty: none yet)
    bool hashed;
    // warp-collective: make lookups refer to ball a's list
    __device__ __forceinline__ void bind(uint32_t a, const uint32_t* nid_, const uint32_t* nslot_, uint32_t cnt_) {
        nid = nid_;
        nslot = nslot_;
        cnt = cnt_;
        hashed = cnt <= kIdTabMax;
        if (!hashed || tab_a == a) return;
        const int lane = threadIdx.x & 31;
        __syncwarp();  // lookups into the previous list are done
        for (int k = lane; k < kIdTabSize; k += 32) t->key[k] = kIdTabEmpty;
        __syncwarp();
        for (uint32_t e = lane; e < cnt; e += 32) {
            const uint32_t id = nid[e];
            uint32_t pos = idtab_hash(id);
            for (int probe = 0; probe < kIdTabSize; ++probe) {  // cnt < kIdTabSize: a free key exists
                if (atomicCAS(&t->key[pos], kIdTabEmpty, id) == kIdTabEmpty) {
                    t->slot[pos] = nslot[e];
                    break;
                }
                pos = (pos + 1) & (kIdTabSize - 1);
            }
        }
        __syncwarp();
        tab_a = a;
    }
    __device__ __forceinline__ double4 operator()(uint32_t c) const {
        if (hashed) {
            uint32_t pos = idtab_hash(c);
            for (int probe = 0; probe < kIdTabSize; ++probe) {
                const uint32_t k = t->key[pos];
                if (k == c) return sph[t->slot[pos]];
                if (k == kIdTabEmpty) break;
                pos = (pos + 1) & (kIdTabSize - 1);
            }
        } else {
            for (uint32_t e = 0; e < cnt; ++e)
                if (nid[e] == c) return sph[nslot[e]];
        }
        return make_double4(0.0, 0.0, 0.0, 0.0);
    }
};

// FP32 adjoint: the contour recomputed in FP32 (relative to a), the gradient formed in
// double from its points; pairs whose recomputation is unsure or overflows are listed for
// the FP64 adjoint.
template <bool VOL>
__global__ void __launch_bounds__(kWarps * 32, 4)
    k_adjoint32(DevBufs b, uint32_t P, float band, const double* __restrict__ u_contact,
                const double* __restrict__ w_eff, const double* __restrict__ v_eff, double* __restrict__ grad) {
    __shared__ IdTab tabs[kWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n = b.n;
    NbSpheres sphere_of{&tabs[w], b.sph, nullptr, nullptr, 0, kIdTabEmpty, false};
    // chunks of 32 consecutive pairs per warp: one coalesced status read per chunk, and
    // consecutive pairs share ball a (one table fill)
    for (size_t c0 = ((size_t)blockIdx.x * kWarps + w) * 32; c0 < P; c0 += (size_t)gridDim.x * kWarps * 32) {
        unsigned todo = __ballot_sync(kFull, c0 + lane < P && (b.p_status[c0 + lane] & kValid));
        while (todo) {
            const uint32_t p = (uint32_t)c0 + (uint32_t)(__ffs(todo) - 1);
            todo &= todo - 1;
            const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
            const uint32_t bid = b.nb_id[eb];
            AdjPair G;
            if (!adjoint_weights(b, p, a, bid, u_contact, w_eff, v_eff, G)) continue;
            const uint32_t off = b.nb_off[a], cnt = b.nb_cnt[a];
            const double4 A4 = b.sph[a], B4 = b.sph[b.nb_slot[eb]];
            PairGeom<float> g;
            const float Ra = (float)A4.w;
            const float4 rb = b.nb_rel[eb];
            g.A = {{0.f, 0.f, 0.f}, Ra};
            g.B = {{rb.x, rb.y, rb.z}, rb.w};
            g.a_id = a;
            g.b_id = bid;
            g.S = Ra + rb.w;
            g.e0 = band * g.S;
            const float4* rel = b.nb_rel + off;
            const uint32_t* nid = b.nb_id + off;
            const uint32_t* nslot = b.nb_slot + off;
            auto nbf = [&](int e) {
                Nb<float> r;
                float4 v = rel[e];
                r.s = {{v.x, v.y, v.z}, v.w};
                r.id = nid[e];
                return r;
            };
            ContourOut<float> co;
            WarpContact r;
            if (!recorded_contour(b, p, a, co, r))
                r = contact_warp<float, true, false, false, kWarps>(g, (int)cnt, (int)(eb - off), nbf, &co);
            if (r.unsure || r.overflow) {
                if (lane == 0) b.redo_list[atomicAdd(b.d_redo_count, 1u)] = p;
                continue;
            }
            if (!r.valid) continue;  // no contact, decided outside the band
            const Sph<double> A = {{A4.x, A4.y, A4.z}, A4.w}, B = {{B4.x, B4.y, B4.z}, B4.w};
            const Sph<double> ic = intersection_circle(A, B);
            G.pa = A.c;
            G.pb = B.c;
            G.Ra = A.r;
            G.Rb = B.r;
            G.q = ic.c;
            G.rho = ic.r;
            G.axis = normalize(B.c - A.c);
            G.a = a;
            G.bid = bid;
            const int len = co.len;
            const int nx = len > 0 ? (lane + 1 < len ? lane + 1 : 0) : 0;
            if (!co.full) sphere_of.bind(a, nid, nslot, cnt);
            // the FP32 topology with FP64 vertices and arc angles
            V3<double> y = widen(co.q.p);
            if (!co.full && lane < len) y = snap_vertex(G, y, co.q.lid, co.q.rid, sphere_of);
            const V3<double> P0 = A.c + y;
            const V3<double> P1 = mk<double>(__shfl_sync(kFull, P0.x, nx), __shfl_sync(kFull, P0.y, nx),
                                             __shfl_sync(kFull, P0.z, nx));
            const uint32_t nlid = __shfl_sync(kFull, co.q.lid, nx);
            double ang = 0.0;
            if (!co.full && lane < len && co.q.rid == a && nlid == a && co.q.ang > 0.f) {
                const V3<double> v1 = P0 - G.q, v2 = P1 - G.q;
                ang = atan2(dot(cross(v1, v2), G.axis), dot(v1, v2));
                if (ang < 0.0) ang += kTau;
                // a nearly full or nearly empty arc keeps the FP32 branch of the angle
                if (fabs((double)co.q.ang - ang) > 1.0) ang = (double)co.q.ang;
            }
            adjoint_pair<VOL>(G, co.full, len, P0, P1, ang, co.q.rid, nlid, sphere_of, grad, n);
        }
    }
}

// Tessellation network elements from the FP32 contour (tessellation network of
// vt_network.cu): the FP32 topology gives every vertex's defining planes, and the vertex
// is placed in double from them (snap_vertex), so positions, chord lengths and arc
// angles are FP64 values.  A pair whose FP32 contour is unsure, overflows, merged two
// points (the kept point's ids no longer define it), or has a vertex the snap cannot
// place is listed for the FP64 element kernel instead.
#ifndef VT_NET32_MINB
#define VT_NET32_MINB 6  // 80 registers (a little spill) for 24 warps per SM: 10% faster than 4
#endif
__global__ void __launch_bounds__(kWarps * 32, VT_NET32_MINB)
    k_net_elements32(DevBufs b, uint32_t P, float band, const uint32_t* __restrict__ voff, NetSlots sl,
                     uint32_t* __restrict__ fp64_list, uint32_t* __restrict__ fp64_count) {
    __shared__ IdTab tabs[kWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n = b.n;
    const int periodic = b.periodic;
    NbSpheres sphere_of{&tabs[w], b.sph, nullptr, nullptr, 0, kIdTabEmpty, false};
    // chunks of 32 consecutive pairs per warp: one coalesced read of the slot offsets per
    // chunk, and consecutive pairs share ball a (one table fill)
    for (size_t c0 = ((size_t)blockIdx.x * kWarps + w) * 32; c0 < P; c0 += (size_t)gridDim.x * kWarps * 32) {
        uint32_t vo = 0, vn = 0;
        if (c0 + lane < P) {
            vo = voff[c0 + lane];
            vn = voff[c0 + lane + 1];
        }
        unsigned todo = __ballot_sync(kFull, vn != vo);  // pairs with a contact
        while (todo) {
            const int k = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t p = (uint32_t)c0 + (uint32_t)k;
            const uint32_t slot = __shfl_sync(kFull, vo, k);
            const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
            const uint32_t bid = b.nb_id[eb];
            const uint32_t off = b.nb_off[a], cnt = b.nb_cnt[a];
            const double4 A4 = b.sph[a], B4 = b.sph[b.nb_slot[eb]];
            PairGeom<float> g;
            const float Ra = (float)A4.w;
            const float4 rb = b.nb_rel[eb];
            g.A = {{0.f, 0.f, 0.f}, Ra};
            g.B = {{rb.x, rb.y, rb.z}, rb.w};
            g.a_id = a;
            g.b_id = bid;
            g.S = Ra + rb.w;
            g.e0 = band * g.S;
            const float4* rel = b.nb_rel + off;
            const uint32_t* nid = b.nb_id + off;
            const uint32_t* nslot = b.nb_slot + off;
            auto nbf = [&](int e) {
                Nb<float> r;
                float4 v = rel[e];
                r.s = {{v.x, v.y, v.z}, v.w};
                r.id = nid[e];
                return r;
            };
            ContourOut<float> co;
            WarpContact r;
            if (!recorded_contour(b, p, a, co, r))
                r = contact_warp<float, true, false, false, kWarps>(g, (int)cnt, (int)(eb - off), nbf, &co);
            bool fp64 = r.unsure || r.overflow || !r.valid || r.merged;
            const Sph<double> A = {{A4.x, A4.y, A4.z}, A4.w}, B = {{B4.x, B4.y, B4.z}, B4.w};
            const Sph<double> ic = intersection_circle(A, B);
            const uint32_t base = slot * (uint32_t)kNetSlot;
            if (!fp64 && co.full) {  // an uncut contact: one SAS edge, no vertex
                if (lane == 0) {
                    sl.e_ids[base] = net_edge_ids(a, bid, kNetNull, periodic, n);
                    sl.e_len[base] = kTau * ic.r;
                    sl.v_cnt[slot] = 0;
                    sl.e_cnt[slot] = 1;
                    sl.base[slot] = base;
                }
                continue;
            }
            const int len = co.len;
            V3<double> P0 = mk<double>(0, 0, 0), P1 = P0;
            double ang = 0.0;
            bool arc = false;
            if (!fp64) {
                AdjPair G;
                G.pa = A.c;
                G.pb = B.c;
                G.Ra = A.r;
                G.Rb = B.r;
                G.q = ic.c;
                G.rho = ic.r;
                G.axis = normalize(B.c - A.c);
                G.a = a;
                G.bid = bid;
                sphere_of.bind(a, nid, nslot, cnt);
                bool ok = true;
                V3<double> y = widen(co.q.p);
                if (lane < len) y = snap_vertex(G, y, co.q.lid, co.q.rid, sphere_of, &ok);
                P0 = A.c + y;
                const int nx = len > 0 ? (lane + 1 < len ? lane + 1 : 0) : 0;
                P1 = mk<double>(__shfl_sync(kFull, P0.x, nx), __shfl_sync(kFull, P0.y, nx),
                                __shfl_sync(kFull, P0.z, nx));
                const uint32_t nlid = __shfl_sync(kFull, co.q.lid, nx);
                arc = lane < len && co.q.rid == a;
                if (arc && nlid == a && co.q.ang > 0.f) {
                    const V3<double> v1 = P0 - G.q, v2 = P1 - G.q;
                    ang = atan2(dot(cross(v1, v2), G.axis), dot(v1, v2));
                    if (ang < 0.0) ang += kTau;
                    if (fabs((double)co.q.ang - ang) > 1e-3) ok = false;  // the 0 / 2 pi branch is unclear
                }
                // elements with equal ids inside one contour (arcs of one contact, both ends of
                // an arc cut by the same ball): the network keeps the first in contour order,
                // which the FP64 contour decides
                const bool on = lane < len;
                const uint32_t third = arc ? kNetNull : co.q.rid;
                const uint32_t vl = co.q.lid == a ? kNetNull : co.q.lid;
                const unsigned long long ek = on ? (unsigned long long)third : (1ull << 40) + lane;
                const unsigned long long vk = on ? ((unsigned long long)vl << 32 | third) : (1ull << 63) + lane;
                // both matches on every lane: a collective that some lanes skip (a short-circuit
                // ||) pairs the warp's later collectives wrongly
                const unsigned me = __match_any_sync(kFull, ek), mv = __match_any_sync(kFull, vk);
                const bool dup = __popc(me) > 1 || __popc(mv) > 1;
                fp64 = __any_sync(kFull, !ok || dup);
            }
            if (fp64) {
                if (lane == 0) {
                    sl.v_cnt[slot] = 0;
                    sl.e_cnt[slot] = 0;
                    sl.base[slot] = base;
                    fp64_list[atomicAdd(fp64_count, 1u)] = p;
                }
                continue;
            }
            if (lane < len) {
                const Pt<float>& cp = co.q;
                sl.e_ids[base + lane] = net_edge_ids(a, bid, arc ? kNetNull : cp.rid, periodic, n);
                sl.e_len[base + lane] = arc ? ang * ic.r : norm(P1 - P0);
                sl.v_ids[base + lane] =
                    net_vertex_ids(a, bid, cp.lid == a ? kNetNull : cp.lid, arc ? kNetNull : cp.rid, periodic, n);
                sl.v_xyz[3 * (size_t)(base + lane)] = P0.x;
                sl.v_xyz[3 * (size_t)(base + lane) + 1] = P0.y;
                sl.v_xyz[3 * (size_t)(base + lane) + 2] = P0.z;
            }
            if (lane == 0) {
                sl.v_cnt[slot] = (uint32_t)len;
                sl.e_cnt[slot] = (uint32_t)len;
                sl.base[slot] = base;
            }
        }
    }
}

}  // namespace

void launch_net_elements_f32(const DevBufs& b, uint32_t P, const uint32_t* voff, NetSlots sl, uint32_t* fp64_list,
                             uint32_t* fp64_count, cudaStream_t s) {
    size_t g = ((size_t)P + 32 * kWarps - 1) / (32 * kWarps);
    if (g < 1) g = 1;
    if (g > 148 * 64) g = 148 * 64;
    k_net_elements32<<<(unsigned)g, kWarps * 32, 0, s>>>(b, P, b.fp32_band, voff, sl, fp64_list, fp64_count);
    count_launch();
}

void launch_adjoint_f32(const DevBufs& b, uint32_t P, const double* u_contact, const double* w_eff,
                        const double* v_eff, double* grad, cudaStream_t s) {
    size_t g = ((size_t)P + 32 * kWarps - 1) / (32 * kWarps);
    if (g < 1) g = 1;
    if (g > 148 * 64) g = 148 * 64;
    if (v_eff)
        k_adjoint32<true><<<(unsigned)g, kWarps * 32, 0, s>>>(b, P, b.fp32_band, u_contact, w_eff, v_eff, grad);
    else
        k_adjoint32<false><<<(unsigned)g, kWarps * 32, 0, s>>>(b, P, b.fp32_band, u_contact, w_eff, v_eff, grad);
    count_launch();
}

template <bool FULL, bool XM, bool REC, int W>
void launch_c32_kernel(const DevBufs& b, uint32_t P, cudaStream_t s) {
    uint32_t* queue = b.c32_chunk > 0 ? b.c32_queue : nullptr;
    size_t g;
    if (queue) {
        static int blocks_per_sm = 0;  // resident blocks of this variant (per process)
        if (blocks_per_sm == 0)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_contact32<FULL, XM, REC, W>, W * 32, 0);
        int sms = 148;
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g = (size_t)sms * (size_t)(blocks_per_sm > 0 ? blocks_per_sm : 1);
        cudaMemsetAsync(queue, 0, sizeof(uint32_t), s);
    } else {
        g = (P + W - 1) / W;
        if (g > (size_t)148 * 16 * 32 / W) g = (size_t)148 * 16 * 32 / W;
    }
    if (g < 1) g = 1;
    k_contact32<FULL, XM, REC, W><<<(unsigned)g, W * 32, 0, s>>>(b, P, b.fp32_band, queue, (uint32_t)b.c32_chunk);
    count_launch();
}

template <int W>
void launch_c32(const DevBufs& b, uint32_t P, int full, cudaStream_t s) {
    if (full && b.p_arcm)  // the updateable tessellation records arc and face moments
        launch_c32_kernel<true, true, false, W>(b, P, s);
    else if (full && b.rec_off)  // the network's element kernel reuses the contours
        launch_c32_kernel<true, false, true, W>(b, P, s);
    else if (full)
        launch_c32_kernel<true, false, false, W>(b, P, s);
    else
        launch_c32_kernel<false, false, false, W>(b, P, s);
}

void launch_contact_f32(const DevBufs& b, uint32_t P, int full, cudaStream_t s) {
    if (b.c32_warps == 2)
        launch_c32<2>(b, P, full, s);
    else if (b.c32_warps == 8)
        launch_c32<8>(b, P, full, s);
    else
        launch_c32<4>(b, P, full, s);
}

}  // namespace vt

