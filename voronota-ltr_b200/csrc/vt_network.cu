// vt_network.cu -- the tessellation network (with_cell_vertices): cell vertices and
// edges of the radical tessellation, deduplicated (contact.rs:119-177,
// tessellation.rs:334-401).
//
//   1. every valid pair's contour is recomputed in FP64 (warp per pair) and emits one edge
//      per contour segment -- ids (a, b, the cutting neighbour or NULL on an arc), length
//      of the chord or arc -- and one vertex per contour point -- ids (a, b, left id,
//      right id with a's id as NULL), position; an uncut contact emits one SAS edge; a
//      contour that outgrows the warp is listed for the serial kernel (vt_contact64.cu);
//   2. ids are taken mod n for periodic images and sorted within the element;
//   3. elements are compacted, stably sorted by their ids (radix sort on two key words,
//      low word first; an id takes B = bits(n) bits with NULL mapped to n, so it still
//      sorts after every ball id, and a word holds two ids: 2B bits instead of 64) and
//      deduplicated keeping the first of equal ids, i.e. the first in pair and contour
//      order (the reference sorts unstably and keeps an unspecified one).
#include <cub/cub.cuh>

#include "vt_contact.cuh"
#include "vt_pipeline.cuh"

namespace vt {

namespace {

constexpr int kWarps = 4;
constexpr int kSlot = kNetSlot;  // elements of one pair (a warp contour holds <= 32 points)

__device__ __forceinline__ Sph<double> sph_of(double4 v) { return {{v.x, v.y, v.z}, v.w}; }

__global__ void k_valid_flags(const uint8_t* __restrict__ status, uint32_t P, uint32_t* __restrict__ flags) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x)
        flags[p] = (status[p] & kValid) ? 1u : 0u;
}

__global__ void __launch_bounds__(kWarps * 32)
    k_net_elements(DevBufs b, uint32_t P, const uint32_t* __restrict__ voff, NetSlots sl,
                   const uint32_t* __restrict__ list, const uint32_t* __restrict__ list_count) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n = b.n;
    const int periodic = b.periodic;
    const uint32_t count = list ? *list_count : P;
    for (uint32_t it = blockIdx.x * kWarps + w; it < count; it += gridDim.x * kWarps) {
        const uint32_t p = list ? list[it] : it;
        const uint32_t slot = voff[p];
        if (voff[p + 1] == slot) continue;  // no contact
        const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
        const uint32_t off = b.nb_off[a], cnt = b.nb_cnt[a];
        PairGeom<double> g;
        g.A = sph_of(b.sph[a]);
        g.B = sph_of(b.sph[b.nb_slot[eb]]);
        g.a_id = a;
        g.b_id = b.nb_id[eb];
        g.e0 = 0.0;
        g.S = g.A.r + g.B.r;
        const double4* sph = b.sph;
        const uint32_t* nslot = b.nb_slot + off;
        const uint32_t* nid = b.nb_id + off;
        auto nbf = [&](int e) {
            Nb<double> r;
            r.s = sph_of(sph[nslot[e]]);
            r.id = nid[e];
            return r;
        };
        ContourOut<double> co;
        WarpContact r = contact_warp<double, false, false>(g, (int)cnt, (int)(eb - off), nbf, &co);
        const uint32_t base = slot * (uint32_t)kSlot;
        if (!r.valid) {  // the contour outgrew the warp: the serial kernel emits this pair
            if (lane == 0) {
                sl.v_cnt[slot] = 0;
                sl.e_cnt[slot] = 0;
                sl.base[slot] = base;
                const uint32_t j = r.overflow ? atomicAdd(sl.ov_count, 1u) : sl.ov_cap;
                if (j < sl.ov_cap)
                    sl.ov_list[j] = p;
                else
                    atomicOr(b.err, kErrNetwork);
            }
            continue;
        }
        if (co.full) {  // an uncut contact: one SAS edge, no vertex
            if (lane == 0) {
                sl.e_ids[base] = net_edge_ids(a, g.b_id, kNetNull, periodic, n);
                sl.e_len[base] = kTau * co.ic.r;
                sl.v_cnt[slot] = 0;
                sl.e_cnt[slot] = 1;
                sl.base[slot] = base;
            }
            continue;
        }
        const int len = co.len;
        const int nx = len > 0 ? (lane + 1 < len ? lane + 1 : 0) : 0;
        const Pt<double> nxt = shfl_pt(co.q, nx);
        if (lane < len) {
            const Pt<double>& cp = co.q;
            const bool arc = cp.rid == a;
            sl.e_ids[base + lane] = net_edge_ids(a, g.b_id, arc ? kNetNull : cp.rid, periodic, n);
            sl.e_len[base + lane] = arc ? cp.ang * co.ic.r : norm(cp.p - nxt.p);
            sl.v_ids[base + lane] =
                net_vertex_ids(a, g.b_id, cp.lid == a ? kNetNull : cp.lid, arc ? kNetNull : cp.rid, periodic, n);
            sl.v_xyz[3 * (size_t)(base + lane)] = cp.p.x;
            sl.v_xyz[3 * (size_t)(base + lane) + 1] = cp.p.y;
            sl.v_xyz[3 * (size_t)(base + lane) + 2] = cp.p.z;
        }
        if (lane == 0) {
            sl.v_cnt[slot] = (uint32_t)len;
            sl.e_cnt[slot] = (uint32_t)len;
            sl.base[slot] = base;
        }
    }
}

// dense arrays: key words (hi, lo) and the element's index; thread per pair.  An id
// takes B bits, NULL (0xffffffff) becoming n, above every ball id.
__device__ __forceinline__ unsigned long long net_key_id(uint32_t id, uint32_t n) {
    return id == kNetNull ? (unsigned long long)n : (unsigned long long)id;
}
__global__ void k_net_compact(uint32_t V, const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ off,
                              NetSlots sl, int vertices, uint32_t n, int B, unsigned long long* __restrict__ key_hi,
                              unsigned long long* __restrict__ key_lo, uint32_t* __restrict__ src) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint32_t c = cnt[v], o = off[v], base = sl.base[v];
        for (uint32_t k = 0; k < c; ++k) {
            const uint32_t i = base + k;
            const uint4 id = vertices ? net_vid(sl, i) : net_eid(sl, i);
            key_hi[o + k] = (net_key_id(id.x, n) << B) | net_key_id(id.y, n);
            key_lo[o + k] = vertices ? ((net_key_id(id.z, n) << B) | net_key_id(id.w, n)) : net_key_id(id.z, n);
            src[o + k] = i;
        }
    }
}
__global__ void k_first_flags(const unsigned long long* __restrict__ hi, const unsigned long long* __restrict__ lo,
                              uint32_t m, uint32_t* __restrict__ flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        flags[i] = (i == 0 || hi[i] != hi[i - 1] || lo[i] != lo[i - 1]) ? 1u : 0u;
}
__global__ void k_net_gather_v(uint32_t m, const uint32_t* __restrict__ uoff, const uint32_t* __restrict__ src,
                               NetSlots sl, uint32_t* __restrict__ out_ids, double* __restrict__ out_xyz) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (uoff[i + 1] == uoff[i]) continue;
        const uint32_t o = uoff[i], s = src[i];
        const uint4 id = net_vid(sl, s);
        out_ids[4 * (size_t)o] = id.x;
        out_ids[4 * (size_t)o + 1] = id.y;
        out_ids[4 * (size_t)o + 2] = id.z;
        out_ids[4 * (size_t)o + 3] = id.w;
        for (int k = 0; k < 3; ++k) out_xyz[3 * (size_t)o + k] = net_vxyz(sl, s, k);
    }
}
__global__ void k_net_gather_e(uint32_t m, const uint32_t* __restrict__ uoff, const uint32_t* __restrict__ src,
                               NetSlots sl, uint32_t* __restrict__ out_ids, double* __restrict__ out_len) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (uoff[i + 1] == uoff[i]) continue;
        const uint32_t o = uoff[i], s = src[i];
        const uint4 id = net_eid(sl, s);
        out_ids[3 * (size_t)o] = id.x;
        out_ids[3 * (size_t)o + 1] = id.y;
        out_ids[3 * (size_t)o + 2] = id.z;
        out_len[o] = net_elen(sl, s);
    }
}

int gb(size_t n) { return grid_blocks(n, 256, 148 * 16); }

}  // namespace

void launch_valid_flags(const DevBufs& b, uint32_t P, uint32_t* flags, cudaStream_t s) {
    k_valid_flags<<<gb(P), 256, 0, s>>>(b.p_status, P, flags); count_launch();
}
void launch_net_elements(const DevBufs& b, uint32_t P, const uint32_t* voff, NetSlots sl, const uint32_t* list,
                         const uint32_t* count, cudaStream_t s) {
    k_net_elements<<<grid_blocks(P, kWarps, 148 * 64), kWarps * 32, 0, s>>>(b, P, voff, sl, list, count);
    count_launch();
}
size_t net_slot_capacity() { return kSlot; }

void set_hex_table_network() {
    double hs[8], hc[8];
    int n = 0;
    hex_table_values(hs, hc, &n);
    cudaMemcpyToSymbol(c_hex_sin, hs, sizeof(hs));
    cudaMemcpyToSymbol(c_hex_cos, hc, sizeof(hc));
    cudaMemcpyToSymbol(c_hex_n, &n, sizeof(int));
}

int net_key_bits(uint32_t n) {
    int B = 1;
    while (B < 32 && ((uint64_t)1 << B) <= (uint64_t)n) ++B;  // 2^B > n: ids 0..n-1 and NULL as n
    return B;
}
void launch_net_keys(uint32_t V, const uint32_t* cnt, const uint32_t* off, const NetSlots& sl, int vertices,
                     uint32_t n, unsigned long long* key_hi, unsigned long long* key_lo, uint32_t* src,
                     cudaStream_t s) {
    k_net_compact<<<gb(V), 256, 0, s>>>(V, cnt, off, sl, vertices, n, net_key_bits(n), key_hi, key_lo, src);
    count_launch();
}

size_t net_sort_temp_bytes(uint32_t m) {
    size_t bytes = 0;
    cub::DoubleBuffer<unsigned long long> k(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> v(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, k, v, (int)(m > 0 ? m : 1));
    return bytes + 256;
}

namespace {
__global__ void k_iota(uint32_t m, uint32_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) out[i] = i;
}
__global__ void k_gather_u64(uint32_t m, const uint32_t* __restrict__ idx, const unsigned long long* __restrict__ in,
                             unsigned long long* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) out[i] = in[idx[i]];
}
__global__ void k_gather_u32(uint32_t m, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ in,
                             uint32_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) out[i] = in[idx[i]];
}
}  // namespace

// Stable LSD sort of m keys (hi, lo): by lo, then by hi, carrying the dense index; only
// the low bits_lo / bits_hi bits of the words are sorted on (the rest are zero).  On
// return hi_s/lo_s hold the sorted keys and order[i] the dense index of sorted element i.
void net_sort(uint32_t m, const unsigned long long* hi, const unsigned long long* lo, int bits_hi, int bits_lo,
              NetSortBufs t, cudaStream_t s) {
    if (m == 0) return;
    k_iota<<<gb(m), 256, 0, s>>>(m, t.idx_a); count_launch();
    cudaMemcpyAsync(t.key_a, lo, 8 * (size_t)m, cudaMemcpyDeviceToDevice, s);
    size_t tb = t.temp_bytes;
    {
        cub::DoubleBuffer<unsigned long long> k(t.key_a, t.key_b);
        cub::DoubleBuffer<uint32_t> v(t.idx_a, t.idx_b);
        cub::DeviceRadixSort::SortPairs(t.temp, tb, k, v, (int)m, 0, bits_lo, s);
        count_launch();
        if (v.Current() != t.idx_a) cudaMemcpyAsync(t.idx_a, v.Current(), 4 * (size_t)m, cudaMemcpyDeviceToDevice, s);
    }
    k_gather_u64<<<gb(m), 256, 0, s>>>(m, t.idx_a, hi, t.key_a); count_launch();
    {
        tb = t.temp_bytes;
        cub::DoubleBuffer<unsigned long long> k(t.key_a, t.key_b);
        cub::DoubleBuffer<uint32_t> v(t.idx_a, t.idx_b);
        cub::DeviceRadixSort::SortPairs(t.temp, tb, k, v, (int)m, 0, bits_hi, s);
        count_launch();
        if (k.Current() != t.hi_s) cudaMemcpyAsync(t.hi_s, k.Current(), 8 * (size_t)m, cudaMemcpyDeviceToDevice, s);
        if (v.Current() != t.order) cudaMemcpyAsync(t.order, v.Current(), 4 * (size_t)m, cudaMemcpyDeviceToDevice, s);
    }
    k_gather_u64<<<gb(m), 256, 0, s>>>(m, t.order, lo, t.lo_s); count_launch();
}

void launch_net_unique(uint32_t m, const NetSortBufs& t, uint32_t* flags, cudaStream_t s) {
    k_first_flags<<<gb(m), 256, 0, s>>>(t.hi_s, t.lo_s, m, flags); count_launch();
}
void launch_net_gather(uint32_t m, const uint32_t* uoff, const uint32_t* order, const uint32_t* src_dense,
                       uint32_t* src_tmp, const NetSlots& sl, int vertices, uint32_t* out_ids, double* out_vals,
                       cudaStream_t s) {
    k_gather_u32<<<gb(m), 256, 0, s>>>(m, order, src_dense, src_tmp); count_launch();
    if (vertices)
        k_net_gather_v<<<gb(m), 256, 0, s>>>(m, uoff, src_tmp, sl, out_ids, out_vals);
    else
        k_net_gather_e<<<gb(m), 256, 0, s>>>(m, uoff, src_tmp, sl, out_ids, out_vals);
    count_launch();
}

}  // namespace vt
