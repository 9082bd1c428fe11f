// vt_network.cu -- the tessellation network (with_cell_vertices): cell vertices and
// edges of the radical tessellation, deduplicated (contact.rs:119-177,
// tessellation.rs:334-401).
//
//   1. every valid pair emits one edge per contour segment -- ids (a, b, the cutting
//      neighbour or NULL on an arc), length of the chord or arc -- and one vertex per
//      contour point -- ids (a, b, left id, right id with a's id as NULL), position; an
//      uncut contact emits one SAS edge.  FP64 mode recomputes the contours here in FP64
//      (warp per pair); FP32 mode takes the contours the contact kernel recorded and
//      places their vertices in double (k_net_elements32, vt_contact32.cu), and the pairs
//      that kernel cannot settle come here.  A contour that outgrows the warp is listed
//      for the serial kernel (vt_contact64.cu);
//   2. ids are taken mod n for periodic images and sorted within the element;
//   3. elements are put in id order and deduplicated keeping the first of equal ids, i.e.
//      the first in pair and contour order (the reference sorts unstably and keeps an
//      unspecified one): bucketed by their first id (a counting pass, a scan, a scatter),
//      each bucket reduced to its distinct id tuples (first occurrence, through a hash
//      table, for buckets of more than 32 elements) and sorted by (remaining ids, dense
//      index) -- a warp's bitonic sort in registers for buckets of up to 128 elements, a
//      block's otherwise.  The remaining ids are packed into one 64-bit key (NULL as n,
//      after every ball id) or, for vertices of 2^21 balls and more, two.
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

// ---- deduplication: bucket by the first id, sort each bucket, keep the first of equal ids ----
namespace {

constexpr int kBigSmem = 2048;  // bucket size the block sort holds in shared memory

__device__ __forceinline__ uint4 net_ids(const NetSlots& sl, uint32_t i, int vertices) {
    return vertices ? net_vid(sl, i) : net_eid(sl, i);
}
__device__ __forceinline__ uint32_t net_bucket(uint32_t id0, uint32_t n) { return id0 < n ? id0 : n; }
__device__ __forceinline__ unsigned long long net_key_id(uint32_t id, uint32_t n) {
    return id == kNetNull ? (unsigned long long)n : (unsigned long long)id;  // NULL after every ball id
}

// A bucket element: the ids after the first and the element's dense index j (pair then
// contour order), ordered by (ids, j).  Narrow form (WIDE = false): the ids packed B bits
// each into k1, NULL as n (2^B > n): edges always, vertices while 3 B <= 64.  Wide form:
// k1 = id1 << 32 | id2, k2 = id3.
template <bool WIDE>
struct NbKey {
    unsigned long long k1, k2;
    uint32_t j;
    __device__ __forceinline__ static NbKey pad() { return {~0ull, ~0ull, 0xffffffffu}; }
    __device__ __forceinline__ bool less(const NbKey& o) const {
        if (k1 != o.k1) return k1 < o.k1;
        if (WIDE && k2 != o.k2) return k2 < o.k2;
        return j < o.j;
    }
    __device__ __forceinline__ bool same_ids(const NbKey& o) const { return k1 == o.k1 && (!WIDE || k2 == o.k2); }
    __device__ __forceinline__ NbKey xor_lane(int m) const {
        NbKey r;
        r.k1 = __shfl_xor_sync(kFull, k1, m);
        r.k2 = WIDE ? __shfl_xor_sync(kFull, k2, m) : 0ull;
        r.j = __shfl_xor_sync(kFull, j, m);
        return r;
    }
    __device__ __forceinline__ NbKey from_lane(int src) const {
        NbKey r;
        r.k1 = __shfl_sync(kFull, k1, src);
        r.k2 = WIDE ? __shfl_sync(kFull, k2, src) : 0ull;
        r.j = __shfl_sync(kFull, j, src);
        return r;
    }
    __device__ __forceinline__ NbKey up_lane() const {
        NbKey r;
        r.k1 = __shfl_up_sync(kFull, k1, 1);
        r.k2 = WIDE ? __shfl_up_sync(kFull, k2, 1) : 0ull;
        r.j = __shfl_up_sync(kFull, j, 1);
        return r;
    }
    __device__ __forceinline__ static NbKey load(const unsigned long long* k1s, const unsigned long long* k2s,
                                                 const uint32_t* js, uint32_t i) {
        return {k1s[i], WIDE ? k2s[i] : 0ull, js[i]};
    }
    __device__ __forceinline__ void store(unsigned long long* k1s, unsigned long long* k2s, uint32_t* js,
                                          uint32_t i) const {
        k1s[i] = k1;
        if (WIDE) k2s[i] = k2;
        js[i] = j;
    }
};

// The key of an element with sorted ids id (first id already the bucket)
template <bool WIDE>
__device__ __forceinline__ NbKey<WIDE> nb_key(uint4 id, int vertices, uint32_t n, int B, uint32_t j) {
    NbKey<WIDE> k;
    k.j = j;
    k.k2 = 0ull;
    if (WIDE) {  // vertices only
        k.k1 = (unsigned long long)id.y << 32 | id.z;
        k.k2 = id.w;
    } else if (vertices) {
        k.k1 = (net_key_id(id.y, n) << (2 * B)) | (net_key_id(id.z, n) << B) | net_key_id(id.w, n);
    } else {
        k.k1 = (net_key_id(id.y, n) << B) | net_key_id(id.z, n);
    }
    return k;
}

// The counting (FILL = false) and scatter (FILL = true) passes, lanes over the dense
// elements: a warp takes 32 consecutive pair slots, whose elements are the dense range
// [off[v0], off[v0 + 32]), and finds each lane's slot by a shuffle binary search over the
// slots' offsets (coalesced reads, every lane busy although a contour has ~5 vertices).
// Lanes of one bucket share one atomic; the scatter places them in lane order after it,
// and records each element's slot index by dense index for the gather.
template <bool FILL, bool WIDE>
__global__ void k_nb_pass(uint32_t V, const uint32_t* __restrict__ off, NetSlots sl, int vertices, uint32_t n, int B,
                          NetBuckets t) {
    const int lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    const uint32_t groups = (V + 31) / 32;
    for (uint32_t g = blockIdx.x * wpb + (threadIdx.x >> 5); g < groups; g += gridDim.x * wpb) {
        const uint32_t v0 = g * 32, v = v0 + lane;
        const uint32_t o = v < V ? off[v] : 0xffffffffu;  // non-decreasing over the lanes
        const uint32_t base = v < V ? sl.base[v] : 0u;
        const uint32_t d0 = __shfl_sync(kFull, o, 0);
        const uint32_t d1 = off[v0 + 32 < V ? v0 + 32 : V];
        for (uint32_t j0 = d0; j0 < d1; j0 += 32) {
            const uint32_t j = j0 + lane;  // dense index
            const bool on = j < d1;
            int L = 0;  // the last slot whose offset is <= j
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
                if (__shfl_sync(kFull, o, L + step) <= j) L += step;
            const uint32_t e = __shfl_sync(kFull, base, L) + (j - __shfl_sync(kFull, o, L));
            uint4 id = make_uint4(0u, 0u, 0u, 0u);
            uint32_t bk = 0xffffffffu;
            if (on) {
                id = net_ids(sl, e, vertices);
                bk = net_bucket(id.x, n);
            }
            const unsigned grp = __match_any_sync(kFull, bk);
            const int leader = __ffs(grp) - 1;
            uint32_t r = 0;
            if (on && lane == leader) r = atomicAdd(FILL ? &t.cur[bk] : &t.cnt[bk], (uint32_t)__popc(grp));
            if constexpr (FILL) {
                r = __shfl_sync(kFull, r, leader);
                if (on) {
                    const uint32_t pos = t.off[bk] + r + (uint32_t)__popc(grp & ((1u << lane) - 1u));
                    nb_key<WIDE>(id, vertices, n, B, j).store(t.k1, t.k2, t.idx, pos);
                    t.srcd[j] = e;
                }
            }
        }
    }
}

// Bitonic sort of the N = 32 E elements a warp holds in registers, element index
// i = 32 r + lane in register r: distances below 32 exchange through shuffles, larger
// ones between a thread's own registers.  Elements past the bucket hold the padding key.
template <bool WIDE, int E>
__device__ __forceinline__ void warp_bitonic(NbKey<WIDE> (&x)[E]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32 * E; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const int r2 = r ^ (j >> 5);
                    if (r2 < r) continue;
                    const bool up = ((32 * r + lane) & k) == 0;  // this block ascending
                    if (up ? x[r2].less(x[r]) : x[r].less(x[r2])) {
                        const NbKey<WIDE> tmp = x[r];
                        x[r] = x[r2];
                        x[r2] = tmp;
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const NbKey<WIDE> y = x[r].xor_lane(j);
                    const int i = 32 * r + lane;
                    const bool keep_min = ((i & j) == 0) == ((i & k) == 0);
                    if (keep_min ? y.less(x[r]) : x[r].less(y)) x[r] = y;
                }
            }
        }
    }
}

// One bucket of c <= 32 E elements at o: sorted in registers, then the dense index of the
// first of each run of equal ids written, in order, to the start of the bucket's range.
template <bool WIDE, int E>
__device__ __forceinline__ void warp_bucket(NetBuckets& t, uint32_t bk, uint32_t o, uint32_t c) {
    const int lane = threadIdx.x & 31;
    NbKey<WIDE> x[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const uint32_t i = 32 * r + lane;
        x[r] = i < c ? NbKey<WIDE>::load(t.k1, t.k2, t.idx, o + i) : NbKey<WIDE>::pad();
    }
    if (c > 1) warp_bitonic<WIDE, E>(x);
    uint32_t u = 0;
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const uint32_t i = 32 * r + lane;
        NbKey<WIDE> p = x[r].up_lane();
        if (r > 0) {  // lane 0's predecessor is lane 31 of the previous register
            const NbKey<WIDE> q = x[r > 0 ? r - 1 : 0].from_lane(31);
            if (lane == 0) p = q;
        }
        const bool first = i < c && (i == 0 || !p.same_ids(x[r]));
        const unsigned fm = __ballot_sync(kFull, first);
        if (first) t.idx[o + u + __popc(fm & ((1u << lane) - 1u))] = x[r].j;
        u += (uint32_t)__popc(fm);
    }
    if (lane == 0) t.ucnt[bk] = u;
}

// The per-warp hash table of warp_bucket_distinct (256 slots: keys, smallest dense index),
// for blocks of at most 8 warps.
__device__ __forceinline__ unsigned long long* warp_hash_keys() {
    __shared__ unsigned long long s_keys[8][256];
    return s_keys[threadIdx.x >> 5];
}
__device__ __forceinline__ uint32_t* warp_hash_first() {
    __shared__ uint32_t s_first[8][256];
    return s_first[threadIdx.x >> 5];
}

// Narrow keys, a bucket of 33 to 32 E elements: most of a bucket repeats (a vertex sits
// in up to six contours, an edge in three), so the warp first keeps each id tuple's first
// occurrence (the smallest dense index) through an open-addressing table in shared memory
// (twice as many slots as elements, multiplicative hashing, linear probing), then sorts
// only those, one per lane, and writes their dense indices in id order.  Returns false,
// having written nothing, when more than 32 distinct tuples remain.
template <int E>
__device__ __forceinline__ bool warp_bucket_distinct(NetBuckets& t, uint32_t bk, uint32_t o, uint32_t c) {
    const int lane = threadIdx.x & 31;
    constexpr int bits = E <= 2 ? 7 : 8;
    constexpr uint32_t T = 1u << bits;
    unsigned long long* hk = warp_hash_keys();
    uint32_t* hj = warp_hash_first();
    __syncwarp();  // the previous bucket's reads of the table are done
    for (uint32_t k = lane; k < T; k += 32) {
        hk[k] = ~0ull;
        hj[k] = 0xffffffffu;
    }
    __syncwarp();
    NbKey<false> x[E];
    uint32_t slot[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const uint32_t i = 32 * r + lane;
        slot[r] = 0;
        x[r] = NbKey<false>::pad();
        if (i < c) {
            x[r] = NbKey<false>::load(t.k1, t.k2, t.idx, o + i);
            uint32_t h = (uint32_t)((x[r].k1 * 0x9E3779B97F4A7C15ull) >> (64 - bits));
            for (uint32_t probe = 0; probe < T; ++probe) {  // T > 2 c: a free slot exists
                const unsigned long long prev = atomicCAS(&hk[h], ~0ull, x[r].k1);
                if (prev == ~0ull || prev == x[r].k1) break;
                h = (h + 1) & (T - 1);
            }
            atomicMin(&hj[h], x[r].j);
            slot[r] = h;
        }
    }
    __syncwarp();
    bool rep[E];
    uint32_t U = 0;
#pragma unroll
    for (int r = 0; r < E; ++r) {
        rep[r] = 32 * r + lane < c && hj[slot[r]] == x[r].j;
        U += (uint32_t)__popc(__ballot_sync(kFull, rep[r]));
    }
    if (U > 32) return false;
    __syncwarp();  // all reads of the table done: its first 32 slots take the survivors
    uint32_t base = 0;
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const unsigned m = __ballot_sync(kFull, rep[r]);
        if (rep[r]) {
            const uint32_t at = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
            hk[at] = x[r].k1;
            hj[at] = x[r].j;
        }
        base += (uint32_t)__popc(m);
    }
    __syncwarp();
    NbKey<false> y[1];
    y[0] = (uint32_t)lane < U ? NbKey<false>{hk[lane], 0ull, hj[lane]} : NbKey<false>::pad();
    if (U > 1) warp_bitonic<false, 1>(y);
    if ((uint32_t)lane < U) t.idx[o + lane] = y[0].j;
    if (lane == 0) t.ucnt[bk] = U;
    return true;
}

// warp per bucket of at most kWarpSort elements (1, 2 or 4 per lane); larger buckets are
// listed for k_nb_sort_big
constexpr uint32_t kWarpSort = 128;
template <bool WIDE>
__global__ void k_nb_sort_small(uint32_t NB, NetBuckets t) {
    const int lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    for (uint32_t bk = blockIdx.x * wpb + (threadIdx.x >> 5); bk < NB; bk += gridDim.x * wpb) {
        const uint32_t o = t.off[bk], c = t.off[bk + 1] - o;
        if (c <= 32) {
            warp_bucket<WIDE, 1>(t, bk, o, c);
        } else if (c <= kWarpSort) {
            bool done = false;
            if constexpr (!WIDE)
                done = c <= 64 ? warp_bucket_distinct<2>(t, bk, o, c) : warp_bucket_distinct<4>(t, bk, o, c);
            if (!done) {
                if (c <= 64)
                    warp_bucket<WIDE, 2>(t, bk, o, c);
                else
                    warp_bucket<WIDE, 4>(t, bk, o, c);
            }
        } else if (lane == 0) {
            t.big[atomicAdd(t.big + NB, 1u)] = bk;
        }
    }
}

// One bitonic sort of c elements across a block, all comparators ascending (each merge
// starts by comparing mirrored positions), so that positions past c act as the largest
// keys and are never touched: sorts any c in place.
template <bool WIDE>
__device__ void block_bitonic(unsigned long long* k1, unsigned long long* k2, uint32_t* js, uint32_t c) {
    uint32_t N = 1;
    while (N < c) N <<= 1;
    for (uint32_t k = 2; k <= N; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t q = threadIdx.x; q < N / 2; q += blockDim.x) {
                const uint32_t i = (q / j) * 2 * j + (q % j);
                const uint32_t l = j == (k >> 1) ? (i ^ (k - 1)) : (i + j);
                if (l < c) {
                    const NbKey<WIDE> a = NbKey<WIDE>::load(k1, k2, js, i), b = NbKey<WIDE>::load(k1, k2, js, l);
                    if (b.less(a)) {
                        b.store(k1, k2, js, i);
                        a.store(k1, k2, js, l);
                    }
                }
            }
            __syncthreads();
        }
    }
}

// block per listed bucket of more than kWarpSort elements: sorted in shared memory up to
// kBigSmem elements, in place in global memory beyond; then warp 0 writes the dense index
// of the first of each run of equal ids to the start of the bucket's range (positions at
// or before the one being read, so the in-place form reads every element before it is
// overwritten).
template <bool WIDE>
__global__ void __launch_bounds__(256) k_nb_sort_big(uint32_t NB, NetBuckets t) {
    __shared__ unsigned long long s1[kBigSmem], s2[WIDE ? kBigSmem : 1];
    __shared__ uint32_t sj[kBigSmem];
    const uint32_t count = t.big[NB];
    const int lane = threadIdx.x & 31;
    for (uint32_t it = blockIdx.x; it < count; it += gridDim.x) {
        const uint32_t bk = t.big[it];
        const uint32_t o = t.off[bk], c = t.off[bk + 1] - o;
        unsigned long long *K1 = t.k1 + o, *K2 = WIDE ? t.k2 + o : nullptr;
        uint32_t* J = t.idx + o;
        if (c <= (uint32_t)kBigSmem) {
            for (uint32_t i = threadIdx.x; i < c; i += blockDim.x)
                NbKey<WIDE>::load(K1, K2, J, i).store(s1, s2, sj, i);
            __syncthreads();
            K1 = s1;
            K2 = s2;
            J = sj;
        }
        block_bitonic<WIDE>(K1, K2, J, c);
        if (threadIdx.x < 32) {
            uint32_t u = 0;
            NbKey<WIDE> q = NbKey<WIDE>::pad();
            for (uint32_t base = 0; base < c; base += 32) {
                const uint32_t i = base + lane;
                const bool in = i < c;
                const NbKey<WIDE> x = in ? NbKey<WIDE>::load(K1, K2, J, i) : NbKey<WIDE>::pad();
                NbKey<WIDE> p = x.up_lane();
                if (lane == 0) p = q;
                const bool first = in && (i == 0 || !p.same_ids(x));
                const unsigned fm = __ballot_sync(kFull, first);
                if (first) t.idx[o + u + __popc(fm & ((1u << lane) - 1u))] = x.j;
                u += (uint32_t)__popc(fm);
                q = x.from_lane(31);
            }
            if (lane == 0) t.ucnt[bk] = u;
        }
        __syncthreads();
    }
}

// warp per bucket: its distinct elements to the output, at uoff[bucket]
__global__ void k_nb_gather(uint32_t NB, NetBuckets t, NetSlots sl, int vertices, uint32_t* __restrict__ out_ids,
                            double* __restrict__ out_vals) {
    const int lane = threadIdx.x & 31;
    const uint32_t wpb = blockDim.x >> 5;
    for (uint32_t bk = blockIdx.x * wpb + (threadIdx.x >> 5); bk < NB; bk += gridDim.x * wpb) {
        const uint32_t u = t.ucnt[bk], o = t.off[bk], uo = t.uoff[bk];
        for (uint32_t j = lane; j < u; j += 32) {
            const uint32_t s = t.srcd[t.idx[o + j]];
            const size_t w = (size_t)uo + j;
            if (vertices) {
                const uint4 id = net_vid(sl, s);
                out_ids[4 * w] = id.x;
                out_ids[4 * w + 1] = id.y;
                out_ids[4 * w + 2] = id.z;
                out_ids[4 * w + 3] = id.w;
                for (int k = 0; k < 3; ++k) out_vals[3 * w + k] = net_vxyz(sl, s, k);
            } else {
                const uint4 id = net_eid(sl, s);
                out_ids[3 * w] = id.x;
                out_ids[3 * w + 1] = id.y;
                out_ids[3 * w + 2] = id.z;
                out_vals[w] = net_elen(sl, s);
            }
        }
    }
}

int gw(size_t items) { return grid_blocks(items, 8, 148 * 32); }  // 8 warps per 256-thread block

template <bool WIDE>
void dedup_kernels(uint32_t V, const uint32_t* off, const NetSlots& sl, int vertices, uint32_t n, int B,
                   NetBuckets t, uint32_t* scan_tmp, cudaStream_t s) {
    const uint32_t NB = n + 1;
    const size_t groups = ((size_t)V + 31) / 32;
    k_nb_pass<false, WIDE><<<gw(groups), 256, 0, s>>>(V, off, sl, vertices, n, B, t); count_launch();
    scan_u32(t.cnt, t.off, NB, scan_tmp, s);
    k_nb_pass<true, WIDE><<<gw(groups), 256, 0, s>>>(V, off, sl, vertices, n, B, t); count_launch();
    k_nb_sort_small<WIDE><<<gw(NB), 256, 0, s>>>(NB, t); count_launch();
    k_nb_sort_big<WIDE><<<148 * 4, 256, 0, s>>>(NB, t); count_launch();
    scan_u32(t.ucnt, t.uoff, NB, scan_tmp, s);
}

}  // namespace

int net_key_bits(uint32_t n) {
    int B = 1;
    while (B < 32 && ((uint64_t)1 << B) <= (uint64_t)n) ++B;  // 2^B > n: ids 0..n-1 and NULL as n
    return B;
}

void launch_net_dedup(uint32_t V, const uint32_t* off, const NetSlots& sl, int vertices, int wide, uint32_t n,
                      NetBuckets t, uint32_t* scan_tmp, cudaStream_t s) {
    const uint32_t NB = n + 1;
    cudaMemsetAsync(t.cnt, 0, 4 * (size_t)NB, s);
    cudaMemsetAsync(t.cur, 0, 4 * (size_t)NB, s);
    cudaMemsetAsync(t.big + NB, 0, 4, s);
    const int B = net_key_bits(n);
    if (vertices && (wide || 3 * B > 64))
        dedup_kernels<true>(V, off, sl, vertices, n, B, t, scan_tmp, s);
    else
        dedup_kernels<false>(V, off, sl, vertices, n, B, t, scan_tmp, s);
}
void launch_net_dedup_gather(uint32_t n, const NetBuckets& t, const NetSlots& sl, int vertices, uint32_t* out_ids,
                             double* out_vals, cudaStream_t s) {
    const uint32_t NB = n + 1;
    k_nb_gather<<<gw(NB), 256, 0, s>>>(NB, t, sl, vertices, out_ids, out_vals); count_launch();
}

}  // namespace vt
