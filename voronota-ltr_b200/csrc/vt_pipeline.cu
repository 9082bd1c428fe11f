// vt_pipeline.cu -- grid build, neighbour search, pair list, cells, periodic dedup,
// output compaction and totals.  All arithmetic here is FP64 and follows the reference
// operation by operation (compiled with --fmad=false).
#include <atomic>
#include <cfloat>
#include <cmath>

#include "vt_geom.cuh"
#include "vt_pipeline.cuh"

namespace vt {

namespace {

constexpr int kBlock = 256;
constexpr int kSearchWarps = 4;  // warps per block of the search kernels
constexpr int kCellWarps = 8;

__device__ __forceinline__ Sph<double> sph_of(double4 v) { return {{v.x, v.y, v.z}, v.w}; }

// ---- prepare: R = r + probe (types.rs:58-63) and the bounding-box partials ----
__global__ void k_prepare(const double* __restrict__ xyzr, uint32_t n, double probe, double4* __restrict__ sph,
                          uint32_t* __restrict__ slot_id, BBox* __restrict__ partials, uint32_t* __restrict__ err) {
    __shared__ double s[7][kBlock];
    double mn0 = DBL_MAX, mn1 = DBL_MAX, mn2 = DBL_MAX, mx0 = -DBL_MAX, mx1 = -DBL_MAX, mx2 = -DBL_MAX, mr = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x = xyzr[4 * (size_t)i], y = xyzr[4 * (size_t)i + 1], z = xyzr[4 * (size_t)i + 2];
        double r = xyzr[4 * (size_t)i + 3];
        double R = r + probe;
        if (!isfinite(x) || !isfinite(y) || !isfinite(z) || !isfinite(r) || r < 0.0) atomicOr(err, (uint32_t)kErrInvalid);
        sph[i] = make_double4(x, y, z, R);
        slot_id[i] = i;
        mn0 = fmin(mn0, x);
        mn1 = fmin(mn1, y);
        mn2 = fmin(mn2, z);
        mx0 = fmax(mx0, x);
        mx1 = fmax(mx1, y);
        mx2 = fmax(mx2, z);
        mr = fmax(mr, R);
    }
    int t = threadIdx.x;
    s[0][t] = mn0;
    s[1][t] = mn1;
    s[2][t] = mn2;
    s[3][t] = mx0;
    s[4][t] = mx1;
    s[5][t] = mx2;
    s[6][t] = mr;
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (t < o) {
            for (int k = 0; k < 3; ++k) s[k][t] = fmin(s[k][t], s[k][t + o]);
            for (int k = 3; k < 7; ++k) s[k][t] = fmax(s[k][t], s[k][t + o]);
        }
        __syncthreads();
    }
    if (t == 0) {
        BBox b;
        for (int k = 0; k < 3; ++k) {
            b.mn[k] = s[k][0];
            b.mx[k] = s[k + 3][0];
        }
        b.max_r = s[6][0];
        partials[blockIdx.x] = b;
    }
}

__global__ void k_bbox_final(const BBox* __restrict__ p, int nb, BBox* out) {
    __shared__ double s[7][kBlock];
    const int t = threadIdx.x;
    double v[7] = {DBL_MAX, DBL_MAX, DBL_MAX, -DBL_MAX, -DBL_MAX, -DBL_MAX, 0.0};
    for (int i = t; i < nb; i += blockDim.x) {
        for (int k = 0; k < 3; ++k) {
            v[k] = fmin(v[k], p[i].mn[k]);
            v[k + 3] = fmax(v[k + 3], p[i].mx[k]);
        }
        v[6] = fmax(v[6], p[i].max_r);
    }
    for (int k = 0; k < 7; ++k) s[k][t] = v[k];
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (t < o) {
            for (int k = 0; k < 3; ++k) s[k][t] = fmin(s[k][t], s[k][t + o]);
            for (int k = 3; k < 7; ++k) s[k][t] = fmax(s[k][t], s[k][t + o]);
        }
        __syncthreads();
    }
    if (t == 0) {
        BBox b;
        for (int k = 0; k < 3; ++k) {
            b.mn[k] = s[k][0];
            b.mx[k] = s[k + 3][0];
        }
        b.max_r = s[6][0];
        *out = b;
    }
}

// ---- periodic images (types.rs:323-375): only images within `reach` of the balls'
// bounding box can intersect a ball, so only those are materialised.
struct PBoxArg {
    double v[9];
};
__device__ __forceinline__ bool in_reach(double4 p, const BBox& bb, double reach) {
    return p.x >= bb.mn[0] - reach && p.x <= bb.mx[0] + reach && p.y >= bb.mn[1] - reach &&
           p.y <= bb.mx[1] + reach && p.z >= bb.mn[2] - reach && p.z <= bb.mx[2] + reach;
}
__global__ void k_image_count(const double4* __restrict__ sph, uint32_t n, PBoxArg pb, const BBox* __restrict__ bb,
                              double reach, uint32_t* __restrict__ cnt) {
    BBox b = *bb;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double4 s = sph[j];
        uint32_t c = 0;
        for (int g = 0; g < 26; ++g) {
            int sx, sy, sz;
            neighbor_shift(g, sx, sy, sz);
            if (in_reach(shift_sphere(s, pb.v, sx, sy, sz), b, reach)) ++c;
        }
        cnt[j] = c;
    }
}
__global__ void k_image_fill(double4* __restrict__ sph, uint32_t* __restrict__ slot_id, uint32_t n, PBoxArg pb,
                             const BBox* __restrict__ bb, double reach, const uint32_t* __restrict__ off,
                             uint32_t* __restrict__ d_nslots) {
    BBox b = *bb;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double4 s = sph[j];
        uint32_t o = n + off[j];
        for (int g = 0; g < 26; ++g) {
            int sx, sy, sz;
            neighbor_shift(g, sx, sy, sz);
            double4 p = shift_sphere(s, pb.v, sx, sy, sz);
            if (in_reach(p, b, reach)) {
                sph[o] = p;
                slot_id[o] = (uint32_t)(g + 1) * n + j;
                ++o;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_nslots = n + off[n];
}

// ---- uniform grid: counting sort of the slots by cell ----
__global__ void k_cell_hist(const double4* __restrict__ sph, const uint32_t* __restrict__ d_nslots, GridDev g,
                            uint32_t* __restrict__ cnt) {
    uint32_t ns = *d_nslots;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x)
        atomicAdd(&cnt[slot_cell(g, sph[s])], 1u);
}
__global__ void k_cell_scatter(const double4* __restrict__ sph, const uint32_t* __restrict__ slot_id,
                               const uint32_t* __restrict__ d_nslots, GridDev g, uint32_t* __restrict__ cursor,
                               double4* __restrict__ c_pos, uint32_t* __restrict__ c_id, uint32_t* __restrict__ c_slot,
                               int slot_is_id) {
    uint32_t ns = *d_nslots;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
        double4 p = sph[s];
        uint32_t at = atomicAdd(&cursor[slot_cell(g, p)], 1u);
        c_pos[at] = p;
        c_id[at] = slot_id[s];
        c_slot[at] = slot_is_id ? slot_id[s] : s;
    }
}

// ---- neighbour search: find_colliding_ids (spheres_searcher.rs:253-326), one warp per
// ball over the 3x3x3 cell stencil (9 contiguous rows of 3 cells in key order).
__device__ __forceinline__ bool same_group(const int32_t* g, uint64_t ng, uint32_t a, uint32_t b) {
    return g != nullptr && a < ng && b < ng && g[a] == g[b];  // tessellation.rs:323-328
}
__device__ __forceinline__ bool vless(double va, uint32_t ia, double vb, uint32_t ib) {
    // ValuedId::cmp (types.rs:176-184): by value, ties and NaN by index
    if (va < vb) return true;
    if (va > vb) return false;
    return ia < ib;
}

// The count pass waits on candidate loads: 9 resident blocks (56 registers) hide a little
// more of that latency than the 8 that 64 registers allow.
// Resident blocks per SM: the count pass at 9 (56 registers); the fill pass at 7, as many as
// its 16 KB of sort buffers allow under the default carveout (71 registers, no spill; 95
// registers and 5 blocks left it latency bound: 0.57 -> 0.47 ms at 100k balls).
template <bool FILL>
__global__ void __launch_bounds__(kSearchWarps * 32, FILL ? 7 : 9) k_search(DevBufs b, int want_rel) {
    __shared__ double s_val[kSearchWarps][kSortCap];
    __shared__ uint32_t s_id[kSearchWarps][kSortCap];
    __shared__ uint32_t s_slot[kSearchWarps][kSortCap];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    GridDev g = b.grid;
    uint32_t cbase = 0;  // first cell of the ball's structure (batched grids)
    const uint32_t n = b.n;
    Dec<double, false> d;
    const uint32_t rows = b.frontier ? b.n_frontier : n;
    for (uint32_t row = blockIdx.x * kSearchWarps + w; row < rows; row += gridDim.x * kSearchWarps) {
        const uint32_t i = b.frontier ? b.frontier[row] : row;
        if (b.grids) {
            const uint32_t st = b.ball_struct[i];
            g = b.grids[st];
            cbase = b.cell_base[st];
        }
        const double4 A4 = b.sph[i];
        const Sph<double> A = sph_of(A4);
        // a row longer than the warp sort buffer is written unsorted to the CSR by the
        // fill pass and sorted there by k_big_sort
        const uint32_t row_cnt = FILL ? b.nb_cnt[row] : 0u;
        const bool big = row_cnt > (uint32_t)kSortCap;
        const uint32_t off = FILL ? b.nb_off[row] : 0u;
        uint32_t hits = 0, np = 0;
        bool hidden = false;
        // fill pass of a row whose hits the count pass listed (at most kHitCap): read them
        // instead of scanning the stencil again
        if (FILL && b.hit_idx && row_cnt <= (uint32_t)kHitCap) {
            if constexpr (FILL) {
                for (uint32_t e = lane; e < row_cnt; e += 32) {
                    const uint32_t idx = b.hit_idx[(size_t)row * kHitCap + e];
                    s_val[w][e] = dist_to_ic_center(A, sph_of(b.c_pos[idx]));  // spheres_searcher.rs:312-316
                    s_id[w][e] = b.c_id[idx];
                    s_slot[w][e] = b.c_slot[idx];
                }
            }
            hits = row_cnt;
        } else {
        int cx = cell_coord(A4.x, g.ox, g.cell, g.dx), cy = cell_coord(A4.y, g.oy, g.cell, g.dy),
            cz = cell_coord(A4.z, g.oz, g.cell, g.dz);
        // stencil rows (y, z) of up to 2 half + 1 cells in x, one per lane; a row whose y and
        // z slabs lie beyond the reach from the centre is empty, and a row's x-range is cut
        // to the cells within reach (every intersecting ball is closer than the reach, and
        // floor is monotone, so the cut loses none)
        const int side = 2 * g.half + 1;
        uint32_t rbeg = 0, rcnt = 0;
        if (lane < side * side) {
            const int y = cy + lane / side - g.half, z = cz + lane % side - g.half;
            if (y >= 0 && y < g.dy && z >= 0 && z < g.dz) {
                const double ylo = g.oy + y * g.cell, zlo = g.oz + z * g.cell;
                const double ey = fmax(fmax(ylo - A4.y, A4.y - (ylo + g.cell)), 0.0);
                const double ez = fmax(fmax(zlo - A4.z, A4.z - (zlo + g.cell)), 0.0);
                const double rem = g.reach * g.reach - ey * ey - ez * ez;
                if (rem >= 0.0) {
                    const double ext = sqrt(rem);
                    int x0 = cell_coord(A4.x - ext, g.ox, g.cell, g.dx), x1 = cell_coord(A4.x + ext, g.ox, g.cell, g.dx);
                    x0 = x0 > cx - g.half ? x0 : cx - g.half;
                    x1 = x1 < cx + g.half ? x1 : cx + g.half;
                    if (x0 <= x1) {
                        rbeg = b.cell_start[cbase + cell_key(g, x0, y, z)];
                        rcnt = b.cell_start[cbase + cell_key(g, x1, y, z) + 1] - rbeg;
                    }
                }
            }
        }
        uint32_t incl = rcnt;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t t0 = 0; t0 < total && !hidden; t0 += 32) {
            uint32_t t = t0 + lane;
            bool hit = false, hid = false;
            double val = 0.0;
            uint32_t cid = 0, cslot = 0;
            // candidate t lies in the first row whose inclusive count exceeds it
            int r = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const uint32_t v = __shfl_sync(0xffffffffu, incl, r + step - 1);
                if (v <= t) r += step;
            }
            r = r > 31 ? 31 : r;
            const uint32_t r_end = __shfl_sync(0xffffffffu, incl, r);
            const uint32_t r_cnt = __shfl_sync(0xffffffffu, rcnt, r);
            const uint32_t r_beg = __shfl_sync(0xffffffffu, rbeg, r);
            uint32_t idx = 0;
            if (t < total) {
                idx = r_beg + (t - (r_end - r_cnt));
                cid = b.c_id[idx];
                if (cid != i) {
                    const Sph<double> C = sph_of(b.c_pos[idx]);
                    if (sphere_intersects(d, A, C, 0.0)) {
                        // hidden central ball (spheres_searcher.rs:295-303)
                        bool eqs = fabs(C.r - A.r) <= kEps && fabs(C.c.x - A.c.x) <= kEps &&
                                   fabs(C.c.y - A.c.y) <= kEps && fabs(C.c.z - A.c.z) <= kEps;
                        if (sphere_contains(d, C, A, 0.0, 0.0) && (!eqs || i > cid)) {
                            hid = true;
                        } else if (!sphere_contains(d, A, C, 0.0, 0.0)) {  // :305-310
                            hit = true;
                            val = dist_to_ic_center(A, C);  // :312-316
                            cslot = b.c_slot[idx];
                        }
                    }
                }
            }
            if (__any_sync(0xffffffffu, hid)) {
                hidden = true;
                break;
            }
            unsigned m = __ballot_sync(0xffffffffu, hit);
            uint32_t pos = hits + __popc(m & ((1u << lane) - 1u));
            if constexpr (FILL) {
                if (hit) {
                    if (big) {
                        if (pos < row_cnt) {  // the count pass found exactly row_cnt
                            b.nb_id[off + pos] = cid;
                            b.nb_slot[off + pos] = cslot;
                            b.nb_val[off + pos] = val;
                        }
                    } else if (pos < (uint32_t)kSortCap) {
                        s_val[w][pos] = val;
                        s_id[w][pos] = cid;
                        s_slot[w][pos] = cslot;
                    }
                }
            }
            if (!FILL && hit && b.hit_idx && pos < (uint32_t)kHitCap)
                b.hit_idx[(size_t)row * kHitCap + pos] = idx;  // for the fill pass
            if (!FILL) {  // pairs this ball generates (collect_collision_pairs, tessellation.rs:298-319)
                const uint32_t bc = b.periodic ? cid % n : cid;
                const bool gen = hit && !b.no_pairs && !same_group(b.groups, b.n_groups, i, bc) &&
                                 ((b.periodic && cid >= n) || i < cid);
                np += __popc(__ballot_sync(0xffffffffu, gen));
            }
            hits += __popc(m);
        }
        }  // stencil scan
        const uint32_t cnt = hidden ? 0 : hits;
        __syncwarp();
        if (!FILL) {
            if (lane == 0) {
                b.nb_cnt[row] = cnt;
                if (!b.no_pairs) b.nb_npair[row] = hidden ? 0u : np;
                b.excluded[i] = hidden ? 1 : 0;
                if (cnt > (uint32_t)kSortCap) b.big_list[atomicAdd(b.d_big_count, 1u)] = row;
            }
            __syncwarp();
            continue;
        }
        if (big) continue;
        // bitonic sort of (value, id) (spheres_searcher.rs:324); keys are distinct within a
        // row.  Up to 64 entries (nearly every ball): in registers, two per lane, partners
        // exchanged by shuffles; longer rows: in shared memory.
        uint32_t n2 = 2;
        while (n2 < cnt) n2 <<= 1;
        if (n2 <= 64) {
            double v[2];
            uint32_t id[2], sl[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t t = lane + 32u * h;
                v[h] = t < cnt ? s_val[w][t] : INFINITY;
                id[h] = t < cnt ? s_id[w][t] : 0xffffffffu;
                sl[h] = t < cnt ? s_slot[w][t] : 0u;
            }
            for (uint32_t k = 2; k <= n2; k <<= 1) {
                for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
                    if (jj == 32) {  // k = 64: element lane against lane + 32, ascending
                        if (vless(v[1], id[1], v[0], id[0])) {
                            const double tv = v[0];
                            const uint32_t ti = id[0], ts = sl[0];
                            v[0] = v[1];
                            id[0] = id[1];
                            sl[0] = sl[1];
                            v[1] = tv;
                            id[1] = ti;
                            sl[1] = ts;
                        }
                        continue;
                    }
                    const bool lower = (lane & jj) == 0;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint32_t t = lane + 32u * h;
                        const double pv = __shfl_xor_sync(0xffffffffu, v[h], jj);
                        const uint32_t pi = __shfl_xor_sync(0xffffffffu, id[h], jj);
                        const uint32_t ps = __shfl_xor_sync(0xffffffffu, sl[h], jj);
                        const bool keep_min = lower == ((t & k) == 0);
                        const bool take = keep_min ? vless(pv, pi, v[h], id[h]) : vless(v[h], id[h], pv, pi);
                        if (take) {
                            v[h] = pv;
                            id[h] = pi;
                            sl[h] = ps;
                        }
                    }
                }
            }
            __syncwarp();
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t t = lane + 32u * h;
                if (t < cnt) {
                    s_val[w][t] = v[h];
                    s_id[w][t] = id[h];
                    s_slot[w][t] = sl[h];
                }
            }
            __syncwarp();
        } else {
            for (uint32_t e = cnt + lane; e < n2; e += 32) {
                s_val[w][e] = INFINITY;
                s_id[w][e] = 0xffffffffu;
                s_slot[w][e] = 0;
            }
            __syncwarp();
            for (uint32_t k = 2; k <= n2; k <<= 1) {
                for (uint32_t jj = k >> 1; jj > 0; jj >>= 1) {
                    for (uint32_t t = lane; t < n2; t += 32) {
                        uint32_t ixj = t ^ jj;
                        if (ixj > t) {
                            bool up = (t & k) == 0;
                            double vt = s_val[w][t], vx = s_val[w][ixj];
                            uint32_t it = s_id[w][t], ix = s_id[w][ixj];
                            bool sw = up ? vless(vx, ix, vt, it) : vless(vt, it, vx, ix);
                            if (sw) {
                                s_val[w][t] = vx;
                                s_val[w][ixj] = vt;
                                s_id[w][t] = ix;
                                s_id[w][ixj] = it;
                                uint32_t st = s_slot[w][t];
                                s_slot[w][t] = s_slot[w][ixj];
                                s_slot[w][ixj] = st;
                            }
                        }
                    }
                    __syncwarp();
                }
            }
        }
        uint32_t prank = b.no_pairs ? 0u : b.pair_off[row];
        for (uint32_t e0 = 0; e0 < cnt; e0 += 32) {
            uint32_t e = e0 + lane;
            bool gen = false;
            uint32_t bid = 0, bslot = 0;
            if (e < cnt) {
                bid = s_id[w][e];
                bslot = s_slot[w][e];
                uint32_t bc = b.periodic ? bid % n : bid;
                gen = !b.no_pairs && !same_group(b.groups, b.n_groups, i, bc) && ((b.periodic && bid >= n) || i < bid);
            }
            unsigned m = __ballot_sync(0xffffffffu, gen);
            if (e < cnt) {
                b.nb_id[off + e] = bid;
                b.nb_slot[off + e] = bslot;
                b.nb_val[off + e] = s_val[w][e];
                int32_t pidx = -1;
                if (gen) {
                    pidx = (int32_t)(prank + __popc(m & ((1u << lane) - 1u)));
                    b.pair_a[pidx] = i;
                    b.pair_e[pidx] = off + e;
                }
                if (!b.no_pairs) b.nb_pair[off + e] = pidx;
                if (want_rel) {
                    double4 C = b.sph[bslot];
                    b.nb_rel[off + e] = make_float4((float)(C.x - A4.x), (float)(C.y - A4.y), (float)(C.z - A4.z),
                                                    (float)C.w);
                }
            }
            prank += __popc(m);
        }
        __syncwarp();
    }
}

// ---- rows longer than the warp sort buffer: a block per row sorts the row in place in
// global memory by (value, id) with an ascending bitonic network over the next power of
// two (comparators reaching past the row's end are skipped: the missing elements act as
// +infinity), then generates the row's pairs in sorted order (block scan of the flags).
constexpr int kBigThreads = 1024;
__device__ __forceinline__ void big_cmpswap(const DevBufs& b, uint32_t lo, uint32_t hi) {
    const double vl = b.nb_val[lo], vh = b.nb_val[hi];
    const uint32_t il = b.nb_id[lo], ih = b.nb_id[hi];
    if (vless(vh, ih, vl, il)) {
        const uint32_t sl = b.nb_slot[lo], sh = b.nb_slot[hi];
        b.nb_val[lo] = vh;
        b.nb_val[hi] = vl;
        b.nb_id[lo] = ih;
        b.nb_id[hi] = il;
        b.nb_slot[lo] = sh;
        b.nb_slot[hi] = sl;
    }
}
__global__ void __launch_bounds__(kBigThreads) k_big_sort(DevBufs b, int want_rel) {
    __shared__ uint32_t s_warp[kBigThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint32_t n = b.n, nbig = *b.d_big_count;
    for (uint32_t k = blockIdx.x; k < nbig; k += gridDim.x) {
        const uint32_t row = b.big_list[k];
        const uint32_t i = b.frontier ? b.frontier[row] : row;
        const uint32_t off = b.nb_off[row], cnt = b.nb_cnt[row];
        uint32_t n2 = 1;
        while (n2 < cnt) n2 <<= 1;
        for (uint32_t size = 2; size <= n2; size <<= 1) {
            const uint32_t half = size >> 1;
            for (uint32_t t = tid; t < (n2 >> 1); t += kBigThreads) {  // flip step
                const uint32_t g = t / half, p = t % half;
                const uint32_t lo = g * size + p, hi = g * size + size - 1 - p;
                if (hi < cnt) big_cmpswap(b, off + lo, off + hi);
            }
            __syncthreads();
            for (uint32_t stride = half >> 1; stride > 0; stride >>= 1) {
                for (uint32_t t = tid; t < (n2 >> 1); t += kBigThreads) {
                    const uint32_t g = t / stride, p = t % stride;
                    const uint32_t lo = g * 2 * stride + p, hi = lo + stride;
                    if (hi < cnt) big_cmpswap(b, off + lo, off + hi);
                }
                __syncthreads();
            }
        }
        const double4 A4 = b.sph[i];
        uint32_t prank = b.no_pairs ? 0u : b.pair_off[row];
        for (uint32_t base = 0; base < cnt; base += kBigThreads) {
            const uint32_t e = base + tid;
            bool gen = false;
            uint32_t bid = 0;
            if (e < cnt) {
                bid = b.nb_id[off + e];
                const uint32_t bc = b.periodic ? bid % n : bid;
                gen = !b.no_pairs && !same_group(b.groups, b.n_groups, i, bc) && ((b.periodic && bid >= n) || i < bid);
            }
            const unsigned m = __ballot_sync(0xffffffffu, gen);
            if (lane == 0) s_warp[w] = __popc(m);
            __syncthreads();
            uint32_t before = 0, total = 0;
            for (int q = 0; q < kBigThreads / 32; ++q) {
                before += q < w ? s_warp[q] : 0u;
                total += s_warp[q];
            }
            if (e < cnt) {
                int32_t pidx = -1;
                if (gen) {
                    pidx = (int32_t)(prank + before + __popc(m & ((1u << lane) - 1u)));
                    b.pair_a[pidx] = i;
                    b.pair_e[pidx] = off + e;
                }
                if (!b.no_pairs) b.nb_pair[off + e] = pidx;
                if (want_rel) {
                    const double4 C = b.sph[b.nb_slot[off + e]];
                    b.nb_rel[off + e] = make_float4((float)(C.x - A4.x), (float)(C.y - A4.y), (float)(C.z - A4.z),
                                                    (float)C.w);
                }
            }
            prank += total;
            __syncthreads();
        }
    }
}

// ---- cells: compute_cells (tessellation.rs:607-658) as a per-ball warp reduction ----
__device__ __forceinline__ double wsum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Pair index of the pair between ball i and its neighbour entry e (CSR position):
// pairs (i, j) with j > i or j a periodic image sit in i's own list; pairs (j, i) with
// j < i are found by locating i in j's sorted list by its (value, id) key.
__device__ __forceinline__ int32_t incident_pair(const DevBufs& b, uint32_t i, double4 Si, uint32_t e,
                                                 bool* side_a) {
    const uint32_t n = b.n;
    uint32_t j = b.nb_id[e];
    *side_a = true;
    if ((b.periodic && j >= n) || j > i) return b.nb_pair[e];
    double v = dist_to_ic_center(sph_of(b.sph[j]), sph_of(Si));
    uint32_t lo = b.nb_off[j], hi = lo + b.nb_cnt[j];
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (vless(b.nb_val[mid], b.nb_id[mid], v, i))
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo < b.nb_off[j] + b.nb_cnt[j] && b.nb_id[lo] == i) {
        *side_a = false;
        return b.nb_pair[lo];
    }
    return -1;
}

// 5 resident blocks per SM (48 registers, no spill): the kernel waits on dependent loads
// (the binary searches), so warps in flight matter more than registers
__global__ void __launch_bounds__(kCellWarps * 32, 5) k_cells(DevBufs b, float cell_band, int only_dirty) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n = b.n;
    for (uint32_t i = blockIdx.x * kCellWarps + w; i < n; i += gridDim.x * kCellWarps) {
        if (only_dirty && !b.ball_dirty[i]) continue;
        const uint32_t cnt = b.nb_cnt[i], off = b.nb_off[i];
        const double4 Si = b.sph[i];
        double area = 0, arc = 0, spos = 0, sneg = 0, ppos = 0, pneg = 0;
        uint32_t count = 0;
        for (uint32_t e = lane; e < cnt; e += 32) {
            bool side_a;
            int32_t p = incident_pair(b, i, Si, off + e, &side_a);
            if (p >= 0 && (b.p_status[p] & kValid)) {
                double sa = side_a ? b.p_sa_a[p] : b.p_sa_b[p];
                double pv = side_a ? b.p_pv_a[p] : b.p_pv_b[p];
                ++count;
                area += b.p_area[p];
                arc += b.p_arc[p];
                spos += fmax(sa, 0.0);
                sneg -= fmin(sa, 0.0);
                ppos += fmax(pv, 0.0);
                pneg -= fmin(pv, 0.0);
            }
        }
        area = wsum_d(area);
        arc = wsum_d(arc);
        spos = wsum_d(spos);
        sneg = wsum_d(sneg);
        ppos = wsum_d(ppos);
        pneg = wsum_d(pneg);
        for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
        if (lane == 0) {
            const double r = Si.w;
            uint8_t flag = 0;
            double sas = 0.0, vol = 0.0;
            if (count > 0) {  // CellContactSummary::compute_sas (types.rs:623-663)
                flag = 1;
                bool unsure = false;
                cell_from_sums(count, arc, spos, sneg, ppos, pneg, r, cell_band, &unsure, &sas, &vol);
                if (unsure) {
                    uint32_t at = atomicAdd(b.d_cell_redo_count, 1u);
                    b.cell_redo_list[at] = i;
                }
            } else if (cnt == 0 && !(b.detached_excl && b.excluded[i])) {
                // compute_sas_detached (types.rs:666-675); the updateable tessellation also
                // requires the ball not to be excluded (updateable.rs:680-685)
                flag = 1;
                sas = 4.0 * kPi * r * r;
                vol = sas * r / 3.0;
            }
            b.cell_flag[i] = flag;
            b.cell_sas[i] = sas;
            b.cell_vol[i] = vol;
        }
    }
}

__global__ void __launch_bounds__(kCellWarps * 32) k_mark_ball_pairs(DevBufs b) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t m = *b.d_cell_redo_count;
    for (uint32_t k = blockIdx.x * kCellWarps + w; k < m; k += gridDim.x * kCellWarps) {
        const uint32_t i = b.cell_redo_list[k];
        const uint32_t cnt = b.nb_cnt[i], off = b.nb_off[i];
        const double4 Si = b.sph[i];
        if (lane == 0) b.ball_dirty[i] = 1;
        for (uint32_t e = lane; e < cnt; e += 32) {
            bool side_a;
            int32_t p = incident_pair(b, i, Si, off + e, &side_a);
            uint32_t j = b.nb_id[off + e];
            if (j < b.n) b.ball_dirty[j] = 1;
            if (p >= 0) {
                uint32_t at = atomicAdd(b.d_redo_count, 1u);
                b.redo_list[at] = (uint32_t)p;
            }
        }
    }
}

// ---- periodic dedup ----
// Full tessellation: compute_canonical_ids (tessellation.rs:556-601) keeps, among the
// boundary contacts (an id >= n), the first one in pair order per unordered canonical
// pair.  Contacts-only: deduplicate_and_canonicalize_contacts (tessellation.rs:172-188)
// keeps the first contact per canonical pair among all contacts.  Pair order is a-major,
// so earlier contacts with the same key sit in a's range before p or, when the canonical
// partner c is smaller than a, anywhere in c's range.
__device__ __forceinline__ bool earlier_same_key(const DevBufs& b, uint32_t lo, uint32_t hi, uint32_t want,
                                                 bool boundary_only) {
    const uint32_t n = b.n;
    for (uint32_t q = lo; q < hi; ++q) {
        if (!(b.p_status[q] & kValid)) continue;
        uint32_t bid = b.nb_id[b.pair_e[q]];
        if (boundary_only && bid < n) continue;
        if (bid % n == want) return true;
    }
    return false;
}
__global__ void k_dedup(DevBufs b, uint32_t P, int contacts_only) {
    const uint32_t n = b.n;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        uint32_t keep = 0;
        if (b.p_status[p] & kValid) {
            keep = 1;
            uint32_t a = b.pair_a[p];
            uint32_t bid = b.nb_id[b.pair_e[p]];
            bool boundary = bid >= n;
            if (contacts_only || boundary) {
                uint32_t c = bid % n;
                bool bo = !contacts_only;
                if (earlier_same_key(b, b.pair_off[a], p, c, bo)) keep = 0;
                if (keep && c < a && earlier_same_key(b, b.pair_off[c], b.pair_off[c + 1], a, bo)) keep = 0;
            }
        }
        b.keep[p] = keep;
    }
}
__global__ void k_keep_plain(DevBufs b, uint32_t P) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x)
        b.keep[p] = (b.p_status[p] & kValid) ? 1u : 0u;
}
__global__ void k_cell_keep(DevBufs b, uint32_t* flags32) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.n; i += gridDim.x * blockDim.x)
        flags32[i] = b.cell_flag[i];
}

// ---- output compaction (pair order, which is the reference's output order) ----
__global__ void k_compact_contacts(DevBufs b, uint32_t P, int contacts_only) {
    const uint32_t n = b.n;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        uint32_t o = b.keep_off[p];
        if (b.keep_off[p + 1] == o) continue;
        uint32_t a = b.pair_a[p];
        uint32_t bid = b.nb_id[b.pair_e[p]];
        uint32_t ia = a, ib = bid;
        if (b.periodic) {
            ia = a % n;
            ib = bid % n;
            if (contacts_only && ib < ia) {  // canonical (min, max)
                uint32_t t = ia;
                ia = ib;
                ib = t;
            }
        }
        b.out_a[o] = ia;
        b.out_b[o] = ib;
        b.out_area[o] = b.p_area[p];
        b.out_arc[o] = b.p_arc[p];
        b.out_central[o] = b.p_central[p];
    }
}
__global__ void k_compact_cells(DevBufs b) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.n; i += gridDim.x * blockDim.x) {
        uint32_t o = b.cell_off[i];
        if (b.cell_off[i + 1] == o) continue;
        b.out_cell_index[o] = i;
        b.out_cell_sas[o] = b.cell_sas[i];
        b.out_cell_vol[o] = b.cell_vol[i];
    }
}

// ---- deterministic totals: fixed grid, fixed tree ----
constexpr int kSumBlocks = 148;
__global__ void k_partial_sums(const double* __restrict__ x0, const uint32_t* __restrict__ cnt0,
                               const double* __restrict__ x1, const double* __restrict__ x2,
                               const uint32_t* __restrict__ cnt1, double* __restrict__ partials) {
    __shared__ double s[3][kBlock];
    uint32_t c0 = *cnt0, c1 = *cnt1;
    double a0 = 0, a1 = 0, a2 = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c0; i += gridDim.x * blockDim.x) a0 += x0[i];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c1; i += gridDim.x * blockDim.x) {
        a1 += x1[i];
        a2 += x2[i];
    }
    int t = threadIdx.x;
    s[0][t] = a0;
    s[1][t] = a1;
    s[2][t] = a2;
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (t < o)
            for (int k = 0; k < 3; ++k) s[k][t] += s[k][t + o];
        __syncthreads();
    }
    if (t < 3) partials[blockIdx.x * 3 + t] = s[t][0];
}
__global__ void k_final_sums(const double* __restrict__ partials, double* __restrict__ totals) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a = 0, s = 0, v = 0;
    for (int k = 0; k < kSumBlocks; ++k) {
        a += partials[3 * k];
        s += partials[3 * k + 1];
        v += partials[3 * k + 2];
    }
    totals[0] = s;
    totals[1] = v;
    totals[2] = a;
}

// ---- pairs that must be recomputed (FP32 unsure -> FP64 warp; overflow -> serial) ----
__global__ void k_collect_redo(DevBufs b, uint32_t P) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        uint8_t st = b.p_status[p];
        if (st & kOverflow) {
            uint32_t at = atomicAdd(b.d_serial_count, 1u);
            b.serial_list[at] = p;
        } else if (st & kUnsure) {
            uint32_t at = atomicAdd(b.d_redo_count, 1u);
            b.redo_list[at] = p;
        }
    }
}

// ---- exclusive scan of u32 (3 phases: tile sums, scan of tile sums, tile scan) ----
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kTile = kScanThreads * kScanPer;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t ws[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t y = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += t;
        }
        ws[lane] = y;
    }
    __syncthreads();
    uint32_t before = w > 0 ? ws[w - 1] : 0u;
    *total = ws[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t* __restrict__ in, size_t n,
                                                             uint32_t* __restrict__ tile_sums) {
    size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kScanPer;
    uint32_t s = 0;
    for (int k = 0; k < kScanPer; ++k)
        if (base + k < n) s += in[base + k];
    uint32_t total;
    block_excl_scan(s, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(uint32_t* __restrict__ sums, size_t ntiles) {
    // single block: exclusive scan of the tile sums in chunks, carrying the prefix
    uint32_t carry = 0;
    for (size_t base = 0; base < ntiles; base += kScanThreads) {
        size_t i = base + threadIdx.x;
        uint32_t v = i < ntiles ? sums[i] : 0u;
        uint32_t total;
        uint32_t ex = block_excl_scan(v, &total);
        if (i < ntiles) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) sums[ntiles] = carry;
}
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const uint32_t* __restrict__ in, size_t n,
                                                             const uint32_t* __restrict__ tile_off,
                                                             uint32_t* __restrict__ out, size_t ntiles) {
    size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kScanPer;
    uint32_t v[kScanPer];
    uint32_t s = 0;
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t ex = block_excl_scan(s, &total) + tile_off[blockIdx.x];
    for (int k = 0; k < kScanPer; ++k) {
        if (base + k < n) out[base + k] = ex;
        ex += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = tile_off[ntiles];
}

int grid_for(size_t n, int block, int cap = 148 * 16) {
    size_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > (size_t)cap) g = cap;
    return (int)g;
}

std::atomic<uint64_t> g_launches{0};

}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

size_t scan_tmp_words_needed(size_t n) { return (n + kTile - 1) / kTile + 2; }

void scan_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* tmp, cudaStream_t s) {
    size_t ntiles = (n + kTile - 1) / kTile;
    if (ntiles == 0) {
        cudaMemsetAsync(out, 0, sizeof(uint32_t), s);
        return;
    }
    k_scan_tiles<<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, n, tmp); count_launch();
    k_scan_sums<<<1, kScanThreads, 0, s>>>(tmp, ntiles); count_launch();
    k_scan_apply<<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, n, tmp, out, ntiles); count_launch();
}

void launch_prepare(const DevBufs& b, const double* d_xyzr, double probe, BBox* d_parts, int nblocks,
                    cudaStream_t s) {
    k_prepare<<<nblocks, kBlock, 0, s>>>(d_xyzr, b.n, probe, b.sph, b.slot_id, d_parts, b.err); count_launch();
}
void launch_bbox_final(const BBox* parts, int nblocks, BBox* out, cudaStream_t s) {
    k_bbox_final<<<1, kBlock, 0, s>>>(parts, nblocks, out); count_launch();
}
void launch_images(const DevBufs& b, double reach, const BBox* d_bbox, uint32_t* img_cnt, uint32_t* img_off,
                   uint32_t* scan_tmp, size_t, cudaStream_t s) {
    PBoxArg pb;
    for (int k = 0; k < 9; ++k) pb.v[k] = b.pbox[k];
    int gb = grid_for(b.n, kBlock);
    k_image_count<<<gb, kBlock, 0, s>>>(b.sph, b.n, pb, d_bbox, reach, img_cnt); count_launch();
    scan_u32(img_cnt, img_off, b.n, scan_tmp, s);
    k_image_fill<<<gb, kBlock, 0, s>>>(b.sph, b.slot_id, b.n, pb, d_bbox, reach, img_off, b.d_nslots); count_launch();
}
void launch_grid(const DevBufs& b, uint32_t ncell, uint32_t max_slots, uint32_t* scan_tmp, size_t, cudaStream_t s) {
    cudaMemsetAsync(b.cell_count, 0, sizeof(uint32_t) * ncell, s);
    int gb = grid_for(max_slots, kBlock);
    k_cell_hist<<<gb, kBlock, 0, s>>>(b.sph, b.d_nslots, b.grid, b.cell_count); count_launch();
    scan_u32(b.cell_count, b.cell_start, ncell, scan_tmp, s);
    cudaMemcpyAsync(b.cell_cursor, b.cell_start, sizeof(uint32_t) * ncell, cudaMemcpyDeviceToDevice, s);
    k_cell_scatter<<<gb, kBlock, 0, s>>>(b.sph, b.slot_id, b.d_nslots, b.grid, b.cell_cursor, b.c_pos, b.c_id,
                                         b.c_slot, b.slot_is_id); count_launch();
}
void launch_search_count(const DevBufs& b, cudaStream_t s) {
    cudaMemsetAsync(b.d_big_count, 0, sizeof(uint32_t), s);
    int gb = grid_for(b.n, kSearchWarps, 148 * 64);
    k_search<false><<<gb, kSearchWarps * 32, 0, s>>>(b, 0); count_launch();
}
void launch_search_fill(const DevBufs& b, int want_rel, uint32_t n_big, cudaStream_t s) {
    int gb = grid_for(b.n, kSearchWarps, 148 * 64);
    k_search<true><<<gb, kSearchWarps * 32, 0, s>>>(b, want_rel); count_launch();
    if (n_big) {
        k_big_sort<<<n_big < 148u * 2u ? n_big : 148u * 2u, kBigThreads, 0, s>>>(b, want_rel); count_launch();
    }
}
void launch_cells(const DevBufs& b, float cell_band, int only_dirty, cudaStream_t s) {
    int gb = grid_for(b.n, kCellWarps, 148 * 32);
    k_cells<<<gb, kCellWarps * 32, 0, s>>>(b, cell_band, only_dirty); count_launch();
}
void launch_mark_ball_pairs(const DevBufs& b, cudaStream_t s) {
    k_mark_ball_pairs<<<64, kCellWarps * 32, 0, s>>>(b); count_launch();
}
void launch_dedup(const DevBufs& b, uint32_t P, int contacts_only, cudaStream_t s) {
    int gb = grid_for(P, kBlock);
    if (b.periodic)
        k_dedup<<<gb, kBlock, 0, s>>>(b, P, contacts_only);
    else
        k_keep_plain<<<gb, kBlock, 0, s>>>(b, P);
    count_launch();
}
void launch_compact(const DevBufs& b, uint32_t P, int contacts_only, uint32_t* scan_tmp, size_t, cudaStream_t s) {
    scan_u32(b.keep, b.keep_off, P, scan_tmp, s);
    k_compact_contacts<<<grid_for(P, kBlock), kBlock, 0, s>>>(b, P, contacts_only); count_launch();
    if (!contacts_only) {
        // cell flags (u8) widened into the keep buffer's tail is avoided: use params_u
        k_cell_keep<<<grid_for(b.n, kBlock), kBlock, 0, s>>>(b, b.params_u); count_launch();
        scan_u32(b.params_u, b.cell_off, b.n, scan_tmp, s);
        k_compact_cells<<<grid_for(b.n, kBlock), kBlock, 0, s>>>(b); count_launch();
    }
}
void launch_totals(const DevBufs& b, uint32_t P, int contacts_only, cudaStream_t s) {
    const uint32_t* ccount = b.keep_off + P;
    const uint32_t* ncell = contacts_only ? b.keep_off + P : b.cell_off + b.n;
    if (contacts_only) {
        // no cells: the cell sums read zero elements from a zero count
        k_partial_sums<<<kSumBlocks, kBlock, 0, s>>>(b.out_area, ccount, b.out_area, b.out_area, b.zero_word,
                                                     b.partials); count_launch();
    } else {
        k_partial_sums<<<kSumBlocks, kBlock, 0, s>>>(b.out_area, ccount, b.out_cell_sas, b.out_cell_vol, ncell,
                                                     b.partials); count_launch();
    }
    k_final_sums<<<1, 32, 0, s>>>(b.partials, b.totals); count_launch();
}
void launch_sums3(const double* x0, const uint32_t* cnt0, const double* x1, const double* x2, const uint32_t* cnt1,
                  double* partials, double* totals, cudaStream_t s) {
    k_partial_sums<<<kSumBlocks, kBlock, 0, s>>>(x0, cnt0, x1, x2, cnt1, partials); count_launch();
    k_final_sums<<<1, 32, 0, s>>>(partials, totals); count_launch();
}
int grid_blocks(size_t n, int block, int cap) { return grid_for(n, block, cap); }

GridDev plan_grid(const BBox& bb, double reach, size_t max_slots, uint32_t* ncell, double cell_scale) {
    double ext[3], cell = reach * (cell_scale > 0.5 ? cell_scale : 0.5);
    for (int k = 0; k < 3; ++k) ext[k] = (bb.mx[k] - bb.mn[k]) + 2.0 * reach;
    auto dims_for = [&](double c, int* d) {
        for (int k = 0; k < 3; ++k) d[k] = (int)std::floor(ext[k] / c) + 1;
    };
    int dd[3];
    dims_for(cell, dd);
    double vol_cells = (double)dd[0] * dd[1] * dd[2];
    const double max_cells = 8.0 * (double)max_slots + 4096.0;
    while (vol_cells > max_cells) {  // sparse inputs: coarser cells keep the grid O(n)
        cell *= std::cbrt(vol_cells / max_cells) * 1.01;
        dims_for(cell, dd);
        vol_cells = (double)dd[0] * dd[1] * dd[2];
    }
    GridDev g;
    g.cell = cell;
    g.reach = reach;
    g.half = cell >= reach ? 1 : 2;  // cell >= reach / 2 always
    g.ox = bb.mn[0] - reach;
    g.oy = bb.mn[1] - reach;
    g.oz = bb.mn[2] - reach;
    g.dx = dd[0];
    g.dy = dd[1];
    g.dz = dd[2];
    *ncell = (uint32_t)(dd[0] * (uint64_t)dd[1] * dd[2]);
    return g;
}
void launch_collect_redo(const DevBufs& b, uint32_t P, cudaStream_t s) {
    cudaMemsetAsync(b.d_redo_count, 0, sizeof(uint32_t), s);
    cudaMemsetAsync(b.d_serial_count, 0, sizeof(uint32_t), s);
    k_collect_redo<<<grid_for(P, kBlock), kBlock, 0, s>>>(b, P); count_launch();
}

}  // namespace vt
