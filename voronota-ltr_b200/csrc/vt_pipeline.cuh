// vt_pipeline.cuh -- device buffers and kernel launchers of the tessellation pipeline.
//
// Data layout in HBM (n balls, m periodic images, E neighbour entries, P pairs):
//   sph      double4[n + m]  x, y, z, R (= r + probe) per slot; slots 0..n-1 are the balls,
//                            slots n.. the periodic images within reach of the structure
//   slot_id  u32[n + m]      reference id of the slot: i for balls, (g+1) n + j for the image
//                            of ball j under NEIGHBOR_SHIFTS[g] (types.rs:351-375)
//   grid     cell_start u32[ncell+1], c_pos double4 / c_id u32 / c_slot u32 [n + m]
//            (slots sorted by cell: a counting sort on the cell key)
//   CSR      nb_off u32[n+1]; nb_id, nb_slot u32[E]; nb_val f64[E]; nb_pair i32[E];
//            nb_rel float4[E] (FP32 path: neighbour centre relative to the ball, and R)
//   pairs    pair_a u32[P], pair_e u32[P] (CSR entry of b in a's list)
//   per pair status u8, area, arc, solid angles a/b, pyramid volumes a/b f64, central u8
//   cells    cell_flag u8[n], cell_sas f64[n], cell_vol f64[n]
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vt {

// Error bits written by kernels into the engine's device status word.
enum DevErr : uint32_t {
    kErrNeighborCap = 1u,  // a ball has more neighbour candidates than the sort buffer holds
    kErrOverflow = 2u,     // a contour exceeded the serial fallback's capacity
    kErrIdRange = 4u,      // ids do not fit 32 bits
    kErrInvalid = 8u,      // non-finite input value or negative radius
    kErrNetwork = 64u,     // a network contour outgrew a warp (32 points): elements not emitted
};

// Per-pair status bits.
enum PairStatus : uint8_t {
    kValid = 1,     // contact exists (area > 0)
    kUnsure = 2,    // FP32 decision inside the band: recompute in FP64
    kOverflow = 4,  // contour needed more than 32 points: recompute serially
};

constexpr int kSortCap = 256;       // neighbour list capacity of the warp sort buffer (longer
                                    // lists go through the block sort, without a limit)
constexpr int kSerialCap = 256;     // contour capacity of the serial fallback
constexpr uint32_t kRecNone = 0xffffffffu;  // a pair whose FP32 contour was not recorded
constexpr int kHitCap = 64;  // hits per row the count pass lists for the fill pass

// Host-visible bounding-box reduction result.
struct BBox {
    double mn[3], mx[3], max_r;
};

// Uniform grid: cells of edge `cell` from (ox, oy, oz), dx x dy x dz of them.  reach is an
// upper bound of R_a + R_c over intersecting balls (2 max R + 0.25), and half = the stencil
// half-width in cells (cell * half >= reach): 1 for cells of at least the reach, 2 for
// cells of half of it (a 5 x 5 x 5 stencil, culled to the rows and x-ranges within reach).
struct GridDev {
    double ox, oy, oz, cell, reach;
    int dx, dy, dz, half;
};

struct DevBufs {
    // inputs / slots
    double4* sph;
    uint32_t* slot_id;
    const int32_t* groups;
    uint64_t n_groups;
    uint32_t n;
    uint32_t* d_nslots;  // device count of slots (n + images)
    int periodic;
    double pbox[9];
    // grid
    GridDev grid;
    uint32_t* cell_count;
    uint32_t* cell_start;
    uint32_t* cell_cursor;
    double4* c_pos;
    uint32_t* c_id;
    uint32_t* c_slot;
    // CSR
    uint32_t* nb_cnt;
    // optional: kHitCap grid indices per search row, the hits the count pass found (rows
    // with more hits are scanned again by the fill pass)
    uint32_t* hit_idx;
    uint32_t* nb_npair;
    uint8_t* excluded;
    uint32_t* nb_off;
    uint32_t* pair_off;
    uint32_t* nb_id;
    uint32_t* nb_slot;
    double* nb_val;
    int32_t* nb_pair;
    float4* nb_rel;
    // pairs
    uint32_t* pair_a;
    uint32_t* pair_e;
    uint8_t* p_status;
    double* p_area;
    double* p_arc;
    uint8_t* p_central;
    double* p_sa_a;
    double* p_sa_b;
    double* p_pv_a;
    double* p_pv_b;
    double* p_arcm;  // optional: first moments of each contact's arcs and area about a (6 per pair)
    // optional (FP32 calls that build the network): the FP32 contact kernel records each
    // valid pair's contour for the network's element kernel, which then need not
    // recompute it.  rec_off[p]: first point in rec_pts / rec_ids, or kRecNone (not
    // recorded: the element kernel recomputes the contour); rec_meta[p]: points << 8 |
    // 1 uncut | 2 merged points | 4 an unsure contour decision; points are taken from a
    // pool of rec_cap with the counter rec_count.
    float4* rec_pts;  // x, y, z relative to a, arc angle
    uint2* rec_ids;   // left id, right id
    uint32_t* rec_off;
    uint32_t* rec_meta;
    uint32_t* rec_count;
    uint32_t rec_cap;
    // recompute lists
    uint32_t* redo_list;
    uint32_t* d_redo_count;
    uint32_t* serial_list;
    uint32_t* d_serial_count;
    double* serial_scratch;  // kSerialCap * 7 doubles per fallback slot
    uint32_t serial_slots;
    // cells
    uint8_t* cell_flag;
    double* cell_sas;
    double* cell_vol;
    // output compaction
    uint32_t* keep;      // per pair 0/1, then scanned
    uint32_t* keep_off;  // P+1
    uint32_t* cell_off;  // n+1
    uint32_t* out_a;
    uint32_t* out_b;
    double* out_area;
    double* out_arc;
    uint8_t* out_central;
    uint32_t* out_cell_index;
    double* out_cell_sas;
    double* out_cell_vol;
    double* totals;     // 3: sas, volume, contact area
    double* partials;   // reduction scratch
    uint32_t* err;        // device error bits
    uint32_t* zero_word;  // a device word that stays 0 (an empty count)
    uint32_t* params_u;   // n words of scratch (cell flags widened for the scan)
    float fp32_band;      // FP32 error floor of a computed length, relative to the pair scale
    // cells whose compute_sas branch is uncertain with FP32 inputs (FP32 path only)
    uint32_t* cell_redo_list;
    uint32_t* d_cell_redo_count;
    uint8_t* ball_dirty;  // balls whose cell is recomputed after the FP64 fixup
    // updateable tessellation (all zero for the stateless path)
    const uint32_t* frontier;  // search only these balls; per-ball CSR arrays are then
    uint32_t n_frontier;       // indexed by frontier position (excluded stays per ball)
    int no_pairs;              // fill pass writes the neighbour lists only
    // rows with more neighbours than the warp sort holds (kSortCap): listed by the count
    // pass, written unsorted by the fill pass, then sorted and paired by a block per row
    uint32_t* big_list;
    uint32_t* d_big_count;
    int slot_is_id;            // grid slots carry reference ids as their sph index
    int detached_excl;         // cells: an empty list is detached only when not excluded
    // batched structures (null for one structure): ball -> structure, the structure's
    // grid and the index of its first cell in the concatenated cell arrays
    const uint32_t* ball_struct;
    const GridDev* grids;
    const uint32_t* cell_base;
    int c32_warps;  // warps per block of the FP32 contact kernel (2, 4 or 8; 0: 4)
    int c32_chunk;  // > 0: persistent FP32 contact launch taking chunks of pairs from
    uint32_t* c32_queue;  // this work counter
};


#ifdef __CUDACC__
// NEIGHBOR_SHIFTS (types.rs:292-302) without the origin: image g of ball j has id (g+1) n + j.
__device__ __forceinline__ void neighbor_shift(int g, int& sx, int& sy, int& sz) {
    int k = g < 13 ? g : g + 1;
    sx = k / 9 - 1;
    sy = (k / 3) % 3 - 1;
    sz = k % 3 - 1;
}
// PeriodicBox::shift_sphere (types.rs:323-347): c.mul_add(wc, b.mul_add(wb, a.mul_add(wa, x)))
__device__ __forceinline__ double4 shift_sphere(double4 s, const double* pb, double wa, double wb, double wc) {
    return make_double4(fma(pb[6], wc, fma(pb[3], wb, fma(pb[0], wa, s.x))),
                        fma(pb[7], wc, fma(pb[4], wb, fma(pb[1], wa, s.y))),
                        fma(pb[8], wc, fma(pb[5], wb, fma(pb[2], wa, s.z))), s.w);
}
// ---- uniform grid cells ----
__device__ __forceinline__ int cell_coord(double x, double o, double cell, int d) {
    double f = floor((x - o) / cell);
    int c = f < 0.0 ? 0 : (f > (double)(d - 1) ? d - 1 : (int)f);
    return c;
}
__device__ __forceinline__ uint32_t cell_key(const GridDev& g, int x, int y, int z) {
    return (uint32_t)x + (uint32_t)g.dx * ((uint32_t)y + (uint32_t)g.dy * (uint32_t)z);
}
__device__ __forceinline__ uint32_t slot_cell(const GridDev& g, double4 p) {
    return cell_key(g, cell_coord(p.x, g.ox, g.cell, g.dx), cell_coord(p.y, g.oy, g.cell, g.dy),
                    cell_coord(p.z, g.oz, g.cell, g.dz));
}

// CellContactSummary::compute_sas (types.rs:623-663) from the accumulated sums of a cell
// with count > 0 contributing contacts.  cell_band > 0 (sums of FP32-derived values):
// *unsure is set when a branch decision lies within cell_band radians per contact of
// its threshold.
__device__ __forceinline__ void cell_from_sums(uint32_t count, double arc, double spos, double sneg, double ppos,
                                               double pneg, double r, float cell_band, bool* unsure, double* sas_out,
                                               double* vol_out) {
    const double kPiD = 3.141592653589793;
    double sas = 0.0, vol = 0.0;
    double diff = fabs(spos - sneg);
    *unsure = false;
    if (cell_band > 0.f && arc > 0.0) {
        double tol_sa = (double)cell_band * count;
        // which sum dominates (the centre inside or outside its own cell): decided only by
        // cells whose centre is close to the cell's boundary, rare, and there the FP32
        // solid angles' error (float vertices, about E / distance per contour point) once
        // exceeded tol_sa (a nearly engulfed ball, 5 contacts); the wider band costs
        // almost no recomputation
        if (fabs(spos - sneg) <= 8.0 * tol_sa + 1e-10) *unsure = true;
        // a nearly buried ball (positive dominance, 4 pi - (spos - sneg) about 0): the
        // sign of its SAS area, i.e. whether it is exposed at all, is within the band
        if (spos > sneg && fabs(fma(4.0, kPiD, -(spos - sneg))) <= tol_sa) *unsure = true;
        double sas_g = spos > sneg ? fma(4.0, kPiD, -(spos - sneg)) * r * r : (sneg - spos) * r * r;
        double vol_g = sas_g * r / 3.0 + ppos - pneg;
        double full_g = 4.0 / 3.0 * kPiD * r * r * r;
        double tol_v = (double)cell_band * count * (ppos + pneg + r * r * r);
        if (fabs(vol_g - full_g) <= tol_v) *unsure = true;
    }
    if (arc > 0.0 && diff > 1e-10) {
        if (spos > sneg) {
            sas = fma(4.0, kPiD, -fmax(spos - sneg, 0.0)) * r * r;
        } else {
            sas = fmax(sneg - spos, 0.0) * r * r;
        }
        vol = (sas * r / 3.0) + ppos - pneg;
        double full = 4.0 / 3.0 * kPiD * r * r * r;
        if (vol > full) {
            sas = 0.0;
            vol = ppos - pneg;
        }
    } else {
        vol = ppos - pneg;
    }
    *sas_out = sas;
    *vol_out = vol;
}
#endif

// Host-side count of kernel launches issued by this library (all devices, all engines).
void count_launch();
uint64_t launch_count();

// ---- launchers (vt_pipeline.cu) ----
void launch_prepare(const DevBufs& b, const double* d_xyzr, double probe, BBox* d_bbox_partials, int nblocks,
                    cudaStream_t s);
void launch_bbox_final(const BBox* partials, int nblocks, BBox* out, cudaStream_t s);
void launch_images(const DevBufs& b, double reach, const BBox* d_bbox, uint32_t* img_cnt, uint32_t* img_off,
                   uint32_t* scan_tmp, size_t scan_tmp_words, cudaStream_t s);
void launch_grid(const DevBufs& b, uint32_t ncell, uint32_t max_slots, uint32_t* scan_tmp, size_t scan_tmp_words,
                 cudaStream_t s);
void launch_search_count(const DevBufs& b, cudaStream_t s);
// n_big: rows the count pass listed in big_list (read back by the caller)
void launch_search_fill(const DevBufs& b, int want_rel, uint32_t n_big, cudaStream_t s);
// cell_band > 0 (FP32 inputs): balls whose compute_sas branch decisions lie within
// cell_band radians per contributing contact of their thresholds go to cell_redo_list.
// only_dirty: recompute only balls flagged in ball_dirty.
void launch_cells(const DevBufs& b, float cell_band, int only_dirty, cudaStream_t s);
// Append every pair incident to a ball of cell_redo_list to redo_list and mark the
// ball and its neighbours dirty.
void launch_mark_ball_pairs(const DevBufs& b, cudaStream_t s);
void launch_dedup(const DevBufs& b, uint32_t P, int contacts_only, cudaStream_t s);
void launch_compact(const DevBufs& b, uint32_t P, int contacts_only, uint32_t* scan_tmp, size_t scan_tmp_words,
                    cudaStream_t s);
void launch_totals(const DevBufs& b, uint32_t P, int contacts_only, cudaStream_t s);
void launch_collect_redo(const DevBufs& b, uint32_t P, cudaStream_t s);
// Deterministic FP64 totals: totals[0] = sum x1[0..*cnt1), totals[1] = sum x2[0..*cnt1),
// totals[2] = sum x0[0..*cnt0) (fixed grid, fixed tree; partials holds 148 * 3 doubles).
void launch_sums3(const double* x0, const uint32_t* cnt0, const double* x1, const double* x2, const uint32_t* cnt1,
                  double* partials, double* totals, cudaStream_t s);
int grid_blocks(size_t n, int block, int cap);
// Cell grid over the bounding box extended by `reach` (cell edge >= reach, so that
// intersecting balls lie in adjacent cells), coarsened for sparse inputs so that the
// number of cells stays O(max_slots).
// cell_scale >= 1 widens the cells (fewer cells, more candidates per ball).
GridDev plan_grid(const BBox& bb, double reach, size_t max_slots, uint32_t* ncell, double cell_scale = 1.0);
size_t scan_tmp_words_needed(size_t n);
void scan_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* tmp, cudaStream_t s);

// ---- adjoint (vt_adjoint.cu): grad (n x 4, overwritten) = dL/d(x, y, z, r) for
// L = sum_i w_sas[i] SAS_i + sum_i v_vol[i] V_i + sum_k u_contact[k] area_k over the last
// full tessellation in b (w_sas, v_vol, u_contact: device arrays or null; w_eff, v_eff:
// n doubles of scratch each).
void launch_adjoint(const DevBufs& b, uint32_t P, const double* w_sas, const double* v_vol, const double* u_contact,
                    double* w_eff, double* v_eff, double* grad, cudaStream_t s);
// FP32 adjoint over all valid pairs (vt_contact32.cu); lists the pairs it cannot decide
// in redo_list for the FP64 adjoint.  v_eff may be null (no volume term).
// Adjoint of the pairs the FP64 adjoint listed in serial_list (contours beyond a warp),
// with the serial contour (vt_contact64.cu).
void launch_adjoint_serial(const DevBufs& b, const double* u_contact, const double* w_eff, const double* v_eff,
                           double* grad, cudaStream_t s);
void launch_adjoint_f32(const DevBufs& b, uint32_t P, const double* u_contact, const double* w_eff,
                        const double* v_eff, double* grad, cudaStream_t s);

// ---- tessellation network (vt_network.cu) ----
// Element storage.  Valid pair number v (slot = exclusive scan of the valid flags) owns
// elements [base[v], base[v] + cnt[v]) of a two-part index space: [0, split) are the warp
// slots (net_slot_capacity() = 32 elements per pair, split = 32 V); [split, ...) is the
// overflow area, kSerialCap elements for each pair whose contour outgrew a warp, filled
// by the serial kernel (launch_net_serial).  Ids: NULL = 0xffffffff; an edge uses the
// x, y, z of its uint4.
constexpr uint32_t kNetNull = 0xffffffffu;
constexpr int kNetSlot = 32;  // elements of one pair in the warp area
struct NetSlots {
    uint4* v_ids;  // warp area
    double* v_xyz;
    uint4* e_ids;
    double* e_len;
    uint4* ov_v_ids;  // overflow area
    double* ov_v_xyz;
    uint4* ov_e_ids;
    double* ov_e_len;
    uint32_t split;
    uint32_t* base;
    uint32_t* v_cnt;
    uint32_t* e_cnt;
    uint32_t* ov_list;   // pairs whose contour outgrew a warp, in no particular order
    uint32_t* ov_count;  // device counter of ov_list
    uint32_t ov_cap;
};
__device__ __forceinline__ uint4 net_vid(const NetSlots& s, uint32_t i) {
    return i < s.split ? s.v_ids[i] : s.ov_v_ids[i - s.split];
}
__device__ __forceinline__ uint4 net_eid(const NetSlots& s, uint32_t i) {
    return i < s.split ? s.e_ids[i] : s.ov_e_ids[i - s.split];
}
__device__ __forceinline__ double net_vxyz(const NetSlots& s, uint32_t i, int k) {
    return i < s.split ? s.v_xyz[3 * (size_t)i + k] : s.ov_v_xyz[3 * (size_t)(i - s.split) + k];
}
__device__ __forceinline__ double net_elen(const NetSlots& s, uint32_t i) {
    return i < s.split ? s.e_len[i] : s.ov_e_len[i - s.split];
}
__device__ __forceinline__ void net_cswap(uint32_t& x, uint32_t& y) {
    if (x > y) {
        const uint32_t t = x;
        x = y;
        y = t;
    }
}
// ids of the edge (a, b, third) and of the vertex (a, b, left, right): periodic image ids
// taken mod n (NULL kept), then sorted (contact.rs:119-177, tessellation.rs:334-360)
__device__ __forceinline__ uint4 net_edge_ids(uint32_t a, uint32_t b, uint32_t third, int periodic, uint32_t n) {
    uint32_t i0 = a, i1 = b, i2 = third;
    if (periodic) {
        i0 %= n;
        i1 %= n;
        if (i2 != kNetNull) i2 %= n;
    }
    net_cswap(i0, i1);
    net_cswap(i1, i2);
    net_cswap(i0, i1);
    return make_uint4(i0, i1, i2, 0u);
}
__device__ __forceinline__ uint4 net_vertex_ids(uint32_t a, uint32_t b, uint32_t l, uint32_t r, int periodic,
                                                uint32_t n) {
    uint32_t v0 = a, v1 = b, v2 = l, v3 = r;
    if (periodic) {
        v0 %= n;
        v1 %= n;
        if (v2 != kNetNull) v2 %= n;
        if (v3 != kNetNull) v3 %= n;
    }
    net_cswap(v0, v1);  // sorting network of 4
    net_cswap(v2, v3);
    net_cswap(v0, v2);
    net_cswap(v1, v3);
    net_cswap(v1, v2);
    return make_uint4(v0, v1, v2, v3);
}
// Deduplication buffers of one element type (m elements, n + 1 buckets by first id).
struct NetBuckets {
    uint32_t* cnt;   // [n + 1] elements per bucket
    uint32_t* off;   // [n + 2] exclusive scan of cnt
    uint32_t* cur;   // [n + 1] fill cursors
    uint32_t* ucnt;  // [n + 1] distinct elements per bucket
    uint32_t* uoff;  // [n + 2] exclusive scan of ucnt
    uint32_t* big;   // [n + 2] buckets too large for a warp's sort; [n + 1] is their count
    unsigned long long* k1;  // [m] by bucket position: the ids after the first (packed)
    unsigned long long* k2;  // [m] the third of them when three do not fit one word
    uint32_t* idx;   // [m] by bucket position: the dense index; after the sort each bucket's
                     // range starts with its distinct elements' dense indices in id order
    uint32_t* srcd;  // [m] by dense index: the element's index in the slot arrays
};
// bits of an id in the packed keys: 2^B > n (ids 0..n-1, NULL as n)
int net_key_bits(uint32_t n);
void launch_valid_flags(const DevBufs& b, uint32_t P, uint32_t* flags, cudaStream_t s);
// FP64 elements of every valid pair, or (list != null) of the *count pairs listed
void launch_net_elements(const DevBufs& b, uint32_t P, const uint32_t* voff, NetSlots slots, const uint32_t* list,
                         const uint32_t* count, cudaStream_t s);
// FP32 mode: elements from the FP32 contour with FP64-placed vertices (vt_contact32.cu);
// pairs it cannot settle are listed for launch_net_elements
void launch_net_elements_f32(const DevBufs& b, uint32_t P, const uint32_t* voff, NetSlots slots, uint32_t* fp64_list,
                             uint32_t* fp64_count, cudaStream_t s);
// the pairs of ov_list through the serial contour (vt_contact64.cu); at most ov_cap
void launch_net_serial(const DevBufs& b, const uint32_t* voff, NetSlots slots, cudaStream_t s);
size_t net_slot_capacity();
// The distinct elements of V pairs (off = exclusive scan of the pairs' element counts,
// the dense order: pair then contour order) in id order, keeping the first in dense order of equal ids:
// elements bucketed by their first id (ids are sorted within an element), each bucket
// sorted by (the other ids, dense index); t.uoff[n + 1] is the distinct count.
// wide: the two-word vertex keys (taken anyway when three ids need more than 64 bits)
void launch_net_dedup(uint32_t V, const uint32_t* off, const NetSlots& slots, int vertices, int wide, uint32_t n,
                      NetBuckets t, uint32_t* scan_tmp, cudaStream_t s);
// the distinct elements to the output arrays (ids, and positions or lengths)
void launch_net_dedup_gather(uint32_t n, const NetBuckets& t, const NetSlots& slots, int vertices,
                             uint32_t* out_ids, double* out_vals, cudaStream_t s);

// ---- contact kernels (vt_contact64.cu / vt_contact32.cu) ----
// mode: 0 = all pairs; 1 = pairs listed in redo_list (count on device)
void launch_contact_f64(const DevBufs& b, uint32_t P, int full, int from_list, cudaStream_t s);
void launch_contact_f32(const DevBufs& b, uint32_t P, int full, cudaStream_t s);
void launch_contact_serial(const DevBufs& b, uint32_t P, int full, cudaStream_t s);
// Upload the FP64 hexagon rotation table (sin/cos from the host C library) to the
// current device; call once per device before the first FP64 contact launch.
void set_hex_table();
// The hexagon table's values (host C library) and the upload into the adjoint's unit.
void hex_table_values(double* hs, double* hc, int* n);
void set_hex_table_adjoint();
void set_hex_table_network();

}  // namespace vt
