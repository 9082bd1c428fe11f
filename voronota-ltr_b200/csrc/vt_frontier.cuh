// vt_frontier.cuh -- device kernels of the updateable tessellation (updateable.rs,
// spheres_container.rs), launched by vt_updateable.cu.
//
// Device state of one updateable tessellation (n balls, E list entries, M table entries):
//   balls      f64[4n]     stored balls (x, y, z, r); spheres R = r + probe in sph
//   sph        double4[n] or, periodic, double4[27n] with image g of ball j at (g+1) n + j,
//              so a neighbour's reference id is also its sph index
//   excl       u8[n]       exclusion statuses (images share their ball's status)
//   lists      cnt u32[n], off u32[n+1], id u32[E], val f64[E], rel float4[E] (FP32 path)
//              -- colliding_ids per ball, sorted by (value, id)
//   table      off u32[n+1]; a, b u32[M] (canonical ids, a <= b); area, arc f64[M];
//              sa, pv f64[M] (solid angle and pyramid volume at the owning ball);
//              flags u8[M] (bit 0 central, bit 1 the owning ball is id a)
//              -- contacts_by_sphere: ball i's entries in the reference's push order
//   cells      flag u8[n] (1 = SasComputed), sas f64[n], vol f64[n]
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "vt_pipeline.cuh"

namespace vt {

struct ListsRef {
    const uint32_t* cnt;
    const uint32_t* off;
    const uint32_t* id;
    const double* val;
    const float4* rel;  // may be null
};

struct TableRef {
    uint32_t* off;
    uint32_t* a;
    uint32_t* b;
    double* area;
    double* arc;
    double* sa;
    double* pv;
    uint8_t* flags;
    // optional: SAS adjoint coefficients of the entry (x, y, z, r): gA = dSAS_owner /
    // d(owner), gB = dSAS_other / d(owner); volume adjoint coefficients through the
    // entry's contact face: vA = dV_owner / d(owner), vB = dV_other / d(owner)
    double4* gA;
    double4* gB;
    double4* vA;
    double4* vB;
};

// Contacts computed by one pass, deduplicated and canonicalised, in the reference's
// order (the order of pairs): ids (a <= b), values oriented to a, and the pair index.
struct NewContacts {
    uint32_t* a;
    uint32_t* b;
    double* area;
    double* arc;
    double* sa_a;
    double* sa_b;
    double* pv_a;
    double* pv_b;
    uint8_t* central;
    uint32_t* pair;
    // optional: SAS adjoint coefficients, dSAS_x / d(y) for x, y in {a, b}, and volume
    // adjoint coefficients dV_x / d(y) through the contact's face
    double4* gaa;
    double4* gab;
    double4* gba;
    double4* gbb;
    double4* vaa;
    double4* vab;
    double4* vba;
    double4* vbb;
};

// Every periodic image at id (g+1) n + j (populate_periodic_spheres, types.rs:351-375).
void launch_images_all(double4* sph, uint32_t n, const double* pbox9, cudaStream_t s);
// Changed-ball filter (spheres_container.rs:86-101): flags[t] = 1 when listed id t
// (ids == null: t itself) is < n and its sphere differs from the stored one.  The new
// ball of entry t is src[4 id .. ] when src_by_id, else src[4 t ..].
void launch_changed_flags(const uint64_t* ids, uint32_t k, const double* src, int src_by_id, uint32_t n,
                          double probe, const double* balls, uint32_t* flags, cudaStream_t s);
// Compacts the flagged entries (off = exclusive scan of flags, k+1 words) into
// changed ids and their new balls, preserving order.
void launch_changed_compact(const uint64_t* ids, uint32_t k, const double* src, int src_by_id, const uint32_t* off,
                            uint32_t* changed, double4* changed_ball, cudaStream_t s);
// *count = min(*count, cap)
void launch_clamp_count(uint32_t* count, uint32_t cap, cudaStream_t s);
// balls[changed[t]] = changed_ball[t] for t < *count
void launch_apply_changed(const uint32_t* changed, const double4* changed_ball, const uint32_t* count,
                          uint32_t max_count, double* balls, cudaStream_t s);
// mark[list[t]] = val where it was 0; *d_new counts the newly marked balls
void launch_mark_list(const uint32_t* list, const uint32_t* count, uint32_t max_count, uint32_t* mark, uint32_t val,
                      uint32_t* d_new, cudaStream_t s);
// Marks the canonical ids (id % n) of the neighbours of the listed balls; a listed ball's
// row in `lists` is row_of[ball] (row_of == null: the ball itself).  Newly marked ids are
// counted in *d_new and, when append != null, appended to it.
void launch_mark_neighbours(const uint32_t* list, const uint32_t* count, uint32_t max_count, const uint32_t* row_of,
                            ListsRef lists, uint32_t n, uint32_t* mark, uint32_t val, uint32_t* d_new,
                            uint32_t* append, cudaStream_t s);
// Marks `id` and the other ends of its table entries (updateable.rs:241-253).
void launch_mark_table_partners(uint32_t id, TableRef tab, uint32_t* mark, cudaStream_t s);
// flags[i] = mark[i] != 0
void launch_nonzero(const uint32_t* mark, uint32_t n, uint32_t* flags, cudaStream_t s);
// list[off[i]] = i for every i with off[i+1] > off[i]
void launch_compact_index(const uint32_t* off, uint32_t n, uint32_t* list, cudaStream_t s);
// row_of[list[t]] = t
void launch_row_of(const uint32_t* list, const uint32_t* count, uint32_t max_count, uint32_t* row_of,
                   cudaStream_t s);
// Spliced list counts: ball i keeps its old row when mark[i] == 0, else takes row
// row_of[i] of t1 (mark 1) or t2 (mark 2).
void launch_splice_counts(uint32_t n, const uint32_t* mark, const uint32_t* row_of, const uint32_t* old_cnt,
                          const uint32_t* c1, const uint32_t* c2, uint32_t* cnt, cudaStream_t s);
void launch_splice_lists(uint32_t n, const uint32_t* mark, const uint32_t* row_of, ListsRef old, ListsRef t1,
                         ListsRef t2, const uint32_t* new_off, uint32_t* id, double* val, float4* rel,
                         cudaStream_t s);
// collect_collision_pairs with involvement (updateable.rs:516-561) over the listed balls
// (list == null: all n).  Count pass writes npair[a]; fill pass writes pair_a, pair_e
// (list entry of b) and nb_pair (pair index or -1) for every entry of a listed ball.
// need > 0 keeps only the pairs with an end whose mark is at least need.
void launch_upd_pairs(int fill, const uint32_t* list, const uint32_t* count, uint32_t max_count, uint32_t n,
                      int periodic, ListsRef lists, const uint8_t* excl, const uint32_t* mark, uint32_t need,
                      uint32_t* npair, const uint32_t* pair_off, uint32_t* pair_a, uint32_t* pair_e,
                      int32_t* nb_pair, cudaStream_t s);
// Kept pairs (keep_off = exclusive scan of keep flags) as canonical contacts
// (compute_contact_summaries_with_dedup + deduplicate_and_canonicalize_contacts,
// updateable.rs:565-631).
void launch_new_contacts(uint32_t P, const uint32_t* keep_off, const DevBufs& b, NewContacts nc, cudaStream_t s);
// Table splice (updateable.rs:494-511).  keep_cnt[i]: entries of ball i that stay (all
// when i is not involved, else those whose other end is not involved; 0 when old.off is
// null); new_cnt[i] += new contacts incident to i.
void launch_table_counts(uint32_t n, const uint32_t* mark, TableRef old, uint32_t* keep_cnt, cudaStream_t s);
void launch_table_new_counts(const NewContacts& nc, const uint32_t* nc_count, uint32_t max_nc, uint32_t* new_cnt,
                             cudaStream_t s);
void launch_add_u32(const uint32_t* x, const uint32_t* y, uint32_t n, uint32_t* out, cudaStream_t s);
void launch_table_copy_kept(uint32_t n, const uint32_t* mark, TableRef old, TableRef nw, cudaStream_t s);
// New entries go after the kept ones of each ball, in contact order: a scatter of contact
// indices (cursor zeroed, n words) and a per-ball ranking that writes the entries.
void launch_table_scatter_new(const NewContacts& nc, const uint32_t* nc_count, uint32_t max_nc, TableRef nw,
                              const uint32_t* keep_cnt, uint32_t* cursor, uint32_t* tmp_k, cudaStream_t s);
void launch_table_write_new(uint32_t n, const NewContacts& nc, TableRef nw, const uint32_t* keep_cnt,
                            const uint32_t* new_cnt, const uint32_t* tmp_k, uint32_t* err, cudaStream_t s);
// Cells of the listed balls from their table entries (recompute_cells_for_affected,
// updateable.rs:691-727).  cell_band > 0: balls with an uncertain compute_sas branch
// get unsure[i] = 1.
// keep_empty: a listed ball without table entries keeps its cell state (the FP64 refresh of
// uncertain cells, whose neighbours need not be affected by the operation).
void launch_table_cells(const uint32_t* list, const uint32_t* count, uint32_t max_count, TableRef tab,
                        const double4* sph, const uint8_t* excl, uint8_t* cell_flag, double* cell_sas,
                        double* cell_vol, float cell_band, uint8_t* unsure, cudaStream_t s, int keep_empty = 0);
// Contact-table bit: a recomputed contact found no entry to overwrite (launch_table_update).
constexpr uint32_t kErrRefresh = 128u;
// Overwrites the values of the existing entries (same canonical ids) of every contact in
// nc; the entries keep their place in each ball's order.
void launch_table_update(const NewContacts& nc, const uint32_t* nc_count, uint32_t max_nc, TableRef tab,
                         uint32_t* err, cudaStream_t s);
// Appends to out the listed balls whose flag is set (in no particular order; the count
// goes to *d_out, zeroed by the caller).
void launch_list_flagged(const uint32_t* list, const uint32_t* count, uint32_t max_count, const uint8_t* flag,
                         uint32_t* out, uint32_t* d_out, cudaStream_t s);
// grad (n x 4, overwritten) = d(sum_i w_i SAS_i + sum_i v_i V_i)/d(x, y, z, r) from the
// table's adjoint coefficients (w == null: every w_i = w_default; v == null: no volume
// term; balls without a cell, or with zero SAS for the SAS term, weigh 0).
void launch_table_grad(uint32_t n, TableRef tab, const double* w, double w_default, const double* v,
                       const uint8_t* cell_flag, const double* cell_sas, const double4* sph, double* grad,
                       cudaStream_t s);
// Summary (updateable.rs:332-378): entries owned by their id a, in table order.
void launch_owner_flags(const uint8_t* flags, uint32_t M, uint32_t* out, cudaStream_t s);
void launch_summary_contacts(TableRef tab, uint32_t M, const uint32_t* off, uint32_t* a, uint32_t* b, double* area,
                             double* arc, uint8_t* central, cudaStream_t s);
void launch_cell_flags_u32(const uint8_t* flag, uint32_t n, uint32_t* out, cudaStream_t s);
void launch_summary_cells(const uint32_t* off, uint32_t n, const double* sas, const double* vol, uint32_t* index,
                          double* osas, double* ovol, cudaStream_t s);

}  // namespace vt
