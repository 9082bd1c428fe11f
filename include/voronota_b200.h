/*
 * voronota_b200.h -- C ABI of the B200 radical-tessellation library (libvoronota_b200.so).
 *
 * Drop-in boundary for voronota-ltr's tessellation hot path.  Plain pointers and sizes,
 * integer status codes, no exceptions across the ABI, nothing aborts.
 *
 * Balls are N x 4 row-major doubles (x, y, z, r) -- the layout of the reference's
 * numpy input (src/python.rs:69-88) and of `&[Ball]` (src/types.rs:12-21).  A periodic
 * box is 9 doubles: the lattice vectors a, b, c (PeriodicBox, src/types.rs:292-320;
 * from_corners(min, max) is the diagonal box (max - min)).  Pass NULL for no box.
 * Groups: optional int32 per ball; as in the reference (src/tessellation.rs:323-328)
 * only ids below n_groups are compared.
 *
 * Ids are 32-bit: n must satisfy 27 * n < 2^32 (periodic image ids are (g+1) n + i).
 * Inputs must be finite with r >= 0; anything else returns VT_ERR_INVALID (the
 * reference accepts such inputs silently and returns meaningless results).
 */
#ifndef VORONOTA_B200_H
#define VORONOTA_B200_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define VT_OK 0
#define VT_ERR_INVALID 1   /* malformed input (NaN/inf, r < 0, n too large, null pointer) */
#define VT_ERR_OOM 2       /* device or host allocation failed */
#define VT_ERR_CUDA 3      /* CUDA runtime error (message: vt_last_error()) */
#define VT_ERR_CAPACITY 4  /* a neighbour list or contour exceeded the kernels' capacity */
#define VT_ERR_TIMEOUT 5   /* a bounded device wait expired */
#define VT_ERR_NO_DEVICE 6 /* no CUDA device */

/* arithmetic of the contact kernel */
#define VT_FP64 0        /* plain FP64: the reference's arithmetic on the GPU */
#define VT_FP32_FIXUP 1  /* FP32 bulk; pairs with a decision inside the FP32 error band
                            are recomputed in FP64 */

typedef struct vt_result vt_result; /* library-owned host result */
typedef struct vt_engine vt_engine; /* device workspace + stream, one per device/thread */

/* Replaces compute_tessellation(balls, probe, periodic_box, groups, false)
 * (src/tessellation.rs:37-48).  Contacts come in the reference's output order: pair
 * order, i.e. by id_a, then by a's neighbour order (src/tessellation.rs:298-319,
 * 238-253); periodic contacts are deduplicated as deduplicate_periodic_contacts
 * (src/tessellation.rs:527-601) with ids taken mod n.  Cells are ascending by index
 * (src/tessellation.rs:649-657).  Uses a per-device engine shared by the process. */
int vt_compute_tessellation(const double* xyzr, uint64_t n, double probe, const double* periodic_box9,
                            const int32_t* groups, uint64_t n_groups, int precision, vt_result** out);

/* Replaces compute_contacts_only (src/tessellation.rs:125-166): no cells; periodic
 * contacts are canonicalised to (min, max) ids and deduplicated keeping the first in
 * pair order (the reference's HashMap order is unspecified; pair order is a valid one). */
int vt_compute_contacts_only(const double* xyzr, uint64_t n, double probe, const double* periodic_box9,
                             const int32_t* groups, uint64_t n_groups, int precision, vt_result** out);

/* compute_tessellation(..., with_cell_vertices = true) (src/tessellation.rs:37-48,
 * 334-401): the result also holds the tessellation network -- cell vertices (4 ball ids
 * in ascending order, 0xffffffff for NULL, i.e. a vertex on the SAS, and x, y, z) and
 * cell edges (3 ids, NULL on the SAS, and the length), each sorted by ids and
 * deduplicated (of several elements with equal ids the first in pair order is kept; the
 * reference keeps an unspecified one).  Contours are recomputed in FP64 for the network. */
int vt_compute_tessellation_network(const double* xyzr, uint64_t n, double probe, const double* periodic_box9,
                                    const int32_t* groups, uint64_t n_groups, int precision, vt_result** out);
uint64_t vt_result_num_vertices(const vt_result* r);
uint64_t vt_result_num_edges(const vt_result* r);
int vt_result_vertices(const vt_result* r, uint32_t* ids4, double* xyz3);
int vt_result_edges(const vt_result* r, uint32_t* ids3, double* length);

/* compute_solvent_spheres (src/solvent_spheres.rs:131-169): weighted pseudo-solvent
 * spheres on the exposed surface.  Stage 1 tessellates the balls with `probe`; a sample
 * point p = centre + v (r + probe) of an exposed ball (cell sas_area > 0), v one of the
 * subdivided-icosahedron directions of `depth` (0..4: 12, 42, 162, 642, 2562; larger
 * clamps to 4), is kept when it is strictly closer (distance minus radius) to its ball
 * than to every contact partner; stage 2 tessellates the atoms (radius max(r - probe +
 * volume_probe, 0.01)) and the spheres (radius probe + volume_probe) with probe 0, and a
 * sphere's weight is its stage-2 cell volume (0 without a cell).  Spheres come in the
 * reference's order: cells by ball index, then direction order.  VT_ERR_INVALID (with the
 * reference's message in vt_last_error) for a negative or non-finite probe or volume
 * probe, a negative depth, non-finite coordinates or a non-positive radius. */
typedef struct vt_solvent_result vt_solvent_result;
int vt_compute_solvent_spheres(const double* xyzr, uint64_t n, double probe, double volume_probe, int depth,
                               const double* periodic_box9, int precision, vt_solvent_result** out);
uint64_t vt_solvent_count(const vt_solvent_result* r);
/* The unit sample directions of a depth (clamped to 0..4), x y z each; returns their count
 * (12, 42, 162, 642, 2562).  Host code only: needs no GPU. */
int vt_icosahedron(int depth, double* xyz3);
int vt_solvent_get(const vt_solvent_result* r, double* xyz3, double* radius, double* weight, uint32_t* parent);
void vt_solvent_free(vt_solvent_result* r);

/* Result accessors: TessellationResult + the Results trait (src/types.rs:187-269). */
uint64_t vt_result_num_balls(const vt_result* r);
uint64_t vt_result_num_contacts(const vt_result* r);
uint64_t vt_result_num_cells(const vt_result* r);
/* Copy out the contacts (arrays of num_contacts); any pointer may be NULL. */
int vt_result_contacts(const vt_result* r, uint32_t* id_a, uint32_t* id_b, double* area, double* arc_length,
                       uint8_t* central);
/* Copy out the cells (arrays of num_cells); any pointer may be NULL. */
int vt_result_cells(const vt_result* r, uint32_t* index, double* sas_area, double* volume);
/* total_sas_area / total_volume / total_contact_area (src/types.rs:230-252), summed on
 * the device in FP64 with a fixed reduction tree. */
void vt_result_totals(const vt_result* r, double* total_sas_area, double* total_volume,
                      double* total_contact_area);
void vt_result_free(vt_result* r);
/* Read-only views of a result's arrays, valid until vt_result_free (no copy; the arrays
 * live in page-locked host memory the device wrote directly). */
typedef struct vt_result_view {
    uint64_t num_contacts, num_cells;
    const uint32_t* id_a;
    const uint32_t* id_b;
    const double* area;
    const double* arc_length;
    const uint8_t* central;
    const uint32_t* cell_index;
    const double* cell_sas_area;
    const double* cell_volume;
} vt_result_view;
int vt_result_view_get(const vt_result* r, vt_result_view* view);

/* ---- engine: explicit device, stream and device-resident inputs ---- */
int vt_engine_create(int device, vt_engine** out);
void vt_engine_destroy(vt_engine* e);
/* cudaStream_t to run on (NULL: the engine's own stream). */
int vt_engine_set_stream(vt_engine* e, void* stream);
/* One tessellation on device-resident input (d_xyzr: N x 4 doubles on the engine's
 * device; d_groups: device int32 or NULL).  The box is read from host memory.  Results
 * stay in device memory until vt_engine_download / vt_engine_device_outputs. */
int vt_engine_compute_device(vt_engine* e, const double* d_xyzr, uint64_t n, double probe,
                             const double* periodic_box9, const int32_t* d_groups, uint64_t n_groups,
                             int precision, int contacts_only);
/* Same from host memory (copied in on the engine's stream). */
int vt_engine_compute_host(vt_engine* e, const double* xyzr, uint64_t n, double probe,
                           const double* periodic_box9, const int32_t* groups, uint64_t n_groups,
                           int precision, int contacts_only);
int vt_engine_download(vt_engine* e, vt_result** out);
/* Engine calls also build the tessellation network (on) or not (off, the default). */
int vt_engine_set_network(vt_engine* e, int on);
/* The network's vertex deduplication packs the three ids after the first into one 64-bit
 * key while 3 bits(n) <= 64 (fewer than 2^21 balls) and uses two words beyond; on: always
 * two words (the same results; lets tests cover that form on small inputs). */
int vt_engine_set_network_wide_keys(vt_engine* e, int on);

typedef struct vt_stats {
    uint64_t num_balls, num_slots, num_entries, num_pairs, num_contacts, num_cells;
    uint64_t num_fp64_redo;   /* FP32 pairs recomputed in FP64 */
    uint64_t num_serial;      /* pairs recomputed by the serial (large-contour) kernel */
    double total_sas_area, total_volume, total_contact_area;
    uint32_t device_error_bits;
    uint64_t num_kernel_launches; /* kernels this library launched during the call */
    uint64_t num_cell_redo;       /* FP32 path: cells whose SAS branch needed FP64 inputs */
    uint64_t fp32_kernel;         /* 1 when the FP32 contact kernel ran */
    uint64_t num_host_syncs;      /* waits of the host for the stream (each reads device counts) */
} vt_stats;
int vt_engine_stats(const vt_engine* e, vt_stats* out);

/* Per-stage device times (CUDA events on the engine's stream) of the last call, when
 * timing is on:  [0] prepare  [1] periodic images  [2] grid  [3] neighbour count
 * [4] neighbour fill  [5] contact kernel  [6] FP64 recompute  [7] serial fallback
 * [8] cells  [9] dedup/compaction/totals  [10] whole call (first to last event,
 * including the waits for the three small device->host reads).  Unused stages are 0. */
#define VT_NUM_STAGES 11
/* FP32 path: the error budget E assumed for a contour point coordinate, in float ulps of
 * the pair's length scale R_a + R_b (default 16).  Decisions within an E-derived band of
 * their threshold, and ill-conditioned constructions, send the pair to FP64.  Larger is
 * more conservative (more pairs recomputed in FP64). */
int vt_engine_set_fp32_band(vt_engine* e, double ulps);
int vt_engine_set_timing(vt_engine* e, int on);
/* FP32 mode runs the FP32 contact kernel only when a call (or, in a batch, a structure)
 * has at least this many candidate pairs (default 2048, about 130 balls), and the FP64
 * kernel below it.  A tiny structure's total SAS area is the sum of few contacts, so the
 * FP32 rounding of their solid angles is not averaged out (it adds up coherently on a
 * symmetric input), and such a call is latency bound, so FP64 costs it nothing
 * measurable.  0 forces the FP32 kernel. */
int vt_engine_set_fp32_min_pairs(vt_engine* e, uint64_t min_pairs);
int vt_engine_stage_times(const vt_engine* e, double* ms);

/* Autotuner (no counterpart in the reference): times candidate launch configurations on
 * this input and keeps the fastest for later calls of the engine -- warps per block of the
 * FP32 contact kernel (2, 4 or 8; one warp per pair), its launch form (grid-stride, or
 * persistent with warps taking chunks of 4 or 16 pairs from a work counter; chunk 0 is
 * grid-stride) and the grid cell edge as a multiple of the reach 2 max R + 0.25 (0.5,
 * 0.75, 1 or 1.25; below 1 the neighbour search scans a 5 x 5 x 5 cell stencil culled to
 * the rows and x-ranges within reach).  Results do not depend on any of them.  A new
 * engine (and the one behind the stateless calls) starts with 2 warps, chunks of 4 pairs
 * and scale 0.5.  vt_engine_set_tuning accepts scales in [0.5, 4].
 * batch_offsets: NULL for one structure, else as vt_engine_compute_batch_device. */
int vt_engine_autotune_device(vt_engine* e, const double* d_xyzr, uint64_t n, double probe,
                              const double* periodic_box9, int precision, const uint64_t* batch_offsets,
                              uint64_t num_structures);
int vt_engine_get_tuning(const vt_engine* e, int* warps, double* cell_scale, int* chunk);
int vt_engine_set_tuning(vt_engine* e, int warps, double cell_scale, int chunk);

typedef struct vt_device_outputs {
    const uint32_t* id_a;
    const uint32_t* id_b;
    const double* area;
    const double* arc_length;
    const uint8_t* central;
    const uint32_t* cell_index;
    const double* cell_sas_area;
    const double* cell_volume;
    const double* totals; /* 3 doubles: sas area, volume, contact area */
} vt_device_outputs;
int vt_engine_device_outputs(const vt_engine* e, vt_device_outputs* out);

/* ---- gradient ----
 * No counterpart in the reference: the adjoint of
 *     L = sum_i w_sas[i] SAS_i + sum_i v_volume[i] V_i + sum_k u_contact[k] area_k
 * with respect to every ball's x, y, z and r (SAS_i and V_i of a ball without a cell
 * count as 0; contact k is the k-th contact of the tessellation's output; V_i is the
 * cell volume of compute_sas, types.rs:623-663).  The backward pass recomputes each
 * contact's contour and differentiates the final region analytically (boundary
 * velocities of its edges and arcs; the pyramid volumes through the radical planes'
 * distances); it does not store contours.  Balls of periodic images accumulate into the
 * ball they image; the box is fixed.  Contours of more than 32 points (beyond a warp) are
 * differentiated by a serial kernel; a contour beyond its 256 points is not
 * (VT_ERR_CAPACITY). */
/* After vt_engine_compute_device/_host (full tessellation, one structure): device arrays
 * d_w_sas and d_v_volume (n doubles each) and d_u_contact (one per contact) may each be
 * NULL (no such term); d_grad: n x 4 doubles, overwritten. */
int vt_engine_grad_device(vt_engine* e, const double* d_w_sas, const double* d_v_volume, const double* d_u_contact,
                          double* d_grad);
/* Whether later FP32+fixup computations of the engine keep each contact's FP32 contour
 * (about 24 bytes per contour point in device memory) so that vt_engine_grad_device reads
 * it instead of recomputing it (no counterpart in the reference; off by default; vt_grad
 * and the torch.autograd front end turn it on for their forward). */
int vt_engine_set_keep_contours(vt_engine* e, int on);
/* Forward (as vt_compute_tessellation, no groups) + adjoint on host arrays; u_contact
 * must have num_contacts = the tessellation's contact count entries. */
int vt_grad(const double* xyzr, uint64_t n, double probe, const double* periodic_box9, int precision,
            const double* w_sas, const double* v_volume, const double* u_contact, uint64_t num_contacts,
            double* grad_out);

/* ---- batched structures ----
 * No counterpart in the reference (which tessellates one structure per call): S
 * independent structures concatenated in one N x 4 ball array, structure s being balls
 * [offsets[s], offsets[s+1]) (offsets[0] = 0, non-decreasing, offsets[S] = N).  Each
 * structure is tessellated exactly as compute_tessellation would tessellate it alone
 * (non-periodic; its own grid); the work runs as one pass over all structures.  Contacts
 * and cells of structure s are the ranges [contact_off[s], contact_off[s+1]) and
 * [cell_off[s], cell_off[s+1]) of the concatenated arrays, with ball ids local to the
 * structure, in the same order a single call returns them. */
typedef struct vt_batch_result vt_batch_result;
int vt_compute_batch(const double* xyzr, const uint64_t* offsets, uint64_t num_structures, double probe,
                     int precision, vt_batch_result** out);
/* Device-resident balls (offsets stay in host memory). */
int vt_engine_compute_batch_device(vt_engine* e, const double* d_xyzr, const uint64_t* offsets,
                                   uint64_t num_structures, double probe, int precision, int contacts_only);
int vt_engine_download_batch(vt_engine* e, vt_batch_result** out);
uint64_t vt_batch_num_structures(const vt_batch_result* r);
uint64_t vt_batch_num_contacts(const vt_batch_result* r); /* all structures */
uint64_t vt_batch_num_cells(const vt_batch_result* r);
/* contact_off and cell_off: S + 1 entries each (either may be NULL). */
int vt_batch_ranges(const vt_batch_result* r, uint64_t* contact_off, uint64_t* cell_off);
int vt_batch_contacts(const vt_batch_result* r, uint32_t* id_a, uint32_t* id_b, double* area, double* arc_length,
                      uint8_t* central);
int vt_batch_cells(const vt_batch_result* r, uint32_t* index, double* sas_area, double* volume);
/* 3 doubles per structure: total SAS area, total volume, total contact area. */
int vt_batch_totals(const vt_batch_result* r, double* totals3);
void vt_batch_free(vt_batch_result* r);

/* ---- updateable tessellation ----
 * Replaces UpdateableTessellation (src/updateable.rs:154-742) with its state held on the
 * device: stored balls, exclusion statuses, neighbour lists, the per-ball contact table
 * and the cells.  An update recomputes only the affected balls (the changed balls and
 * their old and new neighbours): neighbour search of those balls, the pairs with both
 * ends affected, their contacts, and the affected cells.  One handle per host thread;
 * each handle owns a CUDA stream on its device.  Return values of the reference's bool
 * methods come back through the int* arguments (may be NULL).
 *
 * Behaviour follows the reference, with one deviation: the neighbour grid is rebuilt
 * from the stored balls, so a ball that crossed a grid cell is not left registered in
 * its old cell (src/spheres_searcher.rs:144-175 removes it from the cell of its new
 * position).  Summary contact order is the reference's: by owning ball, then in the
 * order the contacts were added (src/updateable.rs:332-378). */
typedef struct vt_updateable vt_updateable;
/* new() / with_backup() (src/updateable.rs:154-182); precision VT_FP64 or VT_FP32_FIXUP. */
int vt_upd_create(int device, int with_backup, int precision, vt_updateable** out);
void vt_upd_destroy(vt_updateable* h);
int vt_upd_set_stream(vt_updateable* h, void* stream);
/* init(balls, probe, periodic_box) (src/updateable.rs:187-201); *ok = its return value. */
int vt_upd_init(vt_updateable* h, const double* xyzr, uint64_t n, double probe, const double* periodic_box9,
                int* ok);
/* update(balls) (src/updateable.rs:207-209): every ball compared with the stored one. */
int vt_upd_update(vt_updateable* h, const double* xyzr, uint64_t n, int* changed);
/* update_with_changed(balls, changed_ids) (src/updateable.rs:215-220): only the listed
 * balls are read; ids >= n are ignored. */
int vt_upd_update_with_changed(vt_updateable* h, const double* xyzr, uint64_t n, const uint64_t* ids, uint64_t k,
                               int* changed);
/* Device-resident variants: d_xyzr (n x 4 doubles) and d_ids on the handle's device,
 * ordered on the handle's stream; no host copy of the balls. */
int vt_upd_init_device(vt_updateable* h, const double* d_xyzr, uint64_t n, double probe,
                       const double* periodic_box9, int* ok);
int vt_upd_update_with_changed_device(vt_updateable* h, const double* d_xyzr, uint64_t n, const uint64_t* d_ids,
                                      uint64_t k, int* changed);
/* set_exclusion(id, excluded) (src/updateable.rs:226-271). */
int vt_upd_set_exclusion(vt_updateable* h, uint64_t id, int excluded, int* changed);
/* restore() (src/updateable.rs:277-322): back to the state before the last operation
 * (handles created with backup); *ok = its return value. */
int vt_upd_restore(vt_updateable* h, int* ok);
/* summary() (src/updateable.rs:332-378) as a result object (free with vt_result_free). */
int vt_upd_summary(vt_updateable* h, vt_result** out);
/* total SAS area, volume and contact area of the current summary (3 doubles). */
int vt_upd_totals(vt_updateable* h, double* totals3);
/* last_update_was_full_reinit(), changed_ids(), affected_ids() (src/updateable.rs:380-400). */
int vt_upd_last_full_reinit(const vt_updateable* h);
uint64_t vt_upd_num_changed(const vt_updateable* h);
int vt_upd_changed_ids(vt_updateable* h, uint64_t* out);
uint64_t vt_upd_num_affected(vt_updateable* h);
int vt_upd_affected_ids(vt_updateable* h, uint64_t* out);
/* Adjoint of sum_i w_sas[i] SAS_i over the current state (no counterpart in the
 * reference; the gradient of vt_engine_grad_device restricted to SAS terms): d_w_sas (n
 * doubles on the device, NULL: all 1, the total SAS) and d_grad (n x 4 doubles on the
 * device, overwritten with dL/d(x, y, z, r)).  VT_ERR_INVALID when an operation since
 * the last full computation ran with the adjoint off (vt_upd_set_adjoint). */
int vt_upd_grad_sas(vt_updateable* h, const double* d_w_sas, double* d_grad);
/* Adjoint of sum_i w_sas[i] SAS_i + sum_i v_volume[i] V_i over the current state (no
 * counterpart in the reference): d_w_sas and d_v_volume (n doubles each on the device)
 * may each be NULL (no such term); d_grad (n x 4 doubles on the device) is overwritten
 * with dL/d(x, y, z, r).  V_i is the cell volume of the handle's summary; its adjoint
 * integrates the normal velocity of the cell's boundary (each contact face moves with
 * its radical plane, the exposed sphere with the ball), from per-entry coefficients that
 * the operations record with the SAS ones (vt_upd_set_adjoint).  Same refusal as
 * vt_upd_grad_sas. */
int vt_upd_grad(vt_updateable* h, const double* d_w_sas, const double* d_v_volume, double* d_grad);
/* Whether operations record the arc and face moments behind vt_upd_grad_sas and
 * vt_upd_grad (on by default; no counterpart in the reference).  Off saves about a tenth
 * of an update's time; the adjoint is then refused until a full computation (init, or an
 * update past the full-reinit threshold) has run with it on again. */
int vt_upd_set_adjoint(vt_updateable* h, int on);
/* counters of the last operation: list entries, pairs recomputed, FP64 redo, cells */
int vt_upd_stats(const vt_updateable* h, vt_stats* out);
/* Per-stage device times (CUDA events on the handle's stream) of the last
 * update_with_changed / update that did not fall back to a full reinit, when timing is
 * on (no counterpart in the reference):  [0] changed filter and marks  [1] apply, spheres,
 * images, grid  [2] frontier neighbour searches  [3] list splice and affected set
 * [4] pair generation  [5] contacts (FP32 or FP64, band recompute, serial)  [6] dedup,
 * contact-table splice, cells  [7] FP64 refresh of uncertain cells  [8] cell count,
 * error word  [9] the whole update (first to last event, including the host's reads of
 * device counts between stages).  Unused stages are 0. */
#define VT_UPD_NUM_STAGES 10
int vt_upd_set_timing(vt_updateable* h, int on);
int vt_upd_stage_times(const vt_updateable* h, double* ms);

/* ---- contact descriptors without device allocation ----
 * No counterpart in the reference: an entry point for callers that cannot call
 * cudaMalloc/cudaFree while they run (a custom call inside a framework whose allocator
 * owns the device, a real-time loop that must not hit the allocator, a plugin host that
 * only hands out pre-allocated buffers).  It runs the serial contour kernel
 * (construct_contact_descriptor for each pair; no neighbour search) with its scratch in a
 * static device array of VT_NOALLOC_SCRATCH_BYTES that every GPU loading this library
 * holds until the process exits; it allocates nothing.
 *
 * All pointers are device memory on the current device.  d_spheres: num_spheres x 4
 * doubles (x, y, z, R with R = r + probe).  Neighbour lists are per sphere: sphere a's
 * list is d_nb_index[d_nb_offsets[a] .. d_nb_offsets[a+1]) in find_colliding_ids order
 * (sorted by distance to the intersection-circle centre, then index).  Pair k is
 * (d_pair_a[k], d_pair_b[k]).  Outputs per pair: status (1 contact, 0 none), area, arc
 * length, central, and, if d_solid_a is not NULL, solid angles and pyramid volumes (all
 * four or none).  Results equal the regular FP64 path's for the same lists.
 *
 * Limit: every listed a must have at most VT_NOALLOC_MAX_NEIGHBORS neighbours (the
 * scratch holds 192 contour points per pair, the peak a 57-entry list can reach);
 * otherwise the call returns VT_ERR_CAPACITY before computing anything.  Malformed input
 * (a pair or neighbour index not below num_spheres, offsets not ascending within the
 * index array of d_nb_offsets[num_spheres] entries, a non-finite coordinate or a
 * negative radius among the spheres the pairs read) returns VT_ERR_INVALID, also before
 * any contact is computed.  The first call on a device looks up the
 * scratch's device address and uploads a small table, so make it before any stream
 * capture.  Calls share the one scratch array: calls that overlap on the GPU race and
 * must be serialised (one stream, or host-side ordering).  The call returns after its
 * work on `stream` (a cudaStream_t, NULL for the default stream) has finished. */
#define VT_NOALLOC_MAX_NEIGHBORS 57
#define VT_NOALLOC_SCRATCH_BYTES 9437440
int vt_contact_descriptors_noalloc(const double* d_spheres, uint64_t num_spheres, const uint32_t* d_nb_offsets,
                                   const uint32_t* d_nb_index, const uint32_t* d_pair_a, const uint32_t* d_pair_b,
                                   uint64_t num_pairs, uint8_t* d_status, double* d_area, double* d_arc_length,
                                   uint8_t* d_central, double* d_solid_a, double* d_solid_b, double* d_pyramid_a,
                                   double* d_pyramid_b, void* stream);

/* Human-readable status, and the message of the calling thread's last error. */
const char* vt_status_string(int status);
const char* vt_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
