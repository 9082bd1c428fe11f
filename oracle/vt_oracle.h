/*
 * vt_oracle.h -- C API of the CPU oracle (test infrastructure, NOT product code).
 *
 * The oracle is a plain C++ f64 restatement of voronota-ltr's radical-tessellation
 * hot path (src/geometry.rs, src/spheres_searcher.rs, src/contact.rs,
 * src/tessellation.rs, src/types.rs, src/spheres_container.rs, src/updateable.rs).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * always as the checker / the timed CPU baseline, never as a product path.
 *
 * Ids are uint64 (the reference uses usize).  A periodic box is given by its three
 * lattice vectors (9 doubles: a.xyz, b.xyz, c.xyz); corners map to diagonal vectors
 * exactly as PeriodicBox::from_corners (types.rs:304-310).
 */
#ifndef VT_ORACLE_H
#define VT_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct vto_result vto_result;
typedef struct vto_upd vto_upd;

/* Number of OpenMP threads used for the per-ball and per-pair loops (<=0: all). */
void vto_set_threads(int n);
int vto_get_threads(void);
/* Incremental grid update of SpheresSearcher::update (spheres_searcher.rs:144-175).
 * on (default): exactly as the reference, whose removal looks a moved sphere up in its
 * NEW cell, leaving a stale registration in the old cell when the sphere crossed a
 * cell boundary.  off: removal uses the old position, so incremental updates equal a
 * full recompute (the contract the reference's tests/updateable.rs asserts). */
void vto_set_faithful_grid_update(int on);

/* compute_tessellation (tessellation.rs:37) when contacts_only == 0, else
 * compute_contacts_only (tessellation.rs:125).  Returns 0 on success. */
int vto_compute(const double* xyzr, uint64_t n, double probe, const double* pbox9,
                const int32_t* groups, uint64_t n_groups, int contacts_only,
                vto_result** out);

uint64_t vto_num_balls(const vto_result* r);
uint64_t vto_num_contacts(const vto_result* r);
uint64_t vto_num_cells(const vto_result* r);
void vto_get_contacts(const vto_result* r, uint64_t* id_a, uint64_t* id_b, double* area,
                      double* arc_length, uint8_t* central);
void vto_get_cells(const vto_result* r, uint64_t* index, double* sas_area, double* volume);

/* Internals kept for stage-by-stage parity checks of the GPU kernels. */
/* neighbour CSR for balls 0..n-1 (find_colliding_ids results, sorted) */
uint64_t vto_num_neighbor_entries(const vto_result* r);
void vto_get_neighbors(const vto_result* r, uint64_t* offsets /* n+1 */, uint64_t* ids,
                       double* values);
/* candidate pairs (collect_collision_pairs order) and per-pair descriptors.
 * valid[k] = 1 when the pair produced a contact (area > 0). Values of invalid
 * pairs are 0.  Descriptor ids are the pair's own (a, b) before canonicalisation. */
uint64_t vto_num_pairs(const vto_result* r);
void vto_get_pairs(const vto_result* r, uint64_t* a, uint64_t* b, uint8_t* valid,
                   double* area, double* arc_length, uint8_t* central,
                   double* solid_a, double* solid_b, double* pyr_a, double* pyr_b);
void vto_free(vto_result* r);
/* Tessellation network (with_cell_vertices, contact.rs:119-177, tessellation.rs:334-401):
 * when on, vto_compute (full tessellation) also builds the deduplicated vertices (4 sorted
 * ball ids, NULL id = UINT64_MAX, and x, y, z) and edges (3 sorted ids and length). */
void vto_set_network(int on);
uint64_t vto_num_vertices(const vto_result* r);
uint64_t vto_num_edges(const vto_result* r);
void vto_get_vertices(const vto_result* r, uint64_t* ids4, double* xyz3);
void vto_get_edges(const vto_result* r, uint64_t* ids3, double* length);

/* UpdateableTessellation (updateable.rs:154-742). */
vto_upd* vto_upd_create(int with_backup);
void vto_upd_destroy(vto_upd* h);
int vto_upd_init(vto_upd* h, const double* xyzr, uint64_t n, double probe, const double* pbox9);
int vto_upd_update(vto_upd* h, const double* xyzr, uint64_t n);
int vto_upd_update_with_changed(vto_upd* h, const double* xyzr, uint64_t n,
                                const uint64_t* changed, uint64_t k);
int vto_upd_set_exclusion(vto_upd* h, uint64_t id, int excluded);
int vto_upd_restore(vto_upd* h);
int vto_upd_last_full_reinit(const vto_upd* h);
uint64_t vto_upd_num_changed(const vto_upd* h);
void vto_upd_get_changed(const vto_upd* h, uint64_t* ids);
uint64_t vto_upd_num_affected(const vto_upd* h);
void vto_upd_get_affected(const vto_upd* h, uint64_t* ids);
/* summary() (updateable.rs:332-378) as a result object; free with vto_free. */
vto_result* vto_upd_summary(const vto_upd* h);

/* compute_solvent_spheres (solvent_spheres.rs:131-169): 0 ok, 1 invalid probe,
 * 2 invalid volume probe, 3 invalid ball.  Spheres in the reference's order (cells by
 * index, then icosahedron vertex order); x, y, z, radius, weight per sphere. */
typedef struct vto_solvent vto_solvent;
int vto_icosahedron(int depth, double* xyz3);
int vto_solvent_spheres(const double* xyzr, uint64_t n, double probe, double volume_probe, int depth,
                        const double* pbox9, vto_solvent** out);
uint64_t vto_solvent_count(const vto_solvent* s);
void vto_solvent_get(const vto_solvent* s, double* xyzrw5, uint64_t* parent);
void vto_solvent_free(vto_solvent* s);

#ifdef __cplusplus
}
#endif
#endif
