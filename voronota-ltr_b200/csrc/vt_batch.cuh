// vt_batch.cuh -- launchers of the batched tessellation (vt_batch.cu).
//
// Layout: S structures concatenated; off u32[S+1] gives each structure's ball range.
//   ball_struct u32[N]   structure of each ball
//   grids GridDev[S], cell_base u32[S+1]: structure s owns cells
//                        [cell_base[s], cell_base[s+1]) of the concatenated grid
//   outputs: contacts and cells of structure s are the ranges
//            [contact_range[s], contact_range[s+1]) and [cell_range[s], cell_range[s+1])
//            of the compacted arrays, with ids local to the structure
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "vt_pipeline.cuh"

namespace vt {

// ball_struct, per-structure bounding boxes, grids and cell counts (ncell u32[S]).
void launch_batch_grid_setup(const uint32_t* off, uint32_t S, uint32_t N, const double4* sph, uint32_t* ball_struct,
                             BBox* bboxes, GridDev* grids, uint32_t* ncell, double cell_scale, cudaStream_t s);
// Counting sort of the balls into the concatenated grid (b.cell_base filled).
void launch_batch_grid(const DevBufs& b, uint32_t N, uint32_t total_cells, uint32_t* scan_tmp, cudaStream_t s);
// FP32 mode: the pairs of structures with fewer than min_pairs candidate pairs are marked
// for the FP64 recompute (a single call on such a structure runs FP64).
void launch_batch_small_unsure(const DevBufs& b, const uint32_t* off, uint32_t P, uint64_t min_pairs,
                               cudaStream_t s);
// Per-structure contact / cell ranges, local ids, per-structure totals (3 doubles per
// structure: SAS area, volume, contact area).
void launch_batch_outputs(const DevBufs& b, const uint32_t* off, uint32_t S, uint32_t P, int contacts_only,
                          uint32_t* contact_range, uint32_t* cell_range, double* totals, cudaStream_t s);

}  // namespace vt
