// vt_solvent.cuh -- launchers of compute_solvent_spheres' device stages (vt_solvent.cu).
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "vt_pipeline.cuh"

namespace vt {

// Device buffers of one solvent-sphere call (n balls, M stage-1 cells, K directions).
struct SolventBufs {
    uint8_t* exposed;     // n
    uint32_t* deg;        // n + 1: partner counts of exposed balls
    uint32_t* poff;       // n + 1: their exclusive scan
    uint32_t* cursor;     // n
    uint32_t* partners;   // poff[n]
    const double* dirs;   // 3 K unit directions
    uint32_t* mask;       // M * ceil(K / 32) ballot words
    uint32_t* count;      // M + 1 kept points per cell
    uint32_t* soff;       // M + 2: their exclusive scan
    double* sol_xyz;      // 3 S
    uint32_t* sol_parent; // S
};

// SubdividedIcosahedron::new (subdivided_icosahedron.rs:53-125): unit directions, the 12
// icosahedron vertices and then, per depth (clamped to 0..4), each face split in four
// with an edge's midpoint appended the first time the edge is met.
std::vector<double> icosahedron_directions(int depth);

// exposed flags and the partners CSR from the stage-1 outputs (C contacts, M cells)
void launch_solvent_partners(const uint32_t* a, const uint32_t* b, uint32_t C, const uint32_t* cell_index,
                             const double* cell_sas, uint32_t M, uint32_t n, SolventBufs& t, uint32_t* scan_tmp,
                             cudaStream_t s);
// kept-point ballot words and per-cell counts
void launch_solvent_mask(const double* xyzr, const uint32_t* cell_index, const double* cell_sas, uint32_t M,
                         const SolventBufs& t, uint32_t K, double probe, cudaStream_t s);
// kept points (t.soff filled) and the combined stage-2 balls (n atoms, then the spheres)
void launch_solvent_write(const double* xyzr, const uint32_t* cell_index, uint32_t M, const SolventBufs& t,
                          uint32_t K, double probe, double volume_probe, uint32_t n, double* combined,
                          cudaStream_t s);
// weights = stage-2 cell volumes of the spheres (0 for a sphere without a cell)
void launch_solvent_weights(const uint32_t* cell_index, const double* cell_vol, uint32_t M, uint32_t n, uint32_t S,
                            double* weight, cudaStream_t s);

}  // namespace vt
