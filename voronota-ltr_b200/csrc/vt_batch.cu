// vt_batch.cu -- kernels of the batched tessellation: many independent structures
// concatenated into one ball array and tessellated by one launch per stage.
//
// Every structure gets its own cell grid (its own bounding box and cell edge, as a
// single-structure call would), laid out one after the other in the cell arrays, so the
// neighbour search of a ball only ever sees balls of its own structure.  Pairs, contacts
// and cells are then global arrays in which each structure owns a contiguous range.
#include <cfloat>
#include <cmath>

#include "vt_batch.cuh"

namespace vt {

namespace {

constexpr int kBlock = 256;

__global__ void k_ball_struct(const uint32_t* __restrict__ off, uint32_t S, uint32_t* __restrict__ ball_struct) {
    for (uint32_t s = blockIdx.x; s < S; s += gridDim.x)
        for (uint32_t i = off[s] + threadIdx.x; i < off[s + 1]; i += blockDim.x) ball_struct[i] = s;
}

// per-structure bounding box and max R (block per structure, fixed reduction tree)
__global__ void k_struct_bbox(const double4* __restrict__ sph, const uint32_t* __restrict__ off, uint32_t S,
                              BBox* __restrict__ out) {
    __shared__ double sh[7][kBlock];
    const int t = threadIdx.x;
    for (uint32_t s = blockIdx.x; s < S; s += gridDim.x) {
        double v[7] = {DBL_MAX, DBL_MAX, DBL_MAX, -DBL_MAX, -DBL_MAX, -DBL_MAX, 0.0};
        for (uint32_t i = off[s] + t; i < off[s + 1]; i += blockDim.x) {
            const double4 p = sph[i];
            v[0] = fmin(v[0], p.x);
            v[1] = fmin(v[1], p.y);
            v[2] = fmin(v[2], p.z);
            v[3] = fmax(v[3], p.x);
            v[4] = fmax(v[4], p.y);
            v[5] = fmax(v[5], p.z);
            v[6] = fmax(v[6], p.w);
        }
        for (int k = 0; k < 7; ++k) sh[k][t] = v[k];
        __syncthreads();
        for (int o = kBlock / 2; o > 0; o >>= 1) {
            if (t < o) {
                for (int k = 0; k < 3; ++k) sh[k][t] = fmin(sh[k][t], sh[k][t + o]);
                for (int k = 3; k < 7; ++k) sh[k][t] = fmax(sh[k][t], sh[k][t + o]);
            }
            __syncthreads();
        }
        if (t == 0) {
            BBox b;
            for (int k = 0; k < 3; ++k) {
                b.mn[k] = sh[k][0];
                b.mx[k] = sh[k + 3][0];
            }
            b.max_r = sh[6][0];
            out[s] = b;
        }
        __syncthreads();
    }
}

// plan_grid per structure: cell edge = cell_scale x max(2 max R + 0.25, 1) (cell_scale >=
// 0.5), coarsened so that the structure's grid has at most 8 n_s + 4096 cells
__global__ void k_struct_grid(const BBox* __restrict__ bb, const uint32_t* __restrict__ off, uint32_t S,
                              double cell_scale, GridDev* __restrict__ grids, uint32_t* __restrict__ ncell) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        const uint32_t ns = off[s + 1] - off[s];
        GridDev g{};
        if (ns == 0) {
            g.cell = 1.0;
            g.reach = 1.0;
            g.half = 1;
            g.dx = g.dy = g.dz = 1;
            grids[s] = g;
            ncell[s] = 0;
            continue;
        }
        const BBox b = bb[s];
        const double reach = fmax(2.0 * b.max_r + 0.25, 1.0);
        double ext[3];
        for (int k = 0; k < 3; ++k) ext[k] = (b.mx[k] - b.mn[k]) + 2.0 * reach;
        double cell = reach * (cell_scale > 0.5 ? cell_scale : 0.5);
        int d[3];
        for (int k = 0; k < 3; ++k) d[k] = (int)floor(ext[k] / cell) + 1;
        double vol = (double)d[0] * d[1] * d[2];
        const double max_cells = 8.0 * (double)ns + 4096.0;
        for (int it = 0; it < 64 && vol > max_cells; ++it) {
            cell *= cbrt(vol / max_cells) * 1.01;
            for (int k = 0; k < 3; ++k) d[k] = (int)floor(ext[k] / cell) + 1;
            vol = (double)d[0] * d[1] * d[2];
        }
        g.cell = cell;
        g.reach = reach;
        g.half = cell >= reach ? 1 : 2;
        g.ox = b.mn[0] - reach;
        g.oy = b.mn[1] - reach;
        g.oz = b.mn[2] - reach;
        g.dx = d[0];
        g.dy = d[1];
        g.dz = d[2];
        grids[s] = g;
        ncell[s] = (uint32_t)(d[0] * d[1] * d[2]);
    }
}

__global__ void k_batch_cell_hist(const double4* __restrict__ sph, uint32_t N, const uint32_t* __restrict__ bs,
                                  const GridDev* __restrict__ grids, const uint32_t* __restrict__ base,
                                  uint32_t* __restrict__ cnt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const uint32_t s = bs[i];
        atomicAdd(&cnt[base[s] + slot_cell(grids[s], sph[i])], 1u);
    }
}
__global__ void k_batch_cell_scatter(const double4* __restrict__ sph, uint32_t N, const uint32_t* __restrict__ bs,
                                     const GridDev* __restrict__ grids, const uint32_t* __restrict__ base,
                                     uint32_t* __restrict__ cursor, double4* __restrict__ c_pos,
                                     uint32_t* __restrict__ c_id, uint32_t* __restrict__ c_slot) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const uint32_t s = bs[i];
        const double4 p = sph[i];
        const uint32_t at = atomicAdd(&cursor[base[s] + slot_cell(grids[s], p)], 1u);
        c_pos[at] = p;
        c_id[at] = i;
        c_slot[at] = i;
    }
}

// contact and cell ranges of each structure in the compacted outputs
__global__ void k_batch_offsets(const uint32_t* __restrict__ off, uint32_t S, const uint32_t* __restrict__ pair_off,
                                const uint32_t* __restrict__ keep_off, const uint32_t* __restrict__ cell_off,
                                uint32_t* __restrict__ contact_range, uint32_t* __restrict__ cell_range) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s <= S; s += gridDim.x * blockDim.x) {
        const uint32_t first = off[s];
        contact_range[s] = keep_off[pair_off[first]];
        cell_range[s] = cell_off ? cell_off[first] : 0u;
    }
}
// ids local to the structure
__global__ void k_batch_localize(uint32_t* __restrict__ ids, const uint32_t* __restrict__ count,
                                 const uint32_t* __restrict__ bs, const uint32_t* __restrict__ off) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        ids[k] -= off[bs[ids[k]]];
}
__global__ void k_batch_localize_pair(uint32_t* __restrict__ a, uint32_t* __restrict__ b,
                                      const uint32_t* __restrict__ count, const uint32_t* __restrict__ bs,
                                      const uint32_t* __restrict__ off) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t base = off[bs[a[k]]];
        a[k] -= base;
        b[k] -= base;
    }
}

// pairs of structures with fewer than min_pairs candidate pairs: FP64 like a single call on
// such a structure (marked unsure, so the FP64 recompute takes them)
__global__ void k_batch_small_unsure(const uint32_t* __restrict__ pair_a, const uint32_t* __restrict__ bs,
                                     const uint32_t* __restrict__ off, const uint32_t* __restrict__ pair_off,
                                     uint32_t P, uint64_t min_pairs, uint8_t* __restrict__ status) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const uint32_t s = bs[pair_a[p]];
        if ((uint64_t)(pair_off[off[s + 1]] - pair_off[off[s]]) < min_pairs && !(status[p] & kOverflow))
            status[p] |= kUnsure;
    }
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int o = kBlock / 2; o > 0; o >>= 1) {
        if (t < o) sh[t] += sh[t + o];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}
// per-structure totals (Results, types.rs:230-252): block per structure, fixed tree
__global__ void k_batch_totals(const uint32_t* __restrict__ crange, const uint32_t* __restrict__ mrange, uint32_t S,
                               const double* __restrict__ area, const double* __restrict__ sas,
                               const double* __restrict__ vol, double* __restrict__ totals) {
    __shared__ double sh[kBlock];
    for (uint32_t s = blockIdx.x; s < S; s += gridDim.x) {
        double a = 0.0, x = 0.0, v = 0.0;
        for (uint32_t k = crange[s] + threadIdx.x; k < crange[s + 1]; k += blockDim.x) a += area[k];
        if (mrange)
            for (uint32_t k = mrange[s] + threadIdx.x; k < mrange[s + 1]; k += blockDim.x) {
                x += sas[k];
                v += vol[k];
            }
        a = block_sum(a, sh);
        x = block_sum(x, sh);
        v = block_sum(v, sh);
        if (threadIdx.x == 0) {
            totals[3 * s] = x;
            totals[3 * s + 1] = v;
            totals[3 * s + 2] = a;
        }
    }
}

int gb(size_t n) { return grid_blocks(n, kBlock, 148 * 16); }

}  // namespace

void launch_batch_grid_setup(const uint32_t* off, uint32_t S, uint32_t N, const double4* sph, uint32_t* ball_struct,
                             BBox* bboxes, GridDev* grids, uint32_t* ncell, double cell_scale, cudaStream_t s) {
    const int sb = (int)(S < 148u * 8u ? S : 148u * 8u);
    k_ball_struct<<<sb > 0 ? sb : 1, kBlock, 0, s>>>(off, S, ball_struct); count_launch();
    k_struct_bbox<<<sb > 0 ? sb : 1, kBlock, 0, s>>>(sph, off, S, bboxes); count_launch();
    k_struct_grid<<<gb(S), kBlock, 0, s>>>(bboxes, off, S, cell_scale > 1.0 ? cell_scale : 1.0, grids, ncell);
    count_launch();
    (void)N;
}
void launch_batch_grid(const DevBufs& b, uint32_t N, uint32_t total_cells, uint32_t* scan_tmp, cudaStream_t s) {
    cudaMemsetAsync(b.cell_count, 0, sizeof(uint32_t) * total_cells, s);
    k_batch_cell_hist<<<gb(N), kBlock, 0, s>>>(b.sph, N, b.ball_struct, b.grids, b.cell_base, b.cell_count);
    count_launch();
    scan_u32(b.cell_count, b.cell_start, total_cells, scan_tmp, s);
    cudaMemcpyAsync(b.cell_cursor, b.cell_start, sizeof(uint32_t) * total_cells, cudaMemcpyDeviceToDevice, s);
    k_batch_cell_scatter<<<gb(N), kBlock, 0, s>>>(b.sph, N, b.ball_struct, b.grids, b.cell_base, b.cell_cursor,
                                                  b.c_pos, b.c_id, b.c_slot);
    count_launch();
}
void launch_batch_small_unsure(const DevBufs& b, const uint32_t* off, uint32_t P, uint64_t min_pairs,
                               cudaStream_t s) {
    if (P == 0 || min_pairs == 0) return;
    k_batch_small_unsure<<<gb(P), kBlock, 0, s>>>(b.pair_a, b.ball_struct, off, b.pair_off, P, min_pairs, b.p_status);
    count_launch();
}
void launch_batch_outputs(const DevBufs& b, const uint32_t* off, uint32_t S, uint32_t P, int contacts_only,
                          uint32_t* contact_range, uint32_t* cell_range, double* totals, cudaStream_t s) {
    k_batch_offsets<<<gb(S + 1), kBlock, 0, s>>>(off, S, b.pair_off, b.keep_off, contacts_only ? nullptr : b.cell_off,
                                                 contact_range, cell_range);
    count_launch();
    const uint32_t* ccount = b.keep_off + P;
    k_batch_localize_pair<<<gb(P), kBlock, 0, s>>>(b.out_a, b.out_b, ccount, b.ball_struct, off); count_launch();
    if (!contacts_only) {
        k_batch_localize<<<gb(b.n), kBlock, 0, s>>>(b.out_cell_index, b.cell_off + b.n, b.ball_struct, off);
        count_launch();
    }
    const int sb = (int)(S < 148u * 8u ? S : 148u * 8u);
    k_batch_totals<<<sb > 0 ? sb : 1, kBlock, 0, s>>>(contact_range, contacts_only ? nullptr : cell_range, S,
                                                      b.out_area, b.out_cell_sas, b.out_cell_vol, totals);
    count_launch();
}

}  // namespace vt
