// vt_solvent.cu -- compute_solvent_spheres (solvent_spheres.rs:131-345) on the device:
// the stages between the two tessellations (compiled with --fmad=false, so positions and
// distances are the reference's f64 values and every keep/drop decision matches it).
//
//   exposed     ball i is exposed when its cell has sas_area > 0
//   partners    CSR of each exposed ball's contact partners (both ends of every output
//               contact; a periodic self-contact lists the ball twice, as the reference's
//               neighbour graph does)
//   mask/count  warp per cell, lanes over the sample directions: a point p = c + v (r +
//               probe) is kept when |p - c_j| - r_j > |p - c| - r for every partner j;
//               one ballot word per 32 directions
//   write       kept points in cell order then direction order (a scan of the counts and
//               the ballot ranks), with the combined stage-2 ball array
//   weights     a solvent sphere's weight is the stage-2 volume of its cell
#include <cmath>
#include <map>
#include <vector>

#include "vt_solvent.cuh"

namespace vt {

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = 8;

__global__ void k_exposed(const uint32_t* __restrict__ cell_index, const double* __restrict__ cell_sas, uint32_t M,
                          uint8_t* __restrict__ exposed) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x)
        if (cell_sas[k] > 0.0) exposed[cell_index[k]] = 1;
}

__global__ void k_partner_count(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint32_t C,
                                const uint8_t* __restrict__ exposed, uint32_t* __restrict__ deg) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
        if (exposed[a[k]]) atomicAdd(&deg[a[k]], 1u);
        if (exposed[b[k]]) atomicAdd(&deg[b[k]], 1u);
    }
}

// the order of a ball's partners does not change the result (every partner is tested)
__global__ void k_partner_fill(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint32_t C,
                               const uint8_t* __restrict__ exposed, uint32_t* __restrict__ cursor,
                               uint32_t* __restrict__ partners) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
        if (exposed[a[k]]) partners[atomicAdd(&cursor[a[k]], 1u)] = b[k];
        if (exposed[b[k]]) partners[atomicAdd(&cursor[b[k]], 1u)] = a[k];
    }
}

__device__ __forceinline__ double dist3(double px, double py, double pz, double cx, double cy, double cz) {
    const double dx = px - cx, dy = py - cy, dz = pz - cz;
    return sqrt((dx * dx + dy * dy) + dz * dz);
}

__device__ __forceinline__ bool keep_point(const double* __restrict__ xyzr, const uint32_t* __restrict__ partners,
                                           uint32_t p0, uint32_t p1, double px, double py, double pz, double cx,
                                           double cy, double cz, double r) {
    const double da = dist3(px, py, pz, cx, cy, cz) - r;
    for (uint32_t e = p0; e < p1; ++e) {
        const double* q = xyzr + 4 * (size_t)partners[e];
        if (dist3(px, py, pz, q[0], q[1], q[2]) - q[3] <= da) return false;
    }
    return true;
}

__global__ void __launch_bounds__(kWarps * 32)
    k_solvent_mask(const double* __restrict__ xyzr, const uint32_t* __restrict__ cell_index,
                   const double* __restrict__ cell_sas, uint32_t M, const uint32_t* __restrict__ poff,
                   const uint32_t* __restrict__ partners, const double* __restrict__ dirs, uint32_t K, double probe,
                   uint32_t* __restrict__ mask, uint32_t* __restrict__ count) {
    const int lane = threadIdx.x & 31;
    const uint32_t words = (K + 31) / 32;
    for (uint32_t k = blockIdx.x * kWarps + (threadIdx.x >> 5); k < M; k += gridDim.x * kWarps) {
        uint32_t total = 0;
        if (cell_sas[k] > 0.0) {
            const uint32_t i = cell_index[k];
            const double cx = xyzr[4 * (size_t)i], cy = xyzr[4 * (size_t)i + 1], cz = xyzr[4 * (size_t)i + 2];
            const double r = xyzr[4 * (size_t)i + 3], R = r + probe;
            const uint32_t p0 = poff[i], p1 = poff[i + 1];
            for (uint32_t w = 0; w < words; ++w) {
                const uint32_t j = w * 32 + lane;
                bool ok = false;
                if (j < K) {
                    const double px = cx + dirs[3 * j] * R, py = cy + dirs[3 * j + 1] * R,
                                 pz = cz + dirs[3 * j + 2] * R;
                    ok = keep_point(xyzr, partners, p0, p1, px, py, pz, cx, cy, cz, r);
                }
                const uint32_t bits = __ballot_sync(0xffffffffu, ok);
                if (lane == 0) mask[(size_t)k * words + w] = bits;
                total += __popc(bits);
            }
        } else if (lane == 0) {
            for (uint32_t w = 0; w < words; ++w) mask[(size_t)k * words + w] = 0u;
        }
        if (lane == 0) count[k] = total;
    }
}

__global__ void __launch_bounds__(kWarps * 32)
    k_solvent_write(const double* __restrict__ xyzr, const uint32_t* __restrict__ cell_index, uint32_t M,
                    const double* __restrict__ dirs, uint32_t K, double probe, double volume_probe,
                    const uint32_t* __restrict__ mask, const uint32_t* __restrict__ soff, uint32_t n,
                    double* __restrict__ sol_xyz, uint32_t* __restrict__ sol_parent, double* __restrict__ combined) {
    const int lane = threadIdx.x & 31;
    const uint32_t words = (K + 31) / 32;
    for (uint32_t k = blockIdx.x * kWarps + (threadIdx.x >> 5); k < M; k += gridDim.x * kWarps) {
        if (soff[k + 1] == soff[k]) continue;
        const uint32_t i = cell_index[k];
        const double cx = xyzr[4 * (size_t)i], cy = xyzr[4 * (size_t)i + 1], cz = xyzr[4 * (size_t)i + 2];
        const double R = xyzr[4 * (size_t)i + 3] + probe;
        uint32_t at = soff[k];
        for (uint32_t w = 0; w < words; ++w) {
            const uint32_t bits = mask[(size_t)k * words + w];
            const uint32_t j = w * 32 + lane;
            if ((bits >> lane) & 1u) {
                const uint32_t s = at + __popc(bits & ((1u << lane) - 1u));
                const double px = cx + dirs[3 * j] * R, py = cy + dirs[3 * j + 1] * R, pz = cz + dirs[3 * j + 2] * R;
                sol_xyz[3 * (size_t)s] = px;
                sol_xyz[3 * (size_t)s + 1] = py;
                sol_xyz[3 * (size_t)s + 2] = pz;
                sol_parent[s] = i;
                double* c = combined + 4 * ((size_t)n + s);
                c[0] = px;
                c[1] = py;
                c[2] = pz;
                c[3] = probe + volume_probe;
            }
            at += __popc(bits);
        }
    }
}

// original atoms of the stage-2 input: radius max(r - probe + volume_probe, 0.01)
__global__ void k_combined_atoms(const double* __restrict__ xyzr, uint32_t n, double probe, double volume_probe,
                                 double* __restrict__ combined) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double* b = xyzr + 4 * (size_t)i;
        double* c = combined + 4 * (size_t)i;
        c[0] = b[0];
        c[1] = b[1];
        c[2] = b[2];
        c[3] = fmax(b[3] - probe + volume_probe, 0.01);
    }
}

__global__ void k_solvent_weights(const uint32_t* __restrict__ cell_index, const double* __restrict__ cell_vol,
                                  uint32_t M, uint32_t n, uint32_t S, double* __restrict__ weight) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
        const uint32_t idx = cell_index[k];
        if (idx >= n && idx - n < S) weight[idx - n] = cell_vol[k];
    }
}

int gb(size_t n) { return grid_blocks(n, kBlock, 148 * 16); }

struct Dir {
    double x, y, z;
};
Dir unit(double x, double y, double z) {
    const double nn = std::sqrt((x * x + y * y) + z * z);
    return {x / nn, y / nn, z / nn};
}

}  // namespace

std::vector<double> icosahedron_directions(int depth) {
    if (depth < 0) depth = 0;
    if (depth > 4) depth = 4;
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<Dir> v = {unit(t, 1.0, 0.0),  unit(-t, 1.0, 0.0),  unit(t, -1.0, 0.0), unit(-t, -1.0, 0.0),
                                 unit(1.0, 0.0, t),  unit(1.0, 0.0, -t),  unit(-1.0, 0.0, t), unit(-1.0, 0.0, -t),
                                 unit(0.0, t, 1.0),  unit(0.0, -t, 1.0),  unit(0.0, t, -1.0), unit(0.0, -t, -1.0)};
    struct Face {
        uint32_t v[3];
    };
    std::vector<Face> faces = {{{0, 8, 4}},  {{1, 10, 7}}, {{2, 9, 11}}, {{7, 3, 1}},  {{0, 5, 10}},
                               {{3, 9, 6}},  {{3, 11, 9}}, {{8, 6, 4}},  {{2, 4, 9}},  {{3, 7, 11}},
                               {{4, 2, 0}},  {{9, 4, 6}},  {{2, 11, 5}}, {{0, 10, 8}}, {{5, 0, 2}},
                               {{10, 5, 7}}, {{1, 6, 8}},  {{1, 8, 10}}, {{6, 1, 3}},  {{11, 7, 5}}};
    for (int d = 0; d < depth; ++d) {
        std::map<uint64_t, uint32_t> mid_of;  // edge (lo, hi) -> midpoint vertex
        std::vector<Face> next;
        next.reserve(4 * faces.size());
        for (const Face& f : faces) {
            const uint32_t ends[3][2] = {{f.v[1], f.v[2]}, {f.v[0], f.v[2]}, {f.v[0], f.v[1]}};
            uint32_t m[3];
            for (int e = 0; e < 3; ++e) {
                const uint32_t lo = ends[e][0] < ends[e][1] ? ends[e][0] : ends[e][1];
                const uint32_t hi = ends[e][0] < ends[e][1] ? ends[e][1] : ends[e][0];
                const uint64_t key = ((uint64_t)lo << 32) | hi;
                auto it = mid_of.find(key);
                if (it == mid_of.end()) {
                    const Dir p = v[ends[e][0]];
                    const Dir q = v[ends[e][1]];
                    v.push_back(unit((p.x + q.x) * 0.5, (p.y + q.y) * 0.5, (p.z + q.z) * 0.5));
                    it = mid_of.emplace(key, (uint32_t)(v.size() - 1)).first;
                }
                m[e] = it->second;
            }
            next.push_back({{f.v[0], m[1], m[2]}});
            next.push_back({{f.v[1], m[0], m[2]}});
            next.push_back({{f.v[2], m[0], m[1]}});
            next.push_back({{m[0], m[1], m[2]}});
        }
        faces.swap(next);
    }
    std::vector<double> out(3 * v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        out[3 * i] = v[i].x;
        out[3 * i + 1] = v[i].y;
        out[3 * i + 2] = v[i].z;
    }
    return out;
}

void launch_solvent_partners(const uint32_t* a, const uint32_t* b, uint32_t C, const uint32_t* cell_index,
                             const double* cell_sas, uint32_t M, uint32_t n, SolventBufs& t, uint32_t* scan_tmp,
                             cudaStream_t s) {
    cudaMemsetAsync(t.exposed, 0, n, s);
    cudaMemsetAsync(t.deg, 0, sizeof(uint32_t) * (n + 1), s);
    if (M) {
        k_exposed<<<gb(M), kBlock, 0, s>>>(cell_index, cell_sas, M, t.exposed); count_launch();
    }
    if (C) {
        k_partner_count<<<gb(C), kBlock, 0, s>>>(a, b, C, t.exposed, t.deg); count_launch();
    }
    scan_u32(t.deg, t.poff, n, scan_tmp, s);
    cudaMemcpyAsync(t.cursor, t.poff, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s);
    if (C) {
        k_partner_fill<<<gb(C), kBlock, 0, s>>>(a, b, C, t.exposed, t.cursor, t.partners); count_launch();
    }
}

void launch_solvent_mask(const double* xyzr, const uint32_t* cell_index, const double* cell_sas, uint32_t M,
                         const SolventBufs& t, uint32_t K, double probe, cudaStream_t s) {
    if (!M) return;
    k_solvent_mask<<<grid_blocks(M, kWarps, 148 * 32), kWarps * 32, 0, s>>>(
        xyzr, cell_index, cell_sas, M, t.poff, t.partners, t.dirs, K, probe, t.mask, t.count);
    count_launch();
}

void launch_solvent_write(const double* xyzr, const uint32_t* cell_index, uint32_t M, const SolventBufs& t,
                          uint32_t K, double probe, double volume_probe, uint32_t n, double* combined,
                          cudaStream_t s) {
    if (n) {
        k_combined_atoms<<<gb(n), kBlock, 0, s>>>(xyzr, n, probe, volume_probe, combined); count_launch();
    }
    if (M) {
        k_solvent_write<<<grid_blocks(M, kWarps, 148 * 32), kWarps * 32, 0, s>>>(
            xyzr, cell_index, M, t.dirs, K, probe, volume_probe, t.mask, t.soff, n, t.sol_xyz, t.sol_parent, combined);
        count_launch();
    }
}

void launch_solvent_weights(const uint32_t* cell_index, const double* cell_vol, uint32_t M, uint32_t n, uint32_t S,
                            double* weight, cudaStream_t s) {
    cudaMemsetAsync(weight, 0, sizeof(double) * (S ? S : 1), s);
    if (M) {
        k_solvent_weights<<<gb(M), kBlock, 0, s>>>(cell_index, cell_vol, M, n, S, weight); count_launch();
    }
}

}  // namespace vt
