// vt_engine.cu -- host orchestration of the tessellation pipeline and the C ABI.
//
// One engine = one device, one stream, one grow-only workspace.  A call runs:
//   prepare (R = r + probe, bbox)  -> [read bbox]  -> periodic images -> cell grid
//   -> neighbour count -> scans -> [read E, P] -> neighbour fill + pair list
//   -> contact kernel (FP64 or FP32) -> collect unsure/overflow -> FP64 recompute
//   -> serial fallback -> cells -> dedup -> compaction -> totals -> [read counts]
// Three small device->host reads size the next stage's buffers; everything else stays
// on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/voronota_b200.h"
#include "vt_host.cuh"
#include "vt_pipeline.cuh"
#include "vt_batch.cuh"
#include "vt_solvent.cuh"

using namespace vt;

namespace {

thread_local std::string g_last_error;

}  // namespace

namespace vt {
void set_last_error(const std::string& msg) { g_last_error = msg; }

namespace {
std::mutex g_pool_mu;
std::vector<std::pair<size_t, void*>> g_pool;  // free page-locked blocks (capacity, pointer)
size_t g_pool_bytes = 0;
constexpr size_t kPoolMaxBytes = size_t(4) << 30;  // cached page-locked memory kept for reuse
}  // namespace

void* host_block_acquire(size_t bytes, size_t* cap, bool* pinned) {
    size_t c = 64 * 1024;
    while (c < bytes) c <<= 1;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        for (size_t k = 0; k < g_pool.size(); ++k)
            if (g_pool[k].first == c) {
                void* p = g_pool[k].second;
                g_pool[k] = g_pool.back();
                g_pool.pop_back();
                g_pool_bytes -= c;
                *cap = c;
                *pinned = true;
                return p;
            }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, c) == cudaSuccess) {
        *cap = c;
        *pinned = true;
        return p;
    }
    cudaGetLastError();
    p = std::malloc(c);
    *cap = c;
    *pinned = false;
    return p;
}

void host_block_release(void* p, size_t cap, bool pinned) {
    if (!pinned) {
        std::free(p);
        return;
    }
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (g_pool_bytes + cap <= kPoolMaxBytes) {
            g_pool.emplace_back(cap, p);
            g_pool_bytes += cap;
            return;
        }
    }
    cudaFreeHost(p);
}
}  // namespace vt

// Host copy of a batched result: all structures' contacts and cells concatenated (ids
// local to their structure) and the per-structure ranges and totals.
struct vt_batch_result {
    uint64_t S = 0;
    std::unique_ptr<vt_result> all;
    std::vector<uint64_t> contact_off, cell_off;  // S + 1
    std::vector<double> totals;                   // 3 per structure
};

// Host copy of compute_solvent_spheres' output.
struct vt_solvent_result {
    std::vector<double> xyz, radius, weight;
    std::vector<uint32_t> parent;
};

struct vt_engine {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    // workspace
    DBuf<double> xyzr;
    DBuf<int32_t> groups;
    DBuf<double4> sph, c_pos;
    DBuf<uint32_t> slot_id, c_id, c_slot, cell_count, cell_start, cell_cursor;
    DBuf<uint32_t> nb_cnt, nb_npair, nb_off, pair_off, nb_id, nb_slot;
    DBuf<uint8_t> excluded;
    DBuf<double> nb_val;
    DBuf<int32_t> nb_pair;
    DBuf<float4> nb_rel;
    DBuf<uint32_t> pair_a, pair_e;
    DBuf<uint8_t> p_status, p_central;
    DBuf<double> p_area, p_arc, p_sa_a, p_sa_b, p_pv_a, p_pv_b;
    DBuf<uint32_t> redo_list, serial_list, keep, keep_off, cell_off, flags32, big_list;
    DBuf<double> serial_scratch;
    DBuf<uint8_t> cell_flag, ball_dirty;
    DBuf<uint32_t> cell_redo;
    DBuf<double> cell_sas, cell_vol;
    DBuf<uint32_t> out_a, out_b, out_cell_index;
    DBuf<double> out_area, out_arc, out_cell_sas, out_cell_vol;
    DBuf<uint8_t> out_central;
    DBuf<double> totals, partials;
    DBuf<uint32_t> words;  // [0] err, [1] zero, [2] nslots, [3] redo count, [4] serial count
    DBuf<BBox> bbox_parts, bbox;
    DBuf<uint32_t> img_cnt, img_off, scan_tmp;
    // pinned readback
    uint32_t* h_words = nullptr;  // 8 words
    BBox* h_bbox = nullptr;
    // stage timing
    bool timing = false;
    cudaEvent_t ev0[VT_NUM_STAGES] = {}, ev1[VT_NUM_STAGES] = {};
    bool used[VT_NUM_STAGES] = {};
    double stage_ms[VT_NUM_STAGES] = {};
    void t_begin(int k) {
        if (!timing) return;
        VT_CUDA(cudaEventRecord(ev0[k], stream));
        used[k] = true;
    }
    void t_end(int k) {
        if (timing) VT_CUDA(cudaEventRecord(ev1[k], stream));
    }
    void t_collect() {
        for (int k = 0; k < VT_NUM_STAGES; ++k) {
            stage_ms[k] = 0.0;
            if (timing && used[k]) {
                float ms = 0.f;
                VT_CUDA(cudaEventElapsedTime(&ms, ev0[k], ev1[k]));
                stage_ms[k] = ms;
            }
        }
    }
    // tessellation network (with_cell_vertices) of the last call
    bool network = false;
    bool net_wide_keys = false;  // force the two-word vertex keys of the deduplication
    uint64_t net_nv = 0, net_ne = 0;
    DBuf<uint32_t> net_flags, net_voff, net_vcnt, net_ecnt, net_off_v, net_off_e;
    DBuf<uint4> net_vids, net_eids, net_ov_vids, net_ov_eids;
    DBuf<double> net_vxyz, net_elen, net_ov_vxyz, net_ov_elen;
    DBuf<uint32_t> net_base, net_ov_list, net_fp64_list;
    // FP32 contours recorded by the contact kernel for the network's element kernel and
    // the adjoint (network calls, and calls with keep_contours set)
    bool keep_contours = false;
    DBuf<uint32_t> hit_idx;  // the count pass's hits per ball, for the fill pass
    DBuf<float4> rec_pts;
    DBuf<uint2> rec_ids;
    DBuf<uint32_t> rec_off, rec_meta;
    NetSlots net_slots{};
    DBuf<uint32_t> net_bcnt, net_boff, net_bcur, net_bucnt, net_buoff, net_big, net_bidx, net_bsrcd;
    DBuf<unsigned long long> net_k1, net_k2;
    DBuf<uint32_t> out_net_vid, out_net_eid;
    DBuf<double> out_net_vxyz, out_net_elen;

    // one element type (m elements of V pairs): bucket by first id, sort the buckets, keep
    // the first of equal ids, gather
    uint64_t net_unique(uint32_t V, const uint32_t* off, uint32_t m, int vertices) {
        if (m == 0) return 0;
        const uint32_t n = (uint32_t)bufs.n, NB = n + 1;
        net_bcnt.ensure(NB);
        net_boff.ensure(NB + 1);
        net_bcur.ensure(NB);
        net_bucnt.ensure(NB);
        net_buoff.ensure(NB + 1);
        net_big.ensure(NB + 1);
        net_k1.ensure(m);
        const bool wide = vertices && (net_wide_keys || 3 * net_key_bits(n) > 64);
        net_k2.ensure(wide ? m : 1);  // the wide key form only
        net_bidx.ensure(m);
        net_bsrcd.ensure(m);
        NetBuckets t{net_bcnt.p, net_boff.p, net_bcur.p, net_bucnt.p, net_buoff.p, net_big.p,
                     net_k1.p,   net_k2.p,   net_bidx.p, net_bsrcd.p};
        ensure_scan(NB + 1);
        launch_net_dedup(V, off, net_slots, vertices, wide ? 1 : 0, n, t, scan_tmp.p, stream);
        VT_CUDA(cudaMemcpyAsync(h_words + 15, net_buoff.p + NB, 4, cudaMemcpyDeviceToHost, stream));
        sync();
        const uint32_t U = h_words[15];
        if (vertices) {
            out_net_vid.ensure(4 * (size_t)U + 4);
            out_net_vxyz.ensure(3 * (size_t)U + 3);
            launch_net_dedup_gather(n, t, net_slots, 1, out_net_vid.p, out_net_vxyz.p, stream);
        } else {
            out_net_eid.ensure(3 * (size_t)U + 3);
            out_net_elen.ensure((size_t)U + 1);
            launch_net_dedup_gather(n, t, net_slots, 0, out_net_eid.p, out_net_elen.p, stream);
        }
        return U;
    }

    // assemble_tessellation_network over the pairs of the last run (after compaction)
    int build_network(uint32_t P) {
        DevBufs& b = bufs;
        net_nv = net_ne = 0;
        if (P == 0) return VT_OK;
        net_flags.ensure(P + 1);
        net_voff.ensure(P + 2);
        launch_valid_flags(b, P, net_flags.p, stream);
        ensure_scan(P + 1);
        scan_u32(net_flags.p, net_voff.p, P, scan_tmp.p, stream);
        VT_CUDA(cudaMemcpyAsync(h_words + 15, net_voff.p + P, 4, cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 13, b.d_serial_count, 4, cudaMemcpyDeviceToHost, stream));
        sync();
        const uint32_t V = h_words[15];
        if (V == 0) return VT_OK;
        // the pairs whose warp contour overflowed in the contact stage overflow here too
        // (same FP64 contour arithmetic); a margin, and the kernel reports any excess
        const uint32_t ov_cap = h_words[13] + 16;
        const size_t cap = (size_t)V * net_slot_capacity(), ov = (size_t)ov_cap * kSerialCap;
        if (cap + ov >= (size_t)UINT32_MAX) {
            g_last_error = "tessellation network too large for 32-bit element indices";
            return VT_ERR_CAPACITY;
        }
        net_vids.ensure(cap);
        net_eids.ensure(cap);
        net_vxyz.ensure(3 * cap);
        net_elen.ensure(cap);
        net_ov_vids.ensure(ov);
        net_ov_eids.ensure(ov);
        net_ov_vxyz.ensure(3 * ov);
        net_ov_elen.ensure(ov);
        net_vcnt.ensure(V + 1);
        net_ecnt.ensure(V + 1);
        net_base.ensure(V + 1);
        net_ov_list.ensure(ov_cap + 1);  // [ov_cap] is the counter
        VT_CUDA(cudaMemsetAsync(net_ov_list.p + ov_cap, 0, 4, stream));
        NetSlots& sl = net_slots;
        sl = NetSlots{net_vids.p, net_vxyz.p, net_eids.p, net_elen.p, net_ov_vids.p, net_ov_vxyz.p, net_ov_eids.p,
                      net_ov_elen.p, (uint32_t)cap, net_base.p, net_vcnt.p, net_ecnt.p, net_ov_list.p,
                      net_ov_list.p + ov_cap, ov_cap};
        if (b.nb_rel) {  // FP32 mode: FP32 contours with FP64-placed vertices, FP64 for the rest
            net_fp64_list.ensure(V + 1);  // [V] is the counter
            VT_CUDA(cudaMemsetAsync(net_fp64_list.p + V, 0, 4, stream));
            launch_net_elements_f32(b, P, net_voff.p, sl, net_fp64_list.p, net_fp64_list.p + V, stream);
            launch_net_elements(b, P, net_voff.p, sl, net_fp64_list.p, net_fp64_list.p + V, stream);
        } else {
            launch_net_elements(b, P, net_voff.p, sl, nullptr, nullptr, stream);
        }
        launch_net_serial(b, net_voff.p, sl, stream);
        net_off_v.ensure(V + 2);
        net_off_e.ensure(V + 2);
        ensure_scan(V + 1);
        scan_u32(net_vcnt.p, net_off_v.p, V, scan_tmp.p, stream);
        scan_u32(net_ecnt.p, net_off_e.p, V, scan_tmp.p, stream);
        VT_CUDA(cudaMemcpyAsync(h_words + 13, net_off_v.p + V, 4, cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 14, net_off_e.p + V, 4, cudaMemcpyDeviceToHost, stream));
        sync();
        const uint32_t Mv = h_words[13], Me = h_words[14];
        net_nv = net_unique(V, net_off_v.p, Mv, 1);
        net_ne = net_unique(V, net_off_e.p, Me, 0);
        return VT_OK;
    }

    // compute_solvent_spheres (solvent_spheres.rs:131-345): stage-1 tessellation, the kept
    // sample points (vt_solvent.cu), stage-2 tessellation of atoms + spheres, weights
    DBuf<uint8_t> sv_exposed;
    DBuf<uint32_t> sv_deg, sv_poff, sv_cursor, sv_partners, sv_mask, sv_count, sv_soff, sv_parent;
    DBuf<double> sv_dirs, sv_xyz, sv_weight, sv_combined;
    int sv_depth = -1;
    uint32_t sv_K = 0;
    uint64_t sv_S = 0;

    int solvent(const double* d_xyzr, uint64_t n, double probe, double volume_probe, int depth,
                const double* pbox9, int precision) {
        sv_S = 0;
        int st = run(d_xyzr, n, probe, pbox9, nullptr, 0, precision, 0);
        if (st != VT_OK || n == 0) return st;
        if (depth != sv_depth) {
            const std::vector<double> dirs = icosahedron_directions(depth);
            sv_dirs.ensure(dirs.size());
            VT_CUDA(cudaMemcpy(sv_dirs.p, dirs.data(), dirs.size() * sizeof(double), cudaMemcpyHostToDevice));
            sv_K = (uint32_t)(dirs.size() / 3);
            sv_depth = depth;
        }
        const uint32_t C = (uint32_t)stats.num_contacts, M = (uint32_t)stats.num_cells, nn = (uint32_t)n;
        const uint32_t words = (sv_K + 31) / 32;
        sv_exposed.ensure(n);
        sv_deg.ensure(n + 1);
        sv_poff.ensure(n + 2);
        sv_cursor.ensure(n + 1);
        sv_partners.ensure(2 * (size_t)C + 1);
        sv_mask.ensure((size_t)M * words + 1);
        sv_count.ensure(M + 1);
        sv_soff.ensure(M + 2);
        SolventBufs t{sv_exposed.p, sv_deg.p,  sv_poff.p,  sv_cursor.p, sv_partners.p, sv_dirs.p,
                      sv_mask.p,    sv_count.p, sv_soff.p, nullptr,     nullptr};
        ensure_scan(std::max<size_t>(n, M) + 1);
        launch_solvent_partners(bufs.out_a, bufs.out_b, C, bufs.out_cell_index, bufs.out_cell_sas, M, nn, t,
                                scan_tmp.p, stream);
        launch_solvent_mask(d_xyzr, bufs.out_cell_index, bufs.out_cell_sas, M, t, sv_K, probe, stream);
        scan_u32(sv_count.p, sv_soff.p, M, scan_tmp.p, stream);
        VT_CUDA(cudaMemcpyAsync(h_words + 15, sv_soff.p + M, 4, cudaMemcpyDeviceToHost, stream));
        sync();
        const uint64_t S = M ? h_words[15] : 0;
        if (S == 0) return VT_OK;
        if (n + S >= (uint64_t)0xffffffffu / 27u) {
            g_last_error = "too many solvent spheres for 32-bit ids";
            return VT_ERR_CAPACITY;
        }
        sv_xyz.ensure(3 * S);
        sv_parent.ensure(S);
        sv_combined.ensure(4 * (n + S));
        t.sol_xyz = sv_xyz.p;
        t.sol_parent = sv_parent.p;
        launch_solvent_write(d_xyzr, bufs.out_cell_index, M, t, sv_K, probe, volume_probe, nn, sv_combined.p, stream);
        st = run(sv_combined.p, n + S, 0.0, pbox9, nullptr, 0, precision, 0);
        if (st != VT_OK) return st;
        sv_weight.ensure(S);
        launch_solvent_weights(bufs.out_cell_index, bufs.out_cell_vol, (uint32_t)stats.num_cells, nn, (uint32_t)S,
                               sv_weight.p, stream);
        sv_S = S;
        sync();
        return VT_OK;
    }

    int download_solvent(double probe, vt_solvent_result** out) {
        std::unique_ptr<vt_solvent_result> r(new vt_solvent_result());
        const size_t S = sv_S;
        r->xyz.resize(3 * S);
        r->radius.assign(S, probe);
        r->weight.resize(S);
        r->parent.resize(S);
        if (S) {
            VT_CUDA(cudaMemcpyAsync(r->xyz.data(), sv_xyz.p, 24 * S, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->weight.data(), sv_weight.p, 8 * S, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->parent.data(), sv_parent.p, 4 * S, cudaMemcpyDeviceToHost, stream));
            sync();
        }
        *out = r.release();
        return VT_OK;
    }

    // batched call state
    bool batch = false;
    uint64_t batch_S = 0;
    DBuf<uint32_t> boff, ball_struct, sncell, cell_base, crange, mrange;
    DBuf<BBox> sbbox;
    DBuf<GridDev> sgrid;
    DBuf<double> btotals;
    std::vector<uint32_t> h_crange, h_mrange;
    std::vector<double> h_btot;
    double fp32_band_ulps = 16.0;  // FP32 point error budget E, in float ulps of the pair scale
    uint64_t fp32_min_pairs = 2048;  // FP32 mode: fewer candidate pairs run the FP64 kernel
    // launch configuration, set by the autotuner or by hand
    // launch configuration of the FP32 contact kernel until the autotuner or the caller
    // sets one: what the autotuner picks on protein-like inputs of 20k-200k balls
    int c32_warps = 2;        // warps per block of the FP32 contact kernel
    int c32_chunk = 4;        // > 0: persistent FP32 contact launch, pairs taken in chunks
    double cell_scale = 0.5;  // grid cell edge / the reach 2 max R + 0.25 (0.5 .. 4; below 1: a 5^3 stencil)
    // state of the last call
    vt_stats stats{};
    bool contacts_only = false;
    bool have_result = false;
    DevBufs bufs{};
    // FP32 path: per-contributing-contact error budget (radians) of a cell's solid-angle
    // sums; cells within it of a compute_sas branch threshold are recomputed from FP64
    static constexpr float kCellBand = 4e-6f;

    void init(int dev) {
        device = dev;
        VT_CUDA(cudaSetDevice(dev));
        VT_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
        stream = own;
        VT_CUDA(cudaMallocHost(&h_words, 16 * sizeof(uint32_t)));
        VT_CUDA(cudaMallocHost(&h_bbox, sizeof(BBox)));
        words.ensure(16);
        totals.ensure(4);
        partials.ensure(148 * 3 + 8);
        bbox.ensure(1);
        bbox_parts.ensure(1024);
        set_hex_table();
        VT_CUDA(cudaGetLastError());
        for (int k = 0; k < VT_NUM_STAGES; ++k) {
            VT_CUDA(cudaEventCreate(&ev0[k]));
            VT_CUDA(cudaEventCreate(&ev1[k]));
        }
    }
    ~vt_engine() {
        cudaSetDevice(device);
        if (own) cudaStreamSynchronize(own);
        DBuf<double>* dd[] = {&xyzr, &nb_val, &p_area, &p_arc, &p_sa_a, &p_sa_b, &p_pv_a, &p_pv_b, &serial_scratch,
                              &cell_sas, &cell_vol, &out_area, &out_arc, &out_cell_sas, &out_cell_vol, &totals,
                              &partials};
        for (auto* b : dd) b->release();
        DBuf<uint32_t>* du[] = {&slot_id, &c_id, &c_slot, &cell_count, &cell_start, &cell_cursor, &nb_cnt,
                                &nb_npair, &nb_off, &pair_off, &nb_id, &nb_slot, &pair_a, &pair_e, &redo_list,
                                &serial_list, &keep, &keep_off, &cell_off, &flags32, &out_a, &out_b,
                                &out_cell_index, &words, &img_cnt, &img_off, &scan_tmp};
        for (auto* b : du) b->release();
        groups.release();
        sph.release();
        c_pos.release();
        excluded.release();
        nb_pair.release();
        nb_rel.release();
        p_status.release();
        p_central.release();
        cell_flag.release();
        ball_dirty.release();
        cell_redo.release();
        out_central.release();
        bbox_parts.release();
        bbox.release();
        if (h_words) cudaFreeHost(h_words);
        if (h_bbox) cudaFreeHost(h_bbox);
        for (int k = 0; k < VT_NUM_STAGES; ++k) {
            if (ev0[k]) cudaEventDestroy(ev0[k]);
            if (ev1[k]) cudaEventDestroy(ev1[k]);
        }
        if (own) cudaStreamDestroy(own);
    }

    void sync() {
        ++stats.num_host_syncs;
        VT_CUDA(cudaStreamSynchronize(stream));
    }

    void ensure_scan(size_t n) { scan_tmp.ensure(scan_tmp_words_needed(n) + 8); }

    // batch_off (host, S+1 ball offsets): S independent structures concatenated in d_in,
    // tessellated together (non-periodic); outputs are per-structure ranges with local ids.
    int run(const double* d_in, uint64_t n64, double probe, const double* pbox9, const int32_t* d_groups,
            uint64_t n_groups, int precision, int contacts_only_, const uint64_t* batch_off = nullptr,
            uint64_t S = 0) {
        VT_CUDA(cudaSetDevice(device));
        contacts_only = contacts_only_ != 0;
        have_result = false;
        batch = batch_off != nullptr;
        batch_S = batch ? S : 0;
        stats = vt_stats{};
        stats.num_balls = n64;
        net_nv = net_ne = 0;
        const uint64_t launches0 = launch_count();
        for (int k = 0; k < VT_NUM_STAGES; ++k) {
            used[k] = false;
            stage_ms[k] = 0.0;
        }
        if (n64 == 0) {  // tessellation.rs:131-133, 205-207
            if (batch) {
                h_crange.assign(S + 1, 0);
                h_mrange.assign(S + 1, 0);
                h_btot.assign(3 * S, 0.0);
            }
            have_result = true;
            return VT_OK;
        }
        const uint32_t n = (uint32_t)n64;
        const bool periodic = pbox9 != nullptr;
        const size_t max_slots = periodic ? (size_t)n * 27 : (size_t)n;
        DevBufs& b = bufs;
        b = DevBufs{};
        b.n = n;
        b.periodic = periodic ? 1 : 0;
        if (periodic)
            for (int k = 0; k < 9; ++k) b.pbox[k] = pbox9[k];
        b.groups = d_groups;
        b.n_groups = d_groups ? n_groups : 0;
        b.fp32_band = (float)(fp32_band_ulps * 1.1920928955078125e-07);
        b.c32_warps = c32_warps;
        b.c32_chunk = c32_chunk;
        b.c32_queue = words.p + 14;

        sph.ensure(max_slots);
        slot_id.ensure(max_slots);
        b.sph = sph.p;
        b.slot_id = slot_id.p;
        b.err = words.p;
        b.d_nslots = words.p + 2;
        b.d_redo_count = words.p + 3;
        b.d_serial_count = words.p + 4;
        VT_CUDA(cudaMemsetAsync(words.p, 0, 16 * sizeof(uint32_t), stream));

        // 1. prepare + bounding box
        t_begin(10);
        int nblk = (int)std::min<size_t>((n + 255) / 256, 1024);
        t_begin(0);
        launch_prepare(b, d_in, probe, bbox_parts.p, nblk, stream);
        launch_bbox_final(bbox_parts.p, nblk, bbox.p, stream);
        t_end(0);
        VT_CUDA(cudaMemcpyAsync(h_bbox, bbox.p, sizeof(BBox), cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 7, words.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        sync();
        if (h_words[7] & kErrInvalid) {  // k_prepare's input check
            stats.device_error_bits = h_words[7];
            g_last_error = "non-finite input or negative radius";
            return VT_ERR_INVALID;
        }
        const BBox bb = *h_bbox;
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(bb.mn[k]) || !std::isfinite(bb.mx[k])) {
                g_last_error = "non-finite coordinates";
                return VT_ERR_INVALID;
            }
        // cell edge >= 2 max R + margin: intersecting balls lie in adjacent cells
        // (the reference uses max(2R + 0.25), spheres_searcher.rs:74-77)
        double reach = std::max(2.0 * bb.max_r + 0.25, 1.0);

        // 2. periodic images within reach of the structure
        if (periodic) {
            img_cnt.ensure(n);
            img_off.ensure(n + 1);
            ensure_scan(n);
            t_begin(1);
            launch_images(b, reach, bbox.p, img_cnt.p, img_off.p, scan_tmp.p, scan_tmp.cap, stream);
            t_end(1);
        } else {
            VT_CUDA(cudaMemcpyAsync(b.d_nslots, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        }

        // 3. grid over the extended box (cells of edge >= reach); batched: one grid per
        // structure, concatenated
        uint32_t ncell = 0;
        if (batch) {
            std::vector<uint32_t> h_off(S + 1);
            for (uint64_t k = 0; k <= S; ++k) h_off[k] = (uint32_t)batch_off[k];
            boff.ensure(S + 1);
            VT_CUDA(cudaMemcpyAsync(boff.p, h_off.data(), 4 * (S + 1), cudaMemcpyHostToDevice, stream));
            ball_struct.ensure(n);
            sbbox.ensure(S);
            sgrid.ensure(S);
            sncell.ensure(S + 1);
            cell_base.ensure(S + 1);
            launch_batch_grid_setup(boff.p, (uint32_t)S, n, sph.p, ball_struct.p, sbbox.p, sgrid.p, sncell.p, cell_scale,
                                    stream);
            ensure_scan(S + 1);
            scan_u32(sncell.p, cell_base.p, S, scan_tmp.p, stream);
            VT_CUDA(cudaMemcpyAsync(h_words + 12, cell_base.p + S, 4, cudaMemcpyDeviceToHost, stream));
            sync();  // h_off is pageable
            ncell = h_words[12];
            b.ball_struct = ball_struct.p;
            b.grids = sgrid.p;
            b.cell_base = cell_base.p;
        } else {
            b.grid = plan_grid(bb, reach, max_slots, &ncell, cell_scale);
        }
        cell_count.ensure(ncell + 1);
        cell_start.ensure(ncell + 1);
        cell_cursor.ensure(ncell + 1);
        c_pos.ensure(max_slots);
        c_id.ensure(max_slots);
        c_slot.ensure(max_slots);
        b.cell_count = cell_count.p;
        b.cell_start = cell_start.p;
        b.cell_cursor = cell_cursor.p;
        b.c_pos = c_pos.p;
        b.c_id = c_id.p;
        b.c_slot = c_slot.p;
        ensure_scan(std::max<size_t>(ncell, n) + 1);
        t_begin(2);
        if (batch)
            launch_batch_grid(b, n, ncell, scan_tmp.p, stream);
        else
            launch_grid(b, ncell, (uint32_t)max_slots, scan_tmp.p, scan_tmp.cap, stream);
        t_end(2);

        // 4. neighbour counts
        nb_cnt.ensure(n);
        nb_npair.ensure(n);
        excluded.ensure(n);
        nb_off.ensure(n + 1);
        pair_off.ensure(n + 1);
        b.nb_cnt = nb_cnt.p;
        b.nb_npair = nb_npair.p;
        b.excluded = excluded.p;
        b.nb_off = nb_off.p;
        b.pair_off = pair_off.p;
        big_list.ensure(n + 1);
        b.big_list = big_list.p;
        hit_idx.ensure((size_t)n * kHitCap);
        b.hit_idx = hit_idx.p;
        b.d_big_count = words.p + 6;
        t_begin(3);
        launch_search_count(b, stream);
        scan_u32(nb_cnt.p, nb_off.p, n, scan_tmp.p, stream);
        scan_u32(nb_npair.p, pair_off.p, n, scan_tmp.p, stream);
        t_end(3);
        VT_CUDA(cudaMemcpyAsync(h_words + 0, nb_off.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 1, pair_off.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 2, words.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 3, b.d_nslots, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 10, b.d_big_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        sync();
        const uint32_t E = h_words[0], P = h_words[1], n_big = h_words[10];
        stats.num_entries = E;
        stats.num_pairs = P;
        stats.num_slots = h_words[3];
        if (h_words[2] & kErrNeighborCap) {
            g_last_error = "a ball has more than 256 neighbour candidates";
            stats.device_error_bits = h_words[2];
            return VT_ERR_CAPACITY;
        }

        // 5. neighbour lists + pair list
        const bool fp32 = precision == VT_FP32_FIXUP && P >= fp32_min_pairs;
        stats.fp32_kernel = fp32 ? 1 : 0;
        nb_id.ensure(E);
        nb_slot.ensure(E);
        nb_val.ensure(E);
        nb_pair.ensure(E);
        if (fp32) nb_rel.ensure(E);
        pair_a.ensure(P);
        pair_e.ensure(P);
        b.nb_id = nb_id.p;
        b.nb_slot = nb_slot.p;
        b.nb_val = nb_val.p;
        b.nb_pair = nb_pair.p;
        b.nb_rel = fp32 ? nb_rel.p : nullptr;
        b.pair_a = pair_a.p;
        b.pair_e = pair_e.p;
        t_begin(4);
        launch_search_fill(b, fp32 ? 1 : 0, n_big, stream);
        t_end(4);

        // 6. contacts
        p_status.ensure(P);
        p_central.ensure(P);
        p_area.ensure(P);
        p_arc.ensure(P);
        p_sa_a.ensure(P);
        p_sa_b.ensure(P);
        p_pv_a.ensure(P);
        p_pv_b.ensure(P);
        redo_list.ensure(2 * (size_t)P);  // the cell fixup may list a pair from both ends
        serial_list.ensure(P);
        const uint32_t serial_slots = 2048;
        serial_scratch.ensure((size_t)serial_slots * kSerialCap * 6);
        b.p_status = p_status.p;
        b.p_central = p_central.p;
        b.p_area = p_area.p;
        b.p_arc = p_arc.p;
        b.p_sa_a = p_sa_a.p;
        b.p_sa_b = p_sa_b.p;
        b.p_pv_a = p_pv_a.p;
        b.p_pv_b = p_pv_b.p;
        b.redo_list = redo_list.p;
        b.serial_list = serial_list.p;
        b.serial_scratch = serial_scratch.p;
        b.serial_slots = serial_slots;
        const int full = contacts_only ? 0 : 1;
        if (fp32 && (network || keep_contours) && !contacts_only && !batch && P > 0) {
            // a pool of 3 points per candidate pair (valid pairs, about half, hold about 6);
            // pairs past it are recomputed by the element kernel
            const size_t cap = std::min<size_t>(3 * (size_t)P + 64, (size_t)0xfffffff0u);
            rec_pts.ensure(cap);
            rec_ids.ensure(cap);
            rec_off.ensure(P);
            rec_meta.ensure(P);
            b.rec_pts = rec_pts.p;
            b.rec_ids = rec_ids.p;
            b.rec_off = rec_off.p;
            b.rec_meta = rec_meta.p;
            b.rec_count = words.p + 7;
            b.rec_cap = (uint32_t)cap;
            VT_CUDA(cudaMemsetAsync(b.rec_count, 0, sizeof(uint32_t), stream));
        }
        if (P > 0) {
            if (fp32) {
                t_begin(5);
                launch_contact_f32(b, P, full, stream);
                t_end(5);
                t_begin(6);
                if (batch) launch_batch_small_unsure(b, boff.p, P, fp32_min_pairs, stream);
                launch_collect_redo(b, P, stream);
                launch_contact_f64(b, P, full, 1, stream);
                t_end(6);
            } else {
                t_begin(5);
                launch_contact_f64(b, P, full, 0, stream);
                t_end(5);
            }
            VT_CUDA(cudaMemcpyAsync(h_words + 4, b.d_redo_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            t_begin(7);
            launch_collect_redo(b, P, stream);
            launch_contact_serial(b, P, full, stream);
            t_end(7);
        }

        // 7. cells, dedup, compaction, totals
        cell_flag.ensure(n);
        cell_sas.ensure(n);
        cell_vol.ensure(n);
        keep.ensure(P + 1);
        keep_off.ensure(P + 1);
        cell_off.ensure(n + 1);
        flags32.ensure(n);
        out_a.ensure(P);
        out_b.ensure(P);
        out_area.ensure(P);
        out_arc.ensure(P);
        out_central.ensure(P);
        out_cell_index.ensure(n);
        out_cell_sas.ensure(n);
        out_cell_vol.ensure(n);
        b.cell_flag = cell_flag.p;
        b.cell_sas = cell_sas.p;
        b.cell_vol = cell_vol.p;
        b.keep = keep.p;
        b.keep_off = keep_off.p;
        b.cell_off = cell_off.p;
        b.params_u = flags32.p;
        b.out_a = out_a.p;
        b.out_b = out_b.p;
        b.out_area = out_area.p;
        b.out_arc = out_arc.p;
        b.out_central = out_central.p;
        b.out_cell_index = out_cell_index.p;
        b.out_cell_sas = out_cell_sas.p;
        b.out_cell_vol = out_cell_vol.p;
        b.totals = totals.p;
        b.partials = partials.p;
        b.zero_word = words.p + 1;
        cell_redo.ensure(n);
        ball_dirty.ensure(n);
        b.cell_redo_list = cell_redo.p;
        b.d_cell_redo_count = words.p + 5;
        b.ball_dirty = ball_dirty.p;
        ensure_scan(std::max<size_t>(P, n) + 1);
        if (!contacts_only) {
            t_begin(8);
            if (fp32 && P > 0) {
                // cells whose compute_sas branch is uncertain on FP32 inputs: recompute all
                // their pairs in FP64, then the cells of those balls and their neighbours
                VT_CUDA(cudaMemsetAsync(ball_dirty.p, 0, n, stream));
                launch_cells(b, kCellBand, 0, stream);
                VT_CUDA(cudaMemsetAsync(b.d_redo_count, 0, sizeof(uint32_t), stream));
                launch_mark_ball_pairs(b, stream);
                launch_contact_f64(b, P, full, 1, stream);
                launch_cells(b, 0.f, 1, stream);
                VT_CUDA(cudaMemcpyAsync(h_words + 9, b.d_cell_redo_count, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                        stream));
            } else {
                launch_cells(b, 0.f, 0, stream);
            }
            t_end(8);
        }
        t_begin(9);
        launch_dedup(b, P, contacts_only ? 1 : 0, stream);
        launch_compact(b, P, contacts_only ? 1 : 0, scan_tmp.p, scan_tmp.cap, stream);
        launch_totals(b, P, contacts_only ? 1 : 0, stream);
        if (batch) {
            crange.ensure(S + 1);
            mrange.ensure(S + 1);
            btotals.ensure(3 * S + 1);
            launch_batch_outputs(b, boff.p, (uint32_t)S, P, contacts_only ? 1 : 0, crange.p, mrange.p, btotals.p,
                                 stream);
            h_crange.resize(S + 1);
            h_mrange.resize(S + 1);
            h_btot.resize(3 * S);
        }
        t_end(9);
        t_end(10);

        net_nv = net_ne = 0;
        if (network && !contacts_only && !batch) {
            int nst = build_network(P);
            if (nst != VT_OK) return nst;
        }
        VT_CUDA(cudaMemcpyAsync(h_words + 5, keep_off.p + P, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        if (!contacts_only)
            VT_CUDA(cudaMemcpyAsync(h_words + 6, cell_off.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 7, words.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 8, b.d_serial_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        double h_tot[3];
        VT_CUDA(cudaMemcpyAsync(h_tot, totals.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        if (batch) {
            VT_CUDA(cudaMemcpyAsync(h_crange.data(), crange.p, 4 * (S + 1), cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(h_mrange.data(), mrange.p, 4 * (S + 1), cudaMemcpyDeviceToHost, stream));
            if (S) VT_CUDA(cudaMemcpyAsync(h_btot.data(), btotals.p, 8 * 3 * S, cudaMemcpyDeviceToHost, stream));
        }
        sync();
        VT_CUDA(cudaGetLastError());
        t_collect();
        stats.num_kernel_launches = launch_count() - launches0;
        stats.num_contacts = P > 0 ? h_words[5] : 0;
        stats.num_cells = contacts_only ? 0 : h_words[6];
        stats.num_fp64_redo = (P > 0 && fp32) ? h_words[4] : 0;
        stats.num_serial = P > 0 ? h_words[8] : 0;
        stats.num_cell_redo = (fp32 && P > 0 && !contacts_only) ? h_words[9] : 0;
        stats.device_error_bits = h_words[7];
        stats.total_sas_area = contacts_only ? 0.0 : h_tot[0];
        stats.total_volume = contacts_only ? 0.0 : h_tot[1];
        stats.total_contact_area = h_tot[2];
        if (h_words[7] & (kErrOverflow | kErrNeighborCap | kErrNetwork)) {
            g_last_error = "contour or neighbour capacity exceeded";
            return VT_ERR_CAPACITY;
        }
        if (h_words[7] & kErrInvalid) {
            g_last_error = "non-finite input or negative radius";
            return VT_ERR_INVALID;
        }
        have_result = true;
        return VT_OK;
    }

    int download(vt_result** out) {
        if (!have_result) {
            g_last_error = "no result";
            return VT_ERR_INVALID;
        }
        VT_CUDA(cudaSetDevice(device));
        std::unique_ptr<vt_result> r(new vt_result());
        r->num_balls = stats.num_balls;
        const size_t C = stats.num_contacts, M = stats.num_cells;
        r->a.resize(C);
        r->b.resize(C);
        r->area.resize(C);
        r->arc.resize(C);
        r->central.resize(C);
        r->cell_index.resize(M);
        r->cell_sas.resize(M);
        r->cell_vol.resize(M);
        if (C) {
            VT_CUDA(cudaMemcpyAsync(r->a.data(), out_a.p, C * 4, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->b.data(), out_b.p, C * 4, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->area.data(), out_area.p, C * 8, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->arc.data(), out_arc.p, C * 8, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->central.data(), out_central.p, C, cudaMemcpyDeviceToHost, stream));
        }
        if (M) {
            VT_CUDA(cudaMemcpyAsync(r->cell_index.data(), out_cell_index.p, M * 4, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->cell_sas.data(), out_cell_sas.p, M * 8, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->cell_vol.data(), out_cell_vol.p, M * 8, cudaMemcpyDeviceToHost, stream));
        }
        if (network && !contacts_only && !batch) {
            r->has_network = true;
            const size_t V = net_nv, E = net_ne;
            r->net_vid.resize(4 * V);
            r->net_vxyz.resize(3 * V);
            r->net_eid.resize(3 * E);
            r->net_elen.resize(E);
            if (V) {
                VT_CUDA(cudaMemcpyAsync(r->net_vid.data(), out_net_vid.p, 16 * V, cudaMemcpyDeviceToHost, stream));
                VT_CUDA(cudaMemcpyAsync(r->net_vxyz.data(), out_net_vxyz.p, 24 * V, cudaMemcpyDeviceToHost, stream));
            }
            if (E) {
                VT_CUDA(cudaMemcpyAsync(r->net_eid.data(), out_net_eid.p, 12 * E, cudaMemcpyDeviceToHost, stream));
                VT_CUDA(cudaMemcpyAsync(r->net_elen.data(), out_net_elen.p, 8 * E, cudaMemcpyDeviceToHost, stream));
            }
        }
        sync();
        r->totals[0] = stats.total_sas_area;
        r->totals[1] = stats.total_volume;
        r->totals[2] = stats.total_contact_area;
        *out = r.release();
        return VT_OK;
    }

    // Autotuner: times the candidate launch configurations on this input (CUDA events per
    // stage) and keeps the fastest -- warps per block of the FP32 contact kernel by its
    // stage time, then the grid cell scale by the grid + neighbour-search stage times.
    int autotune(const double* d_in, uint64_t n, double probe, const double* pbox9, int precision,
                 const uint64_t* batch_off, uint64_t S) {
        const bool old_timing = timing;
        timing = true;
        auto stage_sum = [&](std::initializer_list<int> ks, double* out) -> int {
            double best = 1e300;
            for (int rep = 0; rep < 2; ++rep) {
                int st = run(d_in, n, probe, pbox9, nullptr, 0, precision, 0, batch_off, S);
                if (st != VT_OK) return st;
                double t = 0.0;
                for (int k : ks) t += stage_ms[k];
                if (rep > 0) best = std::min(best, t);  // the first run warms up
            }
            *out = best;
            return VT_OK;
        };
        int st = VT_OK;
        if (precision == VT_FP32_FIXUP) {
            // warps per block with the grid-stride launch, then the persistent launch's
            // chunk size at the best width
            int best_w = c32_warps, best_c = 0;
            double best_t = 1e300;
            for (int wv : {2, 4, 8}) {
                c32_warps = wv;
                c32_chunk = 0;
                double t = 0.0;
                st = stage_sum({5}, &t);
                if (st != VT_OK) break;
                if (t < best_t) {
                    best_t = t;
                    best_w = wv;
                }
            }
            c32_warps = best_w;
            for (int ch : {4, 16}) {
                if (st != VT_OK) break;
                c32_chunk = ch;
                double t = 0.0;
                st = stage_sum({5}, &t);
                if (st != VT_OK) break;
                if (t < best_t) {
                    best_t = t;
                    best_c = ch;
                }
            }
            c32_chunk = best_c;
        }
        if (st == VT_OK) {
            double best_s = cell_scale, best_t = 1e300;
            for (double sc : {0.5, 0.75, 1.0, 1.25}) {
                cell_scale = sc;
                double t = 0.0;
                st = stage_sum({2, 3, 4}, &t);
                if (st != VT_OK) break;
                if (t < best_t) {
                    best_t = t;
                    best_s = sc;
                }
            }
            cell_scale = best_s;
        }
        timing = old_timing;
        return st;
    }

    // adjoint of the last full tessellation (device arrays)
    DBuf<double> w_eff, v_eff, grad_w, grad_v, grad_u, grad_out;
    int grad_device(const double* d_w, const double* d_v, const double* d_u, double* d_grad) {
        if (!have_result || contacts_only || batch) {
            g_last_error = "the gradient needs the result of a full single-structure tessellation";
            return VT_ERR_INVALID;
        }
        VT_CUDA(cudaSetDevice(device));
        const uint32_t n = (uint32_t)stats.num_balls;
        if (n == 0) return VT_OK;
        w_eff.ensure(n);
        v_eff.ensure(n);
        VT_CUDA(cudaMemsetAsync(words.p, 0, sizeof(uint32_t), stream));
        launch_adjoint(bufs, (uint32_t)stats.num_pairs, d_w, d_v, d_u, w_eff.p, v_eff.p, d_grad, stream);
        VT_CUDA(cudaMemcpyAsync(h_words + 13, words.p, 4, cudaMemcpyDeviceToHost, stream));
        sync();
        VT_CUDA(cudaGetLastError());
        if (h_words[13] & 32u) {
            g_last_error = "a contact whose contour has more than 256 points is not differentiated";
            return VT_ERR_CAPACITY;
        }
        return VT_OK;
    }

    int download_batch(vt_batch_result** out) {
        if (!have_result || !batch) {
            g_last_error = "no batched result";
            return VT_ERR_INVALID;
        }
        vt_result* all = nullptr;
        int st = download(&all);
        if (st != VT_OK) return st;
        std::unique_ptr<vt_batch_result> r(new vt_batch_result());
        r->all.reset(all);
        r->S = batch_S;
        r->contact_off.assign(h_crange.begin(), h_crange.end());
        r->cell_off.assign(h_mrange.begin(), h_mrange.end());
        r->totals = h_btot;
        *out = r.release();
        return VT_OK;
    }
};


namespace {

int validate_host(const double* xyzr, uint64_t n, double probe, const double* pbox9, const int32_t* groups,
                  uint64_t n_groups) {
    if (n > 0 && !xyzr) {
        g_last_error = "null balls pointer";
        return VT_ERR_INVALID;
    }
    if (n_groups > 0 && !groups) {
        g_last_error = "null groups pointer";
        return VT_ERR_INVALID;
    }
    if (n >= (uint64_t)0xffffffffu / 27u) {
        g_last_error = "too many balls for 32-bit ids";
        return VT_ERR_INVALID;
    }
    if (!std::isfinite(probe)) {
        g_last_error = "non-finite probe";
        return VT_ERR_INVALID;
    }
    if (pbox9)
        for (int k = 0; k < 9; ++k)
            if (!std::isfinite(pbox9[k])) {
                g_last_error = "non-finite periodic box";
                return VT_ERR_INVALID;
            }
    return VT_OK;
}

// The balls themselves are checked on the device (k_prepare: a non-finite value or a
// negative radius ends the call with VT_ERR_INVALID before any other work); a host
// caller's error then names the first bad ball, found here.
void name_invalid_ball(const double* xyzr, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) {
        const double* v = xyzr + 4 * i;
        if (!std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2]) || !std::isfinite(v[3]) ||
            v[3] < 0.0) {
            g_last_error = "ball " + std::to_string(i) + ": non-finite value or negative radius";
            return;
        }
    }
}

std::mutex g_engines_mu;
std::vector<std::unique_ptr<vt_engine>> g_engines;
std::vector<std::unique_ptr<std::mutex>> g_engine_mu;

int validate_batch_offsets(const uint64_t* off, uint64_t S) {
    if (S == 0 || S >= 0xffffffffu) {
        g_last_error = "number of structures must be in [1, 2^32)";
        return VT_ERR_INVALID;
    }
    if (off[0] != 0) {
        g_last_error = "offsets[0] must be 0";
        return VT_ERR_INVALID;
    }
    for (uint64_t s = 0; s < S; ++s)
        if (off[s + 1] < off[s]) {
            g_last_error = "offsets must be non-decreasing";
            return VT_ERR_INVALID;
        }
    return VT_OK;
}

int host_compute(vt_engine* e, const double* xyzr, uint64_t n, double probe, const double* pbox9,
                 const int32_t* groups, uint64_t n_groups, int precision, int contacts_only,
                 const uint64_t* batch_off = nullptr, uint64_t S = 0) {
    int st = validate_host(xyzr, n, probe, pbox9, groups, n_groups);
    if (st != VT_OK) return st;
    if (precision != VT_FP64 && precision != VT_FP32_FIXUP) {
        g_last_error = "unknown precision";
        return VT_ERR_INVALID;
    }
    VT_CUDA(cudaSetDevice(e->device));
    const double* d_in = nullptr;
    const int32_t* d_g = nullptr;
    if (n) {
        e->xyzr.ensure(4 * n);
        VT_CUDA(cudaMemcpyAsync(e->xyzr.p, xyzr, 4 * n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        d_in = e->xyzr.p;
    }
    if (groups && n_groups) {
        e->groups.ensure(n_groups);
        VT_CUDA(cudaMemcpyAsync(e->groups.p, groups, n_groups * sizeof(int32_t), cudaMemcpyHostToDevice,
                                e->stream));
        d_g = e->groups.p;
    }
    st = e->run(d_in, n, probe, pbox9, d_g, n_groups, precision, contacts_only, batch_off, S);
    if (st == VT_ERR_INVALID && (e->stats.device_error_bits & kErrInvalid)) name_invalid_ball(xyzr, n);
    return st;
}

template <typename F>
int with_default_engine(F&& f) {
    return guarded([&]() -> int {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            g_last_error = "no CUDA device";
            return VT_ERR_NO_DEVICE;
        }
        int dev = 0;
        VT_CUDA(cudaGetDevice(&dev));
        vt_engine* e;
        std::mutex* mu;
        {
            std::lock_guard<std::mutex> lk(g_engines_mu);
            if ((int)g_engines.size() < ndev) {
                g_engines.resize(ndev);
                g_engine_mu.resize(ndev);
            }
            if (!g_engines[dev]) {
                std::unique_ptr<vt_engine> ne(new vt_engine());
                ne->init(dev);
                g_engines[dev] = std::move(ne);
                g_engine_mu[dev].reset(new std::mutex());
            }
            e = g_engines[dev].get();
            mu = g_engine_mu[dev].get();
        }
        std::lock_guard<std::mutex> lk(*mu);
        return f(e);
    });
}

int stateless(const double* xyzr, uint64_t n, double probe, const double* pbox9, const int32_t* groups,
              uint64_t n_groups, int precision, int contacts_only, vt_result** out) {
    if (!out) {
        g_last_error = "null result pointer";
        return VT_ERR_INVALID;
    }
    *out = nullptr;
    return with_default_engine([&](vt_engine* e) -> int {
        int st = host_compute(e, xyzr, n, probe, pbox9, groups, n_groups, precision, contacts_only);
        if (st != VT_OK) return st;
        return e->download(out);
    });
}

}  // namespace

extern "C" {

int vt_compute_tessellation(const double* xyzr, uint64_t n, double probe, const double* periodic_box9,
                            const int32_t* groups, uint64_t n_groups, int precision, vt_result** out) {
    return stateless(xyzr, n, probe, periodic_box9, groups, n_groups, precision, 0, out);
}
int vt_compute_contacts_only(const double* xyzr, uint64_t n, double probe, const double* periodic_box9,
                             const int32_t* groups, uint64_t n_groups, int precision, vt_result** out) {
    return stateless(xyzr, n, probe, periodic_box9, groups, n_groups, precision, 1, out);
}

int vt_compute_batch(const double* xyzr, const uint64_t* offsets, uint64_t num_structures, double probe,
                     int precision, vt_batch_result** out) {
    if (!out) return VT_ERR_INVALID;
    *out = nullptr;
    if (!offsets) {
        g_last_error = "null offsets";
        return VT_ERR_INVALID;
    }
    int st = validate_batch_offsets(offsets, num_structures);
    if (st != VT_OK) return st;
    const uint64_t n = offsets[num_structures];
    return with_default_engine([&](vt_engine* e) -> int {
        int s2 = host_compute(e, xyzr, n, probe, nullptr, nullptr, 0, precision, 0, offsets, num_structures);
        if (s2 != VT_OK) return s2;
        return e->download_batch(out);
    });
}
int vt_engine_autotune_device(vt_engine* e, const double* d_xyzr, uint64_t n, double probe,
                              const double* periodic_box9, int precision, const uint64_t* batch_offsets,
                              uint64_t num_structures) {
    if (!e || (n && !d_xyzr)) return VT_ERR_INVALID;
    if (precision != VT_FP64 && precision != VT_FP32_FIXUP) return VT_ERR_INVALID;
    if (batch_offsets) {
        int st = validate_batch_offsets(batch_offsets, num_structures);
        if (st != VT_OK) return st;
        if (periodic_box9 || batch_offsets[num_structures] != n) {
            g_last_error = "batched autotuning: no periodic box, offsets[S] must equal n";
            return VT_ERR_INVALID;
        }
    }
    return guarded([&]() {
        return e->autotune(d_xyzr, n, probe, periodic_box9, precision, batch_offsets,
                           batch_offsets ? num_structures : 0);
    });
}
int vt_engine_get_tuning(const vt_engine* e, int* warps, double* cell_scale, int* chunk) {
    if (!e) return VT_ERR_INVALID;
    if (warps) *warps = e->c32_warps;
    if (cell_scale) *cell_scale = e->cell_scale;
    if (chunk) *chunk = e->c32_chunk;
    return VT_OK;
}
int vt_engine_set_tuning(vt_engine* e, int warps, double cell_scale, int chunk) {
    if (!e || (warps != 2 && warps != 4 && warps != 8) || !(cell_scale >= 0.5) || !(cell_scale <= 4.0) ||
        chunk < 0 || chunk > 256)
        return VT_ERR_INVALID;
    e->c32_warps = warps;
    e->cell_scale = cell_scale;
    e->c32_chunk = chunk;
    return VT_OK;
}
int vt_engine_grad_device(vt_engine* e, const double* d_w_sas, const double* d_v_volume, const double* d_u_contact,
                          double* d_grad) {
    if (!e || !d_grad) return VT_ERR_INVALID;
    return guarded([&]() { return e->grad_device(d_w_sas, d_v_volume, d_u_contact, d_grad); });
}
int vt_grad(const double* xyzr, uint64_t n, double probe, const double* periodic_box9, int precision,
            const double* w_sas, const double* v_volume, const double* u_contact, uint64_t num_contacts,
            double* grad_out) {
    if (n && !grad_out) return VT_ERR_INVALID;
    return with_default_engine([&](vt_engine* e) -> int {
        const bool keep = e->keep_contours;
        e->keep_contours = true;  // the adjoint reads the forward's FP32 contours
        int st = host_compute(e, xyzr, n, probe, periodic_box9, nullptr, 0, precision, 0);
        e->keep_contours = keep;
        if (st != VT_OK) return st;
        if (n == 0) return VT_OK;
        if (u_contact && num_contacts != e->stats.num_contacts) {
            g_last_error = "u_contact must have one weight per contact of the tessellation (" +
                           std::to_string(e->stats.num_contacts) + ")";
            return VT_ERR_INVALID;
        }
        e->grad_w.ensure(n);
        e->grad_v.ensure(n);
        e->grad_u.ensure(num_contacts + 1);
        e->grad_out.ensure(4 * n);
        if (w_sas)
            VT_CUDA(cudaMemcpyAsync(e->grad_w.p, w_sas, 8 * n, cudaMemcpyHostToDevice, e->stream));
        if (v_volume)
            VT_CUDA(cudaMemcpyAsync(e->grad_v.p, v_volume, 8 * n, cudaMemcpyHostToDevice, e->stream));
        if (u_contact && num_contacts)
            VT_CUDA(cudaMemcpyAsync(e->grad_u.p, u_contact, 8 * num_contacts, cudaMemcpyHostToDevice, e->stream));
        st = e->grad_device(w_sas ? e->grad_w.p : nullptr, v_volume ? e->grad_v.p : nullptr,
                            u_contact ? e->grad_u.p : nullptr, e->grad_out.p);
        if (st != VT_OK) return st;
        VT_CUDA(cudaMemcpyAsync(grad_out, e->grad_out.p, 32 * n, cudaMemcpyDeviceToHost, e->stream));
        e->sync();
        return VT_OK;
    });
}

uint64_t vt_batch_num_structures(const vt_batch_result* r) { return r ? r->S : 0; }
uint64_t vt_batch_num_contacts(const vt_batch_result* r) { return r ? r->all->a.size() : 0; }
uint64_t vt_batch_num_cells(const vt_batch_result* r) { return r ? r->all->cell_index.size() : 0; }
int vt_batch_ranges(const vt_batch_result* r, uint64_t* contact_off, uint64_t* cell_off) {
    if (!r) return VT_ERR_INVALID;
    if (contact_off) std::memcpy(contact_off, r->contact_off.data(), 8 * (r->S + 1));
    if (cell_off) std::memcpy(cell_off, r->cell_off.data(), 8 * (r->S + 1));
    return VT_OK;
}
int vt_batch_contacts(const vt_batch_result* r, uint32_t* id_a, uint32_t* id_b, double* area, double* arc_length,
                      uint8_t* central) {
    if (!r) return VT_ERR_INVALID;
    return vt_result_contacts(r->all.get(), id_a, id_b, area, arc_length, central);
}
int vt_batch_cells(const vt_batch_result* r, uint32_t* index, double* sas_area, double* volume) {
    if (!r) return VT_ERR_INVALID;
    return vt_result_cells(r->all.get(), index, sas_area, volume);
}
int vt_batch_totals(const vt_batch_result* r, double* totals3) {
    if (!r || (!totals3 && r->S)) return VT_ERR_INVALID;
    if (r->S) std::memcpy(totals3, r->totals.data(), 8 * 3 * r->S);
    return VT_OK;
}
void vt_batch_free(vt_batch_result* r) { delete r; }
int vt_engine_compute_batch_device(vt_engine* e, const double* d_xyzr, const uint64_t* offsets,
                                   uint64_t num_structures, double probe, int precision, int contacts_only) {
    if (!e || !offsets) return VT_ERR_INVALID;
    int st = validate_batch_offsets(offsets, num_structures);
    if (st != VT_OK) return st;
    const uint64_t n = offsets[num_structures];
    if (n && !d_xyzr) return VT_ERR_INVALID;
    if (precision != VT_FP64 && precision != VT_FP32_FIXUP) return VT_ERR_INVALID;
    return guarded([&]() {
        return e->run(d_xyzr, n, probe, nullptr, nullptr, 0, precision, contacts_only, offsets, num_structures);
    });
}
int vt_engine_download_batch(vt_engine* e, vt_batch_result** out) {
    if (!e || !out) return VT_ERR_INVALID;
    *out = nullptr;
    return guarded([&]() { return e->download_batch(out); });
}

int vt_compute_tessellation_network(const double* xyzr, uint64_t n, double probe, const double* periodic_box9,
                                    const int32_t* groups, uint64_t n_groups, int precision, vt_result** out) {
    if (!out) return VT_ERR_INVALID;
    *out = nullptr;
    return with_default_engine([&](vt_engine* e) -> int {
        e->network = true;
        int st = host_compute(e, xyzr, n, probe, periodic_box9, groups, n_groups, precision, 0);
        e->network = false;
        if (st != VT_OK) return st;
        e->network = true;
        st = e->download(out);
        e->network = false;
        return st;
    });
}
int vt_compute_solvent_spheres(const double* xyzr, uint64_t n, double probe, double volume_probe, int depth,
                               const double* periodic_box9, int precision, vt_solvent_result** out) {
    if (!out) return VT_ERR_INVALID;
    *out = nullptr;
    // validate_params / validate_balls (solvent_spheres.rs:164-194), same messages
    char msg[160];
    if (!std::isfinite(probe) || probe < 0.0) {
        std::snprintf(msg, sizeof msg, "invalid probe radius: %g (must be non-negative and finite)", probe);
        g_last_error = msg;
        return VT_ERR_INVALID;
    }
    if (!std::isfinite(volume_probe) || volume_probe < 0.0) {
        std::snprintf(msg, sizeof msg, "invalid volume probe: %g (must be non-negative and finite)", volume_probe);
        g_last_error = msg;
        return VT_ERR_INVALID;
    }
    if (depth < 0) {
        g_last_error = "negative subdivision depth";
        return VT_ERR_INVALID;
    }
    if (n > 0 && !xyzr) {
        g_last_error = "null balls pointer";
        return VT_ERR_INVALID;
    }
    for (uint64_t i = 0; i < n; ++i) {
        const double* b = xyzr + 4 * i;
        const char* why = nullptr;
        if (!std::isfinite(b[0]) || !std::isfinite(b[1]) || !std::isfinite(b[2]))
            why = "coordinates must be finite";
        else if (!std::isfinite(b[3]) || b[3] <= 0.0)
            why = "radius must be positive and finite";
        if (why) {
            std::snprintf(msg, sizeof msg, "invalid ball at index %llu: %s", (unsigned long long)i, why);
            g_last_error = msg;
            return VT_ERR_INVALID;
        }
    }
    if (precision != VT_FP64 && precision != VT_FP32_FIXUP) {
        g_last_error = "unknown precision";
        return VT_ERR_INVALID;
    }
    return with_default_engine([&](vt_engine* e) -> int {
        int st = validate_host(xyzr, n, probe, periodic_box9, nullptr, 0);
        if (st != VT_OK) return st;
        VT_CUDA(cudaSetDevice(e->device));
        const double* d_in = nullptr;
        if (n) {
            e->xyzr.ensure(4 * n);
            VT_CUDA(cudaMemcpyAsync(e->xyzr.p, xyzr, 4 * n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
            d_in = e->xyzr.p;
        }
        st = e->solvent(d_in, n, probe, volume_probe, depth > 4 ? 4 : depth, periodic_box9, precision);
        if (st != VT_OK) return st;
        return e->download_solvent(probe, out);
    });
}
int vt_icosahedron(int depth, double* xyz3) {
    const std::vector<double> d = icosahedron_directions(depth);
    if (xyz3) std::memcpy(xyz3, d.data(), d.size() * sizeof(double));
    return (int)(d.size() / 3);
}
uint64_t vt_solvent_count(const vt_solvent_result* r) { return r ? r->weight.size() : 0; }
int vt_solvent_get(const vt_solvent_result* r, double* xyz3, double* radius, double* weight, uint32_t* parent) {
    if (!r) return VT_ERR_INVALID;
    const size_t S = r->weight.size();
    if (!S) return VT_OK;
    if (xyz3) std::memcpy(xyz3, r->xyz.data(), 24 * S);
    if (radius) std::memcpy(radius, r->radius.data(), 8 * S);
    if (weight) std::memcpy(weight, r->weight.data(), 8 * S);
    if (parent) std::memcpy(parent, r->parent.data(), 4 * S);
    return VT_OK;
}
void vt_solvent_free(vt_solvent_result* r) { delete r; }

int vt_engine_set_fp32_min_pairs(vt_engine* e, uint64_t min_pairs) {
    if (!e) return VT_ERR_INVALID;
    e->fp32_min_pairs = min_pairs;
    return VT_OK;
}
int vt_engine_set_keep_contours(vt_engine* e, int on) {
    if (!e) return VT_ERR_INVALID;
    e->keep_contours = on != 0;
    return VT_OK;
}
int vt_engine_set_network(vt_engine* e, int on) {
    if (!e) return VT_ERR_INVALID;
    e->network = on != 0;
    return VT_OK;
}
int vt_engine_set_network_wide_keys(vt_engine* e, int on) {
    if (!e) return VT_ERR_INVALID;
    e->net_wide_keys = on != 0;
    return VT_OK;
}
uint64_t vt_result_num_vertices(const vt_result* r) { return r ? r->net_vxyz.size() / 3 : 0; }
uint64_t vt_result_num_edges(const vt_result* r) { return r ? r->net_elen.size() : 0; }
int vt_result_vertices(const vt_result* r, uint32_t* ids4, double* xyz3) {
    if (!r || !r->has_network) return VT_ERR_INVALID;
    const size_t V = r->net_vxyz.size() / 3;
    if (V && ids4) std::memcpy(ids4, r->net_vid.data(), 16 * V);
    if (V && xyz3) std::memcpy(xyz3, r->net_vxyz.data(), 24 * V);
    return VT_OK;
}
int vt_result_edges(const vt_result* r, uint32_t* ids3, double* length) {
    if (!r || !r->has_network) return VT_ERR_INVALID;
    const size_t E = r->net_elen.size();
    if (E && ids3) std::memcpy(ids3, r->net_eid.data(), 12 * E);
    if (E && length) std::memcpy(length, r->net_elen.data(), 8 * E);
    return VT_OK;
}

uint64_t vt_result_num_balls(const vt_result* r) { return r ? r->num_balls : 0; }
uint64_t vt_result_num_contacts(const vt_result* r) { return r ? r->a.size() : 0; }
uint64_t vt_result_num_cells(const vt_result* r) { return r ? r->cell_index.size() : 0; }
int vt_result_contacts(const vt_result* r, uint32_t* a, uint32_t* b, double* area, double* arc, uint8_t* central) {
    if (!r) return VT_ERR_INVALID;
    size_t C = r->a.size();
    if (C == 0) return VT_OK;
    if (a) std::memcpy(a, r->a.data(), C * 4);
    if (b) std::memcpy(b, r->b.data(), C * 4);
    if (area) std::memcpy(area, r->area.data(), C * 8);
    if (arc) std::memcpy(arc, r->arc.data(), C * 8);
    if (central) std::memcpy(central, r->central.data(), C);
    return VT_OK;
}
int vt_result_cells(const vt_result* r, uint32_t* index, double* sas, double* vol) {
    if (!r) return VT_ERR_INVALID;
    size_t M = r->cell_index.size();
    if (M == 0) return VT_OK;
    if (index) std::memcpy(index, r->cell_index.data(), M * 4);
    if (sas) std::memcpy(sas, r->cell_sas.data(), M * 8);
    if (vol) std::memcpy(vol, r->cell_vol.data(), M * 8);
    return VT_OK;
}
void vt_result_totals(const vt_result* r, double* s, double* v, double* c) {
    if (!r) return;
    if (s) *s = r->totals[0];
    if (v) *v = r->totals[1];
    if (c) *c = r->totals[2];
}
void vt_result_free(vt_result* r) { delete r; }
int vt_result_view_get(const vt_result* r, vt_result_view* v) {
    if (!r || !v) return VT_ERR_INVALID;
    v->num_contacts = r->a.size();
    v->num_cells = r->cell_index.size();
    v->id_a = r->a.data();
    v->id_b = r->b.data();
    v->area = r->area.data();
    v->arc_length = r->arc.data();
    v->central = r->central.data();
    v->cell_index = r->cell_index.data();
    v->cell_sas_area = r->cell_sas.data();
    v->cell_volume = r->cell_vol.data();
    return VT_OK;
}

int vt_engine_create(int device, vt_engine** out) {
    if (!out) return VT_ERR_INVALID;
    *out = nullptr;
    return guarded([&]() -> int {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            g_last_error = "no CUDA device";
            return VT_ERR_NO_DEVICE;
        }
        if (device < 0 || device >= ndev) {
            g_last_error = "bad device index";
            return VT_ERR_INVALID;
        }
        std::unique_ptr<vt_engine> e(new vt_engine());
        e->init(device);
        *out = e.release();
        return VT_OK;
    });
}
void vt_engine_destroy(vt_engine* e) { delete e; }
int vt_engine_set_stream(vt_engine* e, void* stream) {
    if (!e) return VT_ERR_INVALID;
    e->stream = stream ? (cudaStream_t)stream : e->own;
    return VT_OK;
}
int vt_engine_compute_device(vt_engine* e, const double* d_xyzr, uint64_t n, double probe, const double* pbox9,
                             const int32_t* d_groups, uint64_t n_groups, int precision, int contacts_only) {
    if (!e || (n && !d_xyzr)) return VT_ERR_INVALID;
    if (n >= (uint64_t)0xffffffffu / 27u) {
        g_last_error = "too many balls for 32-bit ids";
        return VT_ERR_INVALID;
    }
    if (precision != VT_FP64 && precision != VT_FP32_FIXUP) return VT_ERR_INVALID;
    return guarded([&]() { return e->run(d_xyzr, n, probe, pbox9, d_groups, n_groups, precision, contacts_only); });
}
int vt_engine_compute_host(vt_engine* e, const double* xyzr, uint64_t n, double probe, const double* pbox9,
                           const int32_t* groups, uint64_t n_groups, int precision, int contacts_only) {
    if (!e) return VT_ERR_INVALID;
    return guarded(
        [&]() { return host_compute(e, xyzr, n, probe, pbox9, groups, n_groups, precision, contacts_only); });
}
int vt_engine_download(vt_engine* e, vt_result** out) {
    if (!e || !out) return VT_ERR_INVALID;
    *out = nullptr;
    return guarded([&]() { return e->download(out); });
}
int vt_engine_stats(const vt_engine* e, vt_stats* out) {
    if (!e || !out) return VT_ERR_INVALID;
    *out = e->stats;
    return VT_OK;
}
int vt_engine_set_fp32_band(vt_engine* e, double ulps) {
    if (!e || !(ulps > 0.0) || !std::isfinite(ulps)) return VT_ERR_INVALID;
    e->fp32_band_ulps = ulps;
    return VT_OK;
}
int vt_engine_set_timing(vt_engine* e, int on) {
    if (!e) return VT_ERR_INVALID;
    e->timing = on != 0;
    return VT_OK;
}
int vt_engine_stage_times(const vt_engine* e, double* ms) {
    if (!e || !ms) return VT_ERR_INVALID;
    for (int k = 0; k < VT_NUM_STAGES; ++k) ms[k] = e->stage_ms[k];
    return VT_OK;
}
int vt_engine_device_outputs(const vt_engine* e, vt_device_outputs* o) {
    if (!e || !o || !e->have_result) return VT_ERR_INVALID;
    o->id_a = e->out_a.p;
    o->id_b = e->out_b.p;
    o->area = e->out_area.p;
    o->arc_length = e->out_arc.p;
    o->central = e->out_central.p;
    o->cell_index = e->out_cell_index.p;
    o->cell_sas_area = e->out_cell_sas.p;
    o->cell_volume = e->out_cell_vol.p;
    o->totals = e->totals.p;
    return VT_OK;
}
const char* vt_status_string(int s) {
    switch (s) {
        case VT_OK: return "ok";
        case VT_ERR_INVALID: return "invalid input";
        case VT_ERR_OOM: return "out of memory";
        case VT_ERR_CUDA: return "CUDA error";
        case VT_ERR_CAPACITY: return "capacity exceeded";
        case VT_ERR_TIMEOUT: return "device wait timed out";
        case VT_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}
const char* vt_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"
