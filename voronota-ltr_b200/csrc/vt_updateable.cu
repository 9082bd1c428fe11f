// vt_updateable.cu -- device-resident UpdateableTessellation (updateable.rs:154-742,
// spheres_container.rs:54-286) and its C ABI.
//
// The state (balls, exclusion statuses, neighbour lists, the per-ball contact table,
// cells) lives on the device.  An update runs, all on the handle's stream:
//   changed filter -> mark changed + old neighbours -> [read counts: no change / full
//   reinit / frontier] -> apply -> spheres, images, grid -> search the frontier ->
//   mark new neighbours of changed balls -> [read] -> search them -> splice the lists ->
//   pairs with both ends involved -> contacts -> periodic dedup -> splice the table ->
//   cells of the affected balls.
// The neighbour grid is rebuilt on every operation from the stored balls, so an
// incremental update equals the reference's documented contract (incremental ==
// recompute of the involved part) without the reference's stale-cell registration
// (spheres_searcher.rs:144-175 removes a moved ball from the cell of its new position).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/voronota_b200.h"
#include "vt_frontier.cuh"
#include "vt_host.cuh"
#include "vt_pipeline.cuh"

using namespace vt;

namespace {

// device word slots of the handle
enum Word : int {
    kWErr = 0,
    kWZero = 1,
    kWSlots = 2,
    kWRedo = 3,
    kWSerial = 4,
    kWCellRedo = 5,
    kWDistinct = 6,  // distinct changed balls
    kWNbrNew = 7,    // neighbours of changed balls newly marked
    kWMore = 8,      // new neighbours of changed balls not yet affected
    kWOne = 9,       // constant 1 (a list length)
    kWId = 10,       // a one-element id list
    kWBig = 11,      // rows of a search longer than the warp sort buffer
    kWUnsure = 12,   // affected balls with an uncertain compute_sas branch (FP32)
    kWMarked = 13,   // balls marked for their FP64 refresh
    kWQueue = 14,    // work counter of the persistent FP32 contact launch
    kWords = 16,
};

struct Lists {
    DBuf<uint32_t> cnt, off, id;
    DBuf<double> val;
    DBuf<float4> rel;
    uint64_t E = 0;
    ListsRef ref(bool with_rel) const { return {cnt.p, off.p, id.p, val.p, with_rel ? rel.p : nullptr}; }
    void swap(Lists& o) {
        cnt.swap(o.cnt);
        off.swap(o.off);
        id.swap(o.id);
        val.swap(o.val);
        rel.swap(o.rel);
        std::swap(E, o.E);
    }
};

struct Table {
    DBuf<uint32_t> off, a, b;
    DBuf<double> area, arc, sa, pv;
    DBuf<uint8_t> flags;
    DBuf<double4> gA, gB;  // SAS adjoint coefficients per entry
    DBuf<double4> vA, vB;  // volume adjoint coefficients per entry
    uint64_t M = 0;
    TableRef ref() const { return {off.p, a.p, b.p, area.p, arc.p, sa.p, pv.p, flags.p, gA.p, gB.p, vA.p, vB.p}; }
    void ensure(size_t n, size_t m) {
        gA.ensure(m);
        gB.ensure(m);
        vA.ensure(m);
        vB.ensure(m);
        off.ensure(n + 1);
        a.ensure(m);
        b.ensure(m);
        area.ensure(m);
        arc.ensure(m);
        sa.ensure(m);
        pv.ensure(m);
        flags.ensure(m);
    }
    void swap(Table& o) {
        off.swap(o.off);
        a.swap(o.a);
        b.swap(o.b);
        area.swap(o.area);
        arc.swap(o.arc);
        sa.swap(o.sa);
        pv.swap(o.pv);
        flags.swap(o.flags);
        gA.swap(o.gA);
        gB.swap(o.gB);
        vA.swap(o.vA);
        vB.swap(o.vB);
        std::swap(M, o.M);
    }
};

// State, updateable.rs:104-124 (container + result + cell summaries + ids).
struct UState {
    uint32_t n = 0;
    double probe = 0.0;
    bool periodic = false;
    double pbox[9] = {};
    DBuf<double> balls;  // 4n: the stored balls (x, y, z, r)
    DBuf<uint8_t> excl;
    Lists lists;
    Table tab;
    DBuf<uint8_t> cell_flag;
    DBuf<double> cell_sas, cell_vol;
    uint64_t num_cells = 0;
    DBuf<uint32_t> changed, affected;
    uint32_t n_changed = 0, n_affected = 0;
    bool affected_dups = false;  // affected keeps duplicated changed ids (no new neighbours)
    bool full = true;
    bool adj_valid = false;  // the table's SAS adjoint coefficients describe this state
    // UpdateableResult::is_empty (updateable.rs:35-37)
    bool empty() const { return n == 0 || num_cells == 0; }
};

void copy_state(UState& d, const UState& s, bool fp32, cudaStream_t st) {
    d.n = s.n;
    d.probe = s.probe;
    d.periodic = s.periodic;
    std::memcpy(d.pbox, s.pbox, sizeof(d.pbox));
    const size_t n = s.n;
    d.balls.copy_from(s.balls, 4 * n, st);
    d.excl.copy_from(s.excl, n, st);
    d.lists.cnt.copy_from(s.lists.cnt, n, st);
    d.lists.off.copy_from(s.lists.off, n + 1, st);
    d.lists.id.copy_from(s.lists.id, s.lists.E, st);
    d.lists.val.copy_from(s.lists.val, s.lists.E, st);
    if (fp32) d.lists.rel.copy_from(s.lists.rel, s.lists.E, st);
    d.lists.E = s.lists.E;
    d.tab.off.copy_from(s.tab.off, n + 1, st);
    d.tab.a.copy_from(s.tab.a, s.tab.M, st);
    d.tab.b.copy_from(s.tab.b, s.tab.M, st);
    d.tab.area.copy_from(s.tab.area, s.tab.M, st);
    d.tab.arc.copy_from(s.tab.arc, s.tab.M, st);
    d.tab.sa.copy_from(s.tab.sa, s.tab.M, st);
    d.tab.pv.copy_from(s.tab.pv, s.tab.M, st);
    d.tab.flags.copy_from(s.tab.flags, s.tab.M, st);
    d.tab.gA.copy_from(s.tab.gA, s.tab.M, st);
    d.tab.gB.copy_from(s.tab.gB, s.tab.M, st);
    d.tab.vA.copy_from(s.tab.vA, s.tab.M, st);
    d.tab.vB.copy_from(s.tab.vB, s.tab.M, st);
    d.tab.M = s.tab.M;
    d.cell_flag.copy_from(s.cell_flag, n, st);
    d.cell_sas.copy_from(s.cell_sas, n, st);
    d.cell_vol.copy_from(s.cell_vol, n, st);
    d.num_cells = s.num_cells;
    d.changed.copy_from(s.changed, s.n_changed, st);
    d.affected.copy_from(s.affected, s.n_affected, st);
    d.n_changed = s.n_changed;
    d.n_affected = s.n_affected;
    d.affected_dups = s.affected_dups;
    d.full = s.full;
    d.adj_valid = s.adj_valid;
}

int check_host_balls(const double* xyzr, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) {
        const double* v = xyzr + 4 * i;
        if (!std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2]) || !std::isfinite(v[3]) ||
            v[3] < 0.0) {
            set_last_error("ball " + std::to_string(i) + ": non-finite value or negative radius");
            return VT_ERR_INVALID;
        }
    }
    return VT_OK;
}

}  // namespace

struct vt_updateable {
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    bool backup_enabled = false;
    bool adjoint = true;  // record arc moments for the SAS adjoint (vt_upd_set_adjoint)
    bool fp32 = false;
    double fp32_band_ulps = 16.0;
    static constexpr float kCellBand = 4e-6f;  // per-contact band of the FP32 cell sums
    std::unique_ptr<UState> cur{new UState()}, bak{new UState()};
    bool has_bak = false;
    bool sph_fresh = false;  // sph/grid built from cur->balls
    vt_stats stats{};

    // workspace
    DBuf<double4> sph, gsph, c_pos, changed_ball;
    DBuf<uint32_t> slot_id, gslot_id, cell_count, cell_start, cell_cursor, c_id, c_slot;
    DBuf<BBox> bbox_parts, bbox;
    DBuf<uint32_t> img_cnt, img_off, scan_tmp, words, big_rows, hit_idx;
    DBuf<uint64_t> ids_in;
    DBuf<double> src_in;
    DBuf<uint32_t> flags, flags_off, mark, row_of, list1, more_list, nflags, noff;
    Lists t1, t2, next_lists;
    DBuf<uint32_t> npair, pair_off, pair_a, pair_e;
    DBuf<int32_t> nb_pair;
    DBuf<uint8_t> p_status, p_central;
    DBuf<double> p_area, p_arc, p_sa_a, p_sa_b, p_pv_a, p_pv_b, serial_scratch;
    DBuf<uint32_t> redo_list, serial_list, keep, keep_off;
    DBuf<uint32_t> nc_a, nc_b, nc_pair;
    DBuf<double> nc_area, nc_arc, nc_sa_a, nc_sa_b, nc_pv_a, nc_pv_b;
    DBuf<uint8_t> nc_central;
    DBuf<double4> nc_gaa, nc_gab, nc_gba, nc_gbb, nc_vaa, nc_vab, nc_vba, nc_vbb;
    DBuf<double> p_arcm;
    Table next_tab;
    DBuf<uint32_t> keep_cnt, new_cnt, tot_cnt, cursor, tmp_k;
    DBuf<uint32_t> cell_redo;
    DBuf<uint8_t> ball_dirty, unsure;
    DBuf<uint32_t> ulist, mark2, nflags2, noff2, aff2;
    DBuf<uint32_t> sum_flags, sum_off, out_a, out_b, out_cell_index;
    DBuf<double> out_area, out_arc, out_cell_sas, out_cell_vol, totals, partials;
    DBuf<uint8_t> out_central;
    uint32_t* h_words = nullptr;
    BBox* h_bbox = nullptr;
    uint32_t ncell = 0;
    GridDev grid{};

    void init_handle(int dev, bool backup, int precision) {
        device = dev;
        backup_enabled = backup;
        fp32 = precision == VT_FP32_FIXUP;
        VT_CUDA(cudaSetDevice(dev));
        VT_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
        stream = own;
        VT_CUDA(cudaMallocHost(&h_words, 32 * sizeof(uint32_t)));
        VT_CUDA(cudaMallocHost(&h_bbox, sizeof(BBox)));
        words.ensure(kWords);
        totals.ensure(4);
        partials.ensure(148 * 3 + 8);
        bbox.ensure(1);
        bbox_parts.ensure(1024);
        set_hex_table();
        VT_CUDA(cudaGetLastError());
    }
    ~vt_updateable() {
        cudaSetDevice(device);
        if (own) cudaStreamSynchronize(own);
        if (h_words) cudaFreeHost(h_words);
        if (h_bbox) cudaFreeHost(h_bbox);
        cur.reset();
        bak.reset();
        for (int k = 0; k < VT_UPD_NUM_STAGES; ++k) {
            if (ev0[k]) cudaEventDestroy(ev0[k]);
            if (ev1[k]) cudaEventDestroy(ev1[k]);
        }
        if (own) cudaStreamDestroy(own);
    }

    void sync() {
        ++stats.num_host_syncs;
        VT_CUDA(cudaStreamSynchronize(stream));
    }

    // stage timing of updates (vt_upd_set_timing)
    bool timing = false;
    cudaEvent_t ev0[VT_UPD_NUM_STAGES] = {}, ev1[VT_UPD_NUM_STAGES] = {};
    bool used[VT_UPD_NUM_STAGES] = {};
    double stage_ms[VT_UPD_NUM_STAGES] = {};
    void t_reset() {
        for (int k = 0; k < VT_UPD_NUM_STAGES; ++k) used[k] = false;
    }
    void t_begin(int k) {
        if (!timing) return;
        if (!ev0[k]) {
            VT_CUDA(cudaEventCreate(&ev0[k]));
            VT_CUDA(cudaEventCreate(&ev1[k]));
        }
        VT_CUDA(cudaEventRecord(ev0[k], stream));
        used[k] = true;
    }
    void t_end(int k) {
        if (timing && used[k]) VT_CUDA(cudaEventRecord(ev1[k], stream));
    }
    // after the operation's final sync
    void t_collect() {
        for (int k = 0; k < VT_UPD_NUM_STAGES; ++k) {
            stage_ms[k] = 0.0;
            if (timing && used[k]) {
                float ms = 0.f;
                VT_CUDA(cudaEventElapsedTime(&ms, ev0[k], ev1[k]));
                stage_ms[k] = ms;
            }
        }
    }
    uint32_t* w(int k) { return words.p + k; }
    void ensure_scan(size_t n) { scan_tmp.ensure(scan_tmp_words_needed(n) + 8); }
    void zero(void* p, size_t bytes) {
        if (bytes) VT_CUDA(cudaMemsetAsync(p, 0, bytes, stream));
    }
    uint32_t read_word(const uint32_t* d) {
        VT_CUDA(cudaMemcpyAsync(h_words, d, 4, cudaMemcpyDeviceToHost, stream));
        sync();
        return h_words[0];
    }

    // ---- spheres, images, grid (from cur->balls) ----
    int build_spheres(UState& S) {
        const uint32_t n = S.n;
        const size_t nslots_max = S.periodic ? (size_t)n * 27 : (size_t)n;
        sph.ensure(nslots_max);
        slot_id.ensure(n);
        DevBufs b{};
        b.n = n;
        b.sph = sph.p;
        b.slot_id = slot_id.p;
        b.err = w(kWErr);
        const int nblk = (int)std::min<size_t>((n + 255) / 256, 1024);
        launch_prepare(b, S.balls.p, S.probe, bbox_parts.p, nblk, stream);
        launch_bbox_final(bbox_parts.p, nblk, bbox.p, stream);
        VT_CUDA(cudaMemcpyAsync(h_bbox, bbox.p, sizeof(BBox), cudaMemcpyDeviceToHost, stream));
        sync();
        const BBox bb = *h_bbox;
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(bb.mn[k]) || !std::isfinite(bb.mx[k]) || !std::isfinite(bb.max_r)) {
                set_last_error("non-finite coordinates");
                return VT_ERR_INVALID;
            }
        const double reach = std::max(2.0 * bb.max_r + 0.25, 1.0);
        DevBufs g = b;  // grid slots: the balls and, periodic, their images within reach
        g.d_nslots = w(kWSlots);
        g.slot_is_id = 1;
        if (S.periodic) {
            launch_images_all(sph.p, n, S.pbox, stream);
            gsph.ensure(nslots_max);
            gslot_id.ensure(nslots_max);
            VT_CUDA(cudaMemcpyAsync(gsph.p, sph.p, n * sizeof(double4), cudaMemcpyDeviceToDevice, stream));
            VT_CUDA(cudaMemcpyAsync(gslot_id.p, slot_id.p, n * 4, cudaMemcpyDeviceToDevice, stream));
            g.sph = gsph.p;
            g.slot_id = gslot_id.p;
            g.periodic = 1;
            for (int k = 0; k < 9; ++k) g.pbox[k] = S.pbox[k];
            img_cnt.ensure(n);
            img_off.ensure(n + 1);
            ensure_scan(n);
            launch_images(g, reach, bbox.p, img_cnt.p, img_off.p, scan_tmp.p, scan_tmp.cap, stream);
        } else {
            VT_CUDA(cudaMemcpyAsync(w(kWSlots), &S.n, 4, cudaMemcpyHostToDevice, stream));
        }
        grid = plan_grid(bb, reach, nslots_max, &ncell, 0.5);  // cells of half the reach, 5^3 stencil
        g.grid = grid;
        cell_count.ensure(ncell);
        cell_start.ensure(ncell + 1);
        cell_cursor.ensure(ncell);
        c_pos.ensure(nslots_max);
        c_id.ensure(nslots_max);
        c_slot.ensure(nslots_max);
        g.cell_count = cell_count.p;
        g.cell_start = cell_start.p;
        g.cell_cursor = cell_cursor.p;
        g.c_pos = c_pos.p;
        g.c_id = c_id.p;
        g.c_slot = c_slot.p;
        ensure_scan(std::max<size_t>(ncell, n) + 1);
        launch_grid(g, ncell, (uint32_t)nslots_max, scan_tmp.p, scan_tmp.cap, stream);
        sph_fresh = true;
        return VT_OK;
    }

    DevBufs base_bufs(UState& S) {
        DevBufs b{};
        b.n = S.n;
        b.periodic = S.periodic ? 1 : 0;
        for (int k = 0; k < 9; ++k) b.pbox[k] = S.pbox[k];
        b.sph = sph.p;
        b.slot_id = slot_id.p;
        b.d_nslots = w(kWSlots);
        b.grid = grid;
        b.cell_count = cell_count.p;
        b.cell_start = cell_start.p;
        b.cell_cursor = cell_cursor.p;
        b.c_pos = c_pos.p;
        b.c_id = c_id.p;
        b.c_slot = c_slot.p;
        b.excluded = S.excl.p;
        b.err = w(kWErr);
        b.zero_word = w(kWZero);
        b.d_redo_count = w(kWRedo);
        b.d_serial_count = w(kWSerial);
        b.d_cell_redo_count = w(kWCellRedo);
        b.fp32_band = (float)(fp32_band_ulps * 1.1920928955078125e-07);
        b.slot_is_id = 1;
        // FP32 contact launch: 2 warps per block, persistent, pairs taken 4 at a time (the
        // form the engine's autotuner picks on the benchmark structures)
        b.c32_warps = 2;
        b.c32_chunk = 4;
        b.c32_queue = w(kWQueue);
        return b;
    }

    // Neighbour lists of the listed balls (list == null: every ball) into L, rows in list
    // order; exclusion statuses of the searched balls into S.excl.
    int search(UState& S, const uint32_t* list, uint32_t m, Lists& L) {
        const uint32_t rows = list ? m : S.n;
        L.cnt.ensure(rows + 1);
        L.off.ensure(rows + 1);
        if (rows == 0) {
            zero(L.off.p, 4);
            L.E = 0;
            return VT_OK;
        }
        DevBufs b = base_bufs(S);
        b.frontier = list;
        b.n_frontier = m;
        b.no_pairs = 1;
        b.nb_cnt = L.cnt.p;
        b.nb_off = L.off.p;
        big_rows.ensure(rows + 1);
        b.big_list = big_rows.p;
        hit_idx.ensure((size_t)rows * kHitCap);
        b.hit_idx = hit_idx.p;
        b.d_big_count = w(kWBig);
        launch_search_count(b, stream);
        ensure_scan(rows + 1);
        scan_u32(L.cnt.p, L.off.p, rows, scan_tmp.p, stream);
        VT_CUDA(cudaMemcpyAsync(h_words, L.off.p + rows, 4, cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 1, w(kWErr), 4, cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 3, w(kWBig), 4, cudaMemcpyDeviceToHost, stream));
        sync();
        if (h_words[1] & kErrNeighborCap) {
            set_last_error("a ball has more than 256 neighbour candidates");
            return VT_ERR_CAPACITY;
        }
        const uint32_t E = h_words[0];
        L.id.ensure(E + 1);
        L.val.ensure(E + 1);
        if (fp32) L.rel.ensure(E + 1);
        b.nb_id = L.id.p;
        b.nb_slot = L.id.p;  // slots are ids: both writes store the same value
        b.nb_val = L.val.p;
        b.nb_rel = fp32 ? L.rel.p : nullptr;
        launch_search_fill(b, fp32 ? 1 : 0, h_words[3], stream);
        L.E = E;
        return VT_OK;
    }

    // Pairs (a, b) of involved balls (mark == null: all), updateable.rs:516-561.
    uint32_t gen_pairs(UState& S, const uint32_t* list, const uint32_t* d_count, uint32_t m, const uint32_t* mk,
                       uint32_t need = 0) {
        const uint32_t n = S.n;
        npair.ensure(n + 1);
        pair_off.ensure(n + 1);
        zero(npair.p, (size_t)n * 4);
        const ListsRef L = S.lists.ref(false);
        launch_upd_pairs(0, list, d_count, m, n, S.periodic ? 1 : 0, L, S.excl.p, mk, need, npair.p, nullptr, nullptr,
                         nullptr, nullptr, stream);
        ensure_scan(n + 1);
        scan_u32(npair.p, pair_off.p, n, scan_tmp.p, stream);
        const uint32_t P = read_word(pair_off.p + n);
        pair_a.ensure(P + 1);
        pair_e.ensure(P + 1);
        nb_pair.ensure(S.lists.E + 1);
        launch_upd_pairs(1, list, d_count, m, n, S.periodic ? 1 : 0, L, S.excl.p, mk, need, npair.p, pair_off.p, pair_a.p,
                         pair_e.p, nb_pair.p, stream);
        return P;
    }

    DevBufs pair_bufs(UState& S, uint32_t P) {
        DevBufs b = base_bufs(S);
        b.nb_cnt = S.lists.cnt.p;
        b.nb_off = S.lists.off.p;
        b.nb_id = S.lists.id.p;
        b.nb_slot = S.lists.id.p;
        b.nb_val = S.lists.val.p;
        b.nb_rel = fp32 ? S.lists.rel.p : nullptr;
        b.nb_pair = nb_pair.p;
        b.pair_off = pair_off.p;
        b.pair_a = pair_a.p;
        b.pair_e = pair_e.p;
        p_status.ensure(P + 1);
        p_central.ensure(P + 1);
        p_area.ensure(P + 1);
        p_arc.ensure(P + 1);
        p_sa_a.ensure(P + 1);
        p_sa_b.ensure(P + 1);
        p_pv_a.ensure(P + 1);
        p_pv_b.ensure(P + 1);
        redo_list.ensure(2 * (size_t)P + 1);
        serial_list.ensure(P + 1);
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
        p_arcm.ensure(6 * (size_t)P + 6);
        b.p_arcm = adjoint ? p_arcm.p : nullptr;
        b.redo_list = redo_list.p;
        b.serial_list = serial_list.p;
        b.serial_scratch = serial_scratch.p;
        b.serial_slots = serial_slots;
        b.cell_flag = S.cell_flag.p;
        b.cell_sas = S.cell_sas.p;
        b.cell_vol = S.cell_vol.p;
        b.cell_redo_list = cell_redo.p;
        b.ball_dirty = ball_dirty.p;
        b.detached_excl = 1;
        return b;
    }

    void contacts(const DevBufs& b, uint32_t P) {
        if (P == 0) return;
        if (fp32) {
            launch_contact_f32(b, P, 1, stream);
            launch_collect_redo(b, P, stream);
            VT_CUDA(cudaMemcpyAsync(h_words + 20, w(kWRedo), 4, cudaMemcpyDeviceToHost, stream));
            launch_contact_f64(b, P, 1, 1, stream);
        } else {
            launch_contact_f64(b, P, 1, 0, stream);
        }
        launch_collect_redo(b, P, stream);
        launch_contact_serial(b, P, 1, stream);
        VT_CUDA(cudaMemcpyAsync(h_words + 21, w(kWSerial), 4, cudaMemcpyDeviceToHost, stream));
    }

    NewContacts nc_ref() {
        return {nc_a.p,    nc_b.p,      nc_area.p,  nc_arc.p,   nc_sa_a.p,  nc_sa_b.p, nc_pv_a.p,
                nc_pv_b.p, nc_central.p, nc_pair.p, nc_gaa.p, nc_gab.p, nc_gba.p, nc_gbb.p,
                nc_vaa.p,  nc_vab.p,    nc_vba.p,   nc_vbb.p};
    }

    // kept contacts of this pass (periodic dedup) as canonical new contacts; the count is
    // keep_off[P] on the device
    void extract_new(const DevBufs& b0, uint32_t P) {
        keep.ensure(P + 1);
        keep_off.ensure(P + 2);
        nc_a.ensure(P + 1);
        nc_b.ensure(P + 1);
        nc_pair.ensure(P + 1);
        nc_area.ensure(P + 1);
        nc_arc.ensure(P + 1);
        nc_sa_a.ensure(P + 1);
        nc_sa_b.ensure(P + 1);
        nc_pv_a.ensure(P + 1);
        nc_pv_b.ensure(P + 1);
        nc_central.ensure(P + 1);
        nc_gaa.ensure(P + 1);
        nc_gab.ensure(P + 1);
        nc_gba.ensure(P + 1);
        nc_gbb.ensure(P + 1);
        nc_vaa.ensure(P + 1);
        nc_vab.ensure(P + 1);
        nc_vba.ensure(P + 1);
        nc_vbb.ensure(P + 1);
        if (P == 0) {
            zero(keep_off.p, 4);
            return;
        }
        DevBufs b = b0;
        b.keep = keep.p;
        b.keep_off = keep_off.p;
        launch_dedup(b, P, 0, stream);
        ensure_scan(P + 1);
        scan_u32(keep.p, keep_off.p, P, scan_tmp.p, stream);
        launch_new_contacts(P, keep_off.p, b, nc_ref(), stream);
    }

    // contacts_by_sphere after removing entries with both ends involved and pushing the
    // new contacts (updateable.rs:494-511); fresh: no old table (full computation)
    void splice_table(UState& S, const uint32_t* mk, bool fresh, uint32_t P) {
        const uint32_t n = S.n;
        keep_cnt.ensure(n + 1);
        new_cnt.ensure(n + 1);
        tot_cnt.ensure(n + 1);
        cursor.ensure(n + 1);
        TableRef old = S.tab.ref();
        if (fresh) old.off = nullptr;
        launch_table_counts(n, mk, old, keep_cnt.p, stream);
        zero(new_cnt.p, (size_t)n * 4);
        const uint32_t* d_nc = keep_off.p + P;
        if (P) launch_table_new_counts(nc_ref(), d_nc, P, new_cnt.p, stream);
        launch_add_u32(keep_cnt.p, new_cnt.p, n, tot_cnt.p, stream);
        const size_t mmax = (fresh ? 0 : S.tab.M) + 2 * (size_t)P + 1;
        next_tab.ensure(n, mmax);
        tmp_k.ensure(mmax);
        ensure_scan(n + 1);
        scan_u32(tot_cnt.p, next_tab.off.p, n, scan_tmp.p, stream);
        // with the adjoint off the coefficients are stale until a full computation: not
        // copied (the adjoints are refused meanwhile)
        TableRef nref = next_tab.ref();
        if (!adjoint) nref.gA = nref.gB = nref.vA = nref.vB = nullptr;
        if (!fresh) launch_table_copy_kept(n, mk, old, nref, stream);
        if (P) {
            zero(cursor.p, (size_t)n * 4);
            launch_table_scatter_new(nc_ref(), d_nc, P, nref, keep_cnt.p, cursor.p, tmp_k.p, stream);
            launch_table_write_new(n, nc_ref(), nref, keep_cnt.p, new_cnt.p, tmp_k.p, w(kWErr), stream);
        }
        S.tab.swap(next_tab);
        S.tab.M = 0;  // known after finish()
    }

    void ensure_cells(UState& S) {
        S.cell_flag.ensure(S.n + 1);
        S.cell_sas.ensure(S.n + 1);
        S.cell_vol.ensure(S.n + 1);
        cell_redo.ensure(S.n + 1);
        ball_dirty.ensure(S.n + 1);
        unsure.ensure(S.n + 1);
    }

    // compute_full_tessellation (updateable.rs:449-474) on the stored balls
    int full_compute(UState& S) {
        const uint32_t n = S.n;
        int st = build_spheres(S);
        if (st != VT_OK) return st;
        S.excl.ensure(n + 1);
        ensure_cells(S);
        st = search(S, nullptr, n, S.lists);
        if (st != VT_OK) return st;
        const uint32_t P = gen_pairs(S, nullptr, nullptr, n, nullptr);
        stats.num_pairs = P;
        DevBufs b = pair_bufs(S, P);
        contacts(b, P);
        // cells from all pair contributions (compute_cells_from_all_summaries, :633-689)
        if (fp32 && P > 0) {
            zero(ball_dirty.p, n);
            zero(w(kWCellRedo), 4);
            launch_cells(b, kCellBand, 0, stream);
            zero(w(kWRedo), 4);
            launch_mark_ball_pairs(b, stream);
            launch_contact_f64(b, P, 1, 1, stream);
            launch_cells(b, 0.f, 1, stream);
        } else {
            launch_cells(b, 0.f, 0, stream);
        }
        extract_new(b, P);
        splice_table(S, nullptr, true, P);
        return VT_OK;
    }

    // FP32 updates: an affected ball whose compute_sas branch is uncertain on its FP32 sums
    // (cell_from_sums' bands) has every contact recomputed in FP64, the table entries kept
    // from earlier operations included (their FP32 values take part in the same sums), and
    // then its cell is recomputed.  The uncertain balls are marked 2 and their neighbours
    // 1; the pairs with an end marked 2 are recomputed, and their FP64 values replace the
    // entries' values in place, so the table keeps the reference's entry order.
    void refresh_unsure_cells(UState& S, const uint32_t* d_count, uint32_t A) {
        const uint32_t n = S.n;
        ulist.ensure(A + 1);
        zero(w(kWUnsure), 4);
        launch_list_flagged(S.affected.p, d_count, A, unsure.p, ulist.p, w(kWUnsure), stream);
        const uint32_t U = read_word(w(kWUnsure));
        stats.num_cell_redo = U;
        if (U == 0) return;
        mark2.ensure(n + 1);
        nflags2.ensure(n + 1);
        noff2.ensure(n + 2);
        aff2.ensure(n + 1);
        zero(mark2.p, (size_t)n * 4);
        launch_mark_list(ulist.p, w(kWUnsure), U, mark2.p, 2, w(kWMarked), stream);
        launch_mark_neighbours(ulist.p, w(kWUnsure), U, nullptr, S.lists.ref(false), n, mark2.p, 1, w(kWMarked),
                               nullptr, stream);
        launch_nonzero(mark2.p, n, nflags2.p, stream);
        ensure_scan(n + 1);
        scan_u32(nflags2.p, noff2.p, n, scan_tmp.p, stream);
        launch_compact_index(noff2.p, n, aff2.p, stream);
        const uint32_t A2 = read_word(noff2.p + n);
        const uint32_t P2 = gen_pairs(S, aff2.p, noff2.p + n, A2, mark2.p, 2);
        DevBufs b = pair_bufs(S, P2);
        if (P2) {
            launch_contact_f64(b, P2, 1, 0, stream);
            launch_collect_redo(b, P2, stream);
            launch_contact_serial(b, P2, 1, stream);
        }
        extract_new(b, P2);
        TableRef tref = S.tab.ref();
        if (!adjoint) tref.gA = tref.gB = tref.vA = tref.vB = nullptr;
        if (P2) launch_table_update(nc_ref(), keep_off.p + P2, P2, tref, w(kWErr), stream);
        // only the uncertain balls' cells are recomputed: all their contacts are FP64 now.
        // Their neighbours keep the cells they have: an affected neighbour was decided
        // outside the band in the first pass (one pair moving from its FP32 to its FP64
        // value stays within it), and a neighbour this operation does not affect keeps its
        // cell in the reference too, while a recomputation could mix FP64 entries with FP32
        // ones this operation wrote for its affected neighbours and, near a threshold, flip
        // its exposure.  A ball without contacts keeps the cell state its last computation
        // gave it (the reference's detached rule applies to affected balls only,
        // updateable.rs:711-719).
        launch_table_cells(ulist.p, w(kWUnsure), U, S.tab.ref(), sph.p, S.excl.p, S.cell_flag.p, S.cell_sas.p,
                           S.cell_vol.p, 0.f, nullptr, stream, 1);
    }

    // update_using_affected (updateable.rs:476-514) for the involved balls (mark != 0),
    // listed sorted in S.affected (count on the device at d_count)
    void update_using_affected(UState& S, const uint32_t* d_count, uint32_t A) {
        t_begin(4);
        const uint32_t P = gen_pairs(S, S.affected.p, d_count, A, mark.p);
        stats.num_pairs = P;
        DevBufs b = pair_bufs(S, P);
        t_end(4);
        t_begin(5);
        contacts(b, P);
        t_end(5);
        t_begin(6);
        extract_new(b, P);
        splice_table(S, mark.p, false, P);
        const float band = (fp32 && P > 0) ? kCellBand : 0.f;
        launch_table_cells(S.affected.p, d_count, A, S.tab.ref(), sph.p, S.excl.p, S.cell_flag.p, S.cell_sas.p,
                           S.cell_vol.p, band, band > 0.f ? unsure.p : nullptr, stream);
        t_end(6);
        if (band > 0.f) {
            t_begin(7);
            refresh_unsure_cells(S, d_count, A);
            t_end(7);
        }
    }

    // table size, cell count and error bits after an operation
    int finish(UState& S) {
        const uint32_t n = S.n;
        // coefficients are whole after a full computation with moments, and stay whole
        // while every update records them
        S.adj_valid = S.full ? adjoint : (S.adj_valid && adjoint);
        t_begin(8);
        nflags.ensure(n + 1);
        noff.ensure(n + 2);
        launch_cell_flags_u32(S.cell_flag.p, n, nflags.p, stream);
        ensure_scan(n + 1);
        scan_u32(nflags.p, noff.p, n, scan_tmp.p, stream);
        VT_CUDA(cudaMemcpyAsync(h_words + 0, S.tab.off.p + n, 4, cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 1, noff.p + n, 4, cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 2, w(kWErr), 4, cudaMemcpyDeviceToHost, stream));
        t_end(8);
        t_end(9);
        sync();
        VT_CUDA(cudaGetLastError());
        t_collect();
        S.tab.M = h_words[0];
        S.num_cells = h_words[1];
        stats.device_error_bits = h_words[2];
        stats.num_fp64_redo = h_words[20];
        stats.num_serial = h_words[21];
        stats.num_entries = S.lists.E;
        stats.num_cells = S.num_cells;
        stats.num_balls = n;
        if (h_words[2] & (kErrOverflow | kErrNeighborCap | 16u)) {
            set_last_error("contour, neighbour or contact-table capacity exceeded");
            return VT_ERR_CAPACITY;
        }
        if (h_words[2] & kErrInvalid) {
            set_last_error("non-finite input or negative radius");
            return VT_ERR_INVALID;
        }
        if (h_words[2] & kErrRefresh) {
            set_last_error("internal: an FP64 cell refresh met a contact missing from the contact table");
            return VT_ERR_CUDA;
        }
        return VT_OK;
    }

    void begin_op() {
        VT_CUDA(cudaSetDevice(device));
        t_reset();
        zero(words.p, kWords * 4);
        const uint32_t one = 1;
        VT_CUDA(cudaMemcpyAsync(w(kWOne), &one, 4, cudaMemcpyHostToDevice, stream));
        h_words[20] = h_words[21] = 0;
        stats = vt_stats{};
    }

    // prepare_for_update (updateable.rs:404-420)
    void prepare_for_update() {
        if (backup_enabled && !cur->empty()) {
            copy_state(*bak, *cur, fp32, stream);
            has_bak = true;
        }
        cur->n_changed = 0;
        cur->n_affected = 0;
        cur->affected_dups = false;
        cur->full = false;
    }

    // init (updateable.rs:187-201) / a full reinit inside an update
    int reinit(const double* d_xyzr, uint32_t n, int* ok) {
        UState& S = *cur;
        S.n = n;
        S.balls.ensure(4 * (size_t)n + 4);
        if (n) VT_CUDA(cudaMemcpyAsync(S.balls.p, d_xyzr, 32 * (size_t)n, cudaMemcpyDeviceToDevice, stream));
        S.n_changed = S.n_affected = 0;
        S.affected_dups = false;
        S.full = true;
        S.lists.E = 0;
        S.tab.M = 0;
        S.num_cells = 0;
        sph_fresh = false;
        if (n == 0) {
            if (ok) *ok = 0;
            return VT_OK;
        }
        int st = full_compute(S);
        if (st == VT_OK) st = finish(S);
        if (ok) *ok = (st == VT_OK && !S.empty()) ? 1 : 0;
        return st;
    }

    int init(const double* d_xyzr, uint32_t n, double probe, const double* pbox9, int* ok) {
        begin_op();
        prepare_for_update();
        UState& S = *cur;
        S.probe = probe;
        S.periodic = pbox9 != nullptr;
        for (int k = 0; k < 9; ++k) S.pbox[k] = pbox9 ? pbox9[k] : 0.0;
        return reinit(d_xyzr, n, ok);
    }

    // update_internal (updateable.rs:422-447) + SpheresContainer::update
    // (spheres_container.rs:71-182).  src: new balls, indexed by id (src_by_id) or packed
    // per listed id; ids == null: every ball is compared.  *need_full: a full reinit from
    // the complete new ball array is required (the caller supplies it).
    int update(const double* src, int src_by_id, const uint64_t* d_ids, uint32_t k, int* changed_out,
               bool* need_full) {
        *need_full = false;
        *changed_out = 0;
        UState& S = *cur;
        const uint32_t n = S.n;
        const uint32_t thr = std::max<uint32_t>(n / 2, 10);  // size_threshold_for_full_reinit
        if (k == 0 || n == 0) return VT_OK;
        t_begin(9);
        t_begin(0);
        flags.ensure(k + 1);
        flags_off.ensure(k + 2);
        S.changed.ensure(k + 1);
        changed_ball.ensure(k + 1);
        launch_changed_flags(d_ids, k, src, src_by_id, n, S.probe, S.balls.p, flags.p, stream);
        ensure_scan(k + 1);
        scan_u32(flags.p, flags_off.p, k, scan_tmp.p, stream);
        launch_changed_compact(d_ids, k, src, src_by_id, flags_off.p, S.changed.p, changed_ball.p, stream);
        uint32_t* d_kc = flags_off.p + k;
        if (!d_ids) launch_clamp_count(d_kc, thr + 1, stream);  // .take(threshold + 1)
        mark.ensure(n + 1);
        zero(mark.p, (size_t)n * 4);
        launch_mark_list(S.changed.p, d_kc, k, mark.p, 1, w(kWDistinct), stream);
        launch_mark_neighbours(S.changed.p, d_kc, k, nullptr, S.lists.ref(false), n, mark.p, 1, w(kWNbrNew), nullptr,
                               stream);
        VT_CUDA(cudaMemcpyAsync(h_words + 0, d_kc, 4, cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 1, w(kWDistinct), 4, cudaMemcpyDeviceToHost, stream));
        VT_CUDA(cudaMemcpyAsync(h_words + 2, w(kWNbrNew), 4, cudaMemcpyDeviceToHost, stream));
        t_end(0);
        sync();
        const uint32_t kc = h_words[0], distinct = h_words[1], nbr_new = h_words[2];
        if (kc == 0) return VT_OK;  // no change: update returns false
        if (kc > thr || (uint64_t)kc + nbr_new > thr) {
            t_reset();  // a full reinit follows: no update stages to report
            *need_full = true;
            return VT_OK;
        }
        // apply, rebuild spheres and grid, search the frontier (changed + old neighbours)
        t_begin(1);
        launch_apply_changed(S.changed.p, changed_ball.p, d_kc, k, S.balls.p, stream);
        int st = build_spheres(S);
        t_end(1);
        if (st != VT_OK) return st;
        t_begin(2);
        const uint32_t A1 = distinct + nbr_new;
        nflags.ensure(n + 1);
        noff.ensure(n + 2);
        list1.ensure(n + 1);
        row_of.ensure(n + 1);
        launch_nonzero(mark.p, n, nflags.p, stream);
        ensure_scan(n + 1);
        scan_u32(nflags.p, noff.p, n, scan_tmp.p, stream);
        launch_compact_index(noff.p, n, list1.p, stream);
        launch_row_of(list1.p, noff.p + n, A1, row_of.p, stream);
        st = search(S, list1.p, A1, t1);
        if (st != VT_OK) return st;
        // new neighbours of changed balls (spheres_container.rs:147-167)
        more_list.ensure(n + 1);
        launch_mark_neighbours(S.changed.p, d_kc, k, row_of.p, t1.ref(false), n, mark.p, 2, w(kWMore), more_list.p,
                               stream);
        const uint32_t more = read_word(w(kWMore));
        if (more) {
            launch_row_of(more_list.p, w(kWMore), more, row_of.p, stream);
            st = search(S, more_list.p, more, t2);
            if (st != VT_OK) return st;
        }
        t_end(2);
        // splice the neighbour lists
        t_begin(3);
        next_lists.cnt.ensure(n + 1);
        next_lists.off.ensure(n + 1);
        launch_splice_counts(n, mark.p, row_of.p, S.lists.cnt.p, t1.cnt.p, more ? t2.cnt.p : nullptr,
                             next_lists.cnt.p, stream);
        scan_u32(next_lists.cnt.p, next_lists.off.p, n, scan_tmp.p, stream);
        const uint32_t E = read_word(next_lists.off.p + n);
        next_lists.id.ensure(E + 1);
        next_lists.val.ensure(E + 1);
        if (fp32) next_lists.rel.ensure(E + 1);
        const ListsRef none{nullptr, nullptr, nullptr, nullptr, nullptr};
        launch_splice_lists(n, mark.p, row_of.p, S.lists.ref(fp32), t1.ref(fp32), more ? t2.ref(fp32) : none,
                            next_lists.off.p, next_lists.id.p, next_lists.val.p, fp32 ? next_lists.rel.p : nullptr,
                            stream);
        next_lists.E = E;
        S.lists.swap(next_lists);
        // affected = changed + old and new neighbours, sorted
        const uint32_t A = A1 + more;
        launch_nonzero(mark.p, n, nflags.p, stream);
        scan_u32(nflags.p, noff.p, n, scan_tmp.p, stream);
        S.affected.ensure(n + 1);
        launch_compact_index(noff.p, n, S.affected.p, stream);
        S.n_changed = kc;
        S.n_affected = A;
        S.affected_dups = more == 0 && kc > distinct;
        S.full = false;
        t_end(3);
        update_using_affected(S, noff.p + n, A);
        st = finish(S);
        if (st != VT_OK) return st;
        *changed_out = 1;
        return VT_OK;
    }

    // set_exclusion (updateable.rs:226-271) after its checks and prepare_for_update
    int exclusion(uint32_t id, bool excluded) {
        UState& S = *cur;
        const uint32_t n = S.n;
        int st = VT_OK;
        if (!sph_fresh) st = build_spheres(S);
        if (st != VT_OK) return st;
        mark.ensure(n + 1);
        zero(mark.p, (size_t)n * 4);
        const uint8_t v = excluded ? 1 : 0;
        if (excluded) {
            launch_mark_table_partners(id, S.tab.ref(), mark.p, stream);
        } else {
            VT_CUDA(cudaMemcpyAsync(w(kWId), &id, 4, cudaMemcpyHostToDevice, stream));
            launch_mark_list(w(kWId), w(kWOne), 1, mark.p, 1, w(kWDistinct), stream);
            launch_mark_neighbours(w(kWId), w(kWOne), 1, nullptr, S.lists.ref(false), n, mark.p, 1, w(kWNbrNew),
                                   nullptr, stream);
        }
        VT_CUDA(cudaMemcpyAsync(S.excl.p + id, &v, 1, cudaMemcpyHostToDevice, stream));
        nflags.ensure(n + 1);
        noff.ensure(n + 2);
        launch_nonzero(mark.p, n, nflags.p, stream);
        ensure_scan(n + 1);
        scan_u32(nflags.p, noff.p, n, scan_tmp.p, stream);
        S.affected.ensure(n + 1);
        launch_compact_index(noff.p, n, S.affected.p, stream);
        const uint32_t A = read_word(noff.p + n);
        S.changed.ensure(2);
        VT_CUDA(cudaMemcpyAsync(S.changed.p, &id, 4, cudaMemcpyHostToDevice, stream));
        S.n_changed = 1;
        S.n_affected = A;
        S.affected_dups = false;
        S.full = false;
        update_using_affected(S, noff.p + n, A);
        return finish(S);
    }

    int summary(vt_result** out) {
        UState& S = *cur;
        std::unique_ptr<vt_result> r(new vt_result());
        const uint32_t n = S.n;
        r->num_balls = n;
        if (n == 0) {
            *out = r.release();
            return VT_OK;
        }
        const uint32_t M = (uint32_t)S.tab.M;
        sum_flags.ensure(M + 1);
        sum_off.ensure(M + 2);
        ensure_scan(std::max<size_t>(M, n) + 1);
        if (M) launch_owner_flags(S.tab.flags.p, M, sum_flags.p, stream);
        scan_u32(sum_flags.p, sum_off.p, M, scan_tmp.p, stream);
        const uint32_t C = read_word(sum_off.p + M);
        out_a.ensure(C + 1);
        out_b.ensure(C + 1);
        out_area.ensure(C + 1);
        out_arc.ensure(C + 1);
        out_central.ensure(C + 1);
        if (M) launch_summary_contacts(S.tab.ref(), M, sum_off.p, out_a.p, out_b.p, out_area.p, out_arc.p,
                                       out_central.p, stream);
        nflags.ensure(n + 1);
        noff.ensure(n + 2);
        launch_cell_flags_u32(S.cell_flag.p, n, nflags.p, stream);
        scan_u32(nflags.p, noff.p, n, scan_tmp.p, stream);
        out_cell_index.ensure(n + 1);
        out_cell_sas.ensure(n + 1);
        out_cell_vol.ensure(n + 1);
        launch_summary_cells(noff.p, n, S.cell_sas.p, S.cell_vol.p, out_cell_index.p, out_cell_sas.p,
                             out_cell_vol.p, stream);
        launch_sums3(out_area.p, sum_off.p + M, out_cell_sas.p, out_cell_vol.p, noff.p + n, partials.p, totals.p,
                     stream);
        const uint32_t K = (uint32_t)S.num_cells;
        r->a.resize(C);
        r->b.resize(C);
        r->area.resize(C);
        r->arc.resize(C);
        r->central.resize(C);
        r->cell_index.resize(K);
        r->cell_sas.resize(K);
        r->cell_vol.resize(K);
        if (C) {
            VT_CUDA(cudaMemcpyAsync(r->a.data(), out_a.p, C * 4, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->b.data(), out_b.p, C * 4, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->area.data(), out_area.p, C * 8, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->arc.data(), out_arc.p, C * 8, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->central.data(), out_central.p, C, cudaMemcpyDeviceToHost, stream));
        }
        if (K) {
            VT_CUDA(cudaMemcpyAsync(r->cell_index.data(), out_cell_index.p, K * 4, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->cell_sas.data(), out_cell_sas.p, K * 8, cudaMemcpyDeviceToHost, stream));
            VT_CUDA(cudaMemcpyAsync(r->cell_vol.data(), out_cell_vol.p, K * 8, cudaMemcpyDeviceToHost, stream));
        }
        double tot[3];
        VT_CUDA(cudaMemcpyAsync(tot, totals.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        sync();
        r->totals[0] = tot[0];
        r->totals[1] = tot[1];
        r->totals[2] = tot[2];
        *out = r.release();
        return VT_OK;
    }

    // adjoint of sum_i w_i SAS_i + sum_i v_i V_i over the current state (w == null: every
    // w_i = w_default; v == null: no volume term), a gather over the table's per-entry
    // coefficients (no contour is recomputed)
    int grad(const double* d_w, double w_default, const double* d_v, double* d_grad) {
        UState& S = *cur;
        const uint32_t n = S.n;
        if (n == 0) return VT_OK;
        if (!S.adj_valid) {
            set_last_error("adjoint unavailable: an operation ran with the adjoint off "
                           "(vt_upd_set_adjoint); enable it and init again");
            return VT_ERR_INVALID;
        }
        if (!sph_fresh) {
            int st = build_spheres(S);
            if (st != VT_OK) return st;
        }
        launch_table_grad(n, S.tab.ref(), d_w, w_default, d_v, S.cell_flag.p, S.cell_sas.p, sph.p, d_grad, stream);
        sync();
        VT_CUDA(cudaGetLastError());
        return VT_OK;
    }

    // totals of the current summary without downloading it: sas, volume, contact area
    int totals3(double* out3) {
        vt_result* r = nullptr;
        int st = summary(&r);
        if (st != VT_OK) return st;
        for (int k = 0; k < 3; ++k) out3[k] = r->totals[k];
        delete r;
        return VT_OK;
    }

    std::vector<uint64_t> ids_of(const DBuf<uint32_t>& d, uint32_t m) {
        std::vector<uint32_t> h(m);
        if (m) {
            VT_CUDA(cudaMemcpyAsync(h.data(), d.p, m * 4, cudaMemcpyDeviceToHost, stream));
            sync();
        }
        return std::vector<uint64_t>(h.begin(), h.end());
    }
    std::vector<uint64_t> affected_ids() {
        UState& S = *cur;
        std::vector<uint64_t> a = ids_of(S.affected, S.n_affected);
        if (!S.affected_dups) return a;
        // the reference's affected list starts from the sorted changed ids, duplicates
        // included, and is deduplicated only when new neighbours were appended
        std::vector<uint64_t> c = ids_of(S.changed, S.n_changed);
        std::sort(c.begin(), c.end());
        std::vector<uint64_t> outv;
        size_t j = 0;
        for (uint64_t id : a) {
            while (j < c.size() && c[j] < id) ++j;
            size_t k = j;
            while (k < c.size() && c[k] == id) ++k;
            size_t mult = std::max<size_t>(1, k - j);
            for (size_t t = 0; t < mult; ++t) outv.push_back(id);
            j = k;
        }
        return outv;
    }
    uint64_t num_affected() {
        UState& S = *cur;
        if (!S.affected_dups) return S.n_affected;
        return affected_ids().size();
    }
};

namespace {

int check_handle(const vt_updateable* h) {
    if (!h) {
        set_last_error("null handle");
        return VT_ERR_INVALID;
    }
    return VT_OK;
}

// host-array entry points: upload, then the device-side operation
int host_update(vt_updateable* h, const double* xyzr, uint64_t n, const uint64_t* ids, uint64_t k, bool all,
                int* changed) {
    if (changed) *changed = 0;
    if (n && !xyzr) return VT_ERR_INVALID;
    if (!all && k && !ids) return VT_ERR_INVALID;
    if (!all && k == 0) return VT_OK;  // update_with_changed with no ids (updateable.rs:216-218)
    if (n >= (uint64_t)0xffffffffu / 27u) {
        set_last_error("too many balls for 32-bit ids");
        return VT_ERR_INVALID;
    }
    return guarded([&]() -> int {
        h->begin_op();
        h->prepare_for_update();
        UState& S = *h->cur;
        int ch = 0;
        auto full = [&]() -> int {
            int st = check_host_balls(xyzr, n);
            if (st != VT_OK) return st;
            h->src_in.ensure(4 * n + 4);
            if (n)
                VT_CUDA(cudaMemcpyAsync(h->src_in.p, xyzr, 32 * n, cudaMemcpyHostToDevice, h->stream));
            st = h->reinit(h->src_in.p, (uint32_t)n, nullptr);
            if (st == VT_OK && changed) *changed = 1;
            return st;
        };
        if (n != S.n) return full();  // spheres_container.rs:77-84
        bool need_full = false;
        int st;
        if (all) {
            st = check_host_balls(xyzr, n);
            if (st != VT_OK) return st;
            h->src_in.ensure(4 * n + 4);
            VT_CUDA(cudaMemcpyAsync(h->src_in.p, xyzr, 32 * n, cudaMemcpyHostToDevice, h->stream));
            st = h->update(h->src_in.p, 1, nullptr, (uint32_t)n, &ch, &need_full);
        } else {
            // pack the listed balls: only those are read (spheres_container.rs:88-95)
            std::vector<double> packed(4 * k, 0.0);
            for (uint64_t t = 0; t < k; ++t)
                if (ids[t] < n) {
                    std::memcpy(&packed[4 * t], xyzr + 4 * ids[t], 32);
                    st = check_host_balls(&packed[4 * t], 1);
                    if (st != VT_OK) return st;
                }
            h->ids_in.ensure(k + 1);
            h->src_in.ensure(4 * k + 4);
            VT_CUDA(cudaMemcpyAsync(h->ids_in.p, ids, 8 * k, cudaMemcpyHostToDevice, h->stream));
            VT_CUDA(cudaMemcpyAsync(h->src_in.p, packed.data(), 32 * k, cudaMemcpyHostToDevice, h->stream));
            h->sync();  // `packed` is pageable host memory
            st = h->update(h->src_in.p, 0, h->ids_in.p, (uint32_t)k, &ch, &need_full);
        }
        if (st != VT_OK) return st;
        if (need_full) return full();
        if (changed) *changed = ch;
        return VT_OK;
    });
}

}  // namespace

extern "C" {

int vt_upd_create(int device, int with_backup, int precision, vt_updateable** out) {
    if (!out) return VT_ERR_INVALID;
    *out = nullptr;
    if (precision != VT_FP64 && precision != VT_FP32_FIXUP) {
        set_last_error("unknown precision");
        return VT_ERR_INVALID;
    }
    return guarded([&]() -> int {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            set_last_error("no CUDA device");
            return VT_ERR_NO_DEVICE;
        }
        if (device < 0 || device >= ndev) {
            set_last_error("bad device index");
            return VT_ERR_INVALID;
        }
        std::unique_ptr<vt_updateable> h(new vt_updateable());
        h->init_handle(device, with_backup != 0, precision);
        *out = h.release();
        return VT_OK;
    });
}
void vt_upd_destroy(vt_updateable* h) { delete h; }
int vt_upd_set_stream(vt_updateable* h, void* stream) {
    if (check_handle(h)) return VT_ERR_INVALID;
    h->stream = stream ? (cudaStream_t)stream : h->own;
    return VT_OK;
}
int vt_upd_init(vt_updateable* h, const double* xyzr, uint64_t n, double probe, const double* periodic_box9,
                int* ok) {
    if (ok) *ok = 0;
    if (check_handle(h) || (n && !xyzr)) return VT_ERR_INVALID;
    if (n >= (uint64_t)0xffffffffu / 27u || !std::isfinite(probe)) {
        set_last_error("too many balls or non-finite probe");
        return VT_ERR_INVALID;
    }
    int st = check_host_balls(xyzr, n);
    if (st != VT_OK) return st;
    return guarded([&]() -> int {
        VT_CUDA(cudaSetDevice(h->device));
        h->src_in.ensure(4 * n + 4);
        if (n) VT_CUDA(cudaMemcpyAsync(h->src_in.p, xyzr, 32 * n, cudaMemcpyHostToDevice, h->stream));
        return h->init(h->src_in.p, (uint32_t)n, probe, periodic_box9, ok);
    });
}
int vt_upd_init_device(vt_updateable* h, const double* d_xyzr, uint64_t n, double probe,
                       const double* periodic_box9, int* ok) {
    if (ok) *ok = 0;
    if (check_handle(h) || (n && !d_xyzr)) return VT_ERR_INVALID;
    if (n >= (uint64_t)0xffffffffu / 27u || !std::isfinite(probe)) {
        set_last_error("too many balls or non-finite probe");
        return VT_ERR_INVALID;
    }
    return guarded([&]() -> int { return h->init(d_xyzr, (uint32_t)n, probe, periodic_box9, ok); });
}
int vt_upd_update(vt_updateable* h, const double* xyzr, uint64_t n, int* changed) {
    if (check_handle(h)) return VT_ERR_INVALID;
    return host_update(h, xyzr, n, nullptr, n, true, changed);
}
int vt_upd_update_with_changed(vt_updateable* h, const double* xyzr, uint64_t n, const uint64_t* ids, uint64_t k,
                               int* changed) {
    if (check_handle(h)) return VT_ERR_INVALID;
    return host_update(h, xyzr, n, ids, k, false, changed);
}
int vt_upd_update_with_changed_device(vt_updateable* h, const double* d_xyzr, uint64_t n, const uint64_t* d_ids,
                                      uint64_t k, int* changed) {
    if (changed) *changed = 0;
    if (check_handle(h) || (n && !d_xyzr) || (k && !d_ids)) return VT_ERR_INVALID;
    if (k == 0) return VT_OK;
    if (n >= (uint64_t)0xffffffffu / 27u || k >= 0xffffffffu) {
        set_last_error("too many balls or ids");
        return VT_ERR_INVALID;
    }
    return guarded([&]() -> int {
        h->begin_op();
        h->prepare_for_update();
        int ch = 0;
        bool need_full = false;
        if (n != h->cur->n) {
            need_full = true;
        } else {
            int st = h->update(d_xyzr, 1, d_ids, (uint32_t)k, &ch, &need_full);
            if (st != VT_OK) return st;
        }
        if (need_full) {
            int st = h->reinit(d_xyzr, (uint32_t)n, nullptr);
            if (st != VT_OK) return st;
            ch = 1;
        }
        if (changed) *changed = ch;
        return VT_OK;
    });
}
int vt_upd_set_exclusion(vt_updateable* h, uint64_t id, int excluded, int* changed) {
    if (changed) *changed = 0;
    if (check_handle(h)) return VT_ERR_INVALID;
    return guarded([&]() -> int {
        UState& S = *h->cur;
        if (S.empty() || id >= S.n) return VT_OK;
        h->begin_op();
        uint8_t curv = 0;
        VT_CUDA(cudaMemcpyAsync(&curv, S.excl.p + id, 1, cudaMemcpyDeviceToHost, h->stream));
        h->sync();
        if ((curv != 0) == (excluded != 0)) return VT_OK;
        h->prepare_for_update();
        int st = h->exclusion((uint32_t)id, excluded != 0);
        if (st != VT_OK) return st;
        if (changed) *changed = 1;
        return VT_OK;
    });
}
int vt_upd_restore(vt_updateable* h, int* ok) {
    if (ok) *ok = 0;
    if (check_handle(h)) return VT_ERR_INVALID;
    if (!h->backup_enabled || !h->has_bak) return VT_OK;
    std::swap(h->cur, h->bak);
    h->has_bak = false;
    h->sph_fresh = false;
    if (ok) *ok = 1;
    return VT_OK;
}
int vt_upd_summary(vt_updateable* h, vt_result** out) {
    if (!out) return VT_ERR_INVALID;
    *out = nullptr;
    if (check_handle(h)) return VT_ERR_INVALID;
    return guarded([&]() -> int {
        VT_CUDA(cudaSetDevice(h->device));
        return h->summary(out);
    });
}
int vt_upd_totals(vt_updateable* h, double* totals3) {
    if (check_handle(h) || !totals3) return VT_ERR_INVALID;
    return guarded([&]() -> int {
        VT_CUDA(cudaSetDevice(h->device));
        return h->totals3(totals3);
    });
}
int vt_upd_grad_sas(vt_updateable* h, const double* d_w_sas, double* d_grad) {
    if (check_handle(h) || !d_grad) return VT_ERR_INVALID;
    return guarded([&]() -> int {
        h->begin_op();
        return h->grad(d_w_sas, 1.0, nullptr, d_grad);
    });
}
int vt_upd_grad(vt_updateable* h, const double* d_w_sas, const double* d_v_volume, double* d_grad) {
    if (check_handle(h) || !d_grad) return VT_ERR_INVALID;
    return guarded([&]() -> int {
        h->begin_op();
        return h->grad(d_w_sas, 0.0, d_v_volume, d_grad);
    });
}
int vt_upd_set_adjoint(vt_updateable* h, int on) {
    if (check_handle(h)) return VT_ERR_INVALID;
    h->adjoint = on != 0;
    return VT_OK;
}
int vt_upd_last_full_reinit(const vt_updateable* h) { return h && h->cur->full ? 1 : 0; }
uint64_t vt_upd_num_changed(const vt_updateable* h) { return h ? h->cur->n_changed : 0; }
int vt_upd_changed_ids(vt_updateable* h, uint64_t* out) {
    if (check_handle(h) || (!out && h->cur->n_changed)) return VT_ERR_INVALID;
    return guarded([&]() -> int {
        std::vector<uint64_t> v = h->ids_of(h->cur->changed, h->cur->n_changed);
        if (!v.empty()) std::memcpy(out, v.data(), v.size() * 8);
        return VT_OK;
    });
}
uint64_t vt_upd_num_affected(vt_updateable* h) {
    if (!h) return 0;
    uint64_t m = 0;
    guarded([&]() -> int {
        m = h->num_affected();
        return VT_OK;
    });
    return m;
}
int vt_upd_affected_ids(vt_updateable* h, uint64_t* out) {
    if (check_handle(h)) return VT_ERR_INVALID;
    return guarded([&]() -> int {
        std::vector<uint64_t> v = h->affected_ids();
        if (!v.empty()) {
            if (!out) return VT_ERR_INVALID;
            std::memcpy(out, v.data(), v.size() * 8);
        }
        return VT_OK;
    });
}
int vt_upd_stats(const vt_updateable* h, vt_stats* out) {
    if (check_handle(h) || !out) return VT_ERR_INVALID;
    *out = h->stats;
    return VT_OK;
}
int vt_upd_set_timing(vt_updateable* h, int on) {
    if (check_handle(h)) return VT_ERR_INVALID;
    h->timing = on != 0;
    return VT_OK;
}
int vt_upd_stage_times(const vt_updateable* h, double* ms) {
    if (check_handle(h) || !ms) return VT_ERR_INVALID;
    for (int k = 0; k < VT_UPD_NUM_STAGES; ++k) ms[k] = h->stage_ms[k];
    return VT_OK;
}

}  // extern "C"
