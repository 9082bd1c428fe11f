"""Benchmark: radical tessellation of a 100,000-ball structure on B200.

Workload (the configuration the headline metric is quoted on): 100,000 balls from the
seeded jittered-lattice generator (2.9 A spacing, +/-0.4 A jitter, protein-like radius
mix; voronota_ltr.workloads.lattice_balls), probe 1.4, compute_tessellation, FP32 bulk
geometry with FP64 recomputation of band pairs.  One step = one full tessellation
(grid, neighbour lists, contacts, cells, compaction, totals).

  value  balls/s with the input resident in HBM (engine API, per-step CUDA events on the
         launching stream; a 256 MiB buffer is written between steps, outside the
         events, to flush the 126 MB L2)
  e2e    balls/s through the public C ABI (vt_compute_tessellation via the Python
         front end) from pinned host memory, results copied back to host arrays; wall
         clock per call, median over the timed steps (mean and extremes reported beside)
  roofline  the contact kernel (the dominant kernel): algorithmic bytes per launch /
         its CUDA-event duration, against the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (a restatement of the reference's Rust code; Rust is not
         in this image) on the host cores

With torchrun (N > 1) each rank tessellates its own structure (seed = rank): independent
replicas, no collective on the data path; value = all ranks' balls / max-over-ranks time
(voronota_ltr.replicas).  The batched leg splits ONE batch of structures across the ranks
(contiguous blocks of about equal ball counts) and reports the whole batch's balls over the
max-over-ranks time.  The contacts-only (groups), updateable trajectory and differentiation
legs run on every rank on its own inputs and report max-over-ranks times; the network leg
times compute_tessellation with with_cell_vertices on the main structure and checks its
vertices and edges against the oracle; the solvent-sphere leg times compute_solvent_spheres
through the C ABI against the CPU oracle.

``--impl reference`` times the reference's algorithm on the host cores instead (the CPU
oracle port: the Rust reference cannot be built here) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "voronota-ltr_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

N_BALLS = 100_000
PROBE = 1.4
METRIC = "balls/s (FP32+FP64 fixup tessellation, 100k-ball structure)"
UNIT = "balls/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_BALLS)
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--upd-n", type=int, default=200_000, help="balls of the periodic updateable trajectory")
    ap.add_argument("--upd-steps", type=int, default=1000, help="steps of the updateable trajectory")
    ap.add_argument("--upd-check-every", type=int, default=100,
                    help="trajectory steps between drift checks against a full recomputation")
    ap.add_argument("--no-contacts-only", action="store_true", help="skip the contacts-only-with-groups leg")
    ap.add_argument("--no-upd", action="store_true", help="skip the updateable trajectory leg")
    ap.add_argument("--no-network", action="store_true", help="skip the tessellation network leg")
    ap.add_argument("--no-solvent", action="store_true", help="skip the solvent-sphere leg")
    ap.add_argument("--solvent-n", type=int, default=20_000, help="balls of the solvent-sphere leg")
    ap.add_argument("--tuning", default=None,
                    help="warps,cell_scale,chunk of the FP32 contact launch instead of autotuning (profiling)")
    ap.add_argument("--batch-count", type=int, default=4096, help="structures of the batched leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched leg")
    ap.add_argument("--grad-n", type=int, default=20_000, help="balls of the differentiation leg")
    ap.add_argument("--no-grad", action="store_true", help="skip the differentiation leg")
    return ap.parse_args()


def headline_config(n, world):
    """The `config` of the headline line, identical in both arms."""
    return {"workload": f"lattice {n} balls per GPU, probe 1.4, compute_tessellation, FP32+fixup",
            "balls_per_gpu": n, "probe": PROBE, "parallelism": f"replicas x{world}",
            "l2": "256 MiB buffer written between timed steps (outside the per-step events)"}


def workload(n, seed):
    from voronota_ltr import workloads as W

    return W.lattice_balls(n, seed)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_value(key):
    """A figure of the contact kernel's committed ncu summary (per launch on the 100k
    lattice), if present: traffic_bytes_per_launch, warp_instructions_per_launch."""
    path = os.path.join(ROOT, "profiles", "contact_kernel_fp32_100k.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(key + ":"):
                    return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


def profiled_traffic():
    """Bytes per contact-kernel launch from the committed ncu summary, if present."""
    return profiled_value("traffic_bytes_per_launch")


def issue_roofline(kernel_ms, sm_mhz, n_balls):
    """The contact kernel's instruction-issue roofline: the warp instructions of one launch
    (ncu, committed summary; valid for the 100k lattice it was measured on) over its
    CUDA-event time, against one instruction per cycle on each of the 4 schedulers of the
    148 SMs at the sampled SM clock."""
    inst = profiled_value("warp_instructions_per_launch")
    if inst is None or not kernel_ms or n_balls != 100_000:
        return None
    peak = 148 * 4 * (sm_mhz or 1965.0) * 1e6
    achieved = inst / (kernel_ms * 1e-3)
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "warp instructions/s",
            "frac": achieved / peak, "instructions_source": "profiles/contact_kernel_fp32_100k.md (ncu)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"vt_clocks_{os.getpid()}_{device}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(balls, seconds=12.0):
    """The CPU oracle on all host cores: balls/s over repeated full tessellations."""
    import oracle as O

    O.set_threads(0)
    cores = O.get_threads()
    O.compute(balls, PROBE)  # warm-up
    times = []
    t_end = time.perf_counter() + seconds
    while len(times) < 2 or (time.perf_counter() < t_end and len(times) < 20):
        t0 = time.perf_counter()
        O.compute(balls, PROBE)
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return {"value": len(balls) / med, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(times)} full tessellations of the {len(balls)}-ball structure, median time"}


def trajectory(n, steps, seed):
    """Periodic cube at 0.033 balls/A^3, r 1.52; each step moves a seeded random 1% of the
    balls by N(0, 0.05 A) per axis (the periodic updateable trajectory workload)."""
    from voronota_ltr import workloads as W

    balls, side = W.periodic_box_balls(n, seed=seed)
    box = {"corners": [(0.0, 0.0, 0.0), (side, side, side)]}
    rng = np.random.default_rng(1000 + seed)
    k = max(1, n // 100)
    moves = []
    for _ in range(steps):
        ids = np.sort(rng.choice(n, k, replace=False)).astype(np.int64)
        moves.append((ids, rng.normal(0.0, 0.05, (k, 3))))
    return balls, box, moves


def _pair_set(a, b):
    a = np.asarray(a, np.int64)
    b = np.asarray(b, np.int64)
    o = np.lexsort((b, a))
    return a[o], b[o], o


def trajectory_drift(u, balls_now, box, n, V, oracle=False):
    """The handle's summary after many FP32 updates against a full recomputation of the
    same positions: the FP64 GPU path (and, with oracle, the CPU oracle): the contact
    pair sets compared exactly, per-contact |dA|, cells, and the totals' relative error."""
    s = u.summary()
    ga, gb, go = _pair_set(s.id_a, s.id_b)
    out = {}
    refs = [("gpu_fp64", V.compute_tessellation_result(balls_now, PROBE, box, precision="fp64"))]
    if oracle:
        import oracle as O

        o = O.compute(balls_now, PROBE, periodic_box=box)
        refs.append(("oracle", V.Result(n, o.contacts_a.astype(np.uint32), o.contacts_b.astype(np.uint32),
                                        o.contacts_area, o.contacts_arc, o.contacts_central,
                                        o.cells_index.astype(np.uint32), o.cells_sas, o.cells_vol,
                                        (o.total_sas_area, o.total_volume, o.total_contact_area))))
    for name, r in refs:
        ra, rb, ro = _pair_set(r.id_a, r.id_b)
        same = len(ra) == len(ga) and np.array_equal(ra, ga) and np.array_equal(rb, gb)
        d = {"contacts_identical": bool(same), "contacts": int(len(ga)),
             "rel_err_total_sas": abs(s.total_sas_area - r.total_sas_area) / r.total_sas_area,
             "rel_err_total_volume": abs(s.total_volume - r.total_volume) / r.total_volume}
        if same:
            d["max_abs_dA"] = float(np.abs(s.area[go] - r.area[ro]).max(initial=0.0))
        cells_same = np.array_equal(s.cell_index, r.cell_index)
        d["cells_identical"] = bool(cells_same)
        if cells_same:
            d["max_abs_d_cell_sas"] = float(np.abs(s.cell_sas_area - r.cell_sas_area).max(initial=0.0))
        out[name] = d
    return out


def updateable_leg(args, rank, torch, V, R):
    """UpdateableTessellation.update_with_changed on the device along the periodic
    trajectory: --upd-steps steps (1,000 by default), each moving 1% of the balls and then
    taking the adjoint of the total SAS.

    Per update: CUDA events on the handle's stream around vt_upd_update_with_changed_device
    (the call returns after its work; inputs already in HBM), and around the adjoint.
    Every --upd-check-every steps the handle's state is compared with a full FP64 GPU
    recomputation of the same positions (outside the events), and at the middle and last
    checkpoints (rank 0) with the CPU oracle's: the drift of the FP32 state whose table
    entries are overwritten in place over the whole trajectory.  Also: the same steps in
    FP64 and with the adjoint off (shorter runs), a full FP32 recompute of the final state,
    and (rank 0) the CPU oracle's own updateable tessellation on the first steps.
    """
    from voronota_ltr.replicas import replica_throughput

    n = args.upd_n
    warm = max(1, args.warmup)
    steps = max(5, args.upd_steps)
    check = max(1, args.upd_check_every)
    balls, box, moves = trajectory(n, warm + steps, rank)
    stream = torch.cuda.current_stream()

    def run(precision, nsteps, adjoint=True, checks=False):
        u = V.UpdateableTessellation(False, precision)
        u.set_stream(stream.cuda_stream)
        u.set_adjoint(adjoint)
        u.set_timing(checks)
        d = torch.from_numpy(balls).cuda()
        torch.cuda.synchronize()
        u.init_device(d.data_ptr(), n, PROBE, box)
        ms, adj, pairs, redo, cref, drift, stages, syncs = [], [], [], [], [], [], [], []
        dg = torch.empty((n, 4), dtype=torch.float64, device="cuda")
        for t, (ids, disp) in enumerate(moves[:warm + nsteps]):
            ti = torch.from_numpy(ids).cuda()
            d[ti, :3] += torch.from_numpy(disp).cuda()
            torch.cuda.synchronize()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            u.update_with_changed_device(d.data_ptr(), n, ti.data_ptr(), len(ids))
            e1.record(stream)
            st = u.stats()
            if checks:
                stages.append(u.stage_times())
            if adjoint:
                u.grad_sas_device(0, dg.data_ptr())  # adjoint of the total SAS
            e2.record(stream)
            e2.synchronize()
            if t >= warm:
                ms.append(e0.elapsed_time(e1))
                adj.append(e1.elapsed_time(e2))
                pairs.append(int(st.num_pairs))
                redo.append(int(st.num_fp64_redo))
                cref.append(int(st.num_cell_redo))
                syncs.append(int(st.num_host_syncs))
                k = t - warm + 1
                if checks and (k % check == 0 or k == nsteps):
                    mid = k == (nsteps // (2 * check)) * check or k == nsteps
                    dd = trajectory_drift(u, d.cpu().numpy(), box, n, V,
                                          oracle=mid and rank == 0 and not args.no_cpu)
                    dd["step"] = k
                    drift.append(dd)
        aff = len(u.affected_ids())
        stage_med = {k: statistics.median(x[k] for x in stages[warm:]) for k in stages[0]} if stages else None
        return u, d, ms, aff, pairs, redo, adj, cref, drift, stage_med, syncs

    u32, d32, ms32, aff, pairs, redo, adj32, cref, drift, ustages, usyncs = run("fp32", steps, checks=True)
    short = min(steps, 100)
    ms64, adj64 = run("fp64", short)[2:7:4]
    ms32na = run("fp32", short, adjoint=False)[2]
    eng = V.Engine()
    eng.set_stream(stream.cuda_stream)
    full = []
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.compute_device(d32.data_ptr(), n, PROBE, V.parse_periodic_box(box), precision="fp32")
        e1.record(stream)
        e1.synchronize()
        full.append(e0.elapsed_time(e1))
    eng.close()
    t32 = R.max(statistics.median(ms32))
    t32na = R.max(statistics.median(ms32na))
    t64 = R.max(statistics.median(ms64))
    a32 = R.max(statistics.median(adj32))
    a64 = R.max(statistics.median(adj64))
    tfull = R.max(statistics.median(full))
    gpu_ok = all(c["gpu_fp64"]["contacts_identical"] for c in drift)
    worst = max((c["gpu_fp64"]["rel_err_total_sas"] for c in drift), default=None)
    worst_v = max((c["gpu_fp64"]["rel_err_total_volume"] for c in drift), default=None)
    out = {
        "workload": f"periodic cube {n} balls, 0.033 balls/A^3, r 1.52, probe 1.4; per step 1% of the balls "
                    "moved by N(0, 0.05 A) per axis, then update_with_changed on the device, then the adjoint "
                    "of the total SAS",
        "steps": steps, "warmup": warm, "steps_fp64_and_adjoint_off_runs": short,
        "ms_per_update_fp32": t32, "ms_per_update_fp64": t64,
        "ms_per_update_fp32_adjoint_off": t32na,
        "ms_adjoint_total_sas_fp32": a32, "ms_adjoint_total_sas_fp64": a64,
        "ms_per_step_update_plus_adjoint_fp32": t32 + a32,
        "ms_per_update_fp32_p90": float(np.percentile(ms32, 90)),
        "ms_full_recompute_fp32": tfull, "speedup_vs_full_recompute": tfull / t32,
        "balls_per_s_fp32": replica_throughput(n, R.world, t32), "max_over_ranks": R.world,
        "affected_per_update": aff, "pairs_per_update": int(statistics.median(pairs)),
        "fp64_redo_pairs_per_update": int(statistics.median(redo)),
        "fp64_cell_refresh_per_update": int(statistics.median(cref)),
        "stages_ms_fp32_median": {k: round(v, 4) for k, v in ustages.items()} if ustages else None,
        "host_gaps_fp32": host_gaps(ustages, ustages["call"], int(statistics.median(usyncs))) if ustages else None,
        "drift_checks": drift,
        "drift_summary": {"checkpoints": len(drift), "contacts_identical_to_full_fp64_at_every_checkpoint": gpu_ok,
                          "max_rel_err_total_sas_vs_full_fp64": worst,
                          "max_rel_err_total_volume_vs_full_fp64": worst_v},
    }
    if rank == 0 and not args.no_cpu:
        out.update(updateable_cpu_check(balls, box, moves[:3], n, torch, V))
    return out


def updateable_cpu_check(balls, box, moves, n, torch, V):
    """The CPU oracle's UpdateableTessellation on the first steps (timed, all host cores),
    and the GPU FP32 handle replaying them: contact count and totals compared."""
    import oracle as O

    O.set_threads(0)
    O.set_faithful_grid_update(False)
    o = O.OracleUpdateable(False)
    b = balls.copy()
    o.init(b, PROBE, box)
    u = V.UpdateableTessellation(False, "fp32")
    u.init(balls, PROBE, box)
    times = []
    for ids, disp in moves:
        b[ids, :3] += disp
        t0 = time.perf_counter()
        o.update_with_changed(b, ids)
        times.append(time.perf_counter() - t0)
        u.update_with_changed(b, ids)
    so, sg = o.summary(), u.summary()
    rel = abs(sg.total_sas_area - so.total_sas_area) / so.total_sas_area
    relv = abs(sg.total_volume - so.total_volume) / so.total_volume
    same = (len(sg.id_a) == len(so.contacts_a) and np.array_equal(sg.id_a, so.contacts_a.astype(np.uint32))
            and np.array_equal(sg.id_b, so.contacts_b.astype(np.uint32)))
    O.set_faithful_grid_update(True)
    return {"cpu_oracle_ms_per_update": 1e3 * statistics.median(times), "cpu_cores": O.get_threads(),
            "cpu_sample": f"{len(times)} updates of the trajectory, median",
            "fp32_vs_oracle_after_updates": {"steps": len(moves), "contacts_identical": bool(same),
                                             "rel_err_total_sas": rel, "rel_err_total_volume": relv}}


def batched_leg(args, rank, torch, V, R):
    """Batched structures: --batch-count structures (4,096 by default), sizes log-uniform in
    [300, 20000], structure i from the lattice generator with seed 1000 + i, FP32+fixup (and
    FP64), in one batched call per step.  With N ranks the batch is split into N contiguous
    blocks of about equal ball counts (replicas.partition_weighted), one batched call per
    rank; throughput = the whole batch's balls / max-over-ranks time.  Per-structure SAS /
    volume error against the CPU oracle on a sample (rank 0)."""
    from voronota_ltr import workloads as W
    from voronota_ltr.replicas import partition_weighted

    sizes_all = W.batch_sizes(args.batch_count)
    lo, hi = partition_weighted(sizes_all, R.world, rank)
    sizes = sizes_all[lo:hi]
    structs = [W.lattice_balls(int(n), 1000 + lo + i) for i, n in enumerate(sizes)]
    balls = np.concatenate(structs) if structs else np.zeros((0, 4))
    off = np.zeros(len(sizes) + 1, np.uint64)
    off[1:] = np.cumsum(sizes)
    d = torch.from_numpy(balls).cuda()
    stream = torch.cuda.current_stream()
    eng = V.Engine()
    eng.set_stream(stream.cuda_stream)
    eng.set_timing(True)

    # autotune on the first 256 structures (a sample of the size distribution), untimed
    ks = min(256, len(sizes))
    tuning = eng.autotune_device(d.data_ptr(), int(off[ks]), PROBE, precision="fp32", offsets=off[:ks + 1])

    def timed(precision, reps, warm):
        for _ in range(warm):
            eng.compute_batch_device(d.data_ptr(), off, PROBE, precision)
        ms = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.compute_batch_device(d.data_ptr(), off, PROBE, precision)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    t64 = R.max(timed("fp64", 1, 0))
    t32 = R.max(timed("fp32", 3, 1))
    stages = eng.stage_times()
    st = eng.stats()
    total_balls = int(sizes_all.sum())
    out = {"workload": f"{len(sizes_all)} structures, sizes log-uniform in [300, 20000] ({total_balls} balls), "
                       "lattice generator seed 1000+i, probe 1.4, one batched call per rank",
           "balls": total_balls, "ranks": R.world, "structures_this_rank": [int(lo), int(hi)],
           "ms_fp32": t32, "balls_per_s_fp32": total_balls / (t32 * 1e-3),
           "ms_fp64": t64, "balls_per_s_fp64": total_balls / (t64 * 1e-3),
           "speedup_vs_fp64": t64 / t32, "max_over_ranks": R.world, "autotuned": tuning,
           "pairs": int(st.num_pairs), "fp64_redo_pairs": int(st.num_fp64_redo),
           "kernel_launches_per_call": int(st.num_kernel_launches)}
    out["host_gaps"] = host_gaps(stages, t32, 4)
    if rank == 0 and not args.no_cpu and len(sizes):
        import oracle as O

        O.set_threads(0)
        r = eng.download_batch()
        rng = np.random.default_rng(0)
        errs = []
        for s in rng.choice(len(sizes), min(16, len(sizes)), replace=False):
            o = O.compute(structs[s], PROBE)
            g = r.structure(int(s))
            errs.append((abs(g.total_sas_area - o.total_sas_area) / o.total_sas_area,
                         abs(g.total_volume - o.total_volume) / o.total_volume))
        errs = np.array(errs)
        out["fp32_vs_oracle_sample"] = {"structures": len(errs), "max_rel_err_sas": float(errs[:, 0].max()),
                                        "max_rel_err_volume": float(errs[:, 1].max()),
                                        "median_rel_err_sas": float(np.median(errs[:, 0]))}
    eng.close()
    return out


def host_gaps(stages, call_ms, syncs):
    """Where a call's device time goes: the stages' CUDA-event times, their sum, and the
    rest of the call (the device idle while the host reads a count back and sizes the next
    buffers), from the engine's stage events; `syncs` = the call's host reads of device
    counts (each one drains the stream)."""
    inner = {k: v for k, v in stages.items() if k != "call"}
    ssum = sum(inner.values())
    return {"call_ms": round(call_ms, 4), "stage_sum_ms": round(ssum, 4),
            "gap_ms": round(call_ms - ssum, 4), "gap_frac": round((call_ms - ssum) / call_ms, 4) if call_ms else None,
            "host_syncs_per_call": syncs}


def contacts_only_leg(args, rank, torch, V, R, balls):
    """compute_contacts_only on the main structure with groups 0 for x < 0 and 1
    otherwise (inter-group contacts only), FP32+fixup and FP64, device-timed like the
    headline, beside compute_tessellation with the same groups; rank 0 checks the
    inter-group pair sets bit for bit and the areas against the CPU oracle."""
    from voronota_ltr import workloads as W

    n = balls.shape[0]
    groups = W.x_sign_groups(balls)
    dg = torch.from_numpy(groups).cuda()
    d = torch.from_numpy(balls).cuda()
    stream = torch.cuda.current_stream()
    eng = V.Engine()
    eng.set_stream(stream.cuda_stream)

    def timed(precision, contacts_only, reps=7, grouped=True):
        ts = []
        for k in range(reps + 2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.compute_device(d.data_ptr(), n, PROBE, None, dg.data_ptr() if grouped else 0, n if grouped else 0,
                               precision=precision, contacts_only=contacts_only)
            e1.record(stream)
            e1.synchronize()
            if k >= 2:
                ts.append(e0.elapsed_time(e1))
        return R.max(statistics.median(ts))

    out = {"workload": f"lattice {n} balls, probe 1.4, groups 0 for x < 0 and 1 otherwise"}
    res = {}
    for prec in ("fp32", "fp64"):
        tc = timed(prec, True)
        res[prec] = eng.download()
        tf = timed(prec, False)
        tc0 = timed(prec, True, grouped=False)
        tf0 = timed(prec, False, grouped=False)
        out[prec] = {"ms_contacts_only": tc, "ms_tessellation_same_groups": tf,
                     "balls_per_s_contacts_only": R.world * n / (tc * 1e-3),
                     "contacts_only_over_tessellation": tc / tf, "contacts": int(len(res[prec].id_a)),
                     "no_groups": {"ms_contacts_only": tc0, "ms_tessellation": tf0,
                                   "contacts_only_over_tessellation": tc0 / tf0}}
    eng.close()
    if rank == 0 and not args.no_cpu:
        import oracle as O

        O.set_threads(0)
        o = O.compute(balls, PROBE, groups=groups, contacts_only=True)
        for prec in ("fp32", "fp64"):
            r = res[prec]
            same = (len(r.id_a) == len(o.contacts_a) and np.array_equal(r.id_a, o.contacts_a.astype(np.uint32))
                    and np.array_equal(r.id_b, o.contacts_b.astype(np.uint32)))
            out[prec]["pair_set_matches_oracle"] = bool(same)
            if same:
                out[prec]["max_abs_dA_vs_oracle"] = float(np.abs(r.area - o.contacts_area).max(initial=0.0))
    return out


def _pair_keys(a, b, n):
    return np.asarray(a, np.int64) * n + np.asarray(b, np.int64)


def _loss_fn(n, w, key_sorted, u_sorted):
    """L = sum w SAS + sum u area, u attached to the contact's ball pair (contacts absent
    from the reference list weigh 0)."""
    def loss(cell_index, cell_sas, ida, idb, area):
        k = _pair_keys(ida, idb, n)
        pos = np.clip(np.searchsorted(key_sorted, k), 0, len(key_sorted) - 1)
        uu = np.where(key_sorted[pos] == k, u_sorted[pos], 0.0)
        return float(np.dot(w[cell_index.astype(np.int64)], cell_sas)) + float(np.dot(uu, area))
    return loss


def grad_leg(args, rank, torch, V, R):
    """The differentiation workload: a 20,000-ball lattice structure, L = sum_i w_i SAS_i +
    sum_ab u_ab area_ab with w ~ U(0,1), u ~ N(0,1) (seeded), and the same with the volume
    term sum_i v_i V_i (v ~ U(0,1)).  Forward + hand-written adjoint timed on the device
    (FP32+fixup and FP64 forwards).  The gradient is checked at 256 random coordinates
    (x, y, z, r) against central differences (h = 1e-4 A, f64; h = 1e-5 where a +-h step
    crosses a contour's change of topology) of the GPU FP64 forward, and (rank 0) of the CPU
    oracle, each oracle difference taken on the sub-structure that determines it
    (oracle.finite_difference_local), for both losses and both forwards."""
    n = args.grad_n
    balls = workload(n, 7 + rank)
    rng = np.random.default_rng(20 + rank)
    w = rng.uniform(0.0, 1.0, n)
    ref = V.compute_tessellation_result(balls, PROBE, precision="fp64")
    u = rng.normal(0.0, 1.0, len(ref.id_a))
    v = np.random.default_rng(40 + rank).uniform(0.0, 1.0, n)
    stream = torch.cuda.current_stream()
    eng = V.Engine()
    eng.set_stream(stream.cuda_stream)
    d = torch.from_numpy(balls).cuda()
    dw = torch.from_numpy(w).cuda()
    du = torch.from_numpy(u).cuda()
    dv = torch.from_numpy(v).cuda()
    dg = torch.empty((n, 4), dtype=torch.float64, device="cuda")

    def timed(precision, with_v, reps=7):
        fwd, bwd = [], []
        for k in range(reps + 2):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            eng.compute_device(d.data_ptr(), n, PROBE, precision=precision)
            e1.record(stream)
            eng.grad_device(dw.data_ptr(), du.data_ptr(), dg.data_ptr(), dv.data_ptr() if with_v else 0)
            e2.record(stream)
            e2.synchronize()
            if k >= 2:
                fwd.append(e0.elapsed_time(e1))
                bwd.append(e1.elapsed_time(e2))
        return R.max(statistics.median(fwd)), R.max(statistics.median(bwd)), dg.cpu().numpy().copy()

    f64, b64, g64 = timed("fp64", False)
    f32p, b32p, _ = timed("fp32", False)  # the forward without kept contours
    eng.set_keep_contours(True)  # as the autograd front end does: the adjoint reads them
    f32, b32, g32 = timed("fp32", False)
    f64v, b64v, g64v = timed("fp64", True)
    f32v, b32v, g32v = timed("fp32", True)
    eng.close()
    key = _pair_keys(ref.id_a, ref.id_b, n)
    order = np.argsort(key)
    loss = _loss_fn(n, w, key[order], u[order])

    def l_gpu(b):
        r = V.compute_tessellation_result(b, PROBE, precision="fp64")
        return loss(r.cell_index, r.cell_sas_area, r.id_a, r.id_b, r.area)

    def fd(lf, i, c, h):
        bp, bm = balls.copy(), balls.copy()
        bp[i, c] += h
        bm[i, c] -= h
        return (lf(bp) - lf(bm)) / (2 * h)

    def rel(g, f):
        return abs(g - f) / (1 + abs(f))

    def summary(errs):
        errs = np.array(errs)
        return {"coordinates": len(errs), "h": 1e-4, "max_rel_err": float(errs.max()),
                "median_rel_err": float(np.median(errs)), "within_1e-5": int((errs <= 1e-5).sum())}

    crng = np.random.default_rng(30 + rank)
    coords = list(zip(crng.choice(n, 256, replace=False).tolist(), crng.integers(0, 4, 256).tolist()))
    errs = []
    for i, c in coords:
        f = fd(l_gpu, i, c, 1e-4)
        e = rel(g64[i, c], f)
        if e > 1e-5:
            e = min(e, rel(g64[i, c], fd(l_gpu, i, c, 1e-5)))
        errs.append(e)
    out = {"workload": f"lattice {n} balls, probe 1.4; L = sum w SAS + sum u area, w ~ U(0,1), u ~ N(0,1); "
                       "with volumes: + sum v V, v ~ U(0,1)",
           "forward_ms_fp32_plain": f32p, "adjoint_ms_after_plain_fp32": b32p,
           "forward_ms_fp32": f32, "adjoint_ms_after_fp32": b32,
           "forward_plus_adjoint_over_forward_fp32": (f32 + b32) / f32p,
           "note": "FP32 forward keeping its contours for the adjoint (autograd's form); the ratios "
                   "divide by the plain forward",
           "forward_ms_fp64": f64, "adjoint_ms_after_fp64": b64,
           "with_volume_term": {"forward_ms_fp32": f32v, "adjoint_ms_after_fp32": b32v,
                                "forward_plus_adjoint_over_forward_fp32": (f32v + b32v) / f32p,
                                "forward_ms_fp64": f64v, "adjoint_ms_after_fp64": b64v},
           "fd_check_gpu_fp64_forward": summary(errs),
           "fp32_vs_fp64_forward_grad_max_abs_diff_xyz": float(np.abs(g32[:, :3] - g64[:, :3]).max())}
    if rank == 0 and not args.no_cpu:
        import oracle as O

        O.set_threads(0)
        o = O.compute(balls, PROBE)
        ko = _pair_keys(o.contacts_a, o.contacts_b, n)
        # u attached to the oracle's contacts by ball pair (the pair sets are identical)
        pos = np.clip(np.searchsorted(key[order], ko), 0, len(key) - 1)
        uo = np.where(key[order][pos] == ko, u[order][pos], 0.0)
        upair = O.loss_weights_by_pair(o.contacts_a, o.contacts_b, uo, n)
        checks = {"sas_area": (None, {"fp64": g64, "fp32": g32}),
                  "sas_area_volume": (v, {"fp64": g64v, "fp32": g32v})}
        for name, (vv, grads) in checks.items():
            errs = {k: [] for k in grads}
            for i, c in coords:
                f = O.finite_difference_local(balls, PROBE, i, c, 1e-4, w, vv, upair)
                f2 = None
                for k, g in grads.items():
                    e = rel(g[i, c], f)
                    if e > 1e-5:
                        if f2 is None:
                            f2 = O.finite_difference_local(balls, PROBE, i, c, 1e-5, w, vv, upair)
                        e = min(e, rel(g[i, c], f2))
                    errs[k].append(e)
            out[f"fd_check_oracle_{name}"] = {f"adjoint_after_{k}": summary(e) for k, e in errs.items()}
    return out


def network_leg(args, rank, torch, V, R, balls):
    """compute_tessellation with with_cell_vertices on the main structure: the device time
    of the call with and without the network (CUDA events, inputs resident), and on rank 0
    the network's ids checked bit for bit against the CPU oracle's, positions and lengths
    within 1e-9 (1 + |x|)."""
    n = balls.shape[0]
    stream = torch.cuda.current_stream()
    eng = V.Engine()
    eng.set_stream(stream.cuda_stream)
    d = torch.from_numpy(balls).cuda()

    def timed(on, reps=5):
        eng.set_network(on)
        ts = []
        for k in range(reps + 2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.compute_device(d.data_ptr(), n, PROBE, precision="fp32")
            e1.record(stream)
            e1.synchronize()
            if k >= 2:
                ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    base = R.max(timed(False))
    with_net = R.max(timed(True))
    r = eng.download()
    eng.set_network(False)
    eng.close()
    out = {"ms_without_network": round(base, 3), "ms_with_network": round(with_net, 3),
           "vertices": int(len(r.vertex_ids)), "edges": int(len(r.edge_ids))}
    if rank == 0:
        import oracle as O

        o = O.compute(balls, PROBE, with_cell_vertices=True)
        null32 = 0xFFFFFFFF

        def oid(x):
            y = x.astype(np.int64)
            y[x == O.NET_NULL] = null32
            return y

        ok = (r.vertex_ids.shape == o.vertex_ids.shape and r.edge_ids.shape == o.edge_ids.shape
              and np.array_equal(r.vertex_ids.astype(np.int64), oid(o.vertex_ids))
              and np.array_equal(r.edge_ids.astype(np.int64), oid(o.edge_ids)))
        out["ids_match_oracle"] = bool(ok)
        if ok:
            out["max_xyz_err"] = float(np.abs(r.vertex_xyz - o.vertex_xyz).max(initial=0.0))
            out["max_len_rel_err"] = float((np.abs(r.edge_length - o.edge_length) / (1 + np.abs(o.edge_length)))
                                           .max(initial=0.0))
    return out


def solvent_leg(args, rank, torch, V, R):
    """compute_solvent_spheres on a lattice structure (depth 2, probe 1.4): the whole call
    through the C ABI from host arrays (two tessellations and the sampling between them),
    against the CPU oracle's time and output on rank 0."""
    n = args.solvent_n
    balls = workload(n, 11 + rank)
    for _ in range(2):
        V.compute_solvent_spheres_result(balls, PROBE, precision="fp32")
    ts = {}
    res = {}
    for prec in ("fp32", "fp64"):
        t = []
        for _ in range(5):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res[prec] = V.compute_solvent_spheres_result(balls, PROBE, precision=prec)
            t.append(time.perf_counter() - t0)
        ts[prec] = R.max(1e3 * statistics.median(t))
    out = {"workload": f"lattice {n} balls, probe 1.4, subdivision depth 2 (162 directions)",
           "spheres": len(res["fp32"]), "ms_fp32": round(ts["fp32"], 3), "ms_fp64": round(ts["fp64"], 3)}
    if rank == 0:
        import oracle as O

        t0 = time.perf_counter()
        o = O.solvent_spheres(balls, PROBE)
        out["cpu_oracle_ms"] = round(1e3 * (time.perf_counter() - t0), 1)
        out["cpu_cores"] = O.get_threads()
        g = res["fp64"]
        out["fp64_positions_parents_match_oracle"] = bool(len(g) == len(o.weight) and np.array_equal(g.xyz, o.xyz)
                                                          and np.array_equal(g.parent.astype(np.uint64), o.parent))
        g32 = res["fp32"]
        if len(g32) == len(o.weight) and len(g) == len(o.weight):
            out["fp64_weight_max_rel_err"] = float((np.abs(g.weight - o.weight) / (1 + np.abs(o.weight))).max(initial=0))
            out["fp32_total_weight_rel_err"] = float(abs(g32.weight.sum() - o.weight.sum()) / o.weight.sum())
            out["fp32_positions_match_oracle"] = bool(np.array_equal(g32.xyz, o.xyz))
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle as O

    balls = workload(args.n, 0)
    O.set_threads(0)
    cores = O.get_threads()
    for _ in range(args.warmup):
        O.compute(balls, PROBE)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.compute(balls, PROBE)
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    value = args.n / med
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": med * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(args.n, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full tessellations of the {args.n}-ball structure, median time"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "CPU oracle (C++ restatement of the reference's Rust code, std::thread over all host "
                "cores); the Rust reference cannot be compiled in this image",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    from voronota_ltr.replicas import Ranks, replica_throughput

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    R = Ranks("nccl")
    world, rank = R.world, R.rank
    barrier, max_over_ranks = R.barrier, R.max

    import voronota_ltr as V

    balls = workload(args.n, rank)
    d_xyzr = torch.from_numpy(balls).cuda()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    eng = V.Engine(local)
    eng.set_stream(stream.cuda_stream)
    if args.tuning:
        w, c, ch = args.tuning.split(",")
        eng.set_tuning(int(w), float(c), int(ch))
        tuning = eng.tuning()
    else:
        tuning = eng.autotune_device(d_xyzr.data_ptr(), args.n, PROBE, precision="fp32")  # untimed set-up
    eng.set_timing(True)

    def device_leg(precision, steps, warmup, sample_clocks):
        for _ in range(warmup):
            eng.compute_device(d_xyzr.data_ptr(), args.n, PROBE, precision=precision)
        barrier()
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
        step_ms, contact_ms, launches = [], [], 0
        t0 = time.perf_counter()
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.compute_device(d_xyzr.data_ptr(), args.n, PROBE, precision=precision)
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            contact_ms.append(eng.stage_times()["contact"])
            launches += int(eng.stats().num_kernel_launches)
        barrier()
        wall = time.perf_counter() - t0
        clocks = sampler.stop() if sampler else None
        st = eng.stats()
        return {"mean_ms": sum(step_ms) / len(step_ms), "contact_ms": sum(contact_ms) / len(contact_ms),
                "last_ms": step_ms[-1],
                "launches": launches, "wall_s": wall, "clocks": clocks, "stats": st,
                "stages": eng.stage_times()}

    fp32 = device_leg("fp32", args.steps, args.warmup, True)
    mean_ms = max_over_ranks(fp32["mean_ms"])
    value = replica_throughput(args.n, world, mean_ms)

    fp64 = None
    if not args.no_fp64:
        fp64 = device_leg("fp64", max(3, args.steps // 2), max(1, args.warmup // 2), False)
        fp64_ms = max_over_ranks(fp64["mean_ms"])

    # e2e through the public API from pinned host memory
    pinned = torch.from_numpy(balls).pin_memory()
    host = pinned.numpy()
    for _ in range(max(1, args.warmup)):
        V.compute_tessellation_result(host, PROBE, precision="fp32")
    barrier()
    e2e_t = []
    res = None
    for _ in range(args.steps):
        t0 = time.perf_counter()
        res = V.compute_tessellation_result(host, PROBE, precision="fp32")
        e2e_t.append(time.perf_counter() - t0)
    barrier()
    # median over the steps: the host side of a shared machine shows rare stalls of a few
    # hundred ms (a 197 ms step among 5.9 ms ones) that a mean would turn into the number
    e2e_ms = max_over_ranks(1e3 * statistics.median(e2e_t))
    C, M = len(res.id_a), len(res.cell_index)
    d2h = C * (4 + 4 + 8 + 8 + 1) + M * (4 + 8 + 8) + 3 * 8
    h2d = balls.nbytes

    st = fp32["stats"]
    P, E = int(st.num_pairs), int(st.num_entries)
    alg_bytes = 58 * P + 20 * E + 40 * args.n
    peak, peak_kind = peaks()
    achieved = alg_bytes / (fp32["contact_ms"] * 1e-3) / 1e9
    traffic = profiled_traffic()

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline(balls)

    con = None if args.no_contacts_only else contacts_only_leg(args, rank, torch, V, R, balls)
    upd = None if args.no_upd else updateable_leg(args, rank, torch, V, R)
    bat = None if args.no_batch else batched_leg(args, rank, torch, V, R)
    grd = None if args.no_grad else grad_leg(args, rank, torch, V, R)
    net = None if args.no_network else network_leg(args, rank, torch, V, R, balls)
    sol = None if args.no_solvent else solvent_leg(args, rank, torch, V, R)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (f64 band fixups, f64 reductions)", "data": "synthetic",
            "config": headline_config(args.n, world),
            "e2e": {"value": world * args.n / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step_median": round(e2e_ms, 3),
                    "ms_per_step_mean": round(1e3 * sum(e2e_t) / len(e2e_t), 3),
                    "ms_per_step_min_median_max": [round(1e3 * x, 3) for x in
                                                   (min(e2e_t), statistics.median(e2e_t), max(e2e_t))]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": "k_contact32",
                         "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": fp32["contact_ms"],
                         "peak_source": peak_kind},
            "issue_roofline": issue_roofline(fp32["contact_ms"], (fp32["clocks"] or {}).get("sm_mhz"), args.n),
            "cpu_baseline": cpu,
            "clocks": fp32["clocks"],
            "gpu_launches": fp32["launches"],
            "fp64_value": (world * args.n / (fp64_ms * 1e-3)) if fp64 else None,
            "speedup_vs_fp64": (fp64_ms / mean_ms) if fp64 else None,
            "counts": {"pairs": P, "neighbor_entries": E, "contacts": int(st.num_contacts),
                       "cells": int(st.num_cells), "fp64_redo_pairs": int(st.num_fp64_redo),
                       "serial_pairs": int(st.num_serial)},
            "stages_ms_fp32": {k: round(v, 4) for k, v in fp32["stages"].items()},
            "stages_ms_fp64": {k: round(v, 4) for k, v in fp64["stages"].items()} if fp64 else None,
            "wall_s_timed_region": fp32["wall_s"],
            "autotuned": tuning,
            "host_gaps_fp32": host_gaps(fp32["stages"], fp32["last_ms"], 3),
            "contacts_only_groups": con,
            "updateable": upd,
            "batched": bat,
            "differentiation": grd,
            "network": net,
            "solvent_spheres": sol,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    R.close()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
