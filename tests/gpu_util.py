"""Helpers for comparing GPU results with the oracle."""
import numpy as np

import oracle as O
import voronota_ltr as V


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def gpu(balls, probe, periodic_box=None, groups=None, precision="fp64", contacts_only=False):
    if contacts_only:
        return V.compute_contacts_only_result(balls, probe, periodic_box, groups, precision)
    return V.compute_tessellation_result(balls, probe, periodic_box, groups, precision)


def compare(g, o, precision, contacts_only=False, ordered=True, total_rel=None, total_abs=None):
    """Pair sets and central bits bit-exact; values within the precision's tolerance.

    FP64: |d| <= 1e-9 (1 + |x|) everywhere (only the summation order of the warp
    reductions and CUDA's vs glibc's transcendentals differ).
    FP32: per-contact |dA| <= 1e-3 A^2 and |d arc| <= 1e-3 A; per-cell |d| <= 1e-2 or
    1e-6 relative, whichever is larger;
    total SAS area and total volume relative error <= 1e-6, with an absolute floor of
    1e-4 (A^2, A^3) for tiny totals: a 17-ball periodic ring with 5 A^2 of SAS carries
    ~1e-5 A^2 of FP32 rounding in its nearly cancelling solid-angle sums (the FP32 kernel
    runs on such small inputs only when forced: fp32_engine below).  `total_rel`
    overrides the relative bound on the totals; `total_abs` = (SAS, volume) absolute
    allowances that replace the floor.
    """
    ga, gb = g.id_a.astype(np.int64), g.id_b.astype(np.int64)
    oa, ob = o.contacts_a.astype(np.int64), o.contacts_b.astype(np.int64)
    assert len(ga) == len(oa), f"contact count {len(ga)} vs oracle {len(oa)}"
    if ordered:
        go = np.arange(len(ga))
        oo = np.arange(len(oa))
    else:
        go = np.lexsort((gb, ga))
        oo = np.lexsort((ob, oa))
    assert np.array_equal(ga[go], oa[oo]), "id_a differ"
    assert np.array_equal(gb[go], ob[oo]), "id_b differ"
    mism = np.nonzero(g.central[go] != o.contacts_central[oo])[0]
    assert len(mism) == 0, f"central bits differ at {mism[:10]}"
    if precision == "fp64":
        tol_area = 1e-9 * (1 + np.abs(o.contacts_area[oo]))
        tol_arc = 1e-9 * (1 + np.abs(o.contacts_arc[oo]))
    else:
        tol_area = tol_arc = 1e-3
    da = np.abs(g.area[go] - o.contacts_area[oo])
    dr = np.abs(g.arc_length[go] - o.contacts_arc[oo])
    assert np.all(da <= tol_area), f"max |dA| {da.max()}"
    assert np.all(dr <= tol_arc), f"max |d arc| {dr.max()}"
    if contacts_only:
        return {"max_dA": float(da.max(initial=0))}
    assert np.array_equal(g.cell_index.astype(np.int64), o.cells_index.astype(np.int64)), "cell index sets differ"
    if precision == "fp64":
        ts = 1e-9 * (1 + np.abs(o.cells_sas))
        tv = 1e-9 * (1 + np.abs(o.cells_vol))
    else:  # FP32 cells: 1e-2 absolute, or 1e-6 relative for a big ball (a 15 A ball holds 15,000 A^3)
        ts = np.maximum(1e-2, 1e-6 * np.abs(o.cells_sas))
        tv = np.maximum(1e-2, 1e-6 * np.abs(o.cells_vol))
    ds = np.abs(g.cell_sas_area - o.cells_sas)
    dv = np.abs(g.cell_volume - o.cells_vol)
    assert np.all(ds <= ts), f"max |d sas| {ds.max()}"
    # exposure (sas_area > 0: what compute_solvent_spheres samples) decided as the oracle
    expo = np.nonzero((g.cell_sas_area > 0) != (o.cells_sas > 0))[0]
    assert len(expo) == 0, f"exposure differs at cells {g.cell_index[expo[:10]]}"
    assert np.all(dv <= tv), f"max |d vol| {dv.max()}"
    rs = abs(g.total_sas_area - o.total_sas_area) / max(abs(o.total_sas_area), 1e-300)
    rv = abs(g.total_volume - o.total_volume) / max(abs(o.total_volume), 1e-300)
    lim = total_rel if total_rel is not None else (1e-11 if precision == "fp64" else 1e-6)
    floor = 0.0 if precision == "fp64" else 1e-4
    fs, fv = total_abs if total_abs is not None else (floor, floor)
    assert rs <= lim or abs(g.total_sas_area - o.total_sas_area) <= fs, f"total SAS rel err {rs}"
    assert rv <= lim or abs(g.total_volume - o.total_volume) <= fv, f"total volume rel err {rv}"
    return {"max_dA": float(da.max(initial=0)), "rel_sas": rs, "rel_vol": rv}


def engine_run(balls, probe, precision="fp32", periodic_box=None, groups=None, contacts_only=False,
               fp32_min_pairs=None):
    """One call through an Engine (host inputs); returns (Result, stats).  fp32_min_pairs=0
    forces the FP32 contact kernel on inputs of any size."""
    e = V.Engine()
    try:
        if fp32_min_pairs is not None:
            e.set_fp32_min_pairs(fp32_min_pairs)
        e.compute_host(balls, probe, periodic_box, groups, precision, contacts_only)
        st = e.stats()
        return e.download(), st
    finally:
        e.close()
