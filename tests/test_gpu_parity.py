"""GPU parity: the CUDA path through the C ABI against the CPU oracle and the reference
goldens.  Pair sets and central bits must match the oracle bit for bit; values within
the tolerances in gpu_util.compare (FP64: 1e-9 relative; FP32+fixup: |dA| <= 1e-3 A^2,
total SAS / volume relative error <= 1e-6)."""
import numpy as np
import pytest

import oracle as O
import voronota_ltr as V
from common import (CENTRAL_POINTS, RING_17, THREE_LINE, central_golden, contact_lookup, goldens, load_balls,
                    sunflower)
from gpu_util import compare, engine_run, gpu
from voronota_ltr import workloads as W

pytestmark = pytest.mark.gpu
G = goldens()
PRECISIONS = ["fp64", "fp32"]


@pytest.mark.parametrize("prec", PRECISIONS)
def test_cs_1x1_golden_and_oracle(prec):
    g = G["cs_1x1"]
    balls = load_balls("cs_1x1")
    r = gpu(balls, g["probe"], precision=prec)
    assert len(r.id_a) == g["contacts"] and len(r.cell_index) == g["cells"]
    assert abs(r.total_contact_area - g["total_contact_area"]) < g["tol"]
    assert abs(r.total_sas_area - g["total_sas_area"]) < g["tol"]
    assert abs(r.total_volume - g["total_volume"]) < g["tol"]
    k = contact_lookup(r.id_a, r.id_b, 0, 1)
    assert abs(r.area[k] - g["contact_0_1_area"]) < g["contact_tol"]
    compare(r, O.compute(balls, g["probe"]), prec)


@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("form", ["corners", "vectors"])
def test_cs_1x1_periodic(prec, form):
    g = G["cs_1x1_periodic"]
    (x1, y1, z1), (x2, y2, z2) = g["corners"]
    box = ({"corners": g["corners"]} if form == "corners"
           else {"vectors": [(x2 - x1, 0, 0), (0, y2 - y1, 0), (0, 0, z2 - z1)]})
    balls = load_balls("cs_1x1")
    r = gpu(balls, g["probe"], periodic_box=box, precision=prec)
    assert len(r.id_a) == g["contacts"] and len(r.cell_index) == g["cells"]
    assert abs(r.total_contact_area - g["total_contact_area"]) < g["tol"]
    assert abs(r.total_sas_area - g["total_sas_area"]) < g["tol"]
    assert abs(r.total_volume - g["total_volume"]) < g["tol"]
    compare(r, O.compute(balls, g["probe"], periodic_box=box), prec)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_2zsk(prec):
    balls = load_balls("2zsk")
    r = gpu(balls, 1.4, precision=prec)
    assert (len(r.id_a), len(r.cell_index)) == (23855, 3545)
    compare(r, O.compute(balls, 1.4), prec)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_3dlb(prec):
    balls = load_balls("3dlb")
    compare(gpu(balls, 1.4, precision=prec), O.compute(balls, 1.4), prec)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_ring17_basic_and_periodic(prec):
    g = G["ring17"]
    r = gpu(RING_17, g["probe"], precision=prec)
    assert len(r.id_a) == g["contacts"] and len(r.cell_index) == g["cells"]
    cells = dict(zip(r.cell_index.tolist(), zip(r.cell_sas_area, r.cell_volume)))
    assert abs(cells[0][0] - g["cell0_sas"]) < g["cell_tol"]
    assert abs(cells[1][1] - g["cell1_vol"]) < g["cell_tol"]
    compare(r, O.compute(RING_17, g["probe"]), prec)
    gp = G["ring17_periodic"]
    box = {"corners": gp["corners"]}
    r = gpu(RING_17, gp["probe"], periodic_box=box, precision=prec)
    k = contact_lookup(r.id_a, r.id_b, 0, 0)
    assert k is not None and abs(r.area[k] - gp["self_contact_0_0_area"]) < gp["self_tol"]
    compare(r, O.compute(RING_17, gp["probe"], periodic_box=box), prec)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_centrality_golden(prec):
    balls = [p + [1.5] for p in CENTRAL_POINTS]
    r = gpu(balls, 1.4, precision=prec)
    got = {(int(a), int(b)): bool(c) for a, b, c in zip(r.id_a, r.id_b, r.central)}
    for a, b, c in central_golden():
        assert got[(min(a, b), max(a, b))] == bool(c)
    compare(r, O.compute(balls, 1.4), prec)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_two_body_groups_contacts_only(prec):
    g = G["two_body_groups"]
    balls = [(0.0, 0.0, 0.0, 1.5), (1.0, 0.0, 0.0, 1.5), (4.0, 0.0, 0.0, 2.0), (5.0, 0.0, 0.0, 2.0)]
    c = V.compute_contacts_only(balls, g["probe"], groups=[0, 0, 1, 1], precision=prec)
    assert len(c) == 1 and (c[0]["id_a"], c[0]["id_b"]) == (1, 2)
    assert abs(c[0]["area"] - g["area"]) < (g["tol"] if prec == "fp64" else 1e-3)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_lattice_2k_config(prec):
    balls = W.lattice_balls(2000, 0)
    compare(gpu(balls, 1.4, precision=prec), O.compute(balls, 1.4), prec)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_lattice_20k_groups_contacts_only(prec):
    balls = W.lattice_balls(20000, 3)
    groups = W.x_sign_groups(balls)
    r = gpu(balls, 1.4, groups=groups, precision=prec, contacts_only=True)
    compare(r, O.compute(balls, 1.4, groups=groups, contacts_only=True), prec, contacts_only=True)
    r = gpu(balls, 1.4, groups=groups, precision=prec)
    compare(r, O.compute(balls, 1.4, groups=groups), prec)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_periodic_random_box(prec):
    balls, side = W.periodic_box_balls(6000, 0.033, 1.52, seed=5)
    box = {"corners": [(0, 0, 0), (side, side, side)]}
    compare(gpu(balls, 1.4, periodic_box=box, precision=prec), O.compute(balls, 1.4, periodic_box=box), prec)
    r = gpu(balls, 1.4, periodic_box=box, precision=prec, contacts_only=True)
    compare(r, O.compute(balls, 1.4, periodic_box=box, contacts_only=True), prec, contacts_only=True)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_edge_cases(prec):
    for balls, probe in [
        (np.zeros((0, 4)), 1.4),
        ([(0.0, 0.0, 0.0, 1.0)], 0.5),
        ([(0, 0, 0, 1.0), (10, 0, 0, 1.0)], 0.5),
        ([(0, 0, 0, 1.0), (0, 0, 0, 0.5), (1, 0, 0, 1.0)], 0.5),  # hidden ball
        ([(0, 0, 0, 1.0), (0, 0, 0, 1.0), (1.5, 0, 0, 1.0)], 0.5),  # identical balls
        (THREE_LINE, 0.5),
        ([(0, 0, 0, 1.0), (0.5, 0, 0, 1.0), (1, 0, 0, 1.0)], 1.0),
        ([(0, 0, 0, 1), (0, 0, 1, 1), (0, 1, 0, 1), (0, 1, 1, 1), (1, 0, 0, 1), (1, 0, 1, 1), (1, 1, 0, 1),
          (1, 1, 1, 1)], 2.0),
    ]:
        r = gpu(balls, probe, precision=prec)
        compare(r, O.compute(balls, probe), prec)


SUNFLOWERS = [(sunflower(40), 0.5), (sunflower(40, rr=0.1, rho=3.3), 0.1), (sunflower(120, rr=0.12, rho=3.3), 0.5)]


@pytest.mark.parametrize("prec", PRECISIONS)
def test_serial_fallback_long_contours(prec):
    """Contours of 40 to 120 points (more than a warp holds) through the serial kernel."""
    for balls, probe in SUNFLOWERS:
        r, st = engine_run(balls, probe, prec)
        assert st.num_serial >= 1
        compare(r, O.compute(balls, probe), prec)
        r = gpu(balls, probe, precision=prec, contacts_only=True)
        compare(r, O.compute(balls, probe, contacts_only=True), prec, contacts_only=True)


def test_fp32_kernel_forced_on_small_inputs():
    """The FP32 kernel (forced below its default minimum of 2048 candidate pairs) on the
    small golden structures and edge cases: pair sets and central bits exact, values within
    the FP32 tolerances."""
    cases = [(RING_17, 1.0, None), (RING_17, G["ring17_periodic"]["probe"], {"corners": G["ring17_periodic"]["corners"]}),
             (load_balls("cs_1x1"), 2.0, None), (THREE_LINE, 0.5, None),
             ([(0, 0, 0, 1.0), (0, 0, 0, 0.5), (1, 0, 0, 1.0)], 0.5, None),
             ([(0, 0, 0, 1), (0, 0, 1, 1), (0, 1, 0, 1), (0, 1, 1, 1), (1, 0, 0, 1), (1, 0, 1, 1), (1, 1, 0, 1),
               (1, 1, 1, 1)], 2.0, None)]
    for balls, probe, box in cases:
        r, st = engine_run(balls, probe, "fp32", periodic_box=box, fp32_min_pairs=0)
        assert st.fp32_kernel == 1
        compare(r, O.compute(balls, probe, periodic_box=box), "fp32")
        r, st = engine_run(balls, probe, "fp32", periodic_box=box)
        assert st.fp32_kernel == 0  # below the default minimum: the FP64 kernel
        compare(r, O.compute(balls, probe, periodic_box=box), "fp64")


def test_fp32_kernel_coherent_rounding():
    """Forced FP32 on the rotationally symmetric sunflowers: every small ball's contact has
    the same geometry, so the FP32 rounding of the solid angles adds up coherently instead
    of averaging out; the totals then stay within 1e-5 relative (not 1e-6), while pair
    sets, central bits and per-contact values meet the FP32 tolerances."""
    for balls, probe in SUNFLOWERS:
        r, st = engine_run(balls, probe, "fp32", fp32_min_pairs=0)
        assert st.fp32_kernel == 1
        compare(r, O.compute(balls, probe), "fp32", total_rel=1e-5)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_long_neighbour_lists(prec):
    """A ball with 646 / 1190 neighbour candidates (beyond the 256 the warp sort holds):
    its list is sorted by the block sort, pairs and contacts as the oracle's."""
    from common import big_ball_in_lattice
    for balls in (big_ball_in_lattice(), big_ball_in_lattice(big_r=14.0, half=20.0)):
        compare(gpu(balls, 1.4, precision=prec), O.compute(balls, 1.4), prec)
        r = gpu(balls, 1.4, precision=prec, contacts_only=True)
        compare(r, O.compute(balls, 1.4, contacts_only=True), prec, contacts_only=True)
    balls = big_ball_in_lattice()
    box = {"corners": [(-16.0, -16.0, -16.0), (16.5, 16.5, 16.5)]}
    compare(gpu(balls, 1.4, periodic_box=box, precision=prec), O.compute(balls, 1.4, periodic_box=box), prec)
    groups = (balls[:, 0] > 0).astype(np.int32)
    compare(gpu(balls, 1.4, groups=groups, precision=prec), O.compute(balls, 1.4, groups=groups), prec)


def test_invalid_input_raises():
    """Bad balls are caught on the device before any other work; the host path's error
    names the first bad ball; the engine stays usable afterwards."""
    good = W.lattice_balls(500, 3)
    for bad in ([(0, 0, float("nan"), 1.0)], [(0, 0, 0, -1.0)], np.vstack([good, [[1.0, float("inf"), 0.0, 1.5]]])):
        with pytest.raises(V.VoronotaError) as ei:
            V.compute_tessellation(bad, 1.4)
        assert ei.value.status == V.VT_ERR_INVALID
        assert "ball %d" % (len(bad) - 1) in str(ei.value)
    import torch
    e = V.Engine()
    d = torch.from_numpy(np.vstack([good, [[0.0, 0.0, float("nan"), 1.0]]])).cuda()
    with pytest.raises(V.VoronotaError):
        e.compute_device(d.data_ptr(), len(good) + 1, 1.4)
    compare(V.compute_tessellation_result(good, 1.4, precision="fp64"), O.compute(good, 1.4), "fp64")
    e.close()


_ORACLE_100K = {}


def _oracle_100k(kind):
    """The oracle's results on the 100k-ball lattice (seed 0, probe 1.4), computed once:
    'full' = compute_tessellation, 'groups' = compute_contacts_only with groups 0 for
    x < 0 and 1 otherwise."""
    if kind not in _ORACLE_100K:
        balls = W.lattice_balls(100000, 0)
        if kind == "full":
            _ORACLE_100K[kind] = O.compute(balls, 1.4)
        else:
            _ORACLE_100K[kind] = O.compute(balls, 1.4, groups=W.x_sign_groups(balls), contacts_only=True)
    return _ORACLE_100K[kind]


def test_fp32_large_lattice_pair_set_and_totals():
    balls = W.lattice_balls(100000, 0)
    o = _oracle_100k("full")
    stats = compare(gpu(balls, 1.4, precision="fp32"), o, "fp32")
    assert stats["rel_sas"] <= 1e-6


def test_fp32_million_ball_lattice():
    """A 1,000,000-ball lattice through the FP32+fixup path: the pair set, central bits and
    cells of the oracle's, the totals within 1e-6 relative."""
    balls = W.lattice_balls(1_000_000, 5)
    O.set_threads(0)
    stats = compare(gpu(balls, 1.4, precision="fp32"), O.compute(balls, 1.4), "fp32")
    assert stats["rel_sas"] <= 1e-6 and stats["rel_vol"] <= 1e-6


def test_fp64_large_lattice():
    """The 100k-ball drop-in configuration through the plain FP64 path."""
    balls = W.lattice_balls(100000, 0)
    compare(gpu(balls, 1.4, precision="fp64"), _oracle_100k("full"), "fp64")


@pytest.mark.parametrize("prec", PRECISIONS)
def test_large_lattice_contacts_only_with_groups(prec):
    """compute_contacts_only on the 100k-ball lattice with groups 0 for x < 0 and 1
    otherwise: the inter-group contact set bit-exact, areas within the precision's
    tolerance, and each contact equal to the same pair's contact in the grouped full
    tessellation (contacts-only == full, tests/contacts_only.rs)."""
    balls = W.lattice_balls(100000, 0)
    groups = W.x_sign_groups(balls)
    r = gpu(balls, 1.4, groups=groups, precision=prec, contacts_only=True)
    compare(r, _oracle_100k("groups"), prec, contacts_only=True)
    g = balls[:, 0] < 0
    assert len(r.id_a) > 1000 and np.all(g[r.id_a.astype(np.int64)] != g[r.id_b.astype(np.int64)])
    full = gpu(balls, 1.4, groups=groups, precision=prec)
    assert np.array_equal(full.id_a, r.id_a) and np.array_equal(full.id_b, r.id_b)
    assert np.allclose(full.area, r.area, rtol=0, atol=1e-10 if prec == "fp64" else 1e-3)


def test_engine_device_path_matches_host_path():
    import torch
    balls = W.lattice_balls(5000, 11)
    e = V.Engine(0)
    e.compute_host(balls, 1.4, precision="fp64")
    h = e.download()
    t = torch.from_numpy(balls).cuda()
    e.compute_device(t.data_ptr(), len(balls), 1.4, precision="fp64")
    torch.cuda.synchronize()
    d = e.download()
    assert np.array_equal(h.id_a, d.id_a) and np.array_equal(h.area, d.area)
    assert np.array_equal(h.cell_sas_area, d.cell_sas_area)
    e.close()


def test_deterministic_reruns():
    balls = W.lattice_balls(8000, 2)
    for prec in PRECISIONS:
        r1 = gpu(balls, 1.4, precision=prec)
        r2 = gpu(balls, 1.4, precision=prec)
        assert np.array_equal(r1.area, r2.area) and np.array_equal(r1.cell_sas_area, r2.cell_sas_area)
        assert r1.total_sas_area == r2.total_sas_area
