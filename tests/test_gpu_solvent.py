"""compute_solvent_spheres on the GPU against the oracle and the reference's expectations
(src/solvent_spheres.rs:371-483, tests/test_python.py:199-293).

The sample points and the keep/drop test run in FP64 with the reference's arithmetic, so
the kept spheres (positions, parents, order) must equal the oracle's bit for bit in both
precisions; weights are stage-2 cell volumes: within 1e-9 (1 + |w|) in FP64, and within
the FP32 per-cell tolerance (1e-2) with the total within 1e-6 relative in FP32.
"""
import numpy as np
import pytest

import oracle as O
import voronota_ltr as V
from common import load_balls
from voronota_ltr import workloads as W

pytestmark = pytest.mark.gpu
PRECISIONS = ["fp64", "fp32"]


def check(balls, probe, prec, volume_probe=0.0, depth=2, periodic_box=None):
    g = V.compute_solvent_spheres_result(balls, probe, volume_probe, depth, periodic_box, prec)
    o = O.solvent_spheres(balls, probe, volume_probe, depth, periodic_box)
    assert len(g) == len(o.weight), (len(g), len(o.weight))
    assert np.array_equal(g.xyz, o.xyz), "positions differ"
    assert np.array_equal(g.parent.astype(np.uint64), o.parent), "parents differ"
    assert np.all(g.radius == probe)
    dw = np.abs(g.weight - o.weight)
    if prec == "fp64":
        assert np.all(dw <= 1e-9 * (1 + np.abs(o.weight))), f"max |dw| {dw.max(initial=0)}"
    else:
        assert np.all(dw <= 1e-2), f"max |dw| {dw.max(initial=0)}"
        tot = abs(o.weight.sum())
        assert abs(g.weight.sum() - o.weight.sum()) <= max(1e-6 * tot, 1e-4)
    return g


def test_reference_python_expectations():  # tests/test_python.py:208-293
    r = V.compute_solvent_spheres([(0, 0, 0, 1.5), (3, 0, 0, 1.5)], probe=1.4)
    assert isinstance(r, list) and len(r) > 0
    assert set(r[0]) == {"x", "y", "z", "radius", "weight", "parent_index"}
    r = V.compute_solvent_spheres([(0, 0, 0, 1.5)], probe=1.4, subdivision_depth=0)
    assert len(r) == 12
    for s in r:
        assert s["parent_index"] == 0 and abs(s["radius"] - 1.4) < 1e-12 and s["weight"] > 0
    assert V.compute_solvent_spheres([], probe=1.4) == []
    assert len(V.compute_solvent_spheres([(0, 0, 0, 1.5), (5, 0, 0, 1.5)], probe=1.4, volume_probe=0.5,
                                         subdivision_depth=0)) > 0
    r = V.compute_solvent_spheres(np.array([[0, 0, 0, 1.5], [5, 0, 0, 1.5]]), probe=1.4, subdivision_depth=0)
    assert len(r) == 24


@pytest.mark.parametrize("prec", PRECISIONS)
def test_reference_unit_cases(prec):  # solvent_spheres.rs:371-461
    g = check([(0.0, 0.0, 0.0, 1.5), (5.0, 0.0, 0.0, 1.5)], 1.4, prec, depth=0)
    assert len(g) == 24 and (g.parent == 0).sum() == 12 and abs(g.weight.sum() - 249.1) < 5.0  # C++ sihsolv
    g = check([(0.0, 0.0, 0.0, 1.5), (2.5, 0.0, 0.0, 1.5)], 1.4, prec, depth=0)
    assert 0 < len(g) < 24
    g = check([(0.0, 0.0, 0.0, 3.0), (2.5, 0.0, 0.0, 1.0)], 1.4, prec, depth=0)
    assert (g.parent == 0).sum() > (g.parent == 1).sum()


@pytest.mark.parametrize("prec", PRECISIONS)
def test_structures_against_oracle(prec):
    check(W.lattice_balls(2000, 5), 1.4, prec, depth=2)
    check(load_balls("2zsk"), 1.4, prec, depth=1)
    check(load_balls("cs_1x1"), 2.0, prec, volume_probe=0.5, depth=3)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_periodic_against_oracle(prec):
    balls, side = W.periodic_box_balls(1500, seed=4)
    check(balls, 1.4, prec, depth=1, periodic_box={"corners": [(0, 0, 0), (side, side, side)]})


def test_depths_and_clamp():
    balls = [(0.0, 0.0, 0.0, 1.5), (4.0, 0.0, 0.0, 1.2), (2.0, 3.0, 0.0, 1.4)]
    counts = [len(check(balls, 1.4, "fp64", depth=d)) for d in range(5)]
    assert counts == sorted(counts) and counts[0] > 0
    a = V.compute_solvent_spheres_result(balls, 1.4, subdivision_depth=9, precision="fp64")
    b = V.compute_solvent_spheres_result(balls, 1.4, subdivision_depth=4, precision="fp64")
    assert np.array_equal(a.xyz, b.xyz) and np.array_equal(a.weight, b.weight)
