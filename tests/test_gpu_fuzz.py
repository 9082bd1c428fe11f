"""Seeded random structures against the oracle.

Each case draws its kind (a random cloud with a wide spread of radii, the jittered
lattice, or a periodic box), its size (60 to 3000 balls, so the oracle takes well under a
second), its probe and, for some, random groups.  FP64 and FP32 (the FP32 kernel forced
on inputs of any size) are compared with the oracle by gpu_util.compare; contacts-only
as well; the tessellation network's vertex and edge ids must equal the oracle's.

The SAS area of an exposed ball is (4 pi - sum of solid angles) R^2, a small difference
of large terms when the ball is nearly buried, so the FP32 error of a total scales with
the sum of 4 pi R^2 over the exposed cells rather than with the total itself.  Where the
total is a small fraction of that sum (packings denser than a protein's: 0.8% in one
case here, against 11-13% on the lattice workloads), the FP32 totals are held to 1e-7 of it (of sum 4 pi R^3 / 3 for the volume)
instead of 1e-6 of the total.
"""
import numpy as np
import pytest

import oracle as O
import voronota_ltr as V
from gpu_util import compare, engine_run
from voronota_ltr import workloads as W

pytestmark = pytest.mark.gpu
NULL32 = 0xFFFFFFFF
CASES = 48


def fuzz_case(k):
    rng = np.random.default_rng(1000 + k)
    kind = ("cloud", "cloud", "lattice", "periodic")[k % 4]
    box = None
    if kind == "cloud":
        n = int(rng.integers(60, 1500))
        rmin = rng.uniform(0.4, 1.6)
        rmax = rmin + rng.uniform(0.0, 2.5)
        side = (n / rng.uniform(0.01, 0.05)) ** (1.0 / 3.0)
        balls = np.column_stack([rng.uniform(0.0, side, (n, 3)), rng.uniform(rmin, rmax, n)])
    elif kind == "lattice":
        balls = W.lattice_balls(int(rng.integers(200, 3000)), 2000 + k)
    else:
        balls, side = W.periodic_box_balls(int(rng.integers(100, 2000)), rng.uniform(0.02, 0.05),
                                           rng.uniform(1.2, 2.0), seed=3000 + k)
        box = {"corners": [(0.0, 0.0, 0.0), (side, side, side)]}
    probe = float(rng.choice([0.0, 0.5, 1.0, 1.4, 2.0]))
    groups = rng.integers(0, 3, len(balls)).astype(np.int32) if k % 5 == 0 else None
    return balls, probe, box, groups


def _ids(ids):
    out = ids.astype(np.int64)
    out[ids == O.NET_NULL] = NULL32
    return out


@pytest.mark.parametrize("k", range(CASES))
def test_random_structure(k):
    balls, probe, box, groups = fuzz_case(k)
    o = O.compute(balls, probe, periodic_box=box, groups=groups, with_cell_vertices=True)
    R = balls[o.cells_index.astype(np.int64), 3] + probe
    exposed = o.cells_sas > 0
    allow = (1e-7 * float((4 * np.pi * R[exposed] ** 2).sum()), 1e-7 * float((4 * np.pi * R[exposed] ** 3 / 3).sum()))
    oc = O.compute(balls, probe, periodic_box=box, groups=groups, contacts_only=True)
    for prec, min_pairs in (("fp64", None), ("fp32", 0)):
        r, st = engine_run(balls, probe, prec, periodic_box=box, groups=groups, fp32_min_pairs=min_pairs)
        compare(r, o, prec, total_abs=allow if prec == "fp32" else None)
        r, _ = engine_run(balls, probe, prec, periodic_box=box, groups=groups, contacts_only=True,
                          fp32_min_pairs=min_pairs)
        compare(r, oc, prec, contacts_only=True)
        # the network (FP32 mode takes its FP32-contour path above 2048 candidate pairs)
        r = V.compute_tessellation_result(balls, probe, box, groups, prec, with_cell_vertices=True)
        assert np.array_equal(r.vertex_ids.astype(np.int64), _ids(o.vertex_ids))
        assert np.array_equal(r.edge_ids.astype(np.int64), _ids(o.edge_ids))
        np.testing.assert_allclose(r.vertex_xyz, o.vertex_xyz, rtol=0,
                                   atol=1e-9 * (1 + np.abs(o.vertex_xyz).max(initial=0)))
        assert np.all(np.abs(r.edge_length - o.edge_length) <= 1e-9 * (1 + np.abs(o.edge_length)))
