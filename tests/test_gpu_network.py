"""GPU tessellation network (compute_tessellation with with_cell_vertices) against the
oracle and the reference's network goldens (src/tessellation.rs:1329-1510).

Ids of every vertex and edge must match the oracle bit for bit (same elements, same
order); positions and lengths come from FP64 contours on both sides and agree within
1e-9 (1 + |x|).  Of several elements with equal ids both keep the first in pair and
contour order, so periodic duplicates (equal ids mod n, shifted positions) agree too.
"""
import numpy as np
import pytest

import oracle as O
import voronota_ltr as V
from common import RING_17, THREE_LINE, goldens, load_balls, sunflower
from gpu_util import compare
from voronota_ltr import workloads as W

pytestmark = pytest.mark.gpu
G = goldens()
PRECISIONS = ["fp64", "fp32"]
NULL32 = 0xFFFFFFFF


def _oracle_ids(ids):
    out = ids.astype(np.int64)
    out[ids == O.NET_NULL] = NULL32
    return out


def check_network(balls, probe, prec, periodic_box=None, groups=None):
    r = V.compute_tessellation_result(balls, probe, periodic_box, groups, prec, with_cell_vertices=True)
    o = O.compute(balls, probe, periodic_box=periodic_box, groups=groups, with_cell_vertices=True)
    compare(r, o, prec)
    assert r.vertex_ids.shape == o.vertex_ids.shape, (r.vertex_ids.shape, o.vertex_ids.shape)
    assert r.edge_ids.shape == o.edge_ids.shape, (r.edge_ids.shape, o.edge_ids.shape)
    assert np.array_equal(r.vertex_ids.astype(np.int64), _oracle_ids(o.vertex_ids))
    assert np.array_equal(r.edge_ids.astype(np.int64), _oracle_ids(o.edge_ids))
    np.testing.assert_allclose(r.vertex_xyz, o.vertex_xyz, rtol=0, atol=1e-9 * (1 + np.abs(o.vertex_xyz).max(initial=0)))
    assert np.all(np.abs(r.edge_length - o.edge_length) <= 1e-9 * (1 + np.abs(o.edge_length)))
    return r


@pytest.mark.parametrize("prec", PRECISIONS)
def test_ring17_counts(prec):  # src/tessellation.rs:1347-1387
    r = check_network(RING_17, 1.0, prec)
    on_sas = int((r.vertex_ids[:, 3] == NULL32).sum())
    assert (len(r.vertex_ids), on_sas, len(r.vertex_ids) - on_sas) == (68, 32, 36)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_cs_1x1_counts(prec):  # src/tessellation.rs:1391-1510
    r = check_network(load_balls("cs_1x1"), 2.0, prec)
    assert (len(r.vertex_ids), len(r.edge_ids)) == (65, 215)


def test_full_circle_edge_dict():  # src/tessellation.rs:1329-1344: an uncut contact
    d = V.compute_tessellation([(0.0, 0.0, 0.0, 1.5), (2.5, 0.0, 0.0, 1.5)], 0.5, with_cell_vertices=True,
                               precision="fp64")
    assert d["cell_vertices"] == []
    assert len(d["cell_edges"]) == 1
    e = d["cell_edges"][0]
    assert e["ball_indices"] == [0, 1, None] and e["is_on_sas"]
    o = O.compute([(0.0, 0.0, 0.0, 1.5), (2.5, 0.0, 0.0, 1.5)], 0.5, with_cell_vertices=True)
    assert abs(e["length"] - o.edge_length[0]) < 1e-12


def test_dict_form_matches_arrays():
    r = V.compute_tessellation_result(RING_17, 1.0, with_cell_vertices=True, precision="fp64")
    d = r.to_dict()
    assert len(d["cell_vertices"]) == len(r.vertex_ids) and len(d["cell_edges"]) == len(r.edge_ids)
    for v, ids, p in zip(d["cell_vertices"], r.vertex_ids.tolist(), r.vertex_xyz.tolist()):
        assert v["ball_indices"] == [None if i == NULL32 else i for i in ids]
        assert (v["x"], v["y"], v["z"]) == tuple(p)
        assert v["is_on_sas"] == (ids[3] == NULL32)
    for e, ids in zip(d["cell_edges"], r.edge_ids.tolist()):
        assert e["is_on_sas"] == (ids[2] == NULL32)
    # without with_cell_vertices the dict has no network keys (python.rs:200-206)
    d0 = V.compute_tessellation(RING_17, 1.0, precision="fp64")
    assert "cell_vertices" not in d0 and "cell_edges" not in d0


@pytest.mark.parametrize("prec", PRECISIONS)
def test_periodic_ring_and_box(prec):
    gp = G["ring17_periodic"]
    check_network(RING_17, gp["probe"], prec, periodic_box={"corners": gp["corners"]})
    g = G["cs_1x1_periodic"]
    check_network(load_balls("cs_1x1"), g["probe"], prec, periodic_box={"corners": g["corners"]})
    balls, side = W.periodic_box_balls(3000, 0.033, 1.52, seed=9)
    check_network(balls, 1.4, prec, periodic_box={"corners": [(0, 0, 0), (side, side, side)]})


@pytest.mark.parametrize("prec", PRECISIONS)
def test_structures_and_groups(prec):
    check_network(load_balls("2zsk"), 1.4, prec)
    balls = W.lattice_balls(4000, 2)
    check_network(balls, 1.4, prec)
    check_network(balls, 1.4, prec, groups=W.x_sign_groups(balls))


def test_edge_cases():
    for balls, probe in [
        (np.zeros((0, 4)), 1.4),
        ([(0.0, 0.0, 0.0, 1.0)], 0.5),
        ([(0, 0, 0, 1.0), (10, 0, 0, 1.0)], 0.5),
        ([(0, 0, 0, 1.0), (0, 0, 0, 1.0), (1.5, 0, 0, 1.0)], 0.5),
        (THREE_LINE, 0.5),
        ([(0, 0, 0, 1), (0, 0, 1, 1), (0, 1, 0, 1), (0, 1, 1, 1), (1, 0, 0, 1), (1, 0, 1, 1), (1, 1, 0, 1),
          (1, 1, 1, 1)], 2.0),
    ]:
        check_network(balls, probe, "fp64")


def test_network_does_not_change_the_rest():
    balls = load_balls("2zsk")
    a = V.compute_tessellation_result(balls, 1.4, precision="fp32")
    b = V.compute_tessellation_result(balls, 1.4, precision="fp32", with_cell_vertices=True)
    assert np.array_equal(a.id_a, b.id_a) and np.array_equal(a.id_b, b.id_b)
    assert np.array_equal(a.area, b.area) and np.array_equal(a.cell_sas_area, b.cell_sas_area)
    assert a.vertex_ids is None and b.vertex_ids is not None


@pytest.mark.parametrize("prec", PRECISIONS)
def test_contours_longer_than_a_warp(prec):
    """Contours of 40, 80 and 120 points go through the serial contour kernel."""
    for balls, probe in [(sunflower(40), 0.5), (sunflower(40, rr=0.1, rho=3.3), 0.1),
                         (sunflower(120, rr=0.12, rho=3.3), 0.5)]:
        r = check_network(balls, probe, prec)
        on_pair = ((r.vertex_ids == 0).any(1) & (r.vertex_ids == 1).any(1)).sum()
        assert on_pair == len(balls) - 2
    box = {"corners": [(-10, -10, -10), (12, 10, 10)]}
    check_network(sunflower(40, rr=0.1, rho=3.3), 0.1, prec, periodic_box=box)


def test_fp32_network_after_larger_calls():
    """A warp of the FP32 element kernel handles several pairs in turn (more pairs than
    resident warps); a slot it counts but leaves unwritten would show the elements of the
    previous, larger calls that still sit in reused device memory."""
    for seed in range(2):
        V.compute_tessellation_result(W.lattice_balls(20000, seed), 1.4, precision="fp32", with_cell_vertices=True)
    balls, side = W.periodic_box_balls(3000, 0.033, 1.52, seed=9)
    for _ in range(2):
        check_network(balls, 1.4, "fp32", periodic_box={"corners": [(0, 0, 0), (side, side, side)]})


@pytest.mark.parametrize("prec", PRECISIONS)
def test_large_deduplication_buckets(prec):
    """The big ball (id 0) among a lattice's small balls: its cell's vertices and edges all
    fall into the bucket of id 0, several thousand elements (the block sort in global
    memory); the sunflower's two large balls give buckets of ~1,400 (the block sort in
    shared memory)."""
    from common import big_ball_in_lattice
    check_network(big_ball_in_lattice(), 1.4, prec)
    check_network(sunflower(120, rr=0.12, rho=3.3), 0.5, prec)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_deduplication_key_forms(prec):
    """The vertex deduplication keys: three ids packed into one word (below 2^21 balls) and
    the two-word form (taken from 2^21 balls on, forced here) give the same network."""
    from common import big_ball_in_lattice
    import torch
    pballs, side = W.periodic_box_balls(3000, 0.033, 1.52, seed=9)
    for balls, probe, box in [(W.lattice_balls(4000, 2), 1.4, None), (big_ball_in_lattice(), 1.4, None),
                              (pballs, 1.4, {"corners": [(0, 0, 0), (side, side, side)]})]:
        out = []
        for wide in (False, True):
            e = V.Engine()
            e.set_network(True)
            e.set_network_wide_keys(wide)
            d = torch.from_numpy(np.ascontiguousarray(balls, dtype=np.float64)).cuda()
            e.compute_device(d.data_ptr(), len(balls), probe, periodic_box=box, precision=prec)
            out.append(e.download())
            e.close()
        a, b = out
        assert len(a.vertex_ids) > 0
        assert np.array_equal(a.vertex_ids, b.vertex_ids) and np.array_equal(a.vertex_xyz, b.vertex_xyz)
        assert np.array_equal(a.edge_ids, b.edge_ids) and np.array_equal(a.edge_length, b.edge_length)
