"""Pins the CPU oracle against the reference's own known answers (CPU only).

Every expected number below is one the reference's tests assert; goldens.json names the
file:line each comes from.  Tolerances are the reference's (0.01 absolute on totals,
tests/common.rs:10).
"""
import numpy as np
import pytest

import oracle as O
from common import (CENTRAL_POINTS, RING_17, THREE_LINE, central_golden, contact_lookup, goldens,
                    load_balls)

G = goldens()


def test_cs_1x1_totals():
    g = G["cs_1x1"]
    r = O.compute(load_balls("cs_1x1"), g["probe"])
    assert len(r.contacts_a) == g["contacts"]
    assert len(r.cells_index) == g["cells"]
    assert abs(r.total_contact_area - g["total_contact_area"]) < g["tol"]
    assert abs(r.total_sas_area - g["total_sas_area"]) < g["tol"]
    assert abs(r.total_volume - g["total_volume"]) < g["tol"]
    k = contact_lookup(r.contacts_a, r.contacts_b, 0, 1)
    assert abs(r.contacts_area[k] - g["contact_0_1_area"]) < g["contact_tol"]
    assert abs(r.contacts_arc[k] - g["contact_0_1_arc"]) < g["contact_tol"]


@pytest.mark.parametrize("form", ["corners", "vectors"])
def test_cs_1x1_periodic(form):
    g = G["cs_1x1_periodic"]
    (x1, y1, z1), (x2, y2, z2) = g["corners"]
    box = ({"corners": g["corners"]} if form == "corners"
           else {"vectors": [(x2 - x1, 0, 0), (0, y2 - y1, 0), (0, 0, z2 - z1)]})
    r = O.compute(load_balls("cs_1x1"), g["probe"], periodic_box=box)
    assert len(r.contacts_a) == g["contacts"]
    assert len(r.cells_index) == g["cells"]
    assert abs(r.total_contact_area - g["total_contact_area"]) < g["tol"]
    assert abs(r.total_sas_area - g["total_sas_area"]) < g["tol"]
    assert abs(r.total_volume - g["total_volume"]) < g["tol"]


def test_2zsk_counts():
    g = G["2zsk"]
    r = O.compute(load_balls("2zsk"), g["probe"])
    assert len(r.contacts_a) == g["contacts"]
    assert len(r.cells_index) == g["cells"]


def test_ring17_basic():
    g = G["ring17"]
    r = O.compute(RING_17, g["probe"])
    assert len(r.contacts_a) == g["contacts"]
    assert len(r.cells_index) == g["cells"]
    cells = {int(i): (s, v) for i, s, v in zip(r.cells_index, r.cells_sas, r.cells_vol)}
    assert abs(cells[0][0] - g["cell0_sas"]) < g["cell_tol"]
    assert abs(cells[0][1] - g["cell0_vol"]) < g["cell_tol"]
    assert abs(cells[1][0] - g["cell1_sas"]) < g["cell_tol"]
    assert abs(cells[1][1] - g["cell1_vol"]) < g["cell_tol"]
    k = contact_lookup(r.contacts_a, r.contacts_b, 0, 1)
    assert abs(r.contacts_area[k] - g["contact_0_1_area"]) < g["c01_tol"]
    assert abs(r.contacts_arc[k] - g["contact_0_1_arc"]) < g["c01_tol"]
    k = contact_lookup(r.contacts_a, r.contacts_b, 1, 2)
    assert abs(r.contacts_area[k] - g["contact_1_2_area"]) < g["c12_tol"]


def test_ring17_periodic():
    g = G["ring17_periodic"]
    r = O.compute(RING_17, g["probe"], periodic_box={"corners": g["corners"]})
    assert len(r.contacts_a) > g["min_contacts_exclusive"]
    assert len(r.cells_index) == g["cells"]
    cells = {int(i): (s, v) for i, s, v in zip(r.cells_index, r.cells_sas, r.cells_vol)}
    assert abs(cells[0][0] - g["cell0_sas"]) < g["cell_tol"]
    assert abs(cells[0][1] - g["cell0_vol"]) < g["cell_tol"]
    k = contact_lookup(r.contacts_a, r.contacts_b, 0, 0)
    assert k is not None
    assert abs(r.contacts_area[k] - g["self_contact_0_0_area"]) < g["self_tol"]


def test_two_body_groups_contacts_only():
    g = G["two_body_groups"]
    balls = [(0.0, 0.0, 0.0, 1.5), (1.0, 0.0, 0.0, 1.5), (4.0, 0.0, 0.0, 2.0), (5.0, 0.0, 0.0, 2.0)]
    r = O.compute(balls, g["probe"], groups=[0, 0, 1, 1], contacts_only=True)
    assert len(r.contacts_a) == g["contacts"]
    assert (int(r.contacts_a[0]), int(r.contacts_b[0])) == (g["id_a"], g["id_b"])
    assert abs(r.contacts_area[0] - g["area"]) < g["tol"]


def test_centrality_golden():
    balls = [p + [1.5] for p in CENTRAL_POINTS]
    r = O.compute(balls, 1.4)
    got = {(int(a), int(b)): bool(c) for a, b, c in zip(r.contacts_a, r.contacts_b, r.contacts_central)}
    gold = central_golden()
    assert len(got) == len(gold)
    for a, b, c in gold:
        assert got[(min(a, b), max(a, b))] == bool(c)


def test_contacts_only_matches_full():  # tests/contacts_only.rs:4-88
    for balls in ([(0, 0, 0, 1.5), (2.5, 0, 0, 1.5), (1.25, 2.0, 0, 1.5)], [p + [1.5] for p in CENTRAL_POINTS]):
        full = O.compute(balls, 1.4)
        only = O.compute(balls, 1.4, contacts_only=True)
        fo = np.lexsort((full.contacts_b, full.contacts_a))
        oo = np.lexsort((only.contacts_b, only.contacts_a))
        assert np.array_equal(full.contacts_a[fo], only.contacts_a[oo])
        assert np.array_equal(full.contacts_b[fo], only.contacts_b[oo])
        assert np.max(np.abs(full.contacts_area[fo] - only.contacts_area[oo])) < 1e-10
        assert np.max(np.abs(full.contacts_arc[fo] - only.contacts_arc[oo])) < 1e-10
        assert np.array_equal(full.contacts_central[fo], only.contacts_central[oo])


def test_contacts_only_periodic_canonical():  # tests/contacts_only.rs:114-142
    balls = [(0.0, 0.0, 0.0, 2.0), (9.0, 0.0, 0.0, 2.0)]
    box = {"corners": [(-5, -5, -5), (5, 5, 5)]}
    full = O.compute(balls, 1.4, periodic_box=box)
    only = O.compute(balls, 1.4, periodic_box=box, contacts_only=True)
    assert len(full.contacts_a) == len(only.contacts_a)
    assert np.all(only.contacts_a < 2) and np.all(only.contacts_b < 2)


def test_grouping_and_edge_cases():  # src/tessellation.rs:666-736, 1210-1283
    r = O.compute(THREE_LINE, 0.5)
    assert len(r.contacts_a) == 2
    r = O.compute(THREE_LINE, 0.5, groups=[0, 0, 0])
    assert len(r.contacts_a) == 0
    r = O.compute(THREE_LINE, 0.5, groups=[0, 0, 1])
    assert [(int(a), int(b)) for a, b in zip(r.contacts_a, r.contacts_b)] == [(1, 2)]
    r = O.compute(THREE_LINE + [(6.0, 0.0, 0.0, 1.0)], 0.5, groups=[0, 0, 1, 1])
    assert [(int(a), int(b)) for a, b in zip(r.contacts_a, r.contacts_b)] == [(1, 2)]
    assert len(r.cells_index) == 2
    r = O.compute([(0.0, 0.0, 0.0, 1.0)], 0.5)
    assert len(r.contacts_a) == 0 and len(r.cells_index) == 1
    assert abs(r.cells_sas[0] - 4 * np.pi * 1.5 ** 2) < 0.01
    r = O.compute(np.zeros((0, 4)), 0.5)
    assert r.num_balls == 0 and len(r.contacts_a) == 0 and len(r.cells_index) == 0
    r = O.compute([(0, 0, 0, 1.0), (10, 0, 0, 1.0)], 0.5)
    assert len(r.contacts_a) == 0 and len(r.cells_index) == 2
    r = O.compute([(0, 0, 0, 1.0), (0, 0, 0, 0.5), (1, 0, 0, 1.0)], 0.5)  # containment
    assert len(r.cells_index) <= 3


def test_thread_count_does_not_change_results():
    balls = load_balls("2zsk")
    O.set_threads(1)
    r1 = O.compute(balls, 1.4)
    O.set_threads(4)
    r4 = O.compute(balls, 1.4)
    O.set_threads(0)
    assert np.array_equal(r1.contacts_a, r4.contacts_a)
    assert np.array_equal(r1.contacts_area, r4.contacts_area)
    assert np.array_equal(r1.cells_sas, r4.cells_sas)


def test_network_ring17():  # src/tessellation.rs:1347-1387 (C++ example output)
    r = O.compute(RING_17, 1.0, with_cell_vertices=True)
    on_sas = int((r.vertex_ids[:, 3] == O.NET_NULL).sum())
    assert (len(r.vertex_ids), on_sas, len(r.vertex_ids) - on_sas) == (68, 32, 36)
    assert len(r.edge_ids) > 0
    # ids sorted within each element, elements sorted and unique
    assert np.all(np.diff(r.vertex_ids.astype(np.float64), axis=1) >= 0)
    keys = [tuple(v) for v in r.vertex_ids.tolist()]
    assert keys == sorted(set(keys))


def test_network_cs_1x1():  # src/tessellation.rs:1391-1510
    r = O.compute(load_balls("cs_1x1"), 2.0, with_cell_vertices=True)
    assert (len(r.vertex_ids), len(r.edge_ids)) == (65, 215)
    assert int((r.vertex_ids[:, 3] == O.NET_NULL).sum()) > len(r.vertex_ids) // 2


def test_network_full_circle_edge():  # src/tessellation.rs:1329-1344: an uncut contact
    r = O.compute([(0.0, 0.0, 0.0, 1.5), (2.5, 0.0, 0.0, 1.5)], 0.5, with_cell_vertices=True)
    assert len(r.vertex_ids) == 0 and len(r.edge_ids) == 1
    assert r.edge_ids[0, 2] == O.NET_NULL


# ---- compute_solvent_spheres (solvent_spheres.rs:371-483, tests/test_python.py:199-293) ----
def test_icosahedron_vertex_counts():  # subdivided_icosahedron.rs:143-152
    for depth, k in enumerate((12, 42, 162, 642, 2562)):
        v = O.icosahedron(depth)
        assert v.shape == (k, 3)
        assert np.abs(np.linalg.norm(v, axis=1) - 1.0).max() < 1e-10
    assert len(O.icosahedron(7)) == 2562  # depth clamps to 4 (:29-38)


def test_solvent_single_sphere():  # solvent_spheres.rs:371-386
    r = O.solvent_spheres([(0.0, 0.0, 0.0, 1.5)], 1.4, subdivision_depth=0)
    assert len(r.weight) == 12 and np.all(r.parent == 0)
    assert np.all(np.abs(r.radius - 1.4) < 1e-10) and np.all(r.weight > 0)


def test_solvent_two_separated_spheres_cpp_golden():  # solvent_spheres.rs:410-441 (C++ sihsolv)
    r = O.solvent_spheres([(0.0, 0.0, 0.0, 1.5), (5.0, 0.0, 0.0, 1.5)], 1.4, 0.0, 0)
    assert len(r.weight) == 24
    assert (r.parent == 0).sum() == 12 and (r.parent == 1).sum() == 12
    assert abs(r.weight.sum() - 249.1) < 5.0


def test_solvent_touching_and_contained():  # solvent_spheres.rs:388-408, 443-461
    r = O.solvent_spheres([(0.0, 0.0, 0.0, 1.5), (2.5, 0.0, 0.0, 1.5)], 1.4, subdivision_depth=0)
    assert 0 < len(r.weight) < 24
    r = O.solvent_spheres([(0.0, 0.0, 0.0, 3.0), (2.5, 0.0, 0.0, 1.0)], 1.4, subdivision_depth=0)
    assert (r.parent == 0).sum() > (r.parent == 1).sum()


def test_solvent_validation_and_empty():  # solvent_spheres.rs:463-483; tests/test_python.py:243-278
    for balls, probe in [([(0.0, 0.0, 0.0, 1.5)], -1.0), ([(0.0, 0.0, 0.0, 1.5)], float("nan")),
                         ([(0.0, 0.0, 0.0, -1.0)], 1.4), ([(float("nan"), 0.0, 0.0, 1.5)], 1.4)]:
        with pytest.raises(ValueError):
            O.solvent_spheres(balls, probe)
    assert len(O.solvent_spheres(np.zeros((0, 4)), 1.4).weight) == 0
    assert len(O.solvent_spheres([(0.0, 0.0, 0.0, 1.5), (5.0, 0.0, 0.0, 1.5)], 1.4, volume_probe=0.5,
                                 subdivision_depth=0).weight) > 0
