"""Updateable tessellation on the CPU oracle, following tests/updateable.rs.

Also documents a reference behaviour found while restating SpheresSearcher::update
(spheres_searcher.rs:144-175): positions are overwritten before the grid removal, so a
ball that crosses a grid-cell boundary keeps a stale registration in its old cell and
can show up twice in a neighbour list.  The oracle reproduces that by default
(``faithful`` mode) and can instead remove by the old position (``fixed`` mode), which
gives the incremental == full-recompute contract that tests/updateable.rs asserts.
"""
import numpy as np
import pytest

import oracle as O
from common import RING_17, THREE_LINE, load_balls


def totals(r):
    return len(r.contacts_a), len(r.cells_index), r.total_contact_area, r.total_sas_area, r.total_volume


def verify_updateable_matches_full(balls, probe, pbox, changed, iters):  # tests/updateable.rs:63-120
    balls = np.array(balls, dtype=np.float64)
    t = O.OracleUpdateable(with_backup=True)
    assert t.init(balls, probe, pbox)
    for it in range(iters):
        for i in changed:
            balls[i, 0] += 0.05 * (it + 1.0)
        assert t.update_with_changed(balls, changed)
        full = O.compute(balls, probe, periodic_box=pbox)
        inc = t.summary()
        assert len(inc.contacts_a) == len(full.contacts_a)
        assert len(inc.cells_index) == len(full.cells_index)
        assert abs(inc.total_contact_area - full.total_contact_area) < 0.1
        assert abs(inc.total_sas_area - full.total_sas_area) < 0.1
    assert t.restore()
    assert len(t.summary().contacts_a) > 0


@pytest.fixture(params=[True, False], ids=["faithful", "fixed"])
def grid_mode(request):
    O.set_faithful_grid_update(request.param)
    yield request.param
    O.set_faithful_grid_update(True)


def test_ring17_no_periodic(grid_mode):
    verify_updateable_matches_full(RING_17, 1.0, None, [0, 8], 3)


def test_three_line(grid_mode):
    verify_updateable_matches_full(THREE_LINE, 0.5, None, [1], 5)


def test_ring_periodic_cpp_port(grid_mode):  # tests/updateable.rs:133-192
    balls = np.array(RING_17, dtype=np.float64)
    box = {"corners": [(-1.6, -1.6, -0.6), (1.6, 1.6, 3.1)]}
    t = O.OracleUpdateable(with_backup=True)
    assert t.init(balls, 1.0, box)
    f0, u0 = O.compute(balls, 1.0, periodic_box=box), t.summary()
    assert len(u0.contacts_a) == len(f0.contacts_a)
    assert abs(u0.total_contact_area - f0.total_contact_area) < 0.01
    for _ in range(5):
        balls[[0, 1], 0] += 0.1
        assert t.update_with_changed(balls, [0, 1])
        f, u = O.compute(balls, 1.0, periodic_box=box), t.summary()
        assert len(u.contacts_a) == len(f.contacts_a)
        assert len(u.cells_index) == len(f.cells_index)
        assert abs(u.total_contact_area - f.total_contact_area) < 0.1
        assert abs(u.total_sas_area - f.total_sas_area) < 0.01
        assert abs(u.total_volume - f.total_volume) < 0.01
    before = t.summary().total_contact_area
    assert t.restore()
    assert abs(before - t.summary().total_contact_area) > 0.01


def test_exclusion_and_restore():  # tests/updateable.rs:194-218
    t = O.OracleUpdateable(with_backup=True)
    assert t.init(THREE_LINE, 0.5)
    s = t.summary()
    assert (len(s.contacts_a), len(s.cells_index)) == (2, 3)
    assert t.set_exclusion(1, True)
    s = t.summary()
    assert (len(s.contacts_a), len(s.cells_index)) == (0, 2)
    assert t.restore()
    s = t.summary()
    assert (len(s.contacts_a), len(s.cells_index)) == (2, 3)


def test_auto_detect_and_no_change():  # tests/updateable.rs:220-250
    balls = np.array([(0.0, 0, 0, 1.0), (2.0, 0, 0, 1.0)])
    t = O.OracleUpdateable()
    assert t.init(balls, 0.5)
    n0 = len(t.summary().contacts_a)
    balls[0, 0] += 0.1
    assert t.update(balls)
    assert len(t.summary().contacts_a) == n0
    assert 0 in t.changed_ids().tolist()
    assert not t.update(balls)


def test_full_reinit_trigger():  # tests/updateable.rs:266-285
    n = 20
    balls = np.array([(i * 2.0, 0, 0, 1.0) for i in range(n)])
    t = O.OracleUpdateable()
    assert t.init(balls, 0.5)
    ids = list(range(n // 2 + 1))
    balls[ids, 0] += 0.1
    assert t.update_with_changed(balls, ids)
    assert t.last_update_was_full_reinit()


def test_2zsk_incremental(grid_mode):  # tests/updateable.rs:287-321
    balls = load_balls("2zsk").copy()
    t = O.OracleUpdateable()
    assert t.init(balls, 1.4)
    s = t.summary()
    assert (len(s.contacts_a), len(s.cells_index)) == (23855, 3545)
    ids = [0, 100, 500]
    balls[ids, 0] += 0.1
    assert t.update_with_changed(balls, ids)
    assert not t.last_update_was_full_reinit()
    full, inc = O.compute(balls, 1.4), t.summary()
    assert len(inc.contacts_a) == len(full.contacts_a)
    assert len(inc.cells_index) == len(full.cells_index)


def _cell_crossing_case():
    """Four balls; ball 2 moves across a grid-cell boundary between updates.

    R = 1 + 0.5, so the grid edge is max(2R + 0.25) = 3.25: ball 2 at x = 3.2 sits in
    cell 0 and at x = 3.3 in cell 1.  Ball 3 (x = 12) pins the grid bounds so the update
    stays incremental.  Ball 0 (x = 6.0, cell 1) sees cells 0..2, i.e. both the stale
    registration of ball 2 in cell 0 and the live one in cell 1.
    """
    return np.array([(6.0, 0.0, 0.0, 1.0), (0.5, 0.0, 0.0, 1.0), (3.2, 0.0, 0.0, 1.0),
                     (12.0, 0.0, 0.0, 1.0)])


def test_reference_stale_grid_registration_duplicates_contact():
    balls = _cell_crossing_case()
    O.set_faithful_grid_update(True)
    t = O.OracleUpdateable()
    assert t.init(balls, 0.5)
    balls[2, 0] = 3.3
    assert t.update_with_changed(balls, [2])
    inc, full = t.summary(), O.compute(balls, 0.5)
    pairs_inc = sorted(zip(inc.contacts_a.tolist(), inc.contacts_b.tolist()))
    pairs_full = sorted(zip(full.contacts_a.tolist(), full.contacts_b.tolist()))
    # faithful restatement: balls 0 and 1 both see ball 2 twice, so both of their
    # contacts with ball 2 are produced twice, unlike the full recompute
    assert pairs_full == [(0, 2), (1, 2)]
    assert pairs_inc == [(0, 2), (0, 2), (1, 2), (1, 2)]


def test_fixed_grid_update_matches_full_on_cell_crossing():
    balls = _cell_crossing_case()
    O.set_faithful_grid_update(False)
    try:
        t = O.OracleUpdateable()
        assert t.init(balls, 0.5)
        balls[2, 0] = 3.3
        assert t.update_with_changed(balls, [2])
        inc, full = t.summary(), O.compute(balls, 0.5)
        assert sorted(zip(inc.contacts_a.tolist(), inc.contacts_b.tolist())) == \
            sorted(zip(full.contacts_a.tolist(), full.contacts_b.tolist()))
        assert abs(inc.total_sas_area - full.total_sas_area) < 1e-9
    finally:
        O.set_faithful_grid_update(True)
