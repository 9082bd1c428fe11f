"""Device-resident UpdateableTessellation against the oracle's restatement of updateable.rs.

Every step compares the GPU handle with the oracle handle driven by the same calls:
return values, changed_ids, affected_ids, last_update_was_full_reinit, and the summary
(contacts in the reference's summary order, bit-exact ids and central bits, values within
the tolerance of the precision; cells).  The oracle runs with the grid-update fix
(removal by the old position), the behaviour the GPU path implements; the reference's
stale-cell registration is documented in tests/test_oracle_updateable.py.
Cases follow tests/updateable.rs (ring-17, three-line, periodic ring, exclusion, restore,
auto-detection, full reinit, 2zsk) plus seeded trajectories on the lattice and periodic
generators.
"""
import numpy as np
import pytest

import oracle as O
import voronota_ltr as V
from common import RING_17, THREE_LINE, load_balls
from gpu_util import compare
from voronota_ltr import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def fixed_grid():
    O.set_faithful_grid_update(False)
    yield
    O.set_faithful_grid_update(True)


class Pair:
    """A GPU handle and an oracle handle driven by the same calls."""

    def __init__(self, precision="fp64", with_backup=True):
        self.precision = precision
        self.g = V.UpdateableTessellation(with_backup=with_backup, precision=precision)
        self.o = O.OracleUpdateable(with_backup=with_backup)

    def call(self, name, *args):
        rg = getattr(self.g, name)(*args)
        ro = getattr(self.o, name)(*args)
        assert rg == ro, f"{name}: gpu {rg} oracle {ro}"
        return rg

    def check(self):
        assert self.g.last_update_was_full_reinit() == self.o.last_update_was_full_reinit()
        assert self.g.changed_ids().tolist() == self.o.changed_ids().tolist(), "changed_ids"
        assert self.g.affected_ids().tolist() == self.o.affected_ids().tolist(), "affected_ids"
        return compare(self.g.summary(), self.o.summary(), self.precision)


PRECISIONS = ["fp64", "fp32"]


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ring17(precision):  # tests/updateable.rs:63-131
    balls = np.array(RING_17, dtype=np.float64)
    p = Pair(precision)
    assert p.call("init", balls, 1.0, None)
    p.check()
    for it in range(3):
        balls[[0, 8], 0] += 0.05 * (it + 1.0)
        assert p.call("update_with_changed", balls, [0, 8])
        p.check()
    assert p.call("restore")
    p.check()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_three_line(precision):
    balls = np.array(THREE_LINE, dtype=np.float64)
    p = Pair(precision)
    assert p.call("init", balls, 0.5, None)
    for it in range(5):
        balls[1, 0] += 0.05 * (it + 1.0)
        assert p.call("update_with_changed", balls, [1])
        p.check()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_ring_periodic(precision):  # tests/updateable.rs:133-192
    balls = np.array(RING_17, dtype=np.float64)
    box = {"corners": [(-1.6, -1.6, -0.6), (1.6, 1.6, 3.1)]}
    p = Pair(precision)
    assert p.call("init", balls, 1.0, box)
    p.check()
    for _ in range(5):
        balls[[0, 1], 0] += 0.1
        assert p.call("update_with_changed", balls, [0, 1])
        p.check()
    assert p.call("restore")
    p.check()


def test_exclusion_and_restore():  # tests/updateable.rs:194-218
    p = Pair()
    assert p.call("init", THREE_LINE, 0.5, None)
    s = p.g.summary()
    assert (len(s.id_a), len(s.cell_index)) == (2, 3)
    assert p.call("set_exclusion", 1, True)
    p.check()
    s = p.g.summary()
    assert (len(s.id_a), len(s.cell_index)) == (0, 2)
    assert not p.call("set_exclusion", 1, True)
    assert p.call("restore")
    p.check()
    assert p.call("set_exclusion", 1, True)
    assert p.call("set_exclusion", 1, False)
    p.check()
    assert not p.call("set_exclusion", 7, True)


def test_auto_detect_and_no_change():  # tests/updateable.rs:220-250
    balls = np.array([(0.0, 0, 0, 1.0), (2.0, 0, 0, 1.0)])
    p = Pair(with_backup=False)
    assert p.call("init", balls, 0.5, None)
    balls[0, 0] += 0.1
    assert p.call("update", balls)
    p.check()
    assert not p.call("update", balls)
    p.check()
    assert not p.call("update_with_changed", balls, [])
    assert not p.call("restore")


def test_full_reinit_trigger():  # tests/updateable.rs:266-285
    n = 20
    balls = np.array([(i * 2.0, 0, 0, 1.0) for i in range(n)])
    p = Pair()
    assert p.call("init", balls, 0.5, None)
    ids = list(range(n // 2 + 1))
    balls[ids, 0] += 0.1
    assert p.call("update_with_changed", balls, ids)
    assert p.g.last_update_was_full_reinit()
    p.check()
    # a different ball count is a full reinit too
    assert p.call("update_with_changed", balls[:15], [0])
    p.check()


def test_duplicate_and_out_of_range_ids():
    balls = W.lattice_balls(400, 3)
    p = Pair()
    assert p.call("init", balls, 1.4, None)
    balls[[5, 9], 1] += 0.07
    assert p.call("update_with_changed", balls, [5, 9, 5, 10**9, 9])
    p.check()
    balls[[5], 1] += 0.07
    assert p.call("update_with_changed", balls, [5, 5, 5])
    p.check()
    assert not p.call("update_with_changed", balls, [1, 2, 10**9])  # unchanged balls
    p.check()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_2zsk_incremental(precision):  # tests/updateable.rs:287-321
    balls = load_balls("2zsk").copy()
    p = Pair(precision)
    assert p.call("init", balls, 1.4, None)
    s = p.g.summary()
    assert (len(s.id_a), len(s.cell_index)) == (23855, 3545)
    p.check()
    ids = [0, 100, 500]
    balls[ids, 0] += 0.1
    assert p.call("update_with_changed", balls, ids)
    assert not p.g.last_update_was_full_reinit()
    p.check()


def _trajectory(p, balls, box, steps, frac, seed):
    rng = np.random.default_rng(seed)
    n = len(balls)
    for _ in range(steps):
        ids = np.sort(rng.choice(n, size=max(1, int(frac * n)), replace=False))
        balls[ids, :3] += rng.normal(0.0, 0.05, size=(len(ids), 3))
        assert p.call("update_with_changed", balls, ids.tolist())
        assert not p.g.last_update_was_full_reinit()
        p.check()


@pytest.mark.parametrize("precision", PRECISIONS)
def test_lattice_trajectory(precision):
    balls = W.lattice_balls(3000, 11)
    p = Pair(precision, with_backup=False)
    assert p.call("init", balls, 1.4, None)
    p.check()
    _trajectory(p, balls, None, 6, 0.01, 5)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_periodic_trajectory(precision):  # the periodic-box trajectory workload, small
    balls, side = W.periodic_box_balls(4000, seed=2)
    box = {"corners": [(0.0, 0.0, 0.0), (side, side, side)]}
    p = Pair(precision)
    assert p.call("init", balls, 1.4, box)
    p.check()
    _trajectory(p, balls, box, 6, 0.01, 9)
    assert p.call("restore")
    p.check()


def test_exclusion_in_structure():
    balls = W.lattice_balls(1500, 4)
    p = Pair()
    assert p.call("init", balls, 1.4, None)
    for i in (3, 700, 1499):
        assert p.call("set_exclusion", i, True)
        p.check()
    assert p.call("set_exclusion", 700, False)
    p.check()
    balls[[700, 701], 2] += 0.1
    assert p.call("update_with_changed", balls, [700, 701])
    p.check()


def test_device_api_matches_host_api():
    import torch

    balls = W.lattice_balls(2500, 8)
    h = V.UpdateableTessellation(precision="fp64")
    d = V.UpdateableTessellation(precision="fp64")
    assert h.init(balls, 1.4)
    t = torch.from_numpy(balls).cuda()
    torch.cuda.synchronize()
    assert d.init_device(t.data_ptr(), len(balls), 1.4)
    rng = np.random.default_rng(1)
    for _ in range(3):
        ids = np.sort(rng.choice(len(balls), 25, replace=False)).astype(np.uint64)
        balls[ids, :3] += rng.normal(0, 0.05, (len(ids), 3))
        assert h.update_with_changed(balls, ids)
        t = torch.from_numpy(balls).cuda()
        ti = torch.from_numpy(ids.view(np.int64)).cuda()
        torch.cuda.synchronize()
        assert d.update_with_changed_device(t.data_ptr(), len(balls), ti.data_ptr(), len(ids))
        a, b = h.summary(), d.summary()
        assert np.array_equal(a.id_a, b.id_a) and np.array_equal(a.id_b, b.id_b)
        assert np.array_equal(a.area, b.area) and np.array_equal(a.cell_sas_area, b.cell_sas_area)
        assert h.affected_ids().tolist() == d.affected_ids().tolist()
        assert d.totals() == (b.total_sas_area, b.total_volume, b.total_contact_area)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_long_neighbour_lists(precision):
    """A big ball with 646 neighbours (beyond the warp sort buffer) moved and changed:
    its frontier list goes through the block sort."""
    from common import big_ball_in_lattice
    balls = big_ball_in_lattice()
    p = Pair(precision)
    assert p.call("init", balls, 1.4, None)
    p.check()
    moved = balls.copy()
    moved[0, :3] += (0.3, -0.2, 0.1)
    moved[0, 3] += 0.4
    moved[5, :3] += 0.2
    assert p.call("update_with_changed", moved, [0, 5])
    p.check()
