"""The hand-written adjoint against central finite differences.

L = sum_i w_i SAS_i + sum_(a,b) u_ab area_ab with seeded w ~ U(0, 1) and u ~ N(0, 1), and
with a volume term sum_i v_i V_i (v ~ U(0, 1))
(u attached to the contact's ball pair, so contacts that appear under a perturbation
carry no weight).  The gradient with respect to x, y, z and r of randomly chosen balls is
checked against central differences with h = 1e-4 A in f64 of the GPU FP64 forward and of
the CPU oracle.  Tolerance: |g - fd| <= 1e-5 (1 + |fd|).  The differences' truncation
error is O(h^2) (about 1e-7 at h = 1e-4) except where a +-h step crosses a change of a
contour's topology (a vertex passing a plane), where it is O(h); there the check is
repeated once with h = 1e-5.  Also: the FP32 forward gives the same gradient, the
torch.autograd front end agrees with the C ABI, and a periodic box.
"""
import numpy as np
import pytest

import oracle as O
import voronota_ltr as V
from voronota_ltr import workloads as W

pytestmark = pytest.mark.gpu

H = 1e-4
TOL = 1e-5


def _weights(balls, probe, seed, box=None):
    r = V.compute_tessellation_result(balls, probe, box, precision="fp64")
    rng = np.random.default_rng(seed)
    w = rng.uniform(0.0, 1.0, len(balls))
    u = rng.normal(0.0, 1.0, len(r.id_a))
    upair = {(int(a), int(b)): float(x) for a, b, x in zip(r.id_a, r.id_b, u)}
    return w, u, upair


def _loss(sas_idx, sas, ida, idb, area, w, upair, vol=None, v=None):
    ls = float(np.dot(w[sas_idx], sas))
    la = sum(upair.get((int(a), int(b)), 0.0) * x for a, b, x in zip(ida, idb, area))
    lv = float(np.dot(v[sas_idx], vol)) if v is not None else 0.0
    return ls + la + lv


def _loss_gpu(balls, probe, w, upair, box=None, v=None):
    r = V.compute_tessellation_result(balls, probe, box, precision="fp64")
    return _loss(r.cell_index.astype(np.int64), r.cell_sas_area, r.id_a, r.id_b, r.area, w, upair,
                 r.cell_volume, v)


def _loss_oracle(balls, probe, w, upair, box=None, v=None):
    o = O.compute(balls, probe, periodic_box=box)
    return _loss(o.cells_index.astype(np.int64), o.cells_sas, o.contacts_a, o.contacts_b, o.contacts_area, w, upair,
                 o.cells_vol, v)


def _coords(n, k, seed):
    rng = np.random.default_rng(seed)
    return [(int(i), int(c)) for i, c in zip(rng.choice(n, k, replace=False), rng.integers(0, 4, k))]


def _fd(loss, balls, i, c, h=H):
    bp, bm = balls.copy(), balls.copy()
    bp[i, c] += h
    bm[i, c] -= h
    return (loss(bp) - loss(bm)) / (2 * h)


def _check_fd(g, loss, balls, i, c):
    fd = _fd(loss, balls, i, c)
    if abs(g - fd) <= TOL * (1 + abs(fd)):
        return
    fd2 = _fd(loss, balls, i, c, H / 10)
    err = abs(g - fd2)
    assert err <= TOL * (1 + abs(fd2)), (f"ball {i} coord {c}: adjoint {g} vs finite differences {fd} (h 1e-4), "
                                        f"{fd2} (h 1e-5)")


def test_adjoint_matches_gpu_finite_differences():
    balls = W.lattice_balls(1500, 21)
    w, u, upair = _weights(balls, 1.4, 1)
    g = V.grad(balls, 1.4, w, u, precision="fp64")
    for i, c in _coords(len(balls), 40, 2):
        _check_fd(g[i, c], lambda b: _loss_gpu(b, 1.4, w, upair), balls, i, c)


def test_adjoint_matches_oracle_finite_differences():
    balls = W.lattice_balls(800, 22)
    w, u, upair = _weights(balls, 1.4, 3)
    g = V.grad(balls, 1.4, w, u, precision="fp64")
    for i, c in _coords(len(balls), 12, 4):
        _check_fd(g[i, c], lambda b: _loss_oracle(b, 1.4, w, upair), balls, i, c)


def _check_fd_local(g, balls, i, c, w, v, upair):
    fd = O.finite_difference_local(balls, 1.4, i, c, H, w, v, upair)
    if abs(g - fd) <= TOL * (1 + abs(fd)):
        return abs(g - fd) / (1 + abs(fd))
    fd2 = O.finite_difference_local(balls, 1.4, i, c, H / 10, w, v, upair)
    err = abs(g - fd2) / (1 + abs(fd2))
    assert err <= TOL, f"ball {i} coord {c}: adjoint {g} vs oracle differences {fd} (h 1e-4), {fd2} (h 1e-5)"
    return err


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_differentiation_config_256_coordinates_vs_oracle(precision):
    """The differentiation workload: 20,000 lattice balls, L = sum w SAS + sum u area with
    w ~ U(0, 1), u ~ N(0, 1); the adjoint after the FP32 and the FP64 forward against the
    oracle's central differences (h = 1e-4 A, f64) at 256 random coordinates (x, y, z, r),
    each difference taken on the sub-structure that determines it
    (oracle.finite_difference_local)."""
    balls = W.lattice_balls(20000, 7)
    o = O.compute(balls, 1.4)
    rng = np.random.default_rng(20)
    w = rng.uniform(0.0, 1.0, len(balls))
    u_o = rng.normal(0.0, 1.0, len(o.contacts_a))
    upair = O.loss_weights_by_pair(o.contacts_a, o.contacts_b, u_o, len(balls))
    r = V.compute_tessellation_result(balls, 1.4, precision=precision)
    k = r.id_a.astype(np.int64) * len(balls) + r.id_b.astype(np.int64)
    pos = np.clip(np.searchsorted(upair[0], k), 0, len(upair[0]) - 1)
    u = np.where(upair[0][pos] == k, upair[1][pos], 0.0)
    g = V.grad(balls, 1.4, w, u, precision=precision)
    errs = [_check_fd_local(g[i, c], balls, i, c, w, None, upair) for i, c in _coords(len(balls), 256, 30)]
    assert len(errs) == 256


def test_volume_adjoint_256_coordinates_vs_oracle():
    """The same 20,000-ball structure with the volume term: L = sum w SAS + sum v V +
    sum u area, v ~ U(0, 1), 256 coordinates against the oracle's central differences."""
    balls = W.lattice_balls(20000, 7)
    o = O.compute(balls, 1.4)
    rng = np.random.default_rng(21)
    w = rng.uniform(0.0, 1.0, len(balls))
    v = rng.uniform(0.0, 1.0, len(balls))
    u = rng.normal(0.0, 1.0, len(o.contacts_a))
    upair = O.loss_weights_by_pair(o.contacts_a, o.contacts_b, u, len(balls))
    g = V.grad(balls, 1.4, w, u, precision="fp64", v_volume=v)
    for i, c in _coords(len(balls), 256, 31):
        _check_fd_local(g[i, c], balls, i, c, w, v, upair)


@pytest.mark.parametrize("k, rr, rho, probe", [(40, 0.1, 3.3, 0.1), (48, 1.0, 3.6, 0.5)])
def test_adjoint_of_contours_beyond_a_warp(k, rr, rho, probe):
    """A contact cut by k small balls on a ring (contours of 40 to 96 points, more than a
    warp holds): the serial adjoint against central differences of the GPU forward and of
    the oracle, for the SAS, area and volume terms (the ring jittered so that no step of
    the differences meets a symmetric degeneracy)."""
    from common import sunflower

    balls = sunflower(k, rr=rr, rho=rho)
    rng = np.random.default_rng(k)
    balls[2:, :3] += rng.uniform(-0.03, 0.03, (k, 3))
    w, u, upair = _weights(balls, probe, 50 + k)
    v = _vweights(len(balls), 60 + k)
    g = V.grad(balls, probe, w, u, precision="fp64", v_volume=v)
    coords = [(0, 0), (0, 1), (0, 3), (1, 0), (1, 2), (1, 3)] + _coords(len(balls), 6, 70 + k)
    for i, c in coords:
        _check_fd(g[i, c], lambda b: _loss_gpu(b, probe, w, upair, v=v), balls, i, c)
    for i, c in coords[:6]:
        _check_fd(g[i, c], lambda b: _loss_oracle(b, probe, w, upair, v=v), balls, i, c)


def test_separate_terms_and_fp32_forward():
    balls = W.lattice_balls(1200, 23)
    w, u, upair = _weights(balls, 1.4, 5)
    g_s = V.grad(balls, 1.4, w, None, precision="fp64")
    g_a = V.grad(balls, 1.4, None, u, precision="fp64")
    g = V.grad(balls, 1.4, w, u, precision="fp64")
    assert np.allclose(g, g_s + g_a, rtol=1e-12, atol=1e-9)
    # FP32 forward: same pair set; the adjoint takes each contour's topology from an FP32
    # recomputation (FP64 for pairs in the band) and its vertices and arc angles in FP64,
    # so x, y, z agree to rounding; r also carries the SAS scaling term 2 w SAS / R with the
    # forward's FP32 cell SAS (per-cell relative error up to ~1e-4)
    g32 = V.grad(balls, 1.4, w, u, precision="fp32")
    assert np.allclose(g32[:, :3], g[:, :3], rtol=1e-9, atol=1e-9)
    assert np.allclose(g32[:, 3], g[:, 3], rtol=1e-4, atol=1e-4)
    for i, c in _coords(len(balls), 10, 6):
        _check_fd(g_s[i, c], lambda b: _loss_gpu(b, 1.4, w, {}), balls, i, c)


def test_periodic_adjoint():
    balls, side = W.periodic_box_balls(1500, seed=7)
    box = {"corners": [(0.0, 0.0, 0.0), (side, side, side)]}
    w, u, upair = _weights(balls, 1.4, 8, box)
    g = V.grad(balls, 1.4, w, u, box, precision="fp64")
    for i, c in _coords(len(balls), 16, 9):
        _check_fd(g[i, c], lambda b: _loss_gpu(b, 1.4, w, upair, box), balls, i, c)


def _vweights(n, seed):
    return np.random.default_rng(seed).uniform(0.0, 1.0, n)


def test_volume_adjoint_matches_gpu_finite_differences():
    balls = W.lattice_balls(1500, 31)
    w, u, upair = _weights(balls, 1.4, 31)
    v = _vweights(len(balls), 32)
    g = V.grad(balls, 1.4, w, u, precision="fp64", v_volume=v)
    for i, c in _coords(len(balls), 40, 33):
        _check_fd(g[i, c], lambda b: _loss_gpu(b, 1.4, w, upair, v=v), balls, i, c)


def test_volume_adjoint_alone_matches_oracle_finite_differences():
    """Only the volume term (w = 0, u = 0), against the CPU oracle; includes exposed and
    buried balls of a small structure and a radius coordinate of each kind."""
    balls = W.lattice_balls(600, 34)
    v = _vweights(len(balls), 35)
    z = np.zeros(len(balls))
    g = V.grad(balls, 1.4, None, None, precision="fp64", v_volume=v)
    g_sum = V.grad(balls, 1.4, z, None, precision="fp64", v_volume=v)
    assert np.allclose(g, g_sum, rtol=1e-12, atol=1e-12)
    for i, c in _coords(len(balls), 16, 36):
        _check_fd(g[i, c], lambda b: _loss_oracle(b, 1.4, z, {}, v=v), balls, i, c)


def test_volume_terms_add_and_fp32_forward():
    balls = W.lattice_balls(1200, 37)
    w, u, upair = _weights(balls, 1.4, 37)
    v = _vweights(len(balls), 38)
    g_v = V.grad(balls, 1.4, None, None, precision="fp64", v_volume=v)
    g_wu = V.grad(balls, 1.4, w, u, precision="fp64")
    g = V.grad(balls, 1.4, w, u, precision="fp64", v_volume=v)
    assert np.allclose(g, g_v + g_wu, rtol=1e-12, atol=1e-9)
    g32 = V.grad(balls, 1.4, w, u, precision="fp32", v_volume=v)
    # x, y, z: the FP32 adjoint snaps vertices to FP64; the volume terms use the forward's
    # FP32 areas and SAS (relative error ~1e-6 per contact, ~1e-4 per cell SAS)
    assert np.allclose(g32[:, :3], g[:, :3], rtol=1e-5, atol=1e-5)
    assert np.allclose(g32[:, 3], g[:, 3], rtol=1e-4, atol=1e-4)


def test_periodic_volume_adjoint():
    balls, side = W.periodic_box_balls(1500, seed=39)
    box = {"corners": [(0.0, 0.0, 0.0), (side, side, side)]}
    w, u, upair = _weights(balls, 1.4, 39, box)
    v = _vweights(len(balls), 40)
    g = V.grad(balls, 1.4, w, u, box, precision="fp64", v_volume=v)
    for i, c in _coords(len(balls), 16, 41):
        _check_fd(g[i, c], lambda b: _loss_gpu(b, 1.4, w, upair, box, v=v), balls, i, c)


@pytest.mark.parametrize("periodic", [False, True])
def test_kept_contours_give_the_same_adjoint(periodic):
    """An FP32 forward that keeps its contours lets the adjoint skip their recomputation;
    the gradient is the one the recomputing adjoint gives."""
    import torch

    if periodic:
        balls, side = W.periodic_box_balls(3000, seed=42)
        box = V.parse_periodic_box({"corners": [(0.0, 0.0, 0.0), (side, side, side)]})
    else:
        balls, box = W.lattice_balls(4000, 42), None
    n = len(balls)
    rng = np.random.default_rng(43)
    d = torch.from_numpy(balls).cuda()
    w = torch.from_numpy(rng.uniform(0.0, 1.0, n)).cuda()
    v = torch.from_numpy(rng.uniform(0.0, 1.0, n)).cuda()
    grads = []
    for keep in (False, True):
        e = V.Engine()
        e.set_keep_contours(keep)
        e.compute_device(d.data_ptr(), n, 1.4, box, precision="fp32")
        r = e.download()
        u = torch.from_numpy(np.random.default_rng(44).normal(0.0, 1.0, len(r.id_a))).cuda()
        g = torch.empty((n, 4), dtype=torch.float64, device="cuda")
        e.grad_device(w.data_ptr(), u.data_ptr(), g.data_ptr(), v.data_ptr())
        torch.cuda.synchronize()
        grads.append(g.cpu().numpy())
        e.close()
    assert np.allclose(grads[0], grads[1], rtol=1e-12, atol=1e-12)


def test_torch_autograd_matches_c_abi():
    import torch

    from voronota_ltr.autograd import tessellate

    balls = W.lattice_balls(1000, 24)
    w, u, _ = _weights(balls, 1.4, 10)
    v = _vweights(len(balls), 11)
    x = torch.from_numpy(balls).cuda().requires_grad_(True)
    sas, vol, area, ida, idb = tessellate(x, 1.4, precision="fp64")
    r = V.compute_tessellation_result(balls, 1.4, precision="fp64")
    assert np.array_equal(ida.cpu().numpy(), r.id_a.astype(np.int64))
    assert np.allclose(vol.detach().cpu().numpy()[r.cell_index.astype(np.int64)], r.cell_volume, rtol=1e-12)
    loss = ((torch.from_numpy(w).cuda() * sas).sum() + (torch.from_numpy(u).cuda() * area).sum()
            + (torch.from_numpy(v).cuda() * vol).sum())
    loss.backward()
    g = V.grad(balls, 1.4, w, u, precision="fp64", v_volume=v)
    assert np.allclose(x.grad.cpu().numpy(), g, rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_updateable_sas_adjoint_matches_stateless(precision):
    import torch

    balls = W.lattice_balls(2000, 25)
    t = V.UpdateableTessellation(precision=precision)
    assert t.init(balls, 1.4)
    rng = np.random.default_rng(3)
    for _ in range(3):
        ids = np.sort(rng.choice(len(balls), 20, replace=False))
        balls[ids, :3] += rng.normal(0.0, 0.05, (20, 3))
        assert t.update_with_changed(balls, ids)
    w = rng.uniform(0.0, 1.0, len(balls))
    dw = torch.from_numpy(w).cuda()
    dg = torch.empty((len(balls), 4), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    t.grad_sas_device(dw.data_ptr(), dg.data_ptr())
    g = V.grad(balls, 1.4, w, None, precision=precision)
    gu = dg.cpu().numpy()
    # The handle's adjoint gathers per-contact coefficients recorded when each contact was
    # computed (arc length and first moment of its arcs): exact for FP64 contacts, FP32
    # rounding of the arc end points otherwise; r also carries 2 w SAS / R with each
    # path's own cell SAS (FP32: per-cell error ~1e-4).
    tol_xyz = 1e-9 if precision == "fp64" else 2e-5
    tol_r = 1e-9 if precision == "fp64" else 1e-4
    assert np.allclose(gu[:, :3], g[:, :3], rtol=tol_xyz, atol=tol_xyz)
    assert np.allclose(gu[:, 3], g[:, 3], rtol=tol_r, atol=tol_r)
    # the total SAS (w = 1)
    t.grad_sas_device(0, dg.data_ptr())
    g1 = V.grad(balls, 1.4, np.ones(len(balls)), None, precision=precision)
    assert np.allclose(dg.cpu().numpy()[:, :3], g1[:, :3], rtol=tol_xyz, atol=tol_xyz)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_updateable_volume_adjoint_matches_stateless(precision):
    """The handle's adjoint of sum w SAS + sum v V (per-entry face coefficients gathered,
    Reynolds' transport form) against the stateless adjoint (pyramid-volume form) on the
    same positions after a few updates: two derivations of one gradient."""
    import torch

    balls = W.lattice_balls(2000, 26)
    t = V.UpdateableTessellation(precision=precision)
    assert t.init(balls, 1.4)
    rng = np.random.default_rng(6)
    for _ in range(3):
        ids = np.sort(rng.choice(len(balls), 20, replace=False))
        balls[ids, :3] += rng.normal(0.0, 0.05, (20, 3))
        assert t.update_with_changed(balls, ids)
    w = rng.uniform(0.0, 1.0, len(balls))
    v = rng.uniform(0.0, 1.0, len(balls))
    dw, dv = torch.from_numpy(w).cuda(), torch.from_numpy(v).cuda()
    dg = torch.empty((len(balls), 4), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    t.grad_device(0, dv.data_ptr(), dg.data_ptr())
    g_v = V.grad(balls, 1.4, None, None, precision=precision, v_volume=v)
    tol = 1e-8 if precision == "fp64" else 1e-4
    assert np.allclose(dg.cpu().numpy(), g_v, rtol=tol, atol=tol)
    t.grad_device(dw.data_ptr(), dv.data_ptr(), dg.data_ptr())
    g = V.grad(balls, 1.4, w, None, precision=precision, v_volume=v)
    assert np.allclose(dg.cpu().numpy(), g, rtol=tol, atol=tol)
    # the SAS-only entry point is the w-only case
    t.grad_sas_device(dw.data_ptr(), dg.data_ptr())
    t2 = torch.empty_like(dg)
    t.grad_device(dw.data_ptr(), 0, t2.data_ptr())
    assert torch.equal(dg, t2)


def test_updateable_volume_adjoint_periodic_finite_differences():
    import torch

    balls, side = W.periodic_box_balls(1500, seed=14)
    box = {"corners": [(0.0, 0.0, 0.0), (side, side, side)]}
    t = V.UpdateableTessellation(precision="fp64")
    assert t.init(balls, 1.4, box)
    rng = np.random.default_rng(7)
    for _ in range(2):
        ids = np.sort(rng.choice(len(balls), 15, replace=False))
        balls[ids, :3] += rng.normal(0.0, 0.05, (15, 3))
        assert t.update_with_changed(balls, ids)
    v = rng.uniform(0.0, 1.0, len(balls))
    dv = torch.from_numpy(v).cuda()
    dg = torch.empty((len(balls), 4), dtype=torch.float64, device="cuda")
    t.grad_device(0, dv.data_ptr(), dg.data_ptr())
    g = dg.cpu().numpy()

    def loss(b):
        u = V.UpdateableTessellation(precision="fp64")
        u.init(b, 1.4, box)
        s = u.summary()
        return float(np.dot(v[s.cell_index.astype(np.int64)], s.cell_volume))

    for i, c in _coords(len(balls), 12, 15):
        _check_fd(g[i, c], loss, balls, i, c)


def test_updateable_sas_adjoint_periodic_finite_differences():
    import torch

    balls, side = W.periodic_box_balls(1500, seed=12)
    box = {"corners": [(0.0, 0.0, 0.0), (side, side, side)]}
    t = V.UpdateableTessellation(precision="fp64")
    assert t.init(balls, 1.4, box)
    rng = np.random.default_rng(4)
    for _ in range(2):
        ids = np.sort(rng.choice(len(balls), 15, replace=False))
        balls[ids, :3] += rng.normal(0.0, 0.05, (15, 3))
        assert t.update_with_changed(balls, ids)
    dg = torch.empty((len(balls), 4), dtype=torch.float64, device="cuda")
    t.grad_sas_device(0, dg.data_ptr())
    g = dg.cpu().numpy()
    w = np.ones(len(balls))

    def loss(b):
        u = V.UpdateableTessellation(precision="fp64")
        u.init(b, 1.4, box)
        s = u.summary()
        return float(np.dot(w[s.cell_index.astype(np.int64)], s.cell_sas_area))

    for i, c in _coords(len(balls), 10, 13):
        _check_fd(g[i, c], loss, balls, i, c)


def test_updateable_adjoint_switch():
    """With the adjoint off the updates give the same summary and grad_sas is refused until
    an init with it on; back on, the adjoint equals a handle that always had it."""
    import torch
    balls, side = W.periodic_box_balls(1500, seed=13)
    box = {"corners": [(0.0, 0.0, 0.0), (side, side, side)]}
    d = torch.from_numpy(balls).cuda()
    on = V.UpdateableTessellation(precision="fp32")
    off = V.UpdateableTessellation(precision="fp32")
    off.set_adjoint(False)
    on.init_device(d.data_ptr(), len(balls), 1.4, box)
    off.init_device(d.data_ptr(), len(balls), 1.4, box)
    rng = np.random.default_rng(5)
    ids = np.sort(rng.choice(len(balls), 15, replace=False)).astype(np.int64)
    d[torch.from_numpy(ids).cuda(), :3] += 0.05
    ti = torch.from_numpy(ids).cuda()
    on.update_with_changed_device(d.data_ptr(), len(balls), ti.data_ptr(), len(ids))
    off.update_with_changed_device(d.data_ptr(), len(balls), ti.data_ptr(), len(ids))
    a, b = on.summary(), off.summary()
    assert np.array_equal(a.id_a, b.id_a) and np.array_equal(a.area, b.area)
    assert np.array_equal(a.cell_sas_area, b.cell_sas_area)
    g = torch.empty((len(balls), 4), dtype=torch.float64, device="cuda")
    with pytest.raises(V.VoronotaError):
        off.grad_sas_device(0, g.data_ptr())
    off.set_adjoint(True)
    off.update_with_changed_device(d.data_ptr(), len(balls), ti.data_ptr(), len(ids))  # no change: still refused
    with pytest.raises(V.VoronotaError):
        off.grad_sas_device(0, g.data_ptr())
    off.init_device(d.data_ptr(), len(balls), 1.4, box)
    off.grad_sas_device(0, g.data_ptr())
    g_on = torch.empty_like(g)
    fresh = V.UpdateableTessellation(precision="fp32")
    fresh.init_device(d.data_ptr(), len(balls), 1.4, box)
    fresh.grad_sas_device(0, g_on.data_ptr())
    assert torch.equal(g, g_on)
