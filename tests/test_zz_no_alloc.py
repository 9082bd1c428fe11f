"""The allocation-free entry point (vt_contact_descriptors_noalloc) against the regular one.

Callers that cannot allocate device memory while they run (a custom call inside a
framework that owns the device allocator, a real-time loop that must not hit
cudaMalloc) use vt_contact_descriptors_noalloc, whose scratch is a static device array.
This test calls it twice in a row through the C ABI on the neighbour lists and pairs of a
2,000-ball structure and checks each call's contacts against vt_compute_tessellation
(FP64 path): the same pair set and central bits, areas and arc lengths within 1e-9
relative (the FP64 tolerance of the other parity tests), and the solid angles and
pyramid volumes both per pair (against the oracle's contact descriptors) and summed per
ball through the reference's compute_sas (against the regular path's cell SAS areas and
volumes).  A random cloud whose listed balls have up to the 57-neighbour limit checks the
long contours the same way.  Neighbour lists longer than the scratch allows are rejected
with VT_ERR_CAPACITY, and malformed input (a neighbour index past the spheres, offsets
out of order, a non-finite coordinate, a negative radius) with VT_ERR_INVALID before any
contact is computed.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
import voronota_ltr as V
from voronota_ltr import workloads as W

pytestmark = pytest.mark.gpu

_c = ctypes.c_void_p


def _bind():
    L = V.library()
    f = L.vt_contact_descriptors_noalloc
    f.argtypes = [_c, ctypes.c_uint64, _c, _c, _c, _c, ctypes.c_uint64] + [_c] * 8 + [_c]
    f.restype = ctypes.c_int
    return L, f


def _inputs(balls, probe):
    o = O.compute(balls, probe, internals=True)
    spheres = np.ascontiguousarray(balls.copy())
    spheres[:, 3] += probe
    return o, spheres


def _close(x, y, tol=1e-9):
    return bool(np.all(np.abs(x - y) <= tol * (1 + np.abs(y))))


def _cells_from_descriptors(n, radii, pa, pb, area, arc, sa, sb, va, vb):
    """Per-ball SAS and volume from per-pair descriptors, following the reference's
    CellContactSummary::add and compute_sas (src/types.rs:589-663); balls without a
    contact get no cell (those are checked elsewhere)."""
    ids = np.concatenate([pa, pb]).astype(np.int64)
    s = np.concatenate([sa, sb])
    v = np.concatenate([va, vb])
    arcs = np.concatenate([arc, arc])
    pos_s = np.bincount(ids, np.maximum(s, 0.0), n)
    neg_s = np.bincount(ids, -np.minimum(s, 0.0), n)
    pos_v = np.bincount(ids, np.maximum(v, 0.0), n)
    neg_v = np.bincount(ids, -np.minimum(v, 0.0), n)
    arc_sum = np.bincount(ids, arcs, n)
    has = np.bincount(ids, np.ones(len(ids)), n) > 0
    sas = np.zeros(n)
    vol = pos_v - neg_v
    for i in np.nonzero(has)[0]:
        r = radii[i]
        diff = abs(pos_s[i] - neg_s[i])
        if arc_sum[i] > 0.0 and diff > 1e-10:
            if pos_s[i] > neg_s[i]:
                sas[i] = (4.0 * np.pi - max(pos_s[i] - neg_s[i], 0.0)) * r * r
            else:
                sas[i] = max(neg_s[i] - pos_s[i], 0.0) * r * r
            v_i = sas[i] * r / 3.0 + pos_v[i] - neg_v[i]
            if v_i > 4.0 / 3.0 * np.pi * r ** 3:
                sas[i] = 0.0
            else:
                vol[i] = v_i
    return has, sas, vol


def _to_dev(x, dev):
    import torch

    if x.dtype == np.uint32:
        x = x.view(np.int32)
    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


def _call(fn, dev, spheres, off, idx, pa, pb, descriptors=True):
    import torch

    P = len(pa)
    t = [_to_dev(x, dev) for x in (spheres, off, idx, pa, pb)]
    st = torch.full((P,), 7, dtype=torch.uint8, device=dev)
    area = torch.full((P,), -1.0, dtype=torch.float64, device=dev)
    arc = torch.full((P,), -1.0, dtype=torch.float64, device=dev)
    cen = torch.full((P,), 7, dtype=torch.uint8, device=dev)
    outs = [torch.full((P,), -7.0, dtype=torch.float64, device=dev) for _ in range(4)]
    torch.cuda.synchronize()
    rc = fn(t[0].data_ptr(), len(spheres), t[1].data_ptr(), t[2].data_ptr(), t[3].data_ptr(), t[4].data_ptr(), P,
            st.data_ptr(), area.data_ptr(), arc.data_ptr(), cen.data_ptr(),
            *([x.data_ptr() for x in outs] if descriptors else [None] * 4), torch.cuda.current_stream().cuda_stream)
    return rc, {"status": st.cpu().numpy(), "area": area.cpu().numpy(), "arc": arc.cpu().numpy(),
                "central": cen.cpu().numpy().astype(bool), "solid_a": outs[0].cpu().numpy(),
                "solid_b": outs[1].cpu().numpy(), "pyr_a": outs[2].cpu().numpy(), "pyr_b": outs[3].cpu().numpy()}


def _check_against_oracle_pairs(r, o, keep, tag):
    """Per-pair outputs against the oracle's contact descriptors of the same pairs."""
    valid = o.pairs["valid"][keep].astype(bool)
    assert np.array_equal(r["status"] == 1, valid), f"{tag}: status differ"
    for k in ("area", "arc", "solid_a", "solid_b", "pyr_a", "pyr_b"):
        assert _close(r[k][valid], o.pairs[k][keep][valid]), f"{tag}: {k} differ"
    assert np.array_equal(r["central"][valid], o.pairs["central"][keep][valid].astype(bool)), f"{tag}: central"


def test_noalloc_matches_regular_entry_point_twice():
    import torch

    L, fn = _bind()
    balls = W.lattice_balls(2000, 0)
    probe = 1.4
    o, spheres = _inputs(balls, probe)
    counts = np.diff(o.nb_offsets.astype(np.int64))
    assert counts.max() <= 57
    ref = V.compute_tessellation_result(balls, probe, precision="fp64")

    dev = torch.device("cuda:0")
    off = o.nb_offsets.astype(np.uint32)
    idx = o.nb_ids.astype(np.uint32)
    pa = o.pairs["a"].astype(np.uint32)
    pb = o.pairs["b"].astype(np.uint32)
    for call in range(2):
        rc, r = _call(fn, dev, spheres, off, idx, pa, pb)
        assert rc == 0, L.vt_last_error()
        s = r["status"]
        assert set(np.unique(s).tolist()) <= {0, 1}, f"call {call}: unexpected status {np.unique(s)}"
        valid = s == 1
        assert np.array_equal(pa[valid], ref.id_a), f"call {call}: id_a differ"
        assert np.array_equal(pb[valid], ref.id_b), f"call {call}: id_b differ"
        assert _close(r["area"][valid], ref.area), f"call {call}"
        assert _close(r["arc"][valid], ref.arc_length), f"call {call}"
        assert np.array_equal(r["central"][valid], ref.central), f"call {call}: central differ"
        _check_against_oracle_pairs(r, o, np.ones(len(pa), bool), f"call {call}")
        # solid angles and pyramid volumes summed per ball against the regular path's cells
        has, sas, vol = _cells_from_descriptors(len(balls), spheres[:, 3], pa[valid], pb[valid], r["area"][valid],
                                                r["arc"][valid], r["solid_a"][valid], r["solid_b"][valid],
                                                r["pyr_a"][valid], r["pyr_b"][valid])
        ci = ref.cell_index.astype(np.int64)
        with_contacts = has[ci]
        assert with_contacts.sum() > 0.9 * len(ci)
        assert _close(sas[ci][with_contacts], ref.cell_sas_area[with_contacts]), f"call {call}: cell SAS"
        assert _close(vol[ci][with_contacts], ref.cell_volume[with_contacts]), f"call {call}: cell volume"


def test_noalloc_long_lists_random_cloud():
    """A random cloud where many listed balls have 50-57 neighbours (the long contours the
    192-point slots are sized for); pairs of balls beyond the limit are left out."""
    import torch

    L, fn = _bind()
    rng = np.random.default_rng(5)
    n, side, probe = 3000, 38.0, 1.4
    balls = np.column_stack([rng.uniform(0, side, (n, 3)), rng.uniform(1.0, 2.2, n)])
    o, spheres = _inputs(balls, probe)
    counts = np.diff(o.nb_offsets.astype(np.int64))
    pa_all = o.pairs["a"].astype(np.int64)
    keep = counts[pa_all] <= 57
    assert ((counts >= 50) & (counts <= 57)).sum() > 100
    dev = torch.device("cuda:0")
    pa = o.pairs["a"][keep].astype(np.uint32)
    pb = o.pairs["b"][keep].astype(np.uint32)
    for call in range(2):
        rc, r = _call(fn, dev, spheres, o.nb_offsets.astype(np.uint32), o.nb_ids.astype(np.uint32), pa, pb)
        assert rc == 0, L.vt_last_error()
        _check_against_oracle_pairs(r, o, keep, f"cloud call {call}")


def test_noalloc_rejects_malformed_input():
    """Each malformed input is refused with VT_ERR_INVALID by the check that runs before
    the contact kernel (which therefore never reads past the caller's buffers)."""
    import torch

    L, fn = _bind()
    dev = torch.device("cuda:0")
    balls = W.lattice_balls(300, 0)
    o, spheres = _inputs(balls, 1.4)
    off = o.nb_offsets.astype(np.uint32)
    idx = o.nb_ids.astype(np.uint32)
    pa = o.pairs["a"].astype(np.uint32)
    pb = o.pairs["b"].astype(np.uint32)
    rc, _ = _call(fn, dev, spheres, off, idx, pa, pb)
    assert rc == 0, L.vt_last_error()
    bad_idx = idx.copy()
    bad_idx[off[pa[0]]] = len(spheres) + 5  # a neighbour of a listed ball past the spheres
    rc, _ = _call(fn, dev, spheres, off, bad_idx, pa, pb)
    assert rc == V.VT_ERR_INVALID and b"index" in L.vt_last_error()
    bad_off = off.copy()
    bad_off[pa[0] + 1] = bad_off[-1] + 3  # a list running past the index array
    rc, _ = _call(fn, dev, spheres, bad_off, idx, pa, pb)
    assert rc == V.VT_ERR_INVALID
    bad_pair = pb.copy()
    bad_pair[-1] = len(spheres)
    rc, _ = _call(fn, dev, spheres, off, idx, pa, bad_pair)
    assert rc == V.VT_ERR_INVALID
    for col, val in ((0, np.nan), (3, -1.0), (2, np.inf)):
        bad = spheres.copy()
        bad[idx[off[pa[0]]], col] = val  # a neighbour the first pair reads
        rc, _ = _call(fn, dev, bad, off, idx, pa, pb, descriptors=False)
        assert rc == V.VT_ERR_INVALID and b"finite" in L.vt_last_error(), (col, val)
    # the entry point still works after the refusals
    rc, r = _call(fn, dev, spheres, off, idx, pa, pb)
    assert rc == 0 and (r["status"] == 1).sum() > 0


def test_noalloc_rejects_long_neighbour_lists():
    import torch

    L, fn = _bind()
    dev = torch.device("cuda:0")
    n = 70
    spheres = np.column_stack([np.arange(n) * 0.1, np.zeros(n), np.zeros(n), np.full(n, 3.0)])
    t_sph = torch.from_numpy(np.ascontiguousarray(spheres)).to(dev)
    offs = np.zeros(n + 1, np.int32)
    offs[1:] = 60  # ball 0 lists 60 neighbours, more than the scratch allows
    t_off = torch.from_numpy(offs).to(dev)
    t_idx = torch.from_numpy(np.arange(1, 61, dtype=np.int32)).to(dev)
    t_pa = torch.zeros(1, dtype=torch.int32, device=dev)
    t_pb = torch.ones(1, dtype=torch.int32, device=dev)
    st = torch.zeros(1, dtype=torch.uint8, device=dev)
    area = torch.zeros(1, dtype=torch.float64, device=dev)
    arc = torch.zeros(1, dtype=torch.float64, device=dev)
    cen = torch.zeros(1, dtype=torch.uint8, device=dev)
    rc = fn(t_sph.data_ptr(), n, t_off.data_ptr(), t_idx.data_ptr(), t_pa.data_ptr(), t_pb.data_ptr(), 1,
            st.data_ptr(), area.data_ptr(), arc.data_ptr(), cen.data_ptr(), None, None, None, None,
            torch.cuda.current_stream().cuda_stream)
    assert rc == V.VT_ERR_CAPACITY
    assert b"57" in L.vt_last_error()
