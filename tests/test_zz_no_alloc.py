"""The allocation-free entry point (vt_contact_descriptors_noalloc) against the regular one.

Callers that cannot allocate device memory while they run (a custom call inside a
framework that owns the device allocator, a real-time loop that must not hit
cudaMalloc) use vt_contact_descriptors_noalloc, whose scratch is a static device array.
This test calls it twice in a row through the C ABI on the neighbour lists and pairs of a
2,000-ball structure and checks each call's contacts against vt_compute_tessellation
(FP64 path): the same pair set and central bits, areas and arc lengths within 1e-9
relative (the FP64 tolerance of the other parity tests).  It also checks that a
neighbour list longer than the scratch allows is rejected with VT_ERR_CAPACITY.
The file is named to be collected last.
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
    t_sph = torch.from_numpy(spheres).to(dev)
    t_off = torch.from_numpy(o.nb_offsets.astype(np.uint32).view(np.int32)).to(dev)
    t_idx = torch.from_numpy(o.nb_ids.astype(np.uint32).view(np.int32)).to(dev)
    pa = o.pairs["a"].astype(np.uint32)
    pb = o.pairs["b"].astype(np.uint32)
    t_pa = torch.from_numpy(pa.view(np.int32)).to(dev)
    t_pb = torch.from_numpy(pb.view(np.int32)).to(dev)
    P = len(pa)
    for call in range(2):
        st = torch.full((P,), 7, dtype=torch.uint8, device=dev)
        area = torch.full((P,), -1.0, dtype=torch.float64, device=dev)
        arc = torch.full((P,), -1.0, dtype=torch.float64, device=dev)
        cen = torch.full((P,), 7, dtype=torch.uint8, device=dev)
        outs = [torch.zeros(P, dtype=torch.float64, device=dev) for _ in range(4)]
        torch.cuda.synchronize()
        rc = fn(t_sph.data_ptr(), len(spheres), t_off.data_ptr(), t_idx.data_ptr(), t_pa.data_ptr(),
                t_pb.data_ptr(), P, st.data_ptr(), area.data_ptr(), arc.data_ptr(), cen.data_ptr(),
                *[x.data_ptr() for x in outs], torch.cuda.current_stream().cuda_stream)
        assert rc == 0, L.vt_last_error()
        s = st.cpu().numpy()
        assert set(np.unique(s).tolist()) <= {0, 1}, f"call {call}: unexpected status {np.unique(s)}"
        valid = s == 1
        assert np.array_equal(pa[valid], ref.id_a), f"call {call}: id_a differ"
        assert np.array_equal(pb[valid], ref.id_b), f"call {call}: id_b differ"
        a = area.cpu().numpy()[valid]
        r = arc.cpu().numpy()[valid]
        c = cen.cpu().numpy()[valid].astype(bool)
        assert np.all(np.abs(a - ref.area) <= 1e-9 * (1 + np.abs(ref.area))), f"call {call}"
        assert np.all(np.abs(r - ref.arc_length) <= 1e-9 * (1 + np.abs(ref.arc_length))), f"call {call}"
        assert np.array_equal(c, ref.central), f"call {call}: central differ"


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
