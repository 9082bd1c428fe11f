"""Batched tessellation: many independent structures in one call.

Each structure of a batch must come out exactly as a single compute_tessellation call on
it alone: the batched path runs the same kernels over a concatenated ball array with
one grid per structure, so contacts (ids local to the structure, order, central bits,
areas, arc lengths) and cells are compared bit for bit with single GPU calls, in both
precisions; per-structure totals (a different summation tree) within 1e-12 relative.
FP32 mode computes a structure with fewer than 2048 candidate pairs in FP64, alone or in
a batch (there its pairs go to the FP64 recompute), so the two agree bit for bit.
Structures are also checked against the oracle, and uneven sizes, empty structures and
malformed offsets are covered.
"""
import numpy as np
import pytest

import oracle as O
import voronota_ltr as V
from gpu_util import compare
from voronota_ltr import workloads as W

pytestmark = pytest.mark.gpu


def _structures(count, lo, hi, seed):
    sizes = W.batch_sizes(count, lo, hi, seed)
    return [W.lattice_balls(int(n), 1000 + i) for i, n in enumerate(sizes)]


def _same(a, b):
    assert np.array_equal(a.id_a, b.id_a) and np.array_equal(a.id_b, b.id_b)
    assert np.array_equal(a.central, b.central)
    assert np.array_equal(a.area, b.area) and np.array_equal(a.arc_length, b.arc_length)
    assert np.array_equal(a.cell_index, b.cell_index)
    assert np.array_equal(a.cell_sas_area, b.cell_sas_area) and np.array_equal(a.cell_volume, b.cell_volume)
    for x, y in ((a.total_sas_area, b.total_sas_area), (a.total_volume, b.total_volume),
                 (a.total_contact_area, b.total_contact_area)):
        assert abs(x - y) <= 1e-12 * max(1.0, abs(y))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_equals_single_calls(precision):
    structs = _structures(40, 30, 3000, 3)
    structs.insert(7, np.zeros((0, 4)))  # an empty structure
    structs.append(np.array([[0.0, 0.0, 0.0, 1.5]]))  # a lone ball: one detached cell
    r = V.compute_batch(structs, 1.4, precision)
    assert len(r) == len(structs)
    for s, balls in enumerate(structs):
        single = V.compute_tessellation_result(balls, 1.4, precision=precision)
        _same(r.structure(s), single)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_against_oracle(precision):
    structs = _structures(12, 300, 4000, 11)
    r = V.compute_batch(structs, 1.4, precision)
    for s, balls in enumerate(structs):
        compare(r.structure(s), O.compute(balls, 1.4), precision)


def test_batch_device_engine_and_offsets_form():
    import torch

    structs = _structures(25, 100, 2000, 5)
    balls = np.concatenate(structs)
    off = np.zeros(len(structs) + 1, np.uint64)
    off[1:] = np.cumsum([len(x) for x in structs])
    host = V.compute_batch((balls, off), 1.4, "fp32")
    e = V.Engine()
    d = torch.from_numpy(balls).cuda()
    torch.cuda.synchronize()
    e.compute_batch_device(d.data_ptr(), off, 1.4, "fp32")
    dev = e.download_batch()
    assert np.array_equal(host.contact_off, dev.contact_off) and np.array_equal(host.cell_off, dev.cell_off)
    assert np.array_equal(host.all.area, dev.all.area)
    # contacts-only batch: same contacts as the full batch, no cells; areas agree within
    # the FP32 tolerance (the full call recomputes in FP64 the pairs of cells whose SAS
    # branch or exposure is within the FP32 band)
    e.compute_batch_device(d.data_ptr(), off, 1.4, "fp32", contacts_only=True)
    co = e.download_batch()
    assert np.array_equal(co.all.id_a, host.all.id_a) and np.array_equal(co.all.id_b, host.all.id_b)
    assert np.abs(co.all.area - host.all.area).max(initial=0) <= 1e-3
    assert len(co.all.cell_index) == 0


def test_batch_rejects_bad_offsets():
    balls = W.lattice_balls(50, 1)
    for off in ([1, 50], [0, 30, 20, 50], [0]):
        with pytest.raises(V.VoronotaError) as ei:
            V.compute_batch((balls, np.array(off, np.uint64)), 1.4)
        assert ei.value.status == V.VT_ERR_INVALID
