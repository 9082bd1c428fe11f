"""The autotuner's launch configurations change speed, never results.

Warps per block of the FP32 contact kernel (2, 4, 8), its persistent work-queue launch
(chunks of 4 or 16 pairs) and the grid cell scale (1, 1.25, 1.5) are swept on one structure (single and periodic) and on a batch: every configuration
gives bit-identical contacts and cells.  The autotuner then picks one of the candidates.
"""
import numpy as np
import pytest

import voronota_ltr as V
from voronota_ltr import workloads as W

pytestmark = pytest.mark.gpu


def _same(a, b):
    for x, y in ((a.id_a, b.id_a), (a.id_b, b.id_b), (a.area, b.area), (a.arc_length, b.arc_length),
                 (a.central, b.central), (a.cell_index, b.cell_index), (a.cell_sas_area, b.cell_sas_area),
                 (a.cell_volume, b.cell_volume)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("periodic", [False, True])
def test_configurations_give_identical_results(periodic):
    import torch

    if periodic:
        balls, side = W.periodic_box_balls(4000, seed=5)
        box = {"corners": [(0.0, 0.0, 0.0), (side, side, side)]}
    else:
        balls, box = W.lattice_balls(5000, 31), None
    e = V.Engine()
    d = torch.from_numpy(balls).cuda()
    torch.cuda.synchronize()
    ref = None
    configs = [(w, c, 0) for w in (2, 4, 8) for c in (0.5, 1.0, 1.5)] + [(2, 0.75, 4), (8, 1.0, 16), (2, 0.5, 4)]
    for w, c, ch in configs:
        e.set_tuning(w, c, ch)
        assert e.tuning() == {"warps_per_block": w, "cell_scale": c, "chunk": ch}
        e.compute_device(d.data_ptr(), len(balls), 1.4, box, precision="fp32")
        r = e.download()
        if ref is None:
            ref = r
        else:
            _same(r, ref)
    with pytest.raises(V.VoronotaError):
        e.set_tuning(3, 1.0)
    with pytest.raises(V.VoronotaError):
        e.set_tuning(2, 0.4)  # finer than half the reach: the stencil would exceed 5^3


def test_autotune_on_a_batch():
    import torch

    structs = [W.lattice_balls(int(n), 500 + i) for i, n in enumerate(W.batch_sizes(60, 300, 5000, 2))]
    balls = np.concatenate(structs)
    off = np.zeros(len(structs) + 1, np.uint64)
    off[1:] = np.cumsum([len(x) for x in structs])
    e = V.Engine()
    d = torch.from_numpy(balls).cuda()
    torch.cuda.synchronize()
    t = e.autotune_device(d.data_ptr(), len(balls), 1.4, precision="fp32", offsets=off)
    assert t["warps_per_block"] in (2, 4, 8) and t["cell_scale"] in (0.5, 0.75, 1.0, 1.25) and t["chunk"] in (0, 4, 16)
    e.compute_batch_device(d.data_ptr(), off, 1.4, "fp32")
    got = e.download_batch()
    ref = V.compute_batch((balls, off), 1.4, "fp32")
    assert np.array_equal(got.all.area, ref.all.area) and np.array_equal(got.contact_off, ref.contact_off)
