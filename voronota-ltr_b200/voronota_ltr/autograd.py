"""torch.autograd front end of the tessellation and its hand-written adjoint.

``tessellate(xyzr, probe)`` takes a CUDA float64 tensor of shape (N, 4) (x, y, z, r) and
returns per-ball SAS areas and cell volumes (0 for balls without a cell), per-contact
areas, and the contacts' ball ids (not differentiable).  Backward runs the library's
adjoint kernel: for upstream gradients w (SAS), v (volumes) and u (areas) it returns
dL/d(x, y, z, r) of L = sum w SAS + sum v volume + sum u area, recomputing the contours
instead of storing them.
"""
from __future__ import annotations

import numpy as np
import torch

from . import Engine, parse_periodic_box


class _Tessellation(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyzr, probe, precision, periodic_box):
        if not xyzr.is_cuda or xyzr.dtype != torch.float64 or xyzr.dim() != 2 or xyzr.shape[1] != 4:
            raise ValueError("xyzr must be a CUDA float64 tensor of shape (N, 4)")
        x = xyzr.detach().contiguous()
        n = x.shape[0]
        eng = Engine(x.device.index or 0)
        eng.set_stream(torch.cuda.current_stream(x.device).cuda_stream)
        eng.set_keep_contours(True)  # backward reads the forward's contours
        pb = None if periodic_box is None else parse_periodic_box(periodic_box)
        eng.compute_device(x.data_ptr(), n, probe, pb, precision=precision)
        r = eng.download()
        sas = torch.zeros(n, dtype=torch.float64, device=x.device)
        vol = torch.zeros(n, dtype=torch.float64, device=x.device)
        if len(r.cell_index):
            idx = torch.from_numpy(r.cell_index.astype(np.int64)).to(x.device)
            sas[idx] = torch.from_numpy(r.cell_sas_area).to(x.device)
            vol[idx] = torch.from_numpy(r.cell_volume).to(x.device)
        area = torch.from_numpy(r.area).to(x.device)
        ida = torch.from_numpy(r.id_a.astype(np.int64)).to(x.device)
        idb = torch.from_numpy(r.id_b.astype(np.int64)).to(x.device)
        ctx.eng = eng
        ctx.n = n
        ctx.mark_non_differentiable(ida, idb)
        return sas, vol, area, ida, idb

    @staticmethod
    def backward(ctx, g_sas, g_vol, g_area, _g_ida, _g_idb):
        n = ctx.n
        dev = next(g.device for g in (g_sas, g_vol, g_area) if g is not None)
        grad = torch.empty((n, 4), dtype=torch.float64, device=dev)

        def arg(g):
            return None if g is None else g.detach().to(torch.float64).contiguous()

        w, v, u = arg(g_sas), arg(g_vol), arg(g_area)
        ctx.eng.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        ctx.eng.grad_device(0 if w is None else w.data_ptr(), 0 if (u is None or u.numel() == 0) else u.data_ptr(),
                            grad.data_ptr(), 0 if v is None else v.data_ptr())
        return grad, None, None, None


def tessellate(xyzr: torch.Tensor, probe: float, precision: str = "fp32", periodic_box=None):
    """(sas (N,), volume (N,), contact_area (C,), id_a (C,), id_b (C,)); differentiable in xyzr."""
    return _Tessellation.apply(xyzr, float(probe), precision, periodic_box)
