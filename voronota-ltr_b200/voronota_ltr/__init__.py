"""B200 radical tessellation -- Python front end mirroring voronota-ltr's bindings.

``compute_tessellation`` takes the same arguments and returns the same dict as the
reference's PyO3 function (src/python.rs:238-264, result_to_dict :189-210):
balls as a list of (x, y, z, r) tuples / lists / {x, y, z, r} dicts or an (N, 4) numpy
array; ``periodic_box`` as ``{"corners": [...]}`` or ``{"vectors": [...]}``; optional
``groups``.  The work runs on the GPU through the C ABI of ``libvoronota_b200.so``
(include/voronota_b200.h); there is no CPU fallback -- without the library or a CUDA
device every call raises.

Extra keyword: ``precision`` -- ``"fp32"`` (FP32 bulk geometry with FP64 recomputation
of every pair whose decisions fall inside the FP32 error band; default) or ``"fp64"``
(the reference's f64 arithmetic on the GPU).
"""
from __future__ import annotations

import ctypes
import os
from typing import Any

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libvoronota_b200.so")

VT_OK = 0
VT_ERR_INVALID = 1
VT_ERR_OOM = 2
VT_ERR_CUDA = 3
VT_ERR_CAPACITY = 4
VT_ERR_TIMEOUT = 5
VT_ERR_NO_DEVICE = 6
VT_FP64 = 0
VT_FP32_FIXUP = 1

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f64p = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p


class VoronotaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


class VoronotaInputError(VoronotaError, ValueError):
    """Invalid input (VT_ERR_INVALID): a ValueError, as the reference's Python module raises."""


class VtStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in (
        "num_balls", "num_slots", "num_entries", "num_pairs", "num_contacts", "num_cells",
        "num_fp64_redo", "num_serial")] + [
        ("total_sas_area", ctypes.c_double), ("total_volume", ctypes.c_double),
        ("total_contact_area", ctypes.c_double), ("device_error_bits", ctypes.c_uint32),
        ("num_kernel_launches", ctypes.c_uint64), ("num_cell_redo", ctypes.c_uint64),
        ("fp32_kernel", ctypes.c_uint64), ("num_host_syncs", ctypes.c_uint64)]

STAGES = ("prepare", "images", "grid", "neighbor_count", "neighbor_fill", "contact", "fp64_recompute",
          "serial_fallback", "cells", "output", "call")
UPD_STAGES = ("changed", "grid", "search", "lists", "pairs", "contacts", "table_cells", "cell_refresh", "finish",
              "call")


class VtDeviceOutputs(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in (
        "id_a", "id_b", "area", "arc_length", "central", "cell_index", "cell_sas_area",
        "cell_volume", "totals")]


_lib = None


def library():
    """Load libvoronota_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise VoronotaError(VT_ERR_CUDA, f"{LIB_PATH} is missing: build it with voronota-ltr_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    args7 = [_f64p, ctypes.c_uint64, ctypes.c_double, _f64p, _i32p, ctypes.c_uint64, ctypes.c_int]
    for name in ("vt_compute_tessellation", "vt_compute_contacts_only"):
        f = getattr(L, name)
        f.argtypes = args7 + [ctypes.POINTER(_vp)]
        f.restype = ctypes.c_int
    for name in ("vt_result_num_balls", "vt_result_num_contacts", "vt_result_num_cells"):
        getattr(L, name).argtypes = [_vp]
        getattr(L, name).restype = ctypes.c_uint64
    L.vt_result_contacts.argtypes = [_vp, _u32p, _u32p, _f64p, _f64p, _u8p]
    L.vt_result_cells.argtypes = [_vp, _u32p, _f64p, _f64p]
    L.vt_result_totals.argtypes = [_vp, _f64p, _f64p, _f64p]
    L.vt_result_totals.restype = None
    L.vt_result_free.argtypes = [_vp]
    L.vt_result_free.restype = None
    L.vt_result_view_get.argtypes = [_vp, ctypes.POINTER(VtResultView)]
    L.vt_compute_tessellation_network.argtypes = args7 + [ctypes.POINTER(_vp)]
    for name in ("vt_result_num_vertices", "vt_result_num_edges"):
        getattr(L, name).argtypes = [_vp]
        getattr(L, name).restype = ctypes.c_uint64
    L.vt_result_vertices.argtypes = [_vp, _u32p, _f64p]
    L.vt_result_edges.argtypes = [_vp, _u32p, _f64p]
    L.vt_engine_set_network.argtypes = [_vp, ctypes.c_int]
    L.vt_engine_set_network_wide_keys.argtypes = [_vp, ctypes.c_int]
    L.vt_engine_set_fp32_min_pairs.argtypes = [_vp, ctypes.c_uint64]
    L.vt_compute_solvent_spheres.argtypes = [_f64p, ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             _f64p, ctypes.c_int, ctypes.POINTER(_vp)]
    L.vt_icosahedron.argtypes = [ctypes.c_int, _f64p]
    L.vt_icosahedron.restype = ctypes.c_int
    L.vt_solvent_count.argtypes = [_vp]
    L.vt_solvent_count.restype = ctypes.c_uint64
    L.vt_solvent_get.argtypes = [_vp, _f64p, _f64p, _f64p, _u32p]
    L.vt_solvent_free.argtypes = [_vp]
    L.vt_solvent_free.restype = None
    L.vt_engine_create.argtypes = [ctypes.c_int, ctypes.POINTER(_vp)]
    L.vt_engine_destroy.argtypes = [_vp]
    L.vt_engine_destroy.restype = None
    L.vt_engine_set_stream.argtypes = [_vp, _vp]
    L.vt_engine_compute_device.argtypes = [_vp, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double, _f64p,
                                           ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
    L.vt_engine_compute_host.argtypes = [_vp, _f64p, ctypes.c_uint64, ctypes.c_double, _f64p, _i32p,
                                         ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
    L.vt_engine_download.argtypes = [_vp, ctypes.POINTER(_vp)]
    L.vt_engine_stats.argtypes = [_vp, ctypes.POINTER(VtStats)]
    L.vt_engine_device_outputs.argtypes = [_vp, ctypes.POINTER(VtDeviceOutputs)]
    L.vt_engine_set_timing.argtypes = [_vp, ctypes.c_int]
    L.vt_engine_set_fp32_band.argtypes = [_vp, ctypes.c_double]
    L.vt_engine_stage_times.argtypes = [_vp, _f64p]
    _ip = ctypes.POINTER(ctypes.c_int)
    L.vt_upd_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]
    L.vt_upd_destroy.argtypes = [_vp]
    L.vt_upd_destroy.restype = None
    L.vt_upd_set_stream.argtypes = [_vp, _vp]
    L.vt_upd_init.argtypes = [_vp, _f64p, ctypes.c_uint64, ctypes.c_double, _f64p, _ip]
    L.vt_upd_init_device.argtypes = [_vp, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double, _f64p, _ip]
    L.vt_upd_update.argtypes = [_vp, _f64p, ctypes.c_uint64, _ip]
    L.vt_upd_update_with_changed.argtypes = [_vp, _f64p, ctypes.c_uint64, _u64p, ctypes.c_uint64, _ip]
    L.vt_upd_update_with_changed_device.argtypes = [_vp, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                                    ctypes.c_uint64, _ip]
    L.vt_upd_set_exclusion.argtypes = [_vp, ctypes.c_uint64, ctypes.c_int, _ip]
    L.vt_upd_restore.argtypes = [_vp, _ip]
    L.vt_upd_summary.argtypes = [_vp, ctypes.POINTER(_vp)]
    L.vt_upd_totals.argtypes = [_vp, _f64p]
    L.vt_upd_last_full_reinit.argtypes = [_vp]
    L.vt_upd_num_changed.argtypes = [_vp]
    L.vt_upd_num_changed.restype = ctypes.c_uint64
    L.vt_upd_changed_ids.argtypes = [_vp, _u64p]
    L.vt_upd_num_affected.argtypes = [_vp]
    L.vt_upd_num_affected.restype = ctypes.c_uint64
    L.vt_upd_affected_ids.argtypes = [_vp, _u64p]
    L.vt_upd_stats.argtypes = [_vp, ctypes.POINTER(VtStats)]
    L.vt_upd_set_timing.argtypes = [_vp, ctypes.c_int]
    L.vt_upd_stage_times.argtypes = [_vp, _f64p]
    L.vt_upd_set_adjoint.argtypes = [_vp, ctypes.c_int]
    L.vt_upd_grad_sas.argtypes = [_vp, ctypes.c_void_p, ctypes.c_void_p]
    L.vt_upd_grad.argtypes = [_vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.vt_compute_batch.argtypes = [_f64p, _u64p, ctypes.c_uint64, ctypes.c_double, ctypes.c_int,
                                   ctypes.POINTER(_vp)]
    L.vt_engine_compute_batch_device.argtypes = [_vp, ctypes.c_void_p, _u64p, ctypes.c_uint64, ctypes.c_double,
                                                 ctypes.c_int, ctypes.c_int]
    L.vt_engine_download_batch.argtypes = [_vp, ctypes.POINTER(_vp)]
    for name in ("vt_batch_num_structures", "vt_batch_num_contacts", "vt_batch_num_cells"):
        getattr(L, name).argtypes = [_vp]
        getattr(L, name).restype = ctypes.c_uint64
    L.vt_batch_ranges.argtypes = [_vp, _u64p, _u64p]
    L.vt_batch_contacts.argtypes = [_vp, _u32p, _u32p, _f64p, _f64p, _u8p]
    L.vt_batch_cells.argtypes = [_vp, _u32p, _f64p, _f64p]
    L.vt_batch_totals.argtypes = [_vp, _f64p]
    L.vt_batch_free.argtypes = [_vp]
    L.vt_batch_free.restype = None
    L.vt_engine_grad_device.argtypes = [_vp, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.vt_engine_set_keep_contours.argtypes = [_vp, ctypes.c_int]
    L.vt_engine_autotune_device.argtypes = [_vp, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double, _f64p,
                                            ctypes.c_int, _u64p, ctypes.c_uint64]
    L.vt_engine_get_tuning.argtypes = [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_int)]
    L.vt_engine_set_tuning.argtypes = [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
    L.vt_grad.argtypes = [_f64p, ctypes.c_uint64, ctypes.c_double, _f64p, ctypes.c_int, _f64p, _f64p, _f64p,
                          ctypes.c_uint64, _f64p]
    L.vt_status_string.argtypes = [ctypes.c_int]
    L.vt_status_string.restype = ctypes.c_char_p
    L.vt_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def _check(status: int) -> None:
    if status != VT_OK:
        L = library()
        msg = L.vt_last_error().decode(errors="replace") or L.vt_status_string(status).decode()
        raise (VoronotaInputError if status == VT_ERR_INVALID else VoronotaError)(status, msg)


def _precision_code(precision) -> int:
    if precision in ("fp32", VT_FP32_FIXUP, "fp32_fixup"):
        return VT_FP32_FIXUP
    if precision in ("fp64", VT_FP64):
        return VT_FP64
    raise ValueError("precision must be 'fp32' or 'fp64'")


# ---- input parsing (src/python.rs:21-120) ----
def _ball_from_sequence(seq, type_name):
    if len(seq) != 4:
        raise ValueError(f"ball {type_name} must have 4 elements (x, y, z, r)")
    return [float(seq[0]), float(seq[1]), float(seq[2]), float(seq[3])]


def _parse_single_ball(obj):
    if isinstance(obj, dict):
        try:
            return [float(obj["x"]), float(obj["y"]), float(obj["z"]), float(obj["r"])]
        except KeyError as e:
            raise KeyError(f"missing '{e.args[0]}'") from None
    if isinstance(obj, tuple):
        return _ball_from_sequence(obj, "tuple")
    if isinstance(obj, list):
        return _ball_from_sequence(obj, "list")
    raise TypeError("ball must be tuple (x,y,z,r), list [x,y,z,r], or dict {x,y,z,r}")


def parse_balls(obj) -> np.ndarray:
    """(N, 4) contiguous float64 array from any accepted ball form."""
    if isinstance(obj, np.ndarray):
        if obj.ndim != 2 or obj.shape[1] != 4:
            raise ValueError("numpy array must have shape (N, 4) for (x, y, z, r)")
        return np.ascontiguousarray(obj, dtype=np.float64)
    if not isinstance(obj, list):
        raise TypeError("balls must be a list or a numpy array")
    if len(obj) == 0:
        return np.zeros((0, 4), np.float64)
    return np.ascontiguousarray(np.array([_parse_single_ball(b) for b in obj], dtype=np.float64))


def parse_periodic_box(obj) -> np.ndarray:
    """9 doubles (lattice vectors a, b, c) from a corners / vectors dict (python.rs:90-120)."""
    if not isinstance(obj, dict):
        raise TypeError("periodic_box must be a dict")
    if "corners" in obj:
        c = [tuple(float(v) for v in p) for p in obj["corners"]]
        if len(c) != 2:
            raise ValueError("corners must have exactly 2 points")
        (x1, y1, z1), (x2, y2, z2) = c
        # PeriodicBox::from_corners (types.rs:304-310)
        return np.array([x2 - x1, 0.0, 0.0, 0.0, y2 - y1, 0.0, 0.0, 0.0, z2 - z1], dtype=np.float64)
    if "vectors" in obj:
        v = [tuple(float(x) for x in p) for p in obj["vectors"]]
        if len(v) != 3:
            raise ValueError("vectors must have exactly 3 direction vectors")
        return np.ascontiguousarray(np.array(v, dtype=np.float64).reshape(9))
    raise ValueError("periodic_box must have 'corners' or 'vectors' key")


def _groups_array(groups):
    if groups is None:
        return None
    return np.ascontiguousarray(np.asarray(groups, dtype=np.int32).reshape(-1))


class VtResultView(ctypes.Structure):
    _fields_ = [("num_contacts", ctypes.c_uint64), ("num_cells", ctypes.c_uint64)] + [
        (k, ctypes.c_void_p) for k in ("id_a", "id_b", "area", "arc_length", "central", "cell_index",
                                       "cell_sas_area", "cell_volume")]


class _ResultOwner:
    """Frees a library result when the last numpy view of its arrays is gone."""

    def __init__(self, L, h):
        self.L, self.h = L, h

    def __del__(self):
        if self.h:
            self.L.vt_result_free(self.h)
            self.h = None


def _view(ptr, count, ctype, dtype, owner):
    if count == 0 or not ptr:
        return np.empty(0, dtype)
    buf = (ctype * count).from_address(ptr)
    buf._owner = owner  # the view keeps the result alive
    return np.frombuffer(buf, dtype=dtype)


class Result:
    """A tessellation result as numpy arrays (zero-copy views of the library's result)."""

    def __init__(self, num_balls, id_a, id_b, area, arc_length, central, cell_index, cell_sas, cell_volume,
                 totals):
        self.num_balls = int(num_balls)
        self.id_a, self.id_b = id_a, id_b
        self.area, self.arc_length, self.central = area, arc_length, central
        self.cell_index, self.cell_sas_area, self.cell_volume = cell_index, cell_sas, cell_volume
        self.total_sas_area, self.total_volume, self.total_contact_area = totals

    @classmethod
    def from_handle(cls, L, h):
        """Wrap a library result without copying: the arrays are views of the result's
        page-locked host memory, and the result is freed when the last of them is gone.
        Takes ownership of `h`."""
        owner = _ResultOwner(L, h)
        v = VtResultView()
        _check(L.vt_result_view_get(h, ctypes.byref(v)))
        C, M = int(v.num_contacts), int(v.num_cells)
        a = _view(v.id_a, C, ctypes.c_uint32, np.uint32, owner)
        b = _view(v.id_b, C, ctypes.c_uint32, np.uint32, owner)
        ar = _view(v.area, C, ctypes.c_double, np.float64, owner)
        arc = _view(v.arc_length, C, ctypes.c_double, np.float64, owner)
        ce = _view(v.central, C, ctypes.c_uint8, np.bool_, owner)
        ci = _view(v.cell_index, M, ctypes.c_uint32, np.uint32, owner)
        cs = _view(v.cell_sas_area, M, ctypes.c_double, np.float64, owner)
        cv = _view(v.cell_volume, M, ctypes.c_double, np.float64, owner)
        t = (ctypes.c_double(), ctypes.c_double(), ctypes.c_double())
        L.vt_result_totals(h, ctypes.byref(t[0]), ctypes.byref(t[1]), ctypes.byref(t[2]))
        r = cls(L.vt_result_num_balls(h), a, b, ar, arc, ce, ci, cs, cv, (t[0].value, t[1].value, t[2].value))
        V, E = int(L.vt_result_num_vertices(h)), int(L.vt_result_num_edges(h))
        vid, vxyz = np.empty((V, 4), np.uint32), np.empty((V, 3))
        eid, elen = np.empty((E, 3), np.uint32), np.empty(E)
        if L.vt_result_vertices(h, vid.ctypes.data_as(_u32p), vxyz.ctypes.data_as(_f64p)) == VT_OK:
            _check(L.vt_result_edges(h, eid.ctypes.data_as(_u32p), elen.ctypes.data_as(_f64p)))
            r.vertex_ids, r.vertex_xyz, r.edge_ids, r.edge_length = vid, vxyz, eid, elen
        return r

    # tessellation network (with_cell_vertices): ids (V, 4) / (E, 3) as uint32 with
    # NULL_ID (on the SAS) = 0xffffffff, positions (V, 3), lengths (E,); None otherwise
    vertex_ids = vertex_xyz = edge_ids = edge_length = None
    NULL_ID = 0xFFFFFFFF

    def sas_areas(self):
        """Per-ball SAS area or None (Results::sas_areas, types.rs:207-213)."""
        out = [None] * self.num_balls
        for i, s in zip(self.cell_index.tolist(), self.cell_sas_area.tolist()):
            out[i] = s
        return out

    def volumes(self):
        """Per-ball volume or None (Results::volumes, types.rs:222-228)."""
        out = [None] * self.num_balls
        for i, v in zip(self.cell_index.tolist(), self.cell_volume.tolist()):
            out[i] = v
        return out

    def to_dict(self) -> dict[str, Any]:
        """The reference's result dict (python.rs:189-210)."""
        contacts = [{"id_a": a, "id_b": b, "area": ar, "arc_length": arc, "central": ce}
                    for a, b, ar, arc, ce in zip(self.id_a.tolist(), self.id_b.tolist(), self.area.tolist(),
                                                 self.arc_length.tolist(), self.central.tolist())]
        cells = [{"index": i, "sas_area": s, "volume": v}
                 for i, s, v in zip(self.cell_index.tolist(), self.cell_sas_area.tolist(),
                                    self.cell_volume.tolist())]
        d = {"num_balls": self.num_balls, "contacts": contacts, "cells": cells,
             "total_sas_area": self.total_sas_area, "total_volume": self.total_volume,
             "total_contact_area": self.total_contact_area}
        if self.vertex_ids is not None:
            # vertices_to_list / edges_to_list (python.rs:153-187)
            def ids(row):
                return [None if i == self.NULL_ID else i for i in row]
            d["cell_vertices"] = [{"ball_indices": ids(v), "x": p[0], "y": p[1], "z": p[2], "is_on_sas": v[3] == self.NULL_ID}
                                  for v, p in zip(self.vertex_ids.tolist(), self.vertex_xyz.tolist())]
            d["cell_edges"] = [{"ball_indices": ids(e), "length": ln, "is_on_sas": e[2] == self.NULL_ID}
                               for e, ln in zip(self.edge_ids.tolist(), self.edge_length.tolist())]
        return d


def _run(fn_name, balls, probe, periodic_box, groups, precision) -> Result:
    L = library()
    x = parse_balls(balls)
    pb = None if periodic_box is None else parse_periodic_box(periodic_box)
    g = _groups_array(groups)
    h = _vp()
    st = getattr(L, fn_name)(x.ctypes.data_as(_f64p), x.shape[0], float(probe),
                             None if pb is None else pb.ctypes.data_as(_f64p),
                             None if g is None else g.ctypes.data_as(_i32p), 0 if g is None else len(g),
                             _precision_code(precision), ctypes.byref(h))
    _check(st)
    return Result.from_handle(L, h)


def compute_tessellation_result(balls, probe, periodic_box=None, groups=None, precision="fp32",
                                with_cell_vertices=False) -> Result:
    """compute_tessellation returning a :class:`Result` of numpy arrays; with
    ``with_cell_vertices`` it also holds the tessellation network (vertex_ids, vertex_xyz,
    edge_ids, edge_length)."""
    fn = "vt_compute_tessellation_network" if with_cell_vertices else "vt_compute_tessellation"
    return _run(fn, balls, probe, periodic_box, groups, precision)


def compute_tessellation(balls, probe, periodic_box=None, groups=None, with_cell_vertices=False,
                         precision="fp32") -> dict[str, Any]:
    """Radical tessellation of balls (python.rs:238-264); returns the reference's dict,
    with "cell_vertices" and "cell_edges" when ``with_cell_vertices``."""
    return compute_tessellation_result(balls, probe, periodic_box, groups, precision, with_cell_vertices).to_dict()


def compute_contacts_only(balls, probe, periodic_box=None, groups=None, precision="fp32") -> list[dict]:
    """compute_contacts_only (tessellation.rs:125-166): list of contact dicts."""
    r = _run("vt_compute_contacts_only", balls, probe, periodic_box, groups, precision)
    return r.to_dict()["contacts"]


def compute_contacts_only_result(balls, probe, periodic_box=None, groups=None, precision="fp32") -> Result:
    return _run("vt_compute_contacts_only", balls, probe, periodic_box, groups, precision)


def grad(balls, probe, w_sas=None, u_contact=None, periodic_box=None, precision="fp64",
         v_volume=None) -> np.ndarray:
    """dL/d(x, y, z, r) (an (N, 4) array) of L = sum_i w_sas[i] SAS_i + sum_i v_volume[i]
    V_i + sum_k u_contact[k] area_k, contact k being the k-th contact of
    compute_tessellation on the same input and V_i the cell volume (no counterpart in the
    reference).  The forward runs in ``precision``; the adjoint recomputes the contours."""
    L = library()
    x = parse_balls(balls)
    pb = None if periodic_box is None else parse_periodic_box(periodic_box)

    def per_ball(a, name):
        if a is None:
            return None
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
        if len(a) != x.shape[0]:
            raise ValueError(f"{name} needs one weight per ball")
        return a

    w = per_ball(w_sas, "w_sas")
    v = per_ball(v_volume, "v_volume")
    u = None if u_contact is None else np.ascontiguousarray(np.asarray(u_contact, dtype=np.float64).reshape(-1))
    out = np.zeros((x.shape[0], 4), np.float64)
    _check(L.vt_grad(x.ctypes.data_as(_f64p), x.shape[0], float(probe),
                     None if pb is None else pb.ctypes.data_as(_f64p), _precision_code(precision),
                     None if w is None else w.ctypes.data_as(_f64p), None if v is None else v.ctypes.data_as(_f64p),
                     None if u is None else u.ctypes.data_as(_f64p), 0 if u is None else len(u),
                     out.ctypes.data_as(_f64p)))
    return out


def icosahedron_directions(depth: int) -> np.ndarray:
    """Sample directions of compute_solvent_spheres (SubdividedIcosahedron,
    subdivided_icosahedron.rs:53-125) as computed by the library (host code)."""
    L = library()
    k = L.vt_icosahedron(int(depth), None)
    out = np.empty((k, 3))
    L.vt_icosahedron(int(depth), out.ctypes.data_as(_f64p))
    return out


class SolventSpheres:
    """compute_solvent_spheres output as arrays: xyz (S, 3), radius, weight (S,), parent
    (S,) ball index."""

    def __init__(self, xyz, radius, weight, parent):
        self.xyz, self.radius, self.weight, self.parent = xyz, radius, weight, parent

    def __len__(self):
        return len(self.weight)

    def to_list(self) -> list[dict]:
        """solvent_spheres_to_list (python.rs:326-342)."""
        return [{"x": p[0], "y": p[1], "z": p[2], "radius": r, "weight": w, "parent_index": i}
                for p, r, w, i in zip(self.xyz.tolist(), self.radius.tolist(), self.weight.tolist(),
                                      self.parent.tolist())]


def compute_solvent_spheres_result(balls, probe, volume_probe=None, subdivision_depth=None, periodic_box=None,
                                   precision="fp32") -> SolventSpheres:
    """compute_solvent_spheres returning arrays (see :func:`compute_solvent_spheres`)."""
    L = library()
    depth = 2 if subdivision_depth is None else int(subdivision_depth)
    if depth < 0:  # the reference takes a u32
        raise OverflowError("can't convert negative int to unsigned")
    x = parse_balls(balls)
    pb = None if periodic_box is None else parse_periodic_box(periodic_box)
    h = _vp()
    _check(L.vt_compute_solvent_spheres(x.ctypes.data_as(_f64p), x.shape[0], float(probe),
                                        0.0 if volume_probe is None else float(volume_probe), depth,
                                        None if pb is None else pb.ctypes.data_as(_f64p), _precision_code(precision),
                                        ctypes.byref(h)))
    try:
        S = int(L.vt_solvent_count(h))
        xyz, rad, w, par = np.empty((S, 3)), np.empty(S), np.empty(S), np.empty(S, np.uint32)
        _check(L.vt_solvent_get(h, xyz.ctypes.data_as(_f64p), rad.ctypes.data_as(_f64p), w.ctypes.data_as(_f64p),
                                par.ctypes.data_as(_u32p)))
    finally:
        L.vt_solvent_free(h)
    return SolventSpheres(xyz, rad, w, par)


def compute_solvent_spheres(balls, probe, volume_probe=None, subdivision_depth=None, periodic_box=None,
                            precision="fp32") -> list[dict]:
    """Weighted pseudo-solvent spheres on the exposed surface (python.rs:344-392): list of
    dicts with x, y, z, radius, weight, parent_index.  Both tessellations run on the GPU
    (``precision`` as for compute_tessellation); the sampling and the keep test between
    them run in FP64 on the device with the reference's arithmetic."""
    return compute_solvent_spheres_result(balls, probe, volume_probe, subdivision_depth, periodic_box,
                                          precision).to_list()


class BatchResult:
    """Results of a batched call: per-structure contacts and cells (ids local to the
    structure), concatenated, with the ranges of each structure and its totals."""

    def __init__(self, contact_off, cell_off, totals, all_result: Result):
        self.contact_off, self.cell_off = contact_off, cell_off
        self.totals = totals  # (S, 3): SAS area, volume, contact area
        self.all = all_result

    @classmethod
    def from_handle(cls, L, h):
        S = L.vt_batch_num_structures(h)
        nc, nm = L.vt_batch_num_contacts(h), L.vt_batch_num_cells(h)
        co = np.empty(S + 1, np.uint64)
        mo = np.empty(S + 1, np.uint64)
        _check(L.vt_batch_ranges(h, co.ctypes.data_as(_u64p), mo.ctypes.data_as(_u64p)))
        a, b = np.empty(nc, np.uint32), np.empty(nc, np.uint32)
        ar, arc, ce = np.empty(nc), np.empty(nc), np.empty(nc, np.uint8)
        _check(L.vt_batch_contacts(h, a.ctypes.data_as(_u32p), b.ctypes.data_as(_u32p), ar.ctypes.data_as(_f64p),
                                   arc.ctypes.data_as(_f64p), ce.ctypes.data_as(_u8p)))
        ci, cs, cv = np.empty(nm, np.uint32), np.empty(nm), np.empty(nm)
        _check(L.vt_batch_cells(h, ci.ctypes.data_as(_u32p), cs.ctypes.data_as(_f64p), cv.ctypes.data_as(_f64p)))
        tot = np.empty((S, 3))
        _check(L.vt_batch_totals(h, tot.ctypes.data_as(_f64p)))
        return cls(co, mo, tot, Result(0, a, b, ar, arc, ce.astype(bool), ci, cs, cv, (0.0, 0.0, 0.0)))

    def __len__(self):
        return len(self.totals)

    def structure(self, s: int, num_balls: int = 0) -> Result:
        c0, c1 = int(self.contact_off[s]), int(self.contact_off[s + 1])
        m0, m1 = int(self.cell_off[s]), int(self.cell_off[s + 1])
        A = self.all
        return Result(num_balls, A.id_a[c0:c1], A.id_b[c0:c1], A.area[c0:c1], A.arc_length[c0:c1],
                      A.central[c0:c1], A.cell_index[m0:m1], A.cell_sas_area[m0:m1], A.cell_volume[m0:m1],
                      tuple(float(x) for x in self.totals[s]))


def _batch_input(structures):
    if isinstance(structures, tuple) and len(structures) == 2:
        balls = np.ascontiguousarray(np.asarray(structures[0], dtype=np.float64).reshape(-1, 4))
        off = np.ascontiguousarray(np.asarray(structures[1], dtype=np.uint64))
        return balls, off
    parts = [parse_balls(x) for x in structures]
    off = np.zeros(len(parts) + 1, np.uint64)
    off[1:] = np.cumsum([len(x) for x in parts])
    balls = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros((0, 4)))
    return balls, off


def compute_batch(structures, probe, precision="fp32") -> BatchResult:
    """Tessellate many independent structures in one pass (no counterpart in the
    reference).  ``structures``: a list of ball arrays, or ``(balls (N, 4), offsets
    (S+1))``.  Each structure's result equals compute_tessellation on it alone."""
    L = library()
    balls, off = _batch_input(structures)
    h = _vp()
    _check(L.vt_compute_batch(balls.ctypes.data_as(_f64p), off.ctypes.data_as(_u64p), len(off) - 1, float(probe),
                              _precision_code(precision), ctypes.byref(h)))
    try:
        return BatchResult.from_handle(L, h)
    finally:
        L.vt_batch_free(h)


class Engine:
    """Explicit engine: a device, a stream and a reusable device workspace.

    ``compute_device`` takes a device pointer (e.g. ``tensor.data_ptr()`` of a contiguous
    float64 CUDA tensor of shape (N, 4)); results stay on the device until
    ``download()``.
    """

    def __init__(self, device: int = 0):
        self._L = library()
        self._h = _vp()
        _check(self._L.vt_engine_create(int(device), ctypes.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None):
            self._L.vt_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_stream(self, stream_ptr: int | None):
        _check(self._L.vt_engine_set_stream(self._h, stream_ptr))

    def compute_device(self, d_xyzr_ptr: int, n: int, probe: float, periodic_box=None, d_groups_ptr: int = 0,
                       n_groups: int = 0, precision="fp32", contacts_only: bool = False):
        pb = None if periodic_box is None else (periodic_box if isinstance(periodic_box, np.ndarray)
                                                else parse_periodic_box(periodic_box))
        if pb is not None:
            pb = np.ascontiguousarray(pb, dtype=np.float64).reshape(9)
        self._pb_keep = pb
        _check(self._L.vt_engine_compute_device(self._h, d_xyzr_ptr, int(n), float(probe),
                                                None if pb is None else pb.ctypes.data_as(_f64p),
                                                d_groups_ptr or None, int(n_groups), _precision_code(precision),
                                                1 if contacts_only else 0))

    def compute_host(self, balls, probe, periodic_box=None, groups=None, precision="fp32",
                     contacts_only=False):
        x = parse_balls(balls)
        pb = None if periodic_box is None else parse_periodic_box(periodic_box)
        g = _groups_array(groups)
        _check(self._L.vt_engine_compute_host(self._h, x.ctypes.data_as(_f64p), x.shape[0], float(probe),
                                              None if pb is None else pb.ctypes.data_as(_f64p),
                                              None if g is None else g.ctypes.data_as(_i32p),
                                              0 if g is None else len(g), _precision_code(precision),
                                              1 if contacts_only else 0))

    def stats(self) -> VtStats:
        s = VtStats()
        _check(self._L.vt_engine_stats(self._h, ctypes.byref(s)))
        return s

    def set_fp32_band(self, ulps: float):
        _check(self._L.vt_engine_set_fp32_band(self._h, float(ulps)))

    def set_fp32_min_pairs(self, min_pairs: int):
        """FP32 mode runs the FP32 contact kernel only from this many candidate pairs
        (default 2048; FP64 below); 0 forces the FP32 kernel."""
        _check(self._L.vt_engine_set_fp32_min_pairs(self._h, int(min_pairs)))

    def set_keep_contours(self, on: bool = True):
        """Later FP32 computations keep their contours for grad_device (faster adjoint,
        about 24 bytes of device memory per contour point)."""
        _check(self._L.vt_engine_set_keep_contours(self._h, 1 if on else 0))

    def set_network(self, on: bool = True):
        """Later compute calls also build the tessellation network (with_cell_vertices)."""
        _check(self._L.vt_engine_set_network(self._h, 1 if on else 0))

    def set_network_wide_keys(self, on: bool = True):
        """The network's vertex deduplication in its two-word key form, which it takes by
        itself from 2^21 balls on (same results)."""
        _check(self._L.vt_engine_set_network_wide_keys(self._h, 1 if on else 0))

    def set_timing(self, on: bool = True):
        _check(self._L.vt_engine_set_timing(self._h, 1 if on else 0))

    def stage_times(self) -> dict:
        buf = (ctypes.c_double * len(STAGES))()
        _check(self._L.vt_engine_stage_times(self._h, buf))
        return dict(zip(STAGES, list(buf)))

    def device_outputs(self) -> VtDeviceOutputs:
        o = VtDeviceOutputs()
        _check(self._L.vt_engine_device_outputs(self._h, ctypes.byref(o)))
        return o

    def autotune_device(self, d_xyzr_ptr: int, n: int, probe: float, periodic_box=None, precision="fp32",
                        offsets=None) -> dict:
        """Time candidate launch configurations on this input and keep the fastest."""
        pb = None if periodic_box is None else parse_periodic_box(periodic_box)
        off = None if offsets is None else np.ascontiguousarray(np.asarray(offsets, dtype=np.uint64))
        _check(self._L.vt_engine_autotune_device(self._h, d_xyzr_ptr, int(n), float(probe),
                                                 None if pb is None else pb.ctypes.data_as(_f64p),
                                                 _precision_code(precision),
                                                 None if off is None else off.ctypes.data_as(_u64p),
                                                 0 if off is None else len(off) - 1))
        return self.tuning()

    def tuning(self) -> dict:
        w, c, ch = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        _check(self._L.vt_engine_get_tuning(self._h, ctypes.byref(w), ctypes.byref(c), ctypes.byref(ch)))
        return {"warps_per_block": w.value, "cell_scale": c.value, "chunk": ch.value}

    def set_tuning(self, warps_per_block: int = 2, cell_scale: float = 0.5, chunk: int = 4):
        """chunk > 0: persistent contact launch taking `chunk` pairs per grab."""
        _check(self._L.vt_engine_set_tuning(self._h, int(warps_per_block), float(cell_scale), int(chunk)))

    def grad_device(self, d_w_ptr, d_u_ptr, d_grad_ptr: int, d_v_ptr=None):
        """Adjoint of the last full tessellation: d_grad (N x 4 doubles on the device) =
        dL/d(x, y, z, r), L = sum w SAS + sum v volume + sum u area (device pointers;
        0/None = no term)."""
        _check(self._L.vt_engine_grad_device(self._h, d_w_ptr or None, d_v_ptr or None, d_u_ptr or None,
                                             d_grad_ptr))

    def compute_batch_device(self, d_xyzr_ptr: int, offsets, probe: float, precision="fp32",
                             contacts_only: bool = False):
        off = np.ascontiguousarray(np.asarray(offsets, dtype=np.uint64))
        _check(self._L.vt_engine_compute_batch_device(self._h, d_xyzr_ptr, off.ctypes.data_as(_u64p), len(off) - 1,
                                                      float(probe), _precision_code(precision),
                                                      1 if contacts_only else 0))

    def download_batch(self) -> BatchResult:
        h = _vp()
        _check(self._L.vt_engine_download_batch(self._h, ctypes.byref(h)))
        try:
            return BatchResult.from_handle(self._L, h)
        finally:
            self._L.vt_batch_free(h)

    def download(self) -> Result:
        h = _vp()
        _check(self._L.vt_engine_download(self._h, ctypes.byref(h)))
        return Result.from_handle(self._L, h)


class UpdateableTessellation:
    """UpdateableTessellation (src/updateable.rs:154-742) with its state on the GPU.

    Same methods and return values as the reference: ``init``, ``update``,
    ``update_with_changed``, ``set_exclusion``, ``restore``, ``summary``,
    ``changed_ids``, ``affected_ids``, ``last_update_was_full_reinit``,
    ``backup_enabled``.  ``summary()`` returns a :class:`Result` (``to_dict()`` gives the
    reference's dict layout).  ``update_with_changed_device`` takes device pointers of a
    float64 (N, 4) ball array and a uint64 id array on the handle's device.
    """

    def __init__(self, with_backup: bool = False, precision="fp64", device: int = 0):
        self._L = library()
        self._h = _vp()
        self._backup = bool(with_backup)
        _check(self._L.vt_upd_create(int(device), 1 if with_backup else 0, _precision_code(precision),
                                     ctypes.byref(self._h)))

    @classmethod
    def with_backup(cls, precision="fp64", device: int = 0) -> "UpdateableTessellation":
        return cls(True, precision, device)

    def close(self):
        if getattr(self, "_h", None):
            self._L.vt_upd_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def backup_enabled(self) -> bool:
        return self._backup

    def set_stream(self, stream_ptr: int | None):
        _check(self._L.vt_upd_set_stream(self._h, stream_ptr))

    def _flag(self, fn, *args) -> bool:
        r = ctypes.c_int(0)
        _check(fn(self._h, *args, ctypes.byref(r)))
        return bool(r.value)

    def init(self, balls, probe: float, periodic_box=None) -> bool:
        x = parse_balls(balls)
        pb = None if periodic_box is None else parse_periodic_box(periodic_box)
        return self._flag(self._L.vt_upd_init, x.ctypes.data_as(_f64p), x.shape[0], float(probe),
                          None if pb is None else pb.ctypes.data_as(_f64p))

    def init_device(self, d_xyzr_ptr: int, n: int, probe: float, periodic_box=None) -> bool:
        pb = None if periodic_box is None else parse_periodic_box(periodic_box)
        return self._flag(self._L.vt_upd_init_device, d_xyzr_ptr, int(n), float(probe),
                          None if pb is None else pb.ctypes.data_as(_f64p))

    def update(self, balls) -> bool:
        x = parse_balls(balls)
        return self._flag(self._L.vt_upd_update, x.ctypes.data_as(_f64p), x.shape[0])

    def update_with_changed(self, balls, changed_ids) -> bool:
        x = parse_balls(balls)
        ids = np.ascontiguousarray(np.asarray(changed_ids, dtype=np.uint64).reshape(-1))
        return self._flag(self._L.vt_upd_update_with_changed, x.ctypes.data_as(_f64p), x.shape[0],
                          ids.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(ids))

    def update_with_changed_device(self, d_xyzr_ptr: int, n: int, d_ids_ptr: int, k: int) -> bool:
        return self._flag(self._L.vt_upd_update_with_changed_device, d_xyzr_ptr, int(n), d_ids_ptr, int(k))

    def set_exclusion(self, idx: int, excluded: bool) -> bool:
        return self._flag(self._L.vt_upd_set_exclusion, int(idx), 1 if excluded else 0)

    def restore(self) -> bool:
        return self._flag(self._L.vt_upd_restore)

    def summary(self) -> Result:
        h = _vp()
        _check(self._L.vt_upd_summary(self._h, ctypes.byref(h)))
        return Result.from_handle(self._L, h)

    def totals(self) -> tuple[float, float, float]:
        """(total SAS area, total volume, total contact area) of the current summary."""
        t = (ctypes.c_double * 3)()
        _check(self._L.vt_upd_totals(self._h, t))
        return t[0], t[1], t[2]

    def last_update_was_full_reinit(self) -> bool:
        return bool(self._L.vt_upd_last_full_reinit(self._h))

    def changed_ids(self) -> np.ndarray:
        out = np.zeros(self._L.vt_upd_num_changed(self._h), np.uint64)
        _check(self._L.vt_upd_changed_ids(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out

    def affected_ids(self) -> np.ndarray:
        out = np.zeros(self._L.vt_upd_num_affected(self._h), np.uint64)
        _check(self._L.vt_upd_affected_ids(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out

    def stats(self) -> VtStats:
        s = VtStats()
        _check(self._L.vt_upd_stats(self._h, ctypes.byref(s)))
        return s

    def grad_sas_device(self, d_w_ptr, d_grad_ptr: int):
        """d_grad (N x 4 doubles on the device) = d(sum w SAS)/d(x, y, z, r) of the current
        state; d_w_ptr 0/None: the total SAS."""
        _check(self._L.vt_upd_grad_sas(self._h, d_w_ptr or None, d_grad_ptr))

    def set_timing(self, on: bool = True):
        """Record per-stage CUDA events in later updates (stage_times)."""
        _check(self._L.vt_upd_set_timing(self._h, 1 if on else 0))

    def stage_times(self) -> dict:
        """Device milliseconds per stage of the last update (UPD_STAGES), with timing on."""
        buf = (ctypes.c_double * len(UPD_STAGES))()
        _check(self._L.vt_upd_stage_times(self._h, buf))
        return dict(zip(UPD_STAGES, list(buf)))

    def grad_device(self, d_w_ptr, d_v_ptr, d_grad_ptr: int):
        """d_grad (N x 4 doubles on the device) = d(sum w SAS + sum v volume)/d(x, y, z, r)
        of the current state; a 0/None weight pointer leaves its term out."""
        _check(self._L.vt_upd_grad(self._h, d_w_ptr or None, d_v_ptr or None, d_grad_ptr))

    def set_adjoint(self, on: bool = True):
        """Record the arc and face moments behind grad_sas_device / grad_device (default
        on).  Off makes updates about a tenth faster; the adjoints then raise until a full
        computation ran with it on again."""
        _check(self._L.vt_upd_set_adjoint(self._h, 1 if on else 0))


__all__ = ["compute_tessellation", "compute_tessellation_result", "compute_contacts_only",
           "compute_solvent_spheres", "compute_solvent_spheres_result", "SolventSpheres", "VoronotaInputError",
           "compute_contacts_only_result", "compute_batch", "BatchResult", "grad", "Engine", "Result", "UpdateableTessellation", "VoronotaError",
           "library", "parse_balls", "parse_periodic_box"]


from .io import compute_tessellation_from_file  # noqa: E402  (file front end, voronota_ltr/io.py)

__all__ += ["compute_tessellation_from_file"]
