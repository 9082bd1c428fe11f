"""ctypes wrapper of the CPU oracle (test infrastructure, not product code).

The oracle is a C++ f64 restatement of voronota-ltr's tessellation hot path
(``oracle/vt_oracle.cpp``).  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` load it, always as the checker or the timed CPU
baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libvt_oracle.so")
_lib = None

_u64p = ctypes.POINTER(ctypes.c_uint64)
_f64p = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)


def build() -> str:
    """Compile the oracle shared library (make) and return its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = ctypes.CDLL(_LIB_PATH)
    vp = ctypes.c_void_p
    L.vto_set_threads.argtypes = [ctypes.c_int]
    L.vto_get_threads.restype = ctypes.c_int
    L.vto_set_faithful_grid_update.argtypes = [ctypes.c_int]
    L.vto_compute.argtypes = [_f64p, ctypes.c_uint64, ctypes.c_double, _f64p, _i32p, ctypes.c_uint64,
                              ctypes.c_int, ctypes.POINTER(vp)]
    L.vto_compute.restype = ctypes.c_int
    for name in ("vto_num_balls", "vto_num_contacts", "vto_num_cells", "vto_num_neighbor_entries",
                 "vto_num_pairs"):
        getattr(L, name).argtypes = [vp]
        getattr(L, name).restype = ctypes.c_uint64
    L.vto_get_contacts.argtypes = [vp, _u64p, _u64p, _f64p, _f64p, _u8p]
    L.vto_get_cells.argtypes = [vp, _u64p, _f64p, _f64p]
    L.vto_get_neighbors.argtypes = [vp, _u64p, _u64p, _f64p]
    L.vto_get_pairs.argtypes = [vp, _u64p, _u64p, _u8p, _f64p, _f64p, _u8p, _f64p, _f64p, _f64p, _f64p]
    L.vto_free.argtypes = [vp]
    L.vto_set_network.argtypes = [ctypes.c_int]
    for name in ("vto_num_vertices", "vto_num_edges"):
        getattr(L, name).argtypes = [vp]
        getattr(L, name).restype = ctypes.c_uint64
    L.vto_get_vertices.argtypes = [vp, _u64p, _f64p]
    L.vto_get_edges.argtypes = [vp, _u64p, _f64p]
    L.vto_upd_create.argtypes = [ctypes.c_int]
    L.vto_upd_create.restype = vp
    L.vto_upd_destroy.argtypes = [vp]
    L.vto_upd_init.argtypes = [vp, _f64p, ctypes.c_uint64, ctypes.c_double, _f64p]
    L.vto_upd_update.argtypes = [vp, _f64p, ctypes.c_uint64]
    L.vto_upd_update_with_changed.argtypes = [vp, _f64p, ctypes.c_uint64, _u64p, ctypes.c_uint64]
    L.vto_upd_set_exclusion.argtypes = [vp, ctypes.c_uint64, ctypes.c_int]
    L.vto_upd_restore.argtypes = [vp]
    L.vto_upd_last_full_reinit.argtypes = [vp]
    for name in ("vto_upd_num_changed", "vto_upd_num_affected"):
        getattr(L, name).argtypes = [vp]
        getattr(L, name).restype = ctypes.c_uint64
    L.vto_upd_get_changed.argtypes = [vp, _u64p]
    L.vto_upd_get_affected.argtypes = [vp, _u64p]
    L.vto_upd_summary.argtypes = [vp]
    L.vto_upd_summary.restype = vp
    L.vto_icosahedron.argtypes = [ctypes.c_int, _f64p]
    L.vto_icosahedron.restype = ctypes.c_int
    L.vto_solvent_spheres.argtypes = [_f64p, ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                      _f64p, ctypes.POINTER(vp)]
    L.vto_solvent_spheres.restype = ctypes.c_int
    L.vto_solvent_count.argtypes = [vp]
    L.vto_solvent_count.restype = ctypes.c_uint64
    L.vto_solvent_get.argtypes = [vp, _f64p, _u64p]
    L.vto_solvent_free.argtypes = [vp]
    _lib = L
    return L


def _p(a, t):
    return a.ctypes.data_as(t)


def pbox_vectors(periodic_box) -> np.ndarray | None:
    """Lattice vectors (3x3) from a reference-style periodic box dict, or None.

    ``{"corners": [(x1,y1,z1), (x2,y2,z2)]}`` maps to diagonal vectors as
    PeriodicBox::from_corners (types.rs:304-310); ``{"vectors": [...]}`` is taken as is.
    """
    if periodic_box is None:
        return None
    if isinstance(periodic_box, np.ndarray):
        return np.ascontiguousarray(periodic_box, dtype=np.float64).reshape(9)
    if "corners" in periodic_box:
        (x1, y1, z1), (x2, y2, z2) = periodic_box["corners"]
        return np.array([x2 - x1, 0, 0, 0, y2 - y1, 0, 0, 0, z2 - z1], dtype=np.float64)
    if "vectors" in periodic_box:
        return np.ascontiguousarray(np.array(periodic_box["vectors"], dtype=np.float64).reshape(9))
    raise ValueError("periodic_box must have 'corners' or 'vectors' key")


@dataclass
class OracleResult:
    num_balls: int
    contacts_a: np.ndarray
    contacts_b: np.ndarray
    contacts_area: np.ndarray
    contacts_arc: np.ndarray
    contacts_central: np.ndarray
    cells_index: np.ndarray
    cells_sas: np.ndarray
    cells_vol: np.ndarray
    nb_offsets: np.ndarray | None = None
    nb_ids: np.ndarray | None = None
    nb_values: np.ndarray | None = None
    pairs: dict = field(default_factory=dict)

    @property
    def total_contact_area(self) -> float:
        return float(np.sum(self.contacts_area))

    @property
    def total_sas_area(self) -> float:
        return float(np.sum(self.cells_sas))

    @property
    def total_volume(self) -> float:
        return float(np.sum(self.cells_vol))


def _read_result(L, h, internals: bool) -> OracleResult:
    nc = L.vto_num_contacts(h)
    a = np.zeros(nc, np.uint64)
    b = np.zeros(nc, np.uint64)
    ar = np.zeros(nc, np.float64)
    arc = np.zeros(nc, np.float64)
    ce = np.zeros(nc, np.uint8)
    L.vto_get_contacts(h, _p(a, _u64p), _p(b, _u64p), _p(ar, _f64p), _p(arc, _f64p), _p(ce, _u8p))
    m = L.vto_num_cells(h)
    ci = np.zeros(m, np.uint64)
    cs = np.zeros(m, np.float64)
    cv = np.zeros(m, np.float64)
    L.vto_get_cells(h, _p(ci, _u64p), _p(cs, _f64p), _p(cv, _f64p))
    res = OracleResult(int(L.vto_num_balls(h)), a, b, ar, arc, ce.astype(bool), ci, cs, cv)
    if internals:
        n = res.num_balls
        ne = L.vto_num_neighbor_entries(h)
        off = np.zeros(n + 1, np.uint64)
        ids = np.zeros(ne, np.uint64)
        vals = np.zeros(ne, np.float64)
        L.vto_get_neighbors(h, _p(off, _u64p), _p(ids, _u64p), _p(vals, _f64p))
        res.nb_offsets, res.nb_ids, res.nb_values = off, ids, vals
        npairs = L.vto_num_pairs(h)
        arrs = {k: np.zeros(npairs, np.uint64) for k in ("a", "b")}
        arrs["valid"] = np.zeros(npairs, np.uint8)
        arrs["central"] = np.zeros(npairs, np.uint8)
        for k in ("area", "arc", "solid_a", "solid_b", "pyr_a", "pyr_b"):
            arrs[k] = np.zeros(npairs, np.float64)
        L.vto_get_pairs(h, _p(arrs["a"], _u64p), _p(arrs["b"], _u64p), _p(arrs["valid"], _u8p),
                        _p(arrs["area"], _f64p), _p(arrs["arc"], _f64p), _p(arrs["central"], _u8p),
                        _p(arrs["solid_a"], _f64p), _p(arrs["solid_b"], _f64p), _p(arrs["pyr_a"], _f64p),
                        _p(arrs["pyr_b"], _f64p))
        res.pairs = arrs
    return res


def set_threads(n: int) -> None:
    lib().vto_set_threads(int(n))


def get_threads() -> int:
    return int(lib().vto_get_threads())


def set_faithful_grid_update(on: bool) -> None:
    lib().vto_set_faithful_grid_update(1 if on else 0)


NET_NULL = np.uint64(0xFFFFFFFFFFFFFFFF)  # NULL_ID of a network element (types.rs:98)


def compute(balls, probe: float, periodic_box=None, groups=None, contacts_only: bool = False,
            internals: bool = False, with_cell_vertices: bool = False) -> OracleResult:
    """compute_tessellation / compute_contacts_only on the CPU oracle.  With
    with_cell_vertices the result also holds the tessellation network: vertex_ids
    (V, 4) and vertex_xyz (V, 3), edge_ids (E, 3) and edge_length (E,); NULL ids are
    NET_NULL."""
    L = lib()
    L.vto_set_network(1 if with_cell_vertices else 0)
    xyzr = np.ascontiguousarray(np.asarray(balls, dtype=np.float64).reshape(-1, 4))
    n = xyzr.shape[0]
    pb = pbox_vectors(periodic_box)
    g = None if groups is None else np.ascontiguousarray(np.asarray(groups, dtype=np.int32))
    h = ctypes.c_void_p()
    rc = L.vto_compute(_p(xyzr, _f64p), n, float(probe), None if pb is None else _p(pb, _f64p),
                       None if g is None else _p(g, _i32p), 0 if g is None else len(g),
                       1 if contacts_only else 0, ctypes.byref(h))
    L.vto_set_network(0)
    if rc != 0:
        raise RuntimeError(f"oracle failed: {rc}")
    try:
        res = _read_result(L, h, internals)
        if with_cell_vertices:
            nv, ne = L.vto_num_vertices(h), L.vto_num_edges(h)
            res.vertex_ids = np.zeros((nv, 4), np.uint64)
            res.vertex_xyz = np.zeros((nv, 3), np.float64)
            res.edge_ids = np.zeros((ne, 3), np.uint64)
            res.edge_length = np.zeros(ne, np.float64)
            L.vto_get_vertices(h, _p(res.vertex_ids, _u64p), _p(res.vertex_xyz, _f64p))
            L.vto_get_edges(h, _p(res.edge_ids, _u64p), _p(res.edge_length, _f64p))
        return res
    finally:
        L.vto_free(h)


class OracleUpdateable:
    """UpdateableTessellation restated on the CPU (updateable.rs)."""

    def __init__(self, with_backup: bool = False):
        self._L = lib()
        self._h = ctypes.c_void_p(self._L.vto_upd_create(1 if with_backup else 0))

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.vto_upd_destroy(self._h)
            self._h = None

    @staticmethod
    def _xyzr(balls):
        return np.ascontiguousarray(np.asarray(balls, dtype=np.float64).reshape(-1, 4))

    def init(self, balls, probe: float, periodic_box=None) -> bool:
        x = self._xyzr(balls)
        pb = pbox_vectors(periodic_box)
        return bool(self._L.vto_upd_init(self._h, _p(x, _f64p), x.shape[0], float(probe),
                                         None if pb is None else _p(pb, _f64p)))

    def update(self, balls) -> bool:
        x = self._xyzr(balls)
        return bool(self._L.vto_upd_update(self._h, _p(x, _f64p), x.shape[0]))

    def update_with_changed(self, balls, changed_ids) -> bool:
        x = self._xyzr(balls)
        ids = np.ascontiguousarray(np.asarray(changed_ids, dtype=np.uint64))
        return bool(self._L.vto_upd_update_with_changed(self._h, _p(x, _f64p), x.shape[0], _p(ids, _u64p),
                                                        len(ids)))

    def set_exclusion(self, idx: int, excluded: bool) -> bool:
        return bool(self._L.vto_upd_set_exclusion(self._h, int(idx), 1 if excluded else 0))

    def restore(self) -> bool:
        return bool(self._L.vto_upd_restore(self._h))

    def last_update_was_full_reinit(self) -> bool:
        return bool(self._L.vto_upd_last_full_reinit(self._h))

    def changed_ids(self) -> np.ndarray:
        k = self._L.vto_upd_num_changed(self._h)
        out = np.zeros(k, np.uint64)
        self._L.vto_upd_get_changed(self._h, _p(out, _u64p))
        return out

    def affected_ids(self) -> np.ndarray:
        k = self._L.vto_upd_num_affected(self._h)
        out = np.zeros(k, np.uint64)
        self._L.vto_upd_get_affected(self._h, _p(out, _u64p))
        return out

    def summary(self) -> OracleResult:
        h = ctypes.c_void_p(self._L.vto_upd_summary(self._h))
        try:
            return _read_result(self._L, h, False)
        finally:
            self._L.vto_free(h)


def icosahedron(depth: int) -> np.ndarray:
    """Unit sample directions of SubdividedIcosahedron (subdivided_icosahedron.rs:53-125)."""
    L = lib()
    k = L.vto_icosahedron(int(depth), None)
    out = np.zeros((k, 3))
    L.vto_icosahedron(int(depth), _p(out, _f64p))
    return out


class SolventResult:
    def __init__(self, xyz, radius, weight, parent):
        self.xyz, self.radius, self.weight, self.parent = xyz, radius, weight, parent


_SOLVENT_ERRORS = {1: "invalid probe radius", 2: "invalid volume probe", 3: "invalid ball"}


def solvent_spheres(balls, probe: float, volume_probe: float = 0.0, subdivision_depth: int = 2,
                    periodic_box=None) -> SolventResult:
    """compute_solvent_spheres (solvent_spheres.rs:131-169) on the CPU."""
    L = lib()
    x = np.ascontiguousarray(np.asarray(balls, dtype=np.float64).reshape(-1, 4))
    pb = pbox_vectors(periodic_box)
    h = ctypes.c_void_p()
    st = L.vto_solvent_spheres(_p(x, _f64p), x.shape[0], float(probe), float(volume_probe), int(subdivision_depth),
                               None if pb is None else _p(pb, _f64p), ctypes.byref(h))
    if st != 0:
        raise ValueError(_SOLVENT_ERRORS.get(st, "invalid input"))
    try:
        k = L.vto_solvent_count(h)
        v = np.zeros((k, 5))
        par = np.zeros(k, np.uint64)
        if k:
            L.vto_solvent_get(h, _p(v, _f64p), _p(par, _u64p))
    finally:
        L.vto_solvent_free(h)
    return SolventResult(v[:, :3].copy(), v[:, 3].copy(), v[:, 4].copy(), par)


def loss_weights_by_pair(id_a, id_b, u, num_balls):
    """(sorted pair keys, weights) of per-contact weights u attached to the contacts' ball
    pairs, so that a loss can look a pair's weight up under any perturbation (a pair that
    is not in the list weighs 0)."""
    key = np.asarray(id_a, np.int64) * int(num_balls) + np.asarray(id_b, np.int64)
    order = np.argsort(key)
    return key[order], np.asarray(u, np.float64)[order]


def finite_difference_local(balls, probe: float, i: int, c: int, h: float, w=None, v=None, upair=None) -> float:
    """Central difference (L(x + h e) - L(x - h e)) / 2h of
    L = sum_j w_j SAS_j + sum_j v_j V_j + sum_(a,b) u_ab area_ab at coordinate c (x, y, z,
    r) of ball i, computed by the oracle on the sub-structure that determines the change.

    Moving ball i changes only contacts whose ends both intersect ball i (a contact is cut
    only by balls intersecting both of its balls) and the cells of the balls intersecting
    i.  Those are computed exactly from the balls within three neighbour hops (each hop at
    most 2 max R): a contact needs the complete neighbour list of its lower ball, and a
    cell all of its contacts.  The terms of balls and contacts farther away are left out
    (they do not change).  upair = loss_weights_by_pair(...) of the full structure; w, v
    are per-ball weights of the full structure (None: no such term).  Non-periodic."""
    balls = np.asarray(balls, np.float64)
    R = balls[:, 3] + probe
    reach = 2.0 * R.max()
    d = np.linalg.norm(balls[:, :3] - balls[i, :3], axis=1)
    sub = np.nonzero(d <= 3.0 * reach + 4.0 * abs(h) + 0.1)[0]
    li = int(np.searchsorted(sub, i))
    # balls whose cells and contacts may change: those intersecting ball i (with margin)
    near = d[sub] <= R[sub] + R[i] + 4.0 * abs(h) + 0.01
    n = len(balls)

    def loss(x):
        o = compute(x, probe)
        total = 0.0
        ci = o.cells_index.astype(np.int64)
        keep = near[ci]
        gi = sub[ci[keep]]
        if w is not None:
            total += float(np.dot(w[gi], o.cells_sas[keep]))
        if v is not None:
            total += float(np.dot(v[gi], o.cells_vol[keep]))
        if upair is not None:
            a = o.contacts_a.astype(np.int64)
            b = o.contacts_b.astype(np.int64)
            m = near[a] | near[b]
            k = sub[a[m]] * n + sub[b[m]]
            ks, us = upair
            pos = np.clip(np.searchsorted(ks, k), 0, max(len(ks) - 1, 0))
            uu = np.where(ks[pos] == k, us[pos], 0.0) if len(ks) else np.zeros(len(k))
            total += float(np.dot(uu, o.contacts_area[m]))
        return total

    xp = balls[sub].copy()
    xm = balls[sub].copy()
    xp[li, c] += h
    xm[li, c] -= h
    return (loss(xp) - loss(xm)) / (2.0 * h)
