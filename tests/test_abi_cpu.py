"""CPU-side checks of the product boundary: the C-ABI library builds, loads and exports
every function include/voronota_b200.h declares; the Python front end parses inputs the
way the reference's bindings do (src/python.rs:21-120).  No GPU compute here."""
import ctypes
import os
import re

import numpy as np
import pytest

import voronota_ltr as V

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "voronota_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(vt_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib_path = V.LIB_PATH
    if not os.path.exists(lib_path):
        import importlib.util
        spec = importlib.util.spec_from_file_location("vt_build", os.path.join(ROOT, "voronota-ltr_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    lib = ctypes.CDLL(lib_path)
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), f"{name} not exported"


def test_status_strings():
    L = V.library()
    assert L.vt_status_string(0) == b"ok"
    assert L.vt_status_string(4) == b"capacity exceeded"


def test_parse_balls_forms():
    ref = np.array([[0, 0, 0, 1.5], [3, 0, 0, 1.5]], dtype=np.float64)
    for form in ([(0, 0, 0, 1.5), (3, 0, 0, 1.5)], [[0, 0, 0, 1.5], [3, 0, 0, 1.5]],
                 [{"x": 0, "y": 0, "z": 0, "r": 1.5}, {"x": 3, "y": 0, "z": 0, "r": 1.5}], ref):
        assert np.array_equal(V.parse_balls(form), ref)
    with pytest.raises(ValueError):
        V.parse_balls([(0, 0, 0)])
    with pytest.raises(ValueError):
        V.parse_balls(np.zeros((3, 3)))
    with pytest.raises(TypeError):
        V.parse_balls([5])
    assert V.parse_balls([]).shape == (0, 4)


def test_parse_periodic_box():
    a = V.parse_periodic_box({"corners": [(0, 0, 0), (200, 250, 300)]})
    b = V.parse_periodic_box({"vectors": [(200, 0, 0), (0, 250, 0), (0, 0, 300)]})
    assert np.array_equal(a, b)
    with pytest.raises(ValueError):
        V.parse_periodic_box({"invalid": "key"})
    with pytest.raises(ValueError):
        V.parse_periodic_box({"corners": [(0, 0, 0)]})


def test_no_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(V.VoronotaError) as ei:
        V.compute_tessellation([(0, 0, 0, 1.5)], 1.4)
    assert ei.value.status == V.VT_ERR_NO_DEVICE


def test_icosahedron_directions_match_oracle():
    """The library's sample directions (host code) are the oracle's bit for bit."""
    import oracle as O
    for depth in range(6):
        assert np.array_equal(V.icosahedron_directions(depth), O.icosahedron(depth))


def test_solvent_input_validation_without_device():
    """compute_solvent_spheres rejects bad parameters before any device work, with the
    reference's ValueError (solvent_spheres.rs:164-194; tests/test_python.py:262-278)."""
    for kw in [dict(balls=[(0.0, 0.0, 0.0, 1.5)], probe=-1.0), dict(balls=[(0.0, 0.0, 0.0, 1.5)], probe=float("nan")),
               dict(balls=[(0.0, 0.0, 0.0, -1.0)], probe=1.4), dict(balls=[(0.0, 0.0, 0.0, 0.0)], probe=1.4),
               dict(balls=[(float("inf"), 0.0, 0.0, 1.0)], probe=1.4),
               dict(balls=[(0.0, 0.0, 0.0, 1.5)], probe=1.4, volume_probe=-0.5)]:
        with pytest.raises(ValueError):
            V.compute_solvent_spheres(**kw)
    with pytest.raises(OverflowError):
        V.compute_solvent_spheres([(0.0, 0.0, 0.0, 1.5)], 1.4, subdivision_depth=-1)
    assert hasattr(V, "compute_solvent_spheres")
