"""The C-ABI library loads and exports every function include/edge_b200.h declares (no GPU needed),
and the host-side argument checks reject bad input before touching a device."""
import ctypes as C
import os
import re

import numpy as np

from edge_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "edge_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(edge_(?:b200|mesh|setup)_\w+)\s*\(", txt)))


def test_every_declared_symbol_is_exported():
    L = _lib.lib()
    names = declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.EXPORTED, n


def test_create_rejects_bad_config_without_gpu():
    L = _lib.lib()
    h = C.c_void_p()
    for cfg in (dict(order=4, n_runs=3, n_rms=0, precision=64), dict(order=4, n_runs=1, n_rms=4, precision=64),
                dict(order=4, n_runs=1, n_rms=0, precision=16), dict(order=9, n_runs=1, n_rms=0, precision=64)):
        c = _lib.Cfg(stream=None, device=0, **cfg)
        rc = L.edge_b200_create(C.byref(c), 10, C.byref(h))
        assert rc in (-1, -5), (cfg, rc)


def test_mesh_rejects_bad_arguments():
    L = _lib.lib()
    h = C.c_void_p()
    ext = np.array([1.0, 1.0, 1.0])
    assert L.edge_mesh_box(0, 1, 1, _lib.ptr(ext), 0.0, 0, 1, 2, C.byref(h)) == -1
    assert L.edge_mesh_box(1, 1, 1, _lib.ptr(ext), 0.6, 0, 1, 2, C.byref(h)) == -1
    assert L.edge_mesh_box(1, 1, 1, _lib.ptr(ext), 0.0, 0, 7, 2, C.byref(h)) == -1
