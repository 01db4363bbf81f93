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


def test_every_listed_configuration_is_compiled_in():
    """Each order's configurations (edge_b200/csrc/inst_o*.inc) are compiled over several objects;
    every listed one must be found by context creation (which then fails only for the missing
    device, EDGE_B200_EDEVICE, on a machine without one), and an unlisted one must not
    (EDGE_B200_ENOTSUP)."""
    import glob
    L = _lib.lib()
    h = C.c_void_p()
    listed = set()
    for path in glob.glob(os.path.join(ROOT, "edge_b200", "csrc", "inst_o*.inc")):
        for m in re.finditer(r"EDGE_B200_CFG\((float|double),\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+)\)", open(path).read()):
            listed.add((int(m.group(2)), int(m.group(3)), int(m.group(4)), int(m.group(5))))
    assert len(listed) > 30
    for order in range(2, 7):
        for runs in (1, 4, 8, 16):
            for rms in (0, 3):
                for prec in (32, 64):
                    c = _lib.Cfg(stream=None, device=0, order=order, n_runs=runs, n_rms=rms, precision=prec)
                    rc = L.edge_b200_create(C.byref(c), 10, C.byref(h))
                    if rc == 0:  # a machine with a device
                        L.edge_b200_destroy(h)
                        assert (order, runs, rms, prec) in listed
                    elif (order, runs, rms, prec) in listed:
                        assert rc == -3, (order, runs, rms, prec, rc)  # found; no device here
                    else:
                        assert rc == -5, (order, runs, rms, prec, rc)
