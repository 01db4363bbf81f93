"""Wave-field VTK files (edge_b200.vtk) on the CPU: structure and round trip of the cell data."""
import os

import numpy as np

from edge_b200 import host, vtk


def test_ascii_round_trip_and_structure(tmp_path):
    m = host.Mesh.box(2, (1e4,) * 3)
    rng = np.random.default_rng(0)
    data = rng.normal(size=(2, 9, m.n_el)).astype(np.float32)
    path = os.path.join(tmp_path, "wf.vtk")
    vtk.write(path, m.ve, m.el_ve, data)
    back = vtk.read_cell_data(path)
    assert sorted(back) == sorted(f"crun_{r}_var_{q}" for r in range(2) for q in range(9))
    for r in range(2):
        for q in range(9):
            np.testing.assert_array_equal(back[f"crun_{r}_var_{q}"], data[r, q])
    text = open(path).read()
    assert f"POINTS {m.n_ve} float" in text and f"CELLS {m.n_el} {5 * m.n_el}" in text
    assert f"CELL_TYPES {m.n_el}" in text


def test_binary_layout(tmp_path):
    m = host.Mesh.box(1, (1.0,) * 3)
    data = np.arange(9 * m.n_el, dtype=np.float32).reshape(1, 9, m.n_el)
    path = os.path.join(tmp_path, "wf.vtk")
    vtk.write(path, m.ve, m.el_ve, data, binary=True)
    raw = open(path, "rb").read()
    head = raw.index(b"SCALARS crun_0_var_3 float 1\nLOOKUP_TABLE default\n")
    start = head + len(b"SCALARS crun_0_var_3 float 1\nLOOKUP_TABLE default\n")
    vals = np.frombuffer(raw[start:start + 4 * m.n_el], ">f4")
    np.testing.assert_array_equal(vals, data[0, 3])
