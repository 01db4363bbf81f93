"""Legacy VTK files of wave-field snapshots (the output of EDGE's io::WaveField, src/io/Vtk.cpp:30-121):
the tet mesh as an unstructured grid and, per fused run and quantity, the element's mode-0
coefficient as cell data named crun_<run>_var_<quantity>."""
import numpy as np


def write(path, ve, el_ve, cell_data, binary=False):
    """cell_data [R][9][nEl] (e.g. Solver.wavefield()); ASCII or big-endian binary legacy VTK 3.0."""
    ve = np.asarray(ve, np.float32)
    el_ve = np.asarray(el_ve, np.int32)
    cell_data = np.asarray(cell_data, np.float32)
    n_el = len(el_ve)
    mode = "wb"
    with open(path, mode) as f:
        w = lambda t: f.write(t.encode())
        w("# vtk DataFile Version 3.0\nedge_b200 wave field\n")
        w("BINARY\n" if binary else "ASCII\n")
        w("DATASET UNSTRUCTURED_GRID\n")
        w(f"POINTS {len(ve)} float\n")
        if binary:
            f.write(ve.astype(">f4").tobytes())
            w("\n")
        else:
            w("\n".join(" ".join(repr(float(c)) for c in p) for p in ve) + "\n")
        w(f"CELLS {n_el} {n_el * 5}\n")
        cells = np.concatenate([np.full((n_el, 1), 4, np.int32), el_ve], axis=1)
        if binary:
            f.write(cells.astype(">i4").tobytes())
            w("\n")
        else:
            w("\n".join(" ".join(str(int(c)) for c in row) for row in cells) + "\n")
        w(f"CELL_TYPES {n_el}\n")
        types = np.full(n_el, 10, np.int32)  # VTK_TETRA
        if binary:
            f.write(types.astype(">i4").tobytes())
            w("\n")
        else:
            w("\n".join(str(int(t)) for t in types) + "\n")
        w(f"CELL_DATA {n_el}\n")
        for r in range(cell_data.shape[0]):
            for q in range(cell_data.shape[1]):
                w(f"SCALARS crun_{r}_var_{q} float 1\nLOOKUP_TABLE default\n")
                if binary:
                    f.write(cell_data[r, q].astype(">f4").tobytes())
                    w("\n")
                else:
                    w("\n".join(repr(float(x)) for x in cell_data[r, q]) + "\n")


def read_cell_data(path):
    """{name: values} of the cell scalars of an ASCII file written by write() (tests)."""
    out, cur, n = {}, None, 0
    lines = open(path).read().split("\n")
    i = 0
    while i < len(lines):
        t = lines[i].split()
        if t and t[0] == "CELL_DATA":
            n = int(t[1])
        elif t and t[0] == "SCALARS":
            cur = t[1]
            vals = [float(x) for x in lines[i + 2:i + 2 + n]]
            out[cur] = np.array(vals, np.float32)
            i += 2 + n
            continue
        i += 1
    return out
