"""Gmsh ASCII mesh files (MSH 2.2 and 4.1) for tet4 meshes, the input EDGE-V reads through the gmsh
API (tools/edge_v/src/io/Gmsh.cpp:60-251): vertices ascending by node tag, 4-node tetrahedra as
elements, and 3-node triangles of 2D physical groups as tagged boundary faces (101 free surface,
105 outflow in the seismic solver, src/impl/seismic/const.inc:144-146).

read_msh(path) -> (ve [nVe][3], el_ve [nEl][4], bf_ve [nBf][3], bf_tag [nBf]) with 0-based vertex
indices; write_msh(path, ...) writes MSH 2.2 (used by the tests and to hand box meshes to other
tools). A face listed in several physical groups keeps the first one read.
"""
import numpy as np

TET4, TRIA3 = 4, 2  # gmsh element types


def _sections(path):
    """{section name: list of token lists (one per line)} of an ASCII .msh file."""
    out, cur, name = {}, None, None
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0].startswith("$"):
                if t[0].startswith("$End"):
                    out.setdefault(name, []).extend(cur or [])
                    cur, name = None, None
                else:
                    name, cur = t[0][1:], []
                continue
            if cur is not None:
                cur.append(t)
    return out


def _finish(node_tags, crds, tets, tris, tri_phys):
    order = np.argsort(node_tags, kind="stable")
    tags_sorted = np.asarray(node_tags, np.int64)[order]
    ve = np.asarray(crds, np.float64)[order]
    if len(np.unique(tags_sorted)) != len(tags_sorted):
        raise ValueError("duplicate node tags")

    def idx(t):
        t = np.asarray(t, np.int64)
        i = np.searchsorted(tags_sorted, t)
        if np.any(i >= len(tags_sorted)) or np.any(tags_sorted[np.minimum(i, len(tags_sorted) - 1)] != t):
            raise ValueError("element refers to a missing node")
        return i

    el_ve = idx(np.asarray(tets, np.int64).reshape(-1)).reshape(-1, 4) if len(tets) else np.zeros((0, 4), np.int64)
    bf_ve = idx(np.asarray(tris, np.int64).reshape(-1)).reshape(-1, 3) if len(tris) else np.zeros((0, 3), np.int64)
    bf_tag = np.asarray(tri_phys, np.int32)
    if len(bf_ve):
        # a face in several physical groups keeps the first one
        key = np.sort(bf_ve, axis=1)
        _, first = np.unique(key, axis=0, return_index=True)
        first.sort()
        bf_ve, bf_tag = bf_ve[first], bf_tag[first]
    return ve, el_ve, bf_ve, bf_tag


def _read_v2(sec):
    nodes = sec["Nodes"]
    n = int(nodes[0][0])
    tags = [int(r[0]) for r in nodes[1:1 + n]]
    crds = [[float(x) for x in r[1:4]] for r in nodes[1:1 + n]]
    els = sec["Elements"]
    m = int(els[0][0])
    tets, tris, phys = [], [], []
    for r in els[1:1 + m]:
        ty, ntag = int(r[1]), int(r[2])
        conn = [int(x) for x in r[3 + ntag:]]
        if ty == TET4:
            tets.append(conn[:4])
        elif ty == TRIA3 and ntag > 0:
            tris.append(conn[:3])
            phys.append(int(r[3]))
    return _finish(tags, crds, tets, tris, phys)


def _read_v4(sec):
    # physical tags of surface entities
    surf_phys = {}
    if "Entities" in sec:
        ent = sec["Entities"]
        npt, ncu, nsu, _ = (int(x) for x in ent[0][:4])
        for r in ent[1 + npt + ncu:1 + npt + ncu + nsu]:
            tag, nph = int(r[0]), int(r[7])
            surf_phys[tag] = [int(x) for x in r[8:8 + nph]]
    nodes = sec["Nodes"]
    nblk = int(nodes[0][0])
    tags, crds = [], []
    i = 1
    for _ in range(nblk):
        parametric, nin = int(nodes[i][2]), int(nodes[i][3])
        if parametric:
            raise ValueError("parametric node coordinates are not supported")
        tags += [int(r[0]) for r in nodes[i + 1:i + 1 + nin]]
        crds += [[float(x) for x in r[:3]] for r in nodes[i + 1 + nin:i + 1 + 2 * nin]]
        i += 1 + 2 * nin
    els = sec["Elements"]
    nblk = int(els[0][0])
    tets, tris, phys = [], [], []
    i = 1
    for _ in range(nblk):
        dim, etag, ty, nin = (int(x) for x in els[i][:4])
        rows = els[i + 1:i + 1 + nin]
        if ty == TET4:
            tets += [[int(x) for x in r[1:5]] for r in rows]
        elif ty == TRIA3 and dim == 2 and surf_phys.get(etag):
            ph = surf_phys[etag][0]
            for r in rows:
                tris.append([int(x) for x in r[1:4]])
                phys.append(ph)
        i += 1 + nin
    return _finish(tags, crds, tets, tris, phys)


def read_msh(path):
    sec = _sections(path)
    if "MeshFormat" not in sec:
        raise ValueError(f"{path}: not a gmsh file")
    version, binary = sec["MeshFormat"][0][0], int(sec["MeshFormat"][0][1])
    if binary:
        raise ValueError(f"{path}: binary gmsh files are not supported")
    if version.startswith("2"):
        return _read_v2(sec)
    if version.startswith("4"):
        return _read_v4(sec)
    raise ValueError(f"{path}: gmsh format {version} is not supported")


def write_msh(path, ve, el_ve, bf_ve=None, bf_tag=None):
    """MSH 2.2 ASCII: node tags 1..nVe, tagged triangles first, then the tetrahedra."""
    ve = np.asarray(ve, np.float64)
    el_ve = np.asarray(el_ve, np.int64)
    bf_ve = np.zeros((0, 3), np.int64) if bf_ve is None else np.asarray(bf_ve, np.int64)
    bf_tag = np.zeros(0, np.int32) if bf_tag is None else np.asarray(bf_tag, np.int32)
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
        f.write(f"$Nodes\n{len(ve)}\n")
        for i, x in enumerate(ve):
            f.write(f"{i + 1} {float(x[0])!r} {float(x[1])!r} {float(x[2])!r}\n")
        f.write("$EndNodes\n")
        f.write(f"$Elements\n{len(bf_ve) + len(el_ve)}\n")
        k = 1
        for t, tag in zip(bf_ve, bf_tag):
            f.write(f"{k} {TRIA3} 2 {int(tag)} {int(tag)} {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")
            k += 1
        for t in el_ve:
            f.write(f"{k} {TET4} 2 1 1 {t[0] + 1} {t[1] + 1} {t[2] + 1} {t[3] + 1}\n")
            k += 1
        f.write("$EndElements\n")
