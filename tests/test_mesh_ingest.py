"""Mesh ingest (edge_mesh_from_arrays, gmsh files): EDGE-V's conventions on arbitrary tet meshes.

A box mesh exported to vertex/element/tagged-face arrays (and to gmsh files) and read back must
give the same connectivity, orientation data and geometry; with the Z-order reordering the mesh is
the same up to the element permutation, and the element update (the oracle) is equivariant under
it, which pins the neighbour face / vertex ids of the reordered mesh.
"""
import os

import numpy as np
import pytest

from edge_b200 import gmsh, host
from helpers import OracleRun, random_dofs


def _export(m):
    bf_ve, tag = m.boundary_faces()
    return m.ve.copy(), m.el_ve.copy(), bf_ve, tag


def _same_mesh(a, b):
    for k in ("el_ve", "el_fa_el", "fid", "vid", "el_fa_type", "fa_el", "fa_type"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    for k in ("ve", "fa_normal", "fa_tangent", "fa_area", "el_vol", "el_india"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)


@pytest.mark.parametrize("jitter", [0.0, 0.2])
def test_arrays_roundtrip_identical(jitter):
    box = host.Mesh.box(3, (1e4,) * 3, jitter=jitter, seed=7)
    m = host.Mesh.from_arrays(*_export(box), reorder=False)
    _same_mesh(m, box)
    assert np.array_equal(m.el_perm, np.arange(box.n_el))


def test_gmsh_v2_roundtrip(tmp_path):
    box = host.Mesh.box(3, (1e4,) * 3, jitter=0.15, seed=11)
    ve, el_ve, bf_ve, tag = _export(box)
    # shuffle the vertex numbering and the element vertex order: the reader and the EDGE-V
    # normalisation must undo both
    rng = np.random.default_rng(0)
    vperm = rng.permutation(len(ve))
    inv = np.argsort(vperm)
    el_sh = inv[el_ve]
    el_sh = np.take_along_axis(el_sh, rng.permuted(np.tile(np.arange(4), (len(el_sh), 1)), axis=1), axis=1)
    path = os.path.join(tmp_path, "box.msh")
    gmsh.write_msh(path, ve[vperm], el_sh, inv[bf_ve], tag)
    ve2, el2, bf2, tag2 = gmsh.read_msh(path)
    np.testing.assert_array_equal(ve2, ve[vperm])
    m = host.Mesh.from_arrays(ve2, el2, bf2, tag2, reorder=False)
    # same elements (vertex sets, mapped back), neighbours and face types; the local vertex and
    # face numbering follows the new vertex ids
    assert np.array_equal(np.sort(vperm[m.el_ve], axis=1), np.sort(box.el_ve, axis=1))
    assert np.array_equal(np.sort(m.el_fa_el, axis=1), np.sort(box.el_fa_el, axis=1))
    np.testing.assert_allclose(m.el_vol, box.el_vol, rtol=1e-12)
    key = lambda mm, vmap: {tuple(sorted(vmap[f])): t for f, t in zip(mm.fa_ve(), mm.fa_type)}
    assert key(m, vperm) == key(box, np.arange(len(ve)))
    # the discrete solution does not depend on the local numbering: receiver traces of a point
    # source agree to rounding (this pins the neighbour face and vertex ids of the new numbering)
    kw = dict(jitter=0.15, seed=11, n_receivers=5, source="random", n_steps=12)
    pa = host.build_problem(3, 3, 1, **kw)
    ra = _receiver_traces(pa, 12)
    assert np.abs(ra).max() > 0
    for reorder in (False, True):
        mm = host.Mesh.from_arrays(ve2, el2, bf2, tag2, reorder=reorder)
        rb = _receiver_traces(host.build_problem(3, 3, 1, mesh=mm, **kw), 12)
        np.testing.assert_allclose(rb, ra, rtol=0, atol=1e-12 * np.abs(ra).max())


def _receiver_traces(prob, steps):
    """Oracle receiver buffers in the order the receiver positions were drawn."""
    r = OracleRun(prob)
    r.step(steps)
    out = np.zeros_like(r.recv["buf"])
    out[prob.receivers["perm"]] = r.recv["buf"]
    return out


def _write_v41(path, ve, el_ve, bf_ve, tag):
    """MSH 4.1 with one volume entity and one surface entity per physical tag."""
    tags = sorted(set(int(t) for t in tag))
    with open(path, "w") as f:
        f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
        f.write(f"$Entities\n0 0 {len(tags)} 1\n")
        for i, t in enumerate(tags):
            f.write(f"{i + 1} 0 0 0 1 1 1 1 {t} 0\n")
        f.write("1 0 0 0 1 1 1 0 0\n$EndEntities\n")
        f.write(f"$Nodes\n1 {len(ve)} 1 {len(ve)}\n3 1 0 {len(ve)}\n")
        for i in range(len(ve)):
            f.write(f"{i + 1}\n")
        for x in ve:
            f.write(f"{float(x[0])!r} {float(x[1])!r} {float(x[2])!r}\n")
        f.write("$EndNodes\n")
        n = len(el_ve) + len(bf_ve)
        f.write(f"$Elements\n{1 + len(tags)} {n} 1 {n}\n")
        k = 1
        for i, t in enumerate(tags):
            sel = bf_ve[tag == t]
            f.write(f"2 {i + 1} 2 {len(sel)}\n")
            for tri in sel:
                f.write(f"{k} {tri[0] + 1} {tri[1] + 1} {tri[2] + 1}\n")
                k += 1
        f.write(f"3 1 4 {len(el_ve)}\n")
        for tet in el_ve:
            f.write(f"{k} {tet[0] + 1} {tet[1] + 1} {tet[2] + 1} {tet[3] + 1}\n")
            k += 1
        f.write("$EndElements\n")


def test_gmsh_v41_reader(tmp_path):
    box = host.Mesh.box(2, (1e4,) * 3, jitter=0.1, seed=3)
    ve, el_ve, bf_ve, tag = _export(box)
    path = os.path.join(tmp_path, "box41.msh")
    _write_v41(path, ve, el_ve, bf_ve, tag)
    ve2, el2, bf2, tag2 = gmsh.read_msh(path)
    np.testing.assert_array_equal(ve2, ve)
    assert np.array_equal(el2, el_ve)
    m = host.Mesh.from_arrays(ve2, el2, bf2, tag2, reorder=False)
    _same_mesh(m, box)


def test_reordered_mesh_is_a_permutation():
    box = host.Mesh.box(4, (1e4,) * 3, jitter=0.2, seed=5)
    ve, el_ve, bf_ve, tag = _export(box)
    rng = np.random.default_rng(1)
    shuffle = rng.permutation(box.n_el)
    m = host.Mesh.from_arrays(ve, el_ve[shuffle], bf_ve, tag, reorder=True)
    src = shuffle[m.el_perm]  # box element of each mesh element
    assert np.array_equal(m.el_ve, box.el_ve[src])
    inv = np.argsort(src)
    nb = m.el_fa_el
    assert np.array_equal(np.where(nb >= 0, src[np.maximum(nb, 0)], -1), box.el_fa_el[src])
    assert np.array_equal(m.fid, box.fid[src]) and np.array_equal(m.vid, box.vid[src])
    np.testing.assert_array_equal(m.el_india, box.el_india[src])
    # Z-order puts face neighbours close: median index distance well below a random order's
    d = np.abs(np.arange(m.n_el)[:, None] - np.where(nb >= 0, nb, np.arange(m.n_el)[:, None]))
    assert np.median(d[nb >= 0]) < m.n_el / 8
    assert len(inv) == m.n_el


def test_element_update_equivariant_under_reordering():
    order, steps = 3, 3
    base = host.build_problem(3, order, 1, jitter=0.2, seed=9, n_receivers=0, source=None)
    ve, el_ve, bf_ve, tag = _export(base.mesh)
    m = host.Mesh.from_arrays(ve, el_ve, bf_ve, tag, reorder=True)
    re = host.build_problem(3, order, 1, seed=9, n_receivers=0, source=None, mesh=m)
    e0, _ = random_dofs(base, seed=4)
    a = OracleRun(base, e0)
    b = OracleRun(re, np.ascontiguousarray(e0[m.el_perm]))
    a.step(steps)
    b.step(steps)
    # the same physics; the renumbered setup rounds its geometry in another order
    got, want = b.state["dofsE"], a.state["dofsE"][m.el_perm]
    assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)


def test_ingest_errors():
    box = host.Mesh.box(2, (1e4,) * 3)
    ve, el_ve, bf_ve, tag = _export(box)
    with pytest.raises(RuntimeError, match="ENOTSUP"):
        host.Mesh.from_arrays(ve, el_ve, bf_ve, np.full_like(tag, 106))
    with pytest.raises(RuntimeError, match="EMESH"):
        host.Mesh.from_arrays(ve, el_ve, bf_ve[:-1], tag[:-1], default_type=-1)
    # untagged boundary faces take the default type
    m = host.Mesh.from_arrays(ve, el_ve, default_type=host.FACE_OUTFLOW, reorder=False)
    assert set(np.unique(m.fa_type[m.fa_el[:, 1] < 0])) == {host.FACE_OUTFLOW}
    # a face shared by three elements
    bad = np.concatenate([el_ve, el_ve[:1]])
    with pytest.raises(RuntimeError, match="EMESH"):
        host.Mesh.from_arrays(ve, bad, bf_ve, tag)
    # a flat element
    flat = ve.copy()
    e = el_ve[0]
    flat[e[3]] = (flat[e[0]] + flat[e[1]] + flat[e[2]]) / 3
    with pytest.raises(RuntimeError, match="EMESH"):
        host.Mesh.from_arrays(flat, el_ve, bf_ve, tag)


@pytest.mark.parametrize("jitter", [0.1, 0.2])
def test_box_jitter_moves_interior_vertices_only(jitter):
    n, ext = 6, 1e4
    box = host.Mesh.box(n, (ext,) * 3, jitter=jitter, seed=3)
    h = ext / n
    grid = box.ve / h
    off = np.abs(grid - np.round(grid)).max(axis=1)
    on_boundary = np.any((np.abs(box.ve) < 1e-9) | (np.abs(box.ve - ext) < 1e-9 * ext), axis=1)
    assert np.all(off[on_boundary] < 1e-9)             # boundary vertices stay on the box planes
    interior = ~on_boundary
    assert np.mean(off[interior] > 1e-6) > 0.9        # nearly every interior vertex moved
    assert np.all(off[interior] <= jitter + 1e-9)      # ... by at most jitter * h per coordinate
    assert np.all(box.el_vol > 0)
    normals = box.fa_normal
    assert np.mean(np.any(np.abs(normals) > 1 - 1e-12, axis=1)) < 0.5  # generic face orientations
