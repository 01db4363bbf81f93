"""Box meshes and elastic element data for the CPU reference runs (TEST INFRASTRUCTURE ONLY).

Only ``tests/`` and the CPU legs of ``bench.py`` use this module. It restates, in numpy, the
EDGE-V conventions the reference's solver consumes for a box of cubes split into six tets along the
main diagonal, so that the reference's own kernels (``oracle/_ref``) can be fed without the CUDA
library:

* element vertices sorted ascending, then the last two swapped when the Jacobian determinant is
  negative (tools/edge_v/src/mesh/Mesh.cpp:312-313, geom/Tet4.cpp:80-112);
* local face f of an element with vertices a<b<c<d in face-parameter order (0,2,1), (0,1,3),
  (0,3,2), (1,2,3) (tools/edge_pre/edge_pre/types/Tet.py:89-97); faces numbered in order of first
  appearance, the smaller element on the left (Mesh.cpp:288-375);
* neighbour face ids (geom/Generic.cpp:92-116) and vertex ids (geom/Tet4.cpp:114-229);
* face frames: tangents from the first edge and its orthogonalised partner, normal away from the
  left element's fourth vertex (geom/Tria3.cpp:48-120, Mesh.cpp:763-841);
* boundary faces on the top plane z = ext get ``bc_top``, the others ``bc_sides``
  (1 free surface, 2 outflow).

Element data come from the reference's compiled ``Elasticity::star`` / ``Elasticity::fs`` (through
``oracle/ref.py``), with the star matrices of AderDgInit::initStar (AderDgInit.hpp:129-174) and the
face scaling -2 area / detJ of AderDgInit::initFs (AderDgInit.hpp:568-646).
"""
import ctypes as C

import numpy as np

FACE_INNER, FACE_FREE_SURFACE, FACE_OUTFLOW = 0, 1, 2
FA_VE = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]])
PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def box(n, ext=1e4, bc_top=FACE_FREE_SURFACE, bc_sides=FACE_OUTFLOW):
    """n^3 cubes x 6 tets of the box [0, ext]^3 (no jitter). Returns a dict of the mesh arrays."""
    v1 = n + 1
    h = ext / n
    k, j, i = np.meshgrid(np.arange(v1), np.arange(v1), np.arange(v1), indexing="ij")
    ve = np.stack([i.ravel() * h, j.ravel() * h, k.ravel() * h], axis=1).astype(np.float64)
    vid = lambda a, b, c: a + v1 * (b + v1 * c)
    ck, cj, ci = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    el = np.zeros((n ** 3, 6, 4), np.int64)
    for p, perm in enumerate(PERMS):
        idx = [ci.copy(), cj.copy(), ck.copy()]
        el[:, p, 0] = vid(*idx)
        for s in range(3):
            idx[perm[s]] = idx[perm[s]] + 1
            el[:, p, s + 1] = vid(*idx)
    el_ve = np.sort(el.reshape(-1, 4), axis=1)
    n_el = len(el_ve)
    jac = ve[el_ve[:, 1:]] - ve[el_ve[:, :1]]
    det = np.linalg.det(jac)
    flip = det < 0
    el_ve[flip, 2], el_ve[flip, 3] = el_ve[flip, 3].copy(), el_ve[flip, 2].copy()
    # faces in order of first appearance
    fv = np.sort(el_ve[:, FA_VE].reshape(-1, 3), axis=1)
    key = (fv[:, 0] * v1 ** 3 + fv[:, 1]) * v1 ** 3 + fv[:, 2]
    uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
    rank = np.empty(len(uniq), np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(uniq))
    el_fa = rank[inv].reshape(n_el, 4)
    n_fa = len(uniq)
    fa_ve = np.zeros((n_fa, 3), np.int64)
    fa_ve[el_fa.ravel()] = fv
    fa_el = np.full((n_fa, 2), -1, np.int64)
    occ = np.arange(4 * n_el) // 4
    order = np.argsort(el_fa.ravel(), kind="stable")
    sf = el_fa.ravel()[order]
    so = occ[order]
    start = np.r_[0, np.flatnonzero(np.diff(sf)) + 1]
    fa_el[sf[start], 0] = so[start]
    second = start + 1
    ok = second < len(sf)
    ok[ok] &= sf[second[ok]] == sf[start[ok]]
    fa_el[sf[start[ok]], 1] = so[second[ok]]
    # neighbours, boundary types
    a, b = fa_el[el_fa, 0], fa_el[el_fa, 1]
    el_fa_el = np.where(a == np.arange(n_el)[:, None], b, a).astype(np.int32)
    top = np.all(np.abs(ve[fa_ve, 2] - ext) < 1e-9 * ext, axis=1)
    fa_type = np.where(fa_el[:, 1] >= 0, FACE_INNER, np.where(top, bc_top, bc_sides)).astype(np.uint8)
    el_fa_type = fa_type[el_fa]
    # neighbour face and vertex ids
    fid = np.full((n_el, 4), 255, np.uint8)
    vidn = np.full((n_el, 4), 255, np.uint8)
    e_idx, f_idx = np.nonzero(el_fa_el >= 0)
    ne = el_fa_el[e_idx, f_idx]
    match = el_fa[ne] == el_fa[e_idx, f_idx][:, None]
    f_ad = np.argmax(match, axis=1)
    ve0 = np.where(f_idx <= 2, el_ve[e_idx, 0], el_ve[e_idx, 1])
    ve_ad = np.argmax(el_ve[ne] == ve0[:, None], axis=1)
    v_id = np.argmax(FA_VE[f_ad] == ve_ad[:, None], axis=1)
    fid[e_idx, f_idx] = f_ad
    vidn[e_idx, f_idx] = v_id
    # face frames, areas; element volumes
    v = ve[fa_ve]
    d0 = v[:, 1] - v[:, 0]
    d1 = v[:, 2] - v[:, 0]
    alpha = -np.einsum("ij,ij->i", d0, d1) / np.einsum("ij,ij->i", d0, d0)
    n0 = d1 + alpha[:, None] * d0
    d0 = d0 / np.linalg.norm(d0, axis=1)[:, None]
    n0 = n0 / np.linalg.norm(n0, axis=1)[:, None]
    n1 = np.cross(d0, n0)
    left = el_ve[fa_el[:, 0]]
    opp = left.sum(axis=1) - fa_ve.sum(axis=1)  # the left element's vertex off the face
    swap = np.einsum("ij,ij->i", n1, ve[opp] - v[:, 0]) > 0
    t0 = np.where(swap[:, None], n0, d0)
    t1 = np.where(swap[:, None], d0, n0)
    normal = np.cross(t0, t1)
    area = np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1) / 2
    jac = ve[el_ve[:, 1:]] - ve[el_ve[:, :1]]
    vol = np.abs(np.linalg.det(jac)) / 6
    india = 12 * vol / (2 * area[el_fa].sum(axis=1))
    return dict(n_el=n_el, n_fa=n_fa, ve=ve, el_ve=el_ve, el_fa=el_fa, fa_el=fa_el, fa_ve=fa_ve,
                el_fa_el=el_fa_el, fid=fid, vid=vidn, el_fa_type=el_fa_type, fa_type=fa_type,
                fa_normal=normal, fa_tangent=np.stack([t0, t1], axis=1), fa_area=area, el_vol=vol,
                el_india=india, jac=jac)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def elastic_data(L, m, rho, lam, mu):
    """starE[nEl][3][24] and fsE[2][nEl][4][81] from the reference's compiled Elasticity code
    (``L`` = an oracle/_ref library)."""
    n_el = m["n_el"]
    star = np.zeros((n_el, 3, 24))
    ji = np.ascontiguousarray(np.linalg.inv(m["jac"]))
    for e in range(n_el):
        L.ref_star(rho[e], lam[e], mu[e], _p(ji[e]), _p(star[e]))
    fs = np.zeros((2, n_el, 4, 81))
    det = np.linalg.det(m["jac"])
    fl, fr = np.zeros(81), np.zeros(81)
    for fa in range(m["n_fa"]):
        eL, eR = (int(x) for x in m["fa_el"][fa])
        n = np.ascontiguousarray(m["fa_normal"][fa])
        s = np.ascontiguousarray(m["fa_tangent"][fa, 0])
        t = np.ascontiguousarray(m["fa_tangent"][fa, 1])
        mR = eR if eR >= 0 else eL
        fsurf = 1 if m["fa_type"][fa] == FACE_FREE_SURFACE else 0
        fL = int(np.flatnonzero(m["el_fa"][eL] == fa)[0])
        L.ref_fs(rho[eL], rho[mR], lam[eL], lam[mR], mu[eL], mu[mR], _p(n), _p(s), _p(t), fsurf, _p(fl), _p(fr))
        sc = -m["fa_area"][fa] / det[eL] * 2
        fs[0, eL, fL], fs[1, eL, fL] = fl * sc, fr * sc
        if eR >= 0:
            fR = int(np.flatnonzero(m["el_fa"][eR] == fa)[0])
            nm = np.ascontiguousarray(-n)
            L.ref_fs(rho[eR], rho[eL], lam[eR], lam[eL], mu[eR], mu[eL], _p(nm), _p(s), _p(t), 0, _p(fl), _p(fr))
            sc = -m["fa_area"][fa] / det[eR] * 2
            fs[0, eR, fR], fs[1, eR, fR] = fl * sc, fr * sc
    return star, fs
