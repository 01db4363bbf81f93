"""Per-face permuted face bases of the sparse kernels (edge_b200/gen_kernels.py): the local lift of
a face projection and the neighbour path (projection at the neighbour's face fo, orientation V from
kFacePerm, lift at this element's face FA) equal the reference's operators (fluxL, fluxT and
fluxN = fluxL_fo Mface^-1 Ori_v, dg/DgMats setup of AderDgInit) for every (fo, FA, v)."""
import numpy as np
import pytest

from edge_b200 import dgmat, gen_kernels as gk


def _f(m):
    return np.array([[float(x) for x in row] for row in m])


@pytest.mark.parametrize("order", [2, 3, 4, 5, 6])
def test_permuted_face_bases_reproduce_reference_operators(order):
    ex = dgmat.exact_matrices(order)
    fb = gk.face_bases(order)
    sig = [b[0] for b in fb]
    tab = gk.face_perm_table(sig)
    ori_ref = gk.exact_orientations(order)  # [id, r1, r2, reflections 0..2]
    fl = [_f(ex["fluxL"][f]) for f in range(4)]
    ft = [_f(ex["fluxT"][f]) for f in range(4)]
    fl2 = [_f(b[1]) for b in fb]
    ft2 = [_f(b[2]) for b in fb]
    nb = fl[0].shape[0]
    rng = np.random.default_rng(order)
    u = rng.normal(size=(nb, 3))
    for fa in range(4):
        # local term: lift of the own projection
        np.testing.assert_allclose(ft2[fa].T @ (fl2[fa].T @ u), ft[fa].T @ (fl[fa].T @ u), rtol=0, atol=1e-11)
        assert np.count_nonzero(fl2[fa]) <= np.count_nonzero(fl[fa])
        for fo in range(4):
            for v in range(3):
                ref = ft[fa].T @ (_f(ori_ref[3 + v]).T @ (fl[fo].T @ u))
                V = tab[fo][fa][v]
                got = ft2[fa].T @ (_f(ori_ref[3 + V]).T @ (fl2[fo].T @ u))
                np.testing.assert_allclose(got, ref, rtol=0, atol=1e-11)


def test_face_bases_sparsity_order5():
    nnz = [sum(1 for row in b[1] for x in row if x != 0) for b in gk.face_bases(5)]
    assert nnz == [35, 105, 304, 304]


def test_generated_table_matches_generator():
    import os
    import re
    path = os.path.join(os.path.dirname(gk.__file__), "csrc", "gen", "dg_sparse.cuh")
    src = open(path).read()
    body = src[src.index("kFacePerm[5][4][4][3] = ") + len("kFacePerm[5][4][4][3] = "):]
    nums = [int(x) for x in re.findall(r"-?\d+", body[:body.index(";")])]
    want = []
    for o in range(2, 7):
        tab = gk.face_perm_table([b[0] for b in gk.face_bases(o)])
        want += [tab[fo][fa][v] for fo in range(4) for fa in range(4) for v in range(3)]
    assert nums == want


@pytest.mark.parametrize("order", [2, 3, 4, 5, 6])
def test_derivative_directions_keep_the_star_stiffness_sum(order):
    """sum_a star'_a (x) K'_a == sum_dim star_dim (x) K_dim for the generated direction basis
    (stiffT of the recursion and stiffV of the volume), with star'_a = sum_dim DIRS^-1[dim][a]."""
    ex = dgmat.exact_matrices(order)
    inv = np.array([[float(x) for x in row] for row in gk.dirs_inverse()])
    np.testing.assert_allclose(np.array(gk.DIRS, float) @ inv, np.eye(3), atol=0)
    rng = np.random.default_rng(order)
    star = rng.normal(size=(3, 9, 9))
    star2 = np.einsum("da,dij->aij", inv, star)
    for key in ("stiffT", "stiffV"):
        K = np.array([_f(m) for m in ex[key]])
        K2 = np.array([_f(m) for m in gk.combine_dirs(ex[key])])
        ref = np.einsum("dij,dkn->ikjn", star, K)
        got = np.einsum("aij,akn->ikjn", star2, K2)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * np.abs(ref).max())
        assert np.count_nonzero(K2) < np.count_nonzero(K)
