"""The characteristic face mix of the local kernel rests on one property of the elastic flux
solvers: for every face, the element's own flux solver fsE[0] and the one its face reader applies
(fsE[1] of the neighbour at its face, the element's own for a free surface, none for outflow),
stacked into an 18 x 9 matrix, have rank 3 -- the three waves (P, S, S) that leave the element
through the face. The device then mixes each face projection through three characteristic rows
instead of two 9 x 9 blocks. Checked here on the host-built flux solvers (pinned to the reference's
Elasticity code in test_host_setup.py) for heterogeneous, layered, jittered meshes with every face
type, with the oracle's restatement of the factorisation the device builds (column-scaled
Gram-Schmidt with pivoting, each direction orthogonalised twice)."""
import numpy as np
import pytest

import oracle
from edge_b200 import host
from helpers import small_problem


def _pairs(p):
    fs = np.asarray(p.fsE)
    ef, fid, ty = np.asarray(p.mesh.el_fa_el), np.asarray(p.mesh.fid), np.asarray(p.mesh.el_fa_type)
    for e in range(p.n_el):
        for f in range(4):
            t = int(ty[e, f])
            a = fs[0, e, f].reshape(9, 9)
            if t == host.FACE_INNER:
                b = fs[1, ef[e, f], fid[e, f]].reshape(9, 9)
            elif t == host.FACE_FREE_SURFACE:
                b = fs[1, e, f].reshape(9, 9)
            else:
                b = np.zeros((9, 9))
            yield t, np.vstack([a, b])


@pytest.mark.parametrize("bc_sides", [host.FACE_OUTFLOW, host.FACE_FREE_SURFACE])
def test_stacked_flux_solvers_have_rank_three(bc_sides):
    p = small_problem(n=3, order=3, runs=1, jitter=0.2, seed=5, n_steps=2, source=None, n_receivers=0,
                      layers=[3000.0, 6000.0], lognormal_sigma=0.1, bc_sides=bc_sides)
    seen = set()
    for t, S in _pairs(p):
        seen.add(t)
        s = np.linalg.svd(S, compute_uv=False)
        assert s[2] > 1e-3 * s[0]  # three waves
        assert s[3] < 1e-12 * s[0]  # and no more
        V, U0, U1 = oracle.flux_char_factors(S[:9], S[9:] if np.any(S[9:]) else None)
        U = np.vstack([U0, U1])
        # every entry reproduced to rounding relative to its row and its column
        scale = np.minimum(np.abs(S).max(axis=1)[:, None], np.abs(S).max(axis=0)[None, :])
        assert np.all(np.abs(U @ V.T - S) <= 1e-12 * scale + 1e-300)
    assert host.FACE_INNER in seen and bc_sides in seen and host.FACE_FREE_SURFACE in seen
