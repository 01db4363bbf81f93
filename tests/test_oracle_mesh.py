"""The oracle's numpy box mesh (used to feed the reference's own kernels without the CUDA library)
against the host setup in the CUDA library: identical connectivity, face / vertex ids and boundary
types, the same geometry to rounding, and element data from the reference's compiled
Elasticity::star / ::fs equal to the host setup's."""
import numpy as np
import pytest

import mesh as om
import ref as refmod
from edge_b200 import host


@pytest.mark.parametrize("n,top,sides", [(2, 1, 2), (3, 2, 2), (4, 1, 1), (5, 1, 2)])
def test_box_matches_host_setup(n, top, sides):
    m = om.box(n, 1e4, bc_top=top, bc_sides=sides)
    h = host.Mesh.box(n, bc_top=top, bc_sides=sides)
    for k in ("el_ve", "el_fa", "fa_el", "el_fa_el", "fid", "vid", "el_fa_type", "fa_type"):
        np.testing.assert_array_equal(m[k], getattr(h, k), err_msg=k)
    for k in ("ve", "fa_normal", "fa_tangent", "fa_area", "el_vol", "el_india"):
        a, b = m[k], getattr(h, k)
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max(), err_msg=k)


def test_elastic_data_from_reference_matches_host_setup():
    L = refmod.load(4, 1, 0)
    if L is None:
        pytest.skip("reference kernels not built (oracle/_ref)")
    n = 3
    m = om.box(n)
    h = host.Mesh.box(n)
    rng = np.random.default_rng(5)
    rho = rng.uniform(2000, 3000, m["n_el"])
    mu = rho * rng.uniform(2000, 3500, m["n_el"]) ** 2
    lam = rho * rng.uniform(5000, 7000, m["n_el"]) ** 2 - 2 * mu
    star, fs = om.elastic_data(L, m, rho, lam, mu)
    star_h = host.star(h, rho, lam, mu)
    fs_h, _ = host.flux_solvers(h, rho, lam, mu)
    np.testing.assert_allclose(star, star_h, rtol=0, atol=1e-13 * np.abs(star_h).max())
    np.testing.assert_allclose(fs, fs_h, rtol=0, atol=1e-13 * np.abs(fs_h).max())
