"""Device error norms (edge_b200_error_norms) against the same quadrature evaluated with numpy."""
import numpy as np
import pytest

from edge_b200 import host
from edge_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _numpy_norms(prob, dofs, fn, t, n_quad):
    pts, wts = host.tet_quadrature(n_quad)
    V = host.basis_at(prob.order, pts)
    v = prob.mesh.el_ve_crds()
    J = v[:, 1:, :] - v[:, :1, :]
    det = np.abs(np.linalg.det(J))
    x = v[:, None, 0, :] + np.einsum("pa,ead->epd", pts, J)
    ref = fn(x, t)                                      # [E][P][9]
    uh = np.einsum("pb,eqbr->epqr", V, np.asarray(dofs, np.float64))
    d = np.abs(uh - ref[..., None])
    w = wts[None, :, None, None] * det[:, None, None, None]
    return (d * w).sum((0, 1)), np.sqrt((d * d * w).sum((0, 1))), d.max((0, 1))


@pytest.mark.parametrize("precision,order,runs", [(64, 4, 1), (32, 5, 16)])
def test_norms_match_numpy(precision, order, runs):
    ext, P = 1e4, host.FACE_PERIODIC
    prob = host.build_problem(3, order, runs, ext=ext, jitter=0.1, seed=4, n_receivers=0, source=None,
                              bc_top=P, bc_sides=P)
    rho, lam, mu = prob.rho[0], prob.lam[0], prob.mu[0]
    k = [2 * np.pi / ext, 0.0, 2 * np.pi / ext]
    fn = host.plane_wave_p(rho, lam, mu, k)
    e0 = np.repeat(host.project(prob.mesh, order, fn), runs, axis=3)
    s = Solver(prob, precision=precision)
    try:
        s.upload_dofs(e0.astype(s.dtype))
        s.upload_geometry()
        s.step(5)
        l1, l2, li = s.error_norms(host.plane_wave_rows(rho, lam, mu, k), t=s.t)
        e, _ = s.download_dofs()
    finally:
        s.close()
    n1, n2, ni = _numpy_norms(prob, e, fn, 5 * prob.dt, order + 1)
    tol = 1e-10 if precision == 64 else 1e-5
    np.testing.assert_allclose(l1, n1, rtol=tol)
    np.testing.assert_allclose(l2, n2, rtol=tol)
    np.testing.assert_allclose(li, ni, rtol=tol)
    # the DG solution stays close to the wave: x-velocity error well below its norm
    # (amplitude n_x = 1/sqrt(2), rms over the box ext^3 of a sine: 1/2)
    assert np.all(l2[6] < 0.05 * 0.5 * ext ** 1.5)


def test_wavefield_is_mode_zero(tmp_path):
    from edge_b200 import vtk
    prob = host.build_problem(3, 4, 16, seed=6, n_receivers=0, source="random", n_steps=10)
    s = Solver(prob, precision=32)
    try:
        s.upload_dofs(prob.zero_dofs(np.float32)[0])
        s.step(10)
        wf = s.wavefield()
        e, _ = s.download_dofs()
    finally:
        s.close()
    np.testing.assert_array_equal(wf, np.transpose(e[:, :, 0, :], (2, 1, 0)))
    assert np.abs(wf).max() > 0
    path = str(tmp_path / "wf.vtk")
    vtk.write(path, prob.mesh.ve, prob.mesh.el_ve, wf)
    np.testing.assert_array_equal(vtk.read_cell_data(path)["crun_3_var_6"], wf[3, 6])
