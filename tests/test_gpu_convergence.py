"""Convergence order of the plain FP64 path on a plane wave (periodic unit box).

A P plane wave sin(k.x - w t) with k = 2 pi (1, 1, 1) is L2-projected (InitialDofs::dg,
src/setups/InitialDofs.hpp:172-250), advanced to a fixed time on meshes of 2, 4, 8 (and 16) cubes
per direction, and compared with the exact solution in L2 (InitialDofs::err, :277-373). ADER-DG of
order O converges with order O; the observed rate between the two finest meshes must be at least
O - 0.5.
"""
import math

import numpy as np
import pytest

from edge_b200 import host
from edge_b200.solver import Solver

pytestmark = pytest.mark.gpu

RHO, VP, VS = 1.0, 1.0, 0.5
MU = RHO * VS * VS
LAM = RHO * VP * VP - 2 * MU
T_END = 0.25


def _run(order, n):
    mesh = host.Mesh.box(n, (1.0, 1.0, 1.0), bc_top=host.FACE_PERIODIC, bc_sides=host.FACE_PERIODIC)
    ne = mesh.n_el
    rho, lam, mu = np.full(ne, RHO), np.full(ne, LAM), np.full(ne, MU)
    star = host.star(mesh, rho, lam, mu)
    fsE, _ = host.flux_solvers(mesh, rho, lam, mu)
    dt_cfl = host.dt_cfl(mesh, order, rho, lam, mu)
    steps = math.ceil(T_END / dt_cfl)
    dt = T_END / steps
    prob = host.Problem(order=order, runs=1, rm=0, mesh=mesh, rho=rho, lam=lam, mu=mu, starE=star,
                        fsE=fsE, dt=dt, name=f"plane_wave_o{order}_n{n}")
    wave = host.plane_wave_p(RHO, LAM, MU, 2 * np.pi * np.array([1.0, 1.0, 1.0]))
    d0 = host.project(mesh, order, wave)
    s = Solver(prob, precision=64)
    s.upload_dofs(d0)
    s.step(steps)
    d, _ = s.download_dofs()
    err, ref = host.l2_error(mesh, order, d, lambda x: wave(x, T_END))
    return float(np.linalg.norm(err) / np.linalg.norm(ref))


@pytest.mark.parametrize("order,meshes", [(2, (4, 8, 16)), (3, (4, 8, 16)), (4, (2, 4, 8)), (5, (2, 4, 8))])
def test_plane_wave_convergence_order(order, meshes):
    errs = [_run(order, n) for n in meshes]
    rates = [math.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]
    print(f"order {order}: errors {errs} rates {rates}")
    assert errs[-1] < errs[0]
    assert rates[-1] >= order - 0.5, (errs, rates)
