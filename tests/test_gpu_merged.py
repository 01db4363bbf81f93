"""Simulations of one configuration family merged into one context (edge_b200.merged): different
meshes, time steps, point sources and step counts stepped by one persistent launch per kernel and
step, each simulation ending where it ends when stepped alone on a context of its own."""
import numpy as np
import pytest

from edge_b200.merged import MergedFamily
from edge_b200.solver import Solver
from helpers import random_dofs, rel_l2, small_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order,runs,rm,prec,tol", [(4, 8, 0, 32, 1e-6), (5, 16, 0, 32, 1e-6), (4, 8, 3, 32, 1e-6),
                                                    (3, 1, 0, 64, 1e-12)])
def test_merged_family_matches_each_simulation_alone(order, runs, rm, prec, tol):
    specs = [(2, 0.1, 5), (3, 0.15, 9), (2, 0.0, 2), (3, 0.2, 7)]  # (cubes, jitter, steps)
    probs, dofs, steps = [], [], []
    for i, (n, jit, k) in enumerate(specs):
        p = small_problem(n=n, order=order, runs=runs, rm=rm, jitter=jit, seed=21 + i, n_steps=12,
                          source="random", n_receivers=0, layers=[3000.0, 6000.0] if i % 2 else None)
        probs.append(p)
        dofs.append(random_dofs(p, seed=40 + i, scale=1e-2))
        steps.append(k)
    assert len({p.dt for p in probs}) == len(probs)  # every simulation its own time step
    dt = np.float32 if prec == 32 else np.float64
    fam = MergedFamily(probs, steps, dofs=[(e.astype(dt), None if a is None else a.astype(dt)) for e, a in dofs],
                       precision=prec)
    try:
        launches = fam.launch()
        assert launches > 0
        got = [fam.result(i) for i in range(len(probs))]
    finally:
        fam.close()
    for i, (p, (e0, a0), k) in enumerate(zip(probs, dofs, steps)):
        s = Solver(p, precision=prec)
        try:
            s.upload_dofs(e0.astype(dt), None if a0 is None else a0.astype(dt))
            s.step(k)
            e, a = s.download_dofs()
        finally:
            s.close()
        assert rel_l2(got[i][0], e) < tol, i
        if rm:
            assert rel_l2(got[i][1], a) < tol, i
