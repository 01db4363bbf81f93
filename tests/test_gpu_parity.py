"""CUDA path (through the C ABI) against the CPU oracle.

Tolerances: the plain FP64 path must match to relative L2 <= 1e-12 on DOFs, time-integrated DOFs
and receivers; the FP32 fused-run path to <= 1e-4 against the FP64 oracle.
"""
import numpy as np
import pytest

from edge_b200 import host
from edge_b200.solver import Solver
from helpers import OracleRun, random_dofs, rel_l2, small_problem

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-4


def _run_both(prob, precision, n_steps, dofs_seed=1, scale=1.0):
    e0, a0 = random_dofs(prob, seed=dofs_seed, scale=scale)
    orc = OracleRun(prob, e0, a0)
    s = Solver(prob, precision=precision)
    s.keep_tdofs(True)
    s.upload_dofs(e0, a0)
    s.step(n_steps)
    orc.step(n_steps)
    e, a = s.download_dofs()
    t = s.download_tdofs()
    rb, rt, rc = s.receivers()
    return s, orc, e, a, t, (rb, rt, rc)


@pytest.mark.parametrize("order", [2, 3, 4, 5, 6])
def test_fp64_matches_oracle(order):
    prob = small_problem(n=2, order=order, runs=1, jitter=0.15, n_steps=4)
    s, orc, e, a, t, (rb, rt, rc) = _run_both(prob, 64, 4)
    assert s.launches() >= 3 * 4
    assert rel_l2(e, orc.state["dofsE"]) < TOL64
    assert rel_l2(t, orc.state["tDofs"]) < TOL64
    r = orc.recv
    assert np.array_equal(rc, r["count"])
    k = int(rc[0])
    assert k > 0
    np.testing.assert_array_equal(rt[:, :k], r["buftime"][:, :k])
    assert rel_l2(rb[:, :k], r["buf"][:, :k]) < TOL64


@pytest.mark.parametrize("order", [3, 4])
def test_fp64_viscoelastic_matches_oracle(order):
    prob = small_problem(n=2, order=order, runs=1, rm=3, jitter=0.15, n_steps=3)
    s, orc, e, a, t, (rb, rt, rc) = _run_both(prob, 64, 3)
    assert rel_l2(e, orc.state["dofsE"]) < TOL64
    assert rel_l2(a, orc.state["dofsA"]) < TOL64
    k = int(rc[0])
    assert rel_l2(rb[:, :k], orc.recv["buf"][:, :k]) < TOL64


def test_fp64_sources_from_rest():
    """Zero initial state: the wavefield comes from the point source alone."""
    prob = small_problem(n=3, order=4, runs=1, n_steps=12)
    orc = OracleRun(prob)
    s = Solver(prob, precision=64)
    e0, a0 = prob.zero_dofs()
    s.upload_dofs(e0)
    s.step(12)
    orc.step(12)
    e, _ = s.download_dofs()
    assert np.abs(orc.state["dofsE"]).max() > 0
    assert rel_l2(e, orc.state["dofsE"]) < TOL64
    rb, rt, rc = s.receivers()
    k = int(rc[0])
    assert rel_l2(rb[:, :k], orc.recv["buf"][:, :k]) < TOL64


def test_fp64_all_boundary_types():
    """Free surface on every side, then outflow everywhere."""
    for top, sides in ((host.FACE_FREE_SURFACE, host.FACE_FREE_SURFACE), (host.FACE_OUTFLOW, host.FACE_OUTFLOW)):
        prob = small_problem(n=2, order=3, runs=1, jitter=0.1, n_steps=3, bc_top=top, bc_sides=sides)
        s, orc, e, a, t, _ = _run_both(prob, 64, 3)
        assert rel_l2(e, orc.state["dofsE"]) < TOL64


@pytest.mark.parametrize("order,runs,rm", [(3, 16, 0), (4, 16, 0), (5, 16, 0), (6, 16, 0), (4, 8, 3),
                                           (3, 1, 0), (4, 1, 0), (5, 1, 0),
                                           (3, 4, 0), (4, 4, 0), (5, 4, 0), (6, 4, 0),
                                           (3, 8, 0), (4, 8, 0), (5, 8, 0), (6, 8, 0), (3, 8, 3), (5, 8, 3),
                                           (6, 1, 0), (3, 1, 3), (3, 4, 3), (3, 16, 3), (4, 1, 3), (4, 4, 3),
                                           (4, 16, 3), (5, 1, 3), (5, 4, 3), (5, 16, 3), (6, 1, 3), (6, 4, 3),
                                           (6, 8, 3), (6, 16, 3)])
def test_fp32_fused_runs_vs_fp64_oracle(order, runs, rm):
    prob = small_problem(n=2, order=order, runs=runs, rm=rm, jitter=0.15, n_steps=3, source="random")
    s, orc, e, a, t, (rb, rt, rc) = _run_both(prob, 32, 3)
    assert rel_l2(e, orc.state["dofsE"]) < TOL32
    if rm:
        assert rel_l2(a, orc.state["dofsA"]) < TOL32
    k = int(rc[0])
    for r in range(runs):
        assert rel_l2(rb[:, :k, :, r], orc.recv["buf"][:, :k, :, r]) < TOL32


def test_runs_are_independent():
    """Fused run r of a 16-run context equals a 1-run context fed run r's data (FP32)."""
    prob16 = small_problem(n=2, order=4, runs=16, jitter=0.1, n_steps=2, source=None, n_receivers=0)
    prob1 = small_problem(n=2, order=4, runs=1, jitter=0.1, n_steps=2, source=None, n_receivers=0)
    e0, _ = random_dofs(prob16, seed=5)
    s16 = Solver(prob16, precision=32)
    s16.upload_dofs(e0)
    s16.step(2)
    e16, _ = s16.download_dofs()
    s1 = Solver(prob1, precision=32)
    for r in (0, 7, 15):
        s1.upload_dofs(e0[..., r:r + 1])
        s1.step(2, t=0.0)
        e1, _ = s1.download_dofs()
        assert rel_l2(e16[..., r:r + 1], e1) < 1e-6


@pytest.mark.parametrize("order,runs", [(4, 16), (5, 16)])
def test_fp32_heterogeneous_premixed_faces(order, runs):
    """Layered, log-normally perturbed materials: the face projections the local kernel pre-mixes
    with the reading element's flux solver differ from ones mixed with the element's own."""
    prob = small_problem(n=3, order=order, runs=runs, jitter=0.15, n_steps=3, source="random",
                         layers=[3000.0, 6000.0], lognormal_sigma=0.2)
    s, orc, e, a, t, (rb, rt, rc) = _run_both(prob, 32, 3)
    assert rel_l2(e, orc.state["dofsE"]) < TOL32
    k = int(rc[0])
    assert rel_l2(rb[:, :k], orc.recv["buf"][:, :k]) < TOL32


def test_kernel_config_reports_premix():
    # info[1]: 2 where GTS projections leave as characteristic rows, 0 where the neighbour kernel mixes
    from edge_b200._lib import lib, ptr
    cases = [((32, 5, 16, 0), (2, 2, 84)), ((32, 4, 16, 0), (2, 2, 84)), ((32, 5, 8, 0), (4, 2, 84)), ((32, 5, 4, 0), (8, 0, 84)),
             ((64, 5, 1, 0), (32, 0, 82)), ((64, 4, 1, 0), (32, 2, 82)), ((32, 4, 8, 3), (4, 0, 84))]
    for (prec, order, runs, rm), want in cases:
        prob = small_problem(n=2, order=order, runs=runs, rm=rm, n_steps=1, source=None, n_receivers=0)
        s = Solver(prob, precision=prec)
        info = np.zeros(6, np.int32)
        assert lib().edge_b200_kernel_config(s._h, ptr(info)) == 0
        assert tuple(int(x) for x in info[:3]) == want, (prec, order, runs, rm, info)
        assert info[3] >= 148 and info[4] >= 148
        assert info[5] == (info[1] > 0)  # multi-step calls fuse the neighbour step where projections are pre-mixed
        s.close()


def _per_range(a, b, chunks=4):
    n = len(b)
    return [rel_l2(a[n * i // chunks:n * (i + 1) // chunks], b[n * i // chunks:n * (i + 1) // chunks])
            for i in range(chunks)]


@pytest.mark.parametrize("n,order,runs,rm,prec", [(12, 4, 8, 3, 32), (12, 4, 1, 3, 64), (12, 3, 8, 3, 32),
                                                  (10, 5, 16, 0, 32), (12, 4, 16, 0, 32)])
def test_medium_mesh_vs_oracle(n, order, runs, rm, prec):
    """Meshes with many element groups per persistent CTA (10,368 and 6,000 tets; the small cases
    above have one group per CTA), so the kernels' one-group-ahead prefetches all take part:
    jittered layered materials, random DOFs, 4 steps; every quarter of the element range within the
    tolerance, and two runs of the device path bit-identical."""
    prob = small_problem(n=n, order=order, runs=runs, rm=rm, jitter=0.2, n_steps=8, source="random",
                         layers=[4000.0, 5500.0, 6500.0], lognormal_sigma=0.1)
    tol = TOL64 if prec == 64 else TOL32
    s, orc, e, a, t, (rb, rt, rc) = _run_both(prob, prec, 4)
    errs = _per_range(e, orc.state["dofsE"])
    if rm:
        errs += _per_range(a, orc.state["dofsA"])
    assert max(errs) < tol, errs
    e0, a0 = random_dofs(prob, seed=1)
    s.upload_dofs(e0, a0)
    s.step(4, t=0.0)
    e2, a2 = s.download_dofs()
    assert np.array_equal(e, e2)
    if rm:
        assert np.array_equal(a, a2)
