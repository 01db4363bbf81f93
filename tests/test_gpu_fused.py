"""Fused GTS steps (edge_b200_set_fused): the neighbour step of each step runs inside the next
step's local kernel (and receiver kernel); DOFs and receiver samples equal the separate-kernel
steps exactly, also across downloads, uploads and run replacements in the middle of a run."""
import numpy as np
import pytest

from edge_b200._lib import lib
from edge_b200.solver import Solver
from helpers import random_dofs, small_problem

pytestmark = pytest.mark.gpu

CASES = [(5, 16, 32), (4, 8, 32), (3, 1, 64), (4, 1, 64)]  # pre-mixing configurations


def _solver(prob, prec, e0, fused):
    s = Solver(prob, precision=prec)
    assert lib().edge_b200_set_fused(s._h, 1 if fused else 0) == 0
    s.upload_dofs(e0)
    return s


@pytest.mark.parametrize("order,runs,prec", CASES)
def test_fused_steps_equal_separate_kernels(order, runs, prec):
    prob = small_problem(n=3, order=order, runs=runs, jitter=0.15, n_steps=6, source="random",
                         layers=[3000.0, 6000.0], lognormal_sigma=0.2)
    e0, _ = random_dofs(prob, seed=3)
    a, b = _solver(prob, prec, e0, True), _solver(prob, prec, e0, False)
    for k in (1, 3, 2):  # calls of one and of several steps
        a.step(k)
        b.step(k)
    ea, _ = a.download_dofs()
    eb, _ = b.download_dofs()
    np.testing.assert_array_equal(ea, eb)
    ra, rb = a.receivers(), b.receivers()
    np.testing.assert_array_equal(ra[2], rb[2])
    k = int(ra[2][0])
    assert k > 0
    np.testing.assert_array_equal(ra[0][:, :k], rb[0][:, :k])
    a.close()
    b.close()


def test_fused_steps_around_downloads_uploads_and_run_replacement():
    prob = small_problem(n=3, order=5, runs=16, jitter=0.15, n_steps=16, source="random")
    e0, _ = random_dofs(prob, seed=5)
    e1, _ = random_dofs(prob, seed=6)
    a, b = _solver(prob, 32, e0, True), _solver(prob, 32, e0, False)
    a.step(2)
    b.step(2)
    np.testing.assert_array_equal(a.download_dofs()[0], b.download_dofs()[0])  # flush mid-run
    a.step(2)
    b.step(2)
    # a replaced run (serving): the others continue from their completed state
    run = np.ascontiguousarray(e1[..., 7], np.float32)
    for s in (a, b):
        assert lib().edge_b200_set_run_dofs(s._h, 7, run.ctypes.data, None) == 0
        s.step(2)
    np.testing.assert_array_equal(a.download_dofs()[0], b.download_dofs()[0])
    # an upload replaces the DOFs, whatever the face buffers hold (same time for both)
    a.step(1)
    a.upload_dofs(e1)
    b.upload_dofs(e1)
    a.step(2, t=0.0)
    b.step(2, t=0.0)
    np.testing.assert_array_equal(a.download_dofs()[0], b.download_dofs()[0])
    a.close()
    b.close()
