"""edge_b200_step_noalloc against the context-based step (edge_b200_step).

The allocation-free entry point serves callers that cannot allocate device memory while they run
(a host that has given the whole GPU to a fixed memory budget, or one that must not take the
device-wide synchronisation of cudaMalloc / cudaFree inside its time loop). Its scratch lives in a
static device array, so the test hands it only caller-owned device arrays and checks two calls in
a row against the existing entry point, with the tolerances of the other parity tests. This file
sorts last so that a run stopping at the first failure has run every other test first; it must
also pass on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from edge_b200._lib import Cfg, lib
from edge_b200.solver import Solver
from helpers import random_dofs, rel_l2, small_problem

pytestmark = pytest.mark.gpu

ESCRATCH = -9


def _dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a if dtype is None else a.astype(dtype)))
    return t.cuda()


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("order,runs,rm,precision,tol", [(4, 1, 0, 64, 1e-12), (4, 8, 3, 32, 1e-6),
                                                           (5, 16, 0, 32, 1e-6)])
def test_noalloc_matches_context_step(order, runs, rm, precision, tol):
    torch = pytest.importorskip("torch")
    prob = small_problem(n=2, order=order, runs=runs, rm=rm, jitter=0.1, source=None, n_receivers=0)
    dt_np = np.float64 if precision == 64 else np.float32
    e0, a0 = random_dofs(prob, seed=3)
    e0 = e0.astype(dt_np)
    a0 = None if a0 is None else a0.astype(dt_np)

    # existing entry point: 2 steps, then 2 more
    s = Solver(prob, precision=precision)
    s.upload_dofs(e0, a0)
    s.step(2)
    ref2 = s.download_dofs()
    s.step(2)
    ref4 = s.download_dofs()
    s.close()

    # caller-owned device arrays
    m = prob.mesh
    dE = _dev(torch, e0)
    dA = _dev(torch, a0) if rm else None
    star = _dev(torch, prob.starE)
    fsE = _dev(torch, prob.fsE)
    starA = _dev(torch, prob.starA) if rm else None
    srcA = _dev(torch, prob.srcA) if rm else None
    fsA = _dev(torch, prob.fsA) if rm else None
    omega = np.ascontiguousarray(prob.omega, np.float64) if rm else None
    efe = _dev(torch, m.el_fa_el)
    fid = _dev(torch, m.fid)
    vid = _dev(torch, m.vid)
    fty = _dev(torch, m.el_fa_type)
    stream = torch.cuda.current_stream()
    cfg = Cfg(order=order, n_runs=runs, n_rms=rm, precision=precision, stream=C.c_void_p(stream.cuda_stream),
              device=torch.cuda.current_device())
    args = [_p(dE), _p(dA), _p(star), _p(fsE), _p(starA), _p(srcA), _p(fsA),
            None if omega is None else C.c_void_p(omega.ctypes.data), _p(efe), _p(fid), _p(vid), _p(fty)]
    for want in (ref2, ref4):
        rc = lib().edge_b200_step_noalloc(C.byref(cfg), prob.n_el, prob.dt, 2, *args)
        assert rc == 0
        torch.cuda.synchronize()
        assert rel_l2(dE.cpu().numpy(), want[0]) < tol
        if rm:
            assert rel_l2(dA.cpu().numpy(), want[1]) < tol


def test_noalloc_rejects_problems_beyond_the_scratch():
    torch = pytest.importorskip("torch")
    # 4 * 9 * 15 * 16 * 4 bytes of face projections per element at order 5, 16 runs, FP32
    n_el = (32 << 20) // (4 * 9 * 15 * 16 * 4) + 1
    cfg = Cfg(order=5, n_runs=16, n_rms=0, precision=32, stream=None, device=torch.cuda.current_device())
    dummy = torch.zeros(8, device="cuda")
    p = C.c_void_p(dummy.data_ptr())
    rc = lib().edge_b200_step_noalloc(C.byref(cfg), n_el, 1e-3, 1, p, None, p, p, None, None, None, None,
                                      p, p, p, p)
    assert rc == ESCRATCH
