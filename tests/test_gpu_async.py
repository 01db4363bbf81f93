"""Asynchronous DOF transfers (edge_b200_upload_dofs_async / download_dofs_async): a pipeline of
upload, step, download per step gives the same results as the synchronous forms."""
import ctypes as C

import numpy as np
import pytest
import torch

from edge_b200 import _lib
from edge_b200.solver import Solver
from helpers import random_dofs, small_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,runs,rm", [(64, 1, 0), (32, 16, 0), (32, 8, 3)])
def test_pipelined_transfers_match_synchronous(precision, runs, rm):
    prob = small_problem(n=3, order=4, runs=runs, rm=rm, jitter=0.1, n_steps=4, source="random")
    dtype = np.float64 if precision == 64 else np.float32
    inputs = [tuple(None if x is None else x.astype(dtype) for x in random_dofs(prob, seed=s, scale=1e-2))
              for s in range(3)]
    L = _lib.lib()
    # synchronous reference: each input stepped once
    want = []
    s = Solver(prob, precision=precision)
    try:
        for e, a in inputs:
            s.upload_dofs(e, a)
            s.step(1, t=0.0)
            want.append(s.download_dofs())
    finally:
        s.close()
    pins = [tuple(None if x is None else torch.from_numpy(x).pin_memory() for x in inp) for inp in inputs]
    outs = [tuple(None if x is None else torch.empty_like(x).pin_memory() for x in p) for p in pins]
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    s = Solver(prob, precision=precision)
    try:
        for (pe, pa), (oe, oa) in zip(pins, outs):
            assert L.edge_b200_upload_dofs_async(s._h, ptr(pe), ptr(pa)) == 0
            s.step(1, t=0.0)
            assert L.edge_b200_download_dofs_async(s._h, ptr(oe), ptr(oa)) == 0
        assert L.edge_b200_join_transfers(s._h, 0) == 0
        s.sync()
    finally:
        s.close()
    for (we, wa), (oe, oa) in zip(want, outs):
        np.testing.assert_array_equal(oe.numpy(), we)
        if wa is not None:
            np.testing.assert_array_equal(oa.numpy(), wa)
