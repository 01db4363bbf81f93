"""Halo exchange on the device: the parts of a partition as separate contexts on one GPU, their
face rows moved by pack / device copy / unpack between the two halves of every step, against the
one-domain run (the device half of the multi-GPU form; the transport between GPUs is NCCL)."""
import numpy as np
import pytest

from edge_b200 import host, shard
from edge_b200.solver import Solver
from helpers import random_dofs, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_parts,precision,order,runs", [(2, 64, 4, 1), (3, 64, 3, 1), (2, 32, 5, 16)])
def test_parts_match_one_domain(n_parts, precision, order, runs):
    prob = host.build_problem(4, order, runs, jitter=0.15, seed=12, n_receivers=0, source=None)
    e0, _ = random_dofs(prob, seed=5, scale=1e-2)
    dtype = np.float64 if precision == 64 else np.float32
    ref = Solver(prob, precision=precision)
    try:
        ref.upload_dofs(e0.astype(dtype))
        ref.step(6)
        want, _ = ref.download_dofs()
    finally:
        ref.close()
    parts = [shard.PartSolver(prob, p, precision=precision) for p in shard.plan(prob.mesh, n_parts)]
    try:
        for ps in parts:
            ps.upload_owned(e0.astype(dtype))
        t = 0.0
        for _ in range(6):
            for ps in parts:
                ps.phase0(t, prob.dt)
            sent = {ps.part.rank: ps.pack() for ps in parts}
            for ps in parts:
                for q, buf in ps.recv_buf.items():
                    buf.copy_(sent[q][ps.part.rank])
                ps.unpack()
            for ps in parts:
                ps.phase1(t, prob.dt)
            t += prob.dt
        got = np.concatenate([ps.download_owned()[0] for ps in parts])
    finally:
        for ps in parts:
            ps.close()
    assert np.array_equal(got, want) or rel_l2(got, want) < 1e-14
