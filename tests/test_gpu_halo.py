"""Halo exchange on the device: the parts of a partition as separate contexts on one GPU, their
face rows moved by pack / device copy / unpack between the two halves of every step, against the
one-domain run (the device half of the multi-GPU form; the transport between GPUs is NCCL). Every
other step runs the overlapped order: the send elements' local step, the pack, then the inner
elements' local step before the exchanged rows are unpacked."""
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
        for step in range(6):
            # odd steps: the send elements' local step, the pack, then the inner elements' local
            # step (the overlapped order); even steps: the whole local step first
            for ps in parts:
                if step % 2:
                    ps.phase_send(t, prob.dt)
                else:
                    ps.phase0(t, prob.dt)
            sent = {ps.part.rank: ps.pack() for ps in parts}
            if step % 2:
                for ps in parts:
                    ps.phase_inner(t, prob.dt)
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


def test_send_then_inner_equals_whole_local_step():
    """Phases 2 + 3 (send elements, then the rest with the sources) equal phase 0 bit for bit, with
    sources and receivers on."""
    prob = host.build_problem(3, 4, 1, jitter=0.1, seed=4, n_receivers=3, source="explosive", n_steps=8)
    e0, _ = random_dofs(prob, seed=2, scale=1e-2)
    out = []
    for split in (False, True):
        s = Solver(prob, precision=64)
        try:
            from edge_b200._lib import lib
            s._chk(lib().edge_b200_set_owned(s._h, prob.n_el), "set_owned")
            s._chk(lib().edge_b200_set_send_count(s._h, prob.n_el // 3), "set_send_count")
            s.upload_dofs(e0)
            t = 0.0
            for _ in range(4):
                if split:
                    s._chk(lib().edge_b200_step_phase(s._h, t, prob.dt, 2), "phase 2")
                    s._chk(lib().edge_b200_step_phase(s._h, t, prob.dt, 3), "phase 3")
                else:
                    s._chk(lib().edge_b200_step_phase(s._h, t, prob.dt, 0), "phase 0")
                s._chk(lib().edge_b200_step_phase(s._h, t, prob.dt, 1), "phase 1")
                t += prob.dt
            e, _ = s.download_dofs()
            rb, rt, rc = s.receivers()
            out.append((e, rb, rc))
        finally:
            s.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][2], out[1][2]) and int(out[0][2][0]) > 0
    assert np.array_equal(out[0][1], out[1][1])
