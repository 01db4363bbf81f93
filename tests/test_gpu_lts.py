"""Device rate-2 LTS (edge_b200_set_time_groups / edge_b200_step_lts) against the oracle's LTS."""
import numpy as np
import pytest

import oracle
from edge_b200 import host
from edge_b200.solver import Solver
from helpers import OracleRun, random_dofs, rel_l2
from test_lts import _grouped, _lts_state

pytestmark = pytest.mark.gpu


def _device_lts(prob, gf, precision, n_cycles, e0=None, dt_fun=None):
    s = Solver(prob, precision=precision)
    try:
        if e0 is not None:
            s.upload_dofs(e0.astype(s.dtype))
        s.set_time_groups(gf)
        s.step_lts(n_cycles, dt_fun=dt_fun)
        e, _ = s.download_dofs()
        buf, _, cnt = s.receivers()
    finally:
        s.close()
    return e, buf, cnt


@pytest.mark.parametrize("order", [3, 4])
def test_fp64_three_groups_match_oracle(order):
    prob, gf, flags, rel = _grouped(order=order, n=4, n_receivers=6, source="explosive", n_steps=40)
    e0, _ = random_dofs(prob, seed=7, scale=1e-2)
    ref = OracleRun(prob, e0.copy())
    st = _lts_state(prob, e0.copy())
    oracle.lts_cycles(ref.d, st, gf, 0.0, prob.dt, 3, flags, rel, ref.recv, ref.src)
    e, buf, cnt = _device_lts(prob, gf, 64, 3, e0)
    assert rel_l2(e, st["dofsE"]) < 1e-12
    assert np.array_equal(cnt, ref.recv["count"])
    assert rel_l2(buf, ref.recv["buf"]) < 1e-12


def test_fp64_one_group_equals_gts():
    prob = host.build_problem(3, 4, 1, seed=2, n_receivers=4, source="explosive", n_steps=20)
    e0, _ = random_dofs(prob, seed=3, scale=1e-2)
    e_lts, buf_lts, _ = _device_lts(prob, [0, prob.n_el], 64, 8, e0)
    s = Solver(prob, precision=64)
    try:
        s.upload_dofs(e0)
        s.step(8)
        e_gts, _ = s.download_dofs()
        buf_gts, _, _ = s.receivers()
    finally:
        s.close()
    assert rel_l2(e_lts, e_gts) < 1e-13
    assert rel_l2(buf_lts, buf_gts) < 1e-13


def test_fp64_two_group_plane_wave_matches_oracle():
    ext, P, order = 1e4, host.FACE_PERIODIC, 4
    prob = host.build_problem(4, order, 1, ext=ext, seed=5, n_receivers=0, source=None, bc_top=P, bc_sides=P)
    tg = (prob.mesh.centroids()[:, 2] > ext / 2).astype(np.uint8)
    gf = np.searchsorted(tg, [0, 1, 2]).astype(np.int64)
    flags, rel = host.lts_tables(prob.mesh, tg)
    fn = host.plane_wave_p(prob.rho[0], prob.lam[0], prob.mu[0], [2 * np.pi / ext, 0.0, 2 * np.pi / ext])
    e0 = host.project(prob.mesh, order, fn)
    ref = OracleRun(prob, e0.copy())
    st = _lts_state(prob, e0.copy())
    oracle.lts_cycles(ref.d, st, gf, 0.0, prob.dt / 2, 10, flags, rel)
    e, _, _ = _device_lts(prob, gf, 64, 10, e0, dt_fun=prob.dt / 2)
    assert rel_l2(e, st["dofsE"]) < 1e-12


def test_fp32_fused_runs_three_groups_vs_fp64_oracle():
    prob, gf, flags, rel = _grouped(order=4, n=4, runs=16, n_receivers=5, source="random", n_steps=40)
    ref = OracleRun(prob)
    st = _lts_state(prob, None)
    oracle.lts_cycles(ref.d, st, gf, 0.0, prob.dt, 4, flags, rel, ref.recv, ref.src)
    e, buf, _ = _device_lts(prob, gf, 32, 4)
    for r in range(16):
        assert rel_l2(buf[..., r], ref.recv["buf"][..., r]) < 1e-4, r
    assert rel_l2(e, st["dofsE"]) < 1e-4
