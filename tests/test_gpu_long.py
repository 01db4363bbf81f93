"""Long runs on the GPU.

* The plain-method configuration: 10 km box, 12^3 cubes x 6 = 10,368 tets,
  order 4, FP64, one run, free surface on top and outflow elsewhere, explosive source at the centre
  (2 Hz Ricker), 8 seeded receivers, 200 steps at CFL 0.5: DOFs and receivers within rel-L2 1e-12 of
  the oracle.
* Fused-run precision: the FP32 16-run path against the FP64 path run by run (each FP64 run checked
  against the oracle elsewhere), receivers within rel-L2 1e-4 after 200 steps at order 5.
"""
import numpy as np
import pytest

from edge_b200 import host
from edge_b200.solver import Solver
from helpers import OracleRun, rel_l2, single_run

pytestmark = pytest.mark.gpu


def test_plain_fp64_box12_200_steps_matches_oracle():
    prob = host.build_problem(12, 4, 1, rm=0, ext=1e4, seed=3343, source="explosive", f0=2.0,
                              n_receivers=8, n_steps=200, name="box12_o4_r1_fp64")
    assert prob.n_el == 10368
    s = Solver(prob, precision=64)
    e0, _ = prob.zero_dofs()
    s.upload_dofs(e0)
    s.step(200)
    e, _ = s.download_dofs()
    orc = OracleRun(prob)
    orc.step(200)
    assert np.abs(orc.state["dofsE"]).max() > 0
    assert rel_l2(e, orc.state["dofsE"]) < 1e-12
    buf, bt, cnt = s.receivers()
    k = int(cnt[0])
    assert k == int(orc.recv["count"][0]) and k > 400
    np.testing.assert_array_equal(bt[:, :k], orc.recv["buftime"][:, :k])
    assert rel_l2(buf[:, :k], orc.recv["buf"][:, :k]) < 1e-12
    for i in range(prob.receivers["n"]):
        assert rel_l2(buf[i, :k], orc.recv["buf"][i, :k]) < 1e-12


def test_fused_fp32_receivers_vs_plain_fp64_per_run():
    prob = host.build_problem(8, 5, 16, rm=0, ext=1e4, seed=7, source="random", f0=1.5, n_receivers=8,
                              n_steps=200, name="box8_o5_r16")
    s32 = Solver(prob, precision=32)
    e0, _ = prob.zero_dofs(np.float32)
    s32.upload_dofs(e0)
    s32.step(200)
    b32, _, c32 = s32.receivers()
    k = int(c32[0])
    errs = []
    for r in range(16):
        p1 = single_run(prob, r)
        s64 = Solver(p1, precision=64)
        z, _ = p1.zero_dofs()
        s64.upload_dofs(z)
        s64.step(200)
        b64, _, c64 = s64.receivers()
        assert int(c64[0]) == k
        errs.append(rel_l2(b32[:, :k, :, r], b64[:, :k, :, 0]))
        s64.close()
    assert max(errs) < 1e-4, errs
