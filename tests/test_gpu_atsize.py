"""The FP32 error bar at the benchmark configurations' full sizes.

The fused FP32 path is compared run by run with the plain FP64 path (pinned to the oracle to 1e-12
by the other GPU tests) at the stated sizes and step counts:

* 663,552 tets (48^3 cubes x 6), order 5, 16 fused runs with seeded random sources and moment
  tensors, 1.5 Hz Ricker, 8 receivers, 500 steps;
* 1,296,000 tets (60^3 cubes x 6, 20% vertex jitter), three layers with a lognormal perturbation,
  Q in [50, 200], 3 relaxation mechanisms, order 4, 8 fused runs, 400 steps (40 ms of simulated
  time: each run's Ricker peaks at 20 ms, receiver i sits 150 m from run i's source).

Two measures, each with the FP32 bar of 1e-4 per run: the receiver time series (relative L2 over
all receivers, samples and quantities) from rest with the point sources, and the DOFs of every
element after 50 steps from seeded random DOFs (no sources), which reaches every element whatever
the waves' travel time.
"""
import pytest

from edge_b200 import accuracy, workloads

pytestmark = pytest.mark.gpu

TOL = 1e-4
NAMES = ["box48_o5_r16_fp32", "box60j_o4_r8_m3_fp32"]


@pytest.mark.parametrize("name", NAMES)
def test_fused_fp32_receivers_at_full_size(name):
    prob, w = workloads.build(name)
    rep = accuracy.fused_vs_plain(prob, w.steps)
    print(name, rep)
    assert rep["samples_per_receiver"] > w.steps
    assert len(rep["receiver_rel_l2_per_run"]) == w.runs
    assert rep["receiver_rel_l2_max"] < TOL, rep["receiver_rel_l2_per_run"]


@pytest.mark.parametrize("name", NAMES)
def test_fused_fp32_dofs_at_full_size(name):
    prob, w = workloads.build(name, n_receivers=0, source="none")
    rep = accuracy.dofs_fused_vs_plain(prob, 50)
    print(name, rep)
    assert len(rep["dof_rel_l2_per_run"]) == w.runs
    assert rep["dof_rel_l2_max"] < TOL, rep["dof_rel_l2_per_run"]
