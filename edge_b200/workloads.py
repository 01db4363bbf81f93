"""Named synthetic setups of the element update, shared by the bench and the at-size tests.

Each entry restates one benchmark configuration of the path with its sizes (synthetic inputs: there
is no dataset behind them):

* ``box12_o4_r1_fp64`` -- plain method: 10 km box of 12^3 cubes x 6 = 10,368 tets, order 4, FP64,
  one run, explosive source at the centre (2 Hz Ricker), 8 receivers, 200 steps.
* ``box48_o5_r16_fp32`` -- fused-run precision: 48^3 cubes x 6 = 663,552 tets, order 5, 16 fused
  FP32 runs, each with a seeded uniform interior source and a N(0,1) x 1e15 moment tensor (1.5 Hz
  Ricker), 8 receivers, 500 steps.
* ``box60j_o4_r8_m3_fp32`` -- viscoelastic, unstructured: 60^3 cubes x 6 = 1,296,000 tets with
  interior vertices jittered by 20% of the edge length, three horizontal layers (vp 4000 / 5500 /
  6500 m/s from the top, vs = vp / sqrt(3), rho 2670 kg/m^3), a seeded lognormal factor (sigma
  0.1) per element, Qp and Qs uniform in [50, 200], 3 relaxation mechanisms (central frequency
  1 Hz, frequency ratio 100), order 4, 8 fused FP32 runs, 400 steps. The jitter leaves slivers
  (smallest in-diameter 12 m), so the CFL step is 0.1 ms and 400 steps cover about 40 ms: each run's
  Ricker peaks at half that window (f0 = 1.2 / peak time, about 60 Hz) and receiver i sits 150 m
  from run i's source, so that the receivers record signal within the run.
* ``box16_o5_r16_fp32`` / ``box20j_o4_r8_m3_fp32`` -- small cases of the two FP32 kernels
  (24,576 and 48,000 tets; DOFs above the 126 MB L2) for profiler captures.
"""
from dataclasses import dataclass

from . import host


@dataclass(frozen=True)
class Workload:
    cubes: int
    order: int
    runs: int
    rm: int
    precision: int
    source: str
    f0: float
    steps: int
    jitter: float = 0.0
    layered: bool = False
    f0_window: float = 0.0
    receivers_near: float = 0.0


WORKLOADS = {
    "box48_o5_r16_fp32": Workload(48, 5, 16, 0, 32, "random", 1.5, 500),
    "box12_o4_r1_fp64": Workload(12, 4, 1, 0, 64, "explosive", 2.0, 200),
    "box60j_o4_r8_m3_fp32": Workload(60, 4, 8, 3, 32, "random", 2.0, 400, jitter=0.2, layered=True,
                                     f0_window=0.5, receivers_near=150.0),
    "box16_o5_r16_fp32": Workload(16, 5, 16, 0, 32, "random", 1.5, 500),
    "box20j_o4_r8_m3_fp32": Workload(20, 4, 8, 3, 32, "random", 2.0, 400, jitter=0.2, layered=True,
                                     f0_window=0.5, receivers_near=150.0),
}


def build(name, n_receivers=8, seed=3343, source=None):
    """The Problem of a named workload (receiver buffers sized for its stated number of steps);
    source="none" drops the point sources."""
    w = WORKLOADS[name]
    kw = dict(f0_window=w.f0_window or None, receivers_near=w.receivers_near or None)
    if w.layered:
        kw.update(jitter=w.jitter, layers=[4000.0, 5500.0, 6500.0], lognormal_sigma=0.1)
    if w.rm:
        kw.update(q_range=(50.0, 200.0), freq_cen=1.0, freq_rat=100.0)
    src = None if source == "none" else (source or w.source)
    prob = host.build_problem(w.cubes, w.order, w.runs, rm=w.rm, ext=1e4, seed=seed, source=src, f0=w.f0,
                              n_receivers=n_receivers, n_steps=w.steps, name=name, **kw)
    return prob, w
