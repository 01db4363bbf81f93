"""Shared test helpers: build small problems and run the CPU oracle the way the device path runs.

The oracle (oracle/oracle.c) only checks; the device results come from edge_b200.solver.
"""
import numpy as np

import oracle
from edge_b200 import host


def small_problem(n=2, order=4, runs=1, rm=0, jitter=0.0, seed=3343, n_steps=10, source="explosive",
                  n_receivers=4, layers=None, lognormal_sigma=0.0, bc_top=host.FACE_FREE_SURFACE,
                  bc_sides=host.FACE_OUTFLOW):
    return host.build_problem(n, order, runs, rm=rm, ext=1e4, jitter=jitter, seed=seed,
                              n_steps=n_steps, source=source, n_receivers=n_receivers, layers=layers,
                              lognormal_sigma=lognormal_sigma, bc_top=bc_top, bc_sides=bc_sides,
                              freq_cen=1.0, freq_rat=100.0, f0=2.0)


def random_dofs(prob, seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    e = rng.normal(size=(prob.n_el, 9, prob.B, prob.runs)) * scale
    a = rng.normal(size=(prob.n_el, prob.rm, 6, prob.B, prob.runs)) * scale if prob.rm else None
    return e, a


class OracleRun:
    """Runs the oracle over GTS steps with the device path's time and receiver bookkeeping."""

    def __init__(self, prob, dofsE=None, dofsA=None):
        self.prob = prob
        self.d = prob.oracle_dict()
        e, a = prob.zero_dofs()
        self.state = dict(dofsE=np.ascontiguousarray(e if dofsE is None else dofsE, np.float64),
                          dofsA=None if not prob.rm else np.ascontiguousarray(a if dofsA is None else dofsA, np.float64),
                          tDofs=np.zeros((prob.n_el, 9, prob.B, prob.runs)))
        r = prob.receivers
        self.recv = None
        if r and r.get("n", 0):
            n, mb = r["n"], r["maxbuf"]
            self.recv = dict(n=n, el=np.ascontiguousarray(r["el"]), basis=np.ascontiguousarray(r["basis"]),
                             time=np.full(n, r["t_first"]), period=r["period"], maxbuf=mb,
                             buf=np.zeros((n, mb, 9, prob.runs)), buftime=np.zeros((n, mb)),
                             count=np.zeros(n, np.int32))
        self.src = prob.sources if prob.sources and prob.sources.get("n", 0) else None
        self.t = 0.0

    def step(self, n_steps=1, dt=None):
        dt = self.prob.dt if dt is None else dt
        for _ in range(n_steps):
            oracle.step(self.d, self.state, self.t, dt, recv=self.recv, src=self.src)
            self.t += dt


def single_run(prob, r):
    """The one-run problem of fused run r (same mesh and element data, run r's sources)."""
    return prob.single_run(r)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)
