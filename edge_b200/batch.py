"""Uneven batches of simulations stepped together (the batching form of the element update: many
simulations over different meshes, orders, fused-run counts and physics on one GPU).

Each simulation keeps its own context (``Solver``); ``Batch`` hands the contexts to
``edge_b200_batch_create``, which captures two batch steps (every active context's kernels, each
context on a stream of its own; fused steps where the context's own steps are fused) into a CUDA
graph and replays it. Simulations of different lengths drop out as they finish: ``schedule`` splits a run into
segments with a fixed active set (the graph is captured again at each change). Optionally each
context's launch shape is autotuned first (``edge_b200_autotune``).

EDGE runs one solver per process (``src/main.cpp``); there is no reference counterpart for the
batch itself, whose every simulation still computes the reference's GTS step.
"""
import ctypes as C

import numpy as np

from ._lib import lib, ptr


def schedule(n_steps):
    """Segments (active mask, steps) that take simulation k through n_steps[k] steps, each segment
    ending when the next simulation finishes."""
    rem = np.asarray(n_steps, np.int64).copy()
    if np.any(rem < 0):
        raise ValueError("negative step count")
    out = []
    while rem.max(initial=0) > 0:
        active = rem > 0
        k = int(rem[active].min())
        out.append((active.copy(), k))
        rem[active] -= k
    return out


class Batch:
    def __init__(self, solvers, autotune=False):
        self.solvers = list(solvers)
        n = len(self.solvers)
        if n < 1:
            raise ValueError("empty batch")
        self.caps = []
        if autotune:
            for s in self.solvers:
                caps = np.zeros(2, np.int32)
                s._chk(lib().edge_b200_autotune(s._h, s.prob.dt, ptr(caps)), "autotune")
                self.caps.append(tuple(int(c) for c in caps))
        handles = (C.c_void_p * n)(*[s._h.value for s in self.solvers])
        self._t0 = np.array([s.t for s in self.solvers], np.float64)
        self._dt = np.array([s.prob.dt for s in self.solvers], np.float64)
        h = C.c_void_p()
        rc = lib().edge_b200_batch_create(handles, n, ptr(self._t0), ptr(self._dt), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"edge_b200_batch_create failed ({rc})")
        self._h = h

    def _chk(self, rc, what):
        if rc != 0:
            msg = lib().edge_b200_batch_last_error(self._h)
            raise RuntimeError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def run(self, n_steps, sync=True):
        """Advances simulation k by n_steps[k] steps (an int: all by that many)."""
        if np.isscalar(n_steps):
            n_steps = [int(n_steps)] * len(self.solvers)
        segments = schedule(n_steps)
        for active, k in segments:
            a = active.astype(np.int32)
            self._chk(lib().edge_b200_batch_set_active(self._h, ptr(a)), "batch_set_active")
            self._chk(lib().edge_b200_batch_step(self._h, k), "batch_step")
        if sync:
            self.sync()
        for s, m in zip(self.solvers, n_steps):
            s.t = s.t + m * s.prob.dt
        return segments

    def sync(self):
        steps = np.zeros(len(self.solvers), np.int64)
        self._chk(lib().edge_b200_batch_sync(self._h, ptr(steps)), "batch_sync")
        return steps

    def close(self):
        if getattr(self, "_h", None):
            lib().edge_b200_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
