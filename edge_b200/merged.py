"""Simulations of one configuration family merged into one context: one persistent launch per kernel
and step for all of them (the uneven-batch form without a launch per simulation).

A family is the simulations with the same order, fused runs, relaxation mechanisms, precision and
relaxation frequencies; their meshes may differ in size and shape, and so may their time steps,
sources and step counts. ``MergedFamily`` places the meshes side by side as disjoint element
ranges, each padded to a multiple of the 32 / runs elements of a kernel group (padding elements
have no faces, no element data and stay zero), gives every element group its simulation's time step
(edge_b200_set_group_dt) and every point source its simulation's clock
(edge_b200_set_source_clocks), and orders the simulations by decreasing step count: those still
running are then always a prefix of the elements, and a simulation that has finished is dropped by
lowering the stepped range (edge_b200_set_active_elements). Each simulation computes exactly the
steps it would compute alone (every element group holds elements of one simulation only).

EDGE runs one solver per process; there is no reference counterpart for the merging itself.
"""
import types

import numpy as np

from . import host
from ._lib import lib, ptr
from .solver import Solver


def family_key(prob, precision):
    om = tuple(np.round(np.asarray(prob.omega), 12)) if prob.rm else ()
    return (prob.order, prob.runs, prob.rm, precision, om)


def merge(probs, steps):
    """The merged problem of a family (no device work): returns (Problem, info) with info holding
    the simulation order `perm` (most steps first), their `steps`, element `offsets` (each range
    padded to a multiple of the 32 / runs elements of a kernel group), `sizes`, the per-group time
    steps `group_dt` and the per-source clocks `clk0`, `clk_dt` (None without sources)."""
    if not probs:
        raise ValueError("empty family")
    if len({family_key(p, 0) for p in probs}) != 1:
        raise ValueError("simulations of different configurations cannot be merged")
    if any(p.receivers and p.receivers.get("n", 0) for p in probs):
        raise ValueError("merged simulations take no receivers")
    order, runs, rm = probs[0].order, probs[0].runs, probs[0].rm
    E = 32 // runs
    perm = sorted(range(len(probs)), key=lambda i: -int(steps[i]))
    ps = [probs[i] for i in perm]
    sizes = [p.n_el for p in ps]
    padded = [(n + E - 1) // E * E for n in sizes]
    offsets = np.concatenate([[0], np.cumsum(padded)]).astype(np.int64)
    n_el = int(offsets[-1])

    def cat(get, fill, tail, dtype, axis=0):
        parts = []
        for p, n, pad in zip(ps, sizes, padded):
            a = np.asarray(get(p), dtype)
            parts.append(a)
            if pad > n:
                shape = (pad - n,) + tail if axis == 0 else (a.shape[0], pad - n) + tail
                parts.append(np.full(shape, fill, dtype))
        return np.ascontiguousarray(np.concatenate(parts, axis=axis))

    ef = []
    for p, off, n, pad in zip(ps, offsets[:-1], sizes, padded):
        a = np.asarray(p.mesh.el_fa_el, np.int64)
        ef.append(np.where(a >= 0, a + off, -1))
        if pad > n:
            ef.append(np.full((pad - n, 4), -1, np.int64))
    mesh = types.SimpleNamespace(
        n_el=n_el, el_fa_el=np.ascontiguousarray(np.concatenate(ef).astype(np.int32)),
        fid=cat(lambda p: p.mesh.fid, 0, (4,), np.uint8), vid=cat(lambda p: p.mesh.vid, 0, (4,), np.uint8),
        el_fa_type=cat(lambda p: p.mesh.el_fa_type, host.FACE_OUTFLOW, (4,), np.uint8))
    starE = cat(lambda p: p.starE, 0.0, (3, 24), np.float64)
    fsE = cat(lambda p: p.fsE, 0.0, (4, 81), np.float64, axis=1)
    starA = srcA = fsA = None
    if rm:
        starA = cat(lambda p: p.starA, 0.0, (3, 9), np.float64)
        srcA = cat(lambda p: p.srcA, 0.0, (rm, 12), np.float64)
        fsA = cat(lambda p: p.fsA, 0.0, (4, 54), np.float64, axis=1)
    # sources with element offsets; each keeps its simulation's clock
    keep = {k: [] for k in ("el", "run", "scal", "bEval", "t0", "dt", "tsOff", "nPts", "ts")}
    clk0, clk_dt, ts_len = [], [], 0
    for p, off in zip(ps, offsets[:-1]):
        sr = p.sources
        if not sr or not sr.get("n", 0):
            continue
        keep["el"].append(np.asarray(sr["el"], np.int64) + off)
        for k in ("run", "scal", "bEval", "t0", "dt", "nPts"):
            keep[k].append(np.asarray(sr[k]))
        keep["tsOff"].append(np.asarray(sr["tsOff"], np.int64) + ts_len)
        keep["ts"].append(np.asarray(sr["ts"], np.float64))
        ts_len += len(sr["ts"])
        clk0.append(np.zeros(sr["n"]))
        clk_dt.append(np.full(sr["n"], p.dt))
    src = {}
    if keep["el"]:
        src = {k: np.ascontiguousarray(np.concatenate(v)) for k, v in keep.items()}
        src["n"] = len(src["el"])
        src["run"] = src["run"].astype(np.int32)
        clk0, clk_dt = np.ascontiguousarray(np.concatenate(clk0)), np.ascontiguousarray(np.concatenate(clk_dt))
    else:
        clk0 = clk_dt = None
    group_dt = np.ascontiguousarray(np.concatenate([np.full(pad // E, p.dt) for p, pad in zip(ps, padded)]))
    prob = host.Problem(order=order, runs=runs, rm=rm, mesh=mesh, rho=None, lam=None, mu=None, starE=starE, fsE=fsE,
                        dt=float(ps[0].dt), starA=starA, srcA=srcA, fsA=fsA, omega=ps[0].omega, sources=src,
                        receivers={}, name="merged")
    info = dict(perm=perm, steps=[int(steps[i]) for i in perm], offsets=offsets, sizes=sizes, group_dt=group_dt,
                clk0=clk0, clk_dt=clk_dt)
    return prob, info


class MergedFamily:
    def __init__(self, probs, steps, dofs=None, precision=32, device=0, stream=None):
        prob, info = merge(probs, steps)
        self.probs = [probs[i] for i in info["perm"]]
        self.perm, self.steps, self.offsets, self.sizes = info["perm"], info["steps"], info["offsets"], info["sizes"]
        self.order, self.runs, self.rm, self.n_el = prob.order, prob.runs, prob.rm, prob.n_el
        self.precision = precision
        self.solver = Solver(prob, precision=precision, device=device, stream=stream)
        s = self.solver
        self._keep = (info["group_dt"], info["clk0"], info["clk_dt"])
        s._chk(lib().edge_b200_set_group_dt(s._h, ptr(info["group_dt"])), "set_group_dt")
        if info["clk0"] is not None:
            s._chk(lib().edge_b200_set_source_clocks(s._h, ptr(info["clk0"]), ptr(info["clk_dt"])),
                   "set_source_clocks")
        if dofs is not None:
            self.upload([dofs[i] for i in self.perm])

    def upload(self, dofs):
        """Initial DOFs of the simulations in this family's order: [(dofsE, dofsA)]."""
        p0 = self.probs[0]
        dt = np.float32 if self.precision == 32 else np.float64
        e = np.zeros((self.n_el, 9, p0.B, self.runs), dt)
        a = np.zeros((self.n_el, self.rm, 6, p0.B, self.runs), dt) if self.rm else None
        for (de, da), off, n in zip(dofs, self.offsets[:-1], self.sizes):
            e[off:off + n] = de
            if self.rm:
                a[off:off + n] = da
        self.solver.upload_dofs(e, a)

    def launch(self):
        """Queues every simulation's steps on the context's stream (asynchronous): segments of
        fused multi-step calls, each ending where the next simulation finishes."""
        L, s = lib(), self.solver
        done, n_active = 0, len(self.steps)
        launches = 0
        while n_active > 0:
            k = self.steps[n_active - 1] - done
            if k > 0:
                s.step(k, t=0.0)
                launches += s.launches()
                done += k
            while n_active > 0 and self.steps[n_active - 1] <= done:
                n_active -= 1
            s._chk(L.edge_b200_set_active_elements(s._h, int(self.offsets[n_active])), "set_active_elements")
        self.kernel_launches = launches
        return launches

    def result(self, i):
        """(dofsE, dofsA) of simulation i (in the order given to the constructor)."""
        j = self.perm.index(i)
        e, a = self.solver.download_dofs()
        off, n = int(self.offsets[j]), self.sizes[j]
        return e[off:off + n], (a[off:off + n] if a is not None else None)

    def close(self):
        self.solver.close()
