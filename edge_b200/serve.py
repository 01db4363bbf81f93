"""Continuous batching of simulation requests over fused-run slots (the serving form).

A *pool* is one device context (one mesh, order, material) with R fused-run slots and its own CUDA
stream. A request (its own point source, receivers and number of steps) occupies one slot of a
pool of its mesh and order; requests that arrive while others run are admitted as soon as a slot
is free, so the runs of one pool start and end at different times: the pool steps all slots in
lockstep (the fused-run kernels), a slot's DOFs are reset when it is handed to a new request
(edge_b200_set_run_dofs), the sources of a request are time-shifted to its admission time, and
its receivers are read back every chunk of steps. Pools of different meshes or orders run
concurrently on their own streams. New pools are admitted against an HBM budget; idle pools are
closed to free memory. Latency is arrival -> last sample read back.
"""
import math
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import host
from ._lib import lib, ptr
from .solver import Solver


@dataclass
class MeshSpec:
    """A synthetic mesh and homogeneous material the requests refer to by key."""
    n_cubes: int
    ext: float = 1e4
    jitter: float = 0.0
    seed: int = 0
    vp: float = 6000.0
    vs: float = 3464.0
    rho: float = 2670.0


@dataclass
class Request:
    rid: int
    arrival: float                 # seconds after the start of the stream
    mesh: str                      # key into the mesh specs
    order: int
    n_steps: int
    src_pos: np.ndarray            # [3]
    moment: np.ndarray             # [6] Voigt moment tensor (xx, yy, zz, xy, yz, xz)
    rec_pos: np.ndarray            # [k][3]
    f0: float = 1.5
    # filled by the loop
    slot: Optional[int] = None
    pool: Optional["Pool"] = None
    t0: float = 0.0                # pool time at admission
    admitted: Optional[float] = None
    finished: Optional[float] = None
    steps_done: int = 0
    samples: list = field(default_factory=list)  # per chunk: [k][steps][9]

    def result(self):
        """Receiver samples [k][n_steps][9] at local times 0, dt, 2 dt, ..."""
        s = np.concatenate(self.samples, axis=1) if self.samples else np.zeros((len(self.rec_pos), 0, 9))
        return s[:, :self.n_steps]


class MeshCache:
    def __init__(self, specs):
        self.specs = specs
        self.cache = {}

    def get(self, key):
        if key not in self.cache:
            sp = self.specs[key]
            m = host.Mesh.box(sp.n_cubes, (sp.ext,) * 3, jitter=sp.jitter, seed=sp.seed)
            ne = m.n_el
            rho = np.full(ne, sp.rho)
            mu = rho * sp.vs ** 2
            lam = rho * sp.vp ** 2 - 2 * mu
            star = host.star(m, rho, lam, mu)
            fsE, _ = host.flux_solvers(m, rho, lam, mu)
            self.cache[key] = (m, rho, lam, mu, star, fsE)
        return self.cache[key]


def pool_bytes(n_el, order, runs, precision):
    """Device memory of a pool context (DOFs, two face-projection buffers of the fused steps,
    staging, element data: star matrices, flux solvers and the flux-solver pairs of the pre-mixed
    face projections)."""
    p = 8 if precision == 64 else 4
    w = 16 // p
    gb = math.ceil(host.n_modes(order) / w) * w
    gf = math.ceil(host.n_face_modes(order) / w) * w
    return n_el * (9 * runs * gb * p * 2 + 2 * 36 * runs * gf * p + 9 * host.n_modes(order) * runs * p
                   + (72 + 648) * 8 + 4 * 2 * 84 * p + 28)


class Pool:
    def __init__(self, key, order, meshes, runs=16, precision=32, chunk=20, device=0):
        import torch
        self.key, self.order, self.runs, self.chunk = key, order, runs, chunk
        m, rho, lam, mu, star, fsE = meshes.get(key)
        dt = host.dt_cfl(m, order, rho, lam, mu)
        self.prob = host.Problem(order=order, runs=runs, rm=0, mesh=m, rho=rho, lam=lam, mu=mu, starE=star,
                                 fsE=fsE, dt=dt, name=f"pool_{key}_o{order}")
        self.stream = torch.cuda.Stream(device=device)
        self.solver = Solver(self.prob, precision=precision, stream=self.stream.cuda_stream, device=device)
        e, _ = self.prob.zero_dofs(np.float32 if precision == 32 else np.float64)
        self.solver.upload_dofs(e)
        self.slots = [None] * runs
        self.t = 0.0
        self.dirty = True
        self.entries = []     # union receiver list: (request, receiver index)
        self.bytes = pool_bytes(m.n_el, order, runs, precision)
        self.launched = 0

    def busy(self):
        return any(r is not None for r in self.slots)

    def free_slots(self):
        return [i for i, r in enumerate(self.slots) if r is None]

    def admit(self, req, now):
        slot = self.free_slots()[0]
        self.slots[slot] = req
        req.slot, req.pool, req.t0, req.admitted = slot, self, self.t, now
        lib().edge_b200_set_run_dofs(self.solver._h, slot, None, None)
        self.dirty = True

    def _rebuild(self):
        """Sources and receivers of the active requests (after an admission or a completion)."""
        L = lib()
        h = self.solver._h
        act = [r for r in self.slots if r is not None]
        m = self.prob.mesh
        # sources: one per request, Ricker moment rate shifted to the admission time
        dts = self.prob.dt / 10.0
        srcs = []
        for r in act:
            n_ser = int(math.ceil(r.n_steps * self.prob.dt / dts)) + 4
            el, _, be = host.locate(m, self.order, r.src_pos, source=True)
            ser = host.ricker(np.arange(n_ser) * dts, r.f0, 1.2 / r.f0)
            srcs.append((int(el[0]), r.slot, np.concatenate([r.moment, np.zeros(3)]), be[0], r.t0, ser))
        srcs.sort(key=lambda s: (s[0], s[1]))
        if srcs:
            n = len(srcs)
            el = np.array([s[0] for s in srcs], np.int64)
            run = np.array([s[1] for s in srcs], np.int32)
            scal = np.ascontiguousarray([s[2] for s in srcs], np.float64)
            be = np.ascontiguousarray([s[3] for s in srcs], np.float64)
            t0 = np.array([s[4] for s in srcs], np.float64)
            dt = np.full(n, dts)
            npts = np.array([len(s[5]) for s in srcs], np.int64)
            off = np.concatenate([[0], np.cumsum(npts)[:-1]]).astype(np.int64)
            ts = np.ascontiguousarray(np.concatenate([s[5] for s in srcs]), np.float64)
            self._src_keep = (el, run, scal, be, t0, dt, off, npts, ts)
            L.edge_b200_set_sources(h, n, ptr(el), ptr(run), ptr(scal), ptr(be), ptr(t0), ptr(dt), ptr(off),
                                    ptr(npts), len(ts), ptr(ts))
        else:
            L.edge_b200_set_sources(h, 0, None, None, None, None, None, None, None, None, 0, None)
        # receivers: union of the active requests' receivers, grouped by element
        ent = []
        for r in act:
            el, _, basis = host.locate(m, self.order, r.rec_pos)
            for i in range(len(r.rec_pos)):
                ent.append((int(el[i]), r, i, basis[i]))
        ent.sort(key=lambda x: x[0])
        self.entries = [(x[1], x[2]) for x in ent]
        if ent:
            el = np.array([x[0] for x in ent], np.int64)
            basis = np.ascontiguousarray([x[3] for x in ent], np.float64)
            self._rec_keep = (el, basis)
            L.edge_b200_set_receivers(h, len(ent), ptr(el), ptr(basis), self.t, self.prob.dt, self.chunk + 1)
        else:
            L.edge_b200_set_receivers(h, 0, None, None, 0.0, 1.0, 1)
        self.dirty = False

    def launch(self):
        """Queue one chunk of steps on the pool's stream (asynchronous)."""
        if self.dirty:
            self._rebuild()
        else:
            lib().edge_b200_rewind_receivers(self.solver._h, self.t)
        self.solver.step(self.chunk, t=self.t)
        self.t = self.solver.t
        self.launched = self.chunk

    def _read_samples(self, k):
        """{rid: {receiver index: samples [k][9]}} of the last chunk (synchronises the stream)."""
        per = {}
        if self.entries:
            n = len(self.entries)
            buf = np.zeros((n, self.chunk + 1, 9, self.runs))
            self.solver._chk(lib().edge_b200_read_receivers(self.solver._h, ptr(buf), None, None),
                             "read_receivers")
            for j, (r, i) in enumerate(self.entries):
                per.setdefault(r.rid, {})[i] = buf[j, :k, :, r.slot]
        else:
            self.solver.sync()
        return per

    def collect(self, now):
        """Reads back the chunk's receiver samples and retires the requests that reached their
        step count; returns those."""
        if not self.launched:
            return []
        k = self.launched
        self.launched = 0
        per = self._read_samples(k)
        done = []
        for s, r in enumerate(self.slots):
            if r is None:
                continue
            if r.rid in per:
                d = per[r.rid]
                r.samples.append(np.stack([d[i] for i in range(len(r.rec_pos))]))
            r.steps_done += k
            if r.steps_done >= r.n_steps:
                r.finished = now
                self.slots[s] = None
                self.dirty = True
                done.append(r)
        return done

    def close(self):
        self.solver.close()


class Server:
    """The request loop: admission by free slot and HBM budget, chunked lockstep stepping."""

    def __init__(self, specs, runs=16, precision=32, chunk=20, hbm_fraction=0.8, device=0, budget_bytes=None,
                 pool_cls=None):
        self.meshes = MeshCache(specs)
        self.runs, self.precision, self.chunk, self.device = runs, precision, chunk, device
        self.pool_cls = pool_cls or Pool
        if budget_bytes is None:
            import torch
            free, total = torch.cuda.mem_get_info(device)
            self.budget = hbm_fraction * total
            self.base_used = total - free
        else:
            self.budget, self.base_used = float(budget_bytes), 0.0
        self.pools = {}
        self.pools_opened = 0
        self.max_pools = 0

    def _pool_for(self, req):
        key = (req.mesh, req.order)
        p = self.pools.get(key)
        if p is not None and p.free_slots():
            return p
        if p is not None:
            return None
        m = self.meshes.get(req.mesh)[0]
        need = pool_bytes(m.n_el, req.order, self.runs, self.precision)
        used = self.base_used + sum(q.bytes for q in self.pools.values())
        if used + need > self.budget:
            # close idle pools to make room
            for k in [k for k, q in self.pools.items() if not q.busy()]:
                self.pools.pop(k).close()
            used = self.base_used + sum(q.bytes for q in self.pools.values())
            if used + need > self.budget:
                return None
        p = self.pool_cls(req.mesh, req.order, self.meshes, self.runs, self.precision, self.chunk, self.device)
        self.pools[key] = p
        self.pools_opened += 1
        self.max_pools = max(self.max_pools, len(self.pools))
        return p

    def warm(self, keys):
        """Opens the pools of the given (mesh, order) keys ahead of the first request."""
        for mesh, order in keys:
            if (mesh, order) not in self.pools:
                probe = Request(rid=-1, arrival=0.0, mesh=mesh, order=order, n_steps=0,
                                src_pos=np.zeros(3), moment=np.zeros(6), rec_pos=np.zeros((0, 3)))
                if self._pool_for(probe) is None:
                    raise RuntimeError(f"pool {mesh}/o{order} does not fit the HBM budget")
                p = self.pools[(mesh, order)]
                p.solver.step(2, t=0.0)
                p.solver.sync()

    def run(self, requests, clock="wall"):
        """Serves the requests; returns them in the order they finished.

        clock "wall": arrivals and latencies in seconds of wall time (requests are admitted once
        their arrival time has passed). clock "rounds": arrivals and latencies in rounds of the
        loop (one chunk of steps on every active pool), which makes admission deterministic.
        """
        pending = sorted(requests, key=lambda r: r.arrival)
        finished = []
        t_start = time.perf_counter()
        rounds = 0
        qi = 0
        queue = []

        def now():
            return time.perf_counter() - t_start if clock == "wall" else float(rounds)

        while len(finished) < len(requests):
            t = now()
            while qi < len(pending) and pending[qi].arrival <= t:
                queue.append(pending[qi])
                qi += 1
            waiting = []
            for r in queue:
                p = self._pool_for(r)
                if p is None:
                    waiting.append(r)
                else:
                    p.admit(r, t)
            queue = waiting
            active = [p for p in self.pools.values() if p.busy()]
            if not active:
                if queue:
                    raise RuntimeError(f"request {queue[0].rid} does not fit the HBM budget")
                if qi >= len(pending):
                    raise RuntimeError("requests lost")
                if clock == "wall":
                    time.sleep(max(0.0, min(0.01, pending[qi].arrival - t)))
                else:
                    rounds += 1
                continue
            for p in active:
                p.launch()
            rounds += 1
            for p in active:
                finished.extend(p.collect(now()))
        self.wall = time.perf_counter() - t_start
        self.rounds = rounds
        return finished

    def close(self):
        for p in self.pools.values():
            p.close()
        self.pools = {}


def latency_stats(reqs):
    lat = np.array([r.finished - r.arrival for r in reqs])
    return dict(p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)), mean=float(lat.mean()))


def make_stream(n, rate, specs, orders=(3, 4, 5), steps=(100, 400), n_rec=(4, 16), seed=0):
    """Poisson arrivals (mean rate per second) of random requests over the mesh specs."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    keys = sorted(specs)
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        k = keys[rng.integers(len(keys))]
        ext = specs[k].ext
        nr = int(rng.integers(n_rec[0], n_rec[1] + 1))
        out.append(Request(rid=i, arrival=t, mesh=k, order=int(rng.choice(orders)),
                           n_steps=int(rng.integers(steps[0], steps[1] + 1)),
                           src_pos=rng.uniform(0.1 * ext, 0.9 * ext, 3),
                           moment=rng.normal(0.0, 1.0, 6) * 1e15,
                           rec_pos=rng.uniform(0.1 * ext, 0.9 * ext, (nr, 3))))
    return out
