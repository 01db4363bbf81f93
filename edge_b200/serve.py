"""Continuous batching of simulation requests over fused-run slots (the serving form).

A *pool* is one device context (one mesh with its material set, order and physics: elastic or
viscoelastic with 3 mechanisms) with R fused-run slots and its own CUDA stream. A request (its own
point source, receivers and number of steps) occupies one slot of a pool of its mesh, order and
physics; requests that arrive while others run are admitted as soon as a slot is free, so the runs
of one pool start and end at different times: the pool steps all slots in lockstep (the fused-run
kernels), a slot's DOFs (elastic and anelastic) are reset when it is handed to a new request
(edge_b200_set_run_dofs), the sources of a request are time-shifted to its admission time, and its
receivers are read back every chunk of steps. Pools run concurrently on their own streams. New
pools are admitted against an HBM budget; idle pools are closed to free memory. Latency is
arrival -> last sample read back. ``plain_fp64`` runs one request alone on the plain FP64 path, the
reference every served result can be checked against.
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
    """A synthetic mesh and its material set, referred to by key: homogeneous (vp, vs, rho) or
    horizontal vp layers from the top (vs = vp / sqrt(3)) with a seeded lognormal factor per
    element; viscoelastic pools add Qp, Qs uniform in q_range and 3 mechanisms around freq_cen."""
    n_cubes: int
    ext: float = 1e4
    jitter: float = 0.0
    seed: int = 0
    vp: float = 6000.0
    vs: float = 3464.0
    rho: float = 2670.0
    layers: Optional[tuple] = None
    lognormal_sigma: float = 0.0
    q_range: tuple = (50.0, 200.0)
    freq_cen: float = 1.0
    freq_rat: float = 100.0


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
    rm: int = 0                    # relaxation mechanisms (0 elastic, 3 viscoelastic)
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
        self.data_cache = {}

    def get(self, key):
        """(mesh, rho, lam, mu, starE, fsE) of the elastic material set."""
        d = self.data(key, 0)
        return d["mesh"], d["rho"], d["lam"], d["mu"], d["starE"], d["fsE"]

    def data(self, key, rm=0):
        """Mesh, material and element data of a spec for rm mechanisms (a dict; with rm > 0, lam and
        mu are the unrelaxed values and the anelastic data are included)."""
        if (key, rm) not in self.data_cache:
            sp = self.specs[key]
            if key not in self.cache:
                self.cache[key] = host.Mesh.box(sp.n_cubes, (sp.ext,) * 3, jitter=sp.jitter, seed=sp.seed)
            m = self.cache[key]
            rng = np.random.default_rng(sp.seed + 1)
            rho, lam, mu = host.materials(m, sp.ext, sp.vp, sp.vs, sp.rho, sp.layers, sp.lognormal_sigma, rng)
            qp = qs = None
            if rm:
                qp = rng.uniform(sp.q_range[0], sp.q_range[1], m.n_el)
                qs = rng.uniform(sp.q_range[0], sp.q_range[1], m.n_el)
            d = host.element_data(m, rho, lam, mu, rm, qp, qs, sp.freq_cen, sp.freq_rat)
            d.update(mesh=m, rho=rho)
            self.data_cache[(key, rm)] = d
        return self.data_cache[(key, rm)]

    def problem(self, key, order, runs, rm=0):
        d = self.data(key, rm)
        dt = host.dt_cfl(d["mesh"], order, d["rho"], d["lam"], d["mu"])
        return host.Problem(order=order, runs=runs, rm=rm, mesh=d["mesh"], rho=d["rho"], lam=d["lam"],
                            mu=d["mu"], starE=d["starE"], fsE=d["fsE"], dt=dt, starA=d["starA"], srcA=d["srcA"],
                            fsA=d["fsA"], omega=d["omega"], name=f"pool_{key}_o{order}_m{rm}")


def element_data_bytes(n_el, rm=0):
    """Device memory of a mesh's FP64 element data (star matrices, flux solvers, anelastic data)."""
    return n_el * ((72 + 648) + (rm * 12 + 27 + 2 * 4 * 54) * (rm > 0)) * 8


def pool_bytes(n_el, order, runs, precision, rm=0, shared=False):
    """Device memory of a pool context (DOF and anelastic rows, two face-projection buffers of the
    fused steps, staging, the flux-solver pairs of the pre-mixed face projections and, unless
    borrowed from the mesh's anchor context (shared), the element data)."""
    p = 8 if precision == 64 else 4
    w = 16 // p
    gb = math.ceil(host.n_modes(order) / w) * w
    gf = math.ceil(host.n_face_modes(order) / w) * w
    nq = 9 + 6 * rm
    own = n_el * (nq * runs * gb * p * 2 + 2 * 36 * runs * gf * p + nq * host.n_modes(order) * runs * p
                  + 4 * 2 * 84 * p + 28)
    return own + (0 if shared else element_data_bytes(n_el, rm))


class Pool:
    def __init__(self, key, order, meshes, runs=16, precision=32, chunk=20, device=0, rm=0, anchor=None):
        import torch
        self.key, self.order, self.runs, self.chunk, self.rm = key, order, runs, chunk, rm
        self.prob = meshes.problem(key, order, runs, rm)
        m = self.prob.mesh
        self.stream = torch.cuda.Stream(device=device)
        # (a new context's DOFs start at zero; its element data come from the mesh's anchor context)
        self.solver = Solver(self.prob, precision=precision, stream=self.stream.cuda_stream, device=device,
                             share_from=anchor)
        self.slots = [None] * runs
        self.t = 0.0
        self.dirty = True
        self.entries = []     # union receiver list: (request, receiver index)
        self.bytes = pool_bytes(m.n_el, order, runs, precision, rm, shared=anchor is not None)
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
        """Queue one chunk of steps on the pool's stream (asynchronous): `chunk` steps, fewer when
        every active request finishes sooner."""
        if self.dirty:
            self._rebuild()
        else:
            lib().edge_b200_rewind_receivers(self.solver._h, self.t)
        k = max(1, min(self.chunk, max(r.n_steps - r.steps_done for r in self.slots if r is not None)))
        self.members = {r.rid for r in self.slots if r is not None}
        self.solver.step(k, t=self.t)
        self.t = self.solver.t
        self.launched = k

    def take_over(self, old):
        """Moves the running requests of pool `old` (same mesh, order and physics) into this pool's
        first slots: their DOFs are copied run by run on the device (edge_b200_copy_run), the pool
        continues at old's time, and sources and receivers are rebuilt before the next chunk."""
        self.t = old.t
        j = 0
        for i, r in enumerate(old.slots):
            if r is None:
                continue
            self.solver._chk(lib().edge_b200_copy_run(self.solver._h, j, old.solver._h, i), "copy_run")
            r.slot, r.pool = j, self
            self.slots[j] = r
            old.slots[i] = None
            j += 1
        self.dirty = True

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

    def done(self):
        """True when the chunk in flight (if any) has completed on the pool's stream."""
        return self.stream.query()

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
            if r is None or r.rid not in self.members:
                continue  # (admitted while the chunk ran: it starts with the next one)
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
                 pool_cls=None, sizes=None):
        self.meshes = MeshCache(specs)
        self.runs, self.precision, self.chunk, self.device = runs, precision, chunk, device
        # fused-run counts a pool may have (compiled configurations): a pool opens with the fewest
        # runs that hold the requests waiting for it, grows when it is full and more wait, and
        # shrinks when its tail of long requests would leave most slots idle
        if sizes is None:
            sizes = (1, 4, 8, 16) if precision == 32 else (1,)
        self.sizes = tuple(sorted(x for x in sizes if x <= runs)) or (runs,)
        self.resizes = 0
        # element updates the pools computed (all slots) and those of occupied slots
        self.slot_updates_offered = 0
        self.slot_updates_used = 0
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
        # per (mesh, mechanisms): a small context holding the mesh's element data once on the device,
        # which every pool of the mesh borrows (pools open without uploading them)
        self.anchors = {}
        self.share_element_data = True

    def _size_for(self, n):
        for x in self.sizes:
            if x >= n:
                return x
        return self.sizes[-1]

    def _anchor(self, mesh, rm):
        if not self.share_element_data or self.pool_cls is not Pool:
            return None
        if (mesh, rm) not in self.anchors:
            p = self.meshes.problem(mesh, 3, 1, rm)
            s = Solver(p, precision=32, device=self.device)
            s.bytes = element_data_bytes(p.n_el, rm) + pool_bytes(p.n_el, 3, 1, 32, rm, shared=True)
            self.anchors[(mesh, rm)] = s
        return self.anchors[(mesh, rm)]

    def _used(self):
        return (self.base_used + sum(q.bytes for q in self.pools.values())
                + sum(a.bytes for a in self.anchors.values()))

    def _fits(self, req, runs):
        m = self.meshes.data(req.mesh, req.rm)["mesh"]
        shared = self.share_element_data and self.pool_cls is Pool
        need = pool_bytes(m.n_el, req.order, runs, self.precision, req.rm, shared=shared)
        if shared and (req.mesh, req.rm) not in self.anchors:
            need += element_data_bytes(m.n_el, req.rm) + pool_bytes(m.n_el, 3, 1, 32, req.rm, shared=True)
        used = self._used()
        if used + need > self.budget:
            # close idle pools to make room
            for k in [k for k, q in self.pools.items() if not q.busy()]:
                self.pools.pop(k).close()
            # and the anchors of meshes without an open pool (other than the one asked for)
            live = {(k[0], k[2]) for k in self.pools}
            for k in [k for k in self.anchors if k not in live and k != (req.mesh, req.rm)]:
                self.anchors.pop(k).close()
            used = self._used()
        return used + need <= self.budget

    def _open(self, req, runs):
        anchor = self._anchor(req.mesh, req.rm)
        if anchor is not None:
            p = self.pool_cls(req.mesh, req.order, self.meshes, runs, self.precision, self.chunk, self.device,
                              req.rm, anchor=anchor)
        else:
            p = self.pool_cls(req.mesh, req.order, self.meshes, runs, self.precision, self.chunk, self.device,
                              req.rm)
        self.pools_opened += 1
        return p

    def _pool_for(self, req, demand=1):
        """The pool a request joins (opened, or grown, if need be), or None when it must wait.
        demand: requests of the same mesh, order and physics waiting, this one included."""
        key = (req.mesh, req.order, req.rm)
        p = self.pools.get(key)
        if p is not None and p.free_slots():
            return p
        if p is not None:
            # full: grow into a larger pool that also holds the waiting requests (between chunks)
            if p.launched:
                return None
            want = self._size_for(p.runs + demand)
            while want > p.runs and not self._fits(req, want):
                want = max([x for x in self.sizes if x < want] or [p.runs])
            if want <= p.runs:
                return None
            q = self._open(req, want)
            q.take_over(p)
            p.close()
            self.pools[key] = q
            self.resizes += 1
            return q
        # the fewest runs that hold the waiting requests, fewer where the HBM budget requires it
        runs = self._size_for(demand)
        while not self._fits(req, runs):
            smaller = [x for x in self.sizes if x < runs]
            if not smaller:
                return None
            runs = smaller[-1]
        p = self._open(req, runs)
        self.pools[key] = p
        self.max_pools = max(self.max_pools, len(self.pools))
        return p

    def _compact(self, queue):
        """Shrinks pools whose running requests fit a smaller run count when nothing waits for them."""
        waiting = {(r.mesh, r.order, r.rm) for r in queue}
        for key, p in list(self.pools.items()):
            n = sum(1 for r in p.slots if r is not None)
            want = self._size_for(n)
            if n == 0 or p.launched or key in waiting or want >= p.runs:
                continue
            probe = next(r for r in p.slots if r is not None)
            if not self._fits(probe, want):
                continue
            q = self._open(probe, want)
            q.take_over(p)
            p.close()
            self.pools[key] = q
            self.resizes += 1

    def warm(self, keys):
        """Opens the pools of the given (mesh, order[, mechanisms]) keys ahead of the first request."""
        for k in keys:
            mesh, order, rm = (tuple(k) + (0,))[:3]
            if (mesh, order, rm) not in self.pools:
                probe = Request(rid=-1, arrival=0.0, mesh=mesh, order=order, n_steps=0,
                                src_pos=np.zeros(3), moment=np.zeros(6), rec_pos=np.zeros((0, 3)), rm=rm)
                if self._pool_for(probe, self.runs) is None:
                    raise RuntimeError(f"pool {mesh}/o{order}/m{rm} does not fit the HBM budget")
                p = self.pools[(mesh, order, rm)]
                p.solver.step(2, t=0.0)
                p.solver.sync()

    def run(self, requests, clock="wall"):
        """Serves the requests; returns them in the order they finished.

        clock "wall": arrivals and latencies in seconds of wall time (requests are admitted once
        their arrival time has passed); every pool runs its own cycle of chunks -- a pool whose
        chunk has completed on its stream is read back and relaunched at once, so small and large
        pools do not wait for each other. clock "rounds": arrivals and latencies in rounds of the
        loop (one chunk of steps on every active pool, all read back together), which makes
        admission deterministic.
        """
        pending = sorted(requests, key=lambda r: r.arrival)
        finished = []
        t_start = time.perf_counter()
        rounds = 0
        qi = 0
        queue = []
        wall = clock == "wall"

        def now():
            return time.perf_counter() - t_start if wall else float(rounds)

        def launch(p):
            p.launch()
            ne = p.prob.n_el if hasattr(p, "prob") else 1
            self.slot_updates_offered += p.runs * p.launched * ne
            self.slot_updates_used += sum(1 for r in p.slots if r is not None) * p.launched * ne

        def admit(queue):
            t = now()
            waiting = []
            demand = {}
            for r in queue:
                k = (r.mesh, r.order, r.rm)
                demand[k] = demand.get(k, 0) + 1
            for r in queue:
                k = (r.mesh, r.order, r.rm)
                p = self._pool_for(r, demand[k])
                if p is None:
                    waiting.append(r)
                else:
                    p.admit(r, t)
                    demand[k] -= 1
            return waiting

        while len(finished) < len(requests):
            t = now()
            while qi < len(pending) and pending[qi].arrival <= t:
                queue.append(pending[qi])
                qi += 1
            if wall:
                # read back the pools whose chunk completed first, so that their freed slots, growth
                # and shrinking are settled before they are relaunched
                for p in list(self.pools.values()):
                    if p.launched and p.done():
                        finished.extend(p.collect(now()))
                if len(finished) >= len(requests):
                    break
            queue = admit(queue)
            active = [p for p in self.pools.values() if p.busy() or p.launched]
            if not active:
                if queue:
                    raise RuntimeError(f"request {queue[0].rid} does not fit the HBM budget")
                if qi >= len(pending):
                    raise RuntimeError("requests lost")
                if wall:
                    time.sleep(max(0.0, min(0.01, pending[qi].arrival - t)))
                else:
                    rounds += 1
                continue
            if wall:
                progressed = False
                self._compact(queue)
                for p in list(self.pools.values()):
                    if p.busy() and not p.launched:
                        launch(p)
                        progressed = True
                rounds += 1
                if not progressed:
                    time.sleep(0.0002)
            else:
                for p in active:
                    launch(p)
                rounds += 1
                for p in active:
                    finished.extend(p.collect(now()))
                self._compact(queue)
        self.wall = time.perf_counter() - t_start
        self.rounds = rounds
        return finished

    def close(self):
        for p in self.pools.values():
            p.close()
        self.pools = {}
        for a in self.anchors.values():
            a.close()
        self.anchors = {}


def latency_stats(reqs):
    lat = np.array([r.finished - r.arrival for r in reqs])
    return dict(p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)), mean=float(lat.mean()))


def make_stream(n, rate, specs, orders=(3, 4, 5), steps=(100, 400), n_rec=(4, 16), seed=0, visco=0.0,
                visco_orders=(3, 4), mesh_steps=None):
    """Poisson arrivals (mean rate per second) of random requests over the mesh specs; a fraction
    `visco` of them viscoelastic (3 mechanisms, orders from visco_orders). mesh_steps: optional
    per-mesh (lo, hi) step ranges replacing `steps`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    keys = sorted(specs)
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        k = keys[rng.integers(len(keys))]
        ext = specs[k].ext
        nr = int(rng.integers(n_rec[0], n_rec[1] + 1))
        rm = 3 if rng.uniform() < visco else 0
        order = int(rng.choice(visco_orders if rm else orders))
        lo, hi = (mesh_steps or {}).get(k, steps)
        out.append(Request(rid=i, arrival=t, mesh=k, order=order, n_steps=int(rng.integers(lo, hi + 1)),
                           src_pos=rng.uniform(0.1 * ext, 0.9 * ext, 3),
                           moment=rng.normal(0.0, 1.0, 6) * 1e15,
                           rec_pos=rng.uniform(0.1 * ext, 0.9 * ext, (nr, 3)), rm=rm))
    return out


def plain_fp64(req, meshes, device=0):
    """The request alone as a single-run plain FP64 simulation through the C ABI (no serving loop):
    receiver samples [k][n_steps][9] at local times 0, dt, 2 dt, ... like Request.result()."""
    prob = meshes.problem(req.mesh, req.order, 1, req.rm)
    m, dt = prob.mesh, prob.dt
    dts = dt / 10.0
    n_ser = int(math.ceil(req.n_steps * dt / dts)) + 4
    el, _, be = host.locate(m, req.order, req.src_pos, source=True)
    prob.sources = dict(n=1, el=el.astype(np.int64), run=np.zeros(1, np.int32),
                        scal=np.concatenate([req.moment, np.zeros(3)])[None].copy(), bEval=be.copy(),
                        t0=np.zeros(1), dt=np.full(1, dts), tsOff=np.zeros(1, np.int64),
                        nPts=np.full(1, n_ser, np.int64), ts=host.ricker(np.arange(n_ser) * dts, req.f0, 1.2 / req.f0))
    prob.receivers = host.make_receivers(m, req.order, req.rec_pos, dt, req.n_steps * dt)
    s = Solver(prob, precision=64, device=device)
    try:
        e, a = prob.zero_dofs()
        s.upload_dofs(e, a)
        s.step(req.n_steps)
        buf, _, cnt = s.receivers()
    finally:
        s.close()
    out = np.zeros((len(req.rec_pos), req.n_steps, 9))
    out[prob.receivers["perm"]] = buf[:, :req.n_steps, :, 0]
    return out
