"""Host logic of the serving loop (admission, queueing, HBM budget, completion) on the CPU.

The device pool is replaced by a stand-in that keeps the slot bookkeeping of edge_b200.serve.Pool
and advances its requests without a GPU; meshes are built by the host library.
"""
import numpy as np

from edge_b200 import serve


class _CpuPool(serve.Pool):
    def __init__(self, key, order, meshes, runs=16, precision=32, chunk=20, device=0, rm=0):
        self.key, self.order, self.runs, self.chunk, self.rm = key, order, runs, chunk, rm
        m = meshes.get(key)[0]
        self.slots = [None] * runs
        self.t = 0.0
        self.dirty = True
        self.entries = []
        self.bytes = serve.pool_bytes(m.n_el, order, runs, precision, rm)
        self.launched = 0
        self.closed = False

    def admit(self, req, now):
        slot = self.free_slots()[0]
        self.slots[slot] = req
        req.slot, req.pool, req.t0, req.admitted = slot, self, self.t, now
        self.dirty = True

    def launch(self):
        self.dirty = False
        k = max(1, min(self.chunk, max(r.n_steps - r.steps_done for r in self.slots if r is not None)))
        self.members = {r.rid for r in self.slots if r is not None}
        self.t += k
        self.launched = k

    def done(self):
        return True

    def take_over(self, old):
        self.t = old.t
        j = 0
        for i, r in enumerate(old.slots):
            if r is not None:
                r.slot, r.pool = j, self
                self.slots[j], old.slots[i] = r, None
                j += 1
        self.dirty = True

    def _read_samples(self, k):
        return {r.rid: {i: np.full((k, 9), float(r.rid)) for i in range(len(r.rec_pos))}
                for r in self.slots if r is not None}

    def close(self):
        self.closed = True


SPECS = {"a": serve.MeshSpec(n_cubes=3), "b": serve.MeshSpec(n_cubes=3, vp=5000.0, vs=2887.0)}


def test_stream_is_seeded():
    a = serve.make_stream(20, 10.0, SPECS, seed=4)
    b = serve.make_stream(20, 10.0, SPECS, seed=4)
    assert [(r.arrival, r.mesh, r.order, r.n_steps) for r in a] == [(r.arrival, r.mesh, r.order, r.n_steps)
                                                                       for r in b]
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))


def test_pool_bytes_grow_with_order_and_runs():
    assert serve.pool_bytes(1000, 5, 16, 32) > serve.pool_bytes(1000, 4, 16, 32)
    assert serve.pool_bytes(1000, 4, 16, 32) > serve.pool_bytes(1000, 4, 8, 32)
    assert serve.pool_bytes(1000, 4, 16, 64) > serve.pool_bytes(1000, 4, 16, 32)


def _reqs():
    rng = np.random.default_rng(0)
    out = []
    for i in range(40):
        out.append(serve.Request(rid=i, arrival=float(i // 8), mesh="a" if i % 4 else "b", order=4,
                                 n_steps=int(rng.integers(10, 90)), src_pos=np.zeros(3), moment=np.zeros(6),
                                 rec_pos=np.zeros((2, 3))))
    return out


def test_slots_queue_and_complete():
    reqs = _reqs()
    srv = serve.Server(SPECS, runs=4, chunk=10, budget_bytes=1e12, pool_cls=_CpuPool, sizes=(4,))
    done = srv.run(reqs, clock="rounds")
    assert sorted(r.rid for r in done) == list(range(40))
    assert srv.max_pools == 2
    for r in done:
        res = r.result()
        assert res.shape == (2, r.n_steps, 9) and (res == r.rid).all()
        assert r.arrival <= r.admitted < r.finished
        # whole chunks: a request holds its slot for ceil(n_steps / chunk) rounds
        assert r.finished - r.admitted == -(-r.n_steps // 10)
    # no slot ever held two requests at once
    for key in ("a", "b"):
        spans = {}
        for r in done:
            if r.mesh == key:
                spans.setdefault(r.slot, []).append((r.admitted, r.finished))
        for iv in spans.values():
            iv.sort()
            assert all(x[1] <= y[0] for x, y in zip(iv, iv[1:]))


def test_budget_admits_one_pool_at_a_time():
    reqs = _reqs()
    big = max(serve.pool_bytes(serve.MeshCache(SPECS).get(k)[0].n_el, 4, 4, 32) for k in SPECS)
    srv = serve.Server(SPECS, runs=4, chunk=10, budget_bytes=1.5 * big, pool_cls=_CpuPool, sizes=(4,))
    done = srv.run(reqs, clock="rounds")
    assert len(done) == 40
    assert srv.max_pools == 1 and srv.pools_opened >= 2


def test_request_larger_than_budget_fails_loudly():
    reqs = _reqs()[:3]
    srv = serve.Server(SPECS, runs=4, chunk=10, budget_bytes=1.0, pool_cls=_CpuPool)
    try:
        srv.run(reqs, clock="rounds")
    except RuntimeError as e:
        assert "budget" in str(e)
    else:
        raise AssertionError("expected a budget error")


def test_viscoelastic_requests_get_pools_of_their_own():
    reqs = _reqs()
    for r in reqs[::3]:
        r.rm = 3
    srv = serve.Server(SPECS, runs=4, chunk=10, budget_bytes=1e12, pool_cls=_CpuPool)
    done = srv.run(reqs, clock="rounds")
    assert len(done) == 40
    assert srv.max_pools == 4  # (mesh a / b) x (elastic / viscoelastic)
    for r in done:
        assert r.pool.rm == r.rm and r.pool.key == r.mesh


def test_stream_physics_and_orders():
    reqs = serve.make_stream(400, 20.0, SPECS, orders=(3, 4, 5, 6), seed=2, visco=0.3, visco_orders=(3, 4),
                             mesh_steps={"a": (100, 200), "b": (300, 400)})
    vis = [r for r in reqs if r.rm]
    assert 80 < len(vis) < 160
    assert {r.order for r in vis} <= {3, 4} and {r.order for r in reqs if not r.rm} == {3, 4, 5, 6}
    assert all(100 <= r.n_steps <= 200 for r in reqs if r.mesh == "a")
    assert all(300 <= r.n_steps <= 400 for r in reqs if r.mesh == "b")


def test_material_sets_and_anelastic_data():
    specs = {"l": serve.MeshSpec(n_cubes=3, layers=(4000.0, 6000.0), lognormal_sigma=0.1, seed=5)}
    mc = serve.MeshCache(specs)
    e, v = mc.data("l", 0), mc.data("l", 3)
    assert e["starA"] is None and v["srcA"].shape == (e["mesh"].n_el, 3, 12) and v["fsA"].shape[-1] == 54
    assert len(np.unique(e["lam"])) > 2                     # layered and perturbed per element
    assert (v["mu"] > e["mu"]).all()                        # unrelaxed moduli exceed the phase values
    assert serve.pool_bytes(1000, 4, 16, 32, 3) > serve.pool_bytes(1000, 4, 16, 32, 0)
    p = mc.problem("l", 4, 8, 3)
    assert p.rm == 3 and p.dt < mc.problem("l", 4, 8, 0).dt


def test_pools_grow_and_shrink_with_demand():
    """Pools open with the fewest runs that hold the waiting requests, grow when full while more
    wait, and shrink to the smallest size holding their running tail; requests keep their
    progress across the moves and every result stays whole."""
    rng = np.random.default_rng(3)
    reqs = [serve.Request(rid=i, arrival=float(i // 6), mesh="a", order=4, n_steps=int(rng.integers(10, 300)),
                          src_pos=np.zeros(3), moment=np.zeros(6), rec_pos=np.zeros((2, 3))) for i in range(30)]
    srv = serve.Server(SPECS, runs=16, chunk=10, budget_bytes=1e12, pool_cls=_CpuPool)
    sizes = []
    orig = srv._open

    def spy(req, runs):
        sizes.append(runs)
        return orig(req, runs)

    srv._open = spy
    done = srv.run(reqs, clock="rounds")
    assert sorted(r.rid for r in done) == list(range(30))
    assert srv.resizes >= 2 and sizes[0] < 16 and max(sizes) == 16 and min(sizes[1:]) < 16
    for r in done:
        res = r.result()
        assert res.shape == (2, r.n_steps, 9) and (res == r.rid).all()
        assert r.steps_done >= r.n_steps


def test_wall_clock_loop_serves_everything():
    reqs = _reqs()
    for i, r in enumerate(reqs):
        r.arrival = 0.0005 * i
    srv = serve.Server(SPECS, runs=16, chunk=10, budget_bytes=1e12, pool_cls=_CpuPool)
    done = srv.run(reqs, clock="wall")
    assert sorted(r.rid for r in done) == list(range(40))
    for r in done:
        assert r.result().shape == (2, r.n_steps, 9) and (r.result() == r.rid).all()
