"""Host logic of the serving loop (admission, queueing, HBM budget, completion) on the CPU.

The device pool is replaced by a stand-in that keeps the slot bookkeeping of edge_b200.serve.Pool
and advances its requests without a GPU; meshes are built by the host library.
"""
import numpy as np

from edge_b200 import serve


class _CpuPool(serve.Pool):
    def __init__(self, key, order, meshes, runs=16, precision=32, chunk=20, device=0):
        self.key, self.order, self.runs, self.chunk = key, order, runs, chunk
        m = meshes.get(key)[0]
        self.slots = [None] * runs
        self.t = 0.0
        self.dirty = True
        self.entries = []
        self.bytes = serve.pool_bytes(m.n_el, order, runs, precision)
        self.launched = 0
        self.closed = False

    def admit(self, req, now):
        slot = self.free_slots()[0]
        self.slots[slot] = req
        req.slot, req.pool, req.t0, req.admitted = slot, self, self.t, now
        self.dirty = True

    def launch(self):
        self.dirty = False
        self.t += self.chunk
        self.launched = self.chunk

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
    srv = serve.Server(SPECS, runs=4, chunk=10, budget_bytes=1e12, pool_cls=_CpuPool)
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
    srv = serve.Server(SPECS, runs=4, chunk=10, budget_bytes=1.5 * big, pool_cls=_CpuPool)
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
