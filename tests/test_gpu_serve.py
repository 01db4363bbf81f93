"""Serving loop (edge_b200.serve): continuous batching of requests over fused-run slots.

A request's receiver traces must not depend on when it is admitted, which slot it gets or which
requests share its pool: the fused runs of the element update are independent, so a request run
alone and the same request run in a mix agree to FP32 rounding (the source time integrals see
shifted time origins). The alone run is itself checked against a plain FP64 run of the same
source and receivers through the C ABI.
"""
import numpy as np
import pytest

from edge_b200 import host, serve
from edge_b200.solver import Solver

pytestmark = pytest.mark.gpu

SPECS = {"a": serve.MeshSpec(n_cubes=4, ext=4e3),
         "b": serve.MeshSpec(n_cubes=3, ext=3e3, vp=5000.0, vs=2887.0, rho=2500.0)}
CHUNK = 10


def _dt(mesh, order):
    m, rho, lam, mu, _, _ = serve.MeshCache(SPECS).get(mesh)
    return host.dt_cfl(m, order, rho, lam, mu)


def _req(rid, arrival, mesh="a", order=4, n_steps=45, seed=None, rm=0):
    rng = np.random.default_rng(1000 + rid if seed is None else seed)
    ext = SPECS[mesh].ext
    dt = _dt(mesh, order)
    return serve.Request(rid=rid, arrival=arrival, mesh=mesh, order=order, n_steps=n_steps,
                         src_pos=rng.uniform(0.35 * ext, 0.65 * ext, 3),
                         moment=rng.normal(0.0, 1.0, 6),
                         rec_pos=rng.uniform(0.1 * ext, 0.9 * ext, (5, 3)),
                         f0=1.2 / (0.3 * n_steps * dt), rm=rm)


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _plain_fp64(req):
    """The request as a single-run FP64 simulation through the C ABI (no serving loop)."""
    return serve.plain_fp64(req, serve.MeshCache(SPECS))


def test_alone_matches_plain_fp64():
    req = _req(0, 0.0)
    srv = serve.Server(SPECS, chunk=CHUNK)
    try:
        done = srv.run([req], clock="rounds")
    finally:
        srv.close()
    assert len(done) == 1 and req.slot == 0 and req.t0 == 0.0
    got = req.result()
    ref = _plain_fp64(req)
    assert got.shape == ref.shape
    assert np.abs(ref).max() > 0
    assert _rel(got, ref) < 1e-4


def test_alone_equals_in_the_mix():
    target = lambda rid, arr: _req(rid, arr, seed=7)
    alone = target(0, 0.0)
    srv = serve.Server(SPECS, chunk=CHUNK)
    try:
        srv.run([alone], clock="rounds")
    finally:
        srv.close()
    # the mix: 20 requests on the target's pool (more than its 16 slots, so some queue), others on
    # a second mesh and a second order that run on their own pools and streams
    mix = [_req(i, float(i // 4), n_steps=25 + 7 * (i % 5)) for i in range(1, 21)]
    mix += [_req(100 + i, float(i), mesh="b", order=3, n_steps=40) for i in range(6)]
    mix += [_req(200 + i, float(i), order=5, n_steps=30) for i in range(4)]
    tgt = target(999, 3.0)
    mix.append(tgt)
    srv = serve.Server(SPECS, chunk=CHUNK)
    try:
        done = srv.run(mix, clock="rounds")
    finally:
        srv.close()
    assert len(done) == len(mix)
    assert srv.max_pools == 3
    # admitted late, and moved between pools of different run counts on its way (device copies of
    # its run's DOFs)
    assert tgt.t0 > 0.0 and srv.resizes > 0, (tgt.t0, srv.resizes)
    a, b = alone.result(), tgt.result()
    assert a.shape == b.shape == (5, 45, 9)
    assert _rel(b, a) < 1e-5
    for r in mix:
        res = r.result()
        assert res.shape == (5, r.n_steps, 9) and np.isfinite(res).all()
        assert r.finished >= r.admitted >= r.arrival


def test_hbm_budget_serialises_pools():
    reqs = [_req(i, 0.0, n_steps=20) for i in range(3)] + [_req(10 + i, 0.0, mesh="b", order=3, n_steps=20)
                                                          for i in range(3)]
    srv = serve.Server(SPECS, chunk=CHUNK, sizes=(16,))
    srv.share_element_data = False  # each pool holds its own element data here: the budget counts pools only
    try:
        big = max(serve.pool_bytes(serve.MeshCache(SPECS).get(k)[0].n_el, o, srv.runs, srv.precision)
                  for k, o in (("a", 4), ("b", 3)))
        srv.budget = srv.base_used + 1.05 * big
        done = srv.run(reqs, clock="rounds")
    finally:
        srv.close()
    assert len(done) == len(reqs)
    assert srv.max_pools == 1 and srv.pools_opened == 2
    first = {r.mesh for r in done[:3]}
    assert len(first) == 1


def test_wall_clock_stream_latency():
    specs_keys = {"a": 4, "b": 3}
    rng = np.random.default_rng(5)
    reqs, t = [], 0.0
    for i in range(40):
        t += rng.exponential(0.01)
        k = "a" if i % 3 else "b"
        reqs.append(_req(i, t, mesh=k, order=specs_keys[k], n_steps=int(rng.integers(20, 60))))
    srv = serve.Server(SPECS, chunk=CHUNK)
    try:
        done = srv.run(reqs, clock="wall")
    finally:
        srv.close()
    assert len(done) == 40
    st = serve.latency_stats(done)
    assert 0 < st["p50"] <= st["p99"]
    for r in done:
        assert r.result().shape == (5, r.n_steps, 9)


def test_viscoelastic_alone_matches_plain_fp64():
    req = _req(0, 0.0, rm=3)
    srv = serve.Server(SPECS, chunk=CHUNK)
    try:
        srv.run([req], clock="rounds")
    finally:
        srv.close()
    got, ref = req.result(), _plain_fp64(req)
    assert np.abs(ref).max() > 0
    assert _rel(got, ref) < 1e-4


def test_viscoelastic_alone_equals_in_the_mix():
    """A viscoelastic request alone and in a mix of elastic and viscoelastic requests on shared
    pools (its own pool is viscoelastic, order 4: 3 mechanisms, 16 runs)."""
    alone = _req(0, 0.0, seed=11, rm=3)
    srv = serve.Server(SPECS, chunk=CHUNK)
    try:
        srv.run([alone], clock="rounds")
    finally:
        srv.close()
    mix = [_req(i, float(i // 4), n_steps=25 + 7 * (i % 5), rm=3 * (i % 2)) for i in range(1, 25)]
    mix += [_req(100 + i, float(i), mesh="b", order=3, n_steps=40, rm=3) for i in range(4)]
    tgt = _req(999, 2.0, seed=11, rm=3)
    mix.append(tgt)
    srv = serve.Server(SPECS, chunk=CHUNK)
    try:
        done = srv.run(mix, clock="rounds")
    finally:
        srv.close()
    assert len(done) == len(mix)
    assert srv.max_pools == 3
    assert tgt.t0 > 0.0
    assert _rel(tgt.result(), alone.result()) < 1e-5
