"""Rate-2 local time stepping: EDGE-V's time groups and the oracle's LTS schedule (CPU).

The oracle's LTS work regions restate AderDg.hpp:384-417 / 620-674 and the rate-2 dependencies of
man_sched.inc; with one time group they must reproduce the GTS step, and with two groups on a
smooth plane wave they must be as accurate as GTS with either step and converge at the scheme's
order.
"""
import numpy as np

import oracle
from edge_b200 import host
from helpers import OracleRun, random_dofs, rel_l2


def _edge_v_groups(mesh, dt_el, n_groups, fun_dt=1.0):
    """EDGE-V's setElTg + normalizeElTgs written out (time/Groups.cpp:47-100)."""
    ts = dt_el / dt_el.min()
    bounds = [fun_dt * 2.0 ** (g + 1) for g in range(n_groups - 1)] + [np.inf]
    tg = np.array([next(g for g, b in enumerate(bounds) if t < b) for t in ts], np.int64)
    while True:
        changed = 0
        for e in range(mesh.n_el):
            for f in range(4):
                ad = mesh.el_fa_el[e, f]
                if ad >= 0 and tg[e] > tg[ad] + 1:
                    tg[e] = tg[ad] + 1
                    changed += 1
        if not changed:
            return tg


def _layered(n=4, order=3, runs=1, layers=(1500.0, 3000.0, 6000.0), **kw):
    return host.build_problem(n, order, runs, layers=list(layers), seed=5, **kw)


def _lts_state(prob, e0):
    e, a = prob.zero_dofs()
    return dict(dofsE=np.ascontiguousarray(e0 if e0 is not None else e), dofsA=a,
                tDofs=np.zeros_like(e), tDofs1=np.zeros_like(e), tDofs2=np.zeros_like(e))


def _grouped(order=3, n=4, n_groups=3, **kw):
    """A layered box (slow layer on top) with its elements sorted into EDGE-V time groups."""
    base = _layered(n=n, order=order, **kw)
    dt_el = host.dt_cfl_el(base.mesh, order, base.rho, base.lam, base.mu)
    tg = host.time_groups(base.mesh, dt_el, n_groups)
    m, perm, gf = host.sort_by_groups(base.mesh, tg)
    prob = _layered(n=n, order=order, mesh=m, **kw)
    flags, rel = host.lts_tables(m, tg[perm])
    return prob, gf, flags, rel


def test_time_groups_follow_edge_v():
    p = _layered(n=5, jitter=0.15)
    dt_el = host.dt_cfl_el(p.mesh, p.order, p.rho, p.lam, p.mu)
    assert np.isclose(dt_el.min(), p.dt)
    for ng in (1, 2, 3, 4):
        tg = host.time_groups(p.mesh, dt_el, ng)
        assert np.array_equal(tg, _edge_v_groups(p.mesh, dt_el, ng))
        host.lts_tables(p.mesh, tg)  # raises if neighbours are more than one group apart
        # every element steps within its CFL limit
        assert np.all(dt_el.min() * 2.0 ** tg <= dt_el * (1 + 1e-12))
    assert len(np.unique(tg)) >= 3


def test_sort_by_groups():
    p = _layered(n=4)
    dt_el = host.dt_cfl_el(p.mesh, p.order, p.rho, p.lam, p.mu)
    tg = host.time_groups(p.mesh, dt_el, 3)
    m, perm, gf = host.sort_by_groups(p.mesh, tg)
    assert gf[0] == 0 and gf[-1] == m.n_el and np.all(np.diff(gf) >= 0)
    assert np.array_equal(np.sort(m.el_ve, axis=1), np.sort(p.mesh.el_ve[perm], axis=1))
    tg2 = host.time_groups(m, host.dt_cfl_el(m, p.order, p.rho[perm], p.lam[perm], p.mu[perm]), 3)
    assert np.array_equal(tg2, tg[perm]) and np.all(np.diff(tg2.astype(int)) >= 0)


def test_one_group_is_gts():
    prob = _layered(n=3, order=4, n_receivers=4, source="explosive", n_steps=10)
    e0, _ = random_dofs(prob, seed=2, scale=1e-3)
    gts = OracleRun(prob, e0.copy())
    gts.step(6)
    lts = OracleRun(prob, e0.copy())
    st = _lts_state(prob, e0.copy())
    flags, rel = host.lts_tables(prob.mesh, np.zeros(prob.n_el, np.uint8))
    oracle.lts_cycles(lts.d, st, [0, prob.n_el], 0.0, prob.dt, 6, flags, rel, lts.recv, lts.src)
    # times are t + k dt here and repeated additions in the GTS run
    assert rel_l2(st["dofsE"], gts.state["dofsE"]) < 1e-13
    assert rel_l2(lts.recv["buf"], gts.recv["buf"]) < 1e-13


def _plane_wave_errors(order, n, ncyc=12):
    """L2 errors against the exact plane wave of GTS (dt), GTS (2 dt) and LTS with the upper half of a
    periodic box in group 1 (2 dt) and the lower half in group 0 (dt); dt = half the CFL step."""
    ext, P = 1e4, host.FACE_PERIODIC
    prob = host.build_problem(n, order, 1, ext=ext, seed=5, n_receivers=0, source=None, bc_top=P, bc_sides=P)
    tg = (prob.mesh.centroids()[:, 2] > ext / 2).astype(np.uint8)
    assert np.all(np.diff(tg.astype(int)) >= 0)  # box elements are ordered by z
    gf = np.searchsorted(tg, [0, 1, 2]).astype(np.int64)
    flags, rel = host.lts_tables(prob.mesh, tg)
    fn = host.plane_wave_p(prob.rho[0], prob.lam[0], prob.mu[0], [2 * np.pi / ext, 0.0, 2 * np.pi / ext])
    e0 = host.project(prob.mesh, order, fn)
    dtf = prob.dt / 2
    t_end = ncyc * 2 * dtf

    def err(d):
        e, r = host.l2_error(prob.mesh, order, d, lambda x: fn(x, t_end))
        return np.linalg.norm(e) / np.linalg.norm(r)

    g1 = OracleRun(prob, e0.copy())
    g1.step(2 * ncyc, dt=dtf)
    g2 = OracleRun(prob, e0.copy())
    g2.step(ncyc, dt=2 * dtf)
    lt = OracleRun(prob, e0.copy())
    st = _lts_state(prob, e0.copy())
    oracle.lts_cycles(lt.d, st, gf, 0.0, dtf, ncyc, flags, rel)
    return err(g1.state["dofsE"]), err(g2.state["dofsE"]), err(st["dofsE"]), rel_l2(st["dofsE"], g1.state["dofsE"])


def test_two_groups_plane_wave_accuracy_and_convergence():
    e1, e2, el, d = _plane_wave_errors(4, 4)
    assert min(e1, e2) * 0.98 <= el <= max(e1, e2) * 1.02
    assert d < 0.2 * el
    f1, f2, fl, _ = _plane_wave_errors(4, 6)
    assert min(f1, f2) * 0.98 <= fl <= max(f1, f2) * 1.02
    rate = np.log(el / fl) / np.log(6 / 4)
    assert rate > 3.5, rate


def test_three_groups_layered_with_sources():
    prob, gf, flags, rel = _grouped(order=3, n=4, n_receivers=6, source="explosive", n_steps=40)
    assert len(gf) == 4 and np.all(np.diff(gf) > 0)
    assert (flags & 1).any() and (flags & 2).any()
    lts = OracleRun(prob)
    st = _lts_state(prob, None)
    oracle.lts_cycles(lts.d, st, gf, 0.0, prob.dt, 8, flags, rel, lts.recv, lts.src)
    # every group sampled every receiver at the same times
    assert np.all(lts.recv["count"] == lts.recv["count"][0]) and lts.recv["count"][0] > 0
    assert np.isfinite(st["dofsE"]).all() and np.abs(st["dofsE"]).max() > 0
