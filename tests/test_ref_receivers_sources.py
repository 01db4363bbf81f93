"""Receivers and point sources pinned to the reference's own code.

* Basis values: the host setup locates receivers and sources in their elements and evaluates the
  element basis there (edge_setup_locate); the reference does the same with
  linalg::Mappings::phyToRefTet4 and dg::Basis::evalBasis (Receivers.cpp:127-143,
  PointSources.hpp:458-495, sources also scaled by the inverse mass matrix and divided by the
  Jacobian determinant), compiled unchanged into oracle/_ref and called through ref_locate_eval.
* Sampling schedule: the reference samples a receiver element while its first receiver's next time
  lies in (t - TOL, t + dt - TOL) (Receivers::getRecvTimeRel, Receivers.cpp:235-248), at the
  relative time |time - t|, writes every receiver of the element and advances each one's time by
  the sampling period (writeRecvAll, Receivers.cpp:250-290), as long as the loop of
  AderDg::local (AderDg.hpp:475-495) finds another time in the step. Restated here step by step and
  compared with the oracle's receiver buffers (the device's sample times equal the oracle's bit for
  bit in tests/test_gpu_parity.py).
"""
import numpy as np
import pytest

import ref
from edge_b200 import dgmat, host
from helpers import OracleRun, small_problem

TOL_TIME = 1e-9  # TOL.TIME of a PP_PRECISION=64 build (constants.hpp:289-300)


def _points(mesh, n, rng):
    """n points strictly inside random elements: (element, physical point)."""
    el = rng.integers(0, mesh.n_el, n)
    w = rng.uniform(0.1, 1.0, (n, 4))
    w /= w.sum(axis=1, keepdims=True)
    crd = mesh.el_ve_crds()[el]  # [n][4][3]
    return el, np.einsum("nv,nvd->nd", w, crd)


@pytest.mark.parametrize("order", [3, 4, 5, 6])
def test_receiver_and_source_basis_match_reference(order):
    L = ref.load(order, 1, 0)
    if L is None:
        pytest.skip("reference kernels not built (no reference checkout)")
    p = small_problem(n=3, order=order, runs=1, jitter=0.2, seed=11, n_steps=2, source=None, n_receivers=0)
    rng = np.random.default_rng(order)
    el0, pts = _points(p.mesh, 40, rng)
    el, refc, basis = host.locate(p.mesh, order, pts, source=False)
    _, _, basis_src = host.locate(p.mesh, order, pts, source=True)
    assert np.array_equal(el, el0)
    minv = np.array([float(x) for x in dgmat.exact_matrices(order)["massInv"]])
    crd = p.mesh.el_ve_crds()
    for i in range(len(pts)):
        ves = np.ascontiguousarray(crd[el[i]].T)  # [3 dims][4 vertices]
        x = np.ascontiguousarray(pts[i])
        r_ref, r_basis, det = np.zeros(3), np.zeros(host.n_modes(order)), np.zeros(1)
        L.ref_locate_eval(ref._p(ves), ref._p(x), ref._p(r_ref), ref._p(r_basis), ref._p(det))
        np.testing.assert_allclose(refc[i], r_ref, rtol=0, atol=1e-12)
        np.testing.assert_allclose(basis[i], r_basis, rtol=0, atol=1e-11 * np.abs(r_basis).max())
        want_src = r_basis * minv / det[0]
        np.testing.assert_allclose(basis_src[i], want_src, rtol=0, atol=1e-11 * np.abs(want_src).max())


def _schedule(el, t_first, period, dt, n_steps):
    """Sample times per receiver by the reference's rule (receivers sorted by element)."""
    n = len(el)
    time = np.full(n, t_first)
    out = [[] for _ in range(n)]
    t = 0.0
    for _ in range(n_steps):
        i = 0
        while i < n:
            j = i
            while j < n and el[j] == el[i]:
                j += 1
            while True:  # AderDg.hpp:475-495
                tr = time[i]
                if not (tr > t - TOL_TIME and tr < t + dt - TOL_TIME):  # getRecvTimeRel
                    break
                for r in range(i, j):  # writeRecvAll: every receiver of the element
                    out[r].append(time[r])
                    time[r] += period
            i = j
        t += dt
    return out


@pytest.mark.parametrize("period_over_dt", [0.37, 1.0, 2.5])
def test_receiver_schedule_follows_reference_rule(period_over_dt):
    p = small_problem(n=2, order=3, runs=1, jitter=0.1, seed=4, n_steps=12, source="explosive", n_receivers=0)
    rng = np.random.default_rng(5)
    el0, pts = _points(p.mesh, 6, rng)
    pts = np.concatenate([pts, pts[:2] + 1e-3])  # two elements with two receivers each
    period = period_over_dt * p.dt
    p.receivers = host.make_receivers(p.mesh, p.order, pts, period, 12 * p.dt, t_first=0.3 * p.dt)
    r = p.receivers
    run = OracleRun(p)
    run.step(12)
    want = _schedule(r["el"], r["t_first"], period, p.dt, 12)
    assert len(set(r["el"].tolist())) < r["n"]  # shared elements present
    for i in range(r["n"]):
        k = int(run.recv["count"][i])
        assert k == len(want[i]) and k > 0
        assert np.array_equal(run.recv["buftime"][i, :k], np.array(want[i]))
