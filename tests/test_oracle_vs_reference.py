"""The oracle's GTS step against the reference's own vanilla kernels (oracle/_ref).

The reference build drives TimePredVanilla / VolIntVanilla / SurfIntVanilla unchanged; both sides
get identical inputs (mesh, element data, DOFs) from the host setup. Skipped where the reference
checkout was never available to compile oracle/_ref.
"""
import numpy as np
import pytest

import ref as refmod
from helpers import OracleRun, random_dofs, rel_l2, small_problem


@pytest.mark.parametrize("order,runs,rm", [(3, 1, 0), (4, 1, 0), (5, 1, 0), (4, 1, 3), (4, 8, 3)])
def test_oracle_step_matches_reference_kernels(order, runs, rm):
    L = refmod.load(order, runs, rm)
    if L is None:
        pytest.skip("reference build (oracle/_ref) unavailable")
    prob = small_problem(n=2, order=order, runs=runs, rm=rm, jitter=0.15, source=None, n_receivers=0)
    e0, a0 = random_dofs(prob, seed=order + 10 * rm)
    orc = OracleRun(prob, e0, a0)
    d = prob.oracle_dict()
    st = dict(dofsE=e0.copy(), dofsA=None if a0 is None else a0.copy(),
              tDofs=np.zeros_like(e0))
    for _ in range(3):
        orc.step()
        refmod.step(L, d, st, 0.0, prob.dt)
    assert rel_l2(orc.state["dofsE"], st["dofsE"]) < 1e-13
    assert rel_l2(orc.state["tDofs"], st["tDofs"]) < 1e-13
    if rm:
        assert rel_l2(orc.state["dofsA"], st["dofsA"]) < 1e-13


@pytest.mark.parametrize("order,runs,n_groups", [(3, 1, 2), (3, 1, 3), (4, 1, 3), (4, 4, 3)])
def test_oracle_lts_matches_reference_aderdg(order, runs, n_groups):
    """The oracle's LTS work regions (summed and half-step time integrals, the "=", "<" and ">"
    gathers) against the reference's own AderDg::local / ::neigh on the same grouped mesh, DOFs and
    rate-2 schedule."""
    import oracle
    from test_lts import _grouped
    L = refmod.load_lts(order, runs)
    if L is None:
        pytest.skip("reference build (oracle/_ref) unavailable")
    prob, gf, flags, rel = _grouped(order=order, n=4, n_groups=n_groups, runs=runs, source=None, n_receivers=0)
    assert (flags & 1).any() and (flags & 2).any()
    e0, _ = random_dofs(prob, seed=3)
    d = prob.oracle_dict()
    st = dict(dofsE=e0.copy(), dofsA=None, tDofs=np.zeros_like(e0), tDofs1=np.zeros_like(e0),
              tDofs2=np.zeros_like(e0))
    oracle.lts_cycles(d, st, gf, 0.0, prob.dt, 2, flags, rel)
    ref = refmod.LtsRun(L, d, flags, rel, e0)
    oracle.lts_schedule(ref.local, ref.neigh, gf, 0.0, prob.dt, 2)
    assert np.abs(st["dofsE"] - e0).max() > 0
    assert rel_l2(st["dofsE"], ref.st["dofsE"]) < 1e-13
    for k in ("tDofs", "tDofs1", "tDofs2"):
        assert rel_l2(st[k], ref.st[k]) < 1e-13, k
