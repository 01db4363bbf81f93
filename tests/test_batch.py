"""Host logic of uneven batches (edge_b200/batch.py): the segments of a batch run."""
import numpy as np
import pytest

from edge_b200.batch import schedule


def test_schedule_takes_every_simulation_through_its_steps():
    n = [5, 2, 0, 9, 5]
    segs = schedule(n)
    done = np.zeros(len(n), np.int64)
    for active, k in segs:
        assert k > 0 and active.any()
        done[active] += k
    np.testing.assert_array_equal(done, n)
    # a segment ends exactly when a simulation finishes: one segment per distinct positive length
    assert len(segs) == len({x for x in n if x > 0})
    # the active sets only shrink
    for (a0, _), (a1, _) in zip(segs, segs[1:]):
        assert np.all(a0 >= a1)


def test_schedule_edge_cases():
    assert schedule([]) == []
    assert schedule([0, 0]) == []
    segs = schedule([3])
    assert len(segs) == 1 and segs[0][1] == 3
    with pytest.raises(ValueError):
        schedule([1, -1])


def test_merged_family_layout():
    """Merging simulations of one configuration family (edge_b200.merged.merge): element ranges
    padded to whole kernel groups, most steps first, connectivity shifted into each range, padding
    elements without faces or data, one time step per group and one clock per source."""
    from edge_b200.merged import merge
    from helpers import small_problem
    probs = [small_problem(n=n, order=4, runs=8, jitter=j, seed=30 + i, source="random", n_receivers=0)
             for i, (n, j) in enumerate([(2, 0.0), (3, 0.1), (2, 0.2)])]
    steps = [4, 9, 6]
    prob, info = merge(probs, steps)
    E = 32 // 8
    assert info["perm"] == [1, 2, 0] and info["steps"] == [9, 6, 4]
    off = info["offsets"]
    assert (off % E == 0).all() and off[-1] == prob.n_el
    ef = prob.mesh.el_fa_el
    for k, i in enumerate(info["perm"]):
        n = probs[i].n_el
        loc = ef[off[k]:off[k] + n]
        assert np.array_equal(np.where(loc >= 0, loc - off[k], -1), probs[i].mesh.el_fa_el)
        assert ((loc < 0) | ((loc >= off[k]) & (loc < off[k] + n))).all()
        assert (ef[off[k] + n:off[k + 1]] == -1).all()
        assert (prob.mesh.el_fa_type[off[k] + n:off[k + 1]] == 2).all()
        assert not prob.starE[off[k] + n:off[k + 1]].any()
        assert np.array_equal(prob.fsE[:, off[k]:off[k] + n], probs[i].fsE)
        assert (info["group_dt"][off[k] // E:off[k + 1] // E] == probs[i].dt).all()
    src = prob.sources
    assert src["n"] == sum(p.sources["n"] for p in probs)
    assert (np.diff(src["el"]) >= 0).all()
    assert len(info["clk0"]) == src["n"] and set(info["clk_dt"]) == {p.dt for p in probs}
