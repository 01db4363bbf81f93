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
