"""Uneven batches through captured CUDA graphs of two batch steps (edge_b200_batch_*), and the
launch-shape autotuner: every simulation of a batch ends where it ends when stepped alone."""
import numpy as np
import pytest

from edge_b200.batch import Batch
from edge_b200.solver import Solver
from helpers import random_dofs, rel_l2, small_problem

pytestmark = pytest.mark.gpu

CASES = [  # (order, runs, mechanisms, precision, cubes, steps, tolerance)
    (3, 1, 0, 32, 2, 3, 1e-6),
    (4, 8, 3, 32, 2, 5, 1e-6),
    (5, 16, 0, 32, 3, 2, 1e-6),
    (6, 4, 0, 32, 2, 4, 1e-6),
    (4, 1, 0, 64, 3, 6, 1e-12),
]


def _pair(order, runs, rm, prec, n, seed):
    prob = small_problem(n=n, order=order, runs=runs, rm=rm, jitter=0.1, n_steps=8, source="random",
                         n_receivers=0, seed=seed)
    e0, a0 = random_dofs(prob, seed=seed)
    out = []
    for _ in range(2):
        s = Solver(prob, precision=prec)
        s.upload_dofs(e0, a0)
        out.append(s)
    return out


def test_batch_matches_each_simulation_alone():
    pairs = [_pair(o, r, rm, p, n, 11 + i) for i, (o, r, rm, p, n, _, _) in enumerate(CASES)]
    steps = [c[5] for c in CASES]
    b = Batch([p[0] for p in pairs])
    segs = b.run(steps)
    assert len(segs) == len(set(steps))
    np.testing.assert_array_equal(b.sync(), steps)
    for (sb, sa), c, k in zip(pairs, CASES, steps):
        sa.step(k)
        eb, ab = sb.download_dofs()
        ea, aa = sa.download_dofs()
        assert rel_l2(eb, ea) < c[6], c
        if c[2]:
            assert rel_l2(ab, aa) < c[6], c
    b.close()
    for p in pairs:
        for s in p:
            s.close()


def test_batch_segments_of_fused_steps():
    """Segments of 1, 6 and 5 steps (a call's first step alone; graph pairs with and without an
    odd step left), over fused and separate-kernel contexts, then a second call and a step of each
    context on its own after it."""
    cases = [(5, 16, 0, 32, 3), (4, 8, 3, 32, 2), (3, 1, 0, 64, 2)]
    steps = [1, 7, 12]
    pairs = [_pair(o, r, rm, p, n, 31 + i) for i, (o, r, rm, p, n) in enumerate(cases)]
    b = Batch([p[0] for p in pairs])
    segs = b.run(steps)
    assert [k for _, k in segs] == [1, 6, 5]
    b.run([2, 3, 0])
    np.testing.assert_array_equal(b.sync(), [3, 10, 12])
    b.close()
    for (sb, sa), c, k in zip(pairs, cases, [3, 10, 12]):
        sb.step(1)
        sa.step(k + 1)
        eb, ab = sb.download_dofs()
        ea, aa = sa.download_dofs()
        tol = 1e-12 if c[3] == 64 else 1e-6
        assert rel_l2(eb, ea) < tol, c
        if c[2]:
            assert rel_l2(ab, aa) < tol, c
    for p in pairs:
        for s in p:
            s.close()


def test_batch_step_form_fixed_at_capture():
    """A context created with separate-kernel steps and switched to fused ones afterwards (no second
    face buffer) keeps separate steps in the batch; a context switched off stays consistent too."""
    from edge_b200._lib import lib
    pairs = [_pair(5, 16, 0, 32, 2, 41), _pair(5, 16, 0, 32, 2, 43)]
    assert lib().edge_b200_set_fused(pairs[0][0]._h, 0) == 0
    b = Batch([p[0] for p in pairs])
    assert lib().edge_b200_set_fused(pairs[0][0]._h, 1) == 0
    b.run([5, 4])
    assert lib().edge_b200_set_fused(pairs[1][0]._h, 0) == 0
    b.run([2, 3])
    np.testing.assert_array_equal(b.sync(), [7, 7])
    b.close()
    for sb, sa in pairs:
        sa.step(7)
        assert rel_l2(sb.download_dofs()[0], sa.download_dofs()[0]) < 1e-6
    for p in pairs:
        for s in p:
            s.close()


def test_batch_refuses_receivers():
    from edge_b200._lib import lib
    import ctypes as C
    prob = small_problem(n=2, order=3, runs=1, n_steps=2, source=None, n_receivers=2)
    s = Solver(prob, precision=32)
    h = C.c_void_p()
    t0 = np.zeros(1)
    dt = np.array([prob.dt])
    from edge_b200._lib import ptr
    rc = lib().edge_b200_batch_create((C.c_void_p * 1)(s._h.value), 1, ptr(t0), ptr(dt), C.byref(h))
    assert rc == -5
    s.close()


@pytest.mark.parametrize("order,runs,prec", [(5, 16, 32), (3, 1, 64)])
def test_autotune_keeps_dofs_and_results(order, runs, prec):
    sa, sb = _pair(order, runs, 0, prec, 3, 5)
    e0, _ = sa.download_dofs()
    b = Batch([sa], autotune=True)
    assert len(b.caps) == 1 and all(c >= 0 for c in b.caps[0])
    e1, _ = sa.download_dofs()
    np.testing.assert_array_equal(e0, e1)  # the autotuner restored what it stepped
    b.close()
    sa.step(3)
    sb.step(3)
    np.testing.assert_array_equal(sa.download_dofs()[0], sb.download_dofs()[0])
    sa.close()
    sb.close()
