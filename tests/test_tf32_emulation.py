"""What tensor-core arithmetic would do to the results, measured on the oracle: the products with
the global DG matrices (stiffness, fluxL, fluxT: the tensor-core candidates) with tf32 operands,
and with the three-product tf32 split, everything else exact, against the FP64 oracle on the
receiver time series and the DOFs after 200 steps (order 5, point source, 8 receivers). The FP32
element update stays within 1e-4 at the receivers (and ~1e-6 in the at-size GPU checks)."""
import numpy as np

import oracle
from helpers import OracleRun, rel_l2, small_problem


def _run(mode, prob):
    oracle.set_mm_mode(mode)
    try:
        r = OracleRun(prob)
        r.step(200)
    finally:
        oracle.set_mm_mode(0)
    k = int(r.recv["count"][0])
    return r.recv["buf"][:, :k], r.state["dofsE"]


def test_tf32_products_error_against_fp64():
    prob = small_problem(n=3, order=5, runs=1, jitter=0.1, n_steps=200, source="explosive", n_receivers=8)
    ref_b, ref_d = _run(0, prob)
    assert np.abs(ref_b).max() > 0
    one_b, one_d = _run(1, prob)
    three_b, three_d = _run(2, prob)
    e1, e3 = rel_l2(one_b, ref_b), rel_l2(three_b, ref_b)
    d1, d3 = rel_l2(one_d, ref_d), rel_l2(three_d, ref_d)
    print(f"tf32 products: receivers {e1:.3e}, DOFs {d1:.3e}; 3xtf32: receivers {e3:.3e}, DOFs {d3:.3e}")
    # the split recovers FP32-level products; plain tf32 is three orders of magnitude coarser
    assert e3 < 1e-5 and d3 < 1e-5
    assert e1 > 100 * e3
