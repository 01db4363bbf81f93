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
    err = {}
    for mode, name in ((1, "tf32"), (2, "3xtf32"), (3, "bf16"), (4, "3xbf16")):
        b, d = _run(mode, prob)
        err[name] = (rel_l2(b, ref_b), rel_l2(d, ref_d))
    print("; ".join(f"{k}: receivers {e:.3e}, DOFs {d:.3e}" for k, (e, d) in err.items()))
    # the tf32 split recovers FP32-level products; plain tf32 is three orders of magnitude coarser
    assert err["3xtf32"][0] < 1e-5 and err["3xtf32"][1] < 1e-5
    assert err["tf32"][0] > 100 * err["3xtf32"][0]
    # plain bf16 is coarser than tf32 (8 against 11 significant bits); the bf16 split keeps about
    # 16 bits, between the two
    assert err["bf16"][0] > err["tf32"][0]
    assert err["3xtf32"][0] < err["3xbf16"][0] < err["tf32"][0]
