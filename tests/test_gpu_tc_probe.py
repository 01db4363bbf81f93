"""The tensor-core probe (tcgen05.mma kind::tf32 and kind::f16 with bf16 operands, operands in
shared memory, accumulator in tensor memory) reproduces the FP32 product of operands exact in its
input type, so its timings measure real work. The probe is the evidence for running the element
update's DG products on the FP32 pipe."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n,k,iters", [("tf32", 16, 8, 1), ("tf32", 64, 32, 1), ("tf32", 128, 32, 3),
                                            ("bf16", 16, 16, 1), ("bf16", 64, 64, 1), ("bf16", 128, 64, 3)])
def test_probe_matches_fp32_product(kind, n, k, iters):
    from edge_b200 import tcprobe
    assert tcprobe.check(n, k, iters, kind=kind) < 1e-5


def test_probe_rejects_allocations_that_do_not_fit_two_per_sm():
    import ctypes as C
    from edge_b200 import tcprobe
    ms = C.c_float()
    # three accumulators of 128 columns round up to 512: two CTAs per SM would wait on each other
    assert tcprobe.lib().edge_b200_probe_tc(1, 1, None, 128, 128, 32, 1, 3, 2, 0, 2, 1, C.byref(ms)) == -1
