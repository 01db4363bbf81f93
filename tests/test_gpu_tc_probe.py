"""The tensor-core probe (tcgen05.mma kind::tf32, operands in shared memory, accumulator in tensor
memory) reproduces the FP32 product of tf32-exact operands, so its timings measure real work. The
probe is the evidence for running the element update's DG products on the FP32 pipe."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,k,iters", [(16, 8, 1), (64, 32, 1), (128, 32, 3)])
def test_probe_matches_fp32_product(n, k, iters):
    from edge_b200 import tcprobe
    assert tcprobe.check(n, k, iters) < 1e-5
