"""The tensor-core probe (csrc/probe/tc_probe.cu, libedge_b200_probe.so): tcgen05.mma kind::tf32
at the shapes the element update's DG products would have, checked against the FP32 product and
timed per instruction. Evidence for the choice of the FP32 pipe for those products; not part of the
element update."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "libedge_b200_probe.so")
        if not os.path.exists(path):
            raise RuntimeError("libedge_b200_probe.so is not built (python -m edge_b200.build)")
        _lib = C.CDLL(path)
        vp = C.c_void_p
        _lib.edge_b200_probe_tc.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            vp, C.POINTER(C.c_float)]
    return _lib


def _tf32(x):
    import torch
    return (x.view(torch.int32) & ~0x1FFF).view(torch.float32)


def check(n, k, iters=1, seed=0):
    """Relative max error of D = iters * A B^T (A [128][k], B [n][k], tf32-exact inputs) from one
    CTA of the probe against the float64 product."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = _tf32(torch.randn(128, k, device="cuda", generator=g))
    B = _tf32(torch.randn(n, k, device="cuda", generator=g))
    D = torch.full((128, n), float("nan"), device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    ms = C.c_float()
    rc = lib().edge_b200_probe_tc(A.data_ptr(), B.data_ptr(), D.data_ptr(), 128, n, k, iters, 1, 1, st.data_ptr(),
                                  C.byref(ms))
    if rc != 0 or int(st.item()) != 0:
        raise RuntimeError(f"probe failed: rc {rc}, status {int(st.item())}")
    ref = iters * (A.double() @ B.double().T)
    return float(((D.double() - ref).abs().max() / ref.abs().max()).item())


def time_shape(n, k=32, iters=4096, blocks=148, acc=1):
    """(milliseconds, instructions per CTA) for `blocks` CTAs each issuing iters x k / 8 MMAs of
    128 x n x 8 (tf32) round robin into `acc` independent accumulators."""
    import torch
    A = torch.randn(128, k, device="cuda")
    B = torch.randn(n, k, device="cuda")
    st = torch.zeros(blocks, dtype=torch.int32, device="cuda")
    ms = C.c_float()
    for _ in range(2):  # the first launch sets the shared-memory attribute and warms the clocks
        rc = lib().edge_b200_probe_tc(A.data_ptr(), B.data_ptr(), None, 128, n, k, iters, acc, blocks,
                                      st.data_ptr(), C.byref(ms))
        if rc != 0 or int(st.sum().item()) != 0:
            raise RuntimeError(f"probe failed: rc {rc}")
    return ms.value, iters * (k // 8) * acc
