"""The tensor-core probe (csrc/probe/tc_probe.cu, libedge_b200_probe.so): tcgen05.mma kind::tf32
and kind::f16 (bf16 operands) at the shapes the element update's DG products would have, checked
against the FP32 product and timed per instruction with one or two issuing CTAs per SM. Evidence for
the choice of the FP32 pipe for those products; not part of the element update."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
KINDS = {"tf32": 0, "bf16": 1}
K_INSTR = {"tf32": 8, "bf16": 16}  # reduction length of one instruction


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "libedge_b200_probe.so")
        if not os.path.exists(path):
            raise RuntimeError("libedge_b200_probe.so is not built (python -m edge_b200.build)")
        _lib = C.CDLL(path)
        vp = C.c_void_p
        _lib.edge_b200_probe_tc.argtypes = [vp, vp, vp] + [C.c_int] * 8 + [vp, C.POINTER(C.c_float)]
    return _lib


def _round(x, kind):
    """x (float32) rounded the way the instruction reads it: tf32 drops the low 13 bits of the
    mantissa (exact inputs: already zero), bf16 rounds to nearest even."""
    import torch
    if kind == "tf32":
        return (x.view(torch.int32) & ~0x1FFF).view(torch.float32)
    return x.to(torch.bfloat16).to(torch.float32)


def check(n, k, iters=1, seed=0, kind="tf32"):
    """Relative max error of D = iters * A B^T (A [128][k], B [n][k], inputs exact in the kind's
    type) from one CTA of the probe against the float64 product."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = _round(torch.randn(128, k, device="cuda", generator=g), kind)
    B = _round(torch.randn(n, k, device="cuda", generator=g), kind)
    D = torch.full((128, n), float("nan"), device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    ms = C.c_float()
    rc = lib().edge_b200_probe_tc(A.data_ptr(), B.data_ptr(), D.data_ptr(), 128, n, k, iters, 1, 1, KINDS[kind], 1,
                                  st.data_ptr(), C.byref(ms))
    if rc != 0 or int(st.item()) != 0:
        raise RuntimeError(f"probe failed: rc {rc}, status {int(st.item())}")
    ref = iters * (A.double() @ B.double().T)
    return float(((D.double() - ref).abs().max() / ref.abs().max()).item())


def time_shape(n, iters=4096, sms=148, acc=1, kind="tf32", per_sm=1):
    """(milliseconds, instructions per SM) for sms x per_sm CTAs each issuing iters x 4 MMAs of
    128 x n x K (K = 8 for tf32, 16 for bf16) round robin into `acc` independent accumulators."""
    import torch
    k = 4 * K_INSTR[kind]
    A = torch.randn(128, k, device="cuda")
    B = torch.randn(n, k, device="cuda")
    blocks = sms * per_sm
    st = torch.zeros(blocks, dtype=torch.int32, device="cuda")
    ms = C.c_float()
    for _ in range(2):  # the first launch sets the shared-memory attribute and warms the clocks
        rc = lib().edge_b200_probe_tc(A.data_ptr(), B.data_ptr(), None, 128, n, k, iters, acc, blocks, KINDS[kind],
                                      per_sm, st.data_ptr(), C.byref(ms))
        if rc != 0 or int(st.sum().item()) != 0:
            raise RuntimeError(f"probe failed: rc {rc}")
    return ms.value, iters * 4 * acc * per_sm


if __name__ == "__main__":
    # one small timing per shape (two launches each): N = 16, the output modes of the smallest DG
    # products, and N = 128, where the tf32 pipe runs near its peak
    for n in (16, 128):
        ms, instr = time_shape(n, iters=256, acc=3)
        print(f"tf32 128x{n}x8, three accumulators: {ms:.3f} ms, {ms * 1e6 / instr:.2f} ns per instruction per SM")
