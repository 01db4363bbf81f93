"""Error of the fused FP32 path stated against the plain FP64 path, run by run, on the device.

A fused FP32 context advances R runs together; each run r is also advanced alone on the FP64 path
(one run, the same mesh, element data and receivers, only run r's point sources), and the receiver
time series of the two are compared by relative L2 over all receivers, samples and the nine
quantities. The FP64 path itself matches the CPU restatement of EDGE's kernels to 1e-12, so this is
the FP32 error against the FP64 reference at sizes where the CPU would take hours. Mode-0
coefficients of the final DOFs (the wave field EDGE writes) are compared the same way.
"""
import time

import numpy as np

from .solver import Solver


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def fused_vs_plain(prob, n_steps, device=0, runs=None):
    """Runs prob for n_steps on the FP32 fused path and each of its runs (or those listed in
    ``runs``) on the FP64 single-run path; returns per-run receiver and wave-field rel-L2."""
    t0 = time.perf_counter()
    s32 = Solver(prob, precision=32, device=device)
    e0, a0 = prob.zero_dofs(np.float32)
    s32.upload_dofs(e0, a0)
    del e0, a0
    s32.step(n_steps)
    b32, t32, c32 = s32.receivers()
    w32 = s32.wavefield()
    s32.close()
    k = int(c32[0])
    runs = list(range(prob.runs)) if runs is None else list(runs)
    recv, wave, recv_max = [], [], []
    for r in runs:
        p1 = prob.single_run(r)
        s64 = Solver(p1, precision=64, device=device)
        z, za = p1.zero_dofs()
        s64.upload_dofs(z, za)
        del z, za
        s64.step(n_steps)
        b64, t64, c64 = s64.receivers()
        w64 = s64.wavefield()
        s64.close()
        if int(c64[0]) != k or not np.array_equal(t32[:, :k], t64[:, :k]):
            raise RuntimeError(f"run {r}: FP32 and FP64 receivers sampled at different times")
        recv.append(rel_l2(b32[:, :k, :, r], b64[:, :k, :, 0]))
        recv_max.append(max(rel_l2(b32[i, :k, :, r], b64[i, :k, :, 0]) for i in range(b32.shape[0])))
        wave.append(rel_l2(w32[r], w64[0]))
    return {"tets": prob.n_el, "order": prob.order, "runs": prob.runs, "mechanisms": prob.rm, "steps": n_steps,
            "receivers": int(b32.shape[0]), "samples_per_receiver": k, "runs_checked": runs,
            "receiver_rel_l2_per_run": recv, "receiver_rel_l2_max": max(recv),
            "worst_single_receiver_rel_l2_per_run": recv_max,
            "wavefield_rel_l2_per_run": wave, "wavefield_rel_l2_max": max(wave),
            "seconds": time.perf_counter() - t0}


class _DeviceArray:
    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape, "typestr": typestr, "version": 3}


def _row_pad(n, precision):
    per = 4 if precision == 32 else 2  # rows padded to 16 bytes
    return (n + per - 1) // per * per


def dofs_fused_vs_plain(prob, n_steps, device=0, runs=None, seed=7, chunks=4):
    """The same check on the DOFs themselves, independent of where waves have travelled: seeded
    random DOFs (elastic and anelastic, N(0, 1) in every mode of every element) are written into
    the FP32 fused context's device rows and, run by run, into an FP64 single-run context; after
    n_steps GTS steps (no sources) the relative L2 of each run's DOFs against its FP64 run is
    reported, over the whole mesh and over `chunks` contiguous element ranges."""
    import torch
    t0 = time.perf_counter()
    B, R, rm, ne = prob.B, prob.runs, prob.rm, prob.n_el
    bare = type(prob)(order=prob.order, runs=R, rm=rm, mesh=prob.mesh, rho=prob.rho, lam=prob.lam, mu=prob.mu,
                      starE=prob.starE, fsE=prob.fsE, dt=prob.dt, starA=prob.starA, srcA=prob.srcA, fsA=prob.fsA,
                      omega=prob.omega, name=prob.name + "_dofs")
    dev = torch.device("cuda", device)
    s32 = Solver(bare, precision=32, device=device)
    out = {"tets": ne, "steps": n_steps, "runs_checked": [], "dof_rel_l2_per_run": [],
           "dof_rel_l2_per_run_per_range": []}
    try:
        G32 = _row_pad(B, 32)
        pe, pa, _ = s32.device_ptrs()
        rows = [torch.as_tensor(_DeviceArray(pe, (ne, 9, R, G32), "<f4"), device=dev)]
        if rm:
            rows.append(torch.as_tensor(_DeviceArray(pa, (ne, 6 * rm, R, G32), "<f4"), device=dev))
        g = torch.Generator(device=dev).manual_seed(seed)
        for x in rows:
            x.normal_(generator=g)
            x[..., B:] = 0
        init = [x[..., :B].to(torch.float64) for x in rows]
        s32.step(n_steps, t=0.0)
        s32.sync()
        res32 = [x[..., :B].clone() for x in rows]
    finally:
        s32.close()
    G64 = _row_pad(B, 64)
    bounds = [ne * i // chunks for i in range(chunks + 1)]
    for r in (range(R) if runs is None else runs):
        p1 = type(prob)(order=prob.order, runs=1, rm=rm, mesh=prob.mesh, rho=prob.rho, lam=prob.lam, mu=prob.mu,
                        starE=prob.starE, fsE=prob.fsE, dt=prob.dt, starA=prob.starA, srcA=prob.srcA, fsA=prob.fsA,
                        omega=prob.omega, name=prob.name + f"_dofs_run{r}")
        s64 = Solver(p1, precision=64, device=device)
        try:
            pe, pa, _ = s64.device_ptrs()
            rows64 = [torch.as_tensor(_DeviceArray(pe, (ne, 9, 1, G64), "<f8"), device=dev)]
            if rm:
                rows64.append(torch.as_tensor(_DeviceArray(pa, (ne, 6 * rm, 1, G64), "<f8"), device=dev))
            for x, x0 in zip(rows64, init):
                x.zero_()
                x[:, :, 0, :B] = x0[:, :, r, :]
            s64.step(n_steps, t=0.0)
            s64.sync()
            num = torch.zeros(chunks, dtype=torch.float64, device=dev)
            den = torch.zeros(chunks, dtype=torch.float64, device=dev)
            for x, x32 in zip(rows64, res32):
                ref = x[:, :, 0, :B]
                d = x32[:, :, r, :].to(torch.float64) - ref
                for c in range(chunks):
                    lo, hi = bounds[c], bounds[c + 1]
                    num[c] += (d[lo:hi] ** 2).sum()
                    den[c] += (ref[lo:hi] ** 2).sum()
        finally:
            s64.close()
        out["runs_checked"].append(r)
        out["dof_rel_l2_per_run"].append(float((num.sum() / den.sum()).sqrt()))
        out["dof_rel_l2_per_run_per_range"].append([float(v) for v in (num / den).sqrt()])
    out["dof_rel_l2_max"] = max(out["dof_rel_l2_per_run"])
    out["seconds"] = time.perf_counter() - t0
    del rows, init, res32
    torch.cuda.empty_cache()
    return out
