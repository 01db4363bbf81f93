"""Properties of the element update at the headline size (48^3 cubes x 6 = 663,552 tets, order 5,
16 fused runs, FP32), where the oracle would take hours: the step is linear in the DOFs (no
sources), fused runs are independent (permuting the runs permutes the results bit for bit), and
nothing overflows. Inputs are written straight into the device rows (no host copies)."""
import numpy as np
import pytest
import torch

from edge_b200 import host
from edge_b200.solver import Solver

pytestmark = pytest.mark.gpu


class _DeviceArray:
    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape, "typestr": typestr, "version": 3}


def test_headline_size_linearity_and_run_independence():
    n, order, runs = 48, 5, 16
    prob = host.build_problem(n, order, runs, seed=3343, n_receivers=0, source=None, n_steps=3)
    B = host.n_modes(order)
    GB = (B + 3) // 4 * 4
    s = Solver(prob, precision=32)
    try:
        ptr = s.device_ptrs()[0]
        rows = torch.as_tensor(_DeviceArray(ptr, (prob.n_el, 9, runs, GB), "<f4"), device="cuda")
        g = torch.Generator(device="cuda").manual_seed(7)

        def rand():
            x = torch.randn((prob.n_el, 9, runs, GB), device="cuda", generator=g) * 1e-3
            x[..., B:] = 0
            return x

        def step(x, k=2):
            rows.copy_(x)
            s.step(k, t=0.0)
            s.sync()
            return rows.clone()

        # (each array is 13.8 GB; in-place arithmetic keeps the peak near 125 GB with the solver)
        x, y = rand(), rand()
        fx, fy = step(x), step(y)
        z = x.clone().mul_(2.0).add_(y, alpha=-0.5)
        del y
        fxy = step(z)
        del z
        assert torch.isfinite(fxy).all()
        norm = fxy.norm().item()
        fxy.add_(fx, alpha=-2.0).add_(fy, alpha=0.5)
        rel = fxy.norm().item() / norm
        assert rel < 1e-5, rel
        del fxy, fy
        # permuting the fused runs permutes the results exactly
        perm = torch.randperm(runs, generator=torch.Generator().manual_seed(3)).to("cuda")
        fp = step(x[:, :, perm].contiguous())
        assert torch.equal(fp, fx[:, :, perm])
        del x, fx, fp
    finally:
        s.close()
