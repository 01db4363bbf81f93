"""Device element update on an ingested (gmsh, renumbered, Z-order reordered) mesh vs the oracle."""
import os

import numpy as np
import pytest

from edge_b200 import gmsh, host
from edge_b200.solver import Solver
from helpers import OracleRun, random_dofs, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [3, 5])
def test_fp64_on_gmsh_mesh_matches_oracle(tmp_path, order):
    box = host.Mesh.box(4, (1e4,) * 3, jitter=0.2, seed=21)
    bf_ve, tag = box.boundary_faces()
    rng = np.random.default_rng(2)
    vperm = rng.permutation(box.n_ve)
    inv = np.argsort(vperm)
    path = os.path.join(tmp_path, "mesh.msh")
    gmsh.write_msh(path, box.ve[vperm], inv[box.el_ve][rng.permutation(box.n_el)], inv[bf_ve], tag)
    m = host.Mesh.from_gmsh(path)
    prob = host.build_problem(4, order, 1, seed=21, n_receivers=6, source="random", n_steps=20, mesh=m)
    e0, _ = random_dofs(prob, seed=3, scale=1e-3)
    ref = OracleRun(prob, e0.copy())
    ref.step(20)
    s = Solver(prob, precision=64)
    try:
        s.upload_dofs(e0)
        s.step(20)
        e, _ = s.download_dofs()
        buf, _, _ = s.receivers()
    finally:
        s.close()
    assert rel_l2(e, ref.state["dofsE"]) < 1e-12
    assert rel_l2(buf, ref.recv["buf"]) < 1e-12
