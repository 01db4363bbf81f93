"""Generate golden DG matrices for the tet4 element with the reference's own sympy code.

Runs only where the reference checkout is mounted (it imports ``tools/edge_pre``). It writes
``dg_tet_deg{D}.npz`` next to this file with the arrays that ``edge_pre.py`` writes as CSV
(``tools/edge_pre/edge_pre.py:500-565``):

* ``mass``   [B][B]      element mass matrix
* ``stiffV`` [3][B][B]   K_d * M^-1
* ``stiffT`` [3][B][B]   K_d^T * M^-1
* ``fluxL``  [4][B][F]   local face projections (premultiplied by the face mass matrix)
* ``fluxN``  [12][B][F]  neighbouring projections, vertex-major (``edge_pre.py:531-535``)
* ``fluxT``  [4][F][B]   face -> element basis, premultiplied by M^-1

The arrays are stored as float64 exactly as ``str(float(x))`` would print them (``io/ArrStr.py``).

Usage: python tests/golden/make_dg_golden.py DEG [DEG ...]
"""
import os
import sys
import types

import numpy as np

REF = os.environ.get("EDGE_REFERENCE", os.path.abspath(os.path.join(os.path.dirname(__file__), "..", "..", "..", "reference")))
sys.path.insert(0, os.path.join(REF, "tools", "edge_pre"))

# the triangle basis module imports matplotlib for plotting only; a stub suffices
_mpl = types.ModuleType("matplotlib")
_mpl.use = lambda *a, **k: None
_mpl.pyplot = types.ModuleType("matplotlib.pyplot")
_be = types.ModuleType("matplotlib.backends")
_pdf = types.ModuleType("matplotlib.backends.backend_pdf")
_pdf.PdfPages = object
sys.modules.setdefault("matplotlib", _mpl)
sys.modules.setdefault("matplotlib.pyplot", _mpl.pyplot)
sys.modules.setdefault("matplotlib.backends", _be)
sys.modules.setdefault("matplotlib.backends.backend_pdf", _pdf)

import sympy  # noqa: E402
import edge_pre.dg.basis.Tet  # noqa: E402
import edge_pre.dg.basis.Tria  # noqa: E402
import edge_pre.dg.basis.Mod  # noqa: E402
import edge_pre.types.Tet  # noqa: E402
import edge_pre.types.Tria  # noqa: E402
import edge_pre.int.Matrices  # noqa: E402


def gen(deg):
    # mirrors the tet branch of tools/edge_pre/edge_pre.py:430-560 (DG part only)
    syms_fa, basis_fa = edge_pre.dg.basis.Tria.gen(deg)
    syms_el, basis_el = edge_pre.dg.basis.Tet.gen(deg)
    syms_el, basis_el = edge_pre.dg.basis.Mod.unify(syms_fa, basis_fa, syms_el, basis_el)
    ty = edge_pre.types.Tet.Tet(deg)
    int_fa = edge_pre.types.Tria.Tria(deg).intEl(syms_fa)
    int_el = ty.intEl(syms_el)
    fa_to_fa = ty.faToFa(syms_fa)
    fa_to_el = ty.faToEl(syms_fa)

    mass = edge_pre.int.Matrices.mass(int_el, basis_el)
    stiff = edge_pre.int.Matrices.stiff(syms_el, basis_el, int_el)
    minv = mass.inv()
    stiffT = [s.transpose() * minv for s in stiff]
    stiffV = [s * minv for s in stiff]
    flux = edge_pre.int.Matrices.flux(basis_fa, basis_el, syms_fa, syms_el, int_fa, fa_to_fa, fa_to_el)
    fluxL = [m * flux[1] for m in flux[0]]
    fluxN = []
    for ve in range(len(flux[2])):
        for fa in range(len(flux[0])):
            fluxN.append(flux[0][fa] * flux[2][ve])
    fluxT = [m.transpose() * minv for m in flux[0]]

    def arr(m):
        return np.array([[float(x) for x in row] for row in m.tolist()], dtype=np.float64)

    return dict(
        mass=arr(mass),
        stiffV=np.stack([arr(m) for m in stiffV]),
        stiffT=np.stack([arr(m) for m in stiffT]),
        fluxL=np.stack([arr(m) for m in fluxL]),
        fluxN=np.stack([arr(m) for m in fluxN]),
        fluxT=np.stack([arr(m) for m in fluxT]),
    )


if __name__ == "__main__":
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for d in [int(x) for x in sys.argv[1:]]:
        mats = gen(d)
        np.savez_compressed(os.path.join(out_dir, f"dg_tet_deg{d}.npz"), **mats)
        print("wrote degree", d, {k: v.shape for k, v in mats.items()})
