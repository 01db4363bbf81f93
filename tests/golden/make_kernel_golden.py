"""Extract the reference's kernel golden vectors into numpy fixtures.

The reference pins its element-update kernels with seeded data and numpy-computed results embedded
in three test includes (read here as text; nothing of the reference is executed):

* ``src/impl/seismic/kernels/TimePred.test.inc`` -- ORDER 4, CK time prediction, elastic and
  2-mechanism viscoelastic (arrays at lines 245-400, raw K^T matrices in the comment at 29-94);
* ``src/impl/seismic/kernels/VolInt.test.inc`` -- ORDER 4, volume integral (arrays 226-410,
  raw K matrices at 29-94);
* ``src/impl/seismic/kernels/SurfInt.test.inc`` -- ORDER 3, local / neighbour / free-surface
  surface integrals, elastic and 3-mechanism viscoelastic (arrays 216-431, raw flux matrices in
  the comment at 28-118).

Every ``float name[d0][d1]... = {...};`` initialiser and every ``l_xxx = [ ... ]`` list in the
python comment becomes one array of ``tests/golden/kernels_<name>.npz``.

Usage: python tests/golden/make_kernel_golden.py
"""
import os
import re
import sys

import numpy as np

REF = os.environ.get("EDGE_REFERENCE", os.path.abspath(os.path.join(os.path.dirname(__file__), "..", "..", "..", "reference")))
KDIR = os.path.join(REF, "src", "impl", "seismic", "kernels")
NUM = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?")


def parse(path):
    txt = open(path).read()
    out = {}
    # C initialisers
    for m in re.finditer(r"float\s+(\w+)((?:\[\d+\])+)\s*=\s*\{", txt):
        name, dims = m.group(1), [int(d) for d in re.findall(r"\[(\d+)\]", m.group(2))]
        depth, i = 1, m.end()
        while depth:
            c = txt[i]
            depth += (c == "{") - (c == "}")
            i += 1
        vals = [float(x) for x in NUM.findall(txt[m.end():i - 1])]
        assert len(vals) == int(np.prod(dims)), (name, len(vals), dims)
        out[name] = np.array(vals, dtype=np.float64).reshape(dims)
    # raw matrices in the python comment
    for m in re.finditer(r"^(l_\w+)\s*=\s*\[", txt, flags=re.M):
        name = m.group(1)
        j = txt.index("]", m.end())
        vals = [float(x) for x in NUM.findall(txt[m.end():j])]
        if len(vals) >= 16:
            out["raw_" + name[2:]] = np.array(vals, dtype=np.float64)
    return out


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    for stem in ("TimePred", "VolInt", "SurfInt"):
        arrs = parse(os.path.join(KDIR, stem + ".test.inc"))
        np.savez_compressed(os.path.join(here, f"kernels_{stem.lower()}.npz"), **arrs)
        print(stem, {k: v.shape for k, v in arrs.items()}, file=sys.stderr)
