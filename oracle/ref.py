"""ctypes bindings of the reference's own kernels compiled into oracle/_ref (test infrastructure).

``load(order, runs, rm)`` returns the library for one configuration, building it from the reference
checkout with ``oracle/ref.mk`` when it is missing and the checkout is present; ``None`` otherwise.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: $EDGE_REFERENCE, else "reference" beside this repository
REF = os.environ.get("EDGE_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
_cache = {}


def path(order, runs, rm):
    return os.path.join(HERE, "_ref", f"libedgeref_O{order}_R{runs}_M{rm}.so")


def load(order=4, runs=1, rm=0):
    key = (order, runs, rm)
    if key in _cache:
        return _cache[key]
    p = path(*key)
    if not os.path.exists(p) and os.path.isdir(os.path.join(REF, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "-f", "ref.mk", f"CFGS={order}_{runs}_{rm}"],
                       check=False, capture_output=True)
    if not os.path.exists(p):
        _cache[key] = None
        return None
    L = C.CDLL(p)
    vp = C.c_void_p
    L.ref_step_phase.argtypes = [C.c_int, C.c_long, C.c_double] + [vp] * 13
    L.ref_series_int.restype = C.c_double
    L.ref_series_int.argtypes = [C.c_double, C.c_double, C.c_long, vp, C.c_double, C.c_double]
    L.ref_star.argtypes = [C.c_double] * 3 + [vp, vp]
    L.ref_trafo.argtypes = [vp] * 5
    L.ref_fs.argtypes = [C.c_double] * 6 + [vp] * 3 + [C.c_int, vp, vp]
    L.ref_frequencies.argtypes = [C.c_int, C.c_double, C.c_double, vp]
    L.ref_locate_eval.argtypes = [vp] * 5
    _cache[key] = L
    return L


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def step(L, prob, state, t, dt, src_apply=None):
    """One GTS step with the reference kernels: local, then src_apply(state) (sources), then neigh."""
    args = [prob["starE"], prob.get("starA"), prob.get("srcA"), prob.get("omega"), prob["fsE"],
            prob.get("fsA"), prob["elFaEl"], prob["fIdElFaEl"], prob["vIdElFaEl"], prob["faType"],
            state["dofsE"], state.get("dofsA"), state["tDofs"]]
    rc = L.ref_step_phase(0, prob["nEl"], dt, *[_p(a) for a in args])
    assert rc == 0
    if src_apply is not None:
        src_apply(state)
    rc = L.ref_step_phase(1, prob["nEl"], dt, *[_p(a) for a in args])
    assert rc == 0


def lts_path(order, runs):
    return os.path.join(HERE, "_ref", f"libedgeref_lts_O{order}_R{runs}.so")


def load_lts(order=3, runs=1):
    """The reference's AderDg class (local / neigh with the LTS branches, elastic) for one
    configuration, built from the reference checkout when missing; None otherwise."""
    key = ("lts", order, runs)
    if key in _cache:
        return _cache[key]
    p = lts_path(order, runs)
    if not os.path.exists(p) and os.path.isdir(os.path.join(REF, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "-f", "ref.mk", f"LTS_CFGS={order}_{runs}", f"_ref/libedgeref_lts_O{order}_R{runs}.so"],
                       check=False, capture_output=True)
    if not os.path.exists(p):
        _cache[key] = None
        return None
    L = C.CDLL(p)
    vp = C.c_void_p
    L.ref_lts_setup.argtypes = [C.c_long] + [vp] * 11
    L.ref_lts_local.argtypes = [C.c_long, C.c_long, C.c_int, C.c_double, C.c_double, vp]
    L.ref_lts_neigh.argtypes = [C.c_long, C.c_long, C.c_int, vp]
    _cache[key] = L
    return L


class LtsRun:
    """The reference's AderDg::local / ::neigh on one mesh with its LTS relations; state arrays
    (dofsE, tDofs, tDofs1, tDofs2, each [nEl][9][B][R]) are held here and updated in place."""

    def __init__(self, L, prob, flags, rel, dofsE):
        self.L = L
        self.st = dict(dofsE=np.ascontiguousarray(dofsE, np.float64))
        for k in ("tDofs", "tDofs1", "tDofs2"):
            self.st[k] = np.zeros_like(self.st["dofsE"])
        self.keep = [np.ascontiguousarray(prob[k]) for k in ("starE", "fsE", "elFaEl", "fIdElFaEl", "vIdElFaEl",
                                                             "faType")]
        self.keep += [np.ascontiguousarray(flags, np.uint8), np.ascontiguousarray(rel, np.uint8)]
        rc = L.ref_lts_setup(prob["nEl"], *[_p(a) for a in self.keep],
                             *[_p(self.st[k]) for k in ("tDofs", "tDofs1", "tDofs2")])
        assert rc == 0

    def local(self, first, n, first_ts, t, dt):
        assert self.L.ref_lts_local(first, n, 1 if first_ts else 0, t, dt, _p(self.st["dofsE"])) == 0

    def neigh(self, first, n, first_ts):
        assert self.L.ref_lts_neigh(first, n, 1 if first_ts else 0, _p(self.st["dofsE"])) == 0
