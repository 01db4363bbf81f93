"""ctypes bindings of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module, and only to check or time against it. It loads ``oracle/liboracle.so`` (built from
``oracle.c`` by ``oracle/Makefile``).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def _opt(a, dtype):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=dtype)
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
        _LIB = C.CDLL(path)
        _LIB.oracle_step.restype = C.c_int
        _LIB.oracle_lts_local.restype = C.c_int
        _LIB.oracle_series_int.restype = C.c_double
        _LIB.oracle_series_int.argtypes = [C.c_double, C.c_double, C.c_long, C.c_void_p, C.c_double,
                                           C.c_double, C.c_double, C.c_double]
    return _LIB


def nmodes(o):
    return o * (o + 1) * (o + 2) // 6 if o > 0 else 0


def ck(O, R, rm, dt, stiffT, starE, dofsE, starA=None, srcA=None, omega=None, dofsA=None):
    B = nmodes(O)
    der = np.zeros((O, 9, B, R))
    tE = np.zeros((9, B, R))
    tA = np.zeros((max(rm, 1), 6, B, R))
    a = [_opt(x, np.float64) for x in (stiffT, starE, starA, srcA, omega, dofsE, dofsA)]
    lib().oracle_ck(C.c_int(O), C.c_int(R), C.c_int(rm), C.c_double(dt), *[_ptr(x) for x in a],
                    _ptr(der), _ptr(tE), _ptr(tA))
    return der, tE, tA[:rm]


def eval_pred(O, R, tau, der):
    B = nmodes(O)
    pred = np.zeros((9, B, R))
    der = _opt(der, np.float64)
    lib().oracle_eval_pred(C.c_int(O), C.c_int(R), C.c_double(tau), _ptr(der), _ptr(pred))
    return pred


def volint(O, R, rm, stiffV, starE, tE, dofsE, starA=None, srcA=None, omega=None, tA=None, dofsA=None):
    dofsE = np.array(dofsE, dtype=np.float64, order="C")
    dofsA = None if dofsA is None else np.array(dofsA, dtype=np.float64, order="C")
    a = [_opt(x, np.float64) for x in (stiffV, starE, starA, srcA, omega, tE, tA)]
    lib().oracle_volint(C.c_int(O), C.c_int(R), C.c_int(rm), *[_ptr(x) for x in a], _ptr(dofsE),
                        _ptr(dofsA))
    return dofsE, dofsA


def surf_local(O, R, rm, fluxL, fluxT, fsE4, tE, dofsE, fsA4=None, omega=None, dofsA=None):
    dofsE = np.array(dofsE, dtype=np.float64, order="C")
    dofsA = None if dofsA is None else np.array(dofsA, dtype=np.float64, order="C")
    a = [_opt(x, np.float64) for x in (fluxL, fluxT, fsE4, fsA4, omega, tE)]
    lib().oracle_surf_local(C.c_int(O), C.c_int(R), C.c_int(rm), *[_ptr(x) for x in a],
                            _ptr(dofsE), _ptr(dofsA))
    return dofsE, dofsA


def surf_neigh(O, R, rm, fa, vId, fId, fluxL, fluxN, fluxT, fsE, tNe, dofsE, fsA=None, upA=None):
    dofsE = np.array(dofsE, dtype=np.float64, order="C")
    B = nmodes(O)
    upA = np.zeros((6, B, R)) if upA is None else np.array(upA, dtype=np.float64, order="C")
    a = [_opt(x, np.float64) for x in (fluxL, fluxN, fluxT, fsE, fsA, tNe)]
    lib().oracle_surf_neigh(C.c_int(O), C.c_int(R), C.c_int(rm), C.c_int(fa), C.c_int(vId),
                            C.c_int(fId), *[_ptr(x) for x in a], _ptr(dofsE), _ptr(upA))
    return dofsE, upA


def series_int(dx, x0, vals, x1, x2, na=0.0, tol=1e-9):
    vals = _opt(vals, np.float64)
    return lib().oracle_series_int(dx, x0, len(vals), _ptr(vals), x1, x2, na, tol)


def step(prob, state, t, dt, recv=None, src=None, tol_time=1e-9):
    """One GTS step of the oracle. ``prob`` is a dict of the element data (see oracle.c),
    ``state`` holds dofsE/dofsA/tDofs (updated in place), ``recv``/``src`` the optional
    receiver and source tables (updated in place where the C code writes)."""
    O, R, rm = prob["order"], prob["runs"], prob["rm"]
    nEl = prob["nEl"]
    L = lib()
    f64 = lambda k: _ptr(prob[k]) if prob.get(k) is not None else None
    if recv is None:
        recv = dict(n=0, el=None, basis=None, time=None, period=1.0, maxbuf=0, buf=None,
                    buftime=None, count=None)
    if src is None:
        src = dict(n=0)
    rc = L.oracle_step(
        C.c_int(O), C.c_int(R), C.c_int(rm), C.c_long(nEl), C.c_double(t), C.c_double(dt),
        f64("stiffT"), f64("stiffV"), f64("fluxL"), f64("fluxN"), f64("fluxT"), f64("starE"),
        f64("starA"), f64("srcA"), f64("omega"), f64("fsE"), f64("fsA"), _ptr(prob["elFaEl"]),
        _ptr(prob["fIdElFaEl"]), _ptr(prob["vIdElFaEl"]), _ptr(prob["faType"]),
        _ptr(state["dofsE"]), _ptr(state.get("dofsA")), _ptr(state["tDofs"]),
        C.c_int(recv["n"]), _ptr(recv["el"]), _ptr(recv["basis"]), _ptr(recv["time"]),
        C.c_double(recv["period"]), C.c_int(recv["maxbuf"]), _ptr(recv["buf"]),
        _ptr(recv["buftime"]), _ptr(recv["count"]),
        C.c_int(src.get("n", 0)), _ptr(src.get("el")), _ptr(src.get("run")), _ptr(src.get("scal")),
        _ptr(src.get("bEval")), _ptr(src.get("t0")), _ptr(src.get("dt")), _ptr(src.get("tsOff")),
        _ptr(src.get("nPts")), _ptr(src.get("ts")), C.c_double(tol_time))
    if rc != 0:
        raise RuntimeError("oracle_step failed (receiver buffer full?)")


def _recv_args(recv):
    if recv is None:
        recv = dict(n=0, el=None, basis=None, time=None, period=1.0, maxbuf=0, buf=None, buftime=None,
                    count=None)
    return [C.c_int(recv["n"]), _ptr(recv["el"]), _ptr(recv["basis"]), _ptr(recv["time"]),
            C.c_double(recv["period"]), C.c_int(recv["maxbuf"]), _ptr(recv["buf"]), _ptr(recv["buftime"]),
            _ptr(recv["count"])]


def _src_args(src):
    src = src or dict(n=0)
    return [C.c_int(src.get("n", 0)), _ptr(src.get("el")), _ptr(src.get("run")), _ptr(src.get("scal")),
            _ptr(src.get("bEval")), _ptr(src.get("t0")), _ptr(src.get("dt")), _ptr(src.get("tsOff")),
            _ptr(src.get("nPts")), _ptr(src.get("ts"))]


def lts_local(prob, state, first, n, first_ts, t, dt, flags, recv=None, src=None, tol_time=1e-9):
    """Local step + sources of the elements [first, first+n) of one LTS time group
    (oracle_lts_local); state holds dofsE/dofsA/tDofs and the LTS buffers tDofs1/tDofs2."""
    O, R, rm = prob["order"], prob["runs"], prob["rm"]
    f64 = lambda k: _ptr(prob[k]) if prob.get(k) is not None else None
    rc = lib().oracle_lts_local(
        C.c_int(O), C.c_int(R), C.c_int(rm), C.c_long(first), C.c_long(n), C.c_int(1 if first_ts else 0),
        C.c_double(t), C.c_double(dt), f64("stiffT"), f64("stiffV"), f64("fluxL"), f64("fluxT"), f64("starE"),
        f64("starA"), f64("srcA"), f64("omega"), f64("fsE"), f64("fsA"), _ptr(flags), _ptr(state["dofsE"]),
        _ptr(state.get("dofsA")), _ptr(state["tDofs"]), _ptr(state.get("tDofs1")), _ptr(state.get("tDofs2")),
        *_recv_args(recv), *_src_args(src), C.c_double(tol_time))
    if rc != 0:
        raise RuntimeError("oracle_lts_local failed (receiver buffer full?)")


def lts_neigh(prob, state, first, n, first_ts, rel):
    """Neighbour step of the elements [first, first+n) of one LTS time group (oracle_lts_neigh)."""
    O, R, rm = prob["order"], prob["runs"], prob["rm"]
    f64 = lambda k: _ptr(prob[k]) if prob.get(k) is not None else None
    lib().oracle_lts_neigh(
        C.c_int(O), C.c_int(R), C.c_int(rm), C.c_long(first), C.c_long(n), C.c_long(prob["nEl"]),
        C.c_int(1 if first_ts else 0), f64("fluxL"), f64("fluxN"), f64("fluxT"), f64("fsE"), f64("fsA"),
        f64("omega"), _ptr(prob["elFaEl"]), _ptr(prob["fIdElFaEl"]), _ptr(prob["vIdElFaEl"]),
        _ptr(prob["faType"]), _ptr(rel), _ptr(state["tDofs"]), _ptr(state.get("tDofs1")),
        _ptr(state.get("tDofs2")), _ptr(state["dofsE"]), _ptr(state.get("dofsA")))


def lts_schedule(local, neigh, group_first, t, dt_fun, n_cycles):
    """The rate-2 order of the work regions over n_cycles steps of the largest time group: at
    fundamental step k (t_k = t + k dt_fun) every group g with k % 2^g == 0 runs
    local(lo, n, first_ts, t_k, 2^g dt_fun), then every group whose step ends runs
    neigh(lo, n, first_ts); the first step of each pair of a group (its step count even) resets the
    two-step sums (TimeGroupStatic.cpp:46-111, man_sched.inc:37-206 sequentialised)."""
    G = len(group_first) - 1
    n_fun = 1 << (G - 1)
    for c in range(n_cycles):
        for k in range(n_fun):
            kk = c * n_fun + k
            for g in range(G):
                if k % (1 << g):
                    continue
                lo, hi = int(group_first[g]), int(group_first[g + 1])
                if hi > lo:
                    local(lo, hi - lo, ((kk >> g) & 1) == 0, t + float(kk) * dt_fun, dt_fun * float(1 << g))
            for g in range(G):
                span = 1 << g
                if (k + 1) % span:
                    continue
                lo, hi = int(group_first[g]), int(group_first[g + 1])
                k0 = kk + 1 - span
                if hi > lo:
                    neigh(lo, hi - lo, ((k0 >> g) & 1) == 0)


def lts_cycles(prob, state, group_first, t, dt_fun, n_cycles, flags, rel, recv=None, src=None):
    """n_cycles steps of the largest time group with the rate-2 schedule (lts_schedule) of the
    oracle's LTS work regions."""
    lts_schedule(lambda lo, n, ft, tk, dt: lts_local(prob, state, lo, n, ft, tk, dt, flags, recv, src),
                 lambda lo, n, ft: lts_neigh(prob, state, lo, n, ft, rel), group_first, t, dt_fun, n_cycles)


# ------------------------------------------------------------------------------------------------
# halo exchange of pre-mixed face rows (numpy restatement, test infrastructure)
# ------------------------------------------------------------------------------------------------
def face_orientations(fluxL, fluxN):
    """O[v] (F x F) with fluxN[4 v + f] = fluxL[f] . O[v] for every local face f: the neighbour
    flux matrices of SurfIntVanilla::neigh (SurfIntVanilla.hpp:274-357, matrix 4 + 4 vId + fId)
    are the local projections followed by the face-vertex orientation. Returns (O [3][F][F], the
    largest residual of the factorisation over all v, f)."""
    O, res = [], 0.0
    for v in range(3):
        o = np.linalg.lstsq(fluxL[0], fluxN[4 * v], rcond=None)[0]
        O.append(o)
        for f in range(4):
            res = max(res, float(np.abs(fluxL[f] @ o - fluxN[4 * v + f]).max() / np.abs(fluxN[4 * v + f]).max()))
    return np.array(O), res


def flux_char_factors(fs0, fs1):
    """Rank-3 factors of a face's stacked flux solvers [fs0; fs1] (18 x 9) = [U0; U1] V^T: fs0 the
    writer's own fsE[0] at the face, fs1 the fsE[1] its reader applies (None: an outflow face). The
    same steps as the device's factor build: columns scaled to unit maximum, Gram-Schmidt with
    pivoting over the scaled rows, each direction orthogonalised twice. Returns (V, U0, U1), each
    9 x 3 (U1 zero without a reader)."""
    S = np.vstack([fs0.reshape(9, 9), np.zeros((9, 9)) if fs1 is None else fs1.reshape(9, 9)])
    c = np.abs(S).max(axis=0)
    c[c == 0] = 1.0
    St = S / c
    R = St.copy()
    Q = np.zeros((3, 9))
    for k in range(3):
        v = R[int(np.argmax((R * R).sum(axis=1)))].copy()
        for _ in range(2):
            for kk in range(k):
                v -= (v @ Q[kk]) * Q[kk]
        n2 = v @ v
        Q[k] = v / np.sqrt(n2) if n2 > 0 else 0.0
        R -= np.outer(R @ Q[k], Q[k])
    U = St @ Q.T
    return c[:, None] * Q.T, U[:9], U[9:]


def face_rows_premixed(prob, tDofs, send):
    """The face rows a part sends for its faces `send` [n][2] = (element, face): the element's
    time-integrated DOFs projected on the face (tDofs . fluxL_face, the face-projected data EDGE's
    MPI path ships, AderDg.hpp:419-473) and mixed with the flux solver of the element that reads
    them (fsE[1] of the face neighbour at its own face id). Returns [n][9][F][R]."""
    fl, fs1 = prob["fluxL"], prob["fsE"][1]
    out = []
    for e, f in send:
        ne, fo = int(prob["elFaEl"][e, f]), int(prob["fIdElFaEl"][e, f])
        proj = np.einsum("qbr,bf->qfr", tDofs[e], fl[f])
        out.append(np.einsum("qp,pfr->qfr", fs1[ne, fo].reshape(9, 9), proj))
    return np.array(out)


def neigh_premixed_faces(prob, dofsE, faces, rows, O):
    """Adds the lifted fluxes of received pre-mixed face rows (SurfIntVanilla::neigh with the mix
    done by the sender): for face (element, face) with row P, dofs += (P . O[vId]) . fluxT_face."""
    ft = prob["fluxT"]
    for (e, f), P in zip(faces, rows):
        s1 = np.einsum("qfr,fg->qgr", P, O[int(prob["vIdElFaEl"][e, f])])
        dofsE[e] += np.einsum("qfr,fb->qbr", s1, ft[f])


def set_mm_mode(mode):
    """Operand rounding of the oracle's products with the DG matrices: 0 none, 1 tf32 operands,
    2 the three-product tf32 split, 3 bf16 operands, 4 the three-product bf16 split (oracle.c
    g_mmMode; for measuring tensor-core arithmetic)."""
    lib().oracle_set_mm_mode(C.c_int(mode))
