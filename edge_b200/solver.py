"""Device element update through the C ABI: the Python counterpart of EDGE's AderDg driver.

``Solver(problem, precision)`` creates a device context (edge_b200_create), uploads the mesh,
element data, sources and receivers of a :class:`edge_b200.host.Problem`, and advances GTS steps
(edge_b200_step: local -> sources -> neighbour per step, as src/impl/seismic/steps.inc:24-77).
There is no CPU fallback: without the built library or a CUDA device the constructor raises.
"""
import ctypes as C

import numpy as np

from ._lib import Cfg, check, lib, ptr


class Solver:
    def __init__(self, prob, precision=64, stream=None, device=0, share_from=None):
        self.prob = prob
        self.precision = precision
        self.dtype = np.float64 if precision == 64 else np.float32
        L = lib()
        cfg = Cfg(order=prob.order, n_runs=prob.runs, n_rms=prob.rm, precision=precision,
                  stream=stream, device=device)
        h = C.c_void_p()
        rc = L.edge_b200_create(C.byref(cfg), prob.n_el, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"edge_b200_create failed ({rc}): order={prob.order} runs={prob.runs} "
                               f"rms={prob.rm} precision={precision}")
        self._h = h
        m = prob.mesh
        self._chk(L.edge_b200_upload_mesh(h, ptr(np.ascontiguousarray(m.el_fa_el)),
                                          ptr(np.ascontiguousarray(m.fid)),
                                          ptr(np.ascontiguousarray(m.vid)),
                                          ptr(np.ascontiguousarray(m.el_fa_type))), "upload_mesh")
        if share_from is not None:
            # element data borrowed from another context of the same mesh (kept alive with this one)
            self._share = share_from
            self._chk(L.edge_b200_share_element_data(h, share_from._h), "share_element_data")
        else:
            c = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
            self._keep = [c(prob.starE), c(prob.fsE), c(prob.starA), c(prob.srcA), c(prob.fsA), c(prob.omega)]
            self._chk(L.edge_b200_upload_element_data(h, *[ptr(a) for a in self._keep]), "upload_element_data")
        s = prob.sources
        if s and s.get("n", 0):
            self._chk(L.edge_b200_set_sources(h, s["n"], ptr(s["el"]), ptr(s["run"]), ptr(s["scal"]),
                                              ptr(s["bEval"]), ptr(s["t0"]), ptr(s["dt"]), ptr(s["tsOff"]),
                                              ptr(s["nPts"]), len(s["ts"]), ptr(s["ts"])), "set_sources")
        r = prob.receivers
        if r and r.get("n", 0):
            self._chk(L.edge_b200_set_receivers(h, r["n"], ptr(r["el"]), ptr(r["basis"]), r["t_first"],
                                                r["period"], r["maxbuf"]), "set_receivers")
        self.t = 0.0

    def _chk(self, rc, what):
        if rc != 0:
            msg = lib().edge_b200_last_error(self._h)
            raise RuntimeError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def upload_dofs(self, dofsE, dofsA=None):
        self._dE = np.ascontiguousarray(dofsE, self.dtype)
        self._dA = None if dofsA is None else np.ascontiguousarray(dofsA, self.dtype)
        self._chk(lib().edge_b200_upload_dofs(self._h, ptr(self._dE), ptr(self._dA)), "upload_dofs")

    def download_dofs(self):
        p = self.prob
        e = np.zeros((p.n_el, 9, p.B, p.runs), self.dtype)
        a = np.zeros((p.n_el, p.rm, 6, p.B, p.runs), self.dtype) if p.rm else None
        self._chk(lib().edge_b200_download_dofs(self._h, ptr(e), ptr(a)), "download_dofs")
        return e, a

    def keep_tdofs(self, enable=True):
        self._chk(lib().edge_b200_keep_tdofs(self._h, 1 if enable else 0), "keep_tdofs")

    def download_tdofs(self):
        p = self.prob
        t = np.zeros((p.n_el, 9, p.B, p.runs), self.dtype)
        self._chk(lib().edge_b200_download_tdofs(self._h, ptr(t)), "download_tdofs")
        return t

    def step(self, n_steps=1, dt=None, t=None):
        dt = self.prob.dt if dt is None else dt
        t0 = self.t if t is None else t
        self._chk(lib().edge_b200_step(self._h, t0, dt, n_steps), "step")
        tt = t0
        for _ in range(n_steps):
            tt += dt
        self.t = tt

    def set_time_groups(self, group_first):
        """Rate-2 LTS time groups: group g = elements [group_first[g], group_first[g+1])."""
        gf = np.ascontiguousarray(group_first, np.int64)
        self.n_groups = len(gf) - 1
        self._chk(lib().edge_b200_set_time_groups(self._h, self.n_groups, ptr(gf)), "set_time_groups")

    def step_lts(self, n_cycles=1, dt_fun=None, t=None):
        """n_cycles steps of the largest group (2^(G-1) fundamental steps of dt_fun each)."""
        dt_fun = self.prob.dt if dt_fun is None else dt_fun
        t0 = self.t if t is None else t
        self._chk(lib().edge_b200_step_lts(self._h, t0, dt_fun, n_cycles), "step_lts")
        self.t = t0 + float(n_cycles * (1 << (self.n_groups - 1))) * dt_fun

    def wavefield(self):
        """Mode-0 coefficients [R][9][nEl] (FP32) of the device DOFs."""
        out = np.zeros((self.prob.runs, 9, self.prob.n_el), np.float32)
        self._chk(lib().edge_b200_wavefield(self._h, ptr(out)), "wavefield")
        return out

    def upload_geometry(self):
        crds = np.ascontiguousarray(self.prob.mesh.el_ve_crds(), np.float64)
        self._chk(lib().edge_b200_upload_geometry(self._h, ptr(crds)), "upload_geometry")

    def error_norms(self, waves, t=None, n_quad=None):
        """L1 / L2 / Linf errors [9][R] against a sum of plane waves (rows k[3], omega, phase,
        amp[9], run) on the device; the collapsed Gauss rule with order+1 points per direction."""
        from . import host
        t = self.t if t is None else t
        pts, wts = host.tet_quadrature(n_quad or self.prob.order + 1)
        V = host.basis_at(self.prob.order, pts)
        w = np.ascontiguousarray(np.atleast_2d(waves), np.float64)
        R = self.prob.runs
        out = [np.zeros((9, R)) for _ in range(3)]
        self._chk(lib().edge_b200_error_norms(self._h, t, len(w), ptr(w), len(pts), ptr(np.ascontiguousarray(pts)),
                                              ptr(np.ascontiguousarray(wts)), ptr(np.ascontiguousarray(V)),
                                              *[ptr(o) for o in out]), "error_norms")
        return out

    def sync(self):
        self._chk(lib().edge_b200_sync(self._h), "sync")

    def launches(self):
        return lib().edge_b200_last_launches(self._h)

    def receivers(self):
        r = self.prob.receivers
        if not r or not r.get("n", 0):
            return None, None, None
        buf = np.zeros((r["n"], r["maxbuf"], 9, self.prob.runs))
        bt = np.zeros((r["n"], r["maxbuf"]))
        cnt = np.zeros(r["n"], np.int32)
        self._chk(lib().edge_b200_read_receivers(self._h, ptr(buf), ptr(bt), ptr(cnt)), "read_receivers")
        return buf, bt, cnt

    def device_ptrs(self):
        e, a, t = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self._chk(lib().edge_b200_device_dofs(self._h, C.byref(e), C.byref(a), C.byref(t)), "device_dofs")
        return e.value, a.value, t.value

    def close(self):
        if getattr(self, "_h", None):
            lib().edge_b200_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
