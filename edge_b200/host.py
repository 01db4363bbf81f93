"""Python mirror of the host setup API (mesh, material, element data, sources, receivers).

Each function wraps the C ABI of ``libedge_b200.so`` (include/edge_b200.h); the semantics are
EDGE's setup (src/impl/seismic/setup.inc) restated in C++ in ``csrc/host.cpp``.
"""
import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from ._lib import check, lib, ptr

FACE_INNER, FACE_FREE_SURFACE, FACE_OUTFLOW, FACE_PERIODIC = 0, 1, 2, 3


def n_modes(order):
    return order * (order + 1) * (order + 2) // 6


def n_face_modes(order):
    return order * (order + 1) // 2


class Mesh:
    """Tet mesh with EDGE-V's conventions (see edge_mesh_box in include/edge_b200.h)."""

    def __init__(self, handle):
        self._h = handle
        nve, nfa, nel = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().edge_mesh_sizes(handle, C.byref(nve), C.byref(nfa), C.byref(nel)), "edge_mesh_sizes")
        self.n_ve, self.n_fa, self.n_el = nve.value, nfa.value, nel.value
        ne, nf = self.n_el, self.n_fa
        self.ve = np.zeros((self.n_ve, 3))
        self.el_ve = np.zeros((ne, 4), np.int64)
        self.el_fa = np.zeros((ne, 4), np.int64)
        self.fa_el = np.zeros((nf, 2), np.int64)
        self.fa_normal = np.zeros((nf, 3))
        self.fa_tangent = np.zeros((nf, 2, 3))
        self.fa_area = np.zeros(nf)
        self.fa_type = np.zeros(nf, np.uint8)
        self.el_vol = np.zeros(ne)
        self.el_india = np.zeros(ne)
        self.el_fa_el = np.zeros((ne, 4), np.int32)
        self.fid = np.zeros((ne, 4), np.uint8)
        self.vid = np.zeros((ne, 4), np.uint8)
        self.el_fa_type = np.zeros((ne, 4), np.uint8)
        check(lib().edge_mesh_arrays(handle, *[ptr(a) for a in (
            self.ve, self.el_ve, self.el_fa, self.fa_el, self.fa_normal, self.fa_tangent,
            self.fa_area, self.fa_type, self.el_vol, self.el_india, self.el_fa_el, self.fid,
            self.vid, self.el_fa_type)]), "edge_mesh_arrays")

    @classmethod
    def box(cls, n, ext=(1e4, 1e4, 1e4), jitter=0.0, seed=0, bc_top=FACE_FREE_SURFACE,
            bc_sides=FACE_OUTFLOW):
        nx, ny, nz = (n, n, n) if np.isscalar(n) else n
        h = C.c_void_p()
        e = np.asarray(ext, dtype=np.float64)
        check(lib().edge_mesh_box(nx, ny, nz, ptr(e), float(jitter), int(seed), bc_top, bc_sides,
                                  C.byref(h)), "edge_mesh_box")
        m = cls(h)
        m.ext = tuple(float(x) for x in ext)
        m.n_cubes = (nx, ny, nz)
        return m

    @classmethod
    def from_arrays(cls, ve, el_ve, bf_ve=None, bf_tag=None, default_type=-1, reorder=True):
        """Mesh of arbitrary tets (edge_mesh_from_arrays): boundary faces bf_ve[n][3] tagged 101
        (free surface) / 105 (outflow); untagged boundary faces get default_type (-1 rejects).
        The input index of each mesh element is kept in ``el_perm``."""
        ve = np.ascontiguousarray(ve, np.float64)
        el_ve = np.ascontiguousarray(el_ve, np.int64)
        bf_ve = np.ascontiguousarray(np.zeros((0, 3)) if bf_ve is None else bf_ve, np.int64)
        bf_tag = np.ascontiguousarray(np.zeros(0) if bf_tag is None else bf_tag, np.int32)
        perm = np.zeros(len(el_ve), np.int64)
        h = C.c_void_p()
        check(lib().edge_mesh_from_arrays(len(ve), ptr(ve), len(el_ve), ptr(el_ve), len(bf_ve), ptr(bf_ve),
                                          ptr(bf_tag), int(default_type), 1 if reorder else 0, ptr(perm),
                                          C.byref(h)), "edge_mesh_from_arrays")
        m = cls(h)
        m.el_perm = perm
        return m

    @classmethod
    def from_gmsh(cls, path, default_type=-1, reorder=True):
        """Mesh of a gmsh ASCII file (MSH 2.2 / 4.1, tets + tagged boundary triangles)."""
        from .gmsh import read_msh
        ve, el_ve, bf_ve, bf_tag = read_msh(path)
        return cls.from_arrays(ve, el_ve, bf_ve, bf_tag, default_type, reorder)

    def boundary_faces(self):
        """(bf_ve [n][3], reference tag [n]) of the boundary faces (101 free surface, 105 outflow)."""
        b = self.fa_el[:, 1] < 0
        tag = np.where(self.fa_type[b] == FACE_FREE_SURFACE, 101, 105).astype(np.int32)
        return np.ascontiguousarray(self.fa_ve()[b]), tag

    def fa_ve(self):
        """Vertices of each face (ascending), from the element faces."""
        out = np.zeros((self.n_fa, 3), np.int64)
        loc = np.array([[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]])
        for f in range(4):
            out[self.el_fa[:, f]] = np.sort(self.el_ve[:, loc[f]], axis=1)
        return out

    def __del__(self):
        if getattr(self, "_h", None):
            lib().edge_mesh_free(self._h)
            self._h = None

    def el_ve_crds(self):
        return self.ve[self.el_ve]  # [nEl][4][3]

    def centroids(self):
        return self.el_ve_crds().mean(axis=1)


def star(mesh, rho, lam, mu):
    out = np.zeros((mesh.n_el, 3, 24))
    a = [np.ascontiguousarray(x, np.float64) for x in (rho, lam, mu)]
    check(lib().edge_setup_star(mesh._h, *[ptr(x) for x in a], ptr(out)), "edge_setup_star")
    return out


def star_anelastic(mesh):
    out = np.zeros((mesh.n_el, 3, 9))
    check(lib().edge_setup_star_anelastic(mesh._h, ptr(out)), "edge_setup_star_anelastic")
    return out


def flux_solvers(mesh, rho, lam, mu, n_rms=0):
    fsE = np.zeros((2, mesh.n_el, 4, 81))
    fsA = np.zeros((2, mesh.n_el, 4, 54)) if n_rms else None
    a = [np.ascontiguousarray(x, np.float64) for x in (rho, lam, mu)]
    check(lib().edge_setup_flux_solvers(mesh._h, n_rms, *[ptr(x) for x in a], ptr(fsE), ptr(fsA)),
          "edge_setup_flux_solvers")
    return fsE, fsA


def frequencies(n_rms, freq_cen, freq_rat):
    out = np.zeros(2 * n_rms - 1)
    check(lib().edge_setup_frequencies(n_rms, freq_cen, freq_rat, ptr(out)), "edge_setup_frequencies")
    return out


def anelastic_coeffs(n_rms, quality, freqs):
    out = np.zeros(n_rms)
    f = np.ascontiguousarray(freqs, np.float64)
    check(lib().edge_setup_anelastic_coeffs(n_rms, quality, ptr(f), ptr(out)), "anelastic_coeffs")
    return out


def elastic_lame(n_rms, freq_ref, freqs, ck, cm, lam_phase, mu_phase):
    le, me = C.c_double(), C.c_double()
    a = [np.ascontiguousarray(x, np.float64) for x in (freqs, ck, cm)]
    check(lib().edge_setup_elastic_lame(n_rms, freq_ref, *[ptr(x) for x in a], lam_phase, mu_phase,
                                        C.byref(le), C.byref(me)), "elastic_lame")
    return le.value, me.value


def attenuation(n_rms, freq_cen, freq_rat, qp, qs, lam, mu):
    """Returns (srcA[nEl][rm][12], omega[rm], lam_unrelaxed, mu_unrelaxed)."""
    lam = np.array(lam, np.float64)
    mu = np.array(mu, np.float64)
    n = len(lam)
    src = np.zeros((n, n_rms, 12))
    om = np.zeros(n_rms)
    qp = np.ascontiguousarray(qp, np.float64)
    qs = np.ascontiguousarray(qs, np.float64)
    check(lib().edge_setup_attenuation(n_rms, freq_cen, freq_rat, n, ptr(qp), ptr(qs), ptr(lam),
                                       ptr(mu), ptr(src), ptr(om)), "edge_setup_attenuation")
    return src, om, lam, mu


def dt_cfl(mesh, order, rho, lam, mu):
    out = C.c_double()
    a = [np.ascontiguousarray(x, np.float64) for x in (rho, lam, mu)]
    check(lib().edge_setup_dt_cfl(mesh._h, order, *[ptr(x) for x in a], C.byref(out)), "dt_cfl")
    return out.value


def dt_cfl_el(mesh, order, rho, lam, mu):
    """Per-element CFL time steps (edge_setup_dt_cfl_el)."""
    out = np.zeros(mesh.n_el)
    a = [np.ascontiguousarray(x, np.float64) for x in (rho, lam, mu)]
    check(lib().edge_setup_dt_cfl_el(mesh._h, order, *[ptr(x) for x in a], ptr(out)), "dt_cfl_el")
    return out


def time_groups(mesh, dt_el, n_groups, fun_dt=1.0):
    """Rate-2 LTS time group of every element (edge_setup_time_groups, EDGE-V's rules)."""
    out = np.zeros(mesh.n_el, np.uint8)
    check(lib().edge_setup_time_groups(mesh._h, ptr(np.ascontiguousarray(dt_el, np.float64)), int(n_groups),
                                       float(fun_dt), ptr(out), None), "time_groups")
    return out


def lts_tables(mesh, el_tg):
    """Element flags (1: a larger neighbour, 2: a smaller one) and per-face relations (0 equal,
    1 this element larger, 2 smaller) of LTS time groups, as the device derives them."""
    el_tg = np.asarray(el_tg, np.int64)
    ne = mesh.el_fa_el.astype(np.int64)
    inner = (mesh.el_fa_type == FACE_INNER) & (ne >= 0)
    d = np.where(inner, el_tg[:, None] - el_tg[np.maximum(ne, 0)], 0)
    if np.abs(d).max(initial=0) > 1:
        raise ValueError("face neighbours differ by more than one time group")
    rel = np.where(d > 0, 1, np.where(d < 0, 2, 0)).astype(np.uint8)
    flags = (np.any(d < 0, axis=1) * 1 + np.any(d > 0, axis=1) * 2).astype(np.uint8)
    return flags, np.ascontiguousarray(rel)


def sort_by_groups(mesh, el_tg):
    """The mesh with its elements ordered by time group and, within a group, elements with a
    smaller neighbour first (they need the half-step integrals), the input index of each new
    element, and group_first [G+1] (element ranges of the groups)."""
    el_tg = np.asarray(el_tg)
    flags, _ = lts_tables(mesh, el_tg)
    perm = np.lexsort(((flags & 2) == 0, el_tg))
    bf_ve, tag = mesh.boundary_faces()
    m = Mesh.from_arrays(mesh.ve, mesh.el_ve[perm], bf_ve, tag, reorder=False)
    n_groups = int(el_tg.max()) + 1
    group_first = np.searchsorted(el_tg[perm], np.arange(n_groups + 1)).astype(np.int64)
    return m, perm, group_first


def locate(mesh, order, xyz, source=False):
    xyz = np.ascontiguousarray(np.atleast_2d(xyz), np.float64)
    n = xyz.shape[0]
    el = np.zeros(n, np.int64)
    ref = np.zeros((n, 3))
    basis = np.zeros((n, n_modes(order)))
    check(lib().edge_setup_locate(mesh._h, order, n, ptr(xyz), ptr(el), ptr(ref), ptr(basis),
                                  1 if source else 0), "edge_setup_locate")
    return el, ref, basis


def eval_basis(order, ref):
    out = np.zeros(n_modes(order))
    r = np.ascontiguousarray(ref, np.float64)
    check(lib().edge_setup_eval_basis(order, ptr(r), ptr(out)), "eval_basis")
    return out


def trafo(n, s, t):
    T, Ti = np.zeros((9, 9)), np.zeros((9, 9))
    a = [np.ascontiguousarray(x, np.float64) for x in (n, s, t)]
    check(lib().edge_setup_trafo(*[ptr(x) for x in a], ptr(T), ptr(Ti)), "trafo")
    return T, Ti


def fs_pair(rho_l, rho_r, lam_l, lam_r, mu_l, mu_r, n, s, t, free_surface=False):
    el, er, al, ar = np.zeros((9, 9)), np.zeros((9, 9)), np.zeros((6, 9)), np.zeros((6, 9))
    a = [np.ascontiguousarray(x, np.float64) for x in (n, s, t)]
    check(lib().edge_setup_fs_pair(rho_l, rho_r, lam_l, lam_r, mu_l, mu_r, *[ptr(x) for x in a],
                                   1 if free_surface else 0, ptr(el), ptr(er), ptr(al), ptr(ar)),
          "fs_pair")
    return el, er, al, ar


def ricker(t, f0, t0):
    a = (np.pi * f0 * (t - t0)) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


@dataclass
class Problem:
    """A complete setup of the element update: mesh, element data, sources, receivers, DOFs."""
    order: int
    runs: int
    rm: int
    mesh: Mesh
    rho: np.ndarray
    lam: np.ndarray
    mu: np.ndarray
    starE: np.ndarray
    fsE: np.ndarray
    dt: float
    starA: Optional[np.ndarray] = None
    srcA: Optional[np.ndarray] = None
    fsA: Optional[np.ndarray] = None
    omega: Optional[np.ndarray] = None
    sources: dict = field(default_factory=dict)
    receivers: dict = field(default_factory=dict)
    name: str = ""

    @property
    def n_el(self):
        return self.mesh.n_el

    @property
    def B(self):
        return n_modes(self.order)

    def zero_dofs(self, dtype=np.float64):
        e = np.zeros((self.n_el, 9, self.B, self.runs), dtype)
        a = np.zeros((self.n_el, self.rm, 6, self.B, self.runs), dtype) if self.rm else None
        return e, a

    def single_run(self, r):
        """The one-run problem of fused run r: same mesh, element data and receivers, with only
        run r's point sources (EDGE runs a fused build's runs independently: no kernel mixes runs)."""
        src = {}
        s = self.sources
        if s and s.get("n", 0):
            keep = [i for i in range(s["n"]) if s["run"][i] == r]
            pick = lambda k: np.ascontiguousarray(s[k][keep])
            src = dict(n=len(keep), el=pick("el"), run=np.zeros(len(keep), np.int32), scal=pick("scal"),
                       bEval=pick("bEval"), t0=pick("t0"), dt=pick("dt"), tsOff=pick("tsOff"), nPts=pick("nPts"),
                       ts=s["ts"])
        return Problem(order=self.order, runs=1, rm=self.rm, mesh=self.mesh, rho=self.rho, lam=self.lam,
                       mu=self.mu, starE=self.starE, fsE=self.fsE, dt=self.dt, starA=self.starA, srcA=self.srcA,
                       fsA=self.fsA, omega=self.omega, sources=src, receivers=self.receivers,
                       name=self.name + f"_run{r}")

    def oracle_dict(self):
        """Element data in the oracle's layout (tests only)."""
        from . import dgmat
        m = dgmat.matrices(self.order)
        d = dict(order=self.order, runs=self.runs, rm=self.rm, nEl=self.n_el,
                 stiffT=m["stiffT"], stiffV=m["stiffV"], fluxL=m["fluxL"], fluxN=m["fluxN"],
                 fluxT=m["fluxT"], starE=self.starE, fsE=self.fsE, starA=self.starA,
                 srcA=self.srcA, fsA=self.fsA, omega=self.omega,
                 elFaEl=np.ascontiguousarray(self.mesh.el_fa_el),
                 fIdElFaEl=np.ascontiguousarray(self.mesh.fid),
                 vIdElFaEl=np.ascontiguousarray(self.mesh.vid),
                 faType=np.ascontiguousarray(self.mesh.el_fa_type))
        return {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in d.items()}


def make_sources(mesh, order, runs, positions, scalings, f0, t_onset, dt_series, n_series):
    """Point sources: run r gets the point positions[r] with Voigt moment tensor scalings[r][9]
    and a Ricker moment-rate series of peak frequency f0 delayed by t_onset, sampled every
    dt_series (PointSources.hpp:525-768 reads the same quantities from HDF5)."""
    positions = np.atleast_2d(positions)
    el, ref, bEval = locate(mesh, order, positions, source=True)
    ts_t = np.arange(n_series) * dt_series
    series = ricker(ts_t, f0, t_onset)
    recs = sorted(range(len(positions)), key=lambda s: (el[s], s % runs))
    src = dict(n=len(positions), el=np.array([el[s] for s in recs], np.int64),
               run=np.array([s % runs for s in recs], np.int32),
               scal=np.ascontiguousarray([scalings[s] for s in recs], np.float64),
               bEval=np.ascontiguousarray([bEval[s] for s in recs], np.float64),
               t0=np.zeros(len(positions)), dt=np.full(len(positions), dt_series),
               tsOff=np.arange(len(positions), dtype=np.int64) * n_series,
               nPts=np.full(len(positions), n_series, np.int64),
               ts=np.ascontiguousarray(np.tile(series, len(positions))))
    return src


def make_receivers(mesh, order, positions, period, t_end, t_first=0.0):
    el, ref, basis = locate(mesh, order, positions, source=False)
    order_idx = np.argsort(el, kind="stable")
    maxbuf = int(np.ceil((t_end - t_first) / period)) + 2
    return dict(n=len(positions), el=np.ascontiguousarray(el[order_idx]),
                basis=np.ascontiguousarray(basis[order_idx]), period=float(period),
                t_first=float(t_first), maxbuf=maxbuf, perm=order_idx,
                positions=np.asarray(positions)[order_idx])


def materials(mesh, ext, vp=6000.0, vs=3464.0, rho=2670.0, layers=None, lognormal_sigma=0.0, rng=None):
    """Per-element (rho, lam, mu): homogeneous, or horizontal layers of vp (listed from the top,
    z = ext, down; vs = vp / sqrt(3)), each element optionally scaled by a seeded lognormal factor."""
    ne = mesh.n_el
    if layers is None:
        vpe = np.full(ne, vp)
    else:
        z = mesh.centroids()[:, 2]
        bounds = np.linspace(0, ext, len(layers) + 1)
        idx = np.clip(np.searchsorted(bounds, z, side="right") - 1, 0, len(layers) - 1)
        vpe = np.asarray(layers, np.float64)[::-1][idx]
    if lognormal_sigma > 0:
        vpe = vpe * rng.lognormal(0.0, lognormal_sigma, ne)
    vse = vpe / np.sqrt(3.0) if layers is not None else np.full(ne, vs) * (vpe / vp)
    rhoe = np.full(ne, rho)
    mu = rhoe * vse ** 2
    lam = rhoe * vpe ** 2 - 2 * mu
    return rhoe, lam, mu


def element_data(mesh, rho, lam, mu, rm=0, qp=None, qs=None, freq_cen=1.0, freq_rat=100.0):
    """Star matrices and flux solvers (and, with rm mechanisms and qualities qp / qs, the anelastic
    data, with lam / mu replaced by the unrelaxed values first, as AderDgInit.hpp:113-115 does)."""
    srcA = omega = starA = fsA = None
    if rm:
        srcA, omega, lam, mu = attenuation(rm, freq_cen, freq_rat, qp, qs, lam, mu)
        starA = star_anelastic(mesh)
    starE = star(mesh, rho, lam, mu)
    fsE, fsA = flux_solvers(mesh, rho, lam, mu, rm)
    return dict(lam=lam, mu=mu, starE=starE, fsE=fsE, starA=starA, srcA=srcA, fsA=fsA, omega=omega)


def build_problem(n_cubes, order, runs, rm=0, ext=1e4, jitter=0.0, seed=3343, vp=6000.0,
                  vs=3464.0, rho=2670.0, layers=None, lognormal_sigma=0.0, q_range=None,
                  freq_cen=1.0, freq_rat=100.0, n_receivers=8, source="explosive", f0=2.0,
                  n_steps=200, period=None, cfl=1.0, bc_top=FACE_FREE_SURFACE,
                  bc_sides=FACE_OUTFLOW, name="", mesh=None, f0_window=None, receivers_near=None):
    """Synthetic setups of the element update (box meshes, homogeneous or layered materials).
    A given ``mesh`` (e.g. Mesh.from_gmsh of a box [0, ext]^3) replaces the generated box.
    Sources are Ricker moment rates peaking at 1.2 / f0; with ``f0_window`` the peak is put at that
    fraction of the simulated time n_steps * dt instead (f0 follows), for runs too short for the
    given f0. With ``receivers_near`` (metres) receiver i sits that far from run (i mod runs)'s
    source in a seeded random direction instead of at a uniform position."""
    rng = np.random.default_rng(seed)
    if mesh is None:
        mesh = Mesh.box(n_cubes, (ext, ext, ext), jitter=jitter, seed=seed, bc_top=bc_top, bc_sides=bc_sides)
    ne = mesh.n_el
    rhoe, lam, mu = materials(mesh, ext, vp, vs, rho, layers, lognormal_sigma, rng)
    qp = qs = None
    if rm:
        lo, hi = q_range if q_range else (50.0, 200.0)
        qp = rng.uniform(lo, hi, ne)
        qs = rng.uniform(lo, hi, ne)
    ed = element_data(mesh, rhoe, lam, mu, rm, qp, qs, freq_cen, freq_rat)
    lam, mu = ed["lam"], ed["mu"]
    starE, fsE, starA, srcA, fsA, omega = (ed[k] for k in ("starE", "fsE", "starA", "srcA", "fsA", "omega"))
    dt = dt_cfl(mesh, order, rhoe, lam, mu) * cfl
    t_end = n_steps * dt
    # sources
    if source == "explosive":
        M0 = 1e15
        pos = np.array([[ext / 2, ext / 2, ext / 2]] * runs)
        scal = np.array([[M0, M0, M0, 0, 0, 0, 0, 0, 0]] * runs, np.float64)
    elif source == "random":
        pos = rng.uniform(0.1 * ext, 0.9 * ext, (runs, 3))
        mt = rng.normal(0.0, 1.0, (runs, 6)) * 1e15
        scal = np.concatenate([mt, np.zeros((runs, 3))], axis=1)
    else:
        pos, scal = None, None
    src = {}
    if pos is not None:
        dts = dt / 10.0
        n_series = int(np.ceil(t_end / dts)) + 4
        t_onset = 1.2 / f0
        if f0_window:
            t_onset = f0_window * t_end
            f0 = 1.2 / t_onset
        src = make_sources(mesh, order, runs, pos, scal, f0, t_onset, dts, n_series)
    rec = {}
    if n_receivers:
        rpos = rng.uniform(0.1 * ext, 0.9 * ext, (n_receivers, 3))
        if receivers_near and pos is not None:
            u = rng.normal(size=(n_receivers, 3))
            u /= np.linalg.norm(u, axis=1)[:, None]
            rpos = pos[np.arange(n_receivers) % runs] + receivers_near * u
        per = period if period else dt * 0.37
        rec = make_receivers(mesh, order, rpos, per, t_end)
    return Problem(order=order, runs=runs, rm=rm, mesh=mesh, rho=rhoe, lam=lam, mu=mu, starE=starE,
                   fsE=fsE, dt=dt, starA=starA, srcA=srcA, fsA=fsA, omega=omega, sources=src,
                   receivers=rec, name=name)


# ------------------------------------------------------------------------------------------------
# initial values and error norms (InitialDofs::dg / ::err, src/setups/InitialDofs.hpp:172-373)
# ------------------------------------------------------------------------------------------------
def tet_quadrature(n):
    """Collapsed (Duffy) Gauss-Legendre rule on the unit tet: points [P][3], weights [P]."""
    x, w = np.polynomial.legendre.leggauss(n)
    x, w = (x + 1) / 2, w / 2
    a, b, c = np.meshgrid(x, x, x, indexing="ij")
    wa, wb, wc = np.meshgrid(w, w, w, indexing="ij")
    xi3 = c
    xi2 = b * (1 - c)
    xi1 = a * (1 - b) * (1 - c)
    wt = wa * wb * wc * (1 - b) * (1 - c) ** 2
    return np.stack([xi1.ravel(), xi2.ravel(), xi3.ravel()], axis=1), wt.ravel()


def basis_at(order, pts):
    """Basis values V[P][B] at reference points (monomial form of the generated basis)."""
    from . import dgmat
    mons = dgmat.basis_monomials(order)
    V = np.zeros((len(pts), len(mons)))
    for b, terms in enumerate(mons):
        for (ea, eb, ec), cf in terms:
            V[:, b] += float(cf) * pts[:, 0] ** ea * pts[:, 1] ** eb * pts[:, 2] ** ec
    return V


def _phys_points(mesh, pts, chunk):
    v = mesh.ve[mesh.el_ve[chunk]]                      # [E][4][3]
    jac = v[:, 1:, :] - v[:, :1, :]                     # [E][3][3]
    x = v[:, None, 0, :] + np.einsum("pa,ead->epd", pts, jac)
    return x, np.abs(np.linalg.det(jac))


def project(mesh, order, fn, runs=1, n_quad=None, chunk=20000):
    """L2 projection of fn(x[..., 3]) -> q[..., 9] onto the DG basis: dofs[nEl][9][B][runs]."""
    from . import dgmat
    pts, wts = tet_quadrature(n_quad or order + 2)
    V = basis_at(order, pts)
    minv = dgmat.matrices(order)["massInv"]
    B = n_modes(order)
    out = np.zeros((mesh.n_el, 9, B, runs))
    for s in range(0, mesh.n_el, chunk):
        idx = np.arange(s, min(s + chunk, mesh.n_el))
        x, _ = _phys_points(mesh, pts, idx)
        q = fn(x)                                        # [E][P][9]
        d = np.einsum("epq,p,pb->eqb", q, wts, V) * minv[None, None, :]
        out[idx] = d[..., None]
    return out


def l2_error(mesh, order, dofs, fn, run=0, n_quad=None, chunk=20000):
    """Per-quantity L2 norms over the mesh of (DG solution - fn) and of fn."""
    pts, wts = tet_quadrature(n_quad or order + 3)
    V = basis_at(order, pts)
    err = np.zeros(9)
    ref = np.zeros(9)
    for s in range(0, mesh.n_el, chunk):
        idx = np.arange(s, min(s + chunk, mesh.n_el))
        x, det = _phys_points(mesh, pts, idx)
        q = fn(x)
        qh = np.einsum("eqb,pb->epq", np.asarray(dofs[idx, :, :, run], np.float64), V)
        err += np.einsum("epq,p,e->q", (qh - q) ** 2, wts, det)
        ref += np.einsum("epq,p,e->q", q ** 2, wts, det)
    return np.sqrt(err), np.sqrt(ref)


def plane_wave_rows(rho, lam, mu, kvec, amp=1.0, run=-1):
    """The P plane wave of plane_wave_p as a row k[3], omega, phase, amp[9], run of the device
    error norms (sin(k.x - omega t) times the eigenvector)."""
    kvec = np.asarray(kvec, np.float64)
    kn = np.linalg.norm(kvec)
    n = kvec / kn
    cp = np.sqrt((lam + 2 * mu) / rho)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]
    sig = np.array([-(lam * (i == j) + 2 * mu * n[i] * n[j]) / cp for i, j in pairs])
    return np.concatenate([kvec, [cp * kn, 0.0], amp * np.concatenate([sig, n]), [run]])


def plane_wave_p(rho, lam, mu, kvec, amp=1.0):
    """P plane wave a = amp sin(k.x - w t): v = n a, sigma = -(lam I + 2 mu n n) a / cp."""
    kvec = np.asarray(kvec, np.float64)
    kn = np.linalg.norm(kvec)
    n = kvec / kn
    cp = np.sqrt((lam + 2 * mu) / rho)
    om = cp * kn
    # Voigt xx, yy, zz, xy, yz, xz
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]
    sig = np.array([-(lam * (i == j) + 2 * mu * n[i] * n[j]) / cp for i, j in pairs])
    vec = np.concatenate([sig, n])

    def fn(x, t=0.0):
        a = amp * np.sin(x @ kvec - om * t)
        return a[..., None] * vec
    return fn
