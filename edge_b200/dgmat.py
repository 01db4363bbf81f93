"""Exact DG matrices of the hierarchical (Dubiner) tetrahedral basis.

This is the build-time generator for the global matrices the element update multiplies with.
It restates, in exact rational arithmetic instead of sympy, what the reference's pre-processor
computes:

* tet basis: ``tools/edge_pre/edge_pre/dg/basis/Tet.py:31-76`` (collapsed coordinates, Jacobi
  polynomials P^(0,0), P^(2p1+1,0), P^(2p1+2p2+2,0), ordered by total degree, then p1, then p2),
  on the unit tet with vertices (0,0,0), (1,0,0), (0,1,0), (0,0,1) (``types/Tet.py:57``);
* triangle (face) basis: ``dg/basis/Tria.py:31-60`` on the unit triangle;
* mass / stiffness: ``int/Matrices.py:92-127`` with stiff_d[i][j] = int(phi_i * d(phi_j)/d xi_d);
* stiffT_d = stiff_d^T M^-1 and stiffV_d = stiff_d M^-1 (``edge_pre.py:500-508``);
* flux matrices: ``int/Matrices.py:140-248`` and ``edge_pre.py:510-521``, with the face maps of
  ``types/Tet.py:75-97`` (faToEl, faToFa). fluxN is ordered vertex-major: id = 4*v + f.

Every entry is an exact rational and is rounded once to binary64. Polynomials are dicts that map an
exponent tuple to a Fraction. Integrals of monomials are closed forms:
int_tet x^a y^b z^c = a! b! c! / (a+b+c+3)!  and  int_tri x^a y^b = a! b! / (a+b+2)!.
"""
from fractions import Fraction
from functools import lru_cache
from math import comb, factorial

# ----------------------------------------------------------------------------------------------
# polynomial helpers (dict: exponent tuple -> Fraction)
# ----------------------------------------------------------------------------------------------


def _padd(p, q, s=1):
    r = dict(p)
    for k, v in q.items():
        r[k] = r.get(k, 0) + s * v
        if r[k] == 0:
            del r[k]
    return r


def _pmul(p, q):
    r = {}
    for k1, v1 in p.items():
        for k2, v2 in q.items():
            k = tuple(a + b for a, b in zip(k1, k2))
            r[k] = r.get(k, 0) + v1 * v2
    return {k: v for k, v in r.items() if v != 0}


def _ppow(p, n, nvars):
    r = {(0,) * nvars: Fraction(1)}
    for _ in range(n):
        r = _pmul(r, p)
    return r


def _lin(coefs, const, nvars):
    """Affine form const + sum coefs[i]*x_i as a polynomial."""
    r = {}
    if const != 0:
        r[(0,) * nvars] = Fraction(const)
    for i, c in enumerate(coefs):
        if c != 0:
            e = [0] * nvars
            e[i] = 1
            r[tuple(e)] = Fraction(c)
    return r


def _hom_jacobi(n, alpha, x, w, nvars):
    """w^n * P_n^(alpha,0)(2x/w - 1) for affine forms x, w (a polynomial)."""
    # P_n^(a,0)(eta) = sum_s C(n+a, n-s) C(n, s) ((eta-1)/2)^s ((eta+1)/2)^(n-s)
    # with (eta-1)/2 = (x-w)/w and (eta+1)/2 = x/w
    xmw = _padd(x, w, -1)
    r = {}
    for s in range(n + 1):
        c = comb(n + alpha, n - s) * comb(n, s)
        term = _pmul(_ppow(xmw, s, nvars), _ppow(x, n - s, nvars))
        r = _padd(r, {k: c * v for k, v in term.items()})
    return r


def _diff(p, i):
    r = {}
    for k, v in p.items():
        if k[i] > 0:
            e = list(k)
            e[i] -= 1
            r[tuple(e)] = r.get(tuple(e), 0) + v * k[i]
    return r


def _subs_affine(p, maps, nout):
    """Substitute x_i = maps[i] (affine polynomials in nout variables)."""
    r = {}
    cache = {}
    for k, v in p.items():
        term = {(0,) * nout: Fraction(v)}
        for i, e in enumerate(k):
            if e:
                key = (i, e)
                if key not in cache:
                    cache[key] = _ppow(maps[i], e, nout)
                term = _pmul(term, cache[key])
        r = _padd(r, term)
    return r


def _int_tet(p):
    s = Fraction(0)
    for (a, b, c), v in p.items():
        s += v * Fraction(factorial(a) * factorial(b) * factorial(c), factorial(a + b + c + 3))
    return s


def _int_tri(p):
    s = Fraction(0)
    for (a, b), v in p.items():
        s += v * Fraction(factorial(a) * factorial(b), factorial(a + b + 2))
    return s


# ----------------------------------------------------------------------------------------------
# bases
# ----------------------------------------------------------------------------------------------


def n_modes_tet(order):
    return order * (order + 1) * (order + 2) // 6


def n_modes_tri(order):
    return order * (order + 1) // 2


@lru_cache(maxsize=None)
def basis_tet(deg):
    """Hierarchical tet basis of degree deg as polynomials in (xi1, xi2, xi3)."""
    x1 = _lin([1, 0, 0], 0, 3)
    x2 = _lin([0, 1, 0], 0, 3)
    x3 = _lin([0, 0, 1], 0, 3)
    s = _lin([0, -1, -1], 1, 3)  # 1 - xi2 - xi3
    t = _lin([0, 0, -1], 1, 3)  # 1 - xi3
    one = _lin([0, 0, 0], 1, 3)
    out = []
    for d in range(deg + 1):
        for p1 in range(d + 1):
            for p2 in range(d + 1):
                for p3 in range(d + 1):
                    if p1 + p2 + p3 != d:
                        continue
                    a = _hom_jacobi(p1, 0, x1, s, 3)
                    b = _hom_jacobi(p2, 2 * p1 + 1, x2, t, 3)
                    c = _hom_jacobi(p3, 2 * p1 + 2 * p2 + 2, x3, one, 3)
                    out.append(_pmul(_pmul(a, b), c))
    return tuple(out)


@lru_cache(maxsize=None)
def basis_tri(deg):
    """Hierarchical triangle basis of degree deg as polynomials in (chi1, chi2)."""
    x1 = _lin([1, 0], 0, 2)
    x2 = _lin([0, 1], 0, 2)
    w = _lin([0, -1], 1, 2)  # 1 - chi2
    one = _lin([0, 0], 1, 2)
    out = []
    for d in range(deg + 1):
        for p in range(d + 1):
            q = d - p
            a = _hom_jacobi(p, 0, x1, w, 2)
            b = _hom_jacobi(q, 2 * p + 1, x2, one, 2)
            out.append(_pmul(a, b))
    return tuple(out)


# face maps of the unit tet (types/Tet.py:75-97): chi -> xi per local face, chi -> chi per vertex id
FA_TO_EL = [
    [([0, 1], 0), ([1, 0], 0), ([0, 0], 0)],
    [([1, 0], 0), ([0, 0], 0), ([0, 1], 0)],
    [([0, 0], 0), ([0, 1], 0), ([1, 0], 0)],
    [([-1, -1], 1), ([1, 0], 0), ([0, 1], 0)],
]
FA_TO_FA = [
    [([0, 1], 0), ([1, 0], 0)],
    [([-1, -1], 1), ([0, 1], 0)],
    [([1, 0], 0), ([-1, -1], 1)],
]


def _inv_diag(m):
    n = len(m)
    for i in range(n):
        for j in range(n):
            if i != j:
                assert m[i][j] == 0, "basis is expected to be orthogonal"
    return [Fraction(1) / m[i][i] for i in range(n)]


@lru_cache(maxsize=None)
def exact_matrices(order):
    """All global DG matrices of the given order (= degree + 1) as nested lists of Fractions."""
    deg = order - 1
    bel = basis_tet(deg)
    bfa = basis_tri(deg)
    nb, nf = len(bel), len(bfa)
    mass = [[_int_tet(_pmul(bel[i], bel[j])) for j in range(nb)] for i in range(nb)]
    minv = _inv_diag(mass)
    stiff = []
    for d in range(3):
        dphi = [_diff(p, d) for p in bel]
        stiff.append([[_int_tet(_pmul(bel[i], dphi[j])) for j in range(nb)] for i in range(nb)])
    stiffT = [[[stiff[d][j][i] * minv[j] for j in range(nb)] for i in range(nb)] for d in range(3)]
    stiffV = [[[stiff[d][i][j] * minv[j] for j in range(nb)] for i in range(nb)] for d in range(3)]

    mass_fa = [[_int_tri(_pmul(bfa[i], bfa[j])) for j in range(nf)] for i in range(nf)]
    minv_fa = _inv_diag(mass_fa)
    proj = []
    for f in range(4):
        maps = [_lin(c, k, 2) for c, k in FA_TO_EL[f]]
        tr = [_subs_affine(p, maps, 2) for p in bel]
        proj.append([[_int_tri(_pmul(tr[i], bfa[j])) for j in range(nf)] for i in range(nb)])
    ori = []
    for v in range(3):
        maps = [_lin(c, k, 2) for c, k in FA_TO_FA[v]]
        tr = [_subs_affine(p, maps, 2) for p in bfa]
        ori.append([[_int_tri(_pmul(tr[i], bfa[j])) for j in range(nf)] for i in range(nf)])

    fluxL = proj
    fluxN = []
    for v in range(3):
        for f in range(4):
            pm = [[proj[f][i][k] * minv_fa[k] for k in range(nf)] for i in range(nb)]
            fluxN.append([[sum(pm[i][k] * ori[v][k][j] for k in range(nf)) for j in range(nf)]
                          for i in range(nb)])
    fluxT = [[[proj[f][i][j] * minv_fa[j] * minv[i] for i in range(nb)] for j in range(nf)]
             for f in range(4)]
    return dict(mass=mass, massInv=minv, stiffT=stiffT, stiffV=stiffV, fluxL=fluxL,
                fluxN=fluxN, fluxT=fluxT)


def matrices(order):
    """DG matrices of the given order as numpy float64 arrays (each entry rounded once)."""
    import numpy as np
    ex = exact_matrices(order)
    return {k: np.array(v, dtype=np.float64) if not isinstance(v[0], Fraction)
            else np.array([float(x) for x in v]) for k, v in ex.items()}


def basis_monomials(order):
    """Monomial form of the tet basis: list (per basis function) of (exponents, coefficient)."""
    return [sorted(p.items()) for p in basis_tet(order - 1)]
