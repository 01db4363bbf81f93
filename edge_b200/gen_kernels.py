"""Writes ``edge_b200/csrc/gen/dg_sparse.cuh``: the products with the global DG matrices as
straight-line, compile-time sparse code, one block per order.

The stiffness matrices of the hierarchical basis are ~18% non-zero and the face matrices ~45%
(orders 3-6), so each product is emitted as the fused multiply-adds of its non-zeros only, with the
matrix entries as literals. Per thread the operand and accumulator rows live in registers:

* ``CkMul<O,D>``      acc[n] += sum_dim sum_k z_dim(k) * (-K^T_dim)[k][n], k < B(O-D+1), n < B(O-D)
                      (derivative D of the Cauchy-Kowalevski recursion; D=1 also serves the
                      viscoelastic case, which never truncates: k < B, n < B(O-1))
* ``VolMul<O>``       acc[n] += sum_dim sum_k z_dim(k) * K_dim M^-1 [k][n], k < B(O-1)
* ``FluxLMul<O,FA>``  s[j]   += sum_k z(k) * fluxL'_FA[k][j]         (projection to face FA)

The first three take the operand as a callable that fills four rows at a time
(``z.template load<k0>(zz)``, zz[dim][i] = operand of row k0+i in direction dim); the caller forms
it from shared memory with 128-bit loads (e.g. a star-matrix mix whose loads serve all three
directions), and groups of rows without non-zeros are skipped entirely. The other two take
register arrays:
* ``FluxTMul<O,FA>``  acc[n] += sum_j s[j] * fluxT'_FA[j][n]         (lift from face FA)
* ``OriMul<O,V>``     s[j]   += sum_k x[k] * (Mface^-1 Ori_V)[k][j]  (V: reflection of the face)

Face bases. Each local face FA of every element keeps its projections in the hierarchical triangle
basis composed with a fixed rotation sigma_FA of the reference triangle's vertices (psi_m o
sigma_FA, orthogonal with the same masses), chosen per order and face to make fluxL'_FA / fluxT'_FA
as sparse as possible: at order 5 the face matrices hold 748 instead of 880 non-zeros (face 0 35
instead of 103, faces 2 and 3 304 instead of 363 / 309). A neighbour's projections at its face fo
reach this element's face FA through sigma_fo o sigma_v o sigma_FA^-1, sigma_v being the
reference's vertex-id map (a reflection, tools/edge_pre/types/Tet.py faToFa); with rotations for
the sigma_FA that is again one of the three reflections, V = ``kFacePerm[O-2][fo][FA][v]``. The
flux operators are the reference's up to this change of face basis, which the lifted flux does
not see.

Derivative directions. The stiffness products run in the reference-coordinate derivative directions
a = 0, 1, 2 given by the rows of ``DIRS`` (K'_a = sum_dim DIRS[a][dim] K_dim) instead of xi1, xi2,
xi3: in the hierarchical basis these combinations cancel exactly where the axis directions do not,
so at order 5 the recursion's products hold 516 instead of 901 non-zeros and the volume's 364
instead of 647. The star matrices change accordingly, star'_a = sum_dim DIRS^-1[dim][a] star_dim
(``kStarDir``, applied when the kernels load them), which keeps sum_dim star_dim K_dim unchanged.

Every accumulator receives its terms in ascending k, as the reference's vanilla kernels sum.

Usage: python -m edge_b200.gen_kernels
"""
import os
from fractions import Fraction

from edge_b200 import dgmat

ORDERS = range(2, 7)

# derivative directions of the stiffness products (rows: combinations of the xi1, xi2, xi3
# derivatives), chosen for the fewest non-zeros at orders 2-6 among combinations with integer
# coefficients in [-4, 4] (every order picks the same three)
DIRS = [(1, 0, 0), (0, 1, -1), (1, -2, 0)]


def dirs_inverse():
    """DIRS^-1 as Fractions (3x3 Gauss-Jordan)."""
    m = [[Fraction(x) for x in row] + [Fraction(int(i == j)) for j in range(3)] for i, row in enumerate(DIRS)]
    for c in range(3):
        p = next(r for r in range(c, 3) if m[r][c] != 0)
        m[c], m[p] = m[p], m[c]
        piv = m[c][c]
        m[c] = [x / piv for x in m[c]]
        for r in range(3):
            if r != c and m[r][c] != 0:
                f = m[r][c]
                m[r] = [x - f * y for x, y in zip(m[r], m[c])]
    return [row[3:] for row in m]


def combine_dirs(mats):
    """K'_a = sum_dim DIRS[a][dim] K_dim for three [k][n] matrices."""
    kk, nn = len(mats[0]), len(mats[0][0])
    return [[[sum(Fraction(DIRS[a][d]) * mats[d][k][n] for d in range(3)) for n in range(nn)] for k in range(kk)]
            for a in range(3)]


def lit(x):
    x = float(x)
    if x == int(x) and abs(x) < 1e15:
        return f"T({int(x)}.0)"
    return f"T({x!r})"


def block(name_tmpl, rows_in, cols_out, mat, kmax, nmax, x="x", acc="acc", neg=False):
    lines = []
    for k in range(kmax):
        for n in range(nmax):
            v = mat[k][n]
            if v == 0:
                continue
            v = -v if neg else v
            lines.append(f"    {acc}[{n}] = fmaT({x}[{k}], {lit(v)}, {acc}[{n}]);")
    return lines


def struct(name, params, body, x="x", acc="acc"):
    s = [f"template <> struct {name}<{params}> {{",
         "  template <typename T>",
         f"  static __device__ __forceinline__ void run(const T *__restrict__ {x}, T *__restrict__ {acc}) {{"]
    s += body
    s += ["  }", "};", ""]
    return s


def block_fused(mat, kmax, nmax, acc="acc", neg=False):
    """Operand produced on the fly: for every row k with a non-zero, ``zk = z(k)`` once, then its
    FMAs. Rows without non-zeros are skipped entirely (no load, no arithmetic)."""
    lines = []
    for k in range(kmax):
        nz = [(n, mat[k][n]) for n in range(nmax) if mat[k][n] != 0]
        if not nz:
            continue
        lines.append(f"    {{ const T zk = z({k});")
        for n, v in nz:
            v = -v if neg else v
            lines.append(f"      {acc}[{n}] = fmaT(zk, {lit(v)}, {acc}[{n}]);")
        lines.append("    }")
    return lines


def block_rows4(mats, kmax, nmax, acc="acc", neg=False):
    """Operands in groups of four rows: for every group k0 = 0, 4, 8, ... holding a non-zero of
    any of the given matrices (one per reference direction), ``z.template load<k0>(zz)`` fills
    zz[dim][i] = operand of row k0+i for direction dim, then the non-zeros of those rows follow.
    Rows k0..k0+3 are read with 128-bit shared-memory loads by the caller."""
    lines = []
    for k0 in range(0, kmax, 4):
        nzs = []
        for dim, mat in enumerate(mats):
            for k in range(k0, min(k0 + 4, kmax)):
                for n in range(nmax):
                    if mat[k][n] != 0:
                        nzs.append((dim, k, n, -mat[k][n] if neg else mat[k][n]))
        if not nzs:
            continue
        lines.append(f"    {{ T zz[{len(mats)}][4]; z.template load<{k0}>(zz);")
        for dim, k, n, v in sorted(nzs, key=lambda t: (t[1], t[0], t[2])):
            lines.append(f"      {acc}[{n}] = fmaT(zz[{dim}][{k - k0}], {lit(v)}, {acc}[{n}]);")
        lines.append("    }")
    return lines


def struct_fused(name, params, body, acc="acc"):
    s = [f"template <> struct {name}<{params}> {{",
         "  template <typename T, typename Z>",
         f"  static __device__ __forceinline__ void run(const Z &z, T *__restrict__ {acc}) {{"]
    s += body
    s += ["  }", "};", ""]
    return s


def main(out=None):
    here = os.path.dirname(os.path.abspath(__file__))
    out = out or os.path.join(here, "csrc", "gen", "dg_sparse.cuh")
    s = ["// generated by edge_b200/gen_kernels.py -- do not edit",
         "// Compile-time sparse products with the global DG matrices (see the generator's docstring).",
         "#pragma once", "",
         "template <typename T> __device__ __forceinline__ T fmaT(T a, T b, T c);",
         "template <> __device__ __forceinline__ float fmaT<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }",
         "template <> __device__ __forceinline__ double fmaT<double>(double a, double b, double c) { return __fma_rn(a, b, c); }",
         "",
         "template <int O, int D> struct CkMul;",
         "template <int O> struct VolMul;",
         "template <int O, int FA> struct FluxLMul;",
         "template <int O, int FA> struct FluxTMul;",
         "template <int O, int V> struct OriMul;", ""]
    nm = dgmat.n_modes_tet
    tables = []
    for o in ORDERS:
        ex = dgmat.exact_matrices(o)
        B, F = nm(o), dgmat.n_modes_tri(o)
        s.append(f"// ---------------- order {o}: B = {B}, F = {F} ----------------")
        stiffT, stiffV = combine_dirs(ex["stiffT"]), combine_dirs(ex["stiffV"])
        for d in range(1, o):
            body = block_rows4(stiffT, nm(o - d + 1), nm(o - d), "acc", neg=True)
            s += struct_fused("CkMul", f"{o}, {d}", body, "acc")
        body = block_rows4(stiffV, nm(o - 1), B, "acc")
        s += struct_fused("VolMul", f"{o}", body, "acc")
        fb = face_bases(o)
        sig = [b[0] for b in fb]
        for f in range(4):
            s += struct_fused("FluxLMul", f"{o}, {f}", block_rows4([fb[f][1]], B, F, "s"), "s")
            s += struct("FluxTMul", f"{o}, {f}", block("", None, None, fb[f][2], F, B, "s", "acc"), "s", "acc")
        # face orientation: Mface^-1 Ori_v of the three reflections
        ori = exact_orientations(o)
        for v in range(3):
            s += struct("OriMul", f"{o}, {v}", block("", None, None, ori[3 + v], F, F, "x", "s"), "x", "s")
        tables.append((o, sig, face_perm_table(sig)))
    inv = dirs_inverse()
    s.append("// star matrices of the derivative directions: star'_a = sum_dim kStarDir[dim][a] * star_dim")
    s.append("__constant__ double kStarDir[3][3] = {" +
             ", ".join("{" + ", ".join(repr(float(inv[d][a])) for a in range(3)) + "}" for d in range(3)) + "};")
    s.append("// orientation (OriMul index) from a neighbour's face fo to this element's face FA with vertex")
    s.append("// id v: kFacePerm[O - 2][fo][FA][v]; face bases sigma_FA per order: " +
             ", ".join(f"O{o} {sig}" for o, sig, _ in tables))
    rows = []
    for o, _, tab in tables:
        rows.append("{" + ", ".join("{" + ", ".join("{" + ", ".join(str(x) for x in tab[fo][fa]) + "}"
                                                   for fa in range(4)) + "}" for fo in range(4)) + "}")
    s.append("__constant__ int8_t kFacePerm[5][4][4][3] = {" + ",\n    ".join(rows) + "};")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "w") as fh:
        fh.write("\n".join(s) + "\n")
    return out


# the six vertex permutations of the reference triangle (0,0), (1,0), (0,1) as affine maps
# chi -> A chi + b, given by the images of chi1 and chi2 (dgmat's FA_TO_FA form); index 0 is the
# identity, 3..5 are the reference's vertex-id maps FA_TO_FA[0..2]
PERMS = [
    [([1, 0], 0), ([0, 1], 0)],
    [([0, 1], 0), ([-1, -1], 1)],
    [([-1, -1], 1), ([1, 0], 0)],
] + [list(m) for m in dgmat.FA_TO_FA]


def _perm_of(maps):
    """Vertex permutation (image index of each reference vertex) of an affine map."""
    verts = [(0, 0), (1, 0), (0, 1)]
    out = []
    for x, y in verts:
        img = tuple(c[0] * x + c[1] * y + k for c, k in maps)
        out.append(verts.index(img))
    return tuple(out)


PERM_VERTS = [_perm_of(m) for m in PERMS]


def compose(*idx):
    """Index of the map idx[0] o idx[1] o ... (the last applied first)."""
    p = (0, 1, 2)
    for i in reversed(idx):
        q = PERM_VERTS[i]
        p = tuple(q[a] for a in p)
    return PERM_VERTS.index(p)


def inverse(i):
    q = PERM_VERTS[i]
    inv = [0, 0, 0]
    for a, b in enumerate(q):
        inv[b] = a
    return PERM_VERTS.index(tuple(inv))


def perm_matrix(order, i):
    """Q[m][j] = int psi_m(sigma_i(chi)) psi_j(chi) / int psi_j^2 (psi_m o sigma_i in the basis)."""
    bfa = dgmat.basis_tri(order - 1)
    nf = len(bfa)
    mfa = [dgmat._int_tri(dgmat._pmul(bfa[j], bfa[j])) for j in range(nf)]
    maps = [dgmat._lin(c, k, 2) for c, k in PERMS[i]]
    tr = [dgmat._subs_affine(p, maps, 2) for p in bfa]
    return [[dgmat._int_tri(dgmat._pmul(tr[m], bfa[j])) / mfa[j] for j in range(nf)] for m in range(nf)]


def face_bases(order):
    """Per face FA: (sigma_FA, fluxL'_FA [B][F], fluxT'_FA [F][B]) with the sparsest face matrices
    (ties: the lowest permutation index)."""
    ex = dgmat.exact_matrices(order)
    nb, nf = dgmat.n_modes_tet(order), dgmat.n_modes_tri(order)
    out = []
    for f in range(4):
        proj = ex["fluxL"][f]
        best = None
        for i in range(3):  # rotations: the neighbour's map stays a reflection
            q = perm_matrix(order, i)
            pp = [[sum(q[m][j] * proj[k][j] for j in range(nf) if q[m][j]) for m in range(nf)] for k in range(nb)]
            nnz = sum(1 for k in range(nb) for m in range(nf) if pp[k][m] != 0)
            if best is None or nnz < best[0]:
                best = (nnz, i, pp)
        _, i, pp = best
        # fluxT'[m][n] = fluxL'[n][m] / |psi_m|^2 / |phi_n|^2 (same masses: sigma preserves area)
        minv = ex["massInv"]
        bfa = dgmat.basis_tri(order - 1)
        mfa_inv = [Fraction(1) / dgmat._int_tri(dgmat._pmul(bfa[m], bfa[m])) for m in range(nf)]
        ft = [[pp[n][m] * mfa_inv[m] * minv[n] for n in range(nb)] for m in range(nf)]
        out.append((i, pp, ft))
    return out


def face_perm_table(sig):
    """V[fo][FA][v]: sigma_fo o sigma_v o sigma_FA^-1 = sigma_V (sigma_v = PERMS[3 + v], a reflection)."""
    out = [[[compose(sig[fo], 3 + v, inverse(sig[fa])) for v in range(3)] for fa in range(4)] for fo in range(4)]
    assert all(x >= 3 for a in out for b in a for x in b), "face permutations must stay reflections"
    return [[[x - 3 for x in b] for b in a] for a in out]


def exact_orientations(order):
    """(Mface^-1 Ori_P)[k][j] for the permutations P of PERMS, exact (same construction as
    dgmat.exact_matrices)."""
    deg = order - 1
    bfa = dgmat.basis_tri(deg)
    nf = len(bfa)
    mass_fa = [[dgmat._int_tri(dgmat._pmul(bfa[i], bfa[j])) for j in range(nf)] for i in range(nf)]
    minv = [Fraction(1) / mass_fa[i][i] for i in range(nf)]
    out = []
    for mp in PERMS:
        maps = [dgmat._lin(c, k, 2) for c, k in mp]
        tr = [dgmat._subs_affine(p, maps, 2) for p in bfa]
        ori = [[dgmat._int_tri(dgmat._pmul(tr[i], bfa[j])) for j in range(nf)] for i in range(nf)]
        out.append([[minv[k] * ori[k][j] for j in range(nf)] for k in range(nf)])
    return out


if __name__ == "__main__":
    print(main())
