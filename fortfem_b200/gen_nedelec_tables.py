"""Exact-rational generator for the first-kind tetrahedral Nedelec tables.

Writes ``fortfem_b200/csrc/nedelec_tables.inc``: for orders 1..6 the dual-basis
coefficient matrix C = M^-1 of the monomial candidate space, and for orders
2..6 the 6 face basis-to-local transforms.  Everything is computed with Python
``fractions`` and rounded to the nearest double only when written.

The definitions restate the reference:

* candidates (3 monomial component families, the two x-cross families and the
  y/z family) -- ``src/elements/tetra_nedelec_arbitrary_order.f90:318-396``
  (runtime) and the generated ``fortfem_tetra_nedelec_candidates_order_*``;
* moments: shifted-Legendre edge moments along the reference tangents, face
  monomial moments against the two face tangents in face parameter space, and
  volume monomial moments -- ``tetra_nedelec_arbitrary_order.f90:203-315`` and
  the exact generator ``tools/codegen/app/gen_tetra_nedelec_coefficients.f90:50-200``;
* face transform = L C^-1 of the face moment matrices under a vertex
  permutation -- ``src/elements/tetra_face_moment_transforms.f90:296-383``.

Order 6 keeps the monomial candidate space but, as the reference does from
order 6, weights the face moments with Dubiner modes and the volume moments
with Koornwinder modes (``tetra_nedelec_arbitrary_order.f90:642-669``).  Those
polynomials come from fortnum in the reference (not vendored); here they are
restated from their standard collapsed-coordinate definitions, so equality
of the order-6 basis with the reference's depends on fortnum's normalisation
and is unpinned; basis-invariant quantities (energies, solutions) compare.

Order 1..4 tables are pinned against the reference's generated tables by
``tests/golden/nedelec_tables.json`` (see ``tests/golden/make_golden.py``).
Run ``python -m fortfem_b200.gen_nedelec_tables`` to regenerate.
"""
from __future__ import annotations

import itertools
import os
from fractions import Fraction
from math import factorial

REF_VERTS = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]
EDGES = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
FACES = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
PERMUTATIONS = [(1, 2, 3), (1, 3, 2), (2, 1, 3), (2, 3, 1), (3, 1, 2), (3, 2, 1)]
MAX_ORDER = 6


def dof_count(k: int) -> int:
    return k * (k + 2) * (k + 3) // 2


# ---------------------------------------------------------------- polynomials
# A scalar polynomial is a dict {(a, b, c): Fraction}; a candidate is a list of
# three such dicts (x, y, z components).

def candidates(k: int):
    cands = []
    for comp in range(3):
        for d in range(k):
            for a in range(d + 1):
                for b in range(d - a + 1):
                    c = d - a - b
                    v = [dict(), dict(), dict()]
                    v[comp][(a, b, c)] = Fraction(1)
                    cands.append(v)
    d = k - 1
    for fam in (4, 5):
        for a in range(d + 1):
            for b in range(d - a + 1):
                c = d - a - b
                v = [dict(), dict(), dict()]
                if fam == 4:
                    v[0][(a, b + 1, c)] = Fraction(-1)
                    v[1][(a + 1, b, c)] = Fraction(1)
                else:
                    v[0][(a, b, c + 1)] = Fraction(-1)
                    v[2][(a + 1, b, c)] = Fraction(1)
                cands.append(v)
    for b in range(d + 1):
        c = d - b
        v = [dict(), dict(), dict()]
        v[1][(0, b, c + 1)] = Fraction(-1)
        v[2][(0, b + 1, c)] = Fraction(1)
        cands.append(v)
    assert len(cands) == dof_count(k)
    return cands


def shifted_legendre(m: int):
    """Coefficients of P_m(2t-1) in powers of t (exact)."""
    # P_m(2t-1) = sum_j (-1)^(m+j) C(m,j) C(m+j,j) t^j
    from math import comb
    return [Fraction((-1) ** (m + j) * comb(m, j) * comb(m + j, j)) for j in range(m + 1)]


def poly1_mul(p, q):
    r = [Fraction(0)] * (len(p) + len(q) - 1)
    for i, a in enumerate(p):
        if a:
            for j, b in enumerate(q):
                r[i + j] += a * b
    return r


def poly1_pow_affine(c0, c1, n):
    p = [Fraction(1)]
    for _ in range(n):
        p = poly1_mul(p, [Fraction(c0), Fraction(c1)])
    return p


def tet_monomial(a, b, c):
    return Fraction(factorial(a) * factorial(b) * factorial(c), factorial(a + b + c + 3))


def tri_monomial(a, b):
    return Fraction(factorial(a) * factorial(b), factorial(a + b + 2))


def poly2_mul(p, q):
    r = {}
    for (i1, j1), a in p.items():
        for (i2, j2), b in q.items():
            key = (i1 + i2, j1 + j2)
            r[key] = r.get(key, Fraction(0)) + a * b
    return r


def affine2_pow(c0, cu, cv, n):
    p = {(0, 0): Fraction(1)}
    lin = {}
    if c0:
        lin[(0, 0)] = Fraction(c0)
    if cu:
        lin[(1, 0)] = Fraction(cu)
    if cv:
        lin[(0, 1)] = Fraction(cv)
    for _ in range(n):
        p = poly2_mul(p, lin)
    return p


def edge_moment(poly, e, m):
    """int_0^1 L_m(t) poly(v_a + t t_e) dt for a scalar monomial dict."""
    va, vb = REF_VERTS[EDGES[e][0]], REF_VERTS[EDGES[e][1]]
    te = [vb[d] - va[d] for d in range(3)]
    leg = shifted_legendre(m)
    total = Fraction(0)
    for (a, b, c), coef in poly.items():
        p = [Fraction(1)]
        for d, n in enumerate((a, b, c)):
            p = poly1_mul(p, poly1_pow_affine(va[d], te[d], n))
        p = poly1_mul(p, leg)
        total += coef * sum(x / (i + 1) for i, x in enumerate(p))
    return total


def face_integral(poly, f, ma, mb):
    """int_T u^ma v^mb poly(v_a + u t1 + v t2) du dv over the unit triangle."""
    va, vb, vc = (REF_VERTS[i] for i in FACES[f])
    t1 = [vb[d] - va[d] for d in range(3)]
    t2 = [vc[d] - va[d] for d in range(3)]
    total = Fraction(0)
    for (a, b, c), coef in poly.items():
        p = {(0, 0): Fraction(1)}
        for d, n in enumerate((a, b, c)):
            p = poly2_mul(p, affine2_pow(va[d], t1[d], t2[d], n))
        for (i, j), x in p.items():
            total += coef * x * tri_monomial(i + ma, j + mb)
    return total


# ------------------------------------------- orthogonal moment weights (k >= 6)
# From order 6 the reference weights face moments by triangle_dubiner and
# volume moments by tetrahedron_koornwinder (tetra_nedelec_arbitrary_order.f90:
# 642-668) instead of monomials.  They are restated here with the standard
# collapsed-coordinate definitions on the reference triangle / tetrahedron
# (Dubiner 1991, Koornwinder 1975; Jacobi polynomials P_n^(alpha,0)), built
# exactly as polynomials with rational coefficients.

def jacobi(n: int, alpha: int):
    """Coefficients of P_n^(alpha,0)(t) in powers of t (exact)."""
    from math import comb
    out = [Fraction(0)] * (n + 1)
    for s_ in range(n + 1):
        c = Fraction(comb(n + alpha, n - s_) * comb(n, s_))
        # ((t-1)/2)^s ((t+1)/2)^(n-s)
        p = poly1_mul(poly1_pow_affine(Fraction(-1, 2), Fraction(1, 2), s_),
                      poly1_pow_affine(Fraction(1, 2), Fraction(1, 2), n - s_))
        for i, x in enumerate(p):
            out[i] += c * x
    return out


def _polyn_mul(p, q):
    r = {}
    for e1, a in p.items():
        for e2, b in q.items():
            key = tuple(x + y for x, y in zip(e1, e2))
            r[key] = r.get(key, Fraction(0)) + a * b
    return {k_: v for k_, v in r.items() if v != 0}


def _polyn_pow(p, n, dim):
    r = {(0,) * dim: Fraction(1)}
    for _ in range(n):
        r = _polyn_mul(r, p)
    return r


def _polyn_add(p, q, scale=Fraction(1)):
    r = dict(p)
    for k_, v in q.items():
        r[k_] = r.get(k_, Fraction(0)) + scale * v
    return {k_: v for k_, v in r.items() if v != 0}


def _collapsed(coef_t, num, den, degree, dim):
    """den^degree * P(num/den) for P = sum coef_t[i] t^i (num, den linear polys)."""
    out = {}
    for i, c in enumerate(coef_t):
        if c:
            term = _polyn_mul(_polyn_pow(num, i, dim), _polyn_pow(den, degree - i, dim))
            out = _polyn_add(out, term, c)
    return out


def dubiner(p: int, q: int):
    """Dubiner polynomial psi_pq(x, y) on the triangle (0,0),(1,0),(0,1)."""
    one_minus_y = {(0, 0): Fraction(1), (0, 1): Fraction(-1)}
    a_num = {(1, 0): Fraction(2), (0, 0): Fraction(-1), (0, 1): Fraction(1)}  # 2x - 1 + y
    A = _collapsed(jacobi(p, 0), a_num, one_minus_y, p, 2)
    B = _collapsed(jacobi(q, 2 * p + 1), {(0, 1): Fraction(2), (0, 0): Fraction(-1)},
                   {(0, 0): Fraction(1)}, q, 2)
    return _polyn_mul(A, B)


def koornwinder(p: int, q: int, r: int):
    """Koornwinder polynomial phi_pqr(x, y, z) on the unit tetrahedron."""
    e = lambda x, y, z: (x, y, z)  # noqa: E731
    one_yz = {e(0, 0, 0): Fraction(1), e(0, 1, 0): Fraction(-1), e(0, 0, 1): Fraction(-1)}
    a_num = {e(1, 0, 0): Fraction(2), e(0, 0, 0): Fraction(-1), e(0, 1, 0): Fraction(1),
             e(0, 0, 1): Fraction(1)}                                    # 2x - 1 + y + z
    one_z = {e(0, 0, 0): Fraction(1), e(0, 0, 1): Fraction(-1)}
    b_num = {e(0, 1, 0): Fraction(2), e(0, 0, 0): Fraction(-1), e(0, 0, 1): Fraction(1)}  # 2y-1+z
    A = _collapsed(jacobi(p, 0), a_num, one_yz, p, 3)
    B = _collapsed(jacobi(q, 2 * p + 1), b_num, one_z, q, 3)
    C = _collapsed(jacobi(r, 2 * p + 2 * q + 2), {e(0, 0, 1): Fraction(2), e(0, 0, 0): Fraction(-1)},
                   {e(0, 0, 0): Fraction(1)}, r, 3)
    return _polyn_mul(_polyn_mul(A, B), C)


def face_weight(k: int, a: int, b: int):
    """Face moment weight in face coordinates: u^a v^b (k <= 5) or Dubiner (k >= 6)."""
    return {(a, b): Fraction(1)} if k <= 5 else dubiner(a, b)


def volume_weight(k: int, a: int, b: int, c: int):
    return {(a, b, c): Fraction(1)} if k <= 5 else koornwinder(a, b, c)


def moment_matrix(k: int):
    cands = candidates(k)
    n = len(cands)
    rows = []
    for e in range(6):
        va, vb = REF_VERTS[EDGES[e][0]], REF_VERTS[EDGES[e][1]]
        te = [vb[d] - va[d] for d in range(3)]
        for m in range(k):
            row = []
            for cand in cands:
                s = Fraction(0)
                for comp in range(3):
                    if te[comp] and cand[comp]:
                        s += te[comp] * edge_moment(cand[comp], e, m)
                row.append(s)
            rows.append(row)
    for f in range(4):
        va, vb, vc = (REF_VERTS[i] for i in FACES[f])
        tangents = ([vb[d] - va[d] for d in range(3)], [vc[d] - va[d] for d in range(3)])
        for tcomp in range(2):
            t = tangents[tcomp]
            for d in range(k - 1):
                for ma in range(d + 1):
                    mb = d - ma
                    w = face_weight(k, ma, mb)
                    row = []
                    for ci, cand in enumerate(cands):
                        s = Fraction(0)
                        for comp in range(3):
                            if t[comp] and cand[comp]:
                                for (wa, wb), wc in w.items():
                                    s += t[comp] * wc * _face_int(k, ci, comp, f, wa, wb, cand)
                        row.append(s)
                    rows.append(row)
    for comp in range(3):
        for d in range(k - 2):
            for a in range(d + 1):
                for b in range(d - a + 1):
                    c = d - a - b
                    w = volume_weight(k, a, b, c)
                    row = []
                    for cand in cands:
                        s = Fraction(0)
                        for (pa, pb, pc), coef in cand[comp].items():
                            for (wa, wb, wc), wv in w.items():
                                s += coef * wv * tet_monomial(pa + wa, pb + wb, pc + wc)
                        row.append(s)
                    rows.append(row)
    assert len(rows) == n
    return rows


_FACE_CACHE = {}


def _face_int(k, ci, comp, f, ma, mb, cand):
    key = (k, ci, comp, f, ma, mb)
    if key not in _FACE_CACHE:
        _FACE_CACHE[key] = face_integral(cand[comp], f, ma, mb)
    return _FACE_CACHE[key]


def exact_inverse(M):
    n = len(M)
    A = [list(r) + [Fraction(int(i == j)) for j in range(n)] for i, r in enumerate(M)]
    for col in range(n):
        piv = next(r for r in range(col, n) if A[r][col] != 0)
        A[col], A[piv] = A[piv], A[col]
        pv = A[col][col]
        inv = 1 / pv
        A[col] = [x * inv for x in A[col]]
        for r in range(n):
            if r != col and A[r][col] != 0:
                f = A[r][col]
                Ar, Ac = A[r], A[col]
                A[r] = [x - f * y for x, y in zip(Ar, Ac)]
    return [row[n:] for row in A]


def coefficients(k: int):
    """Dual-basis coefficients C (n_b x n_b, C[candidate][basis]) as Fractions."""
    return exact_inverse(moment_matrix(k))


# -------------------------------------------------------- face transforms

def _perm_map(perm):
    v2 = [(0, 0), (1, 0), (0, 1)]
    off = v2[perm[0] - 1]
    a1 = (v2[perm[1] - 1][0] - off[0], v2[perm[1] - 1][1] - off[1])
    a2 = (v2[perm[2] - 1][0] - off[0], v2[perm[2] - 1][1] - off[1])
    # affine(row=coordinate, col=edge)
    affine = [[a1[0], a2[0]], [a1[1], a2[1]]]
    return off, affine


def face_moment_matrix(k: int, perm):
    off, aff = _perm_map(perm)
    idx = []
    for comp in range(2):
        for d in range(k - 1):
            for a in range(d + 1):
                idx.append((comp, a, d - a))
    n = len(idx)
    M = [[Fraction(0)] * n for _ in range(n)]
    for col, (bc, bx, by) in enumerate(idx):
        # mapped = off + aff @ (u, v); poly = weight(bx, by) at the mapped point
        pm = {}
        for (wx, wy), wc in face_weight(k, bx, by).items():
            px = affine2_pow(off[0], aff[0][0], aff[0][1], wx)
            py = affine2_pow(off[1], aff[1][0], aff[1][1], wy)
            for key, x in poly2_mul(px, py).items():
                pm[key] = pm.get(key, Fraction(0)) + wc * x
        for row, (mc, mx, my) in enumerate(idx):
            scale = aff[bc][mc]
            if scale == 0:
                continue
            s = Fraction(0)
            for (wx, wy), wc in face_weight(k, mx, my).items():
                for (i, j), x in pm.items():
                    s += wc * x * tri_monomial(i + wx, j + wy)
            M[row][col] = scale * s
    return M


def face_transform(k: int, perm):
    """basis_to_local transform = L C^-1 (tetra_face_moment_transforms.f90:296-327)."""
    C = face_moment_matrix(k, (1, 2, 3))
    L = face_moment_matrix(k, perm)
    Ci = exact_inverse(C)
    n = len(C)
    return [[sum(L[i][m] * Ci[m][j] for m in range(n)) for j in range(n)] for i in range(n)]


# --------------------------------------------------------------- emitter

def _fmt(x: Fraction) -> str:
    return float(x).hex()


def emit(path: str, max_order: int = MAX_ORDER) -> None:
    lines = [
        "// Generated by fortfem_b200/gen_nedelec_tables.py from exact rational",
        "// arithmetic; do not edit.  Column-major (row + n*col) doubles rounded to",
        "// nearest from the exact values.",
        "#pragma once",
        f"#define FFG_NEDELEC_TABLE_MAX_ORDER {max_order}",
    ]
    for k in range(1, max_order + 1):
        C = coefficients(k)
        n = len(C)
        vals = ", ".join(_fmt(C[r][c]) for c in range(n) for r in range(n))
        lines.append(f"static const double kNedelecCoefficients{k}[{n * n}] = {{{vals}}};")
    for k in range(2, max_order + 1):
        m = k * (k - 1)
        blocks = []
        for perm in PERMUTATIONS:
            T = face_transform(k, perm)
            blocks.append("{" + ", ".join(_fmt(T[r][c]) for c in range(m) for r in range(m)) + "}")
        lines.append(f"static const double kFaceTransform{k}[6][{m * m}] = {{{', '.join(blocks)}}};")
    lines.append("static const double *const kNedelecCoefficientTables[] = {nullptr, " +
                 ", ".join(f"kNedelecCoefficients{k}" for k in range(1, max_order + 1)) + "};")
    lines.append("static const double *kFaceTransformTable(int k, int perm_index) {")
    lines.append("  switch (k) {")
    for k in range(2, max_order + 1):
        lines.append(f"    case {k}: return kFaceTransform{k}[perm_index];")
    lines.append("    default: return nullptr;")
    lines.append("  }")
    lines.append("}")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    emit(os.path.join(here, "csrc", "nedelec_tables.inc"))
