"""Arbitrary-order triangle Lagrange assembly and solve on the GPU, through the
C-ABI: CSC patterns bit-exact and values within relative Frobenius 1e-12 of
the oracle (degrees 1..6, cellwise coefficients, both triangle orientations),
the load within 1e-12, degree 1 equal to the P1 forms, and the discrete
space's exactness: a Poisson problem whose solution is a polynomial of the
degree is solved to the nodal values."""
import numpy as np
import pytest

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K

pytestmark = pytest.mark.gpu


def rel_frob(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def mesh(n, seed=3):
    v, t = oracle.unit_square_mesh(n)
    rng = np.random.default_rng(seed)
    inner = (v[:, 0] > 0) & (v[:, 0] < 1) & (v[:, 1] > 0) & (v[:, 1] < 1)
    v = v.copy()
    v[inner] += rng.uniform(-0.15, 0.15, (inner.sum(), 2)) / (n - 1)
    t = t.copy()
    t[::3] = t[::3][:, [0, 2, 1]]          # mixed orientations
    return v, t


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6])
def test_csc_and_load_match_oracle(p):
    v, t = mesh(7)
    rng = np.random.default_rng(p)
    cs = np.exp(rng.standard_normal(len(t)))
    cm = rng.uniform(0.5, 2.0, len(t))
    q = 2 * p
    A, st = ff.assemble_triangle_lagrange_csc(v, t, p, q, 1.3, 0.7, cs, cm)
    assert st.code == 0
    n, cp, ri, val = oracle.triangle_lagrange_csc(v, t, p, q, 1.3, 0.7, cs, cm)
    assert A.nrow == n and np.array_equal(A.col_ptr, cp) and np.array_equal(A.row_idx, ri)
    assert rel_frob(A.val, val) <= 1e-12
    sp, _ = oracle.triangle_lagrange_points(v, t, p, q)
    src = np.sin(3 * sp[..., 0]) + sp[..., 1] ** 2
    rhs, st = ff.assemble_triangle_lagrange_load_samples(v, t, p, src, q)
    assert st.code == 0
    assert rel_frob(rhs, oracle.triangle_lagrange_load_samples(v, t, p, q, src)) <= 1e-12


def test_degree_one_is_the_p1_form():
    v, t = mesh(9)
    A, st = ff.assemble_triangle_lagrange_csc(v, t, 1, 2, 1.1, 0.4)
    assert st.code == 0
    B, st = ff.assemble_scalar_p1_csc(v, t, 0.4, 1.1)
    gd, n = oracle.triangle_lagrange_dof_map(1, t)
    _, pw = oracle.triangle_lagrange_nodes(1)
    dof_vertex = np.zeros(n, int)
    for c in range(len(t)):
        dof_vertex[gd[c]] = t[c][pw.argmax(axis=1)]
    a = oracle.csc_to_scipy(n, A.col_ptr, A.row_idx, A.val).toarray()
    b = oracle.csc_to_scipy(B.nrow, B.col_ptr, B.row_idx, B.val).toarray()
    assert np.abs(a - b[np.ix_(dof_vertex, dof_vertex)]).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.parametrize("p", [2, 3, 4])
def test_polynomial_solution_is_reproduced(p):
    # -lap u = f with u = x^2 + x y - y^2 / 2 + x^p: in the space of degree p
    v, t = mesh(9, 5)
    u = lambda x, y: x ** 2 + x * y - 0.5 * y ** 2 + x ** p
    f = lambda x, y: -(2.0 - 1.0 + p * (p - 1) * x ** (p - 2))
    opts = ff.solver_options(precision="mixed", tolerance=1e-12, preconditioner="jacobi",
                             max_iterations=100000)
    sol, st, stats = ff.solve_triangle_lagrange(v, t, p, f, 1.0, 0.0, u, opts)
    assert st.code == 0
    with ff.Problem(K.FFG_TRIANGLE_LAGRANGE, p, t, len(v), quadrature_degree=2 * p) as P:
        dp = P.dof_points(v)
    assert np.abs(sol - u(dp[:, 0], dp[:, 1])).max() < 1e-9
