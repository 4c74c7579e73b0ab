"""Solution evaluation and point probes on the GPU, through the C-ABI.

Parity against the oracle's restatement of evaluate_tetra_lagrange_solution
(_prepared / _at_point) and evaluate_box_solution_order / probe_box_* (values
within relative 1e-12, per-query statuses and contributing-cell counts
exact), the reference's own known answers (test/
test_tetra_lagrange_poisson_p_convergence.f90: affine Dirichlet data and the
reaction problem reproduced to 1e-12), and at a larger size the property
that a field of the discrete space is returned exactly wherever it is probed.
"""
import numpy as np
import pytest

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K
from fortfem_b200 import synth

pytestmark = pytest.mark.gpu


# The field is sum_b ld_b sum_c C[c, b] cand_c(xi) with the exact dual-basis
# coefficients C, whose largest entries grow with the order (1, 16, 810,
# 7.3e4, 7.3e6, 1.1e7 for orders 1..6) while the field stays O(1): the
# cancellation costs digits in any summation order, so the oracle and the
# GPU (which sum in different orders) agree to about 1e-15 max|C|.
NEDELEC_TOL = {1: 1e-12, 2: 1e-12, 3: 1e-12, 4: 1e-10, 5: 1e-8, 6: 1e-8}


def jittered_box(n, delta=0.1, seed=7):
    v, t = oracle.box_mesh([n, n, n])
    return synth.jitter_interior(v, 1.0 / n, delta, seed), t


def close(a, b, rel=1e-12):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b).max() <= rel * max(1.0, np.abs(b).max())


def queries(v, t, rng, n):
    """Random (cell, reference point) queries, some outside the reference cell
    and some with a cell index out of range."""
    cells = rng.integers(0, len(t), n)
    xi = rng.dirichlet([1, 1, 1, 1], n)[:, 1:]
    xi[::7] += 0.4                 # outside the reference cell
    cells[::11] = len(t) + 3       # no such cell
    return cells.astype(np.int32), xi


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_lagrange_evaluate_matches_oracle(p):
    v, t = jittered_box(3)
    rng = np.random.default_rng(p)
    with ff.Problem(K.FFG_TETRA_LAGRANGE, p, t, len(v), boundary="none") as P:
        u = rng.standard_normal(P.n_dofs)
        cells, xi = queries(v, t, rng, 60)
        val, grad, qst = P.evaluate(v, u, cells, xi)
        # the same queries as physical points
        phys = np.array([v[t[c % len(t), 0]] + (v[t[c % len(t), 1:]] - v[t[c % len(t), 0]]).T @ x
                         for c, x in zip(cells, xi)])
        pval, pgrad, pst = P.evaluate(v, u, cells, phys, physical=True)
    for i, (c, x) in enumerate(zip(cells, xi)):
        ref = oracle.lagrange_evaluate_solution(v, t, p, u, int(c), x)
        if ref is None:
            assert qst[i] == K.FFG_INVALID_INPUT
            continue
        assert qst[i] == 0
        assert close(val[i], ref[0]) and close(grad[i], ref[1], 1e-11)
        refp = oracle.lagrange_evaluate_solution(v, t, p, u, int(c), phys[i], physical=True)
        assert (pst[i] == 0) == (refp is not None)
        if refp is not None:
            assert close(pval[i], refp[0]) and close(pgrad[i], refp[1], 1e-11)


def test_reference_affine_and_reaction_kat():
    # test_tetra_lagrange_poisson_p_convergence.f90:133-181 through the GPU
    # solve and the GPU evaluator
    t = np.array([[0, 1, 2, 4], [0, 3, 1, 4], [0, 2, 3, 4], [1, 3, 2, 4]], np.int32)
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.25, 0.25, 0.25]], float)
    affine = lambda x, y, z: 1.0 + x + 2.0 * y - 3.0 * z
    opts = ff.solver_options(precision="fp64", tolerance=1e-14, preconditioner="jacobi",
                             max_iterations=100)
    u, st, _ = ff.solve_tetra_lagrange_poisson(v, t, 1, lambda x, y, z: 0.0 * x, affine, opts)
    assert st.code == 0
    value, grad, code = ff.evaluate_tetra_lagrange_solution(v, t, 1, u, 0, [0.2, 0.3, 0.1])
    assert code == 0
    assert abs(value - affine(0.225, 0.325, 0.025)) < 1e-12
    assert np.abs(grad - [1.0, 2.0, -3.0]).max() < 1e-12
    u, st, _ = ff.solve_tetra_lagrange_diffusion_reaction(v, t, 1, lambda x, y, z: 2.0 + 0 * x,
                                                           0.0, 1.0, options=opts)
    assert st.code == 0
    value, grad, code = ff.evaluate_tetra_lagrange_solution(v, t, 1, u, 3, [0.2, 0.1, 0.3])
    assert code == 0 and abs(value - 2.0) < 1e-12 and np.abs(grad).max() < 1e-12


def probe_points(v, t, rng, n):
    pts = rng.uniform(-0.05, 1.05, (n, 3))      # some outside the box
    pts[: len(v) // 4] = v[: len(v) // 4]        # mesh vertices: many cells each
    mids = 0.5 * (v[t[:, 0]] + v[t[:, 1]])       # edge midpoints
    pts[len(v) // 4: len(v) // 4 + 10] = mids[:10]
    return pts


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("mode", ["average", "first"])
def test_lagrange_probe_matches_oracle(p, mode):
    v, t = jittered_box(3)
    rng = np.random.default_rng(10 + p)
    pts = probe_points(v, t, rng, 80)
    with ff.Problem(K.FFG_TETRA_LAGRANGE, p, t, len(v), boundary="none") as P:
        u = rng.standard_normal(P.n_dofs)
        val, grad, cnt = P.probe(v, u, pts, mode)
    m = 0 if mode == "average" else 1
    for i, x in enumerate(pts):
        rv, rg, rc = oracle.lagrange_probe(v, t, p, u, x, m)
        assert cnt[i] == rc
        if rc > 0:
            assert close(val[i], rv) and close(grad[i], rg, 1e-11)
    assert (cnt == 0).any() and ((cnt > 1).any() if m == 0 else (cnt <= 1).all())


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6])
def test_nedelec_evaluate_matches_oracle(k):
    v, t = jittered_box(2, 0.1, 11)
    rng = np.random.default_rng(20 + k)
    with ff.Problem(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary="none") as P:
        u = rng.standard_normal(P.n_dofs)
        cells, xi = queries(v, t, rng, 30)
        val, curl, qst = P.evaluate(v, u, cells, xi)
    tol = NEDELEC_TOL[k]
    for i, (c, x) in enumerate(zip(cells, xi)):
        ref = oracle.nedelec_evaluate_solution(v, t, k, u, int(c), x)
        if ref is None:
            assert qst[i] == K.FFG_INVALID_INPUT
            continue
        assert qst[i] == 0
        assert close(val[i], ref[0], tol) and close(curl[i], ref[1], tol)


@pytest.mark.parametrize("k", [1, 2, 3, 4])
@pytest.mark.parametrize("mode", ["average", "first"])
def test_nedelec_probe_matches_oracle(k, mode):
    v, t = jittered_box(2, 0.1, 11)
    rng = np.random.default_rng(30 + k)
    pts = probe_points(v, t, rng, 40)
    with ff.Problem(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary="none") as P:
        u = rng.standard_normal(P.n_dofs)
        val, curl, cnt = P.probe(v, u, pts, mode)
    m = 0 if mode == "average" else 1
    tol = NEDELEC_TOL[k]
    for i, x in enumerate(pts):
        rv, rc, rn = oracle.nedelec_probe(v, t, k, u, x, m)
        assert cnt[i] == rn
        if rn > 0:
            assert close(val[i], rv, tol), np.abs(val[i] - rv).max()
            assert close(curl[i], rc, tol), np.abs(curl[i] - rc).max()
    assert (cnt == 0).any() and ((cnt > 1).any() if m == 0 else (cnt <= 1).all())


def test_full_size_probe_returns_the_discrete_field():
    # 24^3 box (82,944 cells), P2: the nodal interpolant of a quadratic is the
    # quadratic, so 100,000 probes return it and its gradient; the first-cell
    # and average modes agree on the value; cell-hinted evaluation at the
    # same physical points agrees with the probe
    v, t = jittered_box(24, 0.15, 5)
    f = lambda x: 1.0 + x[:, 0] * x[:, 1] - 2.0 * x[:, 2] ** 2 + 0.5 * x[:, 0]
    df = lambda x: np.stack([x[:, 1] + 0.5, x[:, 0], -4.0 * x[:, 2]], 1)
    with ff.Problem(K.FFG_TETRA_LAGRANGE, 2, t, len(v), boundary="none") as P:
        u = f(P.dof_points(v))
        pts = np.random.default_rng(3).uniform(0.0, 1.0, (100000, 3))
        val, grad, cnt = P.probe(v, u, pts)
        assert (cnt >= 1).all()
        assert np.abs(val - f(pts)).max() < 1e-12
        assert np.abs(grad - df(pts)).max() < 1e-10
        val1, _, cnt1 = P.probe(v, u, pts, "first")
        assert (cnt1 == 1).all() and np.abs(val1 - val).max() < 1e-12
        # locate with the probe's own rule on the host for a sample, then evaluate
        sample = pts[:200]
        cells = np.array([oracle_first_cell(v, t, x) for x in sample], np.int32)
        ev, eg, est = P.evaluate(v, u, cells, sample, physical=True)
        assert (est == 0).all() and np.abs(ev - val[:200]).max() < 1e-12


def oracle_first_cell(v, t, x):
    J = np.transpose(v[t[:, 1:]] - v[t[:, :1]], (0, 2, 1))
    xi = np.linalg.solve(J, (x - v[t[:, 0]])[:, :, None])[:, :, 0]
    inside = (xi >= -1e-12).all(1) & (xi.sum(1) <= 1 + 1e-12)
    return int(np.argmax(inside))


def test_degenerate_mesh_and_bad_input():
    v, t = jittered_box(2)
    flat = v.copy()
    flat[t[0, 3]] = flat[t[0, 0]] + 0.5 * (flat[t[0, 1]] - flat[t[0, 0]]) + \
        0.5 * (flat[t[0, 2]] - flat[t[0, 0]])
    with ff.Problem(K.FFG_TETRA_LAGRANGE, 1, t, len(v), boundary="none") as P:
        u = np.ones(P.n_dofs)
        with pytest.raises(ff.FortfemError) as e:
            P.evaluate(flat, u, [1], [[0.1, 0.1, 0.1]])
        assert e.value.code == K.FFG_INVALID_INPUT
        with pytest.raises(ff.FortfemError):
            P.evaluate(v, u[:-1], [1], [[0.1, 0.1, 0.1]])
        val, grad, qst = P.evaluate(v, u, [], np.zeros((0, 3)))
        assert val.size == 0
