"""GPU parity of the sm_100a path against the FP64 CPU oracle (through the C-ABI).

Tolerances: CSC patterns and integer maps bit-exact; FP64-geometry assembled
values within relative Frobenius 1e-12 of the oracle (1e-11 at Nedelec order
5, whose tables carry larger entries); loads 1e-12; solutions against the
oracle's FP64 solve within the stated residual-derived bounds.
"""
import numpy as np
import pytest

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K
from fortfem_b200 import synth

pytestmark = pytest.mark.gpu

FROB = 1e-12


def rel_frob(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def jittered_box(n, delta=0.1, seed=7):
    v, t = oracle.box_mesh([n, n, n])
    return synth.jitter_interior(v, 1.0 / n, delta, seed), t


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("rule", [0, 1])
def test_lagrange_csc_matches_oracle(p, rule):
    v, t = jittered_box(3)
    rng = np.random.default_rng(p)
    cs = np.exp(rng.standard_normal(len(t)))
    cm = rng.uniform(0.5, 2.0, len(t))
    q = 2 * p + 4
    A, st = ff.assemble_tetra_lagrange_stiffness_csc(v, t, p, q, 1.3, 0.7, rule=rule,
                                                     cell_stiffness=cs, cell_mass=cm)
    assert st.code == 0
    n, cp, ri, val = oracle.lagrange_csc(v, t, p, rule, q, 1.3, 0.7, cs, cm)
    assert A.nrow == n and np.array_equal(A.col_ptr, cp) and np.array_equal(A.row_idx, ri)
    assert rel_frob(A.val, val) <= FROB


@pytest.mark.parametrize("p", [1, 2, 3])
def test_lagrange_load_matches_oracle(p):
    v, t = jittered_box(3)
    q = 2 * p + 4
    pts = oracle.lagrange_quadrature_points(v, t, 0, q)
    src = np.sin(pts[..., 0]) * np.cos(2 * pts[..., 1]) + pts[..., 2]
    rhs, st = ff.assemble_tetra_lagrange_scalar_load_samples(v, t, p, q, src)
    assert st.code == 0
    ref = oracle.lagrange_load_samples(v, t, p, src, 0, q)
    assert rel_frob(rhs, ref) <= FROB


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_nedelec_csc_matches_oracle(k):
    v, t = jittered_box(2, 0.1, 11)
    rng = np.random.default_rng(k)
    cc = rng.uniform(0.5, 2.0, len(t))
    cm = rng.uniform(0.5, 2.0, len(t))
    A, st = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, 1.7, 0.9, order=k, cell_curl=cc,
                                                    cell_mass=cm)
    assert st.code == 0
    n, cp, ri, val = oracle.nedelec_csc(v, t, k, 1.7, 0.9, cc, cm)
    assert A.nrow == n and np.array_equal(A.col_ptr, cp) and np.array_equal(A.row_idx, ri)
    assert rel_frob(A.val, val) <= (1e-11 if k == 5 else FROB)


# order 6: the element matrix (216 x 216) is built in global memory instead of
# shared memory; a 6-cell mesh keeps the oracle's quadrature loop short
def test_nedelec_order6_csc_and_load_match_oracle():
    k = 6
    v, t = jittered_box(1, 0.0, 11)
    rng = np.random.default_rng(6)
    cc = rng.uniform(0.5, 2.0, len(t))
    cm = rng.uniform(0.5, 2.0, len(t))
    A, st = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, 1.7, 0.9, order=k, cell_curl=cc,
                                                    cell_mass=cm)
    assert st.code == 0
    n, cp, ri, val = oracle.nedelec_csc(v, t, k, 1.7, 0.9, cc, cm)
    assert A.nrow == n == 1014 and np.array_equal(A.col_ptr, cp) and np.array_equal(A.row_idx, ri)
    assert rel_frob(A.val, val) <= 1e-10
    pts = oracle.nedelec_load_points(v, t, k)
    src = np.stack([np.sin(pts[..., 1]), pts[..., 0] * pts[..., 2], np.cos(pts[..., 0])], -1)
    rhs, st = ff.assemble_tetra_nedelec_vector_load_samples(v, t, k, src)
    assert st.code == 0
    assert rel_frob(rhs, oracle.nedelec_load_samples(v, t, k, src)) <= 1e-10


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_nedelec_load_matches_oracle(k):
    v, t = jittered_box(2, 0.1, 3)
    pts = oracle.nedelec_load_points(v, t, k)
    src = np.stack([np.sin(pts[..., 1]), pts[..., 0] * pts[..., 2], np.cos(pts[..., 0])], -1)
    rhs, st = ff.assemble_tetra_nedelec_vector_load_samples(v, t, k, src)
    assert st.code == 0
    ref = oracle.nedelec_load_samples(v, t, k, src)
    assert rel_frob(rhs, ref) <= FROB


def relabelled_box(n, seed):
    """A jittered box mesh with its vertices renumbered at random: every
    cell's orientation (edge signs, face permutations) follows the order of
    its global vertex indices, so all 24 orders appear."""
    v, t = jittered_box(n, 0.1, seed)
    perm = np.random.default_rng(seed).permutation(len(v))
    v2 = np.empty_like(v)
    v2[perm] = v
    return v2, perm[t].astype(np.int32)


def vertex_order_classes(t):
    return {tuple(np.argsort(np.argsort(c))) for c in t}


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_nedelec_all_vertex_orders_match_oracle(k):
    v, t = relabelled_box(4, 100 + k)
    assert len(vertex_order_classes(t)) == 24
    rng = np.random.default_rng(k)
    cc = rng.uniform(0.5, 2.0, len(t))
    cm = rng.uniform(0.5, 2.0, len(t))
    A, st = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, 1.7, 0.9, order=k, cell_curl=cc,
                                                    cell_mass=cm)
    assert st.code == 0
    n, cp, ri, val = oracle.nedelec_csc(v, t, k, 1.7, 0.9, cc, cm)
    assert A.nrow == n and np.array_equal(A.col_ptr, cp) and np.array_equal(A.row_idx, ri)
    assert rel_frob(A.val, val) <= FROB
    pts = oracle.nedelec_load_points(v, t, k)
    src = np.stack([np.sin(pts[..., 1]), pts[..., 0] * pts[..., 2], np.cos(pts[..., 0])], -1)
    rhs, st = ff.assemble_tetra_nedelec_vector_load_samples(v, t, k, src)
    assert st.code == 0
    assert rel_frob(rhs, oracle.nedelec_load_samples(v, t, k, src)) <= FROB


def test_nedelec_order6_all_vertex_orders_match_oracle():
    v, t = relabelled_box(2, 136)  # 48 cells in 23 of the 24 orders
    assert len(vertex_order_classes(t)) == 23
    A, st = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, 1.7, 0.9, order=6)
    assert st.code == 0
    n, cp, ri, val = oracle.nedelec_csc(v, t, 6, 1.7, 0.9)
    assert np.array_equal(A.col_ptr, cp) and np.array_equal(A.row_idx, ri)
    assert rel_frob(A.val, val) <= 1e-10


def test_p1_csc_matches_oracle():
    v, t = oracle.unit_square_mesh(17)
    v = synth.jitter_interior_2d(v, 1 / 16, 0.1, 4)
    cs = np.exp(np.random.default_rng(4).standard_normal(len(t)))
    A, st = ff.assemble_scalar_p1_csc(v, t, 0.3, 1.1, cs)
    assert st.code == 0
    n, cp, ri, val = oracle.p1_csc(v, t, 0.3, 1.1, cs)
    assert np.array_equal(A.col_ptr, cp) and np.array_equal(A.row_idx, ri)
    assert rel_frob(A.val, val) <= FROB


# test/test_tetra_nedelec_sparse_assembly_slow.f90:31-85 on the GPU-assembled CSC
def test_nedelec_energy_kats_on_gpu():
    verts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1.0]])
    tets = np.array([[0, 1, 2, 3], [0, 2, 1, 4]])
    edges, _, _ = oracle.edge_dof_map(tets)
    field = np.array([1.0, 2.0, -1.0])
    dofs = np.array([field @ (verts[b] - verts[a]) for a, b in edges])
    A, st = ff.assemble_tetra_nedelec_curl_mass_csc(verts, tets, 4.0, 1.5)
    assert abs(dofs @ ff.spmv(A, dofs) - 3.0) < 2e-12
    curl = np.array([1.0, -2.0, 3.0])
    dofs = np.array([(0.5 * np.cross(curl, 0.5 * (verts[a] + verts[b]))) @ (verts[b] - verts[a])
                     for a, b in edges])
    A, st = ff.assemble_tetra_nedelec_curl_mass_csc(verts, tets, 2.0, 0.0)
    assert abs(dofs @ ff.spmv(A, dofs) - 28.0 / 3.0) < 3e-12


# test/test_tetra_lagrange_arbitrary_order_assembly.f90:37-66
def test_lagrange_linear_energy_on_gpu():
    mv = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1.0]])
    tets = np.array([[0, 1, 2, 3], [0, 2, 1, 4]])
    A, st = ff.assemble_tetra_lagrange_stiffness_csc(mv, tets, 1, 4)
    gd, n = oracle.lagrange_dof_map(1, tets)
    coef = np.zeros(n)
    coef[gd.reshape(-1)] = mv[tets.reshape(-1), 0]
    assert abs(coef @ ff.spmv(A, coef) - 1.0 / 3.0) < 2e-12


def test_reduced_system_with_lifting_matches_oracle():
    v, t = jittered_box(3, 0.1, 5)
    p = 2
    kappa = np.exp(np.random.default_rng(5).standard_normal(len(t)))
    with ff.Problem(K.FFG_TETRA_LAGRANGE, p, t, len(v), rule=K.FFG_RULE_DEGREE_TWO) as prob:
        pts = prob.sample_points(v)
        src = np.sin(np.pi * pts[..., 0]) * np.sin(np.pi * pts[..., 1]) * pts[..., 2]
        dofp = prob.dof_points(v)
        con = prob.constrained()
        g = np.where(con, dofp[:, 0] + 2 * dofp[:, 1] - 3 * dofp[:, 2], 0.0)
        A, rhs, free = prob.reduced_system(v, 1.0, 0.0, kappa, None, src, g)
    n, cp, ri, val = oracle.lagrange_csc(v, t, p, 1, 0, 1.0, 0.0, kappa)
    b = oracle.lagrange_load_samples(v, t, p, src, 1, 0)
    ocon, _ = oracle.lagrange_dirichlet(p, v, t)
    assert np.array_equal(con, ocon)
    nf, rcp, rri, rv, rr, ofree = oracle.reduce_constrained(n, cp, ri, val, b, con, g)
    assert np.array_equal(free, ofree)
    assert np.array_equal(A.col_ptr, rcp) and np.array_equal(A.row_idx, rri)
    assert rel_frob(A.val, rv) <= FROB
    assert rel_frob(rhs, rr) <= 1e-12


def _oracle_reduced_solution(v, t, p, rule, q, kappa, src, g):
    import scipy.sparse.linalg as spla
    n, cp, ri, val = oracle.lagrange_csc(v, t, p, rule, q, 1.0, 0.0, kappa)
    b = oracle.lagrange_load_samples(v, t, p, src, rule, q)
    con, _ = oracle.lagrange_dirichlet(p, v, t)
    nf, rcp, rri, rv, rr, free = oracle.reduce_constrained(n, cp, ri, val, b, con, g)
    return n, nf, rcp, rri, rv, rr, free, con


def test_fp64_pcg_mirrors_reference_iterations():
    v, t = jittered_box(5, 0.1, 9)
    p = 2
    kappa = np.exp(np.random.default_rng(9).standard_normal(len(t)))
    with ff.Problem(K.FFG_TETRA_LAGRANGE, p, t, len(v), rule=K.FFG_RULE_DEGREE_TWO) as prob:
        pts = prob.sample_points(v)
        src = 100.0 * np.sin(np.pi * pts[..., 0]) * np.sin(np.pi * pts[..., 1]) * np.sin(np.pi * pts[..., 2])
        opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                                precision="fp64", max_iterations=100000)
        sol, stats = prob.solve(v, 1.0, 0.0, kappa, None, src, None, opts)
        opts.breakdown_guard = "spd"
        sol_spd, stats_spd = prob.solve(v, 1.0, 0.0, kappa, None, src, None, opts)
    n, nf, rcp, rri, rv, rr, free, con = _oracle_reduced_solution(v, t, p, 1, 0, kappa, src, None)
    # the reference's absolute guard |p^T A p| < 1e-14 (advanced_solvers.f90:897): the
    # GPU and the oracle stop at the same iteration with the same verdict
    xo, so = oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=1e-10)
    assert stats.converged == so["converged"]
    assert abs(stats.iterations - so["iterations"]) <= 2
    assert np.abs(sol[free] - xo).max() <= 1e-6 * np.abs(xo).max()
    assert np.all(sol[con] == 0.0)
    # SPD-only guard: both reach the 1e-10 recursive tolerance in the same iterations
    xs, ss = oracle.pcg_sparse(nf, rcp, rri, rv, rr, tol=1e-10, guard=1)
    assert stats_spd.converged and ss["converged"]
    assert abs(stats_spd.iterations - ss["iterations"]) <= 2
    assert np.abs(sol_spd[free] - xs).max() <= 1e-8 * np.abs(xs).max()


def test_mixed_precision_reaches_true_residual_1e10():
    v, t = jittered_box(6, 0.1, 13)
    p = 2
    kappa = np.exp(np.random.default_rng(13).standard_normal(len(t)))
    with ff.Problem(K.FFG_TETRA_LAGRANGE, p, t, len(v), rule=K.FFG_RULE_DEGREE_TWO) as prob:
        pts = prob.sample_points(v)
        src = np.sin(np.pi * pts[..., 0]) * np.sin(np.pi * pts[..., 1]) * np.sin(np.pi * pts[..., 2])
        sol, stats = prob.solve(v, 1.0, 0.0, kappa, None, src)
        sol2, _ = prob.solve(v, 1.0, 0.0, kappa, None, src)
    assert stats.converged and stats.true_relative_residual <= 1e-10
    assert np.array_equal(sol, sol2), "solve is not bit-reproducible"
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    n, nf, rcp, rri, rv, rr, free, con = _oracle_reduced_solution(v, t, p, 1, 0, kappa, src, None)
    Ao = sp.csc_matrix((rv, rri, rcp), shape=(nf, nf))
    x_direct = spla.spsolve(Ao, rr)
    assert np.linalg.norm(rr - Ao @ sol[free]) <= 1.01e-10 * np.linalg.norm(rr)
    assert np.abs(sol[free] - x_direct).max() <= 1e-7 * np.abs(x_direct).max()


def test_host_solve_into_caller_buffer():
    import torch
    v, t = jittered_box(5, 0.1, 17)
    kappa = np.exp(np.random.default_rng(17).standard_normal(len(t)))
    with ff.Problem(K.FFG_TETRA_LAGRANGE, 2, t, len(v), rule=K.FFG_RULE_DEGREE_TWO) as prob:
        pts = prob.sample_points(v)
        src = np.cos(pts[..., 0]) * pts[..., 1]
        sol, _ = prob.solve(v, 1.0, 0.0, kappa, None, src)
        out = torch.zeros(prob.n_dofs, dtype=torch.float64).pin_memory().numpy()
        sol2, st = prob.solve(v, 1.0, 0.0, kappa, None, src, out=out)
        assert st.converged and sol2 is out and np.array_equal(out, sol)
        for bad in (np.zeros(prob.n_dofs, np.float32), np.zeros(prob.n_dofs + 1),
                    np.zeros(2 * prob.n_dofs)[::2]):
            with pytest.raises(ff.FortfemError):
                prob.solve(v, 1.0, 0.0, kappa, None, src, out=bad)


def test_p1_unit_square_solve_matches_reference_dense_path():
    v, t = ff.unit_square_mesh(65)
    opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                            precision="mixed", max_iterations=100000)
    sol, stats = ff.solve_scalar_p1(v, t, load=1.0, options=opts)
    assert stats.converged
    a = oracle.p1_dense(v, t, 0.0, 1.0)
    b = oracle.p1_load(v, t, 1.0)
    bnd = oracle.square_boundary(len(v), t)
    a2, b2 = oracle.p1_eliminate_dense(a, b, bnd.astype(np.uint8), 0.0)
    x_ref = np.linalg.solve(a2, b2)
    assert np.abs(sol - x_ref).max() <= 1e-9 * np.abs(x_ref).max()
    # the reference's dense Jacobi-PCG path (SPD-only breakdown guard, so that it
    # reaches the 1e-10 tolerance on this small-residual system) agrees too
    xp, sp_ = oracle.pcg_dense(a2, b2, tol=1e-10, guard=1)
    assert sp_["converged"]
    assert np.abs(sol - xp).max() <= 1e-8 * np.abs(x_ref).max()


@pytest.mark.parametrize("k", [1, 2, 3])
def test_nedelec_pec_solve_matches_direct(k):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    v, t = oracle.box_mesh([3, 3, 3])
    mu_inv = synth.slab_reluctivity(v, t, (1.0, 10.0, 1.0))
    with ff.Problem(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary="all") as prob:
        pts = prob.sample_points(v)
        src = synth.slab_current(pts)
        opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                                precision="mixed", max_iterations=200000)
        sol, stats = prob.solve(v, 1.0, 1.0, mu_inv, None, src, None, opts)
        con = prob.constrained()
    assert stats.converged and stats.true_relative_residual <= 1e-10
    n, cp, ri, val = oracle.nedelec_csc(v, t, k, 1.0, 1.0, mu_inv)
    b = oracle.nedelec_load_samples(v, t, k, src)
    assert np.array_equal(con, oracle.pec_mask(k, t))
    nf, rcp, rri, rv, rr, free = oracle.reduce_constrained(n, cp, ri, val, b, con)
    x = spla.spsolve(sp.csc_matrix((rv, rri, rcp), shape=(nf, nf)), rr)
    assert np.abs(sol[free] - x).max() <= 1e-7 * np.abs(x).max()


def test_solve_sparse_drop_in_matches_oracle_pcg():
    v, t = oracle.unit_square_mesh(33)
    n, cp, ri, val = oracle.p1_csc(v, t, 1.0, 1.0)
    b = 1e3 * oracle.p1_load(v, t, 1.0)
    A = ff.CscMatrix(n, n, cp, ri, val)
    x = np.zeros(n)
    opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10, max_iterations=10000)
    stats = ff.solve_sparse(A, b, x, opts)
    xo, so = oracle.pcg_sparse(n, cp, ri, val, b, tol=1e-10)
    assert stats.converged == so["converged"]
    assert abs(stats.iterations - so["iterations"]) <= 1
    assert np.abs(x - xo).max() <= 1e-9 * np.abs(xo).max()
    y = ff.spmv(A, x)
    assert np.abs(y - oracle.csc_matvec(n, cp, ri, val, x)).max() <= 1e-12 * np.abs(y).max()


def test_solve_sparse_nonsymmetric_matvec_is_csc():
    n = 5
    rng = np.random.default_rng(0)
    M = rng.standard_normal((n, n))
    import scipy.sparse as sp
    A = sp.csc_matrix(M)
    m = ff.CscMatrix(n, n, A.indptr.astype(np.int64), A.indices.astype(np.int32), A.data)
    x = rng.standard_normal(n)
    assert np.abs(ff.spmv(m, x) - M @ x).max() < 1e-13


def test_invalid_inputs_report_status():
    v, t = oracle.box_mesh([1, 1, 1])
    t_bad = t.copy()
    t_bad[0, 3] = t_bad[0, 2]
    A, st = ff.assemble_tetra_lagrange_stiffness_csc(v, t_bad, 2, 4)
    assert A is None and st.code == K.FFG_INVALID_INPUT
    v2 = v.copy()
    v2[:] = 0.0  # every cell degenerate
    A, st = ff.assemble_tetra_lagrange_stiffness_csc(v2, t, 2, 4)
    assert A is None and st.code == K.FFG_INVALID_INPUT
    with pytest.raises(ff.FortfemError):
        ff.Problem(K.FFG_TETRA_NEDELEC, 9, t, len(v))


def test_p2_full_size_properties():
    """48^3 P2 workload: symmetric matrix, stiffness annihilates constants,
    mixed solve to 1e-10 true residual."""
    case = synth.p2_poisson_case()
    with ff.Problem(K.FFG_TETRA_LAGRANGE, 2, case.cells, len(case.vertices),
                    rule=case.rule, quadrature_degree=0) as prob:
        assert prob.n_dofs == 912673 and prob.n_free == 857375
        pts = prob.sample_points(case.vertices)
        src = case.source(pts[..., 0], pts[..., 1], pts[..., 2])
        sol, stats = prob.solve(case.vertices, 1.0, 0.0, case.cell_coefficient, None, src)
        assert stats.converged and stats.true_relative_residual <= 1e-10
        assert np.isfinite(sol).all() and sol.max() > 0


def test_wall_limit_reports_timeout():
    """A wall limit far below one solve's time: the persistent PCG kernel
    checks it every iteration and returns FFG_TIMEOUT (status -7) through
    solve_sparse and through a problem handle, without waiting on anything."""
    v, t = jittered_box(8, 0.1, 3)
    A, st = ff.assemble_tetra_lagrange_stiffness_csc(v, t, 2, 8, 1.0, 0.0)
    assert st.code == 0
    b = np.random.default_rng(3).standard_normal(A.nrow)
    opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-14,
                            max_iterations=100000, precision="fp64", breakdown_guard="spd",
                            timeout_seconds=1e-9)
    with pytest.raises(ff.FortfemError) as e:
        ff.solve_sparse(A, b, np.zeros(A.nrow), opts)
    assert e.value.code == K.FFG_TIMEOUT
    with ff.Problem(K.FFG_TETRA_LAGRANGE, 2, t, len(v)) as prob:
        pts = prob.sample_points(v)
        src = np.sin(pts[..., 0])
        for precision in ("fp64", "mixed"):
            opts.precision = precision
            with pytest.raises(ff.FortfemError) as e:
                prob.solve(v, 1.0, 0.0, None, None, src, None, opts)
            assert e.value.code == K.FFG_TIMEOUT
        # the next solve on the same handle is unaffected
        opts.timeout_seconds = 60.0
        opts.tolerance = 1e-10
        sol, stats = prob.solve(v, 1.0, 0.0, None, None, src, None, opts)
        assert stats.converged


@pytest.mark.parametrize("family,degree", [(K.FFG_TETRA_LAGRANGE, 2), (K.FFG_TRIANGLE_P1, 1),
                                           (K.FFG_TETRA_NEDELEC, 2)])
def test_mixed16_operator_reaches_the_same_true_residual(family, degree):
    """The inner SpMV on the row-scaled FP16 operator: the reliable updates
    use the FP64 operator, so the solve still stops at a true relative
    residual of 1e-10 and agrees with the FP32-operator solve to the
    residual-derived bound."""
    if family == K.FFG_TRIANGLE_P1:
        v, t = oracle.unit_square_mesh(49)
        v = synth.jitter_interior_2d(v, 1 / 48, 0.1, 2)
    else:
        v, t = jittered_box(6 if family == K.FFG_TETRA_LAGRANGE else 4, 0.1, 2)
    kappa = np.exp(np.random.default_rng(2).standard_normal(len(t)))
    with ff.Problem(family, degree, t, len(v)) as prob:
        pts = prob.sample_points(v)
        if family == K.FFG_TETRA_NEDELEC:
            src = synth.trig_vector_source(3)(pts)
            cb = 20.0
        else:
            src = np.sin(np.pi * pts[..., 0]) + pts[..., 1]
            cb = 0.0
        sols = {}
        for prec in ("mixed", "mixed16"):
            opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                                    precision=prec, max_iterations=100000)
            sols[prec] = prob.solve(v, 1.0, cb, kappa, None, src, None, opts)
    for prec, (x, st) in sols.items():
        assert st.converged and st.true_relative_residual <= 1e-10, (prec, st)
    x32, x16 = sols["mixed"][0], sols["mixed16"][0]
    assert np.abs(x16 - x32).max() <= 1e-6 * np.abs(x32).max()
    print(f"mixed {sols['mixed'][1].iterations} it, mixed16 {sols['mixed16'][1].iterations} it")
