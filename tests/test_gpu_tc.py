"""3xTF32 tensor-core contraction of Nedelec element matrices (orders 3 to 6).

The tcgen05 path computes the same element matrices as the reference's
quadrature loop (assemble_tetra_nedelec_curl_mass_element,
src/assembly/assembly_tetra_nedelec_3d.f90:584-643) with TF32 hi/lo operands
and FP32 accumulation against the oriented reference tensors of each cell's
vertex-order class.  Tolerances:
pattern and right-hand side exact / 1e-12 (the loads stay FP64); matrix
values within 1e-6 relative Frobenius of the FP64 oracle (the split keeps
about 22 bits of every operand, so 1e-7 is expected).
"""
import numpy as np
import pytest

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K
from fortfem_b200 import synth

pytestmark = pytest.mark.gpu

TF32X3 = 1e-6


def rel_frob(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _reduced(prob, v, mu, cm, src, precision):
    prob.set_assembly_precision(precision)
    return prob.reduced_system(v, 1.3, 0.7, mu, cm, src)


@pytest.mark.parametrize("k", [3, 4, 5, 6])
def test_tf32x3_reduced_system_matches_oracle(k):
    m = 3 if k <= 4 else 2
    v, t = oracle.box_mesh([m, m, m])
    v = synth.jitter_interior(v, 1 / m, 0.1, 31 + k)
    # vertices renumbered at random: cells of many vertex-order classes
    perm = np.random.default_rng(k).permutation(len(v))
    v2 = np.empty_like(v)
    v2[perm] = v
    v, t = v2, perm[t].astype(np.int32)
    rng = np.random.default_rng(k)
    mu = rng.uniform(0.5, 2.0, len(t))
    cm = rng.uniform(0.5, 2.0, len(t))
    with ff.Problem(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary="all") as prob:
        pts = prob.sample_points(v)
        src = synth.trig_vector_source(k)(pts)
        R, rhs, free = _reduced(prob, v, mu, cm, src, "tf32x3")
        R64, rhs64, _ = _reduced(prob, v, mu, cm, src, "fp64")
    n, cp, ri, val = oracle.nedelec_csc(v, t, k, 1.3, 0.7, mu, cm)
    b = oracle.nedelec_load_samples(v, t, k, src)
    con = oracle.pec_mask(k, t)
    nf, rcp, rri, rv, rr, ofree = oracle.reduce_constrained(n, cp, ri, val, b, con)
    assert np.array_equal(free, ofree)
    assert np.array_equal(R.col_ptr, rcp) and np.array_equal(R.row_idx, rri)
    err = rel_frob(R.val, rv)
    print(f"order {k}: 3xTF32 matrix rel. Frobenius error {err:.2e}")
    assert err <= TF32X3
    assert rel_frob(rhs, rr) <= 1e-12
    # switching back gives the FP64 parity path
    fp64 = 1e-12 if k <= 4 else (1e-11 if k == 5 else 1e-10)
    assert rel_frob(R64.val, rv) <= fp64 and rel_frob(rhs64, rr) <= 1e-12


@pytest.mark.parametrize("k", [3, 4])
def test_tf32x3_many_cell_groups_match_fp64_path(k):
    """20^3 x 6 cells in 128-cell groups of one vertex-order class on at most
    296 CTAs, so CTAs run several groups and the bulk-copy pipeline wraps
    across groups of different classes; groups at class ends are partial."""
    v, t = oracle.box_mesh([20, 20, 20])
    v = synth.jitter_interior(v, 1 / 20, 0.1, 7)
    t = t[:-5]  # a partial last group
    mu = synth.slab_reluctivity(v, t)
    with ff.Problem(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary="all") as prob:
        R, rhs, _ = _reduced(prob, v, mu, None, None, "tf32x3")
        R64, rhs64, _ = _reduced(prob, v, mu, None, None, "fp64")
    assert np.array_equal(R.row_idx, R64.row_idx)
    err = rel_frob(R.val, R64.val)
    print(f"order {k} 20^3: 3xTF32 vs FP64 rel. Frobenius {err:.2e}")
    assert err <= TF32X3
    assert np.all(rhs == 0.0) and np.all(rhs64 == 0.0)


# test/test_tetra_nedelec_sparse_assembly_slow.f90:31-85: the constant field
# (1, 2, -1) has energy 3 on the two-cell mesh at every order (mass 1, curl 0).
# The energy is what is left of |x|^T |A| |x| (3.0e4 at order 3, 1.2e6 at
# order 4) after cancellation, so the 3xTF32 matrix (about 2^-22 relative per
# entry) reproduces it to 2^-22 |x|^T |A| |x|, checked here with twice that.
@pytest.mark.parametrize("k", [3, 4])
def test_tf32x3_constant_field_energy(k):
    verts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1.0]])
    tets = np.array([[0, 1, 2, 3], [0, 2, 1, 4]], dtype=np.int32)
    field = np.array([1.0, 2.0, -1.0])
    with ff.Problem(K.FFG_TETRA_NEDELEC, k, tets, len(verts), boundary="none") as prob:
        R64, _, _ = _reduced(prob, verts, None, None, None, "fp64")
        R, _, free = _reduced(prob, verts, None, None, None, "tf32x3")
    # interpolate the constant field: the L2 projection solve is exact for it
    n, cp, ri, val = oracle.nedelec_csc(verts, tets, k, 0.0, 1.0)
    pts_l = oracle.nedelec_load_points(verts, tets, k)
    b = oracle.nedelec_load_samples(verts, tets, k, np.broadcast_to(field, pts_l.shape))
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    M = sp.csc_matrix((val, ri, cp), shape=(n, n))
    dofs = spla.spsolve(M, b)
    A = ff.CscMatrix(R.nrow, R.nrow, R.col_ptr, R.row_idx, R.val)
    # R is the full system here (no constraint), curl 1.3 and mass 0.7: the
    # constant field has no curl and |f|^2 vol = 6 * (2 / 6) = 2
    energy = dofs @ ff.spmv(A, dofs)
    A64 = sp.csc_matrix((np.abs(R64.val), R64.row_idx, R64.col_ptr), shape=(R.nrow, R.nrow))
    bound = 2.0 * 2.0 ** -22 * (np.abs(dofs) @ (A64 @ np.abs(dofs)))
    print(f"order {k}: energy error {abs(energy - 1.4):.2e}, bound {bound:.2e}")
    assert abs(energy - 0.7 * 2.0) <= bound
    energy64 = dofs @ ff.spmv(ff.CscMatrix(R.nrow, R.nrow, R64.col_ptr, R64.row_idx, R64.val), dofs)
    assert abs(energy64 - 1.4) <= 1e-8 * 1.4


def test_tf32x3_selection_rules():
    v, t = oracle.box_mesh([1, 1, 1])
    for fam, deg in ((K.FFG_TETRA_NEDELEC, 2), (K.FFG_TETRA_NEDELEC, 1),
                     (K.FFG_TETRA_LAGRANGE, 3)):
        with ff.Problem(fam, deg, t, len(v)) as prob:
            with pytest.raises(ff.FortfemError):
                prob.set_assembly_precision("tf32x3")
            prob.set_assembly_precision("fp64")
    for deg in (3, 4, 5, 6):
        with ff.Problem(K.FFG_TETRA_NEDELEC, deg, t, len(v)) as prob:
            prob.set_assembly_precision("tf32x3")


# The solution of a 3xTF32-assembled system differs from the FP64-assembled
# one by up to cond(A) times the matrix perturbation (measured 9e-5 at order 3
# and 4e-3 at order 4 on this 4^3 x 6 mesh), so the check is the backward
# error: x3 solves the FP64-assembled system up to the 3xTF32 perturbation,
# ||b - A64 x3|| <= 4 * 2^-22 || |A64| |x3| || + 2e-10 ||b||.
@pytest.mark.parametrize("k", [3, 4])
def test_tf32x3_solve_is_backward_stable_for_the_fp64_matrix(k):
    import scipy.sparse as sp
    v, t = oracle.box_mesh([4, 4, 4])
    v = synth.jitter_interior(v, 0.25, 0.1, 5)
    mu = np.random.default_rng(k).uniform(0.5, 2.0, len(t))
    with ff.Problem(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary="all") as prob:
        pts = prob.sample_points(v)
        src = synth.trig_vector_source(k + 10)(pts)
        opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                                precision="mixed", max_iterations=200000)
        prob.set_assembly_precision("tf32x3")
        x3, s3 = prob.solve(v, 1.0, 50.0, mu, None, src, None, opts)
        prob.set_assembly_precision("fp64")
        R, rhs, free = prob.reduced_system(v, 1.0, 50.0, mu, None, src)
    assert s3.converged
    A = sp.csc_matrix((R.val, R.row_idx, R.col_ptr), shape=(R.nrow, R.nrow))
    x = x3[free]
    res = np.linalg.norm(rhs - A @ x)
    bound = 4 * 2.0 ** -22 * np.linalg.norm(abs(A) @ np.abs(x)) + 2e-10 * np.linalg.norm(rhs)
    print(f"order {k}: ||b - A64 x3|| / ||b|| = {res / np.linalg.norm(rhs):.2e}, "
          f"bound {bound / np.linalg.norm(rhs):.2e}")
    assert res <= bound
