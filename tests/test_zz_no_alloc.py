"""ffg_solve_csr_device_noalloc against ffg_solve_sparse (both FP64 Jacobi-PCG).

The allocation-free solver keeps its work vectors in one fixed device array
shared by every call, so two different systems are solved in a row: the
second must not see anything the first left behind.  Both solvers stop on
the same recursive-residual rule but sum in different orders, so iteration
counts may differ by one and solutions agree to 1e-9 of their largest entry
(the tolerance of the solve_sparse parity test).  The SPD breakdown guard is
selected so that both reach the 1e-10 tolerance: with the reference's
absolute |p^T A p| < 1e-14 test both stop early on these O(1) right-hand sides.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest
import torch

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K

TOL = 1e-9
HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "fortfem_gpu.h")


def _systems():
    v, t = oracle.box_mesh([6, 6, 6])
    a3, st = ff.assemble_tetra_lagrange_stiffness_csc(v, t, 2, 6, 1.0, 1.0)
    assert st.code == 0
    v2, t2 = oracle.unit_square_mesh(33)
    a2, st = ff.assemble_scalar_p1_csc(v2, t2, 1.0, 1.0)
    assert st.code == 0
    rng = np.random.default_rng(5)
    return [(a3, rng.standard_normal(a3.nrow)), (a2, rng.standard_normal(a2.nrow))]


def _noalloc(A, b, opts, nnz=None, row_idx=None):
    """Solve through the C-ABI with the matrix and vectors in device memory
    (the CSC arrays of the symmetric matrix read as CSR).  nnz and row_idx
    override what is passed, to hand the kernel a malformed matrix whose
    every array still has its full length."""
    dev = torch.device("cuda:0")
    ri_host = A.row_idx if row_idx is None else row_idx
    rp = torch.from_numpy(np.ascontiguousarray(A.col_ptr, np.int64)).to(dev)
    ci = torch.from_numpy(np.ascontiguousarray(ri_host, np.int32)).to(dev)
    val = torch.from_numpy(np.ascontiguousarray(A.val, np.float64)).to(dev)
    db = torch.from_numpy(np.ascontiguousarray(b, np.float64)).to(dev)
    dx = torch.zeros(A.nrow, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    oc = opts.to_c()
    sc = K.SolverStatsC()
    st = C.c_int(99)
    K.load().ffg_solve_csr_device_noalloc(
        A.nrow, int(A.col_ptr[-1]) if nnz is None else int(nnz), C.c_void_p(rp.data_ptr()),
        C.c_void_p(ci.data_ptr()), C.c_void_p(val.data_ptr()), C.c_void_p(db.data_ptr()),
        C.c_void_p(dx.data_ptr()), C.byref(oc), C.byref(sc), C.c_void_p(stream.cuda_stream),
        C.byref(st))
    return st.value, sc, dx.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_matches_solve_sparse_twice_in_a_row():
    opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                            max_iterations=10000, precision="fp64", breakdown_guard="spd")
    first = None
    for A, b in _systems():
        x_ref = np.zeros(A.nrow)
        ref = ff.solve_sparse(A, b, x_ref, opts)
        st, sc, x = _noalloc(A, b, opts)
        assert st == K.FFG_OK and sc.converged == 1 and ref.converged
        assert abs(sc.iterations - ref.iterations) <= 1
        assert np.abs(x - x_ref).max() <= TOL * np.abs(x_ref).max()
        assert sc.true_relative_residual <= 1e-8
        first = first or (A, b, x)
    # the first system again, after the second left its vectors in the array:
    # the fixed summation order gives the same bits
    A, b, x = first
    st, sc, x2 = _noalloc(A, b, opts)
    assert st == K.FFG_OK and np.array_equal(x, x2)


@pytest.mark.gpu
def test_noalloc_matches_the_oracle_pcg():
    """The same two systems against the CPU restatement of the reference's
    Jacobi-PCG (oracle.pcg_sparse), so that an error shared by both GPU
    solvers (option handling, the Jacobi diagonal) is caught too."""
    opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                            max_iterations=10000, precision="fp64", breakdown_guard="spd")
    for A, b in _systems():
        xo, so = oracle.pcg_sparse(A.nrow, A.col_ptr, A.row_idx, A.val, b, tol=1e-10,
                                   relative=True, max_iterations=10000, jacobi=True, guard=1)
        st, sc, x = _noalloc(A, b, opts)
        assert st == K.FFG_OK and so["converged"]
        assert abs(sc.iterations - so["iterations"]) <= 1
        assert np.abs(x - xo).max() <= TOL * np.abs(xo).max()


@pytest.mark.gpu
def test_noalloc_reports_timeout_and_non_convergence():
    A, b = _systems()[0]
    quick = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                             max_iterations=10000, precision="fp64", breakdown_guard="spd",
                             timeout_seconds=1e-9)
    st, sc, _ = _noalloc(A, b, quick)
    assert st == K.FFG_TIMEOUT and sc.status == K.FFG_TIMEOUT and sc.converged == 0
    assert sc.iterations == 1
    short = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                             max_iterations=1, precision="fp64", breakdown_guard="spd")
    st, sc, _ = _noalloc(A, b, short)
    assert st == K.FFG_NOT_CONVERGED and sc.status == K.FFG_NOT_CONVERGED
    assert sc.converged == 0 and sc.iterations == 1
    # a huge wall limit is clamped, not wrapped to a tiny one
    long = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                            max_iterations=10000, precision="fp64", breakdown_guard="spd",
                            timeout_seconds=1e30)
    st, sc, _ = _noalloc(A, b, long)
    assert st == K.FFG_OK and sc.converged == 1


@pytest.mark.gpu
def test_noalloc_rejects_malformed_csr_before_use():
    """A row pointer that does not end at nnz, and a column index outside
    [0, n), are found by the kernel's check before any indexed access."""
    A, b = _systems()[1]
    opts = ff.SolverOptions(method="pcg", preconditioner="jacobi", tolerance=1e-10,
                            max_iterations=100, precision="fp64", breakdown_guard="spd")
    nnz = int(A.col_ptr[-1])
    st, sc, _ = _noalloc(A, b, opts, nnz=nnz - 1)
    assert st == K.FFG_INVALID_INPUT
    bad = np.array(A.row_idx, np.int32)
    bad[nnz // 2] = A.nrow
    st, sc, _ = _noalloc(A, b, opts, row_idx=bad)
    assert st == K.FFG_INVALID_INPUT
    bad[nnz // 2] = -1
    st, sc, _ = _noalloc(A, b, opts, row_idx=bad)
    assert st == K.FFG_INVALID_INPUT
    # a well-formed call afterwards still solves
    st, sc, _ = _noalloc(A, b, opts.__class__(**{**opts.__dict__, "max_iterations": 10000}))
    assert st == K.FFG_OK


@pytest.mark.gpu
def test_noalloc_rejects_systems_above_its_maximum():
    n = K.FFG_NOALLOC_MAX_ROWS + 1
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    p = C.c_void_p(dummy.data_ptr())
    st = C.c_int(0)
    K.load().ffg_solve_csr_device_noalloc(n, 0, p, p, p, p, p, None, None, None, C.byref(st))
    assert st.value == K.FFG_CAPACITY


def test_noalloc_maximum_matches_header():
    text = open(HEADER).read()
    m = re.search(r"#define FFG_NOALLOC_MAX_ROWS (\d+)", text)
    assert m and int(m.group(1)) == K.FFG_NOALLOC_MAX_ROWS
