"""Complex PML Nedelec assembly on the GPU, through the C-ABI.

Parity with the oracle's restatement of assemble_tetra_nedelec_pml_csc and
assemble_tetra_nedelec_curvilinear_pml_csc (pattern bit-exact, complex values
within relative Frobenius 1e-12; orders 5-6 1e-10, whose dual-basis tables
carry large entries), and the reference's known answers
(test/test_tetra_nedelec_pml_element.f90, test/test_tetra_nedelec_pml_sparse.f90):
unit stretch reduces to curl-curl minus k^2 mass, the operator is complex
symmetric with a nonzero imaginary part, and the order-1 constant-field
energy is exact.
"""
import numpy as np
import pytest

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K
from fortfem_b200 import synth

pytestmark = pytest.mark.gpu


def rel_frob(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def jittered_box(n, delta=0.1, seed=7):
    v, t = oracle.box_mesh([n, n, n])
    return synth.jitter_interior(v, 1.0 / n, delta, seed), t


def stretches(t, rng, curvilinear):
    if not curvilinear:
        return 1.0 + rng.uniform(0, 0.5, (len(t), 3)) + 1j * rng.uniform(0, 0.8, (len(t), 3))
    a = np.eye(3) + 0.2 * rng.standard_normal((len(t), 3, 3))
    return a + 1j * 0.3 * rng.standard_normal((len(t), 3, 3))


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("curvilinear", [False, True])
def test_pml_csc_matches_oracle(k, curvilinear):
    v, t = jittered_box(2 if k <= 4 else 1, 0.1, 11)
    rng = np.random.default_rng(40 + k)
    s = stretches(t, rng, curvilinear)
    fn = ff.assemble_tetra_nedelec_curvilinear_pml_csc if curvilinear else \
        ff.assemble_tetra_nedelec_pml_csc
    A, st = fn(v, t, k, s, 1.3)
    assert st.code == 0
    n, cp, ri, val = oracle.nedelec_pml_csc(v, t, k, s, 1.3, curvilinear=curvilinear)
    assert A.nrow == n and np.array_equal(A.col_ptr, cp) and np.array_equal(A.row_idx, ri)
    assert rel_frob(A.val, val) <= (1e-12 if k <= 4 else 1e-10)
    # complex symmetric (reciprocal) operator with absorption
    M = oracle.csc_to_scipy(n, A.col_ptr, A.row_idx, A.val)
    assert abs(M - M.T).max() <= 1e-12 * abs(M).max()
    assert np.abs(A.val.imag).max() > 1e-3


@pytest.mark.parametrize("k", [1, 2, 3])
def test_unit_stretch_is_curl_minus_mass(k):
    v, t = jittered_box(2, 0.1, 3)
    wave = 1.7
    A, st = ff.assemble_tetra_nedelec_pml_csc(v, t, k, np.ones((len(t), 3)), wave)
    assert st.code == 0
    B, st = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, 1.0, -wave ** 2, order=k)
    assert np.array_equal(A.col_ptr, B.col_ptr) and np.array_equal(A.row_idx, B.row_idx)
    assert np.abs(A.val.imag).max() == 0.0
    assert np.abs(A.val.real - B.val).max() <= 1e-12 * np.abs(B.val).max()
    C, st = ff.assemble_tetra_nedelec_curvilinear_pml_csc(v, t, k, np.tile(np.eye(3), (len(t), 1, 1)),
                                                          wave)
    assert np.abs(C.val - A.val).max() <= 1e-12 * np.abs(B.val).max()


def test_constant_field_energy():
    # test_tetra_nedelec_pml_sparse.f90:21-52
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1]], float)
    t = np.array([[0, 1, 2, 3], [0, 2, 1, 4]], np.int32)
    s = np.array([[1 + 0.6j, 1.0, 1.0]] * 2)
    A, st = ff.assemble_tetra_nedelec_pml_csc(v, t, 1, s, 1.3)
    assert st.code == 0
    edges = oracle.nedelec_dof_map(1, t)["edges"]
    field = np.array([1.0, 2.0, -1.0])
    dofs = np.array([field @ (v[b] - v[a]) for a, b in edges], complex)
    M = oracle.csc_to_scipy(A.nrow, A.col_ptr, A.row_idx, A.val)
    energy = dofs @ (M @ dofs)
    mass = np.array([s[0, 1] * s[0, 2] / s[0, 0], s[0, 0] * s[0, 2] / s[0, 1],
                     s[0, 0] * s[0, 1] / s[0, 2]])
    assert abs(energy - (-1.3 ** 2 / 3.0 * np.sum(mass * field ** 2))) < 3e-12


def test_invalid_stretch_and_wave_number():
    v, t = jittered_box(1)
    s = np.ones((len(t), 3), complex)
    s[2, 1] = 0.0
    A, st = ff.assemble_tetra_nedelec_pml_csc(v, t, 2, s, 1.0)
    assert A is None and st.code == K.FFG_INVALID_INPUT
    A, st = ff.assemble_tetra_nedelec_pml_csc(v, t, 2, np.ones((len(t), 3)), 0.0)
    assert A is None and st.code == K.FFG_INVALID_INPUT
    S = np.tile(np.eye(3, dtype=complex), (len(t), 1, 1))
    S[1] = 0.0
    A, st = ff.assemble_tetra_nedelec_curvilinear_pml_csc(v, t, 2, S, 1.0)
    assert A is None and st.code == K.FFG_INVALID_INPUT
