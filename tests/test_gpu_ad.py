"""Forward (JVP) and reverse (VJP) mode of the tetrahedral Lagrange stiffness +
mass and the Nedelec curl + mass CSC assembly on the GPU, through the C-ABI.

Restates test/test_tetra_lagrange_stiffness_csc_ad.f90 and
test/test_tetra_nedelec_curl_mass_csc_ad.f90 (central differences of complete
reassembly, step 2e-7, relative 5e-8; adjoint identity 3e-10), then checks
parity against the FP64 CPU oracle (patterns bit-exact, tangent values and
adjoints within relative 1e-12; 1e-11 at Nedelec order 5) and, at larger
sizes, the size-independent properties: the adjoint identity, linearity in
the coefficient tangents, the coefficient adjoints as bilinear forms of the
primal, the primal pattern and run-to-run reproducibility.
"""
import numpy as np
import pytest

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K
from fortfem_b200 import synth

pytestmark = pytest.mark.gpu

REL = 1e-12
STEP = 2.0e-7
COEF = (1.7, 0.8, 0.13, -0.09)  # stiffness, mass and their tangents


def rel_frob(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def jittered_box(n, delta=0.1, seed=7):
    v, t = oracle.box_mesh([n, n, n])
    return synth.jitter_interior(v, 1.0 / n, delta, seed), t


def reference_case():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], float)
    t = np.array([[0, 1, 2, 3], [1, 2, 3, 4]], np.int32)
    vd = np.array([[0.01, -0.02, 0.015], [-0.03, 0.01, 0.02], [0.025, -0.015, 0.005],
                   [-0.01, 0.03, -0.02], [0.02, -0.01, 0.025]])
    return v, t, vd


def test_reference_csc_ad_case():
    v, t, vd = reference_case()
    k, m, kd, md = COEF
    p, q, h = 2, 6, STEP
    A, st = ff.assemble_tetra_lagrange_stiffness_csc(v, t, p, q, k, m)
    assert st.code == 0
    D, st = ff.assemble_tetra_lagrange_stiffness_csc_jvp(v, t, p, q, k, m, vd, kd, md)
    assert st.code == 0
    assert np.array_equal(D.col_ptr, A.col_ptr) and np.array_equal(D.row_idx, A.row_idx)
    plus, _ = ff.assemble_tetra_lagrange_stiffness_csc(v + h * vd, t, p, q, k + h * kd, m + h * md)
    minus, _ = ff.assemble_tetra_lagrange_stiffness_csc(v - h * vd, t, p, q, k - h * kd, m - h * md)
    err = np.abs(D.val - (plus.val - minus.val) / (2 * h)).max() / max(1.0, np.abs(D.val).max())
    assert err < 5e-8
    e = np.arange(1, len(A.val) + 1, dtype=float)
    bar = 0.003 * e - 0.00001 * e ** 2
    vbar, sbar, mbar, st = ff.assemble_tetra_lagrange_stiffness_csc_vjp(v, t, p, q, k, m, bar)
    assert st.code == 0
    lhs = bar @ D.val
    rhs = np.sum(vbar * vd) + sbar * kd + mbar * md
    assert abs(lhs - rhs) < 3e-10 * max(1.0, abs(lhs), abs(rhs))


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("rule", [0, 1])
def test_jvp_matches_oracle(p, rule):
    v, t = jittered_box(3)
    vd = np.random.default_rng(p).standard_normal(v.shape) * 0.05
    k, m, kd, md = COEF
    q = 2 * p + 4
    D, st = ff.assemble_tetra_lagrange_stiffness_csc_jvp(v, t, p, q, k, m, vd, kd, md, rule=rule)
    assert st.code == 0
    n, cp, ri, val = oracle.lagrange_csc_jvp(v, t, p, vd, k, m, kd, md, rule=rule, q=q)
    assert D.nrow == n and np.array_equal(D.col_ptr, cp) and np.array_equal(D.row_idx, ri)
    assert rel_frob(D.val, val) <= REL


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("rule", [0, 1])
def test_vjp_matches_oracle(p, rule):
    v, t = jittered_box(3)
    k, m, _, _ = COEF
    q = 2 * p + 4
    nnz = oracle.lagrange_csc(v, t, p, rule, q, k, m)[3].size
    bar = np.random.default_rng(10 + p).standard_normal(nnz)
    vbar, sbar, mbar, st = ff.assemble_tetra_lagrange_stiffness_csc_vjp(v, t, p, q, k, m, bar,
                                                                       rule=rule)
    assert st.code == 0
    ovbar, osbar, ombar = oracle.lagrange_csc_vjp(v, t, p, bar, k, m, rule=rule, q=q)
    assert rel_frob(vbar, ovbar) <= REL
    # coefficient adjoints: relative to the magnitudes of their nnz terms
    unit_k = oracle.lagrange_csc(v, t, p, rule, q, 1.0, 0.0)[3]
    unit_m = oracle.lagrange_csc(v, t, p, rule, q, 0.0, 1.0)[3]
    assert abs(sbar - osbar) <= REL * (np.abs(bar) @ np.abs(unit_k))
    assert abs(mbar - ombar) <= REL * (np.abs(bar) @ np.abs(unit_m))


def test_full_size_properties():
    # 16^3 box, 24576 cells, P2: identities that hold at any size
    v, t = jittered_box(16, 0.15, 3)
    rng = np.random.default_rng(5)
    vd = rng.standard_normal(v.shape) * 0.01
    k, m, kd, md = COEF
    p, q = 2, 8
    A, st = ff.assemble_tetra_lagrange_stiffness_csc(v, t, p, q, k, m)
    assert st.code == 0
    D, st = ff.assemble_tetra_lagrange_stiffness_csc_jvp(v, t, p, q, k, m, vd, kd, md)
    assert st.code == 0
    assert np.array_equal(D.col_ptr, A.col_ptr) and np.array_equal(D.row_idx, A.row_idx)
    bar = rng.standard_normal(len(A.val))
    vbar, sbar, mbar, st = ff.assemble_tetra_lagrange_stiffness_csc_vjp(v, t, p, q, k, m, bar)
    assert st.code == 0
    lhs = bar @ D.val
    rhs = np.sum(vbar * vd) + sbar * kd + mbar * md
    assert abs(lhs - rhs) < 1e-11 * max(1.0, np.abs(bar).sum() * np.abs(D.val).max())
    # a pure coefficient tangent is the primal assembly with that coefficient
    Ks, st = ff.assemble_tetra_lagrange_stiffness_csc_jvp(v, t, p, q, k, m, np.zeros_like(v), kd,
                                                          0.0)
    assert st.code == 0
    Ps, _ = ff.assemble_tetra_lagrange_stiffness_csc(v, t, p, q, kd, 0.0)
    assert rel_frob(Ks.val, Ps.val) <= 1e-14
    Km, st = ff.assemble_tetra_lagrange_stiffness_csc_jvp(v, t, p, q, k, m, np.zeros_like(v), 0.0,
                                                          md)
    Pm, _ = ff.assemble_tetra_lagrange_stiffness_csc(v, t, p, q, 0.0, md)
    assert rel_frob(Km.val, Pm.val) <= 1e-14
    # the coefficient adjoints are the primal's bilinear forms <bar, dA/dk>
    Pk, _ = ff.assemble_tetra_lagrange_stiffness_csc(v, t, p, q, 1.0, 0.0)
    Pmm, _ = ff.assemble_tetra_lagrange_stiffness_csc(v, t, p, q, 0.0, 1.0)
    assert abs(sbar - bar @ Pk.val) <= 1e-12 * np.abs(bar) @ np.abs(Pk.val)
    assert abs(mbar - bar @ Pmm.val) <= 1e-12 * np.abs(bar) @ np.abs(Pmm.val)
    # reproducible run to run
    vbar2, sbar2, mbar2, _ = ff.assemble_tetra_lagrange_stiffness_csc_vjp(v, t, p, q, k, m, bar)
    assert np.array_equal(vbar, vbar2) and sbar == sbar2 and mbar == mbar2


def test_errors():
    v, t, vd = reference_case()
    k, m, kd, md = COEF
    A, _ = ff.assemble_tetra_lagrange_stiffness_csc(v, t, 2, 6, k, m)
    # cotangent of the wrong length
    vbar, sbar, mbar, st = ff.assemble_tetra_lagrange_stiffness_csc_vjp(
        v, t, 2, 6, k, m, np.ones(len(A.val) + 1))
    assert st.code == K.FFG_INVALID_INPUT and not vbar.any() and sbar == 0.0 and mbar == 0.0
    # tangent of the wrong shape
    D, st = ff.assemble_tetra_lagrange_stiffness_csc_jvp(v, t, 2, 6, k, m, vd[:4], kd, md)
    assert D is None and st.code == K.FFG_INVALID_INPUT
    # a flat cell: every vertex of cell 0 in the plane z = 0
    flat = v.copy()
    flat[3] = [0.3, 0.3, 0.0]
    D, st = ff.assemble_tetra_lagrange_stiffness_csc_jvp(flat, t, 2, 6, k, m, vd, kd, md)
    assert D is None and st.code == K.FFG_INVALID_INPUT
    vbar, sbar, mbar, st = ff.assemble_tetra_lagrange_stiffness_csc_vjp(flat, t, 2, 6, k, m,
                                                                       np.ones(len(A.val)))
    assert st.code == K.FFG_INVALID_INPUT and not vbar.any()
    # vertex index out of range
    bad = t.copy()
    bad[1, 3] = 99
    D, st = ff.assemble_tetra_lagrange_stiffness_csc_jvp(v, bad, 2, 6, k, m, vd, kd, md)
    assert D is None and st.code == K.FFG_INVALID_INPUT


# ------------------------------------------------------------------ Nedelec
NED_COEF = (1.7, -0.8, 0.13, -0.09)  # curl, mass and their tangents


def test_reference_nedelec_csc_ad_case():
    # test/test_tetra_nedelec_curl_mass_csc_ad.f90 (order 2)
    v, t, vd = reference_case()
    c, m, cd, md = NED_COEF
    k, h = 2, STEP
    A, st = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, c, m, order=k)
    assert st.code == 0
    D, st = ff.assemble_tetra_nedelec_curl_mass_csc_jvp(v, t, k, c, m, vd, cd, md)
    assert st.code == 0
    assert np.array_equal(D.col_ptr, A.col_ptr) and np.array_equal(D.row_idx, A.row_idx)
    plus, _ = ff.assemble_tetra_nedelec_curl_mass_csc(v + h * vd, t, c + h * cd, m + h * md, order=k)
    minus, _ = ff.assemble_tetra_nedelec_curl_mass_csc(v - h * vd, t, c - h * cd, m - h * md,
                                                       order=k)
    err = np.abs(D.val - (plus.val - minus.val) / (2 * h)).max() / max(1.0, np.abs(D.val).max())
    assert err < 5e-8
    e = np.arange(1, len(A.val) + 1, dtype=float)
    bar = 0.003 * e - 0.00001 * e ** 2
    vbar, cbar, mbar, st = ff.assemble_tetra_nedelec_curl_mass_csc_vjp(v, t, k, c, m, bar)
    assert st.code == 0
    lhs = bar @ D.val
    rhs = np.sum(vbar * vd) + cbar * cd + mbar * md
    assert abs(lhs - rhs) < 3e-10 * max(1.0, abs(lhs), abs(rhs))


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_nedelec_jvp_vjp_match_oracle(k):
    v, t = jittered_box(2, 0.1, 11)
    rng = np.random.default_rng(20 + k)
    vd = rng.standard_normal(v.shape) * 0.05
    c, m, cd, md = NED_COEF
    D, st = ff.assemble_tetra_nedelec_curl_mass_csc_jvp(v, t, k, c, m, vd, cd, md)
    assert st.code == 0
    n, cp, ri, val = oracle.nedelec_csc_jvp(v, t, k, vd, c, m, cd, md)
    assert D.nrow == n and np.array_equal(D.col_ptr, cp) and np.array_equal(D.row_idx, ri)
    tol = 1e-12 if k <= 4 else 1e-11
    assert rel_frob(D.val, val) <= tol
    bar = rng.standard_normal(len(val))
    vbar, cbar, mbar, st = ff.assemble_tetra_nedelec_curl_mass_csc_vjp(v, t, k, c, m, bar)
    assert st.code == 0
    ovbar, ocbar, ombar = oracle.nedelec_csc_vjp(v, t, k, bar, c, m)
    assert rel_frob(vbar, ovbar) <= tol
    # the coefficient adjoints are sums of nnz signed terms <bar, dA/dc>:
    # relative to the sum of their magnitudes
    unit_c = oracle.nedelec_csc(v, t, k, 1.0, 0.0)[3]
    unit_m = oracle.nedelec_csc(v, t, k, 0.0, 1.0)[3]
    assert abs(cbar - ocbar) <= tol * (np.abs(bar) @ np.abs(unit_c))
    assert abs(mbar - ombar) <= tol * (np.abs(bar) @ np.abs(unit_m))


def test_nedelec_order6_ad_identities():
    # order 6 (216 local DoFs): the cotangent lives in global memory; two cells
    v, t, vd = reference_case()
    c, m, cd, md = NED_COEF
    k = 6
    D, st = ff.assemble_tetra_nedelec_curl_mass_csc_jvp(v, t, k, c, m, vd, cd, md)
    assert st.code == 0
    A, st = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, c, m, order=k)
    assert np.array_equal(D.col_ptr, A.col_ptr) and np.array_equal(D.row_idx, A.row_idx)
    bar = np.random.default_rng(6).standard_normal(len(A.val))
    vbar, cbar, mbar, st = ff.assemble_tetra_nedelec_curl_mass_csc_vjp(v, t, k, c, m, bar)
    assert st.code == 0
    lhs = bar @ D.val
    rhs = np.sum(vbar * vd) + cbar * cd + mbar * md
    assert abs(lhs - rhs) < 1e-10 * max(1.0, np.abs(bar) @ np.abs(D.val))
    # a pure coefficient tangent is the primal with that coefficient
    Kc, _ = ff.assemble_tetra_nedelec_curl_mass_csc_jvp(v, t, k, c, m, np.zeros_like(v), cd, 0.0)
    Pc, _ = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, cd, 0.0, order=k)
    assert rel_frob(Kc.val, Pc.val) <= 1e-13


def test_nedelec_full_size_properties():
    # 8^3 box, 3072 cells, order 3: the adjoint identity, the coefficient
    # adjoints as bilinear forms, and reproducibility
    v, t = jittered_box(8, 0.1, 4)
    rng = np.random.default_rng(8)
    vd = rng.standard_normal(v.shape) * 0.01
    c, m, cd, md = NED_COEF
    k = 3
    D, st = ff.assemble_tetra_nedelec_curl_mass_csc_jvp(v, t, k, c, m, vd, cd, md)
    assert st.code == 0
    bar = rng.standard_normal(len(D.val))
    vbar, cbar, mbar, st = ff.assemble_tetra_nedelec_curl_mass_csc_vjp(v, t, k, c, m, bar)
    assert st.code == 0
    lhs = bar @ D.val
    rhs = np.sum(vbar * vd) + cbar * cd + mbar * md
    assert abs(lhs - rhs) < 1e-11 * max(1.0, np.abs(bar) @ np.abs(D.val))
    Pc, _ = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, 1.0, 0.0, order=k)
    Pm, _ = ff.assemble_tetra_nedelec_curl_mass_csc(v, t, 0.0, 1.0, order=k)
    assert abs(cbar - bar @ Pc.val) <= 1e-12 * np.abs(bar) @ np.abs(Pc.val)
    assert abs(mbar - bar @ Pm.val) <= 1e-12 * np.abs(bar) @ np.abs(Pm.val)
    vbar2, cbar2, mbar2, _ = ff.assemble_tetra_nedelec_curl_mass_csc_vjp(v, t, k, c, m, bar)
    assert np.array_equal(vbar, vbar2) and cbar == cbar2 and mbar == mbar2
