"""Pin the CPU oracle against the reference's own known-answer tests.

Each test cites the reference test it restates; tolerances are the reference's.
"""
import json
import math
import os
import sys
from fractions import Fraction

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))


def fact(n):
    return math.factorial(n)


# test/test_tetra_duffy_quadrature.f90:13-36
def test_duffy_exactness():
    for degree in range(8):
        x, y, z, w = oracle.tetra_duffy(degree)
        assert abs(w.sum() - 1.0 / 6.0) < 2e-14
        for zd in range(degree + 1):
            for yd in range(degree - zd + 1):
                for xd in range(degree - yd - zd + 1):
                    num = np.sum(w * x ** xd * y ** yd * z ** zd)
                    exact = fact(xd) * fact(yd) * fact(zd) / fact(xd + yd + zd + 3)
                    assert abs(num - exact) < 4e-14


def test_gauss_legendre_matches_numpy():
    for n in range(1, 12):
        x, w = oracle.gauss_legendre(n, 0.0, 1.0)
        xr, wr = np.polynomial.legendre.leggauss(n)
        assert np.allclose(x, 0.5 * xr + 0.5, atol=1e-15, rtol=0)
        assert np.allclose(w, 0.5 * wr, atol=1e-15, rtol=0)


def test_degree_two_rule_is_degree_two_exact():
    p, w = oracle.degree_two_rule()
    for xd, yd, zd in [(0, 0, 0), (1, 0, 0), (0, 2, 0), (1, 1, 0), (0, 0, 2), (0, 1, 1)]:
        num = np.sum(w * p[:, 0] ** xd * p[:, 1] ** yd * p[:, 2] ** zd)
        exact = fact(xd) * fact(yd) * fact(zd) / fact(xd + yd + zd + 3)
        assert abs(num - exact) < 1e-15


# test/test_structured_tetra_box_mesh.f90:19-51
def test_box_mesh_invariants():
    bounds = ((-1.0, 0.5, 2.0), (1.0, 2.0, 3.5))
    v, t = oracle.box_mesh([2, 1, 3], bounds)
    assert len(v) == 3 * 2 * 4 and len(t) == 36
    assert np.allclose(v.min(0), bounds[0], atol=1e-14) and np.allclose(v.max(0), bounds[1], atol=1e-14)
    J = np.stack([v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]], v[t[:, 3]] - v[t[:, 0]]], axis=2)
    det = np.linalg.det(J)
    assert (det > 0).all()
    assert abs(det.sum() / 6 - 2.0 * 1.5 * 1.5) < 1e-12


# test/test_tetra_lagrange_arbitrary_order.f90:22-73 (partition of unity, nodal property)
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_lagrange_partition_and_nodal(p):
    idx, nodes = oracle.lagrange_indices(p)
    v, g = oracle.lagrange_evaluate(p, [0.13, 0.21, 0.37])
    assert abs(v.sum() - 1.0) < 3e-13 and np.abs(g.sum(0)).max() < 3e-13
    for i, node in enumerate(nodes):
        v, _ = oracle.lagrange_evaluate(p, node)
        e = np.zeros(len(nodes)); e[i] = 1
        assert np.abs(v - e).max() < 3e-13


# test/test_tetra_lagrange_global_dof_map.f90:17-47
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_lagrange_dof_map_shared_face(p):
    tets = np.array([[0, 1, 2, 3], [2, 1, 0, 4]])
    idx, _ = oracle.lagrange_indices(p)
    for faithful in (False, True):
        gd, n = oracle.lagrange_dof_map(p, tets, faithful=faithful)
        shared = [l for l in range(len(idx)) if idx[l, 3] == 0]
        for l in shared:
            assert gd[0, l] in gd[1]
        assert len(shared) == (p + 1) * (p + 2) // 2
        assert n == 2 * (p + 1) * (p + 2) * (p + 3) // 6 - len(shared)


def test_lagrange_dof_map_rejects():
    tets = np.array([[0, 1, 2, 3], [2, 1, 0, 4]])
    with pytest.raises(oracle.OracleError):
        oracle.lagrange_dof_map(0, tets)
    with pytest.raises(oracle.OracleError):
        oracle.lagrange_dof_map(2, np.array([[0, 1, 2, 3], [0, 0, 1, 4]]))


@pytest.mark.parametrize("p", [1, 2, 3])
def test_lagrange_dof_map_hash_equals_faithful(p):
    v, t = oracle.box_mesh([2, 2, 2])
    a, na = oracle.lagrange_dof_map(p, t, faithful=False)
    b, nb = oracle.lagrange_dof_map(p, t, faithful=True)
    assert na == nb and (a == b).all()


# test/test_tetra_lagrange_arbitrary_order_assembly.f90:28-66
def test_lagrange_element_symmetry_and_linear_energy():
    verts = np.array([[0.2, -0.3, 0.1], [2.1, -0.5, 0.4], [0.6, 1.4, -0.2], [-0.1, 0.2, 1.6]])
    for p in range(1, 5):
        m = oracle.lagrange_element(verts.reshape(-1), p, 0, 2 * p + 2)
        assert np.abs(m - m.T).max() < 2e-11
    mv = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1.0]])
    tets = np.array([[0, 1, 2, 3], [0, 2, 1, 4]])
    n, cp, ri, val = oracle.lagrange_csc(mv, tets, 1, 0, 4)
    gd, _ = oracle.lagrange_dof_map(1, tets)
    coef = np.zeros(n)
    coef[gd.reshape(-1)] = mv[tets.reshape(-1), 0]
    y = oracle.csc_matvec(n, cp, ri, val, coef)
    assert abs(coef @ y - 1.0 / 3.0) < 2e-12


def test_lagrange_dirichlet_hash_equals_faithful():
    v, t = oracle.box_mesh([2, 2, 2])
    for p in (1, 2):
        a, pa = oracle.lagrange_dirichlet(p, v, t, faithful=False)
        b, pb = oracle.lagrange_dirichlet(p, v, t, faithful=True)
        assert (a == b).all()
        assert np.allclose(pa[a], pb[b], atol=1e-15)
    # P2 on n^3: interior nodes are (2n-1)^3
    a, _ = oracle.lagrange_dirichlet(2, v, t)
    assert (~a).sum() == 3 ** 3


def test_csc_pattern_value_independent():
    # test/test_tetra_lagrange_stiffness_csc_ad.f90:62-67: pattern unchanged by values
    v, t = oracle.box_mesh([2, 2, 1])
    n1, cp1, ri1, _ = oracle.lagrange_csc(v, t, 2, 1, 0)
    n2, cp2, ri2, _ = oracle.lagrange_csc(v, t, 2, 1, 0, stiffness=0.0, mass=0.0)
    assert n1 == n2 and (cp1 == cp2).all() and (ri1 == ri2).all()


def test_csc_from_triplet_sums_duplicates():
    cp, ri, v = oracle.csc_from_triplet(3, 3, [2, 0, 2, 1], [0, 0, 0, 2], [1.0, 2.0, 3.0, 4.0])
    assert list(cp) == [0, 2, 2, 3] and list(ri) == [0, 2, 1]
    assert list(v) == [2.0, 4.0, 4.0]


# test/test_advanced_solvers.f90:768-797 (sparse Jacobi-PCG agrees with the dense path)
def test_pcg_sparse_matches_dense():
    v, t = oracle.unit_square_mesh(9)
    a = oracle.p1_dense(v, t, mass=1.0, stiffness=1.0)
    n, cp, ri, val = oracle.p1_csc(v, t, mass=1.0, stiffness=1.0)
    b = oracle.p1_load(v, t, 1.0)
    # the reference's absolute breakdown guard |p^T A p| < 1e-14 ends small
    # systems early, so the load is scaled to keep p^T A p above it
    b = 1e3 * b
    xd, sd = oracle.pcg_dense(a, b, tol=1e-10)
    xs, ss = oracle.pcg_sparse(n, cp, ri, val, b, tol=1e-10)
    assert sd["converged"] and ss["converged"]
    assert np.abs(xd - xs).max() < 1e-6
    assert np.abs(a @ xs - b).max() < 1e-8 * np.abs(b).max()


def test_p1_csc_matches_dense_and_boundary():
    v, t = oracle.unit_square_mesh(65)
    assert len(v) == 4225 and len(t) == 8192
    bnd = oracle.square_boundary(len(v), t)
    assert bnd.sum() == 256
    n, cp, ri, val = oracle.p1_csc(v[:400] if False else v, t)
    assert cp[-1] == 29057
    import scipy.sparse as sp
    v9, t9 = oracle.unit_square_mesh(9)
    a = oracle.p1_dense(v9, t9, 0.0, 1.0)
    n9, cp9, ri9, val9 = oracle.p1_csc(v9, t9, 0.0, 1.0)
    assert np.abs(sp.csc_matrix((val9, ri9, cp9), shape=(n9, n9)).toarray() - a).max() < 1e-15


def _constant_field_dofs(k, verts, tets, dm, field):
    """set_constant_field_dofs of test/test_tetra_nedelec_sparse_assembly_slow.f90:92-170."""
    edges, faces, gd = dm["edges"], dm["faces"], dm["global_dofs"]
    dofs = np.zeros(dm["n_global"])
    for e, (a, b) in enumerate(edges):
        dofs[e * k] = field @ (verts[b] - verts[a])
    fdc = k * (k - 1)
    off = k * len(edges)
    for f, fv in enumerate(faces):
        for comp in range(2):
            tang = verts[fv[comp + 1]] - verts[fv[0]]
            mono = 0
            for d in range(k - 1):
                for xd in range(d + 1):
                    yd = d - xd
                    mono += 1
                    dof = off + f * fdc + comp * fdc // 2 + mono - 1
                    if k <= 5:
                        dofs[dof] = (field @ tang) * fact(xd) * fact(yd) / fact(xd + yd + 2)
                    else:  # orthogonal (Dubiner) weights: only the constant one integrates
                        dofs[dof] = 0.5 * (field @ tang) if d == 0 else 0.0
    base = 6 * k + 4 * fdc
    for c, tet in enumerate(tets):
        J = np.stack([verts[tet[1]] - verts[tet[0]], verts[tet[2]] - verts[tet[0]],
                      verts[tet[3]] - verts[tet[0]]], axis=1)
        rf = J.T @ field
        loc = base
        for comp in range(3):
            for d in range(k - 2):
                for xd in range(d + 1):
                    for yd in range(d - xd + 1):
                        zd = d - xd - yd
                        if k <= 5:
                            dofs[gd[c, loc]] = rf[comp] * fact(xd) * fact(yd) * fact(zd) / fact(d + 3)
                        else:  # orthogonal (Koornwinder) weights
                            dofs[gd[c, loc]] = rf[comp] / 6.0 if d == 0 else 0.0
                        loc += 1
    return dofs


# test/test_tetra_nedelec_sparse_assembly_slow.f90:31-85
def test_nedelec_energy_kats():
    verts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1.0]])
    tets = np.array([[0, 1, 2, 3], [0, 2, 1, 4]])
    edges, _, _ = oracle.edge_dof_map(tets)
    assert len(edges) == 9
    field = np.array([1.0, 2.0, -1.0])
    dofs = np.array([field @ (verts[b] - verts[a]) for a, b in edges])
    n, cp, ri, val = oracle.nedelec_csc(verts, tets, 1, 4.0, 1.5)
    y = oracle.csc_matvec(n, cp, ri, val, dofs)
    assert abs(dofs @ y - 3.0) < 2e-12
    curl = np.array([1.0, -2.0, 3.0])
    dofs = np.array([(0.5 * np.cross(curl, 0.5 * (verts[a] + verts[b]))) @ (verts[b] - verts[a])
                     for a, b in edges])
    n, cp, ri, val = oracle.nedelec_csc(verts, tets, 1, 2.0, 0.0)
    y = oracle.csc_matvec(n, cp, ri, val, dofs)
    assert abs(dofs @ y - 28.0 / 3.0) < 3e-12
    for k in range(2, 7):
        dm = oracle.nedelec_dof_map(k, tets)
        dofs = _constant_field_dofs(k, verts, tets, dm, field)
        n, cp, ri, val = oracle.nedelec_csc(verts, tets, k, 4.0, 1.5)
        y = oracle.csc_matvec(n, cp, ri, val, dofs)
        assert abs(dofs @ y - 3.0) < 1e-8, k


# test/test_tetra_nedelec_global_dof_map.f90:22-74 (topology numbers at order 6)
def test_nedelec_order6_topology():
    tets = np.array([[0, 1, 2, 3], [2, 0, 1, 4]])
    for faithful in (False, True):
        dm = oracle.nedelec_dof_map(6, tets, faithful=faithful)
        assert len(dm["edges"]) == 9 and len(dm["faces"]) == 7
        assert dm["global_dofs"].shape[1] == 216 and dm["n_global"] == 384
        fs = 6 * 6
        assert (dm["global_dofs"][0, fs:fs + 30] == dm["global_dofs"][1, fs:fs + 30]).all()
        assert list(dm["face_permutations"][0, 0]) == [1, 2, 3]
        assert list(dm["face_permutations"][1, 0]) == [3, 1, 2]


@pytest.mark.parametrize("k", [2, 3, 4])
def test_nedelec_transform_signs_and_roundtrip(k):
    tets = np.array([[0, 1, 2, 3], [2, 0, 1, 4]])
    dm = oracle.nedelec_dof_map(k, tets)
    T = oracle.nedelec_transform(k, dm["edge_orientations"][1], dm["face_permutations"][1])
    signs = [T[i, i] for i in range(k)]
    assert signs == [(-1.0 if m % 2 == 0 else 1.0) for m in range(k)]  # reversed edge 1
    # shared face: both cells give the same canonical coefficients
    fdc = k * (k - 1); fs = 6 * k
    T0 = oracle.nedelec_transform(k, dm["edge_orientations"][0], dm["face_permutations"][0])
    canonical = np.array([(2 * m - 7) / (m + 2) for m in range(1, fdc + 1)])
    b0 = T0[fs:fs + fdc, fs:fs + fdc] @ canonical
    assert np.allclose(b0, canonical)


def test_nedelec_dof_maps_hash_equals_faithful():
    v, t = oracle.box_mesh([2, 2, 2])
    for k in (1, 2, 3):
        a = oracle.nedelec_dof_map(k, t, faithful=False)
        b = oracle.nedelec_dof_map(k, t, faithful=True)
        for key in ("edges", "faces", "global_dofs", "edge_orientations", "face_permutations"):
            assert (a[key] == b[key]).all(), key
        assert (oracle.pec_mask(k, t, False) == oracle.pec_mask(k, t, True)).all()


def test_whitney_equals_order1_table_basis():
    for pt in ([0.1, 0.2, 0.3], [0.25, 0.25, 0.25], [0.0, 0.5, 0.1]):
        a = oracle.whitney_evaluate(pt)
        b = oracle.nedelec_evaluate(1, pt)
        assert np.abs(a[0] - b[0]).max() < 1e-15 and np.abs(a[1] - b[1]).max() < 1e-15


# The repository's exact generator against the reference's generated tables
def test_generated_tables_match_reference_digests():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import canonical_digest
    from fortfem_b200.gen_nedelec_tables import PERMUTATIONS, coefficients, face_transform
    fx = json.load(open(os.path.join(HERE, "golden", "nedelec_tables.json")))
    for k in (1, 2, 3, 4):
        Cm = coefficients(k)
        n = len(Cm)
        ent = {(r + 1, c + 1): Cm[r][c] for r in range(n) for c in range(n) if Cm[r][c] != 0}
        assert canonical_digest(ent) == fx["coefficients"][str(k)]["digest"]
        for r, c, s in fx["coefficients"][str(k)]["samples"]:
            assert Cm[r - 1][c - 1] == Fraction(s)
    for k in (2, 3, 4):
        for pi, perm in enumerate(PERMUTATIONS):
            T = face_transform(k, perm)
            n = len(T)
            ent = {(r + 1, c + 1): T[r][c] for r in range(n) for c in range(n) if T[r][c] != 0}
            assert canonical_digest(ent) == fx["face_transforms"][f"{k}/{pi + 1}"]["digest"]


def test_emitted_tables_are_rounded_exact_values():
    from fortfem_b200.gen_nedelec_tables import coefficients
    path = os.path.join(os.path.dirname(HERE), "fortfem_b200", "csrc", "nedelec_tables.inc")
    text = open(path).read()
    import re
    for k in (1, 2, 3):
        m = re.search(rf"kNedelecCoefficients{k}\[\d+\] = \{{(.*?)\}};", text)
        vals = [float.fromhex(s.strip()) for s in m.group(1).split(",")]
        Cm = coefficients(k)
        n = len(Cm)
        assert vals == [float(Cm[r][c]) for c in range(n) for r in range(n)]


# ---------------------------------------------------------------- JVP / VJP
# test/test_tetra_lagrange_element_ad.f90:9-79 and
# test/test_tetra_lagrange_stiffness_csc_ad.f90:10-91: central differences of
# complete reassembly (step 2e-7, relative 5e-8) and the adjoint identity
# <Kbar, Kdot> = <vbar, vdot> + kbar kdot + mbar mdot (2e-10 / 3e-10).
AD_STEP = 2.0e-7
AD_COEF = (1.7, 0.8, 0.13, -0.09)  # stiffness, mass and their tangents
AD_VDOT = [[0.01, -0.02, 0.015], [-0.03, 0.01, 0.02], [0.025, -0.015, 0.005],
           [-0.01, 0.03, -0.02], [0.02, -0.01, 0.025]]


def test_lagrange_element_jvp_vjp_kat():
    v = np.array([[0.1, -0.2, 0.3], [1.3, -0.1, 0.25], [0.25, 0.9, 0.35], [0.0, 0.1, 1.4]])
    vd = np.array(AD_VDOT[:4])
    k, m, kd, md = AD_COEF
    p, q, h = 2, 6, AD_STEP
    kdot = oracle.lagrange_element_jvp(v, p, vd, k, m, kd, md, q=q)
    plus = oracle.lagrange_element(v + h * vd, p, q=q, stiffness=k + h * kd, mass=m + h * md)
    minus = oracle.lagrange_element(v - h * vd, p, q=q, stiffness=k - h * kd, mass=m - h * md)
    err = np.abs(kdot - (plus - minus) / (2 * h)).max() / max(1.0, np.abs(kdot).max())
    assert err < 5e-8
    nb = kdot.shape[0]
    r, c = np.meshgrid(np.arange(1, nb + 1), np.arange(1, nb + 1), indexing="ij")
    kbar = 0.002 * r - 0.0015 * c
    vbar, sbar, mbar = oracle.lagrange_element_vjp(v, p, kbar, k, m, q=q)
    lhs = np.sum(kbar * kdot)
    rhs = np.sum(vbar * vd) + sbar * kd + mbar * md
    assert abs(lhs - rhs) < 2e-10 * max(1.0, abs(lhs), abs(rhs))


def test_lagrange_csc_jvp_vjp_kat():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], float)
    t = np.array([[0, 1, 2, 3], [1, 2, 3, 4]], np.int32)
    vd = np.array(AD_VDOT)
    k, m, kd, md = AD_COEF
    p, q, h = 2, 6, AD_STEP
    n, cp, ri, vdot = oracle.lagrange_csc_jvp(v, t, p, vd, k, m, kd, md, q=q)
    n0, cp0, ri0, _ = oracle.lagrange_csc(v, t, p, q=q, stiffness=k, mass=m)
    assert n == n0 and np.array_equal(cp, cp0) and np.array_equal(ri, ri0)
    _, _, _, plus = oracle.lagrange_csc(v + h * vd, t, p, q=q, stiffness=k + h * kd,
                                        mass=m + h * md)
    _, _, _, minus = oracle.lagrange_csc(v - h * vd, t, p, q=q, stiffness=k - h * kd,
                                         mass=m - h * md)
    err = np.abs(vdot - (plus - minus) / (2 * h)).max() / max(1.0, np.abs(vdot).max())
    assert err < 5e-8
    e = np.arange(1, len(vdot) + 1, dtype=float)
    vbar_in = 0.003 * e - 0.00001 * e ** 2
    vbar, sbar, mbar = oracle.lagrange_csc_vjp(v, t, p, vbar_in, k, m, q=q)
    lhs = vbar_in @ vdot
    rhs = np.sum(vbar * vd) + sbar * kd + mbar * md
    assert abs(lhs - rhs) < 3e-10 * max(1.0, abs(lhs), abs(rhs))


# test/test_tetra_nedelec_element_ad.f90 (order 2, quadrature degree 6) and
# test/test_tetra_nedelec_curl_mass_csc_ad.f90 (order 2, two cells): the same
# identities with curl 1.7, mass -0.8 and tangents 0.13, -0.09; orders 1 and 3
# through the same checks.
@pytest.mark.parametrize("k", [1, 2, 3])
def test_nedelec_element_jvp_vjp_kat(k):
    v = np.array([[0.1, -0.2, 0.3], [1.3, -0.1, 0.25], [0.25, 0.9, 0.35], [0.0, 0.1, 1.4]])
    vd = np.array(AD_VDOT[:4])
    c, m, cd, md = 1.7, -0.8, 0.13, -0.09
    q, h = 6, AD_STEP
    kdot = oracle.nedelec_element_jvp(v, k, vd, c, m, cd, md, q=q)
    plus = oracle.nedelec_element(v + h * vd, k, q=q, curl=c + h * cd, mass=m + h * md)
    minus = oracle.nedelec_element(v - h * vd, k, q=q, curl=c - h * cd, mass=m - h * md)
    err = np.abs(kdot - (plus - minus) / (2 * h)).max() / max(1.0, np.abs(kdot).max())
    assert err < 5e-8
    nb = kdot.shape[0]
    r, cc = np.meshgrid(np.arange(1, nb + 1), np.arange(1, nb + 1), indexing="ij")
    kbar = 0.002 * r - 0.0015 * cc
    vbar, cbar, mbar = oracle.nedelec_element_vjp(v, k, kbar, c, m, q=q)
    lhs = np.sum(kbar * kdot)
    rhs = np.sum(vbar * vd) + cbar * cd + mbar * md
    assert abs(lhs - rhs) < 2e-10 * max(1.0, abs(lhs), abs(rhs))


@pytest.mark.parametrize("k", [1, 2, 3])
def test_nedelec_csc_jvp_vjp_kat(k):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], float)
    t = np.array([[0, 1, 2, 3], [1, 2, 3, 4]], np.int32)
    vd = np.array(AD_VDOT)
    c, m, cd, md = 1.7, -0.8, 0.13, -0.09
    h = AD_STEP
    n, cp, ri, vdot = oracle.nedelec_csc_jvp(v, t, k, vd, c, m, cd, md)
    n0, cp0, ri0, _ = oracle.nedelec_csc(v, t, k, c, m)
    assert n == n0 and np.array_equal(cp, cp0) and np.array_equal(ri, ri0)
    _, _, _, plus = oracle.nedelec_csc(v + h * vd, t, k, c + h * cd, m + h * md)
    _, _, _, minus = oracle.nedelec_csc(v - h * vd, t, k, c - h * cd, m - h * md)
    err = np.abs(vdot - (plus - minus) / (2 * h)).max() / max(1.0, np.abs(vdot).max())
    assert err < 5e-8
    e = np.arange(1, len(vdot) + 1, dtype=float)
    vbar_in = 0.003 * e - 0.00001 * e ** 2
    vbar, cbar, mbar = oracle.nedelec_csc_vjp(v, t, k, vbar_in, c, m)
    lhs = vbar_in @ vdot
    rhs = np.sum(vbar * vd) + cbar * cd + mbar * md
    assert abs(lhs - rhs) < 3e-10 * max(1.0, abs(lhs), abs(rhs))


# ---------------------------------------------------------- solution probes
# test/test_tetra_lagrange_poisson_p_convergence.f90:11-19 (four cells around
# an interior vertex), :133-157 (affine Dirichlet data reproduced to 1e-12 by
# evaluate_tetra_lagrange_solution) and :159-181 (reaction with source 2 and
# no essential boundary gives the constant 2, zero gradient).
PROBE_TETS = np.array([[0, 1, 2, 4], [0, 3, 1, 4], [0, 2, 3, 4], [1, 3, 2, 4]], np.int32)
PROBE_VERTS = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.25, 0.25, 0.25]], float)


def _oracle_lagrange_solve(p, stiffness, mass, source, boundary_fn):
    v, t = PROBE_VERTS, PROBE_TETS
    q = 2 * p + 4
    n, cp, ri, val = oracle.lagrange_csc(v, t, p, 0, q, stiffness, mass)
    pts = oracle.lagrange_quadrature_points(v, t, 0, q)
    rhs = oracle.lagrange_load_samples(v, t, p, source(pts), 0, q)
    con, nodes = oracle.lagrange_dirichlet(p, v, t)
    if boundary_fn is None:
        con[:] = False
    g = np.where(con, boundary_fn(nodes) if boundary_fn else 0.0, 0.0)
    nf, rcp, rri, rv, rr, free = oracle.reduce_constrained(n, cp, ri, val, rhs, con, g)
    dense = oracle.csc_to_scipy(nf, rcp, rri, rv).toarray()
    u = g.copy()
    u[free] = np.linalg.solve(dense, rr)
    return u


def test_lagrange_evaluate_affine_and_reaction_kat():
    affine = lambda x: 1.0 + x[..., 0] + 2.0 * x[..., 1] - 3.0 * x[..., 2]
    u = _oracle_lagrange_solve(1, 1.0, 0.0, lambda x: 0.0 * x[..., 0], affine)
    value, grad = oracle.lagrange_evaluate_solution(PROBE_VERTS, PROBE_TETS, 1, u, 0,
                                                    [0.2, 0.3, 0.1])
    assert abs(value - affine(np.array([0.225, 0.325, 0.025]))) < 1e-12
    assert np.abs(grad - [1.0, 2.0, -3.0]).max() < 1e-12
    u = _oracle_lagrange_solve(1, 0.0, 1.0, lambda x: 2.0 + 0.0 * x[..., 0], None)
    value, grad = oracle.lagrange_evaluate_solution(PROBE_VERTS, PROBE_TETS, 1, u, 3,
                                                    [0.2, 0.1, 0.3])
    assert abs(value - 2.0) < 1e-12 and np.abs(grad).max() < 1e-12


def lagrange_node_points(v, t, p):
    """Physical location of every global Lagrange DoF (the cell's affine map of
    its reference nodes)."""
    gd, n = oracle.lagrange_dof_map(p, t)
    _, ref_nodes = oracle.lagrange_indices(p)
    out = np.zeros((n, 3))
    for c in range(len(t)):
        J = (v[t[c, 1:]] - v[t[c, 0]]).T
        out[gd[c]] = v[t[c, 0]] + ref_nodes @ J.T
    return out


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_lagrange_probe_reproduces_its_space(p):
    # nodal interpolation of a degree-p polynomial is exact: every evaluation
    # route returns the polynomial and its gradient
    v, t = oracle.box_mesh([2, 2, 2])
    f = lambda x: (1.0 + x[..., 0] - 2 * x[..., 1] + 0.5 * x[..., 2]) ** p
    df = lambda x: p * (1.0 + x[0] - 2 * x[1] + 0.5 * x[2]) ** (p - 1) * np.array([1, -2, 0.5])
    u = f(lagrange_node_points(v, t, p))
    rng = np.random.default_rng(p)
    for _ in range(5):
        x = rng.uniform(0.05, 0.95, 3)
        for mode in (0, 1):
            val, g, cnt = oracle.lagrange_probe(v, t, p, u, x, mode)
            assert cnt >= 1
            assert abs(val - f(x)) < 1e-12 * max(1, abs(f(x)))
            assert np.abs(g - df(x)).max() < 1e-10 * max(1, np.abs(df(x)).max())
    # a vertex of the box lies in several cells; mode 0 counts them all
    val, g, cnt = oracle.lagrange_probe(v, t, p, u, [0.5, 0.5, 0.5], 0)
    assert cnt > 1 and abs(val - f(np.array([0.5, 0.5, 0.5]))) < 1e-12
    # outside the mesh: no cell
    assert oracle.lagrange_probe(v, t, p, u, [1.5, 0.5, 0.5], 0)[2] == 0


@pytest.mark.parametrize("k", [1, 2, 3])
def test_nedelec_probe_reproduces_its_space(k):
    # the L2 projection of a field of the order-k space is the field itself:
    # k = 1 holds a + b x x (curl 2b); order k holds every degree-(k-1) field
    v, t = oracle.box_mesh([2, 2, 2])
    a, b = np.array([0.3, -0.7, 1.1]), np.array([0.5, 0.2, -0.4])

    def field(x):
        extra = {1: np.zeros(3), 2: np.array([x[1], 0.0, x[0]]),
                 3: np.array([x[1] * x[2], 0.0, x[0] ** 2])}[k]
        return a + np.cross(b, x) + extra

    def curl(x):
        extra = {1: np.zeros(3), 2: np.array([0.0, -1.0, -1.0]),
                 3: np.array([0.0, x[1] - 2 * x[0], -x[2]])}[k]
        return 2 * b + extra

    n, cp, ri, val = oracle.nedelec_csc(v, t, k, 0.0, 1.0)
    pts = oracle.nedelec_load_points(v, t, k)
    samples = np.array([[field(x) for x in cell] for cell in pts])
    rhs = oracle.nedelec_load_samples(v, t, k, samples)
    u = np.linalg.solve(oracle.csc_to_scipy(n, cp, ri, val).toarray(), rhs)
    rng = np.random.default_rng(k)
    for _ in range(4):
        x = rng.uniform(0.05, 0.95, 3)
        for mode in (0, 1):
            fv, fc, cnt = oracle.nedelec_probe(v, t, k, u, x, mode)
            assert cnt >= 1
            assert np.abs(fv - field(x)).max() < 1e-9
            assert np.abs(fc - curl(x)).max() < 1e-8


# ------------------------------------------------------------------ complex PML
# test/test_tetra_nedelec_pml_element.f90: unit stretch reduces to curl-curl
# minus k^2 mass (orders 1-4, 2e-12); an absorbing anisotropic stretch gives a
# complex-symmetric element with a nonzero imaginary part.
PML_TET = np.array([[0, 0, 0], [1.2, 0, 0], [0.1, 0.9, 0], [0, 0.2, 1.1]])


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_pml_element_unit_stretch_kat(k):
    wave = 1.7
    m = oracle.nedelec_pml_element(PML_TET, k, np.ones(3), wave, q=10)
    ref = oracle.nedelec_element(PML_TET, k, q=10, curl=1.0, mass=-wave ** 2)
    assert np.abs(m - ref).max() < 2e-12
    # the same with the curvilinear tensor form and S = I
    mc = oracle.nedelec_pml_element(PML_TET, k, np.eye(3), wave, q=10, curvilinear=True)
    assert np.abs(mc - ref).max() < 2e-12


def test_pml_element_absorbing_kat():
    s = np.array([1 + 0.8j, 1.0, 1.0])
    m = oracle.nedelec_pml_element(PML_TET, 2, s, 1.7, q=10)
    assert np.abs(m - m.T).max() < 2e-12
    assert np.abs(m.imag).max() > 1e-3
    # a diagonal curvilinear stretch is the Cartesian one
    mc = oracle.nedelec_pml_element(PML_TET, 2, np.diag(s), 1.7, q=10, curvilinear=True)
    assert np.abs(mc - m).max() < 1e-12 * np.abs(m).max()


# test/test_tetra_nedelec_pml_sparse.f90:21-52: order-1 global PML mass has the
# exact constant-field energy -k^2/3 sum_a m_a f_a^2 on two unit cells.
def test_pml_csc_constant_field_energy_kat():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, -1]], float)
    t = np.array([[0, 1, 2, 3], [0, 2, 1, 4]], np.int32)
    s = np.array([[1 + 0.6j, 1.0, 1.0]] * 2)
    n, cp, ri, val = oracle.nedelec_pml_csc(v, t, 1, s, 1.3)
    dm = oracle.nedelec_dof_map(1, t)
    edges = dm["edges"]
    field = np.array([1.0, 2.0, -1.0])
    dofs = np.array([field @ (v[b] - v[a]) for a, b in edges.T], complex) \
        if edges.shape[0] == 2 else np.array([field @ (v[b] - v[a]) for a, b in edges], complex)
    A = oracle.csc_to_scipy(n, cp, ri, val)
    energy = dofs @ (A @ dofs)
    mass = np.array([s[0, 1] * s[0, 2] / s[0, 0], s[0, 0] * s[0, 2] / s[0, 1],
                     s[0, 0] * s[0, 1] / s[0, 2]])
    expected = -1.3 ** 2 / 3.0 * np.sum(mass * field ** 2)
    assert abs(energy - expected) < 3e-12


# ------------------------------------------------- arbitrary-order triangles
# test/test_triangle_lagrange_arbitrary_order.f90:16-57 (degrees 0..4):
# Kronecker nodal values, partition of unity, zero gradient sum, and exact
# interpolation of every monomial of the degree.
@pytest.mark.parametrize("p", [0, 1, 2, 3, 4])
def test_triangle_lagrange_basis_kat(p):
    nodes, _ = oracle.triangle_lagrange_nodes(p)
    for d, (x, y) in enumerate(nodes):
        v, _ = oracle.triangle_lagrange_evaluate(p, x, y)
        e = np.zeros(len(v)); e[d] = 1.0
        assert np.abs(v - e).max() < 2e-12
    x, y = 0.23, 0.31
    v, g = oracle.triangle_lagrange_evaluate(p, x, y)
    assert abs(v.sum() - 1.0) < 2e-13 and np.abs(g.sum(axis=0)).max() < 5e-13
    for a in range(p + 1):
        for b in range(p - a + 1):
            c = nodes[:, 0] ** a * nodes[:, 1] ** b
            assert abs(c @ v - x ** a * y ** b) < 2e-12
            grad = [a * x ** (a - 1) * y ** b if a else 0.0, b * x ** a * y ** (b - 1) if b else 0.0]
            assert np.abs(c @ g - grad).max() < 8e-12


def test_triangle_lagrange_element_properties():
    v = np.array([[0.1, 0.2], [1.3, -0.1], [0.4, 0.9]])
    area = 0.5 * abs(np.linalg.det(np.array([v[1] - v[0], v[2] - v[0]])))
    # degree 1 is the P1 element of assemble_scalar_p1_matrix (forms_simple.f90:1702-1717)
    m1 = oracle.triangle_lagrange_element(v, 1, 2, stiffness=1.3, mass=0.7)
    ref = oracle.p1_dense(v, np.array([[0, 1, 2]], np.int32), mass=0.7, stiffness=1.3)
    _, pw = oracle.triangle_lagrange_nodes(1)
    vert = pw.argmax(axis=1)          # local DoF l sits on the vertex with power 1
    assert np.abs(m1 - ref[np.ix_(vert, vert)]).max() < 1e-13
    for p in range(1, 7):
        k = oracle.triangle_lagrange_element(v, p, 2 * p, stiffness=1.0, mass=0.0)
        m = oracle.triangle_lagrange_element(v, p, 2 * p, stiffness=0.0, mass=1.0)
        assert np.abs(k.sum(axis=1)).max() < 1e-11          # constants are in the kernel
        assert abs(m.sum() - area) < 1e-13                   # the mass of 1 is the area
        assert np.abs(k - k.T).max() < 1e-13 and np.linalg.eigvalsh(m).min() > 0


# assemble_tetra_nedelec_weighted_element(_order) (assembly_tetra_nedelec_3d.f90:2406-2514):
# an isotropic tensor c I is the scalar curl coefficient c of the curl-mass
# element (:584-643, order 1 :2357-2404); any symmetric tensor gives a
# symmetric matrix, and the tensor enters linearly.
@pytest.mark.parametrize("k", [1, 2, 3])
def test_weighted_element_reduces_to_curl_mass(k):
    rng = np.random.default_rng(k)
    v = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
         + 0.1 * rng.standard_normal((4, 3))).reshape(-1)
    a = oracle.nedelec_weighted_element(v, k, 1.7 * np.eye(3), 0.9)
    b = (oracle.whitney_element(v, 1.7, 0.9) if k == 1
         else oracle.nedelec_element(v, k, 2 * k + 2, 1.7, 0.9))
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    m = rng.standard_normal((3, 3))
    m = m + m.T
    w = oracle.nedelec_weighted_element(v, k, m, 0.0)
    assert np.abs(w - w.T).max() <= 1e-13 * np.abs(w).max()
    w2 = oracle.nedelec_weighted_element(v, k, 2.0 * m, 0.0)
    assert np.abs(w2 - 2.0 * w).max() <= 1e-13 * np.abs(w).max()
