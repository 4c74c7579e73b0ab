"""Problems built on the device (Lagrange and P1 topologies) against the host
build of the same topology (ffg_build_topology): DoF numbering, Dirichlet set,
free DoFs and the constrained CSC pattern must be equal entry for entry."""
import numpy as np
import pytest

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K
from fortfem_b200 import synth

pytestmark = pytest.mark.gpu

CASES = [
    ("p1", 1, "all"), ("p1", 1, "none"), ("p1", 1, "mask"),
    ("tet", 1, "all"), ("tet", 2, "all"), ("tet", 2, "mask"), ("tet", 3, "all"), ("tet", 4, "none"),
]


def _mesh(kind, p):
    if kind == "p1":
        v, t = oracle.unit_square_mesh(17)
        return synth.jitter_interior_2d(v, 1 / 16, 0.1, 4), t
    n = {1: 5, 2: 4, 3: 2, 4: 2}[p]
    v, t = oracle.box_mesh([n, n + 1, n])
    return synth.jitter_interior(v, 1.0 / n, 0.1, 7), t


@pytest.mark.parametrize("kind,p,boundary", CASES)
def test_device_topology_equals_host_build(kind, p, boundary):
    v, t = _mesh(kind, p)
    fam = K.FFG_TRIANGLE_P1 if kind == "p1" else K.FFG_TETRA_LAGRANGE
    bnd = boundary
    if boundary == "mask":
        n_dofs = ff.build_topology(fam, p, t, len(v), boundary="none")["n_dofs"]
        bnd = (np.random.default_rng(p).random(n_dofs) < 0.2).astype(np.uint8)
    host = ff.build_topology(fam, p, t, len(v), boundary=bnd)
    with ff.Problem(fam, p, t, len(v), boundary=bnd) as prob:
        assert prob.n_dofs == host["n_dofs"] and prob.n_free == host["n_free"]
        assert np.array_equal(prob.constrained(), host["constrained"])
        A, rhs, free = prob.reduced_system(v, 1.0, 0.5)
        assert np.array_equal(A.col_ptr, host["col_ptr"]) and np.array_equal(A.row_idx, host["row_idx"])
        assert np.array_equal(free, np.flatnonzero(~host["constrained"]))
        # the numbering: every local DoF's node lands on its global DoF's point
        pts = prob.dof_points(v)
        gd = host["global_dofs"]
        if kind == "p1":
            nodes = np.concatenate([v, np.zeros((len(v), 1))], 1)[t]
        else:
            idx, _ = oracle.lagrange_indices(p)
            nodes = np.einsum("li,cid->cld", idx / p, v[t])
        assert np.allclose(pts[gd], nodes, atol=1e-14)


def test_device_topology_full_size_p2_counts():
    case = synth.p2_poisson_case()
    host = ff.build_topology(K.FFG_TETRA_LAGRANGE, 2, case.cells, len(case.vertices), boundary="all")
    with ff.Problem(K.FFG_TETRA_LAGRANGE, 2, case.cells, len(case.vertices),
                    rule=case.rule) as prob:
        assert prob.n_dofs == 912673 and prob.n_free == 857375 and prob.nnz == 23881263
        A, _, _ = prob.reduced_system(case.vertices, 1.0, 0.0, case.cell_coefficient)
        assert np.array_equal(A.col_ptr, host["col_ptr"]) and np.array_equal(A.row_idx, host["row_idx"])


_PERMS = np.array([[1, 2, 3], [1, 3, 2], [2, 1, 3], [2, 3, 1], [3, 1, 2], [3, 2, 1]])


def _check_nedelec_maps(prob, k, t):
    """The device build's DoF map, edge orientations and face permutations
    against the oracle's restatement of build_tetra_nedelec_dof_map."""
    topo = prob.topology()
    ref = oracle.nedelec_dof_map(k, t)
    assert prob.n_dofs == ref["n_global"]
    assert np.array_equal(topo["global_dofs"], ref["global_dofs"])
    assert np.array_equal(topo["edge_sign"].astype(np.int32), ref["edge_orientations"])
    assert np.array_equal(_PERMS[topo["face_perm"]], ref["face_permutations"])


NED_CASES = [(1, "all"), (2, "all"), (2, "none"), (3, "all"), (3, "mask"), (4, "all"), (6, "all")]


@pytest.mark.parametrize("k,boundary", NED_CASES)
def test_device_nedelec_topology_equals_host_build(k, boundary):
    n = {1: 4, 2: 3, 3: 2, 4: 2, 6: 1}[k]
    v, t = oracle.box_mesh([n, n + 1, n])
    bnd = boundary
    if boundary == "mask":
        n_dofs = ff.build_topology(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary="none")["n_dofs"]
        bnd = (np.random.default_rng(k).random(n_dofs) < 0.2).astype(np.uint8)
    host = ff.build_topology(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary=bnd)
    with ff.Problem(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary=bnd) as prob:
        assert prob.n_dofs == host["n_dofs"] and prob.n_free == host["n_free"]
        assert np.array_equal(prob.constrained(), host["constrained"])
        assert np.array_equal(prob.topology()["global_dofs"], host["global_dofs"])
        A, rhs, free = prob.reduced_system(v, 1.0, 0.5)
        assert np.array_equal(A.col_ptr, host["col_ptr"]) and np.array_equal(A.row_idx, host["row_idx"])
        assert np.array_equal(free, np.flatnonzero(~host["constrained"]))
        _check_nedelec_maps(prob, k, t)
        if boundary == "all":
            assert np.array_equal(prob.constrained(), oracle.pec_mask(k, t))


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_device_nedelec_topology_slab_24cube(k):
    """The 24^3 x 6 slab mesh: numbering, orientations, permutations and the
    PEC mask against the oracle entry for entry; the constrained pattern
    against the host build for orders 1-2 (the host build of orders 3-4 sorts
    10^8+ couplings on the CPU)."""
    import time
    case = synth.nedelec_slab_case(k, mesh=lambda m: oracle.box_mesh([m, m, m]))
    t0 = time.perf_counter()
    prob = ff.Problem(K.FFG_TETRA_NEDELEC, k, case.cells, len(case.vertices), boundary="all")
    setup = time.perf_counter() - t0
    try:
        print(f"order {k}: device topology setup {setup:.3f} s, {prob.n_dofs} DoFs, nnz {prob.nnz}")
        assert prob.n_dofs == {1: 102024, 2: 542736, 3: 1570968, 4: 3435552}[k]
        _check_nedelec_maps(prob, k, case.cells)
        assert np.array_equal(prob.constrained(), oracle.pec_mask(k, case.cells))
        if k <= 2:
            host = ff.build_topology(K.FFG_TETRA_NEDELEC, k, case.cells, len(case.vertices),
                                     boundary="all")
            A, _, _ = prob.reduced_system(case.vertices, 1.0, 1.0, case.cell_curl)
            assert np.array_equal(A.col_ptr, host["col_ptr"])
            assert np.array_equal(A.row_idx, host["row_idx"])
    finally:
        prob.close()
