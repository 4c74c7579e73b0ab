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
