"""CPU checks of libfortfem_gpu.so: it loads, exports every symbol the header
declares, and its host-side integer topology (DoF numbering, constrained sets,
CSC patterns) is bit-identical to the oracle's restatement of the reference.
No compute kernel is launched here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
import fortfem_b200 as ff
from fortfem_b200 import _capi as K

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "fortfem_gpu.h")).read()
    return sorted(set(re.findall(r"\bvoid\s+(ffg_\w+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = K.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(K.exported_symbols()) == syms


def test_python_constants_match_header():
    text = open(os.path.join(ROOT, "include", "fortfem_gpu.h")).read()
    defines = re.findall(r"#define\s+(FFG_[A-Z0-9_]+)\s+(-?\d+)", text)
    assert len(defines) > 20
    for name, value in defines:
        assert getattr(K, name) == int(value), name


def test_no_device_is_reported_not_faked():
    count = C.c_int(-1)
    st = C.c_int(0)
    K.load().ffg_device_count(C.byref(count), C.byref(st))
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        assert count.value == 0 and st.value == K.FFG_NO_DEVICE
        v, t = oracle.box_mesh([1, 1, 1])
        with pytest.raises(ff.FortfemError) as e:
            ff.Problem(K.FFG_TETRA_LAGRANGE, 1, t, len(v))
        assert e.value.code == K.FFG_NO_DEVICE


def test_box_mesh_matches_oracle():
    for counts in ([1, 1, 1], [2, 3, 1], [5, 4, 3]):
        bounds = [[-1.0, 2.0], [0.5, 1.5], [0.0, 3.0]]
        v, t, st = ff.generate_structured_tetra_box_mesh(bounds, counts)
        assert st.code == 0
        ov, ot = oracle.box_mesh(counts, ((-1.0, 0.5, 0.0), (2.0, 1.5, 3.0)))
        assert np.array_equal(t, ot)
        assert np.array_equal(v, ov)


def test_box_mesh_rejects_bad_input():
    _, _, st = ff.generate_structured_tetra_box_mesh([[0, 1], [0, 1], [0, 1]], [0, 1, 1])
    assert st.code == K.FFG_INVALID_INPUT


def test_unit_square_mesh_matches_oracle():
    v, t = ff.unit_square_mesh(9)
    ov, ot = oracle.unit_square_mesh(9)
    assert np.array_equal(v, ov) and np.array_equal(t, ot)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_lagrange_topology_bit_exact(p):
    v, t = oracle.box_mesh([3, 2, 2])
    topo = ff.build_topology(K.FFG_TETRA_LAGRANGE, p, t, len(v), boundary="none")
    gd, n = oracle.lagrange_dof_map(p, t)
    assert topo["n_dofs"] == n and np.array_equal(topo["global_dofs"], gd)
    # pattern of the unconstrained matrix equals the oracle's triplet->CSC pattern
    nn, cp, ri, _ = oracle.lagrange_csc(v, t, p, 0, 2 * p)
    assert np.array_equal(topo["col_ptr"], cp) and np.array_equal(topo["row_idx"], ri)
    # constrained set equals build_dirichlet_data's
    topo_b = ff.build_topology(K.FFG_TETRA_LAGRANGE, p, t, len(v), boundary="all")
    con, _ = oracle.lagrange_dirichlet(p, v, t, faithful=True)
    assert np.array_equal(topo_b["constrained"], con)
    # reduced pattern equals sparse_direct_solve_constrained's reduction
    nf, rcp, rri, _, _, _ = oracle.reduce_constrained(nn, cp, ri, np.ones(len(ri)), np.zeros(nn), con)
    assert topo_b["n_free"] == nf
    assert np.array_equal(topo_b["col_ptr"], rcp) and np.array_equal(topo_b["row_idx"], rri)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_nedelec_topology_bit_exact(k):
    v, t = oracle.box_mesh([2, 2, 1])
    topo = ff.build_topology(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary="none")
    dm = oracle.nedelec_dof_map(k, t, faithful=True)
    assert topo["n_dofs"] == dm["n_global"]
    assert np.array_equal(topo["global_dofs"], dm["global_dofs"])
    n, cp, ri, _ = oracle.nedelec_csc(v, t, k)
    assert np.array_equal(topo["col_ptr"], cp) and np.array_equal(topo["row_idx"], ri)
    topo_b = ff.build_topology(K.FFG_TETRA_NEDELEC, k, t, len(v), boundary="all")
    assert np.array_equal(topo_b["constrained"], oracle.pec_mask(k, t, faithful=True))


def test_p1_topology_and_boundary():
    v, t = oracle.unit_square_mesh(65)
    topo = ff.build_topology(K.FFG_TRIANGLE_P1, 1, t, len(v), boundary="all")
    assert topo["constrained"].sum() == 256 and topo["n_free"] == 3969
    assert np.array_equal(topo["constrained"], oracle.square_boundary(len(v), t))
    full = ff.build_topology(K.FFG_TRIANGLE_P1, 1, t, len(v), boundary="none")
    n, cp, ri, _ = oracle.p1_csc(v, t)
    assert np.array_equal(full["col_ptr"], cp) and np.array_equal(full["row_idx"], ri)
    assert cp[-1] == 29057 and topo["col_ptr"][-1] == 27281


def test_p2_full_size_counts():
    """Config facts of the 48^3 P2 workload: N = 912,673, nnz = 25,755,265."""
    v, t, _ = ff.generate_structured_tetra_box_mesh([[0, 1], [0, 1], [0, 1]], [48, 48, 48])
    topo = ff.build_topology(K.FFG_TETRA_LAGRANGE, 2, t, len(v), boundary="all")
    assert topo["n_dofs"] == 912673
    assert topo["n_free"] == 95 ** 3
    full = ff.build_topology(K.FFG_TETRA_LAGRANGE, 2, t, len(v), boundary="none")
    assert full["col_ptr"][-1] == 25755265


def test_topology_rejects_bad_cells():
    with pytest.raises(ff.FortfemError):
        ff.build_topology(K.FFG_TETRA_LAGRANGE, 2, np.array([[0, 0, 1, 2]]), 3)
    with pytest.raises(ff.FortfemError):
        ff.build_topology(K.FFG_TETRA_LAGRANGE, 5, np.array([[0, 1, 2, 3]]), 4)
    with pytest.raises(ff.FortfemError):
        ff.build_topology(K.FFG_TETRA_NEDELEC, 1, np.array([[0, 1, 2, 9]]), 4)


@pytest.mark.parametrize("p", [1, 2, 3, 6])
def test_triangle_lagrange_topology_bit_exact(p):
    v, t = oracle.unit_square_mesh(6)
    topo = ff.build_topology(K.FFG_TRIANGLE_LAGRANGE, p, t, len(v), "all")
    gd, n = oracle.triangle_lagrange_dof_map(p, t)
    assert topo["n_dofs"] == n and np.array_equal(topo["global_dofs"], gd)
    assert np.array_equal(topo["constrained"], oracle.triangle_lagrange_boundary(p, t))
    # the constrained pattern is the oracle's CSC restricted to free DoFs
    nn, cp, ri, _ = oracle.triangle_lagrange_csc(v, t, p, 2 * p)
    A = oracle.csc_to_scipy(nn, cp, ri, np.ones(len(ri))).tocsc()
    free = np.flatnonzero(~topo["constrained"])
    R = A[free][:, free].tocsc()
    R.sort_indices()
    assert np.array_equal(topo["col_ptr"], R.indptr) and np.array_equal(topo["row_idx"], R.indices)
