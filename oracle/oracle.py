"""ctypes wrapper of the FP64 CPU oracle (test infrastructure only).

The oracle (``oracle/liboracle.so``, built from ``oracle_core.cpp`` and
``oracle_nedelec.cpp`` by ``oracle/Makefile``) restates the reference's
assembly + Krylov path on the CPU.  Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU legs use this module, as the checker or the timed CPU
baseline.  The product package ``fortfem_b200`` never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
    return _lib


def _arr(x, dtype):
    return np.ascontiguousarray(x, dtype=dtype)


def _p(x):
    return x.ctypes.data_as(C.c_void_p) if x is not None else None


def _call(name, *args, restype=C.c_int):
    f = getattr(lib(), name)
    f.restype = restype
    conv = []
    for a in args:
        if isinstance(a, np.ndarray):
            conv.append(_p(a))
        elif isinstance(a, float):
            conv.append(C.c_double(a))
        elif isinstance(a, bool):
            conv.append(C.c_int(int(a)))
        elif isinstance(a, int):
            conv.append(C.c_int64(a) if abs(a) > 2 ** 31 - 1 else C.c_int(a))
        elif a is None:
            conv.append(None)
        else:
            conv.append(a)
    return f(*conv)


class OracleError(RuntimeError):
    pass


def _check(st, what):
    if st != 0:
        raise OracleError(f"oracle {what} failed with status {st}")


# ------------------------------------------------------------------ quadrature

def gauss_legendre(n, a=0.0, b=1.0):
    x = np.zeros(n); w = np.zeros(n)
    _check(_call("or_gauss_legendre", n, float(a), float(b), x, w), "gauss_legendre")
    return x, w


def tetra_duffy(q):
    n = _call("or_tetra_duffy_count", q)
    x, y, z, w = (np.zeros(n) for _ in range(4))
    _check(_call("or_tetra_duffy", q, x, y, z, w), "tetra_duffy")
    return x, y, z, w


def triangle_duffy(q):
    n = _call("or_triangle_duffy_count", q)
    x, y, w = (np.zeros(n) for _ in range(3))
    _check(_call("or_triangle_duffy", q, x, y, w), "triangle_duffy")
    return x, y, w


def degree_two_rule():
    p = np.zeros(12); w = np.zeros(4)
    _call("or_tetra_degree_two_rule", p, w, restype=None)
    return p.reshape(4, 3), w


# ---------------------------------------------------------------------- meshes

def box_mesh(counts, bounds=((0, 0, 0), (1, 1, 1))):
    counts = _arr(counts, np.int32)
    b = _arr([*bounds[0], *bounds[1]], np.float64)
    nv = int(np.prod(counts + 1)); nt = 6 * int(np.prod(counts))
    v = np.zeros(3 * nv); t = np.zeros(4 * nt, np.int32)
    _check(_call("or_structured_tetra_box_mesh", b, counts, v, t), "box_mesh")
    return v.reshape(nv, 3), t.reshape(nt, 4)


def unit_square_mesh(n):
    v = np.zeros(2 * n * n); t = np.zeros(3 * 2 * (n - 1) ** 2, np.int32)
    _check(_call("or_unit_square_mesh", n, v, t), "unit_square_mesh")
    return v.reshape(-1, 2), t.reshape(-1, 3)


def square_boundary(n_vertices, tris):
    tris = _arr(tris, np.int32)
    out = np.zeros(n_vertices, np.uint8)
    _check(_call("or_square_boundary_vertices", n_vertices, len(tris), tris, out), "boundary")
    return out.astype(bool)


# ---------------------------------------------------------- tetra Lagrange

def lagrange_dof_count(p):
    return _call("or_lagrange_dof_count", p)


def lagrange_indices(p):
    nb = lagrange_dof_count(p)
    idx = np.zeros(4 * nb, np.int32); nodes = np.zeros(3 * nb)
    _check(_call("or_lagrange_barycentric_indices", p, idx, nodes), "indices")
    return idx.reshape(nb, 4), nodes.reshape(nb, 3)


def lagrange_evaluate(p, point):
    nb = lagrange_dof_count(p)
    v = np.zeros(nb); g = np.zeros(3 * nb)
    _check(_call("or_lagrange_evaluate", p, _arr(point, np.float64), v, g), "evaluate")
    return v, g.reshape(nb, 3)


def lagrange_dof_map(p, tets, faithful=False):
    tets = _arr(tets, np.int32)
    nb = lagrange_dof_count(p)
    gd = np.zeros(nb * len(tets), np.int32)
    n = C.c_int(0)
    name = "or_lagrange_dof_map_faithful" if faithful else "or_lagrange_dof_map"
    _check(_call(name, p, len(tets), tets, gd, C.byref(n)), "dof_map")
    return gd.reshape(len(tets), nb), n.value


def lagrange_element(vertices, p, rule=0, q=None, stiffness=1.0, mass=0.0):
    if q is None:
        q = 2 * p + 4
    nb = lagrange_dof_count(p)
    m = np.zeros(nb * nb)
    _check(_call("or_lagrange_element", _arr(vertices, np.float64), p, rule, q, float(stiffness),
                 float(mass), m), "lagrange_element")
    return m.reshape(nb, nb, order="F")


def csc_to_scipy(n, cp, ri, v):
    import scipy.sparse as sp
    return sp.csc_matrix((v, ri, cp), shape=(n, n))


def lagrange_csc(vertices, tets, p, rule=0, q=None, stiffness=1.0, mass=0.0, cell_stiffness=None,
                 cell_mass=None):
    if q is None:
        q = 2 * p + 4
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    cs = None if cell_stiffness is None else _arr(cell_stiffness, np.float64)
    cm = None if cell_mass is None else _arr(cell_mass, np.float64)
    nnz = int(_call("or_lagrange_csc_nnz", p, len(tets), tets, restype=C.c_int64))
    if nnz < 0:
        raise OracleError("lagrange_csc_nnz failed")
    nd = C.c_int(0); nz = C.c_int64(0)
    gd, n = lagrange_dof_map(p, tets)
    cp = np.zeros(n + 1, np.int64); ri = np.zeros(nnz, np.int32); v = np.zeros(nnz)
    _check(_call("or_lagrange_csc", len(vertices), vertices, len(tets), tets, p, rule, q,
                 float(stiffness), float(mass), cs, cm, C.c_int64(nnz), C.byref(nd), C.byref(nz),
                 cp, ri, v), "lagrange_csc")
    return n, cp, ri, v


def lagrange_element_jvp(vertices, p, vertices_dot, stiffness, mass, stiffness_dot, mass_dot,
                         rule=0, q=None):
    if q is None:
        q = 2 * p + 4
    nb = lagrange_dof_count(p)
    m = np.zeros(nb * nb)
    _check(_call("or_lagrange_element_jvp", _arr(vertices, np.float64), p, rule, q,
                 float(stiffness), float(mass), _arr(vertices_dot, np.float64),
                 float(stiffness_dot), float(mass_dot), m), "lagrange_element_jvp")
    return m.reshape(nb, nb, order="F")


def lagrange_element_vjp(vertices, p, matrix_bar, stiffness, mass, rule=0, q=None):
    """(vertices_bar (4,3), stiffness_bar, mass_bar) of one element."""
    if q is None:
        q = 2 * p + 4
    vb = np.zeros(12)
    sb = C.c_double(0.0); mb = C.c_double(0.0)
    _check(_call("or_lagrange_element_vjp", _arr(vertices, np.float64), p, rule, q,
                 float(stiffness), float(mass),
                 _arr(np.asarray(matrix_bar).ravel(order="F"), np.float64), vb, C.byref(sb),
                 C.byref(mb)), "lagrange_element_vjp")
    return vb.reshape(4, 3), sb.value, mb.value


def lagrange_csc_jvp(vertices, tets, p, vertices_dot, stiffness, mass, stiffness_dot, mass_dot,
                     rule=0, q=None):
    """(n, col_ptr, row_idx, values_dot) of assemble_tetra_lagrange_stiffness_csc_jvp."""
    if q is None:
        q = 2 * p + 4
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    nnz = int(_call("or_lagrange_csc_nnz", p, len(tets), tets, restype=C.c_int64))
    if nnz < 0:
        raise OracleError("lagrange_csc_nnz failed")
    nd = C.c_int(0); nz = C.c_int64(0)
    _, n = lagrange_dof_map(p, tets)
    cp = np.zeros(n + 1, np.int64); ri = np.zeros(nnz, np.int32); v = np.zeros(nnz)
    _check(_call("or_lagrange_csc_jvp", len(vertices), vertices, len(tets), tets, p, rule, q,
                 float(stiffness), float(mass), _arr(vertices_dot, np.float64),
                 float(stiffness_dot), float(mass_dot), C.c_int64(nnz), C.byref(nd), C.byref(nz),
                 cp, ri, v), "lagrange_csc_jvp")
    return n, cp, ri, v


def lagrange_csc_vjp(vertices, tets, p, values_bar, stiffness, mass, rule=0, q=None):
    """(vertices_bar (n_vertices,3), stiffness_bar, mass_bar) of
    assemble_tetra_lagrange_stiffness_csc_vjp."""
    if q is None:
        q = 2 * p + 4
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    values_bar = _arr(values_bar, np.float64)
    vb = np.zeros(vertices.size)
    sb = C.c_double(0.0); mb = C.c_double(0.0)
    _check(_call("or_lagrange_csc_vjp", len(vertices), vertices, len(tets), tets, p, rule, q,
                 float(stiffness), float(mass), C.c_int64(values_bar.size), values_bar, vb,
                 C.byref(sb), C.byref(mb)), "lagrange_csc_vjp")
    return vb.reshape(-1, 3), sb.value, mb.value


def lagrange_quadrature_points(vertices, tets, rule=0, q=0):
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    nq = 4 if rule == 1 else _call("or_tetra_duffy_count", q)
    out = np.zeros(3 * nq * len(tets))
    _check(_call("or_lagrange_quadrature_points", len(vertices), vertices, len(tets), tets, rule, q,
                 out), "quadrature_points")
    return out.reshape(len(tets), nq, 3)


def lagrange_load_samples(vertices, tets, p, source_values, rule=0, q=0):
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    _, n = lagrange_dof_map(p, tets)
    rhs = np.zeros(n)
    _check(_call("or_lagrange_load_samples", len(vertices), vertices, len(tets), tets, p, rule, q,
                 _arr(source_values, np.float64), rhs), "load_samples")
    return rhs


def lagrange_dirichlet(p, vertices, tets, faithful=False):
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    _, n = lagrange_dof_map(p, tets)
    con = np.zeros(n, np.uint8); pts = np.zeros(3 * n)
    name = "or_lagrange_dirichlet_faithful" if faithful else "or_lagrange_dirichlet"
    _check(_call(name, p, len(vertices), vertices, len(tets), tets, con, pts), "dirichlet")
    return con.astype(bool), pts.reshape(n, 3)


# ------------------------------------------------------------------------ P1

def p1_dense(vertices, tris, mass=0.0, stiffness=1.0):
    vertices = _arr(vertices, np.float64); tris = _arr(tris, np.int32)
    n = len(vertices)
    a = np.zeros(n * n)
    _check(_call("or_p1_dense_matrix", n, vertices, len(tris), tris, float(mass), float(stiffness),
                 a), "p1_dense")
    return a.reshape(n, n, order="F")


def p1_load(vertices, tris, load=1.0):
    vertices = _arr(vertices, np.float64); tris = _arr(tris, np.int32)
    v = np.zeros(len(vertices))
    _check(_call("or_p1_load", len(vertices), vertices, len(tris), tris, float(load), v), "p1_load")
    return v


def p1_csc(vertices, tris, mass=0.0, stiffness=1.0, cell_stiffness=None):
    vertices = _arr(vertices, np.float64); tris = _arr(tris, np.int32)
    n = len(vertices)
    cs = None if cell_stiffness is None else _arr(cell_stiffness, np.float64)
    nz = C.c_int64(0)
    st = _call("or_p1_csc", n, vertices, len(tris), tris, float(mass), float(stiffness), cs,
               C.c_int64(0), C.byref(nz), None, None, None)
    if st not in (0, -2):
        raise OracleError("p1_csc")
    cp = np.zeros(n + 1, np.int64); ri = np.zeros(nz.value, np.int32); v = np.zeros(nz.value)
    _check(_call("or_p1_csc", n, vertices, len(tris), tris, float(mass), float(stiffness), cs,
                 C.c_int64(nz.value), C.byref(nz), cp, ri, v), "p1_csc")
    return n, cp, ri, v


def p1_eliminate_dense(a, rhs, boundary, value=0.0):
    a = np.asfortranarray(a, dtype=np.float64).copy(order="F")
    flat = a.reshape(-1, order="F").copy()
    rhs = _arr(rhs, np.float64).copy()
    _check(_call("or_p1_dirichlet_eliminate_dense", len(rhs), flat, rhs,
                 _arr(boundary, np.uint8), float(value)), "eliminate")
    return flat.reshape(len(rhs), len(rhs), order="F"), rhs


# --------------------------------------------------------------- sparse/solve

def csc_from_triplet(n_rows, n_cols, rows, cols, vals):
    rows = _arr(rows, np.int32); cols = _arr(cols, np.int32); vals = _arr(vals, np.float64)
    nz = C.c_int64(0)
    st = _call("or_csc_from_triplet", n_rows, n_cols, C.c_int64(len(rows)), rows, cols, vals,
               C.c_int64(0), C.byref(nz), None, None, None)
    if st not in (0, -2):
        raise OracleError("csc_from_triplet")
    cp = np.zeros(n_cols + 1, np.int64); ri = np.zeros(nz.value, np.int32); v = np.zeros(nz.value)
    _check(_call("or_csc_from_triplet", n_rows, n_cols, C.c_int64(len(rows)), rows, cols, vals,
                 C.c_int64(nz.value), C.byref(nz), cp, ri, v), "csc_from_triplet")
    return cp, ri, v


def csc_matvec(n, cp, ri, v, x):
    y = np.zeros(n)
    _call("or_csc_matvec", n, _arr(cp, np.int64), _arr(ri, np.int32), _arr(v, np.float64),
          _arr(x, np.float64), y, restype=None)
    return y


def reduce_constrained(n, cp, ri, v, rhs, constrained, values=None):
    cp = _arr(cp, np.int64); ri = _arr(ri, np.int32); v = _arr(v, np.float64)
    rhs = _arr(rhs, np.float64); con = _arr(constrained, np.uint8)
    cv = None if values is None else _arr(values, np.float64)
    nf = C.c_int(0); nz = C.c_int64(0)
    _check(_call("or_reduce_constrained", n, cp, ri, v, rhs, con, cv, C.byref(nf), C.byref(nz),
                 None, None, None, None, None), "reduce(count)")
    rcp = np.zeros(nf.value + 1, np.int64); rri = np.zeros(nz.value, np.int32)
    rv = np.zeros(nz.value); rr = np.zeros(nf.value); free = np.zeros(nf.value, np.int32)
    _check(_call("or_reduce_constrained", n, cp, ri, v, rhs, con, cv, C.byref(nf), C.byref(nz),
                 rcp, rri, rv, rr, free), "reduce")
    return nf.value, rcp, rri, rv, rr, free


def pcg_sparse(n, cp, ri, v, b, x0=None, tol=1e-10, relative=True, max_iterations=100000,
               jacobi=True, guard=0):
    x = np.zeros(n) if x0 is None else _arr(x0, np.float64).copy()
    stats = np.zeros(4)
    _check(_call("or_pcg_sparse", n, _arr(cp, np.int64), _arr(ri, np.int32), _arr(v, np.float64),
                 _arr(b, np.float64), x, float(tol), int(relative), int(max_iterations),
                 int(jacobi), int(guard), stats), "pcg_sparse")
    return x, {"iterations": int(stats[0]), "converged": bool(stats[1]),
               "final_residual": stats[2], "initial_residual": stats[3]}


def pcg_dense(a, b, x0=None, tol=1e-10, relative=True, max_iterations=100000, jacobi=True,
              guard=0):
    n = len(b)
    flat = np.asfortranarray(a, dtype=np.float64).reshape(-1, order="F").copy()
    x = np.zeros(n) if x0 is None else _arr(x0, np.float64).copy()
    stats = np.zeros(4)
    _check(_call("or_pcg_dense", n, flat, _arr(b, np.float64), x, float(tol), int(relative),
                 int(max_iterations), int(jacobi), int(guard), stats), "pcg_dense")
    return x, {"iterations": int(stats[0]), "converged": bool(stats[1]),
               "final_residual": stats[2], "initial_residual": stats[3]}


# --------------------------------------------------------------- Nedelec

def nedelec_dof_count(k):
    return _call("or_nedelec_dof_count", k)


def nedelec_evaluate(k, point):
    nb = nedelec_dof_count(k)
    v = np.zeros(3 * nb); c = np.zeros(3 * nb)
    _check(_call("or_nedelec_evaluate", k, _arr(point, np.float64), v, c), "nedelec_evaluate")
    return v.reshape(nb, 3), c.reshape(nb, 3)


def whitney_evaluate(point):
    v = np.zeros(18); c = np.zeros(18)
    _check(_call("or_whitney_evaluate", _arr(point, np.float64), v, c), "whitney")
    return v.reshape(6, 3), c.reshape(6, 3)


def edge_dof_map(tets, faithful=False):
    tets = _arr(tets, np.int32)
    nt = len(tets)
    edges = np.zeros(12 * nt, np.int32); gd = np.zeros(6 * nt, np.int32)
    orient = np.zeros(6 * nt, np.int32); ne = C.c_int(0)
    name = "or_edge_dof_map_faithful" if faithful else "or_edge_dof_map"
    _check(_call(name, nt, tets, edges, gd, orient, C.byref(ne)), "edge_dof_map")
    return edges[:2 * ne.value].reshape(-1, 2), gd.reshape(nt, 6), orient.reshape(nt, 6)


def nedelec_dof_map(k, tets, faithful=False):
    tets = _arr(tets, np.int32)
    nt = len(tets); nb = nedelec_dof_count(k)
    ne = C.c_int(0); nf = C.c_int(0); ng = C.c_int(0)
    _check(_call("or_nedelec_dof_map", k, nt, tets, int(faithful), None, C.byref(ne), None,
                 C.byref(nf), None, None, None, C.byref(ng)), "nedelec_dof_map(count)")
    edges = np.zeros(2 * ne.value, np.int32); faces = np.zeros(3 * nf.value, np.int32)
    gd = np.zeros(nb * nt, np.int32); eo = np.zeros(6 * nt, np.int32)
    fp = np.zeros(12 * nt, np.int32)
    _check(_call("or_nedelec_dof_map", k, nt, tets, int(faithful), edges, C.byref(ne), faces,
                 C.byref(nf), gd, eo, fp, C.byref(ng)), "nedelec_dof_map")
    return dict(edges=edges.reshape(-1, 2), faces=faces.reshape(-1, 3), global_dofs=gd.reshape(nt, nb),
                edge_orientations=eo.reshape(nt, 6), face_permutations=fp.reshape(nt, 4, 3),
                n_global=ng.value)


def face_basis_to_local(k, perm):
    m = k * (k - 1)
    t = np.zeros(m * m)
    _check(_call("or_face_basis_to_local", k, _arr(perm, np.int32), t), "face_transform")
    return t.reshape(m, m, order="F")


def nedelec_transform(k, edge_orientations, face_permutations):
    nb = nedelec_dof_count(k)
    t = np.zeros(nb * nb)
    _check(_call("or_nedelec_transform", k, _arr(edge_orientations, np.int32),
                 _arr(face_permutations, np.int32), t), "nedelec_transform")
    return t.reshape(nb, nb, order="F")


def nedelec_element(vertices, k, q=None, curl=1.0, mass=1.0):
    if q is None:
        q = 2 * k
    nb = nedelec_dof_count(k)
    m = np.zeros(nb * nb)
    _check(_call("or_nedelec_element", _arr(vertices, np.float64), k, q, float(curl), float(mass),
                 m), "nedelec_element")
    return m.reshape(nb, nb, order="F")


def whitney_element(vertices, curl=1.0, mass=1.0):
    m = np.zeros(36)
    _check(_call("or_nedelec_whitney_element", _arr(vertices, np.float64), float(curl),
                 float(mass), m), "whitney_element")
    return m.reshape(6, 6, order="F")


def nedelec_csc(vertices, tets, k, curl=1.0, mass=1.0, cell_curl=None, cell_mass=None):
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    cc = None if cell_curl is None else _arr(cell_curl, np.float64)
    cm = None if cell_mass is None else _arr(cell_mass, np.float64)
    nnz = int(_call("or_nedelec_csc_nnz", k, len(tets), tets, restype=C.c_int64))
    if nnz < 0:
        raise OracleError("nedelec_csc_nnz")
    n = nedelec_dof_map(k, tets)["n_global"]
    nd = C.c_int(0); nz = C.c_int64(0)
    cp = np.zeros(n + 1, np.int64); ri = np.zeros(nnz, np.int32); v = np.zeros(nnz)
    _check(_call("or_nedelec_csc", len(vertices), vertices, len(tets), tets, k, float(curl),
                 float(mass), cc, cm, C.c_int64(nnz), C.byref(nd), C.byref(nz), cp, ri, v),
           "nedelec_csc")
    return n, cp, ri, v


def nedelec_weighted_element(vertices, k, tensor, mass=1.0):
    """assemble_tetra_nedelec_weighted_element(_order) with a constant 3 x 3 tensor."""
    n = nedelec_dof_count(k)
    out = np.zeros(n * n)
    t = np.asfortranarray(np.asarray(tensor, np.float64).reshape(3, 3)).reshape(-1, order="F")
    _check(_call("or_nedelec_weighted_element", _arr(vertices, np.float64), k, _arr(t, np.float64),
                 float(mass), out), "nedelec_weighted_element")
    return out.reshape(n, n, order="F")


def nedelec_weighted_csc(vertices, tets, k, cell_tensors, mass=1.0):
    """assemble_tetra_nedelec_weighted_csc with one column-major 3 x 3 tensor per cell
    (cell_tensors of shape (n_cells, 3, 3), entry [c, r, s] = M_c(r, s))."""
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    ten = np.ascontiguousarray(np.transpose(np.asarray(cell_tensors, np.float64), (0, 2, 1)))
    nnz = int(_call("or_nedelec_csc_nnz", k, len(tets), tets, restype=C.c_int64))
    if nnz < 0:
        raise OracleError("nedelec_csc_nnz")
    n = nedelec_dof_map(k, tets)["n_global"]
    nd = C.c_int(0); nz = C.c_int64(0)
    cp = np.zeros(n + 1, np.int64); ri = np.zeros(nnz, np.int32); v = np.zeros(nnz)
    _check(_call("or_nedelec_weighted_csc", len(vertices), vertices, len(tets), tets, k,
                 ten.reshape(-1), float(mass), C.c_int64(nnz), C.byref(nd), C.byref(nz), cp, ri,
                 v), "nedelec_weighted_csc")
    return n, cp, ri, v


def nedelec_element_jvp(vertices, k, vertices_dot, curl, mass, curl_dot, mass_dot, q=None):
    if q is None:
        q = 2 * k + 2
    nb = nedelec_dof_count(k)
    m = np.zeros(nb * nb)
    _check(_call("or_nedelec_element_jvp", _arr(vertices, np.float64), k, q, float(curl),
                 float(mass), _arr(vertices_dot, np.float64), float(curl_dot), float(mass_dot), m),
           "nedelec_element_jvp")
    return m.reshape(nb, nb, order="F")


def nedelec_element_vjp(vertices, k, matrix_bar, curl, mass, q=None):
    """(vertices_bar (4,3), curl_bar, mass_bar) of one element."""
    if q is None:
        q = 2 * k + 2
    vb = np.zeros(12)
    cb = C.c_double(0.0); mb = C.c_double(0.0)
    _check(_call("or_nedelec_element_vjp", _arr(vertices, np.float64), k, q, float(curl),
                 float(mass), _arr(np.asarray(matrix_bar).ravel(order="F"), np.float64), vb,
                 C.byref(cb), C.byref(mb)), "nedelec_element_vjp")
    return vb.reshape(4, 3), cb.value, mb.value


def nedelec_csc_jvp(vertices, tets, k, vertices_dot, curl, mass, curl_dot, mass_dot):
    """(n, col_ptr, row_idx, values_dot) of assemble_tetra_nedelec_curl_mass_csc_jvp."""
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    nnz = int(_call("or_nedelec_csc_nnz", k, len(tets), tets, restype=C.c_int64))
    if nnz < 0:
        raise OracleError("nedelec_csc_nnz")
    n = nedelec_dof_map(k, tets)["n_global"]
    nd = C.c_int(0); nz = C.c_int64(0)
    cp = np.zeros(n + 1, np.int64); ri = np.zeros(nnz, np.int32); v = np.zeros(nnz)
    _check(_call("or_nedelec_csc_jvp", len(vertices), vertices, len(tets), tets, k, float(curl),
                 float(mass), _arr(vertices_dot, np.float64), float(curl_dot), float(mass_dot),
                 C.c_int64(nnz), C.byref(nd), C.byref(nz), cp, ri, v), "nedelec_csc_jvp")
    return n, cp, ri, v


def nedelec_csc_vjp(vertices, tets, k, values_bar, curl, mass):
    """(vertices_bar (n_vertices,3), curl_bar, mass_bar) of
    assemble_tetra_nedelec_curl_mass_csc_vjp."""
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    values_bar = _arr(values_bar, np.float64)
    vb = np.zeros(vertices.size)
    cb = C.c_double(0.0); mb = C.c_double(0.0)
    _check(_call("or_nedelec_csc_vjp", len(vertices), vertices, len(tets), tets, k, float(curl),
                 float(mass), C.c_int64(values_bar.size), values_bar, vb, C.byref(cb),
                 C.byref(mb)), "nedelec_csc_vjp")
    return vb.reshape(-1, 3), cb.value, mb.value


def nedelec_load_points(vertices, tets, k):
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    nq = 4 if k == 1 else _call("or_tetra_duffy_count", 2 * k + 2)
    out = np.zeros(3 * nq * len(tets))
    _check(_call("or_nedelec_load_points", len(vertices), vertices, len(tets), tets, k, out),
           "nedelec_load_points")
    return out.reshape(len(tets), nq, 3)


def nedelec_load_samples(vertices, tets, k, source_values):
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    n = nedelec_dof_map(k, tets)["n_global"]
    rhs = np.zeros(n)
    _check(_call("or_nedelec_load_samples", len(vertices), vertices, len(tets), tets, k,
                 _arr(source_values, np.float64), rhs), "nedelec_load_samples")
    return rhs


def pec_mask(k, tets, faithful=False):
    tets = _arr(tets, np.int32)
    n = nedelec_dof_map(k, tets)["n_global"]
    con = np.zeros(n, np.uint8)
    _check(_call("or_pec_mask", k, len(tets), tets, int(faithful), con), "pec_mask")
    return con.astype(bool)


# ------------------------------------------------------------ solution probes

def lagrange_evaluate_solution(vertices, tets, p, solution, cell, point, physical=False):
    """(value, gradient) of evaluate_tetra_lagrange_solution (reference point)
    or evaluate_tetra_lagrange_solution_at_point (physical point); None when
    the reference rejects the query."""
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    u = _arr(solution, np.float64)
    val = C.c_double(0.0); g = np.zeros(3)
    name = "or_lagrange_evaluate_solution_at_point" if physical else "or_lagrange_evaluate_solution"
    st = _call(name, len(vertices), vertices, len(tets), tets, p, len(u), u, int(cell),
               _arr(point, np.float64), C.byref(val), g)
    return None if st else (val.value, g)


def lagrange_probe(vertices, tets, p, solution, point, mode=0):
    """(value, gradient, count) of the all-cell point probe."""
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    u = _arr(solution, np.float64)
    val = C.c_double(0.0); g = np.zeros(3); cnt = C.c_int(0)
    _call("or_lagrange_probe", len(vertices), vertices, len(tets), tets, p, len(u), u,
          _arr(point, np.float64), int(mode), C.byref(val), g, C.byref(cnt))
    return val.value, g, cnt.value


def nedelec_evaluate_solution(vertices, tets, k, solution, cell, point):
    """(value, curl) at a reference point of one cell; None when rejected."""
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    u = _arr(solution, np.float64)
    v = np.zeros(3); c = np.zeros(3)
    st = _call("or_nedelec_evaluate_solution", len(vertices), vertices, len(tets), tets, k, len(u),
               u, int(cell), _arr(point, np.float64), v, c)
    return None if st else (v, c)


def nedelec_probe(vertices, tets, k, solution, point, mode=0):
    """(value, curl, count) of evaluate_box_solution_order (mode 0) or the
    first-containing-cell probes (mode 1)."""
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    u = _arr(solution, np.float64)
    v = np.zeros(3); c = np.zeros(3); cnt = C.c_int(0)
    _call("or_nedelec_probe", len(vertices), vertices, len(tets), tets, k, len(u), u,
          _arr(point, np.float64), int(mode), v, c, C.byref(cnt))
    return v, c, cnt.value


# ------------------------------------------------------------------ complex PML

def _cplx_in(stretch):
    a = np.ascontiguousarray(stretch, dtype=np.complex128)
    return np.ascontiguousarray(a.view(np.float64).ravel())


def nedelec_pml_element(vertices, k, stretch, wave_number, q=None, curvilinear=False):
    """Complex element matrix of assemble_tetra_nedelec_pml_element (stretch (3,))
    or the curvilinear variant (stretch (3, 3))."""
    if q is None:
        q = 2 * k + 2
    nb = nedelec_dof_count(k)
    m = np.zeros(2 * nb * nb)
    s = np.asarray(stretch, np.complex128)
    if curvilinear:
        s = s.ravel(order="F")
    name = "or_nedelec_curvilinear_pml_element" if curvilinear else "or_nedelec_pml_element"
    _check(_call(name, _arr(vertices, np.float64), k, q, _cplx_in(s), float(wave_number), m), name)
    return m.view(np.complex128).reshape(nb, nb, order="F")


def nedelec_pml_csc(vertices, tets, k, stretch, wave_number, curvilinear=False):
    """(n, col_ptr, row_idx, complex values): stretch (T, 3) or (T, 3, 3)."""
    vertices = _arr(vertices, np.float64); tets = _arr(tets, np.int32)
    s = np.asarray(stretch, np.complex128)
    if curvilinear:
        s = np.transpose(s, (0, 2, 1))  # column-major per cell
    nnz = int(_call("or_nedelec_csc_nnz", k, len(tets), tets, restype=C.c_int64))
    n = nedelec_dof_map(k, tets)["n_global"]
    nd = C.c_int(0); nz = C.c_int64(0)
    cp = np.zeros(n + 1, np.int64); ri = np.zeros(nnz, np.int32); v = np.zeros(2 * nnz)
    name = "or_nedelec_curvilinear_pml_csc" if curvilinear else "or_nedelec_pml_csc"
    _check(_call(name, len(vertices), vertices, len(tets), tets, k, _cplx_in(s),
                 float(wave_number), C.c_int64(nnz), C.byref(nd), C.byref(nz), cp, ri, v), name)
    return n, cp, ri, v.view(np.complex128)


# ------------------------------------------------- arbitrary-order triangle Lagrange

def triangle_lagrange_dof_count(p):
    return (p + 1) * (p + 2) // 2


def triangle_lagrange_nodes(p):
    nb = triangle_lagrange_dof_count(p)
    nodes = np.zeros(2 * nb); pw = np.zeros(3 * nb, np.int32)
    _check(_call("or_triangle_lagrange_nodes", p, nodes, pw), "triangle_lagrange_nodes")
    return nodes.reshape(nb, 2), pw.reshape(nb, 3)


def triangle_lagrange_evaluate(p, x, y):
    """(values (n_b,), gradients (n_b, 2)); None when the point is rejected."""
    nb = triangle_lagrange_dof_count(p)
    v = np.zeros(nb); g = np.zeros(2 * nb)
    st = _call("or_triangle_lagrange_evaluate", p, float(x), float(y), v, g)
    return None if st else (v, g.reshape(nb, 2))


def triangle_lagrange_dof_map(p, tris):
    tris = _arr(tris, np.int32)
    nb = triangle_lagrange_dof_count(p)
    gd = np.zeros(nb * len(tris), np.int32)
    n = C.c_int(0)
    _check(_call("or_triangle_lagrange_dof_map", p, len(tris), tris, gd, C.byref(n)), "dof_map")
    return gd.reshape(len(tris), nb), n.value


def triangle_lagrange_element(vertices, p, q, stiffness=1.0, mass=0.0):
    nb = triangle_lagrange_dof_count(p)
    m = np.zeros(nb * nb)
    _check(_call("or_triangle_lagrange_element", _arr(vertices, np.float64), p, q,
                 float(stiffness), float(mass), m), "triangle_lagrange_element")
    return m.reshape(nb, nb, order="F")


def triangle_lagrange_csc(vertices, tris, p, q, stiffness=1.0, mass=0.0, cell_stiffness=None,
                          cell_mass=None):
    vertices = _arr(vertices, np.float64); tris = _arr(tris, np.int32)
    cs = None if cell_stiffness is None else _arr(cell_stiffness, np.float64)
    cm = None if cell_mass is None else _arr(cell_mass, np.float64)
    nnz = int(_call("or_triangle_lagrange_csc_nnz", p, len(tris), tris, restype=C.c_int64))
    _, n = triangle_lagrange_dof_map(p, tris)
    nd = C.c_int(0); nz = C.c_int64(0)
    cp = np.zeros(n + 1, np.int64); ri = np.zeros(nnz, np.int32); v = np.zeros(nnz)
    _check(_call("or_triangle_lagrange_csc", len(vertices), vertices, len(tris), tris, p, q,
                 float(stiffness), float(mass), cs, cm, C.c_int64(nnz), C.byref(nd), C.byref(nz),
                 cp, ri, v), "triangle_lagrange_csc")
    return n, cp, ri, v


def triangle_lagrange_points(vertices, tris, p, q):
    """(sample points (T, n_q, 2), DoF points (n_dofs, 2))."""
    vertices = _arr(vertices, np.float64); tris = _arr(tris, np.int32)
    nq = _call("or_triangle_duffy_count", q)
    _, n = triangle_lagrange_dof_map(p, tris)
    sp = np.zeros(2 * nq * len(tris)); dp = np.zeros(2 * n)
    _check(_call("or_triangle_lagrange_points", len(vertices), vertices, len(tris), tris, p, q,
                 sp, dp), "triangle_lagrange_points")
    return sp.reshape(len(tris), nq, 2), dp.reshape(n, 2)


def triangle_lagrange_load_samples(vertices, tris, p, q, samples):
    vertices = _arr(vertices, np.float64); tris = _arr(tris, np.int32)
    _, n = triangle_lagrange_dof_map(p, tris)
    rhs = np.zeros(n)
    _check(_call("or_triangle_lagrange_load_samples", len(vertices), vertices, len(tris), tris, p,
                 q, _arr(samples, np.float64), rhs), "triangle_lagrange_load_samples")
    return rhs


def triangle_lagrange_boundary(p, tris):
    tris = _arr(tris, np.int32)
    _, n = triangle_lagrange_dof_map(p, tris)
    out = np.zeros(n, np.uint8)
    _check(_call("or_triangle_lagrange_boundary", p, len(tris), tris, out), "boundary")
    return out.astype(bool)
