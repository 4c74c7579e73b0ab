"""Host-side mirror of fortfem's assembly and solver entry points.

Function names, argument meaning and status behaviour follow the reference
Fortran interfaces (each docstring names the routine it replaces); arrays are
zero-based numpy arrays, and every call goes through the C-ABI of
``libfortfem_gpu.so`` (include/fortfem_gpu.h) to the sm_100a kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, Optional, Union

import numpy as np

from . import _capi as K

ArrayLike = Union[np.ndarray, list, tuple]


class FortfemError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where}: {K.STATUS_TEXT.get(code, 'error')} (status {code})")
        self.code = code


@dataclass
class Status:
    """fortsparse_status_t: code 0 is success."""
    code: int = 0
    message: str = ""

    @classmethod
    def of(cls, code: int, where: str) -> "Status":
        return cls(code, "" if code == 0 else f"{where}: {K.STATUS_TEXT.get(code, 'error')}")


@dataclass
class CscMatrix:
    """csc_t (fortsparse): zero-based column pointers and row indices."""
    nrow: int
    ncol: int
    col_ptr: np.ndarray
    row_idx: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.col_ptr[-1])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csc_matrix((self.val, self.row_idx, self.col_ptr), shape=(self.nrow, self.ncol))


@dataclass
class SolverOptions:
    """solver_options_t (src/solvers/advanced_solvers.f90:32-44) with the
    reference defaults, plus the GPU precision controls."""
    method: str = "auto"
    tolerance: float = 1.0e-6
    max_iterations: int = 1000
    preconditioner: str = "none"
    tolerance_type: str = "relative"
    verbosity: int = 0
    precision: str = "fp64"          # "fp64" (reference semantics), "mixed" or "mixed16"
    inner_tolerance: float = 0.1      # mixed: reliable-update threshold
    max_refinements: int = 1000       # mixed: cap on reliable updates
    timeout_seconds: float = 60.0
    breakdown_guard: str = "absolute"  # "absolute" (reference) or "spd"

    def to_c(self) -> K.SolverOptionsC:
        if self.method not in ("auto", "pcg", "cg"):
            raise FortfemError(K.FFG_INVALID_INPUT, f"method {self.method!r} is not on this path")
        o = K.SolverOptionsC()
        o.version = K.FFG_OPTIONS_VERSION
        o.preconditioner = 1 if (self.preconditioner == "jacobi" and self.method != "cg") else 0
        modes = {"fp64": K.FFG_PRECISION_FP64, "mixed": K.FFG_PRECISION_MIXED,
                 "mixed16": K.FFG_PRECISION_MIXED16}
        if self.precision not in modes:
            raise FortfemError(K.FFG_INVALID_INPUT, f"precision {self.precision!r}")
        o.precision = modes[self.precision]
        o.tolerance_type = 1 if self.tolerance_type == "absolute" else 0
        o.tolerance = float(self.tolerance)
        o.max_iterations = int(self.max_iterations)
        o.max_refinements = int(self.max_refinements)
        o.inner_tolerance = float(self.inner_tolerance)
        o.verbosity = int(self.verbosity)
        o.timeout_seconds = float(self.timeout_seconds)
        o.breakdown_guard = 1 if self.breakdown_guard == "spd" else 0
        return o


def solver_options(**kw) -> SolverOptions:
    """solver_options(...) constructor (advanced_solvers.f90:1430-1465)."""
    return SolverOptions(**kw)


@dataclass
class SolverStats:
    """solver_stats_t (advanced_solvers.f90:47-57) plus GPU fields."""
    converged: bool = False
    iterations: int = 0
    final_residual: float = 0.0
    solve_time: float = 0.0
    method_used: str = "pcg"
    refinements: int = 0
    true_relative_residual: float = 0.0
    assembly_time: float = 0.0
    status: int = 0

    @classmethod
    def from_c(cls, s: K.SolverStatsC) -> "SolverStats":
        return cls(bool(s.converged), s.iterations, s.final_residual, s.solve_seconds, "pcg",
                   s.refinements, s.true_relative_residual, s.assembly_seconds, s.status)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _opt(a, n, dtype=np.float64):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.size != n:
        raise FortfemError(K.FFG_INVALID_INPUT, "array length")
    return a


# ------------------------------------------------------------------ meshes

def generate_structured_tetra_box_mesh(bounds, counts):
    """generate_structured_tetra_box_mesh (src/mesh/structured_tetra_box_mesh.f90:12-70).
    bounds: (3, 2) [[xmin, xmax], [ymin, ymax], [zmin, zmax]]; returns
    (vertices (n, 3), tetrahedra (T, 4) zero-based, Status)."""
    b = np.asarray(bounds, dtype=np.float64)
    flat = _f64([b[0, 0], b[1, 0], b[2, 0], b[0, 1], b[1, 1], b[2, 1]])
    counts = _i32(counts)
    nv = int(np.prod(counts.astype(np.int64) + 1))
    nt = 6 * int(np.prod(counts.astype(np.int64)))
    v = np.zeros((max(nv, 0), 3))
    t = np.zeros((max(nt, 0), 4), np.int32)
    st = C.c_int(0)
    K.load().ffg_structured_tetra_box_mesh(_ptr(flat), _ptr(counts), _ptr(v), _ptr(t), C.byref(st))
    return v, t, Status.of(st.value, "generate_structured_tetra_box_mesh")


def unit_square_mesh(n: int):
    """unit_square_mesh(n) (src/fortfem_api_mesh.f90:128-139): n vertices per side."""
    v = np.zeros((n * n, 2))
    t = np.zeros((2 * (n - 1) ** 2, 3), np.int32)
    st = C.c_int(0)
    K.load().ffg_unit_square_mesh(n, _ptr(v), _ptr(t), C.byref(st))
    if st.value:
        raise FortfemError(st.value, "unit_square_mesh")
    return v, t


# -------------------------------------------------------- drop-in assembly

def _csc_call(fn, args, where, capacity_hint=None):
    lib = K.load()
    nd = C.c_int(0)
    nz = C.c_int64(0)
    st = C.c_int(0)
    getattr(lib, fn)(*args, C.c_int64(0), C.byref(nd), C.byref(nz), None, None, None, C.byref(st))
    if st.value not in (K.FFG_OK, K.FFG_CAPACITY):
        return None, Status.of(st.value, where)
    n = nd.value
    cp = np.zeros(n + 1, np.int64)
    ri = np.zeros(nz.value, np.int32)
    val = np.zeros(nz.value)
    getattr(lib, fn)(*args, C.c_int64(nz.value), C.byref(nd), C.byref(nz), _ptr(cp), _ptr(ri),
                     _ptr(val), C.byref(st))
    if st.value:
        return None, Status.of(st.value, where)
    return CscMatrix(n, n, cp, ri, val), Status()


def assemble_tetra_lagrange_stiffness_csc(mesh_vertices, tetrahedra, degree, quadrature_degree,
                                          stiffness_coefficient=None, mass_coefficient=None,
                                          rule=K.FFG_RULE_DUFFY, cell_stiffness=None,
                                          cell_mass=None):
    """assemble_tetra_lagrange_stiffness_csc
    (src/assembly/assembly_tetra_lagrange_arbitrary_order_3d.f90:276-334).
    Returns (CscMatrix, Status).  cell_* scale the coefficients cellwise."""
    v = _f64(mesh_vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    cs = _opt(cell_stiffness, len(t))
    cm = _opt(cell_mass, len(t))
    args = [len(v), _ptr(v), len(t), _ptr(t), int(degree), int(rule), int(quadrature_degree),
            1.0 if stiffness_coefficient is None else float(stiffness_coefficient),
            0.0 if mass_coefficient is None else float(mass_coefficient), _ptr(cs), _ptr(cm)]
    return _csc_call("ffg_assemble_tetra_lagrange_stiffness_csc", args,
                     "Tetrahedral H1 sparse assembly failed")


def assemble_tetra_lagrange_stiffness_csc_jvp(mesh_vertices, tetrahedra, degree, quadrature_degree,
                                              stiffness_coefficient, mass_coefficient,
                                              mesh_vertices_dot, stiffness_coefficient_dot,
                                              mass_coefficient_dot, rule=K.FFG_RULE_DUFFY):
    """assemble_tetra_lagrange_stiffness_csc_jvp
    (src/assembly/assembly_tetra_lagrange_arbitrary_order_3d.f90:336-391): the
    tangent of the stiffness + mass CSC along (mesh_vertices_dot,
    stiffness_coefficient_dot, mass_coefficient_dot), on the primal pattern.
    Returns (CscMatrix, Status)."""
    where = "Tetrahedral H1 JVP assembly failed"
    v = _f64(mesh_vertices).reshape(-1, 3)
    vd = _f64(mesh_vertices_dot)
    if vd.size != v.size:
        return None, Status.of(K.FFG_INVALID_INPUT, where)
    vd = vd.reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    args = [len(v), _ptr(v), len(t), _ptr(t), int(degree), int(rule), int(quadrature_degree),
            float(stiffness_coefficient), float(mass_coefficient), _ptr(vd),
            float(stiffness_coefficient_dot), float(mass_coefficient_dot)]
    return _csc_call("ffg_assemble_tetra_lagrange_stiffness_csc_jvp", args, where)


def assemble_tetra_lagrange_stiffness_csc_vjp(mesh_vertices, tetrahedra, degree, quadrature_degree,
                                              stiffness_coefficient, mass_coefficient,
                                              matrix_values_bar, rule=K.FFG_RULE_DUFFY):
    """assemble_tetra_lagrange_stiffness_csc_vjp (same file :393-471).
    matrix_values_bar: one cotangent per entry of the primal CSC.  Returns
    (mesh_vertices_bar (n_vertices, 3), stiffness_coefficient_bar,
    mass_coefficient_bar, Status); the adjoints are zero on failure."""
    v = _f64(mesh_vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    vb_in = _f64(matrix_values_bar).ravel()
    vbar = np.zeros_like(v)
    sb = C.c_double(0.0)
    mb = C.c_double(0.0)
    st = C.c_int(0)
    K.load().ffg_assemble_tetra_lagrange_stiffness_csc_vjp(
        len(v), _ptr(v), len(t), _ptr(t), int(degree), int(rule), int(quadrature_degree),
        float(stiffness_coefficient), float(mass_coefficient), C.c_int64(vb_in.size), _ptr(vb_in),
        _ptr(vbar), C.byref(sb), C.byref(mb), C.byref(st))
    return vbar, sb.value, mb.value, Status.of(st.value, "Tetrahedral H1 VJP failed")


def assemble_tetra_lagrange_scalar_load_samples(mesh_vertices, tetrahedra, degree,
                                                quadrature_degree, source_values,
                                                rule=K.FFG_RULE_DUFFY):
    """assemble_tetra_lagrange_scalar_load_samples (same file :473-528).
    source_values: (T, n_q) samples at the rule's points.  Returns (rhs, Status)."""
    v = _f64(mesh_vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    p = Problem(K.FFG_TETRA_LAGRANGE, degree, t, len(v), rule=rule,
                quadrature_degree=quadrature_degree, boundary="none")
    try:
        src = _f64(source_values)
        if src.size != p.samples_per_cell * len(t):
            return None, Status.of(K.FFG_INVALID_INPUT, "Sampled tetrahedral H1 scalar load failed")
        rhs = np.zeros(p.n_dofs)
        st = C.c_int(0)
        K.load().ffg_assemble_tetra_lagrange_scalar_load_samples(
            len(v), _ptr(v), len(t), _ptr(t), int(degree), int(rule), int(quadrature_degree),
            _ptr(src), p.n_dofs, _ptr(rhs), C.byref(st))
        return (rhs if st.value == 0 else None), Status.of(st.value, "Sampled tetrahedral H1 scalar load failed")
    finally:
        p.close()


def assemble_tetra_nedelec_curl_mass_csc(mesh_vertices, tetrahedra, curl_coefficient=None,
                                         mass_coefficient=None, order=None, cell_curl=None,
                                         cell_mass=None):
    """assemble_tetra_nedelec_curl_mass_csc (src/assembly/assembly_tetra_nedelec_3d.f90:2042-2112,
    arbitrary order :2289-2355).  Returns (CscMatrix, Status)."""
    v = _f64(mesh_vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    args = [len(v), _ptr(v), len(t), _ptr(t), 1 if order is None else int(order),
            1.0 if curl_coefficient is None else float(curl_coefficient),
            1.0 if mass_coefficient is None else float(mass_coefficient),
            _ptr(_opt(cell_curl, len(t))), _ptr(_opt(cell_mass, len(t)))]
    return _csc_call("ffg_assemble_tetra_nedelec_curl_mass_csc", args,
                     "Tetrahedral Nedelec assembly failed")


def cell_tensors(coefficient, vertices, tetrahedra) -> np.ndarray:
    """One symmetric 3 x 3 tensor per cell as the C-ABI takes it (9 doubles per
    cell, column-major).  `coefficient` is an (n_cells, 3, 3) array, or a
    tensor_coefficient_3d-style callable f(x, y, z) -> 3 x 3 that is evaluated
    once per cell at its centroid (the caller declares it cellwise constant)."""
    v = _f64(vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    if callable(coefficient):
        cen = v[t].mean(axis=1)
        ten = np.array([np.asarray(coefficient(*c), dtype=np.float64) for c in cen])
    else:
        ten = np.asarray(coefficient, dtype=np.float64)
    ten = ten.reshape(len(t), 3, 3)
    return np.ascontiguousarray(np.transpose(ten, (0, 2, 1))).reshape(-1)


def assemble_tetra_nedelec_weighted_csc(mesh_vertices, tetrahedra, coefficient, mass_coefficient,
                                        order=None):
    """assemble_tetra_nedelec_weighted_csc (src/assembly/assembly_tetra_nedelec_3d.f90:1870-2000)
    with the tensor coefficient constant on each cell (see cell_tensors).
    Returns (CscMatrix, Status)."""
    v = _f64(mesh_vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    ten = cell_tensors(coefficient, v, t)
    args = [len(v), _ptr(v), len(t), _ptr(t), 1 if order is None else int(order), _ptr(ten),
            float(mass_coefficient)]
    return _csc_call("ffg_assemble_tetra_nedelec_weighted_csc", args,
                     "Weighted tetrahedral Nedelec assembly failed")


def assemble_tetra_nedelec_curl_mass_csc_jvp(mesh_vertices, tetrahedra, order, curl_coefficient,
                                             mass_coefficient, mesh_vertices_dot,
                                             curl_coefficient_dot, mass_coefficient_dot):
    """assemble_tetra_nedelec_curl_mass_csc_jvp
    (src/assembly/assembly_tetra_nedelec_3d.f90:2114-2181): the tangent of the
    curl + mass CSC along (mesh_vertices_dot, curl_coefficient_dot,
    mass_coefficient_dot), on the primal pattern.  Returns (CscMatrix, Status)."""
    where = "Tetrahedral Nedelec curl-mass JVP assembly failed"
    v = _f64(mesh_vertices).reshape(-1, 3)
    vd = _f64(mesh_vertices_dot)
    if vd.size != v.size:
        return None, Status.of(K.FFG_INVALID_INPUT, where)
    vd = vd.reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    args = [len(v), _ptr(v), len(t), _ptr(t), int(order), float(curl_coefficient),
            float(mass_coefficient), _ptr(vd), float(curl_coefficient_dot),
            float(mass_coefficient_dot)]
    return _csc_call("ffg_assemble_tetra_nedelec_curl_mass_csc_jvp", args, where)


def assemble_tetra_nedelec_curl_mass_csc_vjp(mesh_vertices, tetrahedra, order, curl_coefficient,
                                             mass_coefficient, matrix_values_bar):
    """assemble_tetra_nedelec_curl_mass_csc_vjp (same file :2183-2287).
    Returns (mesh_vertices_bar (n_vertices, 3), curl_coefficient_bar,
    mass_coefficient_bar, Status); the adjoints are zero on failure."""
    v = _f64(mesh_vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    vb_in = _f64(matrix_values_bar).ravel()
    vbar = np.zeros_like(v)
    cb = C.c_double(0.0)
    mb = C.c_double(0.0)
    st = C.c_int(0)
    K.load().ffg_assemble_tetra_nedelec_curl_mass_csc_vjp(
        len(v), _ptr(v), len(t), _ptr(t), int(order), float(curl_coefficient),
        float(mass_coefficient), C.c_int64(vb_in.size), _ptr(vb_in), _ptr(vbar), C.byref(cb),
        C.byref(mb), C.byref(st))
    return vbar, cb.value, mb.value, Status.of(st.value, "Tetrahedral Nedelec curl-mass VJP failed")


def _pml_call(fn, v, t, order, stretch_pairs, wave_number, where):
    lib = K.load()
    nd = C.c_int(0)
    nz = C.c_int64(0)
    st = C.c_int(0)
    args = [len(v), _ptr(v), len(t), _ptr(t), int(order), _ptr(stretch_pairs), float(wave_number)]
    getattr(lib, fn)(*args, C.c_int64(0), C.byref(nd), C.byref(nz), None, None, None, C.byref(st))
    if st.value not in (K.FFG_OK, K.FFG_CAPACITY):
        return None, Status.of(st.value, where)
    n = nd.value
    cp = np.zeros(n + 1, np.int64)
    ri = np.zeros(nz.value, np.int32)
    val = np.zeros(2 * nz.value)
    getattr(lib, fn)(*args, C.c_int64(nz.value), C.byref(nd), C.byref(nz), _ptr(cp), _ptr(ri),
                     _ptr(val), C.byref(st))
    if st.value:
        return None, Status.of(st.value, where)
    return CscMatrix(n, n, cp, ri, val.view(np.complex128)), Status()


def assemble_tetra_nedelec_pml_csc(mesh_vertices, tetrahedra, order, stretch, wave_number):
    """assemble_tetra_nedelec_pml_csc (src/assembly/assembly_tetra_nedelec_3d.f90:1613-1685):
    stretch (T, 3) complex per cell.  Returns (CscMatrix with complex values, Status)."""
    v = _f64(mesh_vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    s = np.ascontiguousarray(np.asarray(stretch, np.complex128).reshape(len(t), 3))
    return _pml_call("ffg_assemble_tetra_nedelec_pml_csc", v, t, order, s.view(np.float64),
                     wave_number, "Complex tetrahedral Nedelec PML assembly failed")


def assemble_tetra_nedelec_curvilinear_pml_csc(mesh_vertices, tetrahedra, order, stretch,
                                               wave_number):
    """assemble_tetra_nedelec_curvilinear_pml_csc (same file :1372-1444): stretch
    (T, 3, 3) complex, stretch[t] the cell's matrix.  Returns (CscMatrix, Status)."""
    v = _f64(mesh_vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    s = np.asarray(stretch, np.complex128).reshape(len(t), 3, 3)
    s = np.ascontiguousarray(np.transpose(s, (0, 2, 1)))  # column-major per cell
    return _pml_call("ffg_assemble_tetra_nedelec_curvilinear_pml_csc", v, t, order,
                     s.view(np.float64), wave_number,
                     "Curvilinear tetrahedral Nedelec PML assembly failed")


def assemble_tetra_nedelec_vector_load_samples(mesh_vertices, tetrahedra, order, source_values):
    """assemble_tetra_nedelec_vector_load_samples (assembly_tetra_nedelec_3d.f90:128-185).
    source_values: (T, n_q, 3) at the order's load points.  Returns (rhs, Status)."""
    v = _f64(mesh_vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    p = Problem(K.FFG_TETRA_NEDELEC, order, t, len(v), boundary="none")
    try:
        src = _f64(source_values)
        if src.size != 3 * p.samples_per_cell * len(t):
            return None, Status.of(K.FFG_INVALID_INPUT, "Sampled tetrahedral Nedelec vector load failed")
        rhs = np.zeros(p.n_dofs)
        st = C.c_int(0)
        K.load().ffg_assemble_tetra_nedelec_vector_load_samples(
            len(v), _ptr(v), len(t), _ptr(t), int(order), _ptr(src), p.n_dofs, _ptr(rhs),
            C.byref(st))
        return (rhs if st.value == 0 else None), Status.of(st.value, "Sampled tetrahedral Nedelec vector load failed")
    finally:
        p.close()


def assemble_triangle_lagrange_csc(vertices, triangles, degree, quadrature_degree=None,
                                   stiffness_coefficient=1.0, mass_coefficient=0.0,
                                   cell_stiffness=None, cell_mass=None):
    """kappa grad u . grad v + m u v on arbitrary-order triangle Lagrange elements
    (the basis of src/elements/triangle_lagrange_arbitrary_order.f90:29-127)
    in CSC.  quadrature_degree defaults to 2 degree.  Returns (CscMatrix, Status)."""
    v = _f64(vertices).reshape(-1, 2)
    t = _i32(triangles).reshape(-1, 3)
    q = 2 * degree if quadrature_degree is None else quadrature_degree
    args = [len(v), _ptr(v), len(t), _ptr(t), int(degree), int(q), float(stiffness_coefficient),
            float(mass_coefficient), _ptr(_opt(cell_stiffness, len(t))),
            _ptr(_opt(cell_mass, len(t)))]
    return _csc_call("ffg_assemble_triangle_lagrange_csc", args,
                     "Triangle Lagrange assembly failed")


def assemble_triangle_lagrange_load_samples(vertices, triangles, degree, source_values,
                                            quadrature_degree=None):
    """The load of source samples at the rule's points (T, n_q).  Returns (rhs, Status)."""
    v = _f64(vertices).reshape(-1, 2)
    t = _i32(triangles).reshape(-1, 3)
    q = 2 * degree if quadrature_degree is None else quadrature_degree
    p = Problem(K.FFG_TRIANGLE_LAGRANGE, degree, t, len(v), quadrature_degree=q, boundary="none")
    try:
        src = _f64(source_values)
        if src.size != p.samples_per_cell * len(t):
            return None, Status.of(K.FFG_INVALID_INPUT, "Triangle Lagrange load failed")
        rhs = np.zeros(p.n_dofs)
        st = C.c_int(0)
        K.load().ffg_assemble_triangle_lagrange_load_samples(
            len(v), _ptr(v), len(t), _ptr(t), int(degree), int(q), _ptr(src), p.n_dofs,
            _ptr(rhs), C.byref(st))
        return (rhs if st.value == 0 else None), Status.of(st.value, "Triangle Lagrange load failed")
    finally:
        p.close()


def solve_triangle_lagrange(vertices, triangles, degree, source, stiffness_coefficient=1.0,
                            mass_coefficient=0.0, boundary_value=None, options=None,
                            quadrature_degree=None):
    """-div(kappa grad u) + m u = f on arbitrary-order triangles with u = g on
    the boundary edges (boundary_value a vectorised g(x, y) or per-DoF
    values; None: no essential boundary).  Returns (solution, Status, SolverStats)."""
    v = _f64(vertices).reshape(-1, 2)
    t = _i32(triangles).reshape(-1, 3)
    q = 2 * degree if quadrature_degree is None else quadrature_degree
    bmode = "all" if boundary_value is not None else "none"
    with Problem(K.FFG_TRIANGLE_LAGRANGE, degree, t, len(v), quadrature_degree=q,
                 boundary=bmode) as p:
        pts = p.sample_points(v)
        samples = None
        if source is not None:
            samples = np.asarray(source(pts[..., 0], pts[..., 1]), np.float64) if callable(source) \
                else _f64(source)
        g = None
        if boundary_value is not None:
            if callable(boundary_value):
                dp = p.dof_points(v)
                g = np.where(p.constrained(), boundary_value(dp[:, 0], dp[:, 1]), 0.0)
            else:
                g = _f64(boundary_value)
        sol, stats = p.solve(v, stiffness_coefficient, mass_coefficient, None, None, samples, g,
                             options)
        return sol, Status.of(0 if stats.converged else K.FFG_NOT_CONVERGED,
                              "Triangle Lagrange solve failed"), stats


def assemble_scalar_p1_csc(vertices, triangles, mass_coefficient=0.0, stiffness_coefficient=1.0,
                           cell_stiffness=None):
    """assemble_scalar_p1_matrix (src/fortfem_forms_simple.f90:1678-1728) scattered into CSC."""
    v = _f64(vertices).reshape(-1, 2)
    t = _i32(triangles).reshape(-1, 3)
    lib = K.load()
    cs = _opt(cell_stiffness, len(t))
    nz = C.c_int64(0)
    st = C.c_int(0)
    args = [len(v), _ptr(v), len(t), _ptr(t), float(mass_coefficient), float(stiffness_coefficient),
            _ptr(cs)]
    lib.ffg_assemble_scalar_p1_csc(*args, C.c_int64(0), C.byref(nz), None, None, None, C.byref(st))
    if st.value not in (0, K.FFG_CAPACITY):
        return None, Status.of(st.value, "assemble_scalar_p1_matrix")
    n = len(v)
    cp = np.zeros(n + 1, np.int64)
    ri = np.zeros(nz.value, np.int32)
    val = np.zeros(nz.value)
    lib.ffg_assemble_scalar_p1_csc(*args, C.c_int64(nz.value), C.byref(nz), _ptr(cp), _ptr(ri),
                                   _ptr(val), C.byref(st))
    if st.value:
        return None, Status.of(st.value, "assemble_scalar_p1_matrix")
    return CscMatrix(n, n, cp, ri, val), Status()


# -------------------------------------------------------------------- solve

def solve_sparse(A_sparse: CscMatrix, b, x: np.ndarray, opts: Optional[SolverOptions] = None) -> SolverStats:
    """solve_sparse(A_sparse, b, x, opts, stats) (src/solvers/advanced_solvers.f90:135-195):
    x (float64 numpy array) is the initial guess and is overwritten in place."""
    opts = opts or SolverOptions()
    n = A_sparse.nrow
    if A_sparse.ncol != n:
        raise FortfemError(K.FFG_INVALID_INPUT, "solve_sparse: only square matrices are supported")
    b = _f64(b)
    if b.size != n or x.size != n or x.dtype != np.float64 or not x.flags.c_contiguous:
        raise FortfemError(K.FFG_INVALID_INPUT, "solve_sparse: incompatible vector size")
    cp = np.ascontiguousarray(A_sparse.col_ptr, dtype=np.int64)
    ri = _i32(A_sparse.row_idx)
    val = _f64(A_sparse.val)
    oc = opts.to_c()
    sc = K.SolverStatsC()
    st = C.c_int(0)
    K.load().ffg_solve_sparse(n, int(cp[-1]), _ptr(cp), _ptr(ri), _ptr(val), _ptr(b), _ptr(x),
                              C.byref(oc), C.byref(sc), C.byref(st))
    if st.value not in (0, K.FFG_NOT_CONVERGED):
        raise FortfemError(st.value, "solve_sparse")
    return SolverStats.from_c(sc)


def spmv(matrix: CscMatrix, vector) -> np.ndarray:
    """spmv (src/solvers/fortfem_sparse_matrix.f90:46-58): product = A x."""
    x = _f64(vector)
    y = np.zeros(matrix.nrow)
    cp = np.ascontiguousarray(matrix.col_ptr, dtype=np.int64)
    ri = _i32(matrix.row_idx)
    val = _f64(matrix.val)
    st = C.c_int(0)
    K.load().ffg_csc_matvec(matrix.nrow, int(cp[-1]), _ptr(cp), _ptr(ri), _ptr(val), _ptr(x),
                            _ptr(y), C.byref(st))
    if st.value:
        raise FortfemError(st.value, "spmv")
    return y


def build_topology(family: int, degree: int, cells, n_vertices: int, boundary="none"):
    """Host-only topology (ffg_build_topology): returns dict with global_dofs
    (cells x n_b), constrained mask, and the constrained CSC pattern."""
    cells = _i32(cells)
    vpc = 3 if family in (K.FFG_TRIANGLE_P1, K.FFG_TRIANGLE_LAGRANGE) else 4
    nc = cells.size // vpc
    if isinstance(boundary, str):
        mode, mask = _BOUNDARY[boundary], None
    else:
        mode, mask = K.FFG_BOUNDARY_MASK, np.ascontiguousarray(boundary, dtype=np.uint8)
    nd, nf, nz = C.c_int64(0), C.c_int64(0), C.c_int64(0)
    st = C.c_int(0)
    lib = K.load()
    lib.ffg_build_topology(int(family), int(degree), int(n_vertices), nc, _ptr(cells), mode,
                           _ptr(mask), C.c_int64(0), C.c_int64(0), C.byref(nd), C.byref(nf),
                           C.byref(nz), None, None, None, None, C.byref(st))
    if st.value not in (0, K.FFG_CAPACITY):
        raise FortfemError(st.value, "ffg_build_topology")
    if family == K.FFG_TRIANGLE_P1:
        nb = 3
    elif family == K.FFG_TRIANGLE_LAGRANGE:
        nb = (degree + 1) * (degree + 2) // 2
    elif family == K.FFG_TETRA_LAGRANGE:
        nb = (degree + 1) * (degree + 2) * (degree + 3) // 6
    else:
        nb = degree * (degree + 2) * (degree + 3) // 2
    gd = np.zeros((nc, nb), np.int32)
    con = np.zeros(nd.value, np.uint8)
    cp = np.zeros(nf.value + 1, np.int64)
    ri = np.zeros(nz.value, np.int32)
    lib.ffg_build_topology(int(family), int(degree), int(n_vertices), nc, _ptr(cells), mode,
                           _ptr(mask), C.c_int64(nd.value), C.c_int64(nz.value), C.byref(nd),
                           C.byref(nf), C.byref(nz), _ptr(gd), _ptr(con), _ptr(cp), _ptr(ri),
                           C.byref(st))
    if st.value:
        raise FortfemError(st.value, "ffg_build_topology")
    return dict(global_dofs=gd, constrained=con.astype(bool), n_dofs=nd.value, n_free=nf.value,
                col_ptr=cp, row_idx=ri)


_BOUNDARY = {"none": K.FFG_BOUNDARY_NONE, "all": K.FFG_BOUNDARY_ALL}


# ------------------------------------------------- device-resident problems

class Problem:
    """A mesh + element family whose topology, CSC pattern and slot maps live
    in HBM (ffg_problem_create).  ``solve`` assembles and solves the
    constrained system for new geometry, coefficients and sources."""

    def __init__(self, family: int, degree: int, cells, n_vertices: int,
                 rule: int = K.FFG_RULE_DUFFY, quadrature_degree: int = 0,
                 boundary: Union[str, np.ndarray] = "all"):
        self.family = family
        self.degree = degree
        self.cells = _i32(cells)
        self.n_vertices = int(n_vertices)
        triangles = family in (K.FFG_TRIANGLE_P1, K.FFG_TRIANGLE_LAGRANGE)
        self.dim = 2 if triangles else 3
        vpc = 3 if triangles else 4
        n_cells = self.cells.size // vpc
        self.n_cells = n_cells
        if isinstance(boundary, str):
            mode, mask = _BOUNDARY[boundary], None
        else:
            mode, mask = K.FFG_BOUNDARY_MASK, np.ascontiguousarray(boundary, dtype=np.uint8)
        h = C.c_int(0)
        nd, nf, nz = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        spc = C.c_int(0)
        st = C.c_int(0)
        K.load().ffg_problem_create(int(family), int(degree), self.n_vertices, n_cells,
                                    _ptr(self.cells), int(rule), int(quadrature_degree), mode,
                                    _ptr(mask), C.byref(h), C.byref(nd), C.byref(nf), C.byref(nz),
                                    C.byref(spc), C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_create")
        self.handle = h.value
        self.n_dofs = nd.value
        self.n_free = nf.value
        self.nnz = nz.value
        self.samples_per_cell = spc.value
        self.sample_width = 3 if family == K.FFG_TETRA_NEDELEC else 1

    def close(self):
        if getattr(self, "handle", 0):
            st = C.c_int(0)
            K.load().ffg_problem_free(self.handle, C.byref(st))
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def sample_points(self, vertices) -> np.ndarray:
        v = _f64(vertices)
        out = np.zeros((self.n_cells, self.samples_per_cell, 3))
        st = C.c_int(0)
        K.load().ffg_problem_sample_points(self.handle, _ptr(v), _ptr(out), C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_sample_points")
        return out

    def dof_points(self, vertices) -> np.ndarray:
        v = _f64(vertices)
        out = np.zeros((self.n_dofs, 3))
        st = C.c_int(0)
        K.load().ffg_problem_dof_points(self.handle, _ptr(v), _ptr(out), C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_dof_points")
        return out

    def constrained(self) -> np.ndarray:
        out = np.zeros(self.n_dofs, np.uint8)
        st = C.c_int(0)
        K.load().ffg_problem_constrained(self.handle, _ptr(out), C.byref(st))
        return out.astype(bool)

    def topology(self) -> dict:
        """The problem's DoF map (ffg_problem_topology): global_dofs (n_cells x n_b)
        and, for Nedelec, edge_sign (n_cells x 6) and face_perm (n_cells x 4)."""
        gd = np.zeros((self.n_cells, self._nb()), np.int32)
        es = np.zeros((self.n_cells, 6), np.int8)
        fp = np.zeros((self.n_cells, 4), np.uint8)
        st = C.c_int(0)
        K.load().ffg_problem_topology(self.handle, _ptr(gd), _ptr(es), _ptr(fp), C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_topology")
        out = {"global_dofs": gd}
        if self.family == K.FFG_TETRA_NEDELEC:
            out.update(edge_sign=es, face_perm=fp)
        return out

    def _nb(self) -> int:
        k = self.degree
        if self.family == K.FFG_TETRA_NEDELEC:
            return k * (k + 2) * (k + 3) // 2
        if self.family == K.FFG_TETRA_LAGRANGE:
            return (k + 1) * (k + 2) * (k + 3) // 6
        if self.family == K.FFG_TRIANGLE_LAGRANGE:
            return (k + 1) * (k + 2) // 2
        return 3

    def _inputs(self, vertices, cell_a, cell_b, samples, g):
        v = _f64(vertices)
        if v.size != self.n_vertices * self.dim:
            raise FortfemError(K.FFG_INVALID_INPUT, "vertices")
        ca = _opt(cell_a, self.n_cells)
        cb = _opt(cell_b, self.n_cells)
        s = _opt(samples, self.n_cells * self.samples_per_cell * self.sample_width)
        gg = _opt(g, self.n_dofs)
        return v, ca, cb, s, gg

    def solve(self, vertices, coef_a=1.0, coef_b=0.0, cell_a=None, cell_b=None, samples=None,
              constrained_values=None, options: Optional[SolverOptions] = None, out=None):
        """Assemble + constrain + solve with host arrays; returns (solution, SolverStats).
        `out` (float64, n_dofs, C-contiguous) receives the solution; a page-locked
        buffer there makes the device-to-host copy a direct DMA."""
        v, ca, cb, s, g = self._inputs(vertices, cell_a, cell_b, samples, constrained_values)
        opts = options or SolverOptions(precision="mixed", tolerance=1e-10, preconditioner="jacobi",
                                        max_iterations=1000000)
        oc = opts.to_c()
        sc = K.SolverStatsC()
        if out is None:
            sol = np.zeros(self.n_dofs)
        else:
            sol = out
            if sol.dtype != np.float64 or sol.size != self.n_dofs or not sol.flags.c_contiguous:
                raise FortfemError(K.FFG_INVALID_INPUT, "out must be float64, n_dofs, contiguous")
        st = C.c_int(0)
        K.load().ffg_problem_solve(self.handle, _ptr(v), float(coef_a), float(coef_b), _ptr(ca),
                                   _ptr(cb), _ptr(s), _ptr(g), C.byref(oc), _ptr(sol), C.byref(sc),
                                   0, None, C.byref(st))
        if st.value not in (0, K.FFG_NOT_CONVERGED):
            raise FortfemError(st.value, "ffg_problem_solve")
        return sol, SolverStats.from_c(sc)

    def solve_device(self, vertices, solution, coef_a=1.0, coef_b=0.0, cell_a=None, cell_b=None,
                     samples=None, constrained_values=None, options: Optional[SolverOptions] = None,
                     stream=None) -> SolverStats:
        """Same as solve with CUDA tensors (torch) resident in HBM; writes `solution`."""
        def p(t):
            return None if t is None else C.c_void_p(t.data_ptr())
        opts = options or SolverOptions(precision="mixed", tolerance=1e-10, preconditioner="jacobi",
                                        max_iterations=1000000)
        oc = opts.to_c()
        sc = K.SolverStatsC()
        st = C.c_int(0)
        s = None if stream is None else C.c_void_p(int(stream.cuda_stream))
        K.load().ffg_problem_solve(self.handle, p(vertices), float(coef_a), float(coef_b), p(cell_a),
                                   p(cell_b), p(samples), p(constrained_values), C.byref(oc),
                                   p(solution), C.byref(sc), 1, s, C.byref(st))
        if st.value not in (0, K.FFG_NOT_CONVERGED):
            raise FortfemError(st.value, "ffg_problem_solve")
        return SolverStats.from_c(sc)

    def batch_stats(self) -> Optional[SolverStats]:
        """Statistics of this problem's last batched solve (ffg_problem_batch_stats),
        or None while its batch is still running."""
        sc = K.SolverStatsC()
        st = C.c_int(0)
        K.load().ffg_problem_batch_stats(self.handle, C.byref(sc), C.byref(st))
        if st.value == K.FFG_NOT_READY:
            return None
        if st.value not in (0, K.FFG_NOT_CONVERGED):
            raise FortfemError(st.value, "ffg_problem_batch_stats")
        return SolverStats.from_c(sc)

    def phase_times(self) -> dict:
        """Device-side phase profile of the last solve (seconds, CTA 0's view)."""
        out = np.zeros(6)
        st = C.c_int(0)
        K.load().ffg_problem_phase_times(self.handle, _ptr(out), C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_phase_times")
        return {"fp64_continuation": bool(out[0]), "spmv": out[1], "spmv_barrier": out[2],
                "vector": out[3], "vector_barrier": out[4], "residual_replacement": out[5]}

    def reduced_system(self, vertices, coef_a=1.0, coef_b=0.0, cell_a=None, cell_b=None,
                       samples=None, constrained_values=None):
        """The constrained (free x free) CSC, its lifted right-hand side and the free DoFs."""
        v, ca, cb, s, g = self._inputs(vertices, cell_a, cell_b, samples, constrained_values)
        cp = np.zeros(self.n_free + 1, np.int64)
        ri = np.zeros(self.nnz, np.int32)
        val = np.zeros(self.nnz)
        rhs = np.zeros(self.n_free)
        free = np.zeros(self.n_free, np.int32)
        nz = C.c_int64(0)
        st = C.c_int(0)
        K.load().ffg_problem_reduced_system(self.handle, _ptr(v), float(coef_a), float(coef_b),
                                            _ptr(ca), _ptr(cb), _ptr(s), _ptr(g),
                                            C.c_int64(self.nnz), C.byref(nz), _ptr(cp), _ptr(ri),
                                            _ptr(val), _ptr(rhs), _ptr(free), C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_reduced_system")
        return CscMatrix(self.n_free, self.n_free, cp, ri, val), rhs, free

    def autotune(self, vertices, coef_a=1.0, coef_b=0.0, cell_a=None, cell_b=None,
                 samples=None) -> dict:
        """Choose this problem's launch shapes by timing candidates on these inputs
        (ffg_problem_autotune); returns the choice and the measured times."""
        v, ca, cb, s, _ = self._inputs(vertices, cell_a, cell_b, samples, None)
        t = K.TuningC()
        st = C.c_int(0)
        K.load().ffg_problem_autotune(self.handle, _ptr(v), float(coef_a), float(coef_b),
                                      _ptr(ca), _ptr(cb), _ptr(s), 0, C.byref(t), C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_autotune")
        return {name: getattr(t, name) for name, _ in K.TuningC._fields_}

    def set_tuning(self, tuning: dict):
        """Apply launch shapes from an earlier autotune (ffg_problem_set_tuning)."""
        t = K.TuningC()
        for name, _ in K.TuningC._fields_:
            setattr(t, name, tuning.get(name, 0))
        st = C.c_int(0)
        K.load().ffg_problem_set_tuning(self.handle, C.byref(t), C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_set_tuning")

    def set_assembly_precision(self, precision: str):
        """Nedelec orders 3-6: "fp64" (CUDA-core FP64 contraction, the parity
        path) or "tf32x3" (tensor-core 3xTF32 contraction, FP32 accumulation)
        for every following assembly (ffg_problem_set_assembly_precision)."""
        modes = {"fp64": K.FFG_ASSEMBLY_FP64, "tf32x3": K.FFG_ASSEMBLY_TF32X3}
        if precision not in modes:
            raise FortfemError(K.FFG_INVALID_INPUT, f"assembly precision {precision!r}")
        st = C.c_int(0)
        K.load().ffg_problem_set_assembly_precision(self.handle, modes[precision], C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_set_assembly_precision")

    def set_cell_tensor(self, coefficient, vertices=None):
        """Nedelec: a symmetric 3 x 3 tensor per cell (array (n_cells, 3, 3), or a
        callable evaluated at the cell centroids of `vertices`) multiplying the
        curl coefficient in every following assembly; None clears it
        (ffg_problem_set_cell_tensor)."""
        st = C.c_int(0)
        if coefficient is None:
            K.load().ffg_problem_set_cell_tensor(self.handle, None, C.byref(st))
        else:
            if callable(coefficient) and vertices is None:
                raise FortfemError(K.FFG_INVALID_INPUT, "set_cell_tensor: vertices needed")
            ten = cell_tensors(coefficient, vertices if vertices is not None
                               else np.zeros((self.n_vertices, 3)), self.cells)
            K.load().ffg_problem_set_cell_tensor(self.handle, _ptr(ten), C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_set_cell_tensor")

    def evaluate(self, vertices, solution, cells, points, physical=False):
        """Batched evaluation at (cell, point) queries (ffg_problem_evaluate):
        Lagrange (values (n,), gradients (n, 3)), Nedelec (fields (n, 3),
        curls (n, 3)), and the per-query status (0 or FFG_INVALID_INPUT)."""
        v = _f64(vertices)
        u = _f64(solution)
        if u.size != self.n_dofs:
            raise FortfemError(K.FFG_INVALID_INPUT, "solution size")
        c = _i32(cells).ravel()
        x = _f64(points).reshape(-1, 3)
        if len(x) != len(c):
            raise FortfemError(K.FFG_INVALID_INPUT, "one point per cell")
        wv = 3 if self.family == K.FFG_TETRA_NEDELEC else 1
        vals = np.zeros((len(c), wv))
        ders = np.zeros((len(c), 3))
        qst = np.zeros(len(c), np.int32)
        st = C.c_int(0)
        K.load().ffg_problem_evaluate(self.handle, _ptr(v), _ptr(u), len(c), _ptr(c), _ptr(x),
                                      K.FFG_POINT_PHYSICAL if physical else K.FFG_POINT_REFERENCE,
                                      _ptr(vals), _ptr(ders), _ptr(qst), 0, None, C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_evaluate")
        return (vals[:, 0] if wv == 1 else vals), ders, qst

    def probe(self, vertices, solution, points, mode="average"):
        """Point probes without a cell hint (ffg_problem_probe): values,
        derivatives (gradient / curl) and the number of contributing cells per
        point (0: outside the mesh; -1: rejected as the reference's probe)."""
        v = _f64(vertices)
        u = _f64(solution)
        if u.size != self.n_dofs:
            raise FortfemError(K.FFG_INVALID_INPUT, "solution size")
        x = _f64(points).reshape(-1, 3)
        wv = 3 if self.family == K.FFG_TETRA_NEDELEC else 1
        vals = np.zeros((len(x), wv))
        ders = np.zeros((len(x), 3))
        cnt = np.zeros(len(x), np.int32)
        st = C.c_int(0)
        m = {"average": K.FFG_PROBE_AVERAGE, "first": K.FFG_PROBE_FIRST}[mode]
        K.load().ffg_problem_probe(self.handle, _ptr(v), _ptr(u), len(x), _ptr(x), m, _ptr(vals),
                                   _ptr(ders), _ptr(cnt), 0, None, C.byref(st))
        if st.value:
            raise FortfemError(st.value, "ffg_problem_probe")
        return (vals[:, 0] if wv == 1 else vals), ders, cnt


def evaluate_tetra_lagrange_solution(vertices, tetrahedra, degree, solution, tetrahedron,
                                     reference_point):
    """evaluate_tetra_lagrange_solution
    (src/solvers/fortfem_tetra_lagrange_solver_3d.f90:131-150), zero-based
    tetrahedron index.  Returns (value, gradient (3,), status code)."""
    v = _f64(vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    with Problem(K.FFG_TETRA_LAGRANGE, degree, t, len(v), boundary="none") as p:
        u = _f64(solution)
        if u.size != p.n_dofs:
            return 0.0, np.zeros(3), K.FFG_INVALID_INPUT
        try:
            val, grad, qst = p.evaluate(v, u, [tetrahedron], [reference_point])
        except FortfemError as e:
            return 0.0, np.zeros(3), e.code
        return float(val[0]), grad[0], int(qst[0])


def probe_tetra_nedelec_solution(vertices, tetrahedra, order, solution, points, mode="average"):
    """evaluate_box_solution_order (src/solvers/fortfem_magnetic_box_3d.f90:269-343,
    mode "average") or probe_box_az / probe_box_curl (:345-440, mode "first")
    at every point: (fields (n, 3), curls (n, 3), counts)."""
    v = _f64(vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    with Problem(K.FFG_TETRA_NEDELEC, order, t, len(v), boundary="none") as p:
        return p.probe(v, solution, points, mode)


def _samples(source, points, width):
    if source is None:
        return None
    if callable(source):
        vals = np.asarray(source(points[..., 0], points[..., 1], points[..., 2]), dtype=np.float64)
        if width == 3:
            vals = np.stack(np.broadcast_arrays(*vals), axis=-1) if vals.shape[-1] != 3 else vals
        return vals
    return np.asarray(source, dtype=np.float64)


def solve_tetra_lagrange_diffusion_reaction(vertices, tetrahedra, degree, source,
                                            stiffness_coefficient=1.0, mass_coefficient=0.0,
                                            boundary_value=None, options=None,
                                            quadrature_degree=None, rule=K.FFG_RULE_DUFFY,
                                            cell_stiffness=None, cell_mass=None):
    """solve_tetra_lagrange_diffusion_reaction
    (src/solvers/fortfem_tetra_lagrange_solver_3d.f90:64-129) with the sparse
    direct solve replaced by the GPU Jacobi-PCG.  source / boundary_value are
    vectorised callables f(x, y, z) or arrays of samples / DoF values.
    Returns (solution, Status, SolverStats)."""
    v = _f64(vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    q = 2 * degree + 4 if quadrature_degree is None else quadrature_degree
    bmode = "all" if boundary_value is not None else "none"
    with Problem(K.FFG_TETRA_LAGRANGE, degree, t, len(v), rule=rule, quadrature_degree=q,
                 boundary=bmode) as p:
        samples = _samples(source, p.sample_points(v), 1)
        g = None
        if boundary_value is not None:
            if callable(boundary_value):
                pts = p.dof_points(v)
                g = np.where(p.constrained(), boundary_value(pts[:, 0], pts[:, 1], pts[:, 2]), 0.0)
            else:
                g = _f64(boundary_value)
        sol, stats = p.solve(v, stiffness_coefficient, mass_coefficient, cell_stiffness, cell_mass,
                             samples, g, options)
        return sol, Status.of(0 if stats.converged else K.FFG_NOT_CONVERGED,
                              "Tetrahedral H1 diffusion-reaction solve failed"), stats


def solve_tetra_lagrange_poisson(vertices, tetrahedra, degree, source, boundary_value, options=None,
                                 **kw):
    """solve_tetra_lagrange_poisson (fortfem_tetra_lagrange_solver_3d.f90:50-62)."""
    return solve_tetra_lagrange_diffusion_reaction(vertices, tetrahedra, degree, source, 1.0, 0.0,
                                                   boundary_value, options, **kw)


def solve_tetra_nedelec_curl_mass(vertices, tetrahedra, order, source, curl_coefficient,
                                  mass_coefficient, zero_tangential_boundary=False, options=None,
                                  cell_curl=None, cell_mass=None):
    """solve_tetra_nedelec_curl_mass (src/solvers/fortfem_tetra_nedelec_solver_3d.f90:361-414),
    sparse direct solve replaced by the GPU Jacobi-PCG.  Returns (solution, Status, SolverStats)."""
    v = _f64(vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    with Problem(K.FFG_TETRA_NEDELEC, order, t, len(v),
                 boundary="all" if zero_tangential_boundary else "none") as p:
        samples = _samples(source, p.sample_points(v), 3)
        sol, stats = p.solve(v, curl_coefficient, mass_coefficient, cell_curl, cell_mass, samples,
                             None, options)
        return sol, Status.of(0 if stats.converged else K.FFG_NOT_CONVERGED,
                              "Tetrahedral Nedelec curl-mass solve failed"), stats


def solve_tetra_nedelec_weighted_curl_mass(vertices, tetrahedra, order, curl_coefficient, source,
                                           mass_coefficient, zero_tangential_boundary=False,
                                           options=None):
    """solve_tetra_nedelec_weighted_curl_mass (src/solvers/fortfem_tetra_nedelec_solver_3d.f90:41-95)
    with the tensor coefficient constant on each cell (array or callable evaluated
    at the centroids), sparse direct solve replaced by the GPU Jacobi-PCG.
    Returns (solution, Status, SolverStats)."""
    where = "Weighted tetrahedral Nedelec curl-mass solve failed"
    if order < 1 or not mass_coefficient > 0.0:
        return None, Status.of(K.FFG_INVALID_INPUT, where), None
    v = _f64(vertices).reshape(-1, 3)
    t = _i32(tetrahedra).reshape(-1, 4)
    with Problem(K.FFG_TETRA_NEDELEC, order, t, len(v),
                 boundary="all" if zero_tangential_boundary else "none") as p:
        p.set_cell_tensor(coefficient=curl_coefficient, vertices=v)
        samples = _samples(source, p.sample_points(v), 3)
        sol, stats = p.solve(v, 1.0, mass_coefficient, None, None, samples, None, options)
        return sol, Status.of(0 if stats.converged else K.FFG_NOT_CONVERGED, where), stats


_BATCH_MODES = {"cta_per_system": K.FFG_BATCH_CTA_PER_SYSTEM,
                "whole_device": K.FFG_BATCH_WHOLE_DEVICE,
                "cta_groups": K.FFG_BATCH_CTA_GROUPS}


def solve_batch(problems, vertices, solutions, coef_a, coef_b, cell_a=None, cell_b=None,
                samples=None, constrained_values=None, options: Optional[SolverOptions] = None,
                mode: str = "cta_per_system", stream=None) -> None:
    """Enqueue assemble + solve of several device-resident problems on `stream`
    (ffg_problem_solve_batch) and return at once.  All arrays are CUDA
    tensors, one per problem (lists; None entries where a problem has none);
    coef_a / coef_b are sequences of floats.  Collect each result with
    Problem.batch_stats once the stream has passed this call."""
    n = len(problems)
    if n == 0:
        return
    for seq in (vertices, solutions, coef_a, coef_b):
        if len(seq) != n:
            raise FortfemError(K.FFG_INVALID_INPUT, "solve_batch: one entry per problem")

    def ptrs(seq):
        if seq is None or all(t is None for t in seq):
            return None
        if len(seq) != n:
            raise FortfemError(K.FFG_INVALID_INPUT, "solve_batch: one entry per problem")
        return (C.c_void_p * n)(*[None if t is None else t.data_ptr() for t in seq])

    handles = (C.c_int * n)(*[p.handle for p in problems])
    ca = (C.c_double * n)(*[float(a) for a in coef_a])
    cb = (C.c_double * n)(*[float(b) for b in coef_b])
    opts = options or SolverOptions(precision="mixed", tolerance=1e-10, preconditioner="jacobi",
                                    max_iterations=1000000)
    oc = opts.to_c()
    st = C.c_int(0)
    s = None if stream is None else C.c_void_p(int(stream.cuda_stream))
    K.load().ffg_problem_solve_batch(n, handles, ptrs(vertices), ca, cb, ptrs(cell_a), ptrs(cell_b),
                                     ptrs(samples), ptrs(constrained_values), C.byref(oc),
                                     ptrs(solutions), _BATCH_MODES[mode], s, C.byref(st))
    if st.value:
        raise FortfemError(st.value, "ffg_problem_solve_batch")


def solve_scalar_p1(vertices, triangles, load=1.0, stiffness_coefficient=1.0, mass_coefficient=0.0,
                    boundary_value=0.0, options=None, cell_stiffness=None):
    """The compiled P1 problem of solve(a == L, uh, bc)
    (src/solvers/fortfem_solvers_laplacian.f90:59-112): P1 stiffness (+ mass),
    load `load`*area/3, Dirichlet value on all boundary vertices.  The
    boundary rows are eliminated as the reference does; the free block is
    solved on the GPU.  Returns (values, SolverStats)."""
    v = _f64(vertices).reshape(-1, 2)
    t = _i32(triangles).reshape(-1, 3)
    with Problem(K.FFG_TRIANGLE_P1, 1, t, len(v), boundary="all") as p:
        samples = np.full(len(t), float(load)) if np.isscalar(load) else _f64(load)
        g = np.where(p.constrained(), float(boundary_value), 0.0)
        return p.solve(v, stiffness_coefficient, mass_coefficient, cell_stiffness, None, samples, g,
                       options)
