"""ctypes binding of libfortfem_gpu.so (the C-ABI of include/fortfem_gpu.h).

The library is built in-tree by ``python -m fortfem_b200.build``.  Loading
fails loudly when it is missing: there is no CPU fallback in this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfortfem_gpu.so")

FFG_OK = 0
FFG_INVALID_INPUT = -1
FFG_CAPACITY = -2
FFG_BAD_HANDLE = -3
FFG_CUDA_ERROR = -4
FFG_OUT_OF_MEMORY = -5
FFG_NOT_CONVERGED = -6
FFG_TIMEOUT = -7
FFG_NO_DEVICE = -8
FFG_NOT_READY = -9

FFG_TETRA_LAGRANGE = 1
FFG_TETRA_NEDELEC = 2
FFG_TRIANGLE_P1 = 3
FFG_TRIANGLE_LAGRANGE = 4

FFG_RULE_DUFFY = 0
FFG_RULE_DEGREE_TWO = 1

FFG_BOUNDARY_NONE = 0
FFG_BOUNDARY_ALL = 1
FFG_BOUNDARY_MASK = 2

FFG_ASSEMBLY_FP64 = 0
FFG_ASSEMBLY_TF32X3 = 1
FFG_PRECISION_FP64 = 0
FFG_PRECISION_MIXED = 1
FFG_PRECISION_MIXED16 = 2
FFG_OPTIONS_VERSION = 1
FFG_NOALLOC_MAX_ROWS = 65536
FFG_BATCH_CTA_PER_SYSTEM = 0
FFG_BATCH_WHOLE_DEVICE = 1
FFG_BATCH_CTA_GROUPS = 2
FFG_POINT_REFERENCE = 0
FFG_POINT_PHYSICAL = 1
FFG_PROBE_AVERAGE = 0
FFG_PROBE_FIRST = 1
FFG_DIST_WORK_DOUBLES = 1024

STATUS_TEXT = {
    FFG_OK: "ok", FFG_INVALID_INPUT: "invalid input", FFG_CAPACITY: "capacity too small",
    FFG_BAD_HANDLE: "bad handle", FFG_CUDA_ERROR: "CUDA error", FFG_OUT_OF_MEMORY: "out of memory",
    FFG_NOT_CONVERGED: "not converged", FFG_TIMEOUT: "timeout", FFG_NO_DEVICE: "no CUDA device",
    FFG_NOT_READY: "not ready",
}


class SolverOptionsC(C.Structure):
    _fields_ = [("version", C.c_int), ("preconditioner", C.c_int), ("precision", C.c_int),
                ("tolerance_type", C.c_int), ("tolerance", C.c_double),
                ("max_iterations", C.c_int), ("max_refinements", C.c_int),
                ("inner_tolerance", C.c_double), ("verbosity", C.c_int),
                ("timeout_seconds", C.c_double), ("breakdown_guard", C.c_int)]


class SolverStatsC(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("refinements", C.c_int),
                ("status", C.c_int), ("final_residual", C.c_double),
                ("true_relative_residual", C.c_double), ("solve_seconds", C.c_double),
                ("assembly_seconds", C.c_double)]


class TuningC(C.Structure):
    _fields_ = [("element_threads", C.c_int), ("element_ctas_per_sm", C.c_int),
                ("column_threads", C.c_int), ("tc_ctas_per_sm", C.c_int), ("slice_cost", C.c_int),
                ("assembly_ms", C.c_double), ("default_assembly_ms", C.c_double),
                ("solve_ms", C.c_double), ("default_solve_ms", C.c_double)]


i32, i64, f64, vp = C.c_int, C.c_int64, C.c_double, C.c_void_p
pi32, pi64 = C.POINTER(C.c_int), C.POINTER(C.c_int64)

SIGNATURES = {
    "ffg_default_options": (None, [C.POINTER(SolverOptionsC)]),
    "ffg_version": (None, [pi32, pi32, pi32]),
    "ffg_device_count": (None, [pi32, pi32]),
    "ffg_structured_tetra_box_mesh": (None, [vp, vp, vp, vp, pi32]),
    "ffg_unit_square_mesh": (None, [i32, vp, vp, pi32]),
    "ffg_assemble_tetra_lagrange_stiffness_csc": (
        None, [i32, vp, i32, vp, i32, i32, i32, f64, f64, vp, vp, i64, pi32, pi64, vp, vp, vp, pi32]),
    "ffg_assemble_tetra_lagrange_stiffness_csc_jvp": (
        None, [i32, vp, i32, vp, i32, i32, i32, f64, f64, vp, f64, f64, i64, pi32, pi64, vp, vp,
               vp, pi32]),
    "ffg_assemble_tetra_lagrange_stiffness_csc_vjp": (
        None, [i32, vp, i32, vp, i32, i32, i32, f64, f64, i64, vp, vp, vp, vp, pi32]),
    "ffg_assemble_tetra_lagrange_scalar_load_samples": (
        None, [i32, vp, i32, vp, i32, i32, i32, vp, i32, vp, pi32]),
    "ffg_assemble_tetra_nedelec_curl_mass_csc": (
        None, [i32, vp, i32, vp, i32, f64, f64, vp, vp, i64, pi32, pi64, vp, vp, vp, pi32]),
    "ffg_assemble_tetra_nedelec_curl_mass_csc_jvp": (
        None, [i32, vp, i32, vp, i32, f64, f64, vp, f64, f64, i64, pi32, pi64, vp, vp, vp, pi32]),
    "ffg_assemble_tetra_nedelec_curl_mass_csc_vjp": (
        None, [i32, vp, i32, vp, i32, f64, f64, i64, vp, vp, vp, vp, pi32]),
    "ffg_assemble_tetra_nedelec_weighted_csc": (
        None, [i32, vp, i32, vp, i32, vp, f64, i64, pi32, pi64, vp, vp, vp, pi32]),
    "ffg_problem_set_cell_tensor": (None, [i32, vp, pi32]),
    "ffg_problem_set_assembly_precision": (None, [i32, i32, pi32]),
    "ffg_problem_autotune": (
        None, [i32, vp, f64, f64, vp, vp, vp, i32, C.POINTER(TuningC), pi32]),
    "ffg_problem_set_tuning": (None, [i32, C.POINTER(TuningC), pi32]),
    "ffg_assemble_tetra_nedelec_pml_csc": (
        None, [i32, vp, i32, vp, i32, vp, f64, i64, pi32, pi64, vp, vp, vp, pi32]),
    "ffg_assemble_tetra_nedelec_curvilinear_pml_csc": (
        None, [i32, vp, i32, vp, i32, vp, f64, i64, pi32, pi64, vp, vp, vp, pi32]),
    "ffg_problem_assemble": (
        None, [i32, vp, f64, f64, vp, vp, vp, vp, i32, vp, pi32]),
    "ffg_problem_sell_permutation": (None, [i32, vp, pi32]),
    "ffg_problem_system_arrays": (None, [i32, vp, vp, i32, vp, pi32]),
    "ffg_problem_sell_spmv": (None, [i32, vp, vp, vp, pi32]),
    "ffg_dist_start": (None, [i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, pi32]),
    "ffg_dist_update": (None, [i64, vp, f64, vp, vp, vp, vp, vp, vp, vp, vp, vp, pi32]),
    "ffg_dist_dot": (None, [i64, vp, vp, vp, vp, vp, vp, pi32]),
    "ffg_dist_direction": (None, [i64, vp, f64, vp, vp, vp, pi32]),
    "ffg_dist_cgs_dots": (None, [i64, vp, vp, vp, vp, vp, vp, vp, pi32]),
    "ffg_dist_cgs_update": (None, [i64, vp, f64, f64, vp, vp, vp, vp, vp, vp, vp, vp, pi32]),
    "ffg_dist_gather": (None, [i64, vp, vp, vp, vp, pi32]),
    "ffg_dist_scatter": (None, [i64, vp, vp, vp, vp, pi32]),
    "ffg_problem_evaluate": (
        None, [i32, vp, vp, i32, vp, vp, i32, vp, vp, vp, i32, vp, pi32]),
    "ffg_problem_probe": (
        None, [i32, vp, vp, i32, vp, i32, vp, vp, vp, i32, vp, pi32]),
    "ffg_assemble_tetra_nedelec_vector_load_samples": (
        None, [i32, vp, i32, vp, i32, vp, i32, vp, pi32]),
    "ffg_assemble_triangle_lagrange_csc": (
        None, [i32, vp, i32, vp, i32, i32, f64, f64, vp, vp, i64, pi32, pi64, vp, vp, vp, pi32]),
    "ffg_assemble_triangle_lagrange_load_samples": (
        None, [i32, vp, i32, vp, i32, i32, vp, i32, vp, pi32]),
    "ffg_assemble_scalar_p1_csc": (
        None, [i32, vp, i32, vp, f64, f64, vp, i64, pi64, vp, vp, vp, pi32]),
    "ffg_solve_sparse": (
        None, [i32, i64, vp, vp, vp, vp, vp, C.POINTER(SolverOptionsC), C.POINTER(SolverStatsC), pi32]),
    "ffg_csc_matvec": (None, [i32, i64, vp, vp, vp, vp, vp, pi32]),
    "ffg_solve_csr_device_noalloc": (
        None, [i32, i64, vp, vp, vp, vp, vp, C.POINTER(SolverOptionsC), C.POINTER(SolverStatsC),
               vp, pi32]),
    "ffg_build_topology": (
        None, [i32, i32, i32, i32, vp, i32, vp, i64, i64, pi64, pi64, pi64, vp, vp, vp, vp, pi32]),
    "ffg_problem_create": (
        None, [i32, i32, i32, i32, vp, i32, i32, i32, vp, pi32, pi64, pi64, pi64, pi32, pi32]),
    "ffg_problem_sample_points": (None, [i32, vp, vp, pi32]),
    "ffg_problem_dof_points": (None, [i32, vp, vp, pi32]),
    "ffg_problem_constrained": (None, [i32, vp, pi32]),
    "ffg_problem_topology": (None, [i32, vp, vp, vp, pi32]),
    "ffg_problem_solve": (
        None, [i32, vp, f64, f64, vp, vp, vp, vp, C.POINTER(SolverOptionsC), vp,
               C.POINTER(SolverStatsC), i32, vp, pi32]),
    "ffg_problem_reduced_system": (
        None, [i32, vp, f64, f64, vp, vp, vp, vp, i64, pi64, vp, vp, vp, vp, vp, pi32]),
    "ffg_problem_phase_times": (None, [i32, vp, pi32]),
    "ffg_problem_solve_batch": (
        None, [i32, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(SolverOptionsC), vp, i32, vp, pi32]),
    "ffg_problem_batch_stats": (None, [i32, C.POINTER(SolverStatsC), pi32]),
    "ffg_problem_free": (None, [i32, pi32]),
}

_lib = None


def load():
    """Load libfortfem_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing; build it with `python -m fortfem_b200.build` "
                "(nvcc, sm_100a).  There is no CPU fallback.")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def exported_symbols():
    return list(SIGNATURES)
