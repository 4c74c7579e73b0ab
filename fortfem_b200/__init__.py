"""fortfem_b200: the B200 (sm_100a) assembly + preconditioned-CG path of
lazy-fortran/fortfem behind fortfem's own entry points.

Everything here calls libfortfem_gpu.so through its C-ABI
(include/fortfem_gpu.h); importing an entry point that needs the library
raises when it has not been built (``python -m fortfem_b200.build``).
"""
from ._capi import (FFG_BOUNDARY_ALL, FFG_BOUNDARY_MASK, FFG_BOUNDARY_NONE, FFG_RULE_DEGREE_TWO,
                    FFG_RULE_DUFFY, FFG_TETRA_LAGRANGE, FFG_TETRA_NEDELEC,
                    FFG_TRIANGLE_LAGRANGE, FFG_TRIANGLE_P1)
from .api import (CscMatrix, FortfemError, Problem, SolverOptions, SolverStats, Status,
                  assemble_scalar_p1_csc, assemble_tetra_lagrange_scalar_load_samples,
                  assemble_tetra_lagrange_stiffness_csc, assemble_tetra_lagrange_stiffness_csc_jvp,
                  assemble_tetra_lagrange_stiffness_csc_vjp, assemble_tetra_nedelec_curl_mass_csc,
                  assemble_tetra_nedelec_curl_mass_csc_jvp, assemble_tetra_nedelec_curl_mass_csc_vjp,
                  assemble_tetra_nedelec_curvilinear_pml_csc, assemble_tetra_nedelec_pml_csc,
                  assemble_tetra_nedelec_vector_load_samples,
                  assemble_tetra_nedelec_weighted_csc, assemble_triangle_lagrange_csc,
                  assemble_triangle_lagrange_load_samples, build_topology,
                  evaluate_tetra_lagrange_solution, probe_tetra_nedelec_solution,
                  generate_structured_tetra_box_mesh, solve_scalar_p1, solve_sparse,
                  solve_tetra_lagrange_diffusion_reaction, solve_tetra_lagrange_poisson,
                  solve_tetra_nedelec_curl_mass, solve_tetra_nedelec_weighted_curl_mass,
                  solve_triangle_lagrange, solver_options, spmv, cell_tensors,
                  unit_square_mesh)

__all__ = [n for n in dir() if not n.startswith("_")]
