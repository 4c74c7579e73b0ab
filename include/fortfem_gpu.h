/*
 * fortfem_gpu.h -- C-ABI of libfortfem_gpu.so, the B200 (sm_100a) assembly +
 * preconditioned-CG path for lazy-fortran/fortfem.
 *
 * Conventions follow the reference's own C header (include/fortfem.h):
 *   - zero-based indices; vertices are [x0,y0,z0,x1,...] (the Fortran
 *     (3,n_vertices) array) and cells are [v0,v1,v2,v3,...];
 *   - CSC output arrays are caller-owned with a capacity: n_dofs and nnz are
 *     always set for valid input and status is FFG_CAPACITY (-2) when
 *     nnz_capacity is too small (fortfem.h:140-170);
 *   - every entry point ends with `int *status`; nothing aborts across the ABI;
 *   - device-resident objects are positive, process-local integer handles
 *     released by the matching *_free call (fortfem.h:186-197).
 * Host arrays are borrowed for the duration of a call.  Column pointers are
 * int64 so that matrices above 2^31 entries stay addressable.
 *
 * Each entry point cites the reference interface it replaces.  Reference
 * paths are relative to the lazy-fortran/fortfem tree.
 */
#ifndef FORTFEM_GPU_H
#define FORTFEM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: 0, -1, -2, -3 as in src/bindings/fortfem_capi_solver.f90:33-47. */
#define FFG_OK 0
#define FFG_INVALID_INPUT -1
#define FFG_CAPACITY -2
#define FFG_BAD_HANDLE -3
#define FFG_CUDA_ERROR -4
#define FFG_OUT_OF_MEMORY -5
#define FFG_NOT_CONVERGED -6
#define FFG_TIMEOUT -7
#define FFG_NO_DEVICE -8
#define FFG_NOT_READY -9  /* batched work still running on its stream */

/* Element families of a problem handle. */
#define FFG_TETRA_LAGRANGE 1
#define FFG_TETRA_NEDELEC 2
#define FFG_TRIANGLE_P1 3
#define FFG_TRIANGLE_LAGRANGE 4 /* arbitrary-order triangle Lagrange, degree 1..6 */

/* Quadrature rules: FFG_RULE_DUFFY uses tetra_duffy_quadrature(degree)
 * (src/quadrature/tetra_duffy_quadrature.f90:12-51); FFG_RULE_DEGREE_TWO is the
 * 4-point rule tetra_degree_two_quadrature (assembly_tetra_nedelec_3d.f90:2570-2581). */
#define FFG_RULE_DUFFY 0
#define FFG_RULE_DEGREE_TWO 1

/* Essential boundary handling of a problem handle. */
#define FFG_BOUNDARY_NONE 0 /* no constrained DoFs */
#define FFG_BOUNDARY_ALL 1  /* every DoF on an incidence-one face (Lagrange:
                               build_dirichlet_data, fortfem_tetra_lagrange_solver_3d.f90:551-610;
                               Nedelec: build_zero_tangential_mask,
                               fortfem_tetra_nedelec_solver_3d.f90:416-458;
                               P1: find_boundary vertices, mesh_2d.f90:560-603;
                               triangle Lagrange: every DoF on an edge of one triangle) */
#define FFG_BOUNDARY_MASK 2 /* caller-supplied uint8 mask over the global DoFs */

/* Solver precision. */
/* Element contraction of Nedelec problems (ffg_problem_set_assembly_precision) */
#define FFG_ASSEMBLY_FP64 0   /* FP64 CUDA-core contraction (the 1e-12 parity path) */
#define FFG_ASSEMBLY_TF32X3 1 /* 3xTF32 tensor-core contraction, FP32 accumulation (orders 3-6) */
#define FFG_PRECISION_FP64 0  /* FP64 Jacobi-PCG with the reference's stopping rule */
#define FFG_PRECISION_MIXED 1 /* FP32 PCG recurrences, FP64 solution and reliable
                                 FP64 residual updates (defect correction) */
#define FFG_PRECISION_MIXED16 2 /* as FFG_PRECISION_MIXED with the inner SpMV's operator
                                 * stored in FP16, each row scaled by its largest entry
                                 * (4 bytes an entry with the 16-bit column offset
                                 * instead of 6); the residual replacements still use
                                 * the FP64 operator, so the stopping rule is unchanged */

#define FFG_OPTIONS_VERSION 1

/* solver_options_t (src/solvers/advanced_solvers.f90:32-44) plus GPU fields. */
typedef struct {
  int version;           /* FFG_OPTIONS_VERSION */
  int preconditioner;    /* 0 = "none", 1 = "jacobi" */
  int precision;         /* FFG_PRECISION_FP64, _MIXED or _MIXED16 */
  int tolerance_type;    /* 0 = "relative", 1 = "absolute" */
  double tolerance;      /* FP64 mode: on the recursive residual as the reference;
                            mixed mode: on the true FP64 residual ||b-Ax|| (relative to ||b||) */
  int max_iterations;    /* cap on (inner) PCG iterations in total */
  int max_refinements;   /* mixed mode: cap on reliable updates (FP64 residual replacements) */
  double inner_tolerance;/* mixed mode: a reliable update replaces the FP32 recursive
                            residual by b - A x (FP64) whenever it has fallen by this
                            factor since the previous update (default 0.1) */
  int verbosity;         /* > 0 prints per-solve statistics on the host */
  double timeout_seconds;/* device-side wall limit of one solve; <= 0 selects 60 s */
  int breakdown_guard;   /* FP64 mode: 0 = the reference's |p^T A p| < 1e-14 test
                            (advanced_solvers.f90:897), 1 = stop only on p^T A p <= 0 */
} ffg_solver_options;

/* solver_stats_t (src/solvers/advanced_solvers.f90:47-57) plus GPU fields. */
typedef struct {
  int converged;
  int iterations;              /* PCG iterations (inner iterations summed in mixed mode) */
  int refinements;             /* reliable updates performed (mixed mode) */
  int status;                  /* FFG_* of the solve */
  double final_residual;       /* reference meaning: recursive residual 2-norm */
  double true_relative_residual; /* ||b - A x||_2 / ||b||_2 in FP64 at exit */
  double solve_seconds;        /* device time of the solve (CUDA events) */
  double assembly_seconds;     /* device time of assembly + load + reduction */
} ffg_solver_stats;

/* Fill opts with the library defaults (tolerance 1e-10, Jacobi, mixed). */
void ffg_default_options(ffg_solver_options *opts);

/* Library version and the number of visible CUDA devices. */
void ffg_version(int *major, int *minor, int *patch);
void ffg_device_count(int *count, int *status);

/* ------------------------------------------------------------------ meshes */

/* generate_structured_tetra_box_mesh, src/mesh/structured_tetra_box_mesh.f90:12-70.
 * bounds = [xmin,ymin,zmin,xmax,ymax,zmax]; vertices has 3*prod(counts+1)
 * entries and tetrahedra 4*6*prod(counts). */
void ffg_structured_tetra_box_mesh(const double *bounds, const int *counts, double *vertices,
                                   int *tetrahedra, int *status);

/* create_rectangular / unit_square_mesh(n), src/mesh/mesh_2d.f90:90-148 and
 * src/fortfem_api_mesh.f90:128-139: n vertices per side on [0,1]^2. */
void ffg_unit_square_mesh(int n, double *vertices, int *triangles, int *status);

/* ----------------------------------------------------- drop-in assembly */

/* assemble_tetra_lagrange_stiffness_csc,
 * src/assembly/assembly_tetra_lagrange_arbitrary_order_3d.f90:276-334.
 * cell_stiffness / cell_mass (nullable, n_tetrahedra entries) scale the scalar
 * coefficients cellwise as src/fortfem_forms_simple.f90:979-1045 does. */
void ffg_assemble_tetra_lagrange_stiffness_csc(
    int n_vertices, const double *vertices, int n_tetrahedra, const int *tetrahedra, int degree,
    int rule, int quadrature_degree, double stiffness_coefficient, double mass_coefficient,
    const double *cell_stiffness, const double *cell_mass, int64_t nnz_capacity, int *n_dofs,
    int64_t *nnz, int64_t *col_ptr, int *row_ind, double *values, int *status);

/* assemble_tetra_lagrange_stiffness_csc_jvp, same file :336-391: the tangent
 * of the stiffness + mass CSC along (vertices_dot, stiffness_dot, mass_dot),
 * on the primal matrix's pattern (col_ptr/row_ind as the primal call gives).
 * vertices_dot has the shape of vertices.  Capacity as the primal call. */
void ffg_assemble_tetra_lagrange_stiffness_csc_jvp(
    int n_vertices, const double *vertices, int n_tetrahedra, const int *tetrahedra, int degree,
    int rule, int quadrature_degree, double stiffness_coefficient, double mass_coefficient,
    const double *vertices_dot, double stiffness_coefficient_dot, double mass_coefficient_dot,
    int64_t nnz_capacity, int *n_dofs, int64_t *nnz, int64_t *col_ptr, int *row_ind,
    double *values_dot, int *status);

/* assemble_tetra_lagrange_stiffness_csc_vjp, same file :393-471: the adjoints
 * of the vertices (3*n_vertices), the stiffness and the mass coefficient for
 * a cotangent values_bar on the primal CSC pattern (nnz entries, nnz equal to
 * the primal matrix's, else FFG_INVALID_INPUT).  Outputs are zeroed first. */
void ffg_assemble_tetra_lagrange_stiffness_csc_vjp(
    int n_vertices, const double *vertices, int n_tetrahedra, const int *tetrahedra, int degree,
    int rule, int quadrature_degree, double stiffness_coefficient, double mass_coefficient,
    int64_t nnz, const double *values_bar, double *vertices_bar,
    double *stiffness_coefficient_bar, double *mass_coefficient_bar, int *status);

/* assemble_tetra_lagrange_scalar_load_samples, same file :473-528.
 * source_values holds n_q values per cell (n_q of the rule), cell-major. */
void ffg_assemble_tetra_lagrange_scalar_load_samples(
    int n_vertices, const double *vertices, int n_tetrahedra, const int *tetrahedra, int degree,
    int rule, int quadrature_degree, const double *source_values, int n_dofs, double *rhs,
    int *status);

/* assemble_tetra_nedelec_curl_mass_csc, src/assembly/assembly_tetra_nedelec_3d.f90:2042-2112
 * (order 1) and assemble_arbitrary_order_curl_mass_csc :2289-2355 (order >= 2). */
void ffg_assemble_tetra_nedelec_curl_mass_csc(
    int n_vertices, const double *vertices, int n_tetrahedra, const int *tetrahedra, int order,
    double curl_coefficient, double mass_coefficient, const double *cell_curl,
    const double *cell_mass, int64_t nnz_capacity, int *n_dofs, int64_t *nnz, int64_t *col_ptr,
    int *row_ind, double *values, int *status);

/* assemble_tetra_nedelec_curl_mass_csc_jvp, assembly_tetra_nedelec_3d.f90:2114-2181:
 * the tangent of the curl + mass CSC along (vertices_dot, curl_dot, mass_dot) on
 * the primal pattern.  The reference differentiates at quadrature degree 2k+2
 * where its primal uses 2k (order 1: the 4-point rule); both are exact for
 * these integrands, so the values agree to rounding. */
void ffg_assemble_tetra_nedelec_curl_mass_csc_jvp(
    int n_vertices, const double *vertices, int n_tetrahedra, const int *tetrahedra, int order,
    double curl_coefficient, double mass_coefficient, const double *vertices_dot,
    double curl_coefficient_dot, double mass_coefficient_dot, int64_t nnz_capacity, int *n_dofs,
    int64_t *nnz, int64_t *col_ptr, int *row_ind, double *values_dot, int *status);

/* assemble_tetra_nedelec_curl_mass_csc_vjp, same file :2183-2287: vertex, curl
 * and mass adjoints of a cotangent on the primal CSC pattern (nnz entries).
 * Outputs are zeroed first. */
void ffg_assemble_tetra_nedelec_curl_mass_csc_vjp(
    int n_vertices, const double *vertices, int n_tetrahedra, const int *tetrahedra, int order,
    double curl_coefficient, double mass_coefficient, int64_t nnz, const double *values_bar,
    double *vertices_bar, double *curl_coefficient_bar, double *mass_coefficient_bar,
    int *status);

/* assemble_tetra_nedelec_weighted_csc / assemble_arbitrary_order_weighted_csc,
 * assembly_tetra_nedelec_3d.f90:1870-1931 / :1933-2000 (elements :2406-2514):
 * curl M curl + mass_coefficient I with a tensor coefficient M.  A GPU
 * cannot call the reference's Fortran callback (tensor_coefficient_3d,
 * :56-60), so the caller evaluates it once per cell (at the centroid) and
 * declares it constant on each cell: cell_tensors holds 9 doubles per
 * tetrahedron, the column-major 3 x 3 tensor (Fortran value(3,3)).  The
 * tensors must be symmetric (to 1e-12 of their largest entry) and finite,
 * else FFG_INVALID_INPUT.  The reference integrates at degree 2k+2 (order 1:
 * the 4-point rule); the contraction used here is exact for a constant
 * tensor.  Capacity / query protocol as the other CSC entries. */
void ffg_assemble_tetra_nedelec_weighted_csc(int n_vertices, const double *vertices,
                                             int n_tetrahedra, const int *tetrahedra, int order,
                                             const double *cell_tensors, double mass_coefficient,
                                             int64_t nnz_capacity, int *n_dofs, int64_t *nnz,
                                             int64_t *col_ptr, int *row_ind, double *values,
                                             int *status);

/* assemble_tetra_nedelec_pml_csc, assembly_tetra_nedelec_3d.f90:1613-1685 (element
 * :826-887): the complex curl-curl minus k^2 mass operator with the Cartesian PML
 * tensors of cartesian_curl_curl_pml_coefficients (src/boundary/cartesian_helmholtz_pml.f90:94-108).
 * stretch: 3 complex values per tetrahedron as (re, im) pairs (6 doubles per
 * cell); values: nnz complex entries as (re, im) pairs (2 * nnz doubles, the
 * layout of C99 double complex and of Fortran complex(dp), csc_z_t%val).
 * The reference integrates at degree 2k+2, the primal curl-mass at 2k (order 1:
 * the 4-point rule); both are exact for these integrands. */
void ffg_assemble_tetra_nedelec_pml_csc(int n_vertices, const double *vertices, int n_tetrahedra,
                                        const int *tetrahedra, int order, const double *stretch,
                                        double wave_number, int64_t nnz_capacity, int *n_dofs,
                                        int64_t *nnz, int64_t *col_ptr, int *row_ind,
                                        double *values, int *status);

/* assemble_tetra_nedelec_curvilinear_pml_csc, same file :1372-1444 (element
 * :1092-1153), tensors of curvilinear_curl_curl_pml_coefficients
 * (src/boundary/curvilinear_helmholtz_pml.f90:113-131): stretch is a complex
 * 3x3 matrix per tetrahedron, column-major as the Fortran stretch(:, :, t),
 * (re, im) pairs (18 doubles per cell). */
void ffg_assemble_tetra_nedelec_curvilinear_pml_csc(int n_vertices, const double *vertices,
                                                    int n_tetrahedra, const int *tetrahedra,
                                                    int order, const double *stretch,
                                                    double wave_number, int64_t nnz_capacity,
                                                    int *n_dofs, int64_t *nnz, int64_t *col_ptr,
                                                    int *row_ind, double *values, int *status);

/* assemble_tetra_nedelec_vector_load_samples, assembly_tetra_nedelec_3d.f90:128-185
 * (order 1 uses the 4-point rule and edge signs, :2002-2040); source_values
 * holds 3*n_q values per cell. */
void ffg_assemble_tetra_nedelec_vector_load_samples(
    int n_vertices, const double *vertices, int n_tetrahedra, const int *tetrahedra, int order,
    const double *source_values, int n_dofs, double *rhs, int *status);

/* kappa grad u . grad v + m u v on arbitrary-order triangle Lagrange elements
 * (degree 1..6) in CSC.  The reference has the basis
 * (src/elements/triangle_lagrange_arbitrary_order.f90:29-127: Bernstein
 * polynomials made nodal by their inverse Vandermonde matrix) but no assembly
 * routine for it; this one follows its tetrahedral Lagrange assembly
 * (assembly_tetra_lagrange_arbitrary_order_3d.f90:40-105, 276-334) with the
 * triangle Duffy rule of quadrature_degree
 * (src/quadrature/triangle_duffy_quadrature.f90:12-45), |det J| as the area
 * factor, and the first-appearance DoF numbering of the tetrahedral map
 * (tetra_lagrange_global_dof_map.f90:13-99) on triangles.  vertices are
 * [x0,y0,x1,...]; cell_* nullable as above. */
void ffg_assemble_triangle_lagrange_csc(int n_vertices, const double *vertices, int n_triangles,
                                        const int *triangles, int degree, int quadrature_degree,
                                        double stiffness_coefficient, double mass_coefficient,
                                        const double *cell_stiffness, const double *cell_mass,
                                        int64_t nnz_capacity, int *n_dofs, int64_t *nnz,
                                        int64_t *col_ptr, int *row_ind, double *values,
                                        int *status);

/* The load sum_q w_q |det J| f_q phi_i of the same elements; source_values
 * holds n_q samples per triangle (the rule's points, cell-major). */
void ffg_assemble_triangle_lagrange_load_samples(int n_vertices, const double *vertices,
                                                 int n_triangles, const int *triangles,
                                                 int degree, int quadrature_degree,
                                                 const double *source_values, int n_dofs,
                                                 double *rhs, int *status);

/* assemble_scalar_p1_matrix / assemble_scalar_p1_load scattered into CSC,
 * src/fortfem_forms_simple.f90:1678-1761 (the reference builds it dense). */
void ffg_assemble_scalar_p1_csc(int n_vertices, const double *vertices, int n_triangles,
                                const int *triangles, double mass_coefficient,
                                double stiffness_coefficient, const double *cell_stiffness,
                                int64_t nnz_capacity, int64_t *nnz, int64_t *col_ptr,
                                int *row_ind, double *values, int *status);

/* ------------------------------------------------------------------ solve */

/* solve_sparse(A, b, x, opts, stats), src/solvers/advanced_solvers.f90:135-195, with
 * method "pcg": square zero-based CSC in host memory; x is the initial guess
 * on entry and the solution on exit. */
void ffg_solve_sparse(int n, int64_t nnz, const int64_t *col_ptr, const int *row_ind,
                      const double *values, const double *b, double *x,
                      const ffg_solver_options *opts, ffg_solver_stats *stats, int *status);

/* y = A x for a host CSC matrix (spmv / csc_matvec, src/solvers/fortfem_sparse_matrix.f90:46-58). */
void ffg_csc_matvec(int n, int64_t nnz, const int64_t *col_ptr, const int *row_ind,
                    const double *values, const double *x, double *y, int *status);

/* No counterpart in the reference.  FP64 Jacobi-PCG (the FP64 mode of
 * ffg_solve_sparse) on a matrix already in device memory, for callers that
 * may not allocate device memory: codes that own all of the GPU's memory in
 * their own arena, and solve loops that cannot let cudaFree synchronise the
 * device.  It calls no cudaMalloc or cudaFree; its work vectors live in one
 * fixed device array that holds systems of up to FFG_NOALLOC_MAX_ROWS rows
 * (larger n returns FFG_CAPACITY).  row_ptr (n+1), col_ind and values
 * (nnz) are a zero-based CSR matrix in device memory; a symmetric matrix's
 * CSC arrays serve unchanged.  b and x are device vectors, x holding the
 * initial guess on entry and the solution on exit.  opts as ffg_solve_sparse,
 * except that precision is always FP64.  The work runs on `stream` (a
 * cudaStream_t, 0 = default); every call synchronises `stream` before it
 * returns, since it reads its result block back to the host.  The kernel
 * checks the CSR arrays before any indexed access (row_ptr from 0 to nnz,
 * never decreasing; column indices in [0, n)) and a malformed matrix returns
 * FFG_INVALID_INPUT.  The first call with a device current looks up the
 * array's address on that device, so it should come before any stream
 * capture.  All calls share the array: calls whose work overlaps on one GPU
 * race, so serialise them. */
#define FFG_NOALLOC_MAX_ROWS 65536
void ffg_solve_csr_device_noalloc(int n, int64_t nnz, const int64_t *row_ptr,
                                  const int *col_ind, const double *values, const double *b,
                                  double *x, const ffg_solver_options *opts,
                                  ffg_solver_stats *stats, void *stream, int *status);

/* Host-only topology of a problem (no device needed): the global DoF of every
 * local DoF (build_tetra_lagrange_dof_map, tetra_lagrange_global_dof_map.f90:13-79;
 * build_tetra_nedelec_dof_map, tetra_nedelec_global_dof_map.f90:15-105), the
 * constrained mask of boundary_mode and the CSC pattern of the constrained
 * (free x free) system.  Arrays are caller-owned; pass nnz_capacity = 0 and
 * null arrays to query n_dofs and nnz (status FFG_CAPACITY). */
void ffg_build_topology(int family, int degree, int n_vertices, int n_cells, const int *cells,
                        int boundary_mode, const uint8_t *boundary_mask, int64_t dof_capacity,
                        int64_t nnz_capacity, int64_t *n_dofs, int64_t *n_free, int64_t *nnz,
                        int *global_dofs, uint8_t *constrained, int64_t *col_ptr, int *row_ind,
                        int *status);

/* ------------------------------------------------ device-resident problems */

/* Build the topology of an assemble + constrain + solve problem once per mesh
 * (DoF numbering in the reference's first-appearance order, the CSC pattern,
 * the constrained set and the element-to-CSC slot maps) and keep it in HBM.
 * family: FFG_TETRA_LAGRANGE (degree 1..4), FFG_TETRA_NEDELEC (order 1..6) or
 * FFG_TRIANGLE_P1 (degree 1; vertices are then 2-D).  For Lagrange the rule
 * and quadrature degree select the element and load quadrature; Nedelec uses
 * the reference rules (order 1: the 4-point rule; order k >= 2: Duffy 2k for
 * the matrix and 2k+2 for the load).  boundary_mask is read only for
 * FFG_BOUNDARY_MASK.  Returns the global DoF count, the free DoF count, the
 * nonzeros of the constrained (free x free) system and the number of load
 * samples per cell. */
void ffg_problem_create(int family, int degree, int n_vertices, int n_cells, const int *cells,
                        int rule, int quadrature_degree, int boundary_mode,
                        const uint8_t *boundary_mask, int *handle, int64_t *n_dofs,
                        int64_t *n_free, int64_t *nnz, int *samples_per_cell, int *status);

/* Physical sample points (3 * samples_per_cell * n_cells doubles, cell-major)
 * at which the caller evaluates its source; 2-D meshes return (x, y, 0). */
void ffg_problem_sample_points(int handle, const double *vertices, double *points, int *status);

/* Physical location of every global DoF that carries a nodal value (Lagrange,
 * P1): 3 * n_dofs doubles.  Callers evaluate boundary_value there. */
void ffg_problem_dof_points(int handle, const double *vertices, double *points, int *status);

/* The DoF map of the problem, as ffg_build_topology returns it for the host
 * build: global_dofs (n_cells x n_b, the reference's first-appearance
 * numbering) and, for Nedelec, edge_sign (6 per cell: +1 when the local edge
 * runs from the smaller to the larger global vertex, as
 * build_tetra_edge_dof_map, tetra_edge_dof_map.f90:54-60) and face_perm (4
 * per cell: index 0..5 of the local face vertices' ranks 123, 132, 213, 231,
 * 312, 321, the face permutations of build_tetra_nedelec_dof_map,
 * tetra_nedelec_global_dof_map.f90:68-90).  Null arrays are skipped. */
void ffg_problem_topology(int handle, int *global_dofs, int8_t *edge_sign, uint8_t *face_perm,
                          int *status);

/* The constrained mask of the problem (n_dofs bytes, 1 = constrained). */
void ffg_problem_constrained(int handle, uint8_t *mask, int *status);

/* Launch shapes of a problem's kernels and the times that chose them.  Zero
 * shape fields mean the built-in default. */
typedef struct {
  int element_threads;     /* Nedelec FP64 element kernels: threads per CTA (256) */
  int element_ctas_per_sm; /* the matrix kernel's grid target in CTAs per SM (the
                              entry range of a cell tile is split to reach it) */
  int column_threads;      /* column-owner gather: threads per block */
  int tc_ctas_per_sm;      /* 3xTF32 tensor-core kernel: CTAs per SM (1 or 2) */
  int slice_cost;          /* PCG work partition: cost of a slice beyond its entries */
  double assembly_ms;         /* best assembly time measured (device-resident inputs) */
  double default_assembly_ms; /* the built-in defaults, same measurement */
  double solve_ms;            /* best time of a fixed 60-iteration mixed PCG run */
  double default_solve_ms;    /* the built-in partition, same run */
} ffg_tuning;

/* No counterpart in the reference (whose loops have no launch shapes).
 * Chooses the problem's launch shapes by measurement on its own inputs (as
 * ffg_problem_solve takes them): the element matrix kernel's grid (Nedelec
 * FP64) or the tensor-core kernel's CTAs per SM (3xTF32), the column
 * gather's block size, then the PCG work partition's slice cost, each
 * candidate timed with CUDA events (best of three) and the fastest kept for
 * every following assembly and solve of the problem.  Results of assembly and
 * solve do not depend on the shapes except through the CTA partition of the
 * PCG dot products (reduced in a fixed order for a given partition).  Fills
 * `tuning` with the choice and the times. */
void ffg_problem_autotune(int handle, const double *vertices, double coef_a, double coef_b,
                          const double *cell_a, const double *cell_b, const double *samples,
                          int memory, ffg_tuning *tuning, int *status);
/* Apply launch shapes (from an earlier ffg_problem_autotune, possibly of
 * another process); the time fields are ignored. */
void ffg_problem_set_tuning(int handle, const ffg_tuning *tuning, int *status);

/* Nedelec problems of orders 3 to 6: how the element matrices are contracted
 * in every following assembly.  FFG_ASSEMBLY_FP64 (the default) is the FP64
 * oriented reference-tensor contraction on CUDA cores, equal to the
 * reference's quadrature loop (assemble_tetra_nedelec_curl_mass_element,
 * assembly_tetra_nedelec_3d.f90:584-643) to 1e-12.  FFG_ASSEMBLY_TF32X3 runs
 * the contraction as a GEMM on the tensor cores (tcgen05, TF32 hi/lo operand
 * split, three products accumulated in FP32) against the same oriented
 * tensors: entries carry about 1e-7 relative error, the geometry and the
 * loads stay FP64.
 * Other orders and families return FFG_INVALID_INPUT. */
void ffg_problem_set_assembly_precision(int handle, int precision, int *status);

/* Nedelec problems: a symmetric 3 x 3 tensor per cell (9 doubles, column-major,
 * host array) that replaces the scalar curl coefficient's unit tensor in every
 * following assembly of this problem (solve, reduced system, batch): the curl
 * term becomes curl . (curl_coefficient cell_curl[c] M_c) curl, as
 * solve_tetra_nedelec_weighted_curl_mass (src/solvers/fortfem_tetra_nedelec_solver_3d.f90:41-95)
 * with a cellwise-constant tensor callback.  NULL clears it.  Non-symmetric or
 * non-finite tensors return FFG_INVALID_INPUT. */
void ffg_problem_set_cell_tensor(int handle, const double *cell_tensors, int *status);

/* Assemble the constrained system on the device and solve it:
 *   K(c) x = F(f) on the free DoFs, x = g on the constrained DoFs,
 * with K = coef_a * cell_a[c] * (stiffness | curl-curl) + coef_b * cell_b[c] * mass
 * (cell arrays nullable), F from source samples (samples_per_cell values per
 * cell for scalar families, 3 * samples_per_cell for Nedelec) and the lifting
 * -A_fc g of sparse_direct_solve_constrained_real
 * (src/solvers/fortfem_sparse_direct.f90:264-344).  constrained_values
 * (nullable = zero) has n_dofs entries.  memory = 0: all pointers are host
 * memory (synchronous, host<->device copies inside); memory = 1: vertices,
 * cell arrays, samples, constrained_values and solution are device pointers
 * and the call is asynchronous on `stream` (a cudaStream_t) except for the
 * statistics, which are read back at the end.  solution has n_dofs entries. */
void ffg_problem_solve(int handle, const double *vertices, double coef_a, double coef_b,
                       const double *cell_a, const double *cell_b, const double *source_samples,
                       const double *constrained_values, const ffg_solver_options *opts,
                       double *solution, ffg_solver_stats *stats, int memory, void *stream,
                       int *status);

/* Assemble only and return the constrained (free x free) CSC matrix, its
 * lifted right-hand side and the free-DoF list (host memory, capacity rules
 * as above).  This is the reduced system the solve works on. */
void ffg_problem_reduced_system(int handle, const double *vertices, double coef_a, double coef_b,
                                const double *cell_a, const double *cell_b,
                                const double *source_samples, const double *constrained_values,
                                int64_t nnz_capacity, int64_t *nnz, int64_t *col_ptr, int *row_ind,
                                double *values, double *rhs, int *free_dofs, int *status);

/* Device-side profile of the handle's last solve, measured by CTA 0 of the
 * persistent PCG kernel: seconds[0] = 1 if the mixed solve continued in FP64
 * after FP32 stagnation, then seconds in SpMV work, barrier wait after the
 * SpMV, vector work, barrier wait after it, and residual-replacement phases. */
void ffg_problem_phase_times(int handle, double *seconds, int *status);

/* ------------------------------------------------------------ serving */

/* No counterpart in the reference (its solves run one at a time on the CPU).
 * Enqueue assembly and solve of `count` distinct device-resident problems on
 * `stream` and return without waiting, so that a serving loop can keep
 * several batches in flight.  Arguments are those of ffg_problem_solve with
 * memory = 1 (device pointers), one entry per problem: coef_a and coef_b hold
 * `count` values, the other per-problem arrays hold `count` pointers (the
 * arrays cell_a, cell_b, source_samples, constrained_values may be null, as
 * may their entries).  mode FFG_BATCH_CTA_PER_SYSTEM solves every system on
 * one thread block of its own in a single launch (for many small systems;
 * a system's result does not depend on the rest of the batch);
 * FFG_BATCH_WHOLE_DEVICE solves them one after another on the whole GPU (for
 * large systems); FFG_BATCH_CTA_GROUPS solves them side by side in shared
 * cooperative launches, each system on a group of thread blocks sized by its
 * row count alone (16384 rows per block, at least 2, at most one per SM), so
 * that mid-size systems, whose iterations are bound by the grid barrier
 * rather than by bandwidth, share the GPU while a system's result still does
 * not depend on the rest of the batch.  A problem may belong to one
 * unfinished batch at a time. */
#define FFG_BATCH_CTA_PER_SYSTEM 0
#define FFG_BATCH_WHOLE_DEVICE 1
#define FFG_BATCH_CTA_GROUPS 2
void ffg_problem_solve_batch(int count, const int *handles, const double *const *vertices,
                             const double *coef_a, const double *coef_b,
                             const double *const *cell_a, const double *const *cell_b,
                             const double *const *source_samples,
                             const double *const *constrained_values,
                             const ffg_solver_options *opts, double *const *solutions, int mode,
                             void *stream, int *status);

/* Statistics of a problem's last batched solve: FFG_NOT_READY while the
 * stream has not reached the end of its batch; otherwise the solve's status
 * (assembly_seconds: its own assembly; solve_seconds: from the end of its
 * assembly to the end of the batch's solve). */
void ffg_problem_batch_stats(int handle, ffg_solver_stats *stats, int *status);

/* ------------------------------------------------- evaluation and probes */

#define FFG_POINT_REFERENCE 0 /* points are reference coordinates of the query's cell */
#define FFG_POINT_PHYSICAL 1  /* physical points, mapped back by the cell's inverse
                                 Jacobian (invert_tetra_affine_map,
                                 src/geometry/tetra_affine_map.f90:15-33) */
#define FFG_PROBE_AVERAGE 0   /* mean over every containing cell, in cell order */
#define FFG_PROBE_FIRST 1     /* the first containing cell */

/* Batched solution evaluation on a problem's mesh (tetrahedral families).
 * Lagrange: evaluate_tetra_lagrange_solution_prepared and _at_point
 * (src/solvers/fortfem_tetra_lagrange_solver_3d.f90:491-528, :305-325) -
 * values[q] and the physical gradient derivatives[3q..3q+2]; the call fails
 * with FFG_INVALID_INPUT when a cell of the mesh is degenerate, as the
 * reference's evaluator initialisation does (:437-489).  Nedelec: the field
 * values[3q..] and curl derivatives[3q..] of the oriented local DoFs on the
 * query's cell (the per-cell evaluation of evaluate_box_solution_order,
 * src/solvers/fortfem_magnetic_box_3d.f90:313-334).  solution holds n_dofs
 * entries (all DoFs, as ffg_problem_solve returns them).  query_status
 * (nullable) receives 0, or FFG_INVALID_INPUT for a cell index out of range,
 * a degenerate cell or a point outside the reference cell (the basis
 * evaluation's -64 eps test).  memory = 1: every array is device memory and
 * the work runs on `stream`; the call returns when it is done. */
void ffg_problem_evaluate(int handle, const double *vertices, const double *solution,
                          int n_queries, const int *cells, const double *points, int point_kind,
                          double *values, double *derivatives, int *query_status, int memory,
                          void *stream, int *status);

/* Point probes without a cell hint: evaluate_box_solution_order
 * (fortfem_magnetic_box_3d.f90:269-343, FFG_PROBE_AVERAGE) and probe_box_az /
 * probe_box_curl (:345-440, FFG_PROBE_FIRST).  A cell contains a point when
 * det > 0 and the point's reference coordinates are >= -1e-12 with sum <=
 * 1 + 1e-12.  Outputs as ffg_problem_evaluate; counts[q] is the number of
 * cells that contributed (0: the point lies in no cell, values zero; -1: the
 * basis evaluation rejected it on a containing cell, where the reference's
 * probe fails).  Lagrange problems are probed the same way. */
void ffg_problem_probe(int handle, const double *vertices, const double *solution, int n_points,
                       const double *points, int mode, double *values, double *derivatives,
                       int *counts, int memory, void *stream, int *status);

/* ------------------------------------------- one system over several GPUs */

/* No counterpart in the reference (its solve is serial).  Building blocks of
 * the row-block Jacobi-PCG that solves one system sharded over several GPUs
 * (fortfem_b200/sharding.py): every rank owns a set of rows, assembles the
 * cells that touch them (a ghost layer included) as its own problem, and the
 * host loop exchanges the search direction of the ghost rows and all-reduces
 * the dot products between these launches.  Vectors live in device memory in
 * the SELL row order of the rank's problem (ffg_problem_sell_permutation);
 * `owned` (uint8, one per row) selects the rows whose dot products count. */

/* Assemble the constrained system into the problem's device operator and
 * right-hand side without solving (arguments as ffg_problem_solve). */
void ffg_problem_assemble(int handle, const double *vertices, double coef_a, double coef_b,
                          const double *cell_a, const double *cell_b, const double *source_samples,
                          const double *constrained_values, int memory, void *stream, int *status);

/* perm[i] = free-DoF index (position in ffg_build_topology's free list) of
 * SELL row i; n_free entries, host memory. */
void ffg_problem_sell_permutation(int handle, int *perm, int *status);

/* Copy the assembled right-hand side and the Jacobi inverse diagonal (SELL
 * order, n_free each; either pointer may be null) to host (memory = 0) or
 * device (memory = 1) arrays. */
void ffg_problem_system_arrays(int handle, double *rhs, double *dinv, int memory, void *stream,
                               int *status);

/* y = A x with the assembled FP64 operator, device vectors in SELL order. */
void ffg_problem_sell_spmv(int handle, const double *x, double *y, void *stream, int *status);

/* Device work array for the reductions below: FFG_DIST_WORK_DOUBLES doubles. */
#define FFG_DIST_WORK_DOUBLES 1024

/* r = b - ax, z = D^-1 r, p = z on owned rows; dots (device, 3) = (r,r), (r,z), (b,b)
 * over owned rows, summed in a fixed order. */
void ffg_dist_start(int64_t n, const uint8_t *owned, const double *b, const double *ax,
                    const double *dinv, double *r, double *z, double *p, double *work,
                    double *dots, void *stream, int *status);

/* x += alpha p, r -= alpha q, z = D^-1 r on owned rows; dots (device, 2) = (r,r), (r,z). */
void ffg_dist_update(int64_t n, const uint8_t *owned, double alpha, const double *p,
                     const double *q, const double *dinv, double *x, double *r, double *z,
                     double *work, double *dots, void *stream, int *status);

/* dot (device, 1) = (a, b) over owned rows. */
void ffg_dist_dot(int64_t n, const uint8_t *owned, const double *a, const double *b,
                  double *work, double *dot, void *stream, int *status);

/* p = z + beta p on owned rows. */
void ffg_dist_direction(int64_t n, const uint8_t *owned, double beta, const double *z, double *p,
                        void *stream, int *status);

/* Single-reduction form of the same iteration (Chronopoulos-Gear PCG, one
 * all-reduce per iteration): dots (device, 3) = (r, z), (w, z), (r, r) over
 * owned rows with w = A z; then p = z + beta p, s = w + beta s, x += alpha p,
 * r -= alpha s, z = D^-1 r on owned rows. */
void ffg_dist_cgs_dots(int64_t n, const uint8_t *owned, const double *r, const double *z,
                       const double *w, double *work, double *dots, void *stream, int *status);
void ffg_dist_cgs_update(int64_t n, const uint8_t *owned, double alpha, double beta,
                         const double *w, const double *dinv, double *p, double *s, double *x,
                         double *r, double *z, void *stream, int *status);

/* dst[i] = src[idx[i]] (pack a halo) and dst[idx[i]] = src[i] (unpack), i < m. */
void ffg_dist_gather(int64_t m, const int *idx, const double *src, double *dst, void *stream,
                     int *status);
void ffg_dist_scatter(int64_t m, const int *idx, const double *src, double *dst, void *stream,
                      int *status);

/* Release a problem handle (fortfem_factor_free, src/bindings/fortfem_capi_solver.f90:108-124). */
void ffg_problem_free(int handle, int *status);

#ifdef __cplusplus
}
#endif
#endif
