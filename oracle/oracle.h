/*
 * fortfem hot-path ORACLE — test infrastructure only.
 *
 * A plain FP64, single-threaded CPU restatement of the reference algorithms on
 * the assembly + Krylov path of lazy-fortran/fortfem.  Each function names the
 * reference file:line it follows.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU legs may load this library, and only as the checker or as the
 * timed CPU baseline; the product (fortfem_b200, libfortfem_gpu.so) never
 * links, imports or calls it.
 *
 * Conventions: zero-based indices; vertices are [x0,y0,z0,x1,...] (the
 * reference's column-major (3,n) array); tetrahedra are [v0,v1,v2,v3,...];
 * element matrices are column-major n_b x n_b like the reference's Fortran
 * arrays.  Every function returns 0 on success and a non-zero status on the
 * inputs the reference rejects.
 */
#ifndef FORTFEM_ORACLE_H
#define FORTFEM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- quadrature ---- */
int or_gauss_legendre(int n, double a, double b, double *nodes, double *weights);
int or_tetra_duffy_count(int polynomial_degree);
int or_tetra_duffy(int polynomial_degree, double *x, double *y, double *z, double *w);
int or_triangle_duffy_count(int polynomial_degree);
int or_triangle_duffy(int polynomial_degree, double *x, double *y, double *w);
void or_tetra_degree_two_rule(double *points /*3x4*/, double *weights /*4*/);

/* ---- meshes ---- */
int or_structured_tetra_box_mesh(const double *bounds /*xmin,ymin,zmin,xmax,ymax,zmax*/,
                                 const int *counts, double *vertices, int *tetrahedra);
int or_unit_square_mesh(int n, double *vertices, int *triangles);
int or_square_boundary_vertices(int n_vertices, int n_triangles, const int *triangles,
                                uint8_t *is_boundary);

/* ---- tetrahedral Lagrange ---- */
int or_lagrange_dof_count(int degree);
int or_lagrange_barycentric_indices(int degree, int *indices /*4 x n_b*/, double *nodes /*3 x n_b*/);
int or_lagrange_evaluate(int degree, const double *point, double *values, double *gradients);
int or_lagrange_dof_map_faithful(int degree, int n_tets, const int *tets, int *global_dofs, int *n_global);
int or_lagrange_dof_map(int degree, int n_tets, const int *tets, int *global_dofs, int *n_global);
/* rule: 0 = Duffy(quadrature_degree), 1 = the 4-point degree-two rule */
int or_lagrange_element(const double *vertices /*3x4*/, int degree, int rule, int quadrature_degree,
                        double stiffness, double mass, double *matrix);
int64_t or_lagrange_csc_nnz(int degree, int n_tets, const int *tets);
int or_lagrange_csc(int n_vertices, const double *vertices, int n_tets, const int *tets, int degree,
                    int rule, int quadrature_degree, double stiffness, double mass,
                    const double *cell_stiffness, const double *cell_mass,
                    int64_t nnz_capacity, int *n_dofs, int64_t *nnz, int64_t *col_ptr,
                    int *row_idx, double *values);
/* forward (JVP) and reverse (VJP) mode of the element and the CSC assembly */
int or_lagrange_element_jvp(const double *vertices, int degree, int rule, int quadrature_degree,
                            double stiffness, double mass, const double *vertices_dot,
                            double stiffness_dot, double mass_dot, double *matrix_dot);
int or_lagrange_element_vjp(const double *vertices, int degree, int rule, int quadrature_degree,
                            double stiffness, double mass, const double *matrix_bar,
                            double *vertices_bar, double *stiffness_bar, double *mass_bar);
int or_lagrange_csc_jvp(int n_vertices, const double *vertices, int n_tets, const int *tets,
                        int degree, int rule, int quadrature_degree, double stiffness, double mass,
                        const double *vertices_dot, double stiffness_dot, double mass_dot,
                        int64_t nnz_capacity, int *n_dofs, int64_t *nnz, int64_t *col_ptr,
                        int *row_idx, double *values_dot);
int or_lagrange_csc_vjp(int n_vertices, const double *vertices, int n_tets, const int *tets,
                        int degree, int rule, int quadrature_degree, double stiffness, double mass,
                        int64_t nnz, const double *values_bar, double *vertices_bar,
                        double *stiffness_bar, double *mass_bar);
int or_lagrange_load_samples(int n_vertices, const double *vertices, int n_tets, const int *tets,
                             int degree, int rule, int quadrature_degree,
                             const double *source_values /* n_q x T */, double *rhs);
int or_lagrange_quadrature_points(int n_vertices, const double *vertices, int n_tets, const int *tets,
                                  int rule, int quadrature_degree, double *points /*3 x n_q x T*/);
int or_lagrange_dirichlet_faithful(int degree, int n_vertices, const double *vertices, int n_tets,
                                   const int *tets, uint8_t *constrained, double *node_points);
int or_lagrange_dirichlet(int degree, int n_vertices, const double *vertices, int n_tets,
                          const int *tets, uint8_t *constrained, double *node_points);

/* ---- solution probes (evaluation at reference / physical points, point location) ---- */
int or_lagrange_evaluate_solution(int n_vertices, const double *vertices, int n_tets,
                                  const int *tets, int degree, int n_dofs, const double *solution,
                                  int cell, const double *reference_point, double *value,
                                  double *gradient);
int or_lagrange_evaluate_solution_at_point(int n_vertices, const double *vertices, int n_tets,
                                           const int *tets, int degree, int n_dofs,
                                           const double *solution, int cell, const double *point,
                                           double *value, double *gradient);
/* mode 0: average over every containing cell; 1: the first containing cell */
int or_lagrange_probe(int n_vertices, const double *vertices, int n_tets, const int *tets,
                      int degree, int n_dofs, const double *solution, const double *point,
                      int mode, double *value, double *gradient, int *count);

/* ---- arbitrary-order triangle Lagrange (vertices [x0,y0,x1,...]) ---- */
int or_triangle_lagrange_dof_count(int degree);
int or_triangle_lagrange_nodes(int degree, double *nodes /*2 x n_b*/, int *powers /*3 x n_b*/);
int or_triangle_lagrange_evaluate(int degree, double x, double y, double *values,
                                  double *gradients /*2 x n_b*/);
int or_triangle_lagrange_dof_map(int degree, int n_tris, const int *tris, int *global_dofs,
                                 int *n_global);
int or_triangle_lagrange_element(const double *vertices /*2x3*/, int degree, int quadrature_degree,
                                 double stiffness, double mass, double *matrix);
int64_t or_triangle_lagrange_csc_nnz(int degree, int n_tris, const int *tris);
int or_triangle_lagrange_csc(int n_vertices, const double *vertices, int n_tris, const int *tris,
                             int degree, int quadrature_degree, double stiffness, double mass,
                             const double *cell_stiffness, const double *cell_mass,
                             int64_t nnz_capacity, int *n_dofs, int64_t *nnz, int64_t *col_ptr,
                             int *row_idx, double *values);
int or_triangle_lagrange_load_samples(int n_vertices, const double *vertices, int n_tris,
                                      const int *tris, int degree, int quadrature_degree,
                                      const double *samples /* n_q x T */, double *rhs);
int or_triangle_lagrange_points(int n_vertices, const double *vertices, int n_tris,
                                const int *tris, int degree, int quadrature_degree,
                                double *sample_points /*2 x n_q x T*/,
                                double *dof_points /*2 x n_dofs*/);
int or_triangle_lagrange_boundary(int degree, int n_tris, const int *tris, uint8_t *constrained);

/* ---- P1 triangles ---- */
int or_p1_dense_matrix(int n_vertices, const double *vertices, int n_triangles, const int *triangles,
                       double mass, double stiffness, double *matrix /* n x n col-major */);
int or_p1_load(int n_vertices, const double *vertices, int n_triangles, const int *triangles,
               double load, double *vector);
int or_p1_csc(int n_vertices, const double *vertices, int n_triangles, const int *triangles,
              double mass, double stiffness, const double *cell_stiffness,
              int64_t nnz_capacity, int64_t *nnz, int64_t *col_ptr, int *row_idx, double *values);
int or_p1_dirichlet_eliminate_dense(int n, double *matrix, double *rhs, const uint8_t *boundary,
                                    double value);

/* ---- sparse / solver ---- */
int or_csc_from_triplet(int n_rows, int n_cols, int64_t n_triplets, const int *rows, const int *cols,
                        const double *values, int64_t nnz_capacity, int64_t *nnz, int64_t *col_ptr,
                        int *row_idx, double *out_values);
void or_csc_matvec(int n, const int64_t *col_ptr, const int *row_idx, const double *values,
                   const double *x, double *y);
int or_reduce_constrained(int n, const int64_t *col_ptr, const int *row_idx, const double *values,
                          const double *rhs, const uint8_t *constrained,
                          const double *constrained_values, int *n_free, int64_t *nnz_reduced,
                          int64_t *r_col_ptr, int *r_row_idx, double *r_values, double *r_rhs,
                          int *free_dofs);
/* solve_sparse(method=pcg, preconditioner=jacobi|none): returns iterations in stats[0],
 * converged in stats[1], final recursive residual norm in stats[2].  guard 0 is
 * the reference's absolute |p^T A p| < 1e-14 test, guard 1 stops only on
 * p^T A p <= 0 (SPD breakdown). */
int or_pcg_sparse(int n, const int64_t *col_ptr, const int *row_idx, const double *values,
                  const double *b, double *x, double tolerance, int relative, int max_iterations,
                  int jacobi, int guard, double *stats);
int or_pcg_dense(int n, const double *matrix, const double *b, double *x, double tolerance,
                 int relative, int max_iterations, int jacobi, int guard, double *stats);

/* ---- tetrahedral Nedelec (first kind) ---- */
int or_nedelec_dof_count(int order);
int or_nedelec_evaluate(int order, const double *point, double *values /*3 x n_b*/,
                        double *curls /*3 x n_b*/);
int or_whitney_evaluate(const double *point, double *values, double *curls);
int or_edge_dof_map_faithful(int n_tets, const int *tets, int *edges, int *global_dofs,
                             int *orientations, int *n_edges);
int or_edge_dof_map(int n_tets, const int *tets, int *edges, int *global_dofs, int *orientations,
                    int *n_edges);
int or_nedelec_dof_map(int order, int n_tets, const int *tets, int faithful, int *edges, int *n_edges,
                       int *faces, int *n_faces, int *global_dofs, int *edge_orientations,
                       int *face_permutations, int *n_global);
int or_face_basis_to_local(int order, const int *permutation, double *transform);
int or_nedelec_transform(int order, const int *edge_orientations, const int *face_permutations,
                         double *transform);
int or_nedelec_element(const double *vertices, int order, int quadrature_degree, double curl,
                       double mass, double *matrix);
int or_nedelec_whitney_element(const double *vertices, double curl, double mass, double *matrix);
int64_t or_nedelec_csc_nnz(int order, int n_tets, const int *tets);
int or_nedelec_csc(int n_vertices, const double *vertices, int n_tets, const int *tets, int order,
                   double curl, double mass, const double *cell_curl, const double *cell_mass,
                   int64_t nnz_capacity, int *n_dofs, int64_t *nnz, int64_t *col_ptr, int *row_idx,
                   double *values);
int or_nedelec_weighted_element(const double *v, int order, const double *tensor, double mass,
                                double *matrix);
int or_nedelec_weighted_csc(int n_vertices, const double *vertices, int n_tets, const int *tets,
                            int order, const double *tensors, double mass, int64_t cap,
                            int *n_dofs, int64_t *nnz, int64_t *col_ptr, int *row_idx,
                            double *values);
/* forward (JVP) and reverse (VJP) mode of the element and the CSC assembly */
int or_nedelec_element_jvp(const double *vertices, int order, int quadrature_degree, double curl,
                           double mass, const double *vertices_dot, double curl_dot,
                           double mass_dot, double *matrix_dot);
int or_nedelec_element_vjp(const double *vertices, int order, int quadrature_degree, double curl,
                           double mass, const double *matrix_bar, double *vertices_bar,
                           double *curl_bar, double *mass_bar);
int or_nedelec_csc_jvp(int n_vertices, const double *vertices, int n_tets, const int *tets,
                       int order, double curl, double mass, const double *vertices_dot,
                       double curl_dot, double mass_dot, int64_t nnz_capacity, int *n_dofs,
                       int64_t *nnz, int64_t *col_ptr, int *row_idx, double *values_dot);
int or_nedelec_csc_vjp(int n_vertices, const double *vertices, int n_tets, const int *tets,
                       int order, double curl, double mass, int64_t nnz, const double *values_bar,
                       double *vertices_bar, double *curl_bar, double *mass_bar);
/* complex PML variants: stretch 3 (Cartesian) or 9 (curvilinear, column-major)
 * complex values per cell as (re, im) pairs; matrices / values complex
 * (re, im) interleaved, element matrices column-major */
int or_nedelec_pml_element(const double *vertices, int order, int quadrature_degree,
                           const double *stretch, double wave_number, double *matrix);
int or_nedelec_curvilinear_pml_element(const double *vertices, int order, int quadrature_degree,
                                       const double *stretch, double wave_number, double *matrix);
int or_nedelec_pml_csc(int n_vertices, const double *vertices, int n_tets, const int *tets,
                       int order, const double *stretch, double wave_number, int64_t nnz_capacity,
                       int *n_dofs, int64_t *nnz, int64_t *col_ptr, int *row_idx, double *values);
int or_nedelec_curvilinear_pml_csc(int n_vertices, const double *vertices, int n_tets,
                                   const int *tets, int order, const double *stretch,
                                   double wave_number, int64_t nnz_capacity, int *n_dofs,
                                   int64_t *nnz, int64_t *col_ptr, int *row_idx, double *values);
int or_nedelec_evaluate_solution(int n_vertices, const double *vertices, int n_tets,
                                 const int *tets, int order, int n_dofs, const double *solution,
                                 int cell, const double *reference_point, double *value /*3*/,
                                 double *curl /*3*/);
int or_nedelec_probe(int n_vertices, const double *vertices, int n_tets, const int *tets, int order,
                     int n_dofs, const double *solution, const double *point, int mode,
                     double *value /*3*/, double *curl /*3*/, int *count);
int or_nedelec_load_samples(int n_vertices, const double *vertices, int n_tets, const int *tets,
                            int order, const double *source_values /* 3 x n_q x T */, double *rhs);
int or_nedelec_load_points(int n_vertices, const double *vertices, int n_tets, const int *tets,
                           int order, double *points /* 3 x n_q x T */);
int or_pec_mask(int order, int n_tets, const int *tets, int faithful, uint8_t *constrained);

#ifdef __cplusplus
}
#endif
#endif
