// Internal declarations of libfortfem_gpu.so (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/fortfem_gpu.h"

namespace ffg {

// Slot offsets are stored per (incidence pair, local row) as uint16; this value
// marks a local row whose global DoF is constrained (dropped from the system).
constexpr uint16_t kConstrainedSlot = 0xFFFF;
constexpr int kMaxColumnLength = 0xFFFE;

struct Error {
  int status;
  std::string message;
};

// ----------------------------------------------------------------- topology
// Everything that depends on the mesh connectivity only.  Built on the host
// once per mesh and uploaded; reused by every assembly/solve on that mesh.
struct Topology {
  int family = 0;         // FFG_TETRA_LAGRANGE / FFG_TETRA_NEDELEC / FFG_TRIANGLE_P1
  int degree = 0;         // Lagrange degree or Nedelec order
  int nb = 0;             // local DoFs per cell
  int vpc = 0;            // vertices per cell
  int n_cells = 0;
  int n_vertices = 0;
  int64_t n_dofs = 0;
  std::vector<int> cells;        // vpc * n_cells
  std::vector<int> gd;           // nb * n_cells, global DoF of each local DoF
  std::vector<int8_t> edge_sign; // 6 * n_cells (Nedelec)
  std::vector<uint8_t> face_perm;// 4 * n_cells permutation index 0..5 (Nedelec)
  int n_edges = 0, n_faces = 0;
  std::vector<uint8_t> constrained;  // n_dofs
  std::vector<int> free_index;       // n_dofs -> free index or -1
  std::vector<int> free_dofs;        // n_free
  // constrained (free x free) pattern, CSC == CSR by symmetry
  std::vector<int64_t> col_ptr;      // n_free + 1
  std::vector<int> row_idx;          // nnz
  // per free column: incident (cell, local) pairs in ascending cell order
  std::vector<int64_t> inc_ptr;      // n_free + 1
  std::vector<int> inc_cell;
  std::vector<uint8_t> inc_local;
  std::vector<uint16_t> slot;        // inc_count * nb
  int max_column = 0;
  int64_t n_free() const { return (int64_t)free_dofs.size(); }
  int64_t nnz() const { return (int64_t)row_idx.size(); }
};

// Edge signs (6) and face permutation indices (4) of a Nedelec cell from its
// four global vertex indices.
void nedelec_orientation(const int *v, int8_t *sign, uint8_t *perm);
// Build the DoF numbering of a family (first-appearance order of the
// reference).  Returns FFG_OK or FFG_INVALID_INPUT.
int build_dofs(Topology &t, std::string &msg);
// Cell vertices in range and distinct.
bool validate_cells(const Topology &t, std::string &msg);
// Constrained set: boundary_mode FFG_BOUNDARY_NONE / _ALL / _MASK.
int build_constraints(Topology &t, int boundary_mode, const uint8_t *mask, std::string &msg);
// Free numbering, CSC pattern of the free x free block, incidence lists and slots.
int build_pattern(Topology &t, std::string &msg);

// ------------------------------------------------------------ basis tables
struct Rule {
  std::vector<double> x, y, z, w;
  int size() const { return (int)w.size(); }
};
bool make_rule(int rule, int degree, Rule &r);
void gauss_legendre01(int n, double *x, double *w);

int lagrange_dof_count(int p);
void lagrange_indices(int p, std::vector<int> &idx, std::vector<double> &nodes);
void lagrange_eval(int p, const std::vector<int> &idx, const double *pt, double *val, double *grad);
int triangle_lagrange_dof_count(int p);
void triangle_lagrange_indices(int p, std::vector<int> &powers, std::vector<double> &nodes);
bool triangle_lagrange_coefficients(int p, std::vector<double> &C);
void triangle_lagrange_eval(int p, const std::vector<int> &powers, const std::vector<double> &C,
                            double x, double y, double *val, double *grad);
int nedelec_dof_count(int k);
bool nedelec_eval(int k, const double *pt, double *val, double *curl);
// The candidate vector monomials of the order-k first-kind space
// (tetra_nedelec_arbitrary_order.f90:318-396): per candidate two terms of
// (component, sign, x power, y power, z power), component -1 for an unused
// term.  The basis is the candidates times nedelec_coefficients(k)
// (candidate-major, n x n column-major by basis function).
void nedelec_candidate_terms(int k, std::vector<int> &terms);
const double *nedelec_coefficients(int k);
const double *face_transform_table(int k, int perm_index);

// Reference tensors for the per-cell contraction.
struct ElementTables {
  int nb = 0;
  int n_terms = 0;                 // number of reference matrices
  std::vector<double> ref;         // n_terms * nb * nb, column-major per matrix
  int nq_load = 0;
  std::vector<double> load_basis;  // Lagrange: nq_load * nb (w_q phi_i(q));
                                   // Nedelec: nq_load * nb * 3 (w_q v_i(q))
  std::vector<double> load_xi;     // nq_load * 3 reference load points
  // Nedelec orientation transforms (per face permutation) for faces, k(k-1) blocks
  std::vector<double> face_blocks; // 6 * fdc * fdc
};
int build_tables(const Topology &t, int rule, int qdeg, ElementTables &tab, std::string &msg);

// -------------------------------------------------------------- device side
// The solver streams the constrained operator in sliced ELLPACK form
// (SELL-32-sigma): rows in a permuted order sorted by length inside windows of
// sigma rows, 32-row slices stored column-major so that a warp reads 128
// contiguous bytes per step.  Column indices are stored as 16-bit offsets
// from the row (new numbering) when every offset fits, else as int32.
constexpr int kSliceRows = 32;
constexpr int kSellSigma = 4096;

struct HostSell {
  int64_t n = 0, n_slices = 0, padded = 0;
  std::vector<int64_t> soff;   // n_slices + 1 entry offsets
  std::vector<int> perm;       // new row -> old row
  std::vector<int> iperm;      // old row -> new row
  bool narrow = false;
  std::vector<int16_t> dcol;   // narrow: column - row (new numbering)
  std::vector<int> col;        // wide: column (new numbering)
  std::vector<int64_t> pos;    // position of every CSR entry (old row order) in the slices
};
// rp/ci: CSR of the operator (old numbering; for the symmetric constrained
// system this is its CSC).
void build_sell(const std::vector<int64_t> &rp, const std::vector<int> &ci, int sigma,
                HostSell &out);

struct DeviceSell {
  int64_t n = 0, n_slices = 0, padded = 0;
  int64_t *soff = nullptr;
  int16_t *dcol = nullptr;  // exactly one of dcol / col is set
  int *col = nullptr;
  double *val64 = nullptr;  // padded entries, zero in the padding
  float *val32 = nullptr;
  uint16_t *val16 = nullptr;  // FP16 bits of val32 / rscale (FFG_PRECISION_MIXED16, on demand)
  float *rscale = nullptr;    // per-row scale of val16: the row's largest |entry|
  double *dinv64 = nullptr;  // Jacobi inverse diagonal, new numbering
  float *dinv32 = nullptr;
  int *perm = nullptr, *iperm = nullptr;
  int *cta_slice = nullptr;  // grid + 1 slice boundaries of the CTAs
  int *wslice = nullptr;     // the slices of each warp of the grid, warp by warp
  int *woff = nullptr;       // grid * 32 + 1 starts of the warps' lists in wslice
  int2 *inc_range = nullptr; // per SELL row: its column's incidence range (the
                             // slice gather's, built on its first use)
  int grid = 0;
};

// Upload the slice structure (values left zero) and the CTA partition.
int upload_sell(const HostSell &h, int grid, DeviceSell &d);
// Work partition of a SELL operator over `grid` CTAs of 32 warps: cs holds
// grid + 1 CTA slice boundaries, wslice the slices of every warp (warp by
// warp, CTA-major) and woff (grid * 32 + 1) where each warp's list starts.
void sell_partition(const int64_t *soff, int64_t n_slices, int grid, std::vector<int> &cs,
                    std::vector<int> &wslice, std::vector<int> &woff, int slice_cost = 256);
// Re-deal an uploaded operator's slices to CTAs and warps with another slice cost.
int sell_repartition(DeviceSell &d, int slice_cost);
void free_sell(DeviceSell &d);
// The FP16 copy of an operator's FP32 values, row-scaled (allocated on first use).
int sell_half(DeviceSell &d, cudaStream_t s);

struct SolveWork {
  double *r64 = nullptr, *partial = nullptr;
  double *rd = nullptr, *qd = nullptr;      // FP64-mode residual and A p
  double2 *zpd0 = nullptr, *zpd1 = nullptr; // FP64-mode (z, p) pairs, double-buffered
  float *rf = nullptr, *zf = nullptr;       // mixed-mode FP32 r and z = D^-1 r
  float *pf = nullptr, *qf = nullptr;       // mixed-mode FP32 p and q = A p
  float *xf = nullptr;                      // mixed-mode FP32 step of x not yet folded in
  float2 *zpf0 = nullptr, *zpf1 = nullptr;  // mixed-mode (z, p) pairs once q = A p is direct
  unsigned int *barrier = nullptr;
  int *control = nullptr;    // [0] error status
  double *result = nullptr;  // device statistics block
  double *result_host = nullptr;  // pinned copy of the statistics block
  int *control_host = nullptr;    // pinned copy of the control word
  int grid = 0;
  int64_t n = 0;
  // last solve: [0] FP64 continuation taken, then device seconds seen by CTA 0
  // in SpMV work, barrier wait after it, vector work, wait, reliable updates
  double phase_seconds[6] = {0, 0, 0, 0, 0, 0};
};

int solve_work_alloc(SolveWork &w, int64_t n, int grid);
void solve_work_free(SolveWork &w);

// Launch the persistent Jacobi-PCG (FP64 or mixed) on b -> x (both in the
// SELL row numbering).  x holds the initial guess (FP64).  Fills stats.
int pcg_solve(const DeviceSell &A, const double *b, double *x, const ffg_solver_options &opts,
              SolveWork &w, ffg_solver_stats *stats, cudaStream_t stream, std::string &msg);
// Asynchronous halves of pcg_solve: enqueue the cooperative solve (or one
// CTA per system for a batch of independent systems) with the statistics
// copied to each workspace's pinned block, then decode that block once the
// stream has reached it.
int pcg_launch(const DeviceSell &A, const double *b, double *x, const ffg_solver_options &opts,
               SolveWork &w, cudaStream_t stream, std::string &msg);
int pcg_launch_batch(int count, const DeviceSell *const *A, const double *const *b,
                     double *const *x, const ffg_solver_options &opts, SolveWork *const *w,
                     cudaStream_t stream, std::string &msg);
// Independent systems in shared cooperative launches, each on a group of
// pcg_group_ctas(n) CTAs (16384 rows per CTA, at least 2, at most the grid);
// consecutive systems share a launch while their groups fit the grid.
int pcg_group_ctas(int64_t n, int grid);
int pcg_launch_groups(int count, const DeviceSell *const *A, const double *const *b,
                      double *const *x, const ffg_solver_options &opts, SolveWork *const *w,
                      cudaStream_t stream, std::string &msg);
int pcg_collect(SolveWork &w, ffg_solver_stats *stats, std::string &msg);
int pcg_grid_size(int *grid);

// FP64 CSR SpMV y = A x (drop-in matvec).
int csr_spmv64(int64_t n, const int64_t *rp, const int *ci, const double *v, const double *x,
               double *y, cudaStream_t stream);
// Jacobi diagonal and FP32 copy of SELL values (drop-in solve path).
int sell_prepare(DeviceSell &A, const int64_t *csr_rp, const int *csr_ci, const int64_t *pos,
                 bool jacobi, cudaStream_t s);

// Kernel launchers of the assembly (kernels_assemble.cu).
struct DeviceTopology {
  int *cells = nullptr;
  int *gd = nullptr;
  int8_t *edge_sign = nullptr;
  uint8_t *face_perm = nullptr;
  int *free_index = nullptr;
  int64_t *inc_ptr = nullptr;
  int *inc_cell = nullptr;
  uint8_t *inc_local = nullptr;
  uint16_t *slot = nullptr;
  double *ref = nullptr;         // reference tensors
  double *load_basis = nullptr;
  double *face_blocks = nullptr;
  const struct OrientedTables *ort = nullptr;  // Nedelec: oriented tensors and cell classes
};

// Oriented Nedelec tensors (kernels_oriented.cu).  A cell's orientation
// transform T depends only on the order of its four global vertex indices,
// so cells fall in 24 classes (the Lehmer code of that order) and
// T^T R_s T and T^T (w_q v(q)) are tabulated per class; cells are listed
// class by class in tiles of at most 64.
constexpr int kOrtClasses = 24;
constexpr int kOrtTileCells = 64;
struct OrientedTables {
  int order = 0, nb = 0, nql = 0, n_tiles = 0, n_chunks = 0;
  int64_t load_stride = 0;  // doubles per class in `load` (3 nql nb rounded up to even)
  // kOrtClasses x n_chunks x 12 x 128: per class, per 128-entry chunk of the
  // column-major nb x nb matrices, the twelve terms' entries (zero past nb^2)
  double *ref = nullptr;
  double *load = nullptr;  // kOrtClasses x load_stride: row 3q + a (nb values) is T^T (w_q v_a(q))
  int *order_cells = nullptr;  // cells in class order (ascending within a class)
  int4 *tiles = nullptr;       // {class, first position in order_cells, count, 0}
  int class_count[kOrtClasses] = {};
};
// Classes of the cells (host connectivity) and the tables of the classes present.
int ort_build(const Topology &t, const ElementTables &tab, OrientedTables &o);
struct AssemblyInputs;
// Oriented element matrices (n_cells * nb * nb, unless load_only) and element
// loads (n_cells * nb; zero without samples) by the class tables.
int launch_nedelec_oriented(const Topology &t, const OrientedTables &o, const DeviceTopology &dt,
                            const AssemblyInputs &in, double *elem, double *cell_rhs, int *err,
                            cudaStream_t s, bool load_only);
void ort_free(OrientedTables &o);
// Class of a cell with distinct vertex indices v[0..3].
int ort_class(const int *v);

// Lagrange / P1 topology built on the device (topology_gpu.cu): the arrays of
// build_dofs + build_constraints + build_pattern + build_sell, equal entry for
// entry, written straight into the device structures; the host Topology gets
// gd, constrained, free_dofs, col_ptr, row_idx, n_dofs and max_column.
int build_topology_device(Topology &t, int boundary_mode, const uint8_t *mask, int grid,
                          DeviceTopology &dt, int64_t **csc_col_ptr, int **csc_row,
                          DeviceSell &S, std::string &msg);

// Launch shapes chosen by the autotuner (ffg_problem_autotune); zero fields
// keep the built-in defaults.
struct LaunchTuning {
  int ned_threads = 0;      // Nedelec FP64 element kernels: threads per CTA (256)
  int ned_ctas_per_sm = 0;  // grid target of the matrix kernel in CTAs per SM (default 8)
  int col_threads = 0;      // column-owner gather: threads per block
  int tc_ctas_per_sm = 0;   // 3xTF32 tensor-core kernel: CTAs per SM (1 or 2)
  int slice_cost = 0;       // PCG work partition: cost of a slice beyond its entries
};

struct AssemblyInputs {
  const double *vertices = nullptr;  // device
  double coef_a = 1.0, coef_b = 0.0;
  const double *cell_a = nullptr, *cell_b = nullptr;  // device, nullable
  const double *samples = nullptr;                    // device, nullable
  const double *g = nullptr;                          // device constrained values, nullable
  // forward mode: with vertices_dot set, the Nedelec element kernel writes the
  // tangent element matrices along (vertices_dot, coef_a_dot, coef_b_dot)
  const double *vertices_dot = nullptr;               // device, nullable
  double coef_a_dot = 0.0, coef_b_dot = 0.0;
  // Nedelec: 12 contraction weights per cell supplied by the caller (device,
  // nullable); replaces the curl / mass weights computed from the geometry
  const double *geo_override = nullptr;
  const LaunchTuning *tune = nullptr;  // launch shapes (null: defaults)
};

// Per-cell geometry/coefficient block and element right-hand sides.
int launch_cell_geometry(const Topology &t, const ElementTables &tab, const DeviceTopology &dt,
                         const AssemblyInputs &in, double *geo, int geo_stride, double *cell_rhs,
                         int *err, cudaStream_t s);
// 3xTF32 tensor-core contraction of Nedelec element matrices (orders 3 to 6):
// the cells in 128-cell groups of one orientation class and the B operand
// images (TF32 hi / lo) of every (class, 128-entry chunk) of the oriented table.
struct TcPlan {
  int order = 0, n_chunks = 0, n_groups = 0;
  float *bimage = nullptr;  // kOrtClasses x n_chunks x (hi, lo) images, 16 KB each
  int4 *groups = nullptr;   // {class, first position in order_cells, count <= 128, 0}
  size_t image_bytes = 0;
};
bool tc_supported_order(int k);
// floats per cell of the tensor-core element matrices: nb^2 rounded up to 32
int64_t tc_cell_stride(int nb);
int tc_build_plan(const Topology &t, const OrientedTables &o, TcPlan &plan, cudaStream_t s);
void tc_free_plan(TcPlan &plan);
// Oriented element matrices in FP32 (column-major nb x nb, leading dimension
// nb, tc_cell_stride(nb) floats per cell), the weights from the geometry or
// in.geo_override.
int launch_nedelec_tc(const Topology &t, const DeviceTopology &dt, const AssemblyInputs &in,
                      const TcPlan &plan, float *elem, int *err, cudaStream_t s);

// Tensor-weighted Nedelec: the twelve contraction weights of every cell from
// its symmetric 3 x 3 tensor (column-major, 9 per cell, device) and the
// scalar curl / mass coefficients of `in`, for the element kernel's
// caller-weight mode.
int launch_weighted_weights(const Topology &t, const DeviceTopology &dt, const AssemblyInputs &in,
                            const double *tensor, double *geo, int *err, cudaStream_t s);
// Nedelec: oriented element matrices (n_cells * nb * nb) and oriented element
// loads by the class tables of dt.ort.  load_only: the element loads alone
// (the matrices come from the tensor-core kernel).
int launch_nedelec(const Topology &t, const ElementTables &tab, const DeviceTopology &dt,
                   const AssemblyInputs &in, double *elem, double *cell_rhs, int *err,
                   cudaStream_t s, bool load_only = false);
// Column-owner gather into the constrained operator (element matrices from
// `elem`, FP64 nb x nb per cell, or `elem32`, FP32 column-major with leading
// dimension ld32 and cs32 floats per cell).  With `sell` set the
// values go to the slices (FP64 + FP32 copy, Jacobi diagonal, rhs in the
// SELL numbering); otherwise to the CSC value array `csc_val` with the rhs in
// free-DoF order.  row_idx is the CSC row index array (device).
int launch_columns(const Topology &t, const ElementTables &tab, const DeviceTopology &dt,
                   const AssemblyInputs &in, const double *geo, int geo_stride,
                   const double *cell_rhs, const double *elem, const int64_t *col_ptr,
                   const int *row_idx, DeviceSell *sell, double *csc_val, double *rhs,
                   cudaStream_t s, const float *elem32 = nullptr, int ld32 = 0,
                   int64_t cs32 = 0);
int geo_stride_for(const Topology &t, const ElementTables &tab);
// Batched assembly of independent Lagrange-tetrahedron or P1 systems (the
// serving families) into their SELL operators, one launch per phase.
constexpr int kMaxAsmBatch = 48;
struct AsmSys {
  int n_cells = 0, nq = 0, stride = 0, nb = 0;
  int64_t n_free = 0, n_dofs = 0;
  const int *cells = nullptr;
  const double *verts = nullptr;
  double ca = 1.0, cb = 0.0;
  const double *cell_a = nullptr, *cell_b = nullptr, *samples = nullptr;
  double *geo = nullptr;
  int *err = nullptr;
  const int64_t *col_ptr = nullptr;
  const int *row_idx = nullptr;
  const int64_t *inc_ptr = nullptr;
  const int *inc_cell = nullptr;
  const uint8_t *inc_local = nullptr;
  const uint16_t *slot = nullptr;
  const int *gd = nullptr;
  const double *ref = nullptr, *load_basis = nullptr, *g = nullptr;
  const int *iperm = nullptr, *free_index = nullptr;
  const int64_t *soff = nullptr;
  double *val64 = nullptr, *dinv64 = nullptr, *rhs = nullptr, *x = nullptr, *solution = nullptr;
  float *val32 = nullptr, *dinv32 = nullptr;
};
struct AsmBatch {
  int count;
  int64_t cell_begin[kMaxAsmBatch + 1];
  int64_t col_begin[kMaxAsmBatch + 1];
  int64_t dof_begin[kMaxAsmBatch + 1];
  AsmSys sys[kMaxAsmBatch];
};
static_assert(sizeof(AsmBatch) <= 32000, "kernel parameter block too large");
// err = 0, geometry, SELL scatter with x = 0, for `count` systems of `family`
int launch_batch_assembly(int family, int count, const AsmSys *sys, cudaStream_t s);
// full solutions (constrained values from g or 0, free values from x)
int launch_batch_solutions(int count, const AsmSys *sys, cudaStream_t s);


// Forward / reverse mode of the Lagrange stiffness + mass and the Nedelec
// curl + mass assembly (kernels_ad.cu; the Nedelec forward mode runs through
// launch_nedelec with AssemblyInputs::vertices_dot).
// The JVP writes the tangent of the seven contraction weights of every cell
// into `geo` (load samples zero); launch_columns then yields the tangent CSC
// values.  The VJP reads the CSC cotangent values_bar (device, on the pattern
// col_ptr/row_idx) and writes the vertex adjoints (3 n_vertices) and the
// stiffness and mass adjoints (2), all device arrays; it returns once done.
int launch_lagrange_geometry_jvp(const Topology &t, const DeviceTopology &dt,
                                 const double *vertices, const double *vertices_dot, double ca,
                                 double cb, double ca_dot, double cb_dot, double *geo, int stride,
                                 int *err, cudaStream_t s);
int lagrange_vjp(const Topology &t, const DeviceTopology &dt, const int64_t *col_ptr,
                 const int *row_idx, const double *vertices, const double *values_bar, double ca,
                 double cb, double *vertices_bar, double *coef_bar, int *err, cudaStream_t s);
// Reverse mode of the Nedelec curl + mass assembly, same outputs; `elem`
// (n_cells * nb * nb) is the work space of orders whose element matrix does
// not fit in shared memory.
int nedelec_vjp(const Topology &t, const ElementTables &tab, const DeviceTopology &dt,
                const int64_t *col_ptr, const int *row_idx, const double *vertices,
                const double *values_bar, double ca, double cb, double *elem,
                double *vertices_bar, double *coef_bar, int *err, cudaStream_t s);

// ------------------------------------------------------------ complex PML
// The twelve Nedelec contraction weights of the complex PML forms per cell,
// real and imaginary parts (12 doubles per cell each): curl pairs
// (1/det) (J^T Cc J)_ab, mass pairs -k^2 det (J^-1 Cm J^-T)_ab, with
// (Cc, Cm) the Cartesian (stretch: 3 complex per cell) or curvilinear
// (stretch: 3x3 complex per cell, column-major) PML tensors.  Complex
// values are (re, im) pairs.  err: degenerate cell or invalid stretch.
int launch_pml_weights(const Topology &t, const DeviceTopology &dt, const double *vertices,
                       const double *stretch, bool curvilinear, double wave_number,
                       double *geo_re, double *geo_im, int *err, cudaStream_t s);
// values[2i] = re[i], values[2i+1] = im[i]
int launch_interleave(int64_t n, const double *re, const double *im, double *values,
                      cudaStream_t s);

// FP64 y = A x on the SELL layout (vectors in the SELL row order).
int sell_spmv64(const DeviceSell &A, const double *x, double *y, cudaStream_t s);

// --------------------------------------------------- evaluation and probes
// Device tables of the solution evaluators (kernels_probe.cu), built on first use.
struct EvalTables {
  int *lag_idx = nullptr;  // Lagrange: 4 barycentric indices per basis function
  int *terms = nullptr;    // Nedelec: nedelec_candidate_terms
  double *coef = nullptr;  // Nedelec: nedelec_coefficients
};
// Value and derivative (Lagrange gradient / Nedelec curl) of the solution u
// (device, n_dofs) at n_queries (cell, point) pairs, points reference or
// physical; values hold 1 (Lagrange) or 3 (Nedelec) entries per query,
// derivs 3, qstatus (nullable) 0 or FFG_INVALID_INPUT per query.  err is set
// when the Lagrange mesh holds a degenerate cell.  Asynchronous on s.
int evaluate_solution(const Topology &t, const DeviceTopology &dt, const EvalTables &et,
                      const double *vertices, const double *u, int n_queries, const int *qcell,
                      const double *qpoint, int physical, double *values, double *derivs,
                      int *qstatus, int *err, cudaStream_t s);
// Point location over all cells and the evaluation there: the average over
// the containing cells, or the first containing cell when first_only;
// counts per point (0 none, -1 rejected by the basis's point test).
// Returns once done.
int probe_solution(const Topology &t, const DeviceTopology &dt, const EvalTables &et,
                   const double *vertices, const double *u, int n_points, const double *points,
                   int first_only, double *values, double *derivs, int *counts, cudaStream_t s);

}  // namespace ffg
