// C-ABI entry points of libfortfem_gpu.so (declared in include/fortfem_gpu.h).
//
// Handles follow the reference's registry convention (positive process-local
// integers, src/bindings/fortfem_capi_solver.f90:10-13,108-124) but the
// registry here is mutex-protected.  No entry point aborts: every failure is
// reported through *status.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

#include "ffg_internal.h"

namespace ffg {
namespace {

template <class T>
int dalloc(T **p, size_t count) {
  if (count == 0) count = 1;
  if (cudaMalloc((void **)p, count * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return FFG_OUT_OF_MEMORY;
  }
  return FFG_OK;
}

// Device copy of h followed by `pad` zeroed entries.
template <class T>
int upload_padded(T **p, const std::vector<T> &h, size_t pad) {
  if (dalloc(p, h.size() + pad)) return FFG_OUT_OF_MEMORY;
  if (!h.empty() && cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (cudaMemset(*p + h.size(), 0, pad * sizeof(T)) != cudaSuccess) return FFG_CUDA_ERROR;
  return FFG_OK;
}

template <class T>
int zeros_padded(T **p, size_t n, size_t pad) {
  if (dalloc(p, n + pad)) return FFG_OUT_OF_MEMORY;
  if (cudaMemset(*p, 0, (n + pad) * sizeof(T)) != cudaSuccess) return FFG_CUDA_ERROR;
  return FFG_OK;
}

template <class T>
int upload(T **p, const std::vector<T> &h) {
  int st = dalloc(p, h.size());
  if (st) return st;
  if (!h.empty() && cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return FFG_CUDA_ERROR;
  return FFG_OK;
}

// One device-resident problem: topology, tables, pattern, work buffers.
struct Problem {
  Topology topo;
  ElementTables tab;
  DeviceTopology dt;
  HostSell hsell;            // solver layout (host copy: permutation, positions)
  DeviceSell S;              // solver operator (SELL-32-sigma)
  int64_t *csc_col_ptr = nullptr;  // constrained CSC pattern (device)
  int *csc_row = nullptr;
  double *csc_val = nullptr;       // CSC values, allocated on first use
  SolveWork work;
  int rule = 0, qdeg = 0, dim = 3;
  int geo_stride = 0;
  int samples_per_cell = 0;  // scalar samples per cell (x3 for Nedelec)
  double *geo = nullptr, *cell_rhs = nullptr, *elem = nullptr;
  double *rhs = nullptr, *x = nullptr, *full = nullptr;
  double *in_vertices = nullptr, *in_cell_a = nullptr, *in_cell_b = nullptr, *in_samples = nullptr,
         *in_g = nullptr;
  int *free_dofs = nullptr;
  // Nedelec with a per-cell tensor coefficient: the tensors (9 per cell) and
  // the contraction weights computed from them at every assembly
  double *cell_tensor = nullptr, *geo_w = nullptr;
  // Nedelec element contraction: FP64 CUDA cores or 3xTF32 tensor cores
  int assembly_precision = FFG_ASSEMBLY_FP64;
  TcPlan tc;
  OrientedTables ort;  // Nedelec: oriented tensors by vertex-order class (dt.ort)
  LaunchTuning tune;  // launch shapes (autotuned or defaults)
  int *err = nullptr;
  int *err_host = nullptr;   // pinned: degenerate-cell flag of a deferred check
  bool batch_pending = false;  // enqueued by ffg_problem_solve_batch, not yet collected
  EvalTables eval;           // evaluator tables, built on the first evaluate / probe
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

  ~Problem() {
    void *ptrs[] = {dt.cells, dt.gd, dt.edge_sign, dt.face_perm, dt.free_index, dt.inc_ptr,
                    dt.inc_cell, dt.inc_local, dt.slot, dt.ref, dt.load_basis, dt.face_blocks,
                    csc_col_ptr, csc_row, csc_val, geo, cell_rhs, elem, rhs, x, full, in_vertices,
                    in_cell_a, in_cell_b, in_samples, in_g, free_dofs, cell_tensor, geo_w,
                    err, eval.lag_idx,
                    eval.terms, eval.coef};
    for (void *p : ptrs)
      if (p) cudaFree(p);
    free_sell(S);
    tc_free_plan(tc);
    ort_free(ort);
    solve_work_free(work);
    if (err_host) cudaFreeHost(err_host);
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
  }
};

std::mutex g_mutex;
std::map<int, std::shared_ptr<Problem>> g_problems;
int g_next_handle = 1;

std::shared_ptr<Problem> find_problem(int h) {
  std::lock_guard<std::mutex> lock(g_mutex);
  auto it = g_problems.find(h);
  return it == g_problems.end() ? nullptr : it->second;
}

int device_ready() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return FFG_NO_DEVICE;
  }
  return FFG_OK;
}

// Status of a finished solve: a launch or copy error first, then converged,
// then the wall limit (FFG_TIMEOUT) apart from plain non-convergence.
int solve_status(int st, const ffg_solver_stats &s) {
  if (st) return st;
  if (s.converged) return FFG_OK;
  return s.status == FFG_TIMEOUT ? FFG_TIMEOUT : FFG_NOT_CONVERGED;
}

void report(int verbosity, const std::string &msg) {
  if (verbosity > 0 && !msg.empty()) std::fprintf(stderr, "fortfem_gpu: %s\n", msg.c_str());
}

int create_problem(int family, int degree, int n_vertices, int n_cells, const int *cells, int rule,
                   int qdeg, int boundary_mode, const uint8_t *mask, std::shared_ptr<Problem> &out,
                   std::string &msg) {
  int st = device_ready();
  if (st) return st;
  auto P = std::make_shared<Problem>();
  Topology &t = P->topo;
  t.family = family;
  t.degree = degree;
  t.vpc = (family == FFG_TRIANGLE_P1 || family == FFG_TRIANGLE_LAGRANGE) ? 3 : 4;
  P->dim = (family == FFG_TRIANGLE_P1 || family == FFG_TRIANGLE_LAGRANGE) ? 2 : 3;
  t.n_cells = n_cells;
  t.n_vertices = n_vertices;
  if (n_cells < 1 || n_vertices < 1 || !cells) { msg = "empty mesh"; return FFG_INVALID_INPUT; }
  t.cells.assign(cells, cells + (size_t)t.vpc * n_cells);
  int grid = 0;
  if ((st = pcg_grid_size(&grid))) return st;
  // Lagrange, P1 and Nedelec topologies are built on the device; arbitrary-order
  // triangles on the host
  const bool on_device =
      family == FFG_TETRA_LAGRANGE || family == FFG_TRIANGLE_P1 || family == FFG_TETRA_NEDELEC;
  if (on_device) {
    if (!validate_cells(t, msg)) return FFG_INVALID_INPUT;
    if (family == FFG_TRIANGLE_P1 && (t.vpc != 3 || degree != 1)) {
      msg = "P1 triangles only";
      return FFG_INVALID_INPUT;
    }
    if ((st = build_topology_device(t, boundary_mode, mask, grid, P->dt, &P->csc_col_ptr,
                                    &P->csc_row, P->S, msg)))
      return st;
  } else {
    if ((st = build_dofs(t, msg))) return st;
    if ((st = build_constraints(t, boundary_mode, mask, msg))) return st;
    if ((st = build_pattern(t, msg))) return st;
  }
  P->rule = rule;
  P->qdeg = qdeg;
  if ((st = build_tables(t, rule, qdeg, P->tab, msg))) return st;
  P->geo_stride = geo_stride_for(t, P->tab);
  P->samples_per_cell = P->tab.nq_load;
  // device topology
  DeviceTopology &dt = P->dt;
  if (!on_device) {
    if ((st = upload(&dt.cells, t.cells))) return st;
    if ((st = upload(&dt.gd, t.gd))) return st;
    if ((st = upload(&dt.edge_sign, t.edge_sign))) return st;
    if ((st = upload(&dt.face_perm, t.face_perm))) return st;
    if ((st = upload(&dt.free_index, t.free_index))) return st;
    if ((st = upload(&dt.inc_ptr, t.inc_ptr))) return st;
    if ((st = upload(&dt.inc_cell, t.inc_cell))) return st;
    if ((st = upload(&dt.inc_local, t.inc_local))) return st;
    if ((st = upload(&dt.slot, t.slot))) return st;
    // constrained CSC pattern (assembly) and the solver's SELL layout
    if ((st = upload(&P->csc_col_ptr, t.col_ptr))) return st;
    if ((st = upload(&P->csc_row, t.row_idx))) return st;
    build_sell(t.col_ptr, t.row_idx, kSellSigma, P->hsell);
    if ((st = upload_sell(P->hsell, grid, P->S))) return st;
  }
  if (!P->tab.face_blocks.empty() && (st = upload(&dt.face_blocks, P->tab.face_blocks))) return st;
  if (!P->tab.ref.empty() && (st = upload(&dt.ref, P->tab.ref))) return st;
  if (!P->tab.load_basis.empty() && (st = upload(&dt.load_basis, P->tab.load_basis))) return st;
  if (family == FFG_TETRA_NEDELEC) {
    if ((st = ort_build(t, P->tab, P->ort))) return st;
    dt.ort = &P->ort;
  }
  const int64_t nfree = t.n_free();
  // per-step buffers
  const size_t nc = (size_t)n_cells;
  if ((st = dalloc(&P->geo, nc * std::max(P->geo_stride, 1)))) return st;
  if (family == FFG_TETRA_NEDELEC) {
    if ((st = dalloc(&P->cell_rhs, nc * t.nb))) return st;
    if ((st = dalloc(&P->elem, nc * t.nb * t.nb))) return st;
  }
  if ((st = dalloc(&P->rhs, (size_t)nfree))) return st;
  if ((st = dalloc(&P->x, (size_t)nfree))) return st;
  if ((st = dalloc(&P->full, (size_t)t.n_dofs))) return st;
  if ((st = dalloc(&P->in_vertices, (size_t)n_vertices * P->dim))) return st;
  if ((st = dalloc(&P->in_cell_a, nc))) return st;
  if ((st = dalloc(&P->in_cell_b, nc))) return st;
  const int spc = P->samples_per_cell * (family == FFG_TETRA_NEDELEC ? 3 : 1);
  if ((st = dalloc(&P->in_samples, nc * spc))) return st;
  if ((st = dalloc(&P->in_g, (size_t)t.n_dofs))) return st;
  if ((st = upload(&P->free_dofs, t.free_dofs))) return st;
  if ((st = dalloc(&P->err, 4))) return st;
  if (cudaMallocHost((void **)&P->err_host, sizeof(int)) != cudaSuccess) return FFG_OUT_OF_MEMORY;
  *P->err_host = 0;
  if ((st = solve_work_alloc(P->work, nfree, grid))) return st;
  for (auto &e : P->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return FFG_CUDA_ERROR;
  out = P;
  return FFG_OK;
}

// x is in the solver's (SELL) row order: row i is free DoF perm[i].
__global__ void scatter_solution_kernel(int64_t n_free, const int *perm, const int *free_dofs,
                                        const double *x, double *full) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_free) full[free_dofs[perm[i]]] = x[i];
}

// Stage inputs (host or device) and assemble the constrained system: into the
// solver's SELL operator (rhs in SELL order) when `sell`, else into the CSC
// value array (rhs in free-DoF order).
int assemble(Problem &P, const double *vertices, double ca, double cb, const double *cell_a,
             const double *cell_b, const double *samples, const double *g, int memory,
             bool sell, cudaStream_t s, std::string &msg, bool defer_check = false) {
  const Topology &t = P.topo;
  AssemblyInputs in;
  in.coef_a = ca;
  in.coef_b = cb;
  in.tune = &P.tune;
  const size_t nc = (size_t)t.n_cells;
  const int spc = P.samples_per_cell * (t.family == FFG_TETRA_NEDELEC ? 3 : 1);
  if (!vertices) { msg = "vertices missing"; return FFG_INVALID_INPUT; }
  if (memory == 0) {
    auto h2d = [&](double *dst, const double *src, size_t count) -> const double * {
      if (!src) return nullptr;
      cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyHostToDevice, s);
      return dst;
    };
    in.vertices = h2d(P.in_vertices, vertices, (size_t)t.n_vertices * P.dim);
    in.cell_a = h2d(P.in_cell_a, cell_a, nc);
    in.cell_b = h2d(P.in_cell_b, cell_b, nc);
    in.samples = h2d(P.in_samples, samples, nc * spc);
    in.g = h2d(P.in_g, g, (size_t)t.n_dofs);
  } else {
    in.vertices = vertices;
    in.cell_a = cell_a;
    in.cell_b = cell_b;
    in.samples = samples;
    in.g = g;
  }
  if (!sell && !P.csc_val && dalloc(&P.csc_val, (size_t)std::max<int64_t>(t.nnz(), 1)))
    return FFG_OUT_OF_MEMORY;
  if (cudaMemsetAsync(P.err, 0, sizeof(int), s) != cudaSuccess) return FFG_CUDA_ERROR;
  int st;
  const float *elem32 = nullptr;
  int ld32 = 0;
  int64_t cs32 = 0;
  if (t.family == FFG_TETRA_NEDELEC) {
    if (P.cell_tensor) {
      st = launch_weighted_weights(t, P.dt, in, P.cell_tensor, P.geo_w, P.err, s);
      if (st) return st;
      in.geo_override = P.geo_w;
    }
    if (P.assembly_precision == FFG_ASSEMBLY_TF32X3) {
      // matrices on the tensor cores (FP32, leading dimension tc.ld), loads in FP64
      if (!P.tc.bimage && (st = tc_build_plan(t, P.ort, P.tc, s))) return st;
      if (in.samples) {
        st = launch_nedelec(t, P.tab, P.dt, in, P.elem, P.cell_rhs, P.err, s, true);
      } else {
        st = cudaMemsetAsync(P.cell_rhs, 0, sizeof(double) * t.nb * (size_t)t.n_cells, s) ==
                     cudaSuccess
                 ? FFG_OK
                 : FFG_CUDA_ERROR;
      }
      if (st) return st;
      float *e32 = reinterpret_cast<float *>(P.elem);
      st = launch_nedelec_tc(t, P.dt, in, P.tc, e32, P.err, s);
      elem32 = e32;
      ld32 = t.nb;
      cs32 = tc_cell_stride(t.nb);
    } else {
      st = launch_nedelec(t, P.tab, P.dt, in, P.elem, P.cell_rhs, P.err, s);
    }
  } else {
    st = launch_cell_geometry(t, P.tab, P.dt, in, P.geo, P.geo_stride, P.cell_rhs, P.err, s);
  }
  if (st) return st;
  st = launch_columns(t, P.tab, P.dt, in, P.geo, P.geo_stride, P.cell_rhs, P.elem, P.csc_col_ptr,
                      P.csc_row, sell ? &P.S : nullptr, P.csc_val, P.rhs, s, elem32, ld32, cs32);
  if (st) return st;
  if (defer_check) {
    // the flag is read with the statistics, after the stream has passed
    return cudaMemcpyAsync(P.err_host, P.err, sizeof(int), cudaMemcpyDeviceToHost, s) ==
                   cudaSuccess
               ? FFG_OK
               : FFG_CUDA_ERROR;
  }
  int herr = 0;
  if (cudaMemcpyAsync(&herr, P.err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (cudaStreamSynchronize(s) != cudaSuccess) return FFG_CUDA_ERROR;
  if (herr) { msg = "degenerate cell (det <= 64 eps max(1,|J|)^3)"; return herr; }
  return FFG_OK;
}

void fill_default(ffg_solver_options &o) {
  o.version = FFG_OPTIONS_VERSION;
  o.preconditioner = 1;
  o.precision = FFG_PRECISION_MIXED;
  o.tolerance_type = 0;
  o.tolerance = 1.0e-10;
  o.max_iterations = 1000000;
  o.max_refinements = 1000;
  o.inner_tolerance = 0.1;
  o.verbosity = 0;
  o.timeout_seconds = 60.0;
  o.breakdown_guard = 0;
}

int check_options(const ffg_solver_options *o, ffg_solver_options &out) {
  fill_default(out);
  if (!o) return FFG_OK;
  if (o->version != FFG_OPTIONS_VERSION) return FFG_INVALID_INPUT;
  out = *o;
  if (out.precision != FFG_PRECISION_FP64 && out.precision != FFG_PRECISION_MIXED &&
      out.precision != FFG_PRECISION_MIXED16)
    return FFG_INVALID_INPUT;
  if (out.tolerance < 0 || out.max_iterations < 0) return FFG_INVALID_INPUT;
  if (out.inner_tolerance <= 0 || out.inner_tolerance >= 1) out.inner_tolerance = 0.1;
  if (out.max_refinements < 0) out.max_refinements = 0;
  return FFG_OK;
}

__global__ void set_ones_kernel(int64_t n, double *d64, float *d32) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) { d64[i] = 1.0; d32[i] = 1.0f; }
}

struct HostCsr {
  std::vector<int64_t> rp;
  std::vector<int> col;
  std::vector<double> val;
};
// CSC -> CSR (rows ascending within each row by construction of the counting sort)
bool csc_to_csr(int n, const int64_t *cp, const int *ri, const double *v, HostCsr &out) {
  const int64_t nnz = cp[n];
  out.rp.assign((size_t)n + 1, 0);
  for (int64_t k = 0; k < nnz; ++k) {
    if (ri[k] < 0 || ri[k] >= n) return false;
    out.rp[ri[k] + 1]++;
  }
  for (int i = 0; i < n; ++i) out.rp[i + 1] += out.rp[i];
  out.col.assign((size_t)nnz, 0);
  out.val.assign((size_t)nnz, 0.0);
  std::vector<int64_t> pos(out.rp.begin(), out.rp.end() - 1);
  for (int c = 0; c < n; ++c) {
    if (cp[c + 1] < cp[c]) return false;
    for (int64_t k = cp[c]; k < cp[c + 1]; ++k) {
      const int64_t p = pos[ri[k]]++;
      out.col[p] = c;
      out.val[p] = v[k];
    }
  }
  return true;
}

struct DeviceCsrArrays {
  int64_t *rp = nullptr;
  int *ci = nullptr;
  double *v = nullptr;
  ~DeviceCsrArrays() {
    if (rp) cudaFree(rp);
    if (ci) cudaFree(ci);
    if (v) cudaFree(v);
  }
};

// SELL operator of a host CSR with its values, FP32 copy and Jacobi diagonal
// computed on the host.
int upload_sell_with_values(const HostCsr &h, int grid, bool jacobi, HostSell &hs,
                            DeviceSell &d) {
  build_sell(h.rp, h.col, kSellSigma, hs);
  int st = upload_sell(hs, grid, d);
  if (st) return st;
  const int64_t n = (int64_t)h.rp.size() - 1;
  std::vector<double> v64((size_t)std::max<int64_t>(hs.padded, 1), 0.0);
  std::vector<float> v32(v64.size(), 0.0f);
  std::vector<double> d64((size_t)std::max<int64_t>(n, 1), 1.0);
  std::vector<float> d32(d64.size(), 1.0f);
  for (int64_t i = 0; i < n; ++i) {
    double dg = 0.0;
    for (int64_t k = h.rp[i]; k < h.rp[i + 1]; ++k) {
      v64[hs.pos[k]] = h.val[k];
      v32[hs.pos[k]] = (float)h.val[k];
      if (h.col[k] == (int)i) dg = h.val[k];
    }
    // build_sparse_preconditioner("jacobi"), advanced_solvers.f90:1139-1154
    const double di = (jacobi && std::fabs(dg) > 1.0e-14) ? 1.0 / dg : 1.0;
    d64[hs.iperm[i]] = di;
    d32[hs.iperm[i]] = (float)di;
  }
  bool ok = cudaMemcpy(d.val64, v64.data(), sizeof(double) * hs.padded, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(d.val32, v32.data(), sizeof(float) * hs.padded, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(d.dinv64, d64.data(), sizeof(double) * n, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(d.dinv32, d32.data(), sizeof(float) * n, cudaMemcpyHostToDevice) == cudaSuccess;
  return ok ? FFG_OK : FFG_CUDA_ERROR;
}
}  // namespace
}  // namespace ffg

using namespace ffg;

extern "C" {

void ffg_default_options(ffg_solver_options *opts) {
  if (opts) fill_default(*opts);
}

void ffg_version(int *major, int *minor, int *patch) {
  if (major) *major = 0;
  if (minor) *minor = 1;
  if (patch) *patch = 0;
}

void ffg_device_count(int *count, int *status) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) { cudaGetLastError(); n = 0; }
  if (count) *count = n;
  if (status) *status = (n > 0) ? FFG_OK : FFG_NO_DEVICE;
}

void ffg_structured_tetra_box_mesh(const double *bounds, const int *counts, double *vertices,
                                   int *tets, int *status) {
  *status = FFG_INVALID_INPUT;
  if (!bounds || !counts || !vertices || !tets) return;
  for (int d = 0; d < 3; ++d)
    if (counts[d] < 1 || !(bounds[3 + d] > bounds[d])) return;
  const int nx = counts[0], ny = counts[1], nz = counts[2];
  auto vid = [&](int i, int j, int k) { return i + (nx + 1) * (j + (ny + 1) * k); };
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        const int ijk[3] = {i, j, k};
        const int v = vid(i, j, k);
        for (int d = 0; d < 3; ++d)
          vertices[3 * (size_t)v + d] =
              bounds[d] + ((double)ijk[d] / (double)counts[d]) * (bounds[3 + d] - bounds[d]);
      }
  // Kuhn split of each brick into six tetrahedra sharing the main diagonal
  // (add_brick_tetrahedra, structured_tetra_box_mesh.f90:78-94)
  static const int split[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7},
                                  {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};
  size_t cell = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const int brick[8] = {vid(i, j, k),         vid(i + 1, j, k),     vid(i, j + 1, k),
                              vid(i + 1, j + 1, k), vid(i, j, k + 1),     vid(i + 1, j, k + 1),
                              vid(i, j + 1, k + 1), vid(i + 1, j + 1, k + 1)};
        for (int c = 0; c < 6; ++c, ++cell) {
          int *t = tets + 4 * cell;
          for (int n = 0; n < 4; ++n) t[n] = brick[split[c][n]];
          // positive orientation: swap the last two vertices when det < 0 (:56-68)
          double J[9];
          for (int col = 0; col < 3; ++col)
            for (int r = 0; r < 3; ++r)
              J[r + 3 * col] = vertices[3 * (size_t)t[col + 1] + r] - vertices[3 * (size_t)t[0] + r];
          const double det = J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
                             J[6] * (J[1] * J[5] - J[4] * J[2]);
          if (det < 0.0) std::swap(t[2], t[3]);
        }
      }
  *status = FFG_OK;
}

void ffg_unit_square_mesh(int n, double *vertices, int *tris, int *status) {
  *status = FFG_INVALID_INPUT;
  if (n < 2 || !vertices || !tris) return;
  const double dx = 1.0 / (double)(n - 1);
  size_t k = 0;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i, ++k) {
      vertices[2 * k] = i * dx;
      vertices[2 * k + 1] = j * dx;
    }
  k = 0;
  for (int j = 0; j < n - 1; ++j)
    for (int i = 0; i < n - 1; ++i) {
      const int v1 = j * n + i, v2 = j * n + i + 1, v3 = (j + 1) * n + i + 1, v4 = (j + 1) * n + i;
      int *t = tris + 3 * k;
      t[0] = v1; t[1] = v2; t[2] = v3;
      t[3] = v1; t[4] = v3; t[5] = v4;
      k += 2;
    }
  *status = FFG_OK;
}

void ffg_build_topology(int family, int degree, int n_vertices, int n_cells, const int *cells,
                        int boundary_mode, const uint8_t *mask, int64_t dof_cap, int64_t nnz_cap,
                        int64_t *n_dofs, int64_t *n_free, int64_t *nnz, int *global_dofs,
                        uint8_t *constrained, int64_t *col_ptr, int *row_ind, int *status) {
  Topology t;
  t.family = family;
  t.degree = degree;
  t.vpc = (family == FFG_TRIANGLE_P1 || family == FFG_TRIANGLE_LAGRANGE) ? 3 : 4;
  t.n_cells = n_cells;
  t.n_vertices = n_vertices;
  std::string msg;
  if (n_cells < 1 || n_vertices < 1 || !cells) { *status = FFG_INVALID_INPUT; return; }
  t.cells.assign(cells, cells + (size_t)t.vpc * n_cells);
  int st;
  if ((st = build_dofs(t, msg)) || (st = build_constraints(t, boundary_mode, mask, msg)) ||
      (st = build_pattern(t, msg))) {
    *status = st;
    return;
  }
  if (n_dofs) *n_dofs = t.n_dofs;
  if (n_free) *n_free = t.n_free();
  if (nnz) *nnz = t.nnz();
  if (dof_cap < t.n_dofs || nnz_cap < t.nnz() || !global_dofs || !constrained || !col_ptr ||
      !row_ind) {
    *status = FFG_CAPACITY;
    return;
  }
  std::memcpy(global_dofs, t.gd.data(), sizeof(int) * t.gd.size());
  std::memcpy(constrained, t.constrained.data(), t.constrained.size());
  std::memcpy(col_ptr, t.col_ptr.data(), sizeof(int64_t) * t.col_ptr.size());
  std::memcpy(row_ind, t.row_idx.data(), sizeof(int) * t.row_idx.size());
  *status = FFG_OK;
}

void ffg_problem_create(int family, int degree, int n_vertices, int n_cells, const int *cells,
                        int rule, int qdeg, int boundary_mode, const uint8_t *mask, int *handle,
                        int64_t *n_dofs, int64_t *n_free, int64_t *nnz, int *samples_per_cell,
                        int *status) {
  std::shared_ptr<Problem> P;
  std::string msg;
  int st = create_problem(family, degree, n_vertices, n_cells, cells, rule, qdeg, boundary_mode,
                          mask, P, msg);
  if (st) {
    if (handle) *handle = 0;
    *status = st;
    return;
  }
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    const int h = g_next_handle++;
    g_problems[h] = P;
    if (handle) *handle = h;
  }
  if (n_dofs) *n_dofs = P->topo.n_dofs;
  if (n_free) *n_free = P->topo.n_free();
  if (nnz) *nnz = P->topo.nnz();
  if (samples_per_cell) *samples_per_cell = P->samples_per_cell;
  *status = FFG_OK;
}

void ffg_problem_phase_times(int handle, double *seconds, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  if (!seconds) { *status = FFG_INVALID_INPUT; return; }
  for (int i = 0; i < 6; ++i) seconds[i] = P->work.phase_seconds[i];
  *status = FFG_OK;
}

static int ensure_eval_tables(Problem &P) {
  const Topology &t = P.topo;
  if (t.family == FFG_TETRA_LAGRANGE && !P.eval.lag_idx) {
    std::vector<int> idx;
    std::vector<double> nodes;
    lagrange_indices(t.degree, idx, nodes);
    return upload(&P.eval.lag_idx, idx);
  }
  if (t.family == FFG_TETRA_NEDELEC && !P.eval.terms) {
    std::vector<int> terms;
    nedelec_candidate_terms(t.degree, terms);
    const double *C = nedelec_coefficients(t.degree);
    if (!C) return FFG_INVALID_INPUT;
    std::vector<double> coef(C, C + (size_t)t.nb * t.nb);
    int st = upload(&P.eval.terms, terms);
    return st ? st : upload(&P.eval.coef, coef);
  }
  return FFG_OK;
}

// Host or device staging of the evaluation inputs; outputs copied back when
// the caller passed host arrays.
struct EvalStaging {
  double *vertices = nullptr, *u = nullptr, *points = nullptr, *values = nullptr,
         *derivs = nullptr;
  int *cells = nullptr, *flags = nullptr;
  ~EvalStaging() {
    void *ptrs[] = {vertices, u, points, values, derivs, cells, flags};
    for (void *p : ptrs)
      if (p) cudaFree(p);
  }
};

void ffg_problem_evaluate(int handle, const double *vertices, const double *solution,
                          int n_queries, const int *cells, const double *points, int point_kind,
                          double *values, double *derivatives, int *query_status, int memory,
                          void *stream, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  const Topology &t = P->topo;
  if (t.family == FFG_TRIANGLE_P1 || t.family == FFG_TRIANGLE_LAGRANGE || n_queries < 0 || !vertices || !solution ||
      (n_queries > 0 && (!cells || !points || !values || !derivatives)) ||
      (point_kind != FFG_POINT_REFERENCE && point_kind != FFG_POINT_PHYSICAL)) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  int st = ensure_eval_tables(*P);
  if (st) { *status = st; return; }
  cudaStream_t s = (cudaStream_t)stream;
  const int wv = t.family == FFG_TETRA_NEDELEC ? 3 : 1;
  const size_t nq = (size_t)n_queries;
  EvalStaging S;
  const double *dv = vertices, *du = solution, *dp = points;
  const int *dc = cells;
  double *dval = values, *dder = derivatives;
  int *dstat = query_status;
  if (memory == 0) {
    const size_t vb = sizeof(double) * 3 * (size_t)t.n_vertices;
    if ((st = dalloc(&S.vertices, 3 * (size_t)t.n_vertices)) || (st = dalloc(&S.u, t.n_dofs)) ||
        (st = dalloc(&S.points, 3 * nq)) || (st = dalloc(&S.cells, nq)) ||
        (st = dalloc(&S.values, wv * nq)) || (st = dalloc(&S.derivs, 3 * nq)) ||
        (st = dalloc(&S.flags, nq))) {
      *status = st;
      return;
    }
    if (cudaMemcpyAsync(S.vertices, vertices, vb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(S.u, solution, sizeof(double) * t.n_dofs, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        (nq && cudaMemcpyAsync(S.points, points, sizeof(double) * 3 * nq, cudaMemcpyHostToDevice,
                               s) != cudaSuccess) ||
        (nq && cudaMemcpyAsync(S.cells, cells, sizeof(int) * nq, cudaMemcpyHostToDevice, s) !=
                   cudaSuccess)) {
      *status = FFG_CUDA_ERROR;
      return;
    }
    dv = S.vertices; du = S.u; dp = S.points; dc = S.cells;
    dval = S.values; dder = S.derivs; dstat = S.flags;
  }
  if (cudaMemsetAsync(P->err, 0, sizeof(int), s) != cudaSuccess) { *status = FFG_CUDA_ERROR; return; }
  st = evaluate_solution(t, P->dt, P->eval, dv, du, n_queries, dc, dp,
                         point_kind == FFG_POINT_PHYSICAL ? 1 : 0, dval, dder, dstat, P->err, s);
  if (st) { *status = st; return; }
  int herr = 0;
  if (cudaMemcpyAsync(&herr, P->err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  if (memory == 0 && nq) {
    if (cudaMemcpyAsync(values, S.values, sizeof(double) * wv * nq, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(derivatives, S.derivs, sizeof(double) * 3 * nq, cudaMemcpyDeviceToHost,
                        s) != cudaSuccess ||
        (query_status && cudaMemcpyAsync(query_status, S.flags, sizeof(int) * nq,
                                         cudaMemcpyDeviceToHost, s) != cudaSuccess)) {
      *status = FFG_CUDA_ERROR;
      return;
    }
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) { *status = FFG_CUDA_ERROR; return; }
  *status = herr ? herr : FFG_OK;
}

void ffg_problem_probe(int handle, const double *vertices, const double *solution, int n_points,
                       const double *points, int mode, double *values, double *derivatives,
                       int *counts, int memory, void *stream, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  const Topology &t = P->topo;
  if (t.family == FFG_TRIANGLE_P1 || t.family == FFG_TRIANGLE_LAGRANGE || n_points < 0 || !vertices || !solution ||
      (n_points > 0 && (!points || !values || !derivatives || !counts)) ||
      (mode != FFG_PROBE_AVERAGE && mode != FFG_PROBE_FIRST)) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  int st = ensure_eval_tables(*P);
  if (st) { *status = st; return; }
  cudaStream_t s = (cudaStream_t)stream;
  const int wv = t.family == FFG_TETRA_NEDELEC ? 3 : 1;
  const size_t np = (size_t)n_points;
  EvalStaging S;
  const double *dv = vertices, *du = solution, *dp = points;
  double *dval = values, *dder = derivatives;
  int *dcnt = counts;
  if (memory == 0) {
    if ((st = dalloc(&S.vertices, 3 * (size_t)t.n_vertices)) || (st = dalloc(&S.u, t.n_dofs)) ||
        (st = dalloc(&S.points, 3 * np)) || (st = dalloc(&S.values, wv * np)) ||
        (st = dalloc(&S.derivs, 3 * np)) || (st = dalloc(&S.flags, np))) {
      *status = st;
      return;
    }
    if (cudaMemcpyAsync(S.vertices, vertices, sizeof(double) * 3 * (size_t)t.n_vertices,
                        cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(S.u, solution, sizeof(double) * t.n_dofs, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        (np && cudaMemcpyAsync(S.points, points, sizeof(double) * 3 * np, cudaMemcpyHostToDevice,
                               s) != cudaSuccess)) {
      *status = FFG_CUDA_ERROR;
      return;
    }
    dv = S.vertices; du = S.u; dp = S.points;
    dval = S.values; dder = S.derivs; dcnt = S.flags;
  }
  st = probe_solution(t, P->dt, P->eval, dv, du, n_points, dp, mode == FFG_PROBE_FIRST ? 1 : 0,
                      dval, dder, dcnt, s);
  if (st) { *status = st; return; }
  if (memory == 0 && np) {
    if (cudaMemcpyAsync(values, S.values, sizeof(double) * wv * np, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(derivatives, S.derivs, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost,
                        s) != cudaSuccess ||
        cudaMemcpyAsync(counts, S.flags, sizeof(int) * np, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess) {
      *status = FFG_CUDA_ERROR;
      return;
    }
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) { *status = FFG_CUDA_ERROR; return; }
  *status = FFG_OK;
}

void ffg_problem_assemble(int handle, const double *vertices, double ca, double cb,
                          const double *cell_a, const double *cell_b, const double *samples,
                          const double *g, int memory, void *stream, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  if ((memory != 0 && memory != 1) || P->batch_pending) { *status = FFG_INVALID_INPUT; return; }
  std::string msg;
  *status = assemble(*P, vertices, ca, cb, cell_a, cell_b, samples, g, memory, true,
                     (cudaStream_t)stream, msg);
}

void ffg_problem_sell_permutation(int handle, int *perm, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  const int64_t n = P->topo.n_free();
  if (!perm) { *status = FFG_INVALID_INPUT; return; }
  if (n > 0 &&
      cudaMemcpy(perm, P->S.perm, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  *status = FFG_OK;
}

void ffg_problem_system_arrays(int handle, double *rhs, double *dinv, int memory, void *stream,
                               int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  if (memory != 0 && memory != 1) { *status = FFG_INVALID_INPUT; return; }
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = sizeof(double) * (size_t)P->topo.n_free();
  const cudaMemcpyKind kind = memory == 0 ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  if (bytes && ((rhs && cudaMemcpyAsync(rhs, P->rhs, bytes, kind, s) != cudaSuccess) ||
                (dinv && cudaMemcpyAsync(dinv, P->S.dinv64, bytes, kind, s) != cudaSuccess))) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  *status = cudaStreamSynchronize(s) == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

void ffg_problem_sell_spmv(int handle, const double *x, double *y, void *stream, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  if (!x || !y) { *status = FFG_INVALID_INPUT; return; }
  *status = sell_spmv64(P->S, x, y, (cudaStream_t)stream);
}

void ffg_problem_free(int handle, int *status) {
  std::lock_guard<std::mutex> lock(g_mutex);
  auto it = g_problems.find(handle);
  if (it == g_problems.end()) { *status = FFG_BAD_HANDLE; return; }
  g_problems.erase(it);
  *status = FFG_OK;
}

// A symmetric, finite 3 x 3 tensor per cell (column-major): the weighted
// Nedelec path takes only symmetric tensors (reluctivities), whose entries
// agree with their transposes to 1e-12 of the largest entry.
static bool symmetric_tensors(int64_t n_cells, const double *ten) {
  for (int64_t c = 0; c < n_cells; ++c) {
    const double *M = ten + 9 * c;
    double mx = 0.0;
    for (int i = 0; i < 9; ++i) {
      if (!std::isfinite(M[i])) return false;
      mx = std::max(mx, std::fabs(M[i]));
    }
    for (int r = 0; r < 3; ++r)
      for (int e = r + 1; e < 3; ++e)
        if (std::fabs(M[r + 3 * e] - M[e + 3 * r]) > 1e-12 * mx) return false;
  }
  return true;
}

// ---------------------------------------------------------------- autotuner
static void tuning_out(const LaunchTuning &t, ffg_tuning *o) {
  o->element_threads = t.ned_threads;
  o->element_ctas_per_sm = t.ned_ctas_per_sm;
  o->column_threads = t.col_threads;
  o->tc_ctas_per_sm = t.tc_ctas_per_sm;
  o->slice_cost = t.slice_cost;
}

static int valid_tuning(const ffg_tuning &t) {
  auto in = [](int v, std::initializer_list<int> ok) {
    if (v == 0) return true;
    for (int x : ok)
      if (v == x) return true;
    return false;
  };
  return in(t.element_threads, {256}) && t.element_ctas_per_sm >= 0 &&
         t.element_ctas_per_sm <= 32 && in(t.column_threads, {32, 64, 128, 256, 512}) &&
         in(t.tc_ctas_per_sm, {1, 2}) && t.slice_cost >= 0 && t.slice_cost <= (1 << 20);
}

void ffg_problem_set_tuning(int handle, const ffg_tuning *tuning, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  if (!tuning || !valid_tuning(*tuning) || P->batch_pending) { *status = FFG_INVALID_INPUT; return; }
  LaunchTuning t;
  t.ned_threads = tuning->element_threads;
  t.ned_ctas_per_sm = tuning->element_ctas_per_sm;
  t.col_threads = tuning->column_threads;
  t.tc_ctas_per_sm = tuning->tc_ctas_per_sm;
  t.slice_cost = tuning->slice_cost;
  int st = FFG_OK;
  if (P->topo.n_free() > 0 && t.slice_cost != P->tune.slice_cost)
    st = sell_repartition(P->S, t.slice_cost ? t.slice_cost : 256);
  if (!st) P->tune = t;
  *status = st;
}

void ffg_problem_autotune(int handle, const double *vertices, double ca, double cb,
                          const double *cell_a, const double *cell_b, const double *samples,
                          int memory, ffg_tuning *tuning, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  if (!vertices || (memory != 0 && memory != 1) || P->batch_pending) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  const Topology &t = P->topo;
  const size_t nc = (size_t)t.n_cells;
  const int spc = P->samples_per_cell * (t.family == FFG_TETRA_NEDELEC ? 3 : 1);
  // device-resident inputs for every candidate
  const double *v = vertices, *a = cell_a, *b = cell_b, *smp = samples;
  if (memory == 0) {
    auto h2d = [&](double *dst, const double *src, size_t n) -> const double * {
      if (!src) return nullptr;
      return cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess
                 ? dst
                 : nullptr;
    };
    v = h2d(P->in_vertices, vertices, (size_t)t.n_vertices * P->dim);
    a = h2d(P->in_cell_a, cell_a, nc);
    b = h2d(P->in_cell_b, cell_b, nc);
    smp = h2d(P->in_samples, samples, nc * spc);
    if (!v) { *status = FFG_CUDA_ERROR; return; }
  }
  std::string msg;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto time_assembly = [&](const LaunchTuning &cand, double &ms) -> int {
    P->tune = cand;
    ms = 1e30;
    for (int rep = 0; rep < 3; ++rep) {
      cudaEventRecord(e0, 0);
      int st = assemble(*P, v, ca, cb, a, b, smp, nullptr, 1, true, 0, msg);
      cudaEventRecord(e1, 0);
      if (st) return st;
      if (cudaEventSynchronize(e1) != cudaSuccess) return FFG_CUDA_ERROR;
      float f = 0;
      cudaEventElapsedTime(&f, e0, e1);
      ms = std::min(ms, (double)f);
    }
    return FFG_OK;
  };
  ffg_tuning rep;
  std::memset(&rep, 0, sizeof(rep));
  LaunchTuning best;  // defaults
  int st = FFG_OK;
  double best_ms = 0;
  if ((st = time_assembly(best, best_ms))) goto done;
  rep.default_assembly_ms = best_ms;
  {
    // element kernel shapes first, then the column gather's block size
    std::vector<LaunchTuning> cands;
    if (t.family == FFG_TETRA_NEDELEC && P->assembly_precision == FFG_ASSEMBLY_TF32X3) {
      for (int c : {1, 2}) {
        LaunchTuning x = best;
        x.tc_ctas_per_sm = c;
        cands.push_back(x);
      }
    } else if (t.family == FFG_TETRA_NEDELEC) {
      for (int c : {2, 4, 16}) {
        LaunchTuning x = best;
        x.ned_threads = 256;
        x.ned_ctas_per_sm = c;
        cands.push_back(x);
      }
    }
    for (const auto &x : cands) {
      double ms = 0;
      if ((st = time_assembly(x, ms))) goto done;
      if (ms < best_ms) { best_ms = ms; best = x; }
    }
    const LaunchTuning base = best;
    for (int th : {64, 128, 256}) {
      LaunchTuning x = base;
      x.col_threads = th;
      double ms = 0;
      if ((st = time_assembly(x, ms))) goto done;
      if (ms < best_ms) { best_ms = ms; best = x; }
    }
  }
  rep.assembly_ms = best_ms;
  P->tune = best;
  // PCG partition: a fixed 60-iteration mixed run on the assembled system
  if (t.n_free() > 0) {
    if ((st = assemble(*P, v, ca, cb, a, b, smp, nullptr, 1, true, 0, msg))) goto done;
    ffg_solver_options o;
    fill_default(o);
    o.tolerance = 0.0;
    o.max_iterations = 60;
    o.timeout_seconds = 10.0;
    o.breakdown_guard = 1;
    auto time_solve = [&](int cost, double &ms) -> int {
      int s2 = sell_repartition(P->S, cost);
      if (s2) return s2;
      ms = 1e30;
      for (int r = 0; r < 3; ++r) {
        cudaMemset(P->x, 0, sizeof(double) * (size_t)t.n_free());
        ffg_solver_stats stt;
        cudaEventRecord(e0, 0);
        s2 = pcg_solve(P->S, P->rhs, P->x, o, P->work, &stt, 0, msg);
        cudaEventRecord(e1, 0);
        if (s2) return s2;
        if (cudaEventSynchronize(e1) != cudaSuccess) return FFG_CUDA_ERROR;
        float f = 0;
        cudaEventElapsedTime(&f, e0, e1);
        ms = std::min(ms, (double)f);
      }
      return FFG_OK;
    };
    double sms_best = 0;
    if ((st = time_solve(256, sms_best))) goto done;
    rep.default_solve_ms = sms_best;
    int best_cost = 256;
    for (int cost : {16, 64, 128, 512, 1024}) {
      double ms = 0;
      if ((st = time_solve(cost, ms))) goto done;
      if (ms < sms_best) { sms_best = ms; best_cost = cost; }
    }
    rep.solve_ms = sms_best;
    P->tune.slice_cost = best_cost;
    if ((st = sell_repartition(P->S, best_cost))) goto done;
  }
done:
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) {
    report(1, msg);
    P->tune = LaunchTuning();
    sell_repartition(P->S, 256);
    *status = st;
    return;
  }
  tuning_out(P->tune, &rep);
  if (tuning) *tuning = rep;
  *status = FFG_OK;
}

void ffg_problem_set_assembly_precision(int handle, int precision, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  if (P->batch_pending || (precision != FFG_ASSEMBLY_FP64 && precision != FFG_ASSEMBLY_TF32X3)) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  if (precision == FFG_ASSEMBLY_TF32X3 &&
      (P->topo.family != FFG_TETRA_NEDELEC || !tc_supported_order(P->topo.degree))) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  P->assembly_precision = precision;
  *status = FFG_OK;
}

void ffg_problem_set_cell_tensor(int handle, const double *tensors, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  if (P->topo.family != FFG_TETRA_NEDELEC || P->batch_pending) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  if (!tensors) {
    if (P->cell_tensor) cudaFree(P->cell_tensor);
    if (P->geo_w) cudaFree(P->geo_w);
    P->cell_tensor = P->geo_w = nullptr;
    *status = FFG_OK;
    return;
  }
  const size_t nc = (size_t)P->topo.n_cells;
  if (!symmetric_tensors((int64_t)nc, tensors)) { *status = FFG_INVALID_INPUT; return; }
  int st = FFG_OK;
  if (!P->cell_tensor && (st = dalloc(&P->cell_tensor, 9 * std::max<size_t>(nc, 1)))) {
    *status = st;
    return;
  }
  if (!P->geo_w && (st = dalloc(&P->geo_w, 12 * std::max<size_t>(nc, 1)))) {
    *status = st;
    return;
  }
  if (nc && cudaMemcpy(P->cell_tensor, tensors, sizeof(double) * 9 * nc,
                       cudaMemcpyHostToDevice) != cudaSuccess) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  *status = FFG_OK;
}

void ffg_problem_topology(int handle, int *global_dofs, int8_t *edge_sign, uint8_t *face_perm,
                          int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  const Topology &t = P->topo;
  if (global_dofs) std::memcpy(global_dofs, t.gd.data(), sizeof(int) * t.gd.size());
  if (t.family == FFG_TETRA_NEDELEC) {
    if (edge_sign) std::memcpy(edge_sign, t.edge_sign.data(), t.edge_sign.size());
    if (face_perm) std::memcpy(face_perm, t.face_perm.data(), t.face_perm.size());
  }
  *status = FFG_OK;
}

void ffg_problem_constrained(int handle, uint8_t *mask, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  std::memcpy(mask, P->topo.constrained.data(), P->topo.constrained.size());
  *status = FFG_OK;
}

void ffg_problem_sample_points(int handle, const double *vertices, double *points, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  const Topology &t = P->topo;
  const ElementTables &tab = P->tab;
  for (int c = 0; c < t.n_cells; ++c) {
    const int *v = t.cells.data() + (size_t)t.vpc * c;
    if (t.family == FFG_TRIANGLE_P1) {
      // one sample per triangle, at its centroid
      double x = 0, y = 0;
      for (int i = 0; i < 3; ++i) { x += vertices[2 * (size_t)v[i]]; y += vertices[2 * (size_t)v[i] + 1]; }
      points[3 * (size_t)c] = x / 3.0;
      points[3 * (size_t)c + 1] = y / 3.0;
      points[3 * (size_t)c + 2] = 0.0;
      continue;
    }
    if (t.family == FFG_TRIANGLE_LAGRANGE) {
      const double *a = vertices + 2 * (size_t)v[0], *b = vertices + 2 * (size_t)v[1],
                   *d = vertices + 2 * (size_t)v[2];
      for (int q = 0; q < tab.nq_load; ++q) {
        const double *xi = &tab.load_xi[3 * q];
        for (int r = 0; r < 2; ++r)
          points[3 * ((size_t)tab.nq_load * c + q) + r] = a[r] + (b[r] - a[r]) * xi[0] + (d[r] - a[r]) * xi[1];
        points[3 * ((size_t)tab.nq_load * c + q) + 2] = 0.0;
      }
      continue;
    }
    const double *p0 = vertices + 3 * (size_t)v[0];
    for (int q = 0; q < tab.nq_load; ++q) {
      const double *xi = &tab.load_xi[3 * q];
      for (int r = 0; r < 3; ++r) {
        double s = p0[r];
        for (int k = 0; k < 3; ++k) s = s + (vertices[3 * (size_t)v[k + 1] + r] - p0[r]) * xi[k];
        points[3 * ((size_t)tab.nq_load * c + q) + r] = s;
      }
    }
  }
  *status = FFG_OK;
}

void ffg_problem_dof_points(int handle, const double *vertices, double *points, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  const Topology &t = P->topo;
  if (t.family == FFG_TETRA_NEDELEC) { *status = FFG_INVALID_INPUT; return; }
  if (t.family == FFG_TRIANGLE_P1) {
    for (int i = 0; i < t.n_vertices; ++i) {
      points[3 * (size_t)i] = vertices[2 * (size_t)i];
      points[3 * (size_t)i + 1] = vertices[2 * (size_t)i + 1];
      points[3 * (size_t)i + 2] = 0.0;
    }
    *status = FFG_OK;
    return;
  }
  if (t.family == FFG_TRIANGLE_LAGRANGE) {
    std::vector<int> pw;
    std::vector<double> nodes;
    triangle_lagrange_indices(t.degree, pw, nodes);
    for (int c = 0; c < t.n_cells; ++c) {
      const int *v = t.cells.data() + 3 * (size_t)c;
      const double *a = vertices + 2 * (size_t)v[0], *b = vertices + 2 * (size_t)v[1],
                   *d = vertices + 2 * (size_t)v[2];
      for (int l = 0; l < t.nb; ++l) {
        const int g = t.gd[(size_t)t.nb * c + l];
        for (int r = 0; r < 2; ++r)
          points[3 * (size_t)g + r] = a[r] + (b[r] - a[r]) * nodes[2 * l] + (d[r] - a[r]) * nodes[2 * l + 1];
        points[3 * (size_t)g + 2] = 0.0;
      }
    }
    *status = FFG_OK;
    return;
  }
  std::vector<int> idx;
  std::vector<double> nodes;
  lagrange_indices(t.degree, idx, nodes);
  for (int c = 0; c < t.n_cells; ++c) {
    const int *v = t.cells.data() + 4 * (size_t)c;
    const double *p0 = vertices + 3 * (size_t)v[0];
    for (int l = 0; l < t.nb; ++l) {
      const int g = t.gd[(size_t)t.nb * c + l];
      for (int r = 0; r < 3; ++r) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += (vertices[3 * (size_t)v[k + 1] + r] - p0[r]) * nodes[3 * l + k];
        points[3 * (size_t)g + r] = p0[r] + s;
      }
    }
  }
  *status = FFG_OK;
}

void ffg_problem_solve(int handle, const double *vertices, double ca, double cb,
                       const double *cell_a, const double *cell_b, const double *samples,
                       const double *g, const ffg_solver_options *opts, double *solution,
                       ffg_solver_stats *stats, int memory, void *stream, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  ffg_solver_options o;
  if (check_options(opts, o)) { *status = FFG_INVALID_INPUT; return; }
  if (!solution || (memory != 0 && memory != 1) || P->batch_pending) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  cudaStream_t s = (cudaStream_t)stream;
  std::string msg;
  ffg_solver_stats local;
  std::memset(&local, 0, sizeof(local));
  cudaEventRecord(P->ev[0], s);
  int st = assemble(*P, vertices, ca, cb, cell_a, cell_b, samples, g, memory, true, s, msg);
  if (st) { report(o.verbosity, msg); *status = st; if (stats) { local.status = st; *stats = local; } return; }
  cudaEventRecord(P->ev[1], s);
  const Topology &t = P->topo;
  if (!o.preconditioner) {
    set_ones_kernel<<<(unsigned)((t.n_free() + 255) / 256), 256, 0, s>>>(t.n_free(), P->S.dinv64,
                                                                        P->S.dinv32);
  }
  cudaMemsetAsync(P->x, 0, sizeof(double) * (size_t)std::max<int64_t>(t.n_free(), 1), s);
  if (t.n_free() > 0) {
    if (o.precision == FFG_PRECISION_MIXED16) st = sell_half(P->S, s);
    if (!st) st = pcg_solve(P->S, P->rhs, P->x, o, P->work, &local, s, msg);
    if (st) { report(o.verbosity, msg); *status = st; if (stats) { local.status = st; *stats = local; } return; }
  } else {
    local.converged = 1;
  }
  cudaEventRecord(P->ev[2], s);
  // full solution: constrained values (or zero) then the free DoFs
  const double *gdev = (memory == 0) ? (g ? P->in_g : nullptr) : g;
  if (gdev)
    cudaMemcpyAsync(P->full, gdev, sizeof(double) * (size_t)t.n_dofs, cudaMemcpyDeviceToDevice, s);
  else
    cudaMemsetAsync(P->full, 0, sizeof(double) * (size_t)t.n_dofs, s);
  if (t.n_free() > 0)
    scatter_solution_kernel<<<(unsigned)((t.n_free() + 255) / 256), 256, 0, s>>>(
        t.n_free(), P->S.perm, P->free_dofs, P->x, P->full);
  cudaMemcpyAsync(solution, P->full, sizeof(double) * (size_t)t.n_dofs,
                  memory == 0 ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s);
  cudaEventRecord(P->ev[3], s);
  if (cudaEventSynchronize(P->ev[3]) != cudaSuccess) { *status = FFG_CUDA_ERROR; return; }
  float ta = 0, ts = 0;
  cudaEventElapsedTime(&ta, P->ev[0], P->ev[1]);
  cudaEventElapsedTime(&ts, P->ev[1], P->ev[2]);
  local.assembly_seconds = ta * 1e-3;
  local.solve_seconds = ts * 1e-3;
  if (o.verbosity > 0)
    std::fprintf(stderr,
                 "fortfem_gpu: n_free=%lld nnz=%lld it=%d ref=%d converged=%d rel=%.3e "
                 "assembly=%.3f ms solve=%.3f ms\n",
                 (long long)t.n_free(), (long long)t.nnz(), local.iterations, local.refinements,
                 local.converged, local.true_relative_residual, ta, ts);
  if (stats) *stats = local;
  *status = local.status == FFG_NOT_CONVERGED ? FFG_NOT_CONVERGED : local.status;
  if (local.converged) *status = FFG_OK;
}

void ffg_problem_solve_batch(int count, const int *handles, const double *const *vertices,
                             const double *coef_a, const double *coef_b,
                             const double *const *cell_a, const double *const *cell_b,
                             const double *const *samples, const double *const *g,
                             const ffg_solver_options *opts, double *const *solutions, int mode,
                             void *stream, int *status) {
  if (count < 1 || !handles || !vertices || !coef_a || !coef_b || !solutions ||
      (mode != FFG_BATCH_CTA_PER_SYSTEM && mode != FFG_BATCH_WHOLE_DEVICE &&
       mode != FFG_BATCH_CTA_GROUPS)) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  ffg_solver_options o;
  if (check_options(opts, o)) { *status = FFG_INVALID_INPUT; return; }
  std::vector<std::shared_ptr<Problem>> probs((size_t)count);
  for (int i = 0; i < count; ++i) {
    probs[i] = find_problem(handles[i]);
    if (!probs[i]) { *status = FFG_BAD_HANDLE; return; }
    if (probs[i]->batch_pending || !vertices[i] || !solutions[i]) {
      *status = FFG_INVALID_INPUT;
      return;
    }
    for (int j = 0; j < i; ++j)
      if (probs[j] == probs[i]) { *status = FFG_INVALID_INPUT; return; }
  }
  cudaStream_t s = (cudaStream_t)stream;
  std::string msg;
  int st = FFG_OK;
  // Lagrange-tetrahedron and P1 systems with scalar coefficients (the serving
  // families) are assembled together, one launch per phase and family; the
  // rest one system at a time
  std::vector<AsmSys> lag, p1;
  std::vector<AsmSys> all((size_t)count);
  std::vector<char> batched((size_t)count, 0);
  for (int i = 0; i < count; ++i) {
    Problem &P = *probs[i];
    const Topology &t = P.topo;
    if ((t.family != FFG_TETRA_LAGRANGE && t.family != FFG_TRIANGLE_P1) || P.cell_tensor)
      continue;
    AsmSys a;
    a.n_cells = t.n_cells;
    a.nq = P.tab.nq_load;
    a.stride = P.geo_stride;
    a.nb = t.nb;
    a.n_free = t.n_free();
    a.n_dofs = t.n_dofs;
    a.cells = P.dt.cells;
    a.verts = vertices[i];
    a.ca = coef_a[i];
    a.cb = coef_b[i];
    a.cell_a = cell_a ? cell_a[i] : nullptr;
    a.cell_b = cell_b ? cell_b[i] : nullptr;
    a.samples = samples ? samples[i] : nullptr;
    a.geo = P.geo;
    a.err = P.err;
    a.col_ptr = P.csc_col_ptr;
    a.row_idx = P.csc_row;
    a.inc_ptr = P.dt.inc_ptr;
    a.inc_cell = P.dt.inc_cell;
    a.inc_local = P.dt.inc_local;
    a.slot = P.dt.slot;
    a.gd = P.dt.gd;
    a.ref = P.dt.ref;
    a.load_basis = P.dt.load_basis;
    a.g = g ? g[i] : nullptr;
    a.iperm = P.S.iperm;
    a.free_index = P.dt.free_index;
    a.soff = P.S.soff;
    a.val64 = P.S.val64;
    a.val32 = P.S.val32;
    a.dinv64 = P.S.dinv64;
    a.dinv32 = P.S.dinv32;
    a.rhs = P.rhs;
    a.x = P.x;
    a.solution = solutions[i];
    all[i] = a;
    batched[i] = 1;
    (t.family == FFG_TETRA_LAGRANGE ? lag : p1).push_back(a);
  }
  for (int i = 0; i < count; ++i)
    if (batched[i]) cudaEventRecord(probs[i]->ev[0], s);
  if (!lag.empty()) st = launch_batch_assembly(FFG_TETRA_LAGRANGE, (int)lag.size(), lag.data(), s);
  if (!st && !p1.empty()) st = launch_batch_assembly(FFG_TRIANGLE_P1, (int)p1.size(), p1.data(), s);
  for (int i = 0; i < count && !st; ++i) {
    Problem &P = *probs[i];
    const Topology &t = P.topo;
    if (batched[i]) {
      // the degenerate-cell flag is read with the statistics
      if (cudaMemcpyAsync(P.err_host, P.err, sizeof(int), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess)
        st = FFG_CUDA_ERROR;
    } else {
      cudaEventRecord(P.ev[0], s);
      st = assemble(P, vertices[i], coef_a[i], coef_b[i], cell_a ? cell_a[i] : nullptr,
                    cell_b ? cell_b[i] : nullptr, samples ? samples[i] : nullptr,
                    g ? g[i] : nullptr, 1, true, s, msg, true);
      if (st) break;
      cudaMemsetAsync(P.x, 0, sizeof(double) * (size_t)std::max<int64_t>(t.n_free(), 1), s);
    }
    if (!o.preconditioner)
      set_ones_kernel<<<(unsigned)((t.n_free() + 255) / 256), 256, 0, s>>>(t.n_free(), P.S.dinv64,
                                                                          P.S.dinv32);
    cudaEventRecord(P.ev[1], s);
  }
  if (!st) {
    std::vector<const DeviceSell *> A;
    std::vector<const double *> b;
    std::vector<double *> x;
    std::vector<SolveWork *> w;
    for (auto &P : probs)
      if (P->topo.n_free() > 0) {
        A.push_back(&P->S);
        b.push_back(P->rhs);
        x.push_back(P->x);
        w.push_back(&P->work);
      }
    if (o.precision == FFG_PRECISION_MIXED16)
      for (auto &P : probs)
        if (!st && P->topo.n_free() > 0) st = sell_half(P->S, s);
    if (st) {
    } else if (mode == FFG_BATCH_CTA_PER_SYSTEM) {
      if (!A.empty())
        st = pcg_launch_batch((int)A.size(), A.data(), b.data(), x.data(), o, w.data(), s, msg);
    } else if (mode == FFG_BATCH_CTA_GROUPS) {
      if (!A.empty())
        st = pcg_launch_groups((int)A.size(), A.data(), b.data(), x.data(), o, w.data(), s, msg);
    } else {
      for (size_t i = 0; i < A.size() && !st; ++i)
        st = pcg_launch(*A[i], b[i], x[i], o, *w[i], s, msg);
    }
  }
  for (int i = 0; i < count && !st; ++i) cudaEventRecord(probs[i]->ev[2], s);
  {
    std::vector<AsmSys> sols;
    for (int i = 0; i < count; ++i)
      if (batched[i]) sols.push_back(all[i]);
    if (!st && !sols.empty()) st = launch_batch_solutions((int)sols.size(), sols.data(), s);
  }
  for (int i = 0; i < count && !st; ++i) {
    Problem &P = *probs[i];
    const Topology &t = P.topo;
    if (!batched[i]) {
      if (g && g[i])
        cudaMemcpyAsync(P.full, g[i], sizeof(double) * (size_t)t.n_dofs, cudaMemcpyDeviceToDevice,
                        s);
      else
        cudaMemsetAsync(P.full, 0, sizeof(double) * (size_t)t.n_dofs, s);
      if (t.n_free() > 0)
        scatter_solution_kernel<<<(unsigned)((t.n_free() + 255) / 256), 256, 0, s>>>(
            t.n_free(), P.S.perm, P.free_dofs, P.x, P.full);
      cudaMemcpyAsync(solutions[i], P.full, sizeof(double) * (size_t)t.n_dofs,
                      cudaMemcpyDeviceToDevice, s);
    }
    if (cudaEventRecord(P.ev[3], s) != cudaSuccess) st = FFG_CUDA_ERROR;
  }
  if (st) {
    report(o.verbosity, msg);
    *status = st;
    return;
  }
  for (auto &P : probs) P->batch_pending = true;
  *status = FFG_OK;
}

void ffg_problem_batch_stats(int handle, ffg_solver_stats *stats, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  if (!P->batch_pending) { *status = FFG_INVALID_INPUT; return; }
  const cudaError_t q = cudaEventQuery(P->ev[3]);
  if (q == cudaErrorNotReady) { *status = FFG_NOT_READY; return; }
  if (q != cudaSuccess) { cudaGetLastError(); *status = FFG_CUDA_ERROR; return; }
  P->batch_pending = false;
  ffg_solver_stats local;
  std::memset(&local, 0, sizeof(local));
  std::string msg;
  int st = FFG_OK;
  if (*P->err_host) {
    st = *P->err_host;
  } else if (P->topo.n_free() > 0) {
    st = pcg_collect(P->work, &local, msg);
  } else {
    local.converged = 1;
  }
  float ta = 0, ts = 0;
  cudaEventElapsedTime(&ta, P->ev[0], P->ev[1]);
  cudaEventElapsedTime(&ts, P->ev[1], P->ev[2]);
  local.assembly_seconds = ta * 1e-3;
  local.solve_seconds = ts * 1e-3;
  if (st) local.status = st;
  if (stats) *stats = local;
  *status = solve_status(st, local);
}

void ffg_problem_reduced_system(int handle, const double *vertices, double ca, double cb,
                                const double *cell_a, const double *cell_b,
                                const double *samples, const double *g, int64_t cap,
                                int64_t *nnz, int64_t *col_ptr, int *row_ind, double *values,
                                double *rhs, int *free_dofs, int *status) {
  auto P = find_problem(handle);
  if (!P) { *status = FFG_BAD_HANDLE; return; }
  const Topology &t = P->topo;
  if (nnz) *nnz = t.nnz();
  if (cap < t.nnz() || !col_ptr || !row_ind || !values) { *status = FFG_CAPACITY; return; }
  std::string msg;
  int st = assemble(*P, vertices, ca, cb, cell_a, cell_b, samples, g, 0, false, 0, msg);
  if (st) { *status = st; return; }
  std::memcpy(col_ptr, t.col_ptr.data(), sizeof(int64_t) * t.col_ptr.size());
  std::memcpy(row_ind, t.row_idx.data(), sizeof(int) * t.row_idx.size());
  if (cudaMemcpy(values, P->csc_val, sizeof(double) * (size_t)t.nnz(), cudaMemcpyDeviceToHost) != cudaSuccess) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  if (rhs && cudaMemcpy(rhs, P->rhs, sizeof(double) * (size_t)t.n_free(), cudaMemcpyDeviceToHost) != cudaSuccess) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  if (free_dofs) std::memcpy(free_dofs, t.free_dofs.data(), sizeof(int) * t.free_dofs.size());
  *status = FFG_OK;
}

// ------------------------------------------------------------ drop-in assembly
static void full_csc(int family, int degree, int nv, const double *verts, int nt, const int *cells,
                     int rule, int qdeg, double ca, double cb, const double *cell_a,
                     const double *cell_b, int64_t cap, int *n_dofs, int64_t *nnz,
                     int64_t *col_ptr, int *row_ind, double *values, int *status) {
  std::shared_ptr<Problem> P;
  std::string msg;
  int st = create_problem(family, degree, nv, nt, cells, rule, qdeg, FFG_BOUNDARY_NONE, nullptr, P,
                          msg);
  if (st) { *status = st; return; }
  if (n_dofs) *n_dofs = (int)P->topo.n_dofs;
  if (nnz) *nnz = P->topo.nnz();
  if (cap < P->topo.nnz() || !col_ptr || !row_ind || !values) { *status = FFG_CAPACITY; return; }
  st = assemble(*P, verts, ca, cb, cell_a, cell_b, nullptr, nullptr, 0, false, 0, msg);
  if (st) { *status = st; return; }
  std::memcpy(col_ptr, P->topo.col_ptr.data(), sizeof(int64_t) * P->topo.col_ptr.size());
  std::memcpy(row_ind, P->topo.row_idx.data(), sizeof(int) * P->topo.row_idx.size());
  if (cudaMemcpy(values, P->csc_val, sizeof(double) * (size_t)P->topo.nnz(), cudaMemcpyDeviceToHost) !=
      cudaSuccess) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  *status = FFG_OK;
}

static void full_load(int family, int degree, int nv, const double *verts, int nt, const int *cells,
                      int rule, int qdeg, const double *samples, int n_dofs, double *rhs,
                      int *status) {
  std::shared_ptr<Problem> P;
  std::string msg;
  int st = create_problem(family, degree, nv, nt, cells, rule, qdeg, FFG_BOUNDARY_NONE, nullptr, P,
                          msg);
  if (st) { *status = st; return; }
  if (n_dofs != P->topo.n_dofs || !rhs || !samples) { *status = FFG_INVALID_INPUT; return; }
  st = assemble(*P, verts, 0.0, 0.0, nullptr, nullptr, samples, nullptr, 0, false, 0, msg);
  if (st) { *status = st; return; }
  if (cudaMemcpy(rhs, P->rhs, sizeof(double) * (size_t)n_dofs, cudaMemcpyDeviceToHost) != cudaSuccess) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  *status = FFG_OK;
}

void ffg_assemble_tetra_lagrange_stiffness_csc(int nv, const double *verts, int nt, const int *tets,
                                               int degree, int rule, int qdeg, double stiffness,
                                               double mass, const double *cell_stiffness,
                                               const double *cell_mass, int64_t cap, int *n_dofs,
                                               int64_t *nnz, int64_t *col_ptr, int *row_ind,
                                               double *values, int *status) {
  full_csc(FFG_TETRA_LAGRANGE, degree, nv, verts, nt, tets, rule, qdeg, stiffness, mass,
           cell_stiffness, cell_mass, cap, n_dofs, nnz, col_ptr, row_ind, values, status);
}

// Tangent (JVP) of a stiffness/curl + mass CSC on the primal pattern: the
// element kernels run on the tangent weights, the column gather is the primal's.
static void tangent_csc(int family, int degree, int nv, const double *verts, int nt,
                        const int *cells, int rule, int qdeg, double ca, double cb,
                        const double *verts_dot, double ca_dot, double cb_dot, int64_t cap,
                        int *n_dofs, int64_t *nnz, int64_t *col_ptr, int *row_ind,
                        double *values_dot, int *status) {
  std::shared_ptr<Problem> P;
  std::string msg;
  if (!verts || !verts_dot) { *status = FFG_INVALID_INPUT; return; }
  int st = create_problem(family, degree, nv, nt, cells, rule, qdeg, FFG_BOUNDARY_NONE, nullptr, P,
                          msg);
  if (st) { *status = st; return; }
  const Topology &t = P->topo;
  if (n_dofs) *n_dofs = (int)t.n_dofs;
  if (nnz) *nnz = t.nnz();
  if (cap < t.nnz() || !col_ptr || !row_ind || !values_dot) { *status = FFG_CAPACITY; return; }
  double *vdot = nullptr;
  const size_t vbytes = sizeof(double) * 3 * (size_t)nv;
  if ((st = dalloc(&vdot, 3 * (size_t)nv))) { *status = st; return; }
  if (!P->csc_val && (st = dalloc(&P->csc_val, (size_t)std::max<int64_t>(t.nnz(), 1)))) {
    cudaFree(vdot);
    *status = st;
    return;
  }
  AssemblyInputs in;
  in.vertices = P->in_vertices;
  in.coef_a = ca;
  in.coef_b = cb;
  in.vertices_dot = vdot;
  in.coef_a_dot = ca_dot;
  in.coef_b_dot = cb_dot;
  int herr = 0;
  if (cudaMemcpy(P->in_vertices, verts, vbytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(vdot, verts_dot, vbytes, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(P->err, 0, sizeof(int)) != cudaSuccess) {
    st = FFG_CUDA_ERROR;
  } else {
    st = family == FFG_TETRA_LAGRANGE
             ? launch_lagrange_geometry_jvp(t, P->dt, P->in_vertices, vdot, ca, cb, ca_dot, cb_dot,
                                            P->geo, P->geo_stride, P->err, 0)
             : launch_nedelec(t, P->tab, P->dt, in, P->elem, P->cell_rhs, P->err, 0);
    if (!st)
      st = launch_columns(t, P->tab, P->dt, in, P->geo, P->geo_stride, P->cell_rhs, P->elem,
                          P->csc_col_ptr, P->csc_row, nullptr, P->csc_val, P->rhs, 0);
    if (!st) {
      if (cudaMemcpy(&herr, P->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = FFG_CUDA_ERROR;
      else if (herr)
        st = herr;
      else if (cudaMemcpy(values_dot, P->csc_val, sizeof(double) * (size_t)t.nnz(),
                          cudaMemcpyDeviceToHost) != cudaSuccess)
        st = FFG_CUDA_ERROR;
    }
  }
  cudaFree(vdot);
  if (st) { *status = st; return; }
  std::memcpy(col_ptr, t.col_ptr.data(), sizeof(int64_t) * t.col_ptr.size());
  std::memcpy(row_ind, t.row_idx.data(), sizeof(int) * t.row_idx.size());
  *status = FFG_OK;
}

// Adjoint (VJP) of a stiffness/curl + mass CSC: vertex and coefficient
// adjoints of a cotangent on the primal pattern; outputs start at zero.
static void adjoint_csc(int family, int degree, int nv, const double *verts, int nt,
                        const int *cells, int rule, int qdeg, double ca, double cb, int64_t nnz,
                        const double *values_bar, double *verts_bar, double *ca_bar,
                        double *cb_bar, int *status) {
  if (verts_bar && nv > 0) std::memset(verts_bar, 0, sizeof(double) * 3 * (size_t)nv);
  if (ca_bar) *ca_bar = 0.0;
  if (cb_bar) *cb_bar = 0.0;
  if (!verts || !values_bar || !verts_bar || !ca_bar || !cb_bar) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  std::shared_ptr<Problem> P;
  std::string msg;
  int st = create_problem(family, degree, nv, nt, cells, rule, qdeg, FFG_BOUNDARY_NONE, nullptr, P,
                          msg);
  if (st) { *status = st; return; }
  const Topology &t = P->topo;
  if (nnz != t.nnz()) { *status = FFG_INVALID_INPUT; return; }
  double *vb = nullptr, *dvbar = nullptr, *coef = nullptr;
  const size_t vcount = 3 * (size_t)nv;
  if ((st = dalloc(&vb, (size_t)std::max<int64_t>(nnz, 1))) || (st = dalloc(&dvbar, vcount)) ||
      (st = dalloc(&coef, 2))) {
    for (double *p : {vb, dvbar, coef})
      if (p) cudaFree(p);
    *status = st;
    return;
  }
  double hc[2] = {0.0, 0.0};
  int herr = 0;
  if (cudaMemcpy(P->in_vertices, verts, sizeof(double) * vcount, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(vb, values_bar, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemset(P->err, 0, sizeof(int)) != cudaSuccess) {
    st = FFG_CUDA_ERROR;
  } else {
    st = family == FFG_TETRA_LAGRANGE
             ? lagrange_vjp(t, P->dt, P->csc_col_ptr, P->csc_row, P->in_vertices, vb, ca, cb,
                            dvbar, coef, P->err, 0)
             : nedelec_vjp(t, P->tab, P->dt, P->csc_col_ptr, P->csc_row, P->in_vertices, vb, ca,
                           cb, P->elem, dvbar, coef, P->err, 0);
    if (!st) {
      if (cudaMemcpy(&herr, P->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = FFG_CUDA_ERROR;
      else if (herr)
        st = herr;
      else if (cudaMemcpy(verts_bar, dvbar, sizeof(double) * vcount, cudaMemcpyDeviceToHost) !=
                   cudaSuccess ||
               cudaMemcpy(hc, coef, sizeof(hc), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = FFG_CUDA_ERROR;
    }
  }
  for (double *p : {vb, dvbar, coef}) cudaFree(p);
  if (st) {
    std::memset(verts_bar, 0, sizeof(double) * vcount);
    *status = st;
    return;
  }
  *ca_bar = hc[0];
  *cb_bar = hc[1];
  *status = FFG_OK;
}

void ffg_assemble_tetra_lagrange_stiffness_csc_jvp(
    int nv, const double *verts, int nt, const int *tets, int degree, int rule, int qdeg,
    double stiffness, double mass, const double *verts_dot, double stiffness_dot,
    double mass_dot, int64_t cap, int *n_dofs, int64_t *nnz, int64_t *col_ptr, int *row_ind,
    double *values_dot, int *status) {
  tangent_csc(FFG_TETRA_LAGRANGE, degree, nv, verts, nt, tets, rule, qdeg, stiffness, mass,
              verts_dot, stiffness_dot, mass_dot, cap, n_dofs, nnz, col_ptr, row_ind, values_dot,
              status);
}

void ffg_assemble_tetra_lagrange_stiffness_csc_vjp(
    int nv, const double *verts, int nt, const int *tets, int degree, int rule, int qdeg,
    double stiffness, double mass, int64_t nnz, const double *values_bar, double *verts_bar,
    double *stiffness_bar, double *mass_bar, int *status) {
  adjoint_csc(FFG_TETRA_LAGRANGE, degree, nv, verts, nt, tets, rule, qdeg, stiffness, mass, nnz,
              values_bar, verts_bar, stiffness_bar, mass_bar, status);
}

void ffg_assemble_tetra_nedelec_curl_mass_csc_jvp(
    int nv, const double *verts, int nt, const int *tets, int order, double curl, double mass,
    const double *verts_dot, double curl_dot, double mass_dot, int64_t cap, int *n_dofs,
    int64_t *nnz, int64_t *col_ptr, int *row_ind, double *values_dot, int *status) {
  tangent_csc(FFG_TETRA_NEDELEC, order, nv, verts, nt, tets, 0, 0, curl, mass, verts_dot, curl_dot,
              mass_dot, cap, n_dofs, nnz, col_ptr, row_ind, values_dot, status);
}

void ffg_assemble_tetra_nedelec_curl_mass_csc_vjp(
    int nv, const double *verts, int nt, const int *tets, int order, double curl, double mass,
    int64_t nnz, const double *values_bar, double *verts_bar, double *curl_bar, double *mass_bar,
    int *status) {
  adjoint_csc(FFG_TETRA_NEDELEC, order, nv, verts, nt, tets, 0, 0, curl, mass, nnz, values_bar,
              verts_bar, curl_bar, mass_bar, status);
}

void ffg_assemble_tetra_lagrange_scalar_load_samples(int nv, const double *verts, int nt,
                                                     const int *tets, int degree, int rule,
                                                     int qdeg, const double *samples, int n_dofs,
                                                     double *rhs, int *status) {
  full_load(FFG_TETRA_LAGRANGE, degree, nv, verts, nt, tets, rule, qdeg, samples, n_dofs, rhs,
            status);
}

void ffg_assemble_tetra_nedelec_curl_mass_csc(int nv, const double *verts, int nt, const int *tets,
                                              int order, double curl, double mass,
                                              const double *cell_curl, const double *cell_mass,
                                              int64_t cap, int *n_dofs, int64_t *nnz,
                                              int64_t *col_ptr, int *row_ind, double *values,
                                              int *status) {
  full_csc(FFG_TETRA_NEDELEC, order, nv, verts, nt, tets, 0, 0, curl, mass, cell_curl, cell_mass,
           cap, n_dofs, nnz, col_ptr, row_ind, values, status);
}

void ffg_assemble_tetra_nedelec_weighted_csc(int nv, const double *verts, int nt,
                                             const int *tets, int order,
                                             const double *cell_tensors, double mass,
                                             int64_t cap, int *n_dofs, int64_t *nnz,
                                             int64_t *col_ptr, int *row_ind, double *values,
                                             int *status) {
  if (!verts || !cell_tensors || nt < 1) { *status = FFG_INVALID_INPUT; return; }
  if (!symmetric_tensors(nt, cell_tensors)) { *status = FFG_INVALID_INPUT; return; }
  std::shared_ptr<Problem> P;
  std::string msg;
  int st = create_problem(FFG_TETRA_NEDELEC, order, nv, nt, tets, 0, 0, FFG_BOUNDARY_NONE, nullptr,
                          P, msg);
  if (st) { *status = st; return; }
  if (n_dofs) *n_dofs = (int)P->topo.n_dofs;
  if (nnz) *nnz = P->topo.nnz();
  if (cap < P->topo.nnz() || !col_ptr || !row_ind || !values) { *status = FFG_CAPACITY; return; }
  if ((st = dalloc(&P->cell_tensor, 9 * (size_t)nt)) || (st = dalloc(&P->geo_w, 12 * (size_t)nt))) {
    *status = st;
    return;
  }
  if (cudaMemcpy(P->cell_tensor, cell_tensors, sizeof(double) * 9 * (size_t)nt,
                 cudaMemcpyHostToDevice) != cudaSuccess) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  st = assemble(*P, verts, 1.0, mass, nullptr, nullptr, nullptr, nullptr, 0, false, 0, msg);
  if (st) { *status = st; return; }
  std::memcpy(col_ptr, P->topo.col_ptr.data(), sizeof(int64_t) * P->topo.col_ptr.size());
  std::memcpy(row_ind, P->topo.row_idx.data(), sizeof(int) * P->topo.row_idx.size());
  if (cudaMemcpy(values, P->csc_val, sizeof(double) * (size_t)P->topo.nnz(),
                 cudaMemcpyDeviceToHost) != cudaSuccess) {
    *status = FFG_CUDA_ERROR;
    return;
  }
  *status = FFG_OK;
}

// Complex PML curl-curl CSC: the Nedelec element kernel on the real and on
// the imaginary parts of the PML weights, each gathered by the column kernel.
static void pml_csc(bool curvilinear, int nv, const double *verts, int nt, const int *tets,
                    int order, const double *stretch, double wave, int64_t cap, int *n_dofs,
                    int64_t *nnz, int64_t *col_ptr, int *row_ind, double *values, int *status) {
  if (!verts || !stretch || !(wave > 0.0)) { *status = FFG_INVALID_INPUT; return; }
  std::shared_ptr<Problem> P;
  std::string msg;
  int st = create_problem(FFG_TETRA_NEDELEC, order, nv, nt, tets, 0, 0, FFG_BOUNDARY_NONE, nullptr,
                          P, msg);
  if (st) { *status = st; return; }
  const Topology &t = P->topo;
  if (n_dofs) *n_dofs = (int)t.n_dofs;
  if (nnz) *nnz = t.nnz();
  if (cap < t.nnz() || !col_ptr || !row_ind || !values) { *status = FFG_CAPACITY; return; }
  const size_t sw = curvilinear ? 18 : 6;
  const size_t nc = (size_t)nt, nz = (size_t)std::max<int64_t>(t.nnz(), 1);
  double *dstretch = nullptr, *geo_re = nullptr, *geo_im = nullptr, *val_re = nullptr,
         *val_im = nullptr, *out = nullptr;
  auto release = [&]() {
    for (double *p : {dstretch, geo_re, geo_im, val_re, val_im, out})
      if (p) cudaFree(p);
  };
  if ((st = dalloc(&dstretch, sw * nc)) || (st = dalloc(&geo_re, 12 * nc)) ||
      (st = dalloc(&geo_im, 12 * nc)) || (st = dalloc(&val_re, nz)) ||
      (st = dalloc(&val_im, nz)) || (st = dalloc(&out, 2 * nz))) {
    release();
    *status = st;
    return;
  }
  int herr = 0;
  if (cudaMemcpy(P->in_vertices, verts, sizeof(double) * 3 * (size_t)nv, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemcpy(dstretch, stretch, sizeof(double) * sw * nc, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemset(P->err, 0, sizeof(int)) != cudaSuccess) {
    st = FFG_CUDA_ERROR;
  } else {
    st = launch_pml_weights(t, P->dt, P->in_vertices, dstretch, curvilinear, wave, geo_re, geo_im,
                            P->err, 0);
    for (int part = 0; part < 2 && !st; ++part) {
      AssemblyInputs in;
      in.vertices = P->in_vertices;
      in.geo_override = part == 0 ? geo_re : geo_im;
      st = launch_nedelec(t, P->tab, P->dt, in, P->elem, P->cell_rhs, P->err, 0);
      if (!st)
        st = launch_columns(t, P->tab, P->dt, in, P->geo, P->geo_stride, P->cell_rhs, P->elem,
                            P->csc_col_ptr, P->csc_row, nullptr, part == 0 ? val_re : val_im,
                            P->rhs, 0);
    }
    if (!st) st = launch_interleave(t.nnz(), val_re, val_im, out, 0);
    if (!st) {
      if (cudaMemcpy(&herr, P->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        st = FFG_CUDA_ERROR;
      else if (herr)
        st = herr;
      else if (cudaMemcpy(values, out, sizeof(double) * 2 * (size_t)t.nnz(),
                          cudaMemcpyDeviceToHost) != cudaSuccess)
        st = FFG_CUDA_ERROR;
    }
  }
  release();
  if (st) { *status = st; return; }
  std::memcpy(col_ptr, t.col_ptr.data(), sizeof(int64_t) * t.col_ptr.size());
  std::memcpy(row_ind, t.row_idx.data(), sizeof(int) * t.row_idx.size());
  *status = FFG_OK;
}

void ffg_assemble_tetra_nedelec_pml_csc(int nv, const double *verts, int nt, const int *tets,
                                        int order, const double *stretch, double wave_number,
                                        int64_t cap, int *n_dofs, int64_t *nnz, int64_t *col_ptr,
                                        int *row_ind, double *values, int *status) {
  pml_csc(false, nv, verts, nt, tets, order, stretch, wave_number, cap, n_dofs, nnz, col_ptr,
          row_ind, values, status);
}

void ffg_assemble_tetra_nedelec_curvilinear_pml_csc(int nv, const double *verts, int nt,
                                                    const int *tets, int order,
                                                    const double *stretch, double wave_number,
                                                    int64_t cap, int *n_dofs, int64_t *nnz,
                                                    int64_t *col_ptr, int *row_ind,
                                                    double *values, int *status) {
  pml_csc(true, nv, verts, nt, tets, order, stretch, wave_number, cap, n_dofs, nnz, col_ptr,
          row_ind, values, status);
}

void ffg_assemble_tetra_nedelec_vector_load_samples(int nv, const double *verts, int nt,
                                                    const int *tets, int order,
                                                    const double *samples, int n_dofs, double *rhs,
                                                    int *status) {
  full_load(FFG_TETRA_NEDELEC, order, nv, verts, nt, tets, 0, 0, samples, n_dofs, rhs, status);
}

void ffg_assemble_triangle_lagrange_csc(int nv, const double *verts, int nt, const int *tris,
                                        int degree, int qdeg, double stiffness, double mass,
                                        const double *cell_stiffness, const double *cell_mass,
                                        int64_t cap, int *n_dofs, int64_t *nnz, int64_t *col_ptr,
                                        int *row_ind, double *values, int *status) {
  full_csc(FFG_TRIANGLE_LAGRANGE, degree, nv, verts, nt, tris, 0, qdeg, stiffness, mass,
           cell_stiffness, cell_mass, cap, n_dofs, nnz, col_ptr, row_ind, values, status);
}

void ffg_assemble_triangle_lagrange_load_samples(int nv, const double *verts, int nt,
                                                 const int *tris, int degree, int qdeg,
                                                 const double *samples, int n_dofs, double *rhs,
                                                 int *status) {
  full_load(FFG_TRIANGLE_LAGRANGE, degree, nv, verts, nt, tris, 0, qdeg, samples, n_dofs, rhs,
            status);
}

void ffg_assemble_scalar_p1_csc(int nv, const double *verts, int nt, const int *tris, double mass,
                                double stiffness, const double *cell_stiffness, int64_t cap,
                                int64_t *nnz, int64_t *col_ptr, int *row_ind, double *values,
                                int *status) {
  int nd = 0;
  full_csc(FFG_TRIANGLE_P1, 1, nv, verts, nt, tris, 0, 0, stiffness, mass, cell_stiffness, nullptr,
           cap, &nd, nnz, col_ptr, row_ind, values, status);
}

// ------------------------------------------------------------------- solve_sparse

void ffg_solve_sparse(int n, int64_t nnz, const int64_t *col_ptr, const int *row_ind,
                      const double *values, const double *b, double *x,
                      const ffg_solver_options *opts, ffg_solver_stats *stats, int *status) {
  ffg_solver_options o;
  if (n < 1 || !col_ptr || !row_ind || !values || !b || !x || check_options(opts, o) ||
      col_ptr[n] != nnz || col_ptr[0] != 0) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  int st = device_ready();
  if (st) { *status = st; return; }
  HostCsr h;
  if (!csc_to_csr(n, col_ptr, row_ind, values, h)) { *status = FFG_INVALID_INPUT; return; }
  int grid = 0;
  if ((st = pcg_grid_size(&grid))) { *status = st; return; }
  HostSell hs;
  DeviceSell S;
  if ((st = upload_sell_with_values(h, grid, o.preconditioner != 0, hs, S))) {
    free_sell(S);
    *status = st;
    return;
  }
  // b and x in the solver's row order
  std::vector<double> bn(n), xn(n);
  for (int i = 0; i < n; ++i) { bn[hs.iperm[i]] = b[i]; xn[hs.iperm[i]] = x[i]; }
  double *db = nullptr, *dx = nullptr;
  if (dalloc(&db, n) || dalloc(&dx, n)) {
    cudaFree(db); cudaFree(dx); free_sell(S);
    *status = FFG_OUT_OF_MEMORY;
    return;
  }
  cudaMemcpy(db, bn.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dx, xn.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
  SolveWork w;
  std::string msg;
  ffg_solver_stats local;
  std::memset(&local, 0, sizeof(local));
  if (!(st = solve_work_alloc(w, n, grid))) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    if (o.precision == FFG_PRECISION_MIXED16) st = sell_half(S, 0);
    if (!st) st = pcg_solve(S, db, dx, o, w, &local, 0, msg);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    local.solve_seconds = ms * 1e-3;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (!st) {
    cudaMemcpy(xn.data(), dx, sizeof(double) * n, cudaMemcpyDeviceToHost);
    for (int i = 0; i < n; ++i) x[i] = xn[hs.iperm[i]];
  }
  solve_work_free(w);
  free_sell(S);
  cudaFree(db);
  cudaFree(dx);
  report(o.verbosity, msg);
  if (stats) *stats = local;
  *status = solve_status(st, local);
}

void ffg_csc_matvec(int n, int64_t nnz, const int64_t *col_ptr, const int *row_ind,
                    const double *values, const double *x, double *y, int *status) {
  if (n < 1 || !col_ptr || !row_ind || !values || !x || !y || col_ptr[n] != nnz) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  int st = device_ready();
  if (st) { *status = st; return; }
  HostCsr h;
  if (!csc_to_csr(n, col_ptr, row_ind, values, h)) { *status = FFG_INVALID_INPUT; return; }
  DeviceCsrArrays D;
  double *dx = nullptr, *dy = nullptr;
  if (dalloc(&D.rp, h.rp.size()) || dalloc(&D.ci, h.col.size()) || dalloc(&D.v, h.val.size()) ||
      dalloc(&dx, n) || dalloc(&dy, n)) {
    cudaFree(dx); cudaFree(dy);
    *status = FFG_OUT_OF_MEMORY;
    return;
  }
  cudaMemcpy(D.rp, h.rp.data(), sizeof(int64_t) * h.rp.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(D.ci, h.col.data(), sizeof(int) * h.col.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(D.v, h.val.data(), sizeof(double) * h.val.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice);
  st = csr_spmv64(n, D.rp, D.ci, D.v, dx, dy, 0);
  if (!st && cudaMemcpy(y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    st = FFG_CUDA_ERROR;
  cudaFree(dx);
  cudaFree(dy);
  *status = st;
}

}  // extern "C"
