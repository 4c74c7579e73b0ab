// Solution evaluation and point probes (sm_100a): batched gather-evaluate
// kernels for post-processing requests on a solved problem.
//
//  * evaluate: one warp per query (cell, point).  The point is a reference
//    point, or a physical point mapped back by the cell's inverse Jacobian
//    (invert_tetra_affine_map, src/geometry/tetra_affine_map.f90:15-33).
//    Lagrange: value and gradient of evaluate_tetra_lagrange_solution_prepared
//    (src/solvers/fortfem_tetra_lagrange_solver_3d.f90:491-528).  Nedelec:
//    field and curl of the oriented local DoFs T u(gd), covariant map (the
//    per-cell body of evaluate_box_solution_order,
//    src/solvers/fortfem_magnetic_box_3d.f90:313-334).
//  * probe: physical points located without a cell hint.  The reference scans
//    every cell per point (evaluate_box_solution_order :269-343); here a
//    uniform grid of bins over the mesh's bounding box holds, per bin, the
//    cells whose (slightly expanded) bounding boxes meet it, in ascending
//    cell order (stable radix sort of (bin, cell) pairs).  A point's warp
//    walks its bin's cells in that order with the reference's containment
//    test (det > 0, reference coordinates >= -1e-12, sum <= 1 + 1e-12) and
//    averages the contributions (or stops at the first, as probe_box_az /
//    probe_box_curl :345-440 do), so it sums the same cells in the same
//    order as the reference's scan.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>

#include "ffg_internal.h"
#include "tet_geometry.h"

namespace ffg {

namespace {

constexpr int kWarpsPerBlock = 8;
constexpr int kMaxNedelecBasis = 216;  // order 6

struct EvalSpace {
  int family = 0, degree = 0, nb = 0;
  const int *gd = nullptr;         // nb per cell
  const int *lag_idx = nullptr;    // Lagrange: 4 barycentric indices per basis function
  const int *terms = nullptr;      // Nedelec: 10 ints per candidate
  const double *coef = nullptr;    // Nedelec: nb x nb, (candidate, basis) column-major
  const int8_t *edge_sign = nullptr;
  const uint8_t *face_perm = nullptr;
  const double *face_blocks = nullptr;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

// Value and physical gradient of the Lagrange solution on cell c at xi
// (same result on every lane): sum u_i phi_i and J^-T sum u_i grad phi_i,
// with phi_i the cardinal-factor basis of evaluate_tetra_lagrange
// (tetra_lagrange_arbitrary_order.f90:68-116).
__device__ void warp_lagrange(const EvalSpace &E, int c, const double *xi, const double *Ji,
                              const double *__restrict__ u, double out[4]) {
  const int lane = threadIdx.x & 31;
  const int p = E.degree, nb = E.nb;
  const double bary[4] = {1.0 - (xi[0] + xi[1] + xi[2]), xi[0], xi[1], xi[2]};
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = lane; i < nb; i += 32) {
    double f[4], d[4];
    for (int comp = 0; comp < 4; ++comp) {
      const int n = E.lag_idx[4 * i + comp];
      double fact = 1.0, v = 1.0, dv = 0.0;
      for (int q = 2; q <= n; ++q) fact *= q;
      for (int q = 0; q < n; ++q) v *= (p * bary[comp] - q);
      for (int dq = 0; dq < n; ++dq) {
        double term = p;
        for (int q = 0; q < n; ++q)
          if (q != dq) term *= (p * bary[comp] - q);
        dv += term;
      }
      f[comp] = v / fact;
      d[comp] = dv / fact;
    }
    double ld[4];
    for (int comp = 0; comp < 4; ++comp) {
      ld[comp] = d[comp];
      for (int o = 0; o < 4; ++o)
        if (o != comp) ld[comp] *= f[o];
    }
    const double ui = u[E.gd[(size_t)nb * c + i]];
    acc[0] += ui * (f[0] * f[1] * f[2] * f[3]);
    for (int a = 0; a < 3; ++a) acc[1 + a] += ui * (ld[a + 1] - ld[0]);
  }
  for (int a = 0; a < 4; ++a) acc[a] = warp_sum(acc[a]);
  out[0] = acc[0];
  for (int i = 0; i < 3; ++i)
    out[1 + i] = Ji[3 * i] * acc[1] + Ji[3 * i + 1] * acc[2] + Ji[3 * i + 2] * acc[3];
}

// Field and curl of the Nedelec solution on cell c at xi (same on every
// lane).  ld (nb doubles of this warp's shared memory) receives the oriented
// local DoFs T u(gd); the field is sum_cand (sum_i C[cand, i] ld_i) cand(xi).
__device__ void warp_nedelec(const EvalSpace &E, int c, const double *xi, const double *J,
                             double det, const double *Ji, const double *__restrict__ u,
                             double *ld, double out[6]) {
  const int lane = threadIdx.x & 31;
  const int k = E.degree, n = E.nb, fdc = k * (k - 1), edge_end = 6 * k;
  const int *ge = E.gd + (size_t)n * c;
  const int8_t *sg = E.edge_sign + 6 * (size_t)c;
  const uint8_t *fp = E.face_perm + 4 * (size_t)c;
  __syncwarp();
  for (int i = lane; i < n; i += 32) {
    double s;
    if (i < edge_end) {
      s = u[ge[i]];
      if (sg[i / k] == -1 && ((i % k) % 2) == 0) s = -s;
    } else if (i < edge_end + 4 * fdc) {
      // T[st+r][st+m] = B[m*fdc + r] for the face's block B
      const int f = (i - edge_end) / fdc, r = (i - edge_end) % fdc, st = edge_end + f * fdc;
      const double *B = E.face_blocks + (size_t)fp[f] * fdc * fdc;
      s = 0.0;
      for (int m = 0; m < fdc; ++m) s += B[m * fdc + r] * u[ge[st + m]];
    } else {
      s = u[ge[i]];
    }
    ld[i] = s;
  }
  __syncwarp();
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int cand = lane; cand < n; cand += 32) {
    double w = 0.0;
    for (int i = 0; i < n; ++i) w += E.coef[cand + (size_t)n * i] * ld[i];
    double cv[3] = {0.0, 0.0, 0.0}, cc[3] = {0.0, 0.0, 0.0};
    for (int t = 0; t < 2; ++t) {
      const int *tm = E.terms + 10 * cand + 5 * t;
      const int comp = tm[0];
      if (comp < 0) continue;
      const double coef = tm[1];
      const int pw[3] = {tm[2], tm[3], tm[4]};
      cv[comp] += coef * ipow(xi[0], pw[0]) * ipow(xi[1], pw[1]) * ipow(xi[2], pw[2]);
      double der[3];
      for (int dd = 0; dd < 3; ++dd) {
        if (pw[dd] == 0) { der[dd] = 0.0; continue; }
        int r[3] = {pw[0], pw[1], pw[2]};
        r[dd] -= 1;
        der[dd] = coef * pw[dd] * ipow(xi[0], r[0]) * ipow(xi[1], r[1]) * ipow(xi[2], r[2]);
      }
      if (comp == 0) { cc[1] += der[2]; cc[2] -= der[1]; }
      if (comp == 1) { cc[0] -= der[2]; cc[2] += der[0]; }
      if (comp == 2) { cc[0] += der[1]; cc[1] -= der[0]; }
    }
    for (int a = 0; a < 3; ++a) {
      acc[a] += w * cv[a];
      acc[3 + a] += w * cc[a];
    }
  }
  for (int a = 0; a < 6; ++a) acc[a] = warp_sum(acc[a]);
  // covariant map: values J^-T v, curls J c / det
  for (int i = 0; i < 3; ++i) {
    out[i] = Ji[3 * i] * acc[0] + Ji[3 * i + 1] * acc[1] + Ji[3 * i + 2] * acc[2];
    out[3 + i] = (J[i] * acc[3] + J[i + 3] * acc[4] + J[i + 6] * acc[5]) / det;
  }
}

__device__ __forceinline__ void map_to_reference(const double *Ji, const double *v0,
                                                 const double *x, double *xi) {
  for (int i = 0; i < 3; ++i)
    xi[i] = Ji[i] * (x[0] - v0[0]) + Ji[i + 3] * (x[1] - v0[1]) + Ji[i + 6] * (x[2] - v0[2]);
}

// the basis evaluations' own point test: barycentric coordinates >= -64 eps
__device__ __forceinline__ bool in_reference(const double *xi) {
  const double tol = 64.0 * kEps;
  return xi[0] >= -tol && xi[1] >= -tol && xi[2] >= -tol && 1.0 - (xi[0] + xi[1] + xi[2]) >= -tol;
}

// Nedelec's evaluate_tetra_nedelec_first_kind tests sum <= 1 + 64 eps
__device__ __forceinline__ bool in_reference_nedelec(const double *xi) {
  const double tol = 64.0 * kEps;
  return xi[0] >= -tol && xi[1] >= -tol && xi[2] >= -tol && xi[0] + xi[1] + xi[2] <= 1.0 + tol;
}

__device__ __forceinline__ int out_width(int family) { return family == FFG_TETRA_NEDELEC ? 3 : 1; }

__global__ void cells_valid_kernel(int n_cells, const int *__restrict__ cells,
                                   const double *__restrict__ verts, int *err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  double J[9], v0[3];
  tet_jacobian(cells, verts, c, J, v0);
  if (!valid_jacobian(J, det3(J))) atomicCAS(err, 0, FFG_INVALID_INPUT);
}

// One warp per query.  qstatus: 0, or FFG_INVALID_INPUT for a cell index out
// of range, a degenerate cell or a point outside the reference cell.
__global__ void evaluate_kernel(EvalSpace E, int n_cells, const int *__restrict__ cells,
                                const double *__restrict__ verts, const double *__restrict__ u,
                                int n_queries, const int *__restrict__ qcell,
                                const double *__restrict__ qpoint, int physical,
                                double *__restrict__ values, double *__restrict__ derivs,
                                int *__restrict__ qstatus) {
  __shared__ double ld_all[kWarpsPerBlock][kMaxNedelecBasis];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = blockIdx.x * kWarpsPerBlock + warp;
  if (q >= n_queries) return;  // uniform across the warp
  const int wv = out_width(E.family);
  const int c = qcell[q];
  double out[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int st = FFG_INVALID_INPUT;
  if (c >= 0 && c < n_cells) {
    double J[9], Ji[9], v0[3], xi[3];
    tet_jacobian(cells, verts, c, J, v0);
    const double det = det3(J);
    if (valid_jacobian(J, det)) {
      inv3(J, det, Ji);
      const double *x = qpoint + 3 * (size_t)q;
      if (physical) {
        map_to_reference(Ji, v0, x, xi);
      } else {
        xi[0] = x[0]; xi[1] = x[1]; xi[2] = x[2];
      }
      if (E.family == FFG_TETRA_NEDELEC ? in_reference_nedelec(xi) : in_reference(xi)) {
        if (E.family == FFG_TETRA_NEDELEC)
          warp_nedelec(E, c, xi, J, det, Ji, u, ld_all[warp], out);
        else
          warp_lagrange(E, c, xi, Ji, u, out);
        st = FFG_OK;
      }
    }
  }
  if (lane == 0) {
    for (int a = 0; a < wv; ++a) values[(size_t)wv * q + a] = out[a];
    for (int a = 0; a < 3; ++a) derivs[3 * (size_t)q + a] = out[wv + a];
    if (qstatus) qstatus[q] = st;
  }
}

// ------------------------------------------------------------------ bins
struct BinGrid {
  double lo[3], inv_h[3];
  int dims[3];
  double margin;
};

__device__ __forceinline__ int bin_axis(const BinGrid &G, int a, double x) {
  const double t = floor((x - G.lo[a]) * G.inv_h[a]);
  return (int)fmin(fmax(t, 0.0), (double)(G.dims[a] - 1));
}

// Min / max of the vertex coordinates: one CTA, fixed order.
__global__ void bbox_kernel(int n_vertices, const double *__restrict__ verts, double *out) {
  __shared__ double lo[3][256], hi[3][256];
  const int t = threadIdx.x;
  double l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int v = t; v < n_vertices; v += blockDim.x)
    for (int a = 0; a < 3; ++a) {
      const double x = verts[3 * (size_t)v + a];
      l[a] = fmin(l[a], x);
      h[a] = fmax(h[a], x);
    }
  for (int a = 0; a < 3; ++a) {
    lo[a][t] = l[a];
    hi[a][t] = h[a];
  }
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (t < w)
      for (int a = 0; a < 3; ++a) {
        lo[a][t] = fmin(lo[a][t], lo[a][t + w]);
        hi[a][t] = fmax(hi[a][t], hi[a][t + w]);
      }
    __syncthreads();
  }
  if (t == 0)
    for (int a = 0; a < 3; ++a) {
      out[a] = lo[a][0];
      out[3 + a] = hi[a][0];
    }
}

__device__ __forceinline__ void cell_bin_range(const BinGrid &G, const int *cells,
                                               const double *verts, int c, int *b0, int *b1) {
  const int4 t = *reinterpret_cast<const int4 *>(cells + 4 * (size_t)c);
  const int vid[4] = {t.x, t.y, t.z, t.w};
  for (int a = 0; a < 3; ++a) {
    double l = INFINITY, h = -INFINITY;
    for (int n = 0; n < 4; ++n) {
      const double x = verts[3 * (size_t)vid[n] + a];
      l = fmin(l, x);
      h = fmax(h, x);
    }
    b0[a] = bin_axis(G, a, l - G.margin);
    b1[a] = bin_axis(G, a, h + G.margin);
  }
}

__global__ void cell_bin_count_kernel(BinGrid G, int n_cells, const int *__restrict__ cells,
                                      const double *__restrict__ verts, int *__restrict__ count) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  int b0[3], b1[3];
  cell_bin_range(G, cells, verts, c, b0, b1);
  count[c] = (b1[0] - b0[0] + 1) * (b1[1] - b0[1] + 1) * (b1[2] - b0[2] + 1);
}

__global__ void cell_bin_fill_kernel(BinGrid G, int n_cells, const int *__restrict__ cells,
                                     const double *__restrict__ verts,
                                     const int64_t *__restrict__ offset, int *__restrict__ key,
                                     int *__restrict__ val) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  int b0[3], b1[3];
  cell_bin_range(G, cells, verts, c, b0, b1);
  int64_t o = offset[c];
  for (int z = b0[2]; z <= b1[2]; ++z)
    for (int y = b0[1]; y <= b1[1]; ++y)
      for (int x = b0[0]; x <= b1[0]; ++x) {
        key[o] = x + G.dims[0] * (y + G.dims[1] * z);
        val[o] = c;
        ++o;
      }
}

__global__ void widen_kernel(int n, const int *__restrict__ in, int64_t *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

// One warp per point: walk the point's bin in ascending cell order.
// counts[q]: contributing cells; -1 when the basis evaluation rejects the
// point on a containing cell (the reference's probe then fails).
__global__ void probe_kernel(EvalSpace E, BinGrid G, int64_t n_pairs, const int *__restrict__ key,
                             const int *__restrict__ val, const int *__restrict__ cells,
                             const double *__restrict__ verts, const double *__restrict__ u,
                             int n_points, const double *__restrict__ points, int first_only,
                             double *__restrict__ values, double *__restrict__ derivs,
                             int *__restrict__ counts) {
  __shared__ double ld_all[kWarpsPerBlock][kMaxNedelecBasis];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = blockIdx.x * kWarpsPerBlock + warp;
  if (q >= n_points) return;
  const int wv = out_width(E.family);
  const double x[3] = {points[3 * (size_t)q], points[3 * (size_t)q + 1], points[3 * (size_t)q + 2]};
  const int bin = bin_axis(G, 0, x[0]) + G.dims[0] * (bin_axis(G, 1, x[1]) + G.dims[1] * bin_axis(G, 2, x[2]));
  int64_t lo = 0, hi = n_pairs;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (key[mid] < bin) lo = mid + 1; else hi = mid;
  }
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int found = 0;
  for (int64_t p = lo; p < n_pairs && key[p] == bin; ++p) {
    const int c = val[p];
    double J[9], Ji[9], v0[3], xi[3];
    tet_jacobian(cells, verts, c, J, v0);
    const double det = det3(J);
    if (det <= 0.0) continue;
    inv3(J, det, Ji);
    map_to_reference(Ji, v0, x, xi);
    if (xi[0] < -1.0e-12 || xi[1] < -1.0e-12 || xi[2] < -1.0e-12) continue;
    if (xi[0] + xi[1] + xi[2] > 1.0 + 1.0e-12) continue;
    if (!(E.family == FFG_TETRA_NEDELEC ? in_reference_nedelec(xi) : in_reference(xi))) {
      found = -1;
      break;
    }
    double out[6];
    if (E.family == FFG_TETRA_NEDELEC)
      warp_nedelec(E, c, xi, J, det, Ji, u, ld_all[warp], out);
    else
      warp_lagrange(E, c, xi, Ji, u, out);
    for (int a = 0; a < wv + 3; ++a) acc[a] += out[a];
    ++found;
    if (first_only) break;
  }
  if (lane == 0) {
    const double scale = found > 0 ? 1.0 / found : 0.0;
    for (int a = 0; a < wv; ++a) values[(size_t)wv * q + a] = found > 0 ? acc[a] * scale : 0.0;
    for (int a = 0; a < 3; ++a) derivs[3 * (size_t)q + a] = found > 0 ? acc[wv + a] * scale : 0.0;
    counts[q] = found;
  }
}

inline int blocks_for(int64_t n, int t) { return (int)((n + t - 1) / t); }

struct Buf {
  void *p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t bytes) {
    return cudaMalloc(&p, std::max<size_t>(bytes, 16)) == cudaSuccess ? FFG_OK : FFG_OUT_OF_MEMORY;
  }
};

EvalSpace make_space(const Topology &t, const DeviceTopology &dt, const EvalTables &et) {
  EvalSpace E;
  E.family = t.family;
  E.degree = t.degree;
  E.nb = t.nb;
  E.gd = dt.gd;
  E.lag_idx = et.lag_idx;
  E.terms = et.terms;
  E.coef = et.coef;
  E.edge_sign = dt.edge_sign;
  E.face_perm = dt.face_perm;
  E.face_blocks = dt.face_blocks;
  return E;
}

}  // namespace

int evaluate_solution(const Topology &t, const DeviceTopology &dt, const EvalTables &et,
                      const double *vertices, const double *u, int n_queries, const int *qcell,
                      const double *qpoint, int physical, double *values, double *derivs,
                      int *qstatus, int *err, cudaStream_t s) {
  if (t.family != FFG_TETRA_LAGRANGE && t.family != FFG_TETRA_NEDELEC) return FFG_INVALID_INPUT;
  if (t.family == FFG_TETRA_NEDELEC && t.nb > kMaxNedelecBasis) return FFG_INVALID_INPUT;
  if (n_queries <= 0) return FFG_OK;
  // the Lagrange evaluator accepts a mesh only when every cell is valid
  // (initialize_tetra_lagrange_solution_evaluator, :464-479)
  if (t.family == FFG_TETRA_LAGRANGE)
    cells_valid_kernel<<<blocks_for(t.n_cells, 128), 128, 0, s>>>(t.n_cells, dt.cells, vertices,
                                                                  err);
  evaluate_kernel<<<blocks_for(n_queries, kWarpsPerBlock), 32 * kWarpsPerBlock, 0, s>>>(
      make_space(t, dt, et), t.n_cells, dt.cells, vertices, u, n_queries, qcell, qpoint, physical,
      values, derivs, qstatus);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

int probe_solution(const Topology &t, const DeviceTopology &dt, const EvalTables &et,
                   const double *vertices, const double *u, int n_points, const double *points,
                   int first_only, double *values, double *derivs, int *counts, cudaStream_t s) {
  if (t.family != FFG_TETRA_LAGRANGE && t.family != FFG_TETRA_NEDELEC) return FFG_INVALID_INPUT;
  if (t.family == FFG_TETRA_NEDELEC && t.nb > kMaxNedelecBasis) return FFG_INVALID_INPUT;
  if (n_points <= 0) return FFG_OK;
  const int nc = t.n_cells;
  // grid over the bounding box: about one bin per 4 cells, cubes where possible
  Buf box, count, offset, offset64, keys_in, vals_in, keys, vals, temp;
  int st;
  if ((st = box.alloc(6 * sizeof(double)))) return st;
  bbox_kernel<<<1, 256, 0, s>>>(t.n_vertices, vertices, (double *)box.p);
  double hb[6];
  if (cudaMemcpyAsync(hb, box.p, sizeof(hb), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  double ext[3], emax = 0.0;
  for (int a = 0; a < 3; ++a) {
    ext[a] = hb[3 + a] - hb[a];
    if (!std::isfinite(ext[a])) return FFG_INVALID_INPUT;
    emax = std::max(emax, ext[a]);
  }
  if (emax <= 0.0) emax = 1.0;
  for (int a = 0; a < 3; ++a) ext[a] = std::max(ext[a], 1e-9 * emax);
  const double target = std::max(1.0, nc / 4.0);
  const double h = std::cbrt(ext[0] * ext[1] * ext[2] / target);
  BinGrid G;
  int64_t n_bins = 1;
  for (int a = 0; a < 3; ++a) {
    G.dims[a] = (int)std::min(1024.0, std::max(1.0, std::ceil(ext[a] / h)));
    G.lo[a] = hb[a];
    G.inv_h[a] = G.dims[a] / ext[a];
    n_bins *= G.dims[a];
  }
  G.margin = 1e-9 * emax;
  if ((st = count.alloc(sizeof(int) * nc)) || (st = offset64.alloc(sizeof(int64_t) * (nc + 1))) ||
      (st = offset.alloc(sizeof(int64_t) * (nc + 1))))
    return st;
  cell_bin_count_kernel<<<blocks_for(nc, 128), 128, 0, s>>>(G, nc, dt.cells, vertices,
                                                            (int *)count.p);
  widen_kernel<<<blocks_for(nc, 256), 256, 0, s>>>(nc, (const int *)count.p,
                                                   (int64_t *)offset64.p);
  size_t tb = 0;
  if (cub::DeviceScan::ExclusiveSum(nullptr, tb, (const int64_t *)offset64.p,
                                    (int64_t *)offset.p, nc + 1, s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if ((st = temp.alloc(tb))) return st;
  // offset64[nc] is left as it came from the allocation: write a zero there
  if (cudaMemsetAsync((int64_t *)offset64.p + nc, 0, sizeof(int64_t), s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (cub::DeviceScan::ExclusiveSum(temp.p, tb, (const int64_t *)offset64.p, (int64_t *)offset.p,
                                    nc + 1, s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  int64_t n_pairs = 0;
  if (cudaMemcpyAsync(&n_pairs, (int64_t *)offset.p + nc, sizeof(int64_t), cudaMemcpyDeviceToHost,
                      s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (n_pairs <= 0 || n_pairs > (int64_t)INT32_MAX) return FFG_INVALID_INPUT;
  if ((st = keys_in.alloc(sizeof(int) * n_pairs)) || (st = vals_in.alloc(sizeof(int) * n_pairs)) ||
      (st = keys.alloc(sizeof(int) * n_pairs)) || (st = vals.alloc(sizeof(int) * n_pairs)))
    return st;
  cell_bin_fill_kernel<<<blocks_for(nc, 128), 128, 0, s>>>(
      G, nc, dt.cells, vertices, (const int64_t *)offset.p, (int *)keys_in.p, (int *)vals_in.p);
  int end_bit = 1;
  while (end_bit < 31 && (1LL << end_bit) < n_bins) ++end_bit;
  Buf temp2;
  size_t tb2 = 0;
  if (cub::DeviceRadixSort::SortPairs(nullptr, tb2, (const int *)keys_in.p, (int *)keys.p,
                                      (const int *)vals_in.p, (int *)vals.p, (int)n_pairs, 0,
                                      end_bit, s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if ((st = temp2.alloc(tb2))) return st;
  if (cub::DeviceRadixSort::SortPairs(temp2.p, tb2, (const int *)keys_in.p, (int *)keys.p,
                                      (const int *)vals_in.p, (int *)vals.p, (int)n_pairs, 0,
                                      end_bit, s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  probe_kernel<<<blocks_for(n_points, kWarpsPerBlock), 32 * kWarpsPerBlock, 0, s>>>(
      make_space(t, dt, et), G, n_pairs, (const int *)keys.p, (const int *)vals.p, dt.cells,
      vertices, u, n_points, points, first_only, values, derivs, counts);
  if (cudaGetLastError() != cudaSuccess) return FFG_CUDA_ERROR;
  // the scratch buffers are released on return: let the stream pass them first
  return cudaStreamSynchronize(s) == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace ffg
