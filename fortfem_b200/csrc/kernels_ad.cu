// Forward (JVP) and reverse (VJP) mode of the tetrahedral Lagrange stiffness
// + mass CSC assembly: assemble_tetra_lagrange_stiffness_csc_jvp and _vjp
// (src/assembly/assembly_tetra_lagrange_arbitrary_order_3d.f90:336-391 and
// :393-471, element routines :107-180 and :182-274), and of the Nedelec curl
// + mass CSC assembly, assemble_tetra_nedelec_curl_mass_csc_jvp and _vjp
// (src/assembly/assembly_tetra_nedelec_3d.f90:2114-2181 and :2183-2287,
// element routines :645-719 and :721-806).
//
// Both reuse the contraction the primal assembly runs on: every element
// matrix is K = sum_s geo_s R^s with seven reference tensors R^s (six
// symmetric pairs (a,b) of the gradient term, weight kappa det (J^-1 J^-T)_ab,
// and the mass term, weight m det); Nedelec has twelve (curl pairs, weight
// (c/det) (J^T J)_ab, and mass pairs, weight m det (J^-1 J^-T)_ab) and the
// orientation transform T around them.  The reference integrates the
// derivatives at quadrature degree 2k+2 where its primal uses 2k or the
// 4-point rule; every one of these rules integrates the polynomial
// integrands exactly, so the tensors serve both.
//
// JVP: K is linear in geo, so the tangent element matrix is sum_s geo'_s R^s
// with geo' the derivative of the seven weights along (v', kappa', m').  One
// thread per cell writes geo'; the column-owner gather of the primal
// assembly turns it into CSC values on the primal pattern, the same pattern
// csc_from_triplet gives the reference's tangent triplets.
//
// VJP: one warp per cell reads the cotangent of each of its nb x nb element
// entries from the merged CSC pattern (csc_value_bar_at, :836-851, as a
// binary search down the sorted column), contracts it with the seven
// tensors (Q_s = sum_ij Kbar_ij R^s_ij) and pulls Q back through the cell's
// geometry by hand-derived adjoints of det, J^-1 and the vertex->J map.  The
// vertex adjoints are then gathered per vertex over its cells in ascending
// cell order (the order the reference accumulates them in), without atomics.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>

#include "ffg_internal.h"
#include "tet_geometry.h"

namespace ffg {

namespace {

constexpr int kCellBar = 14;  // 12 vertex adjoints (node-major), stiffness, mass

__device__ __forceinline__ void pair_of(int s, int &a, int &b) {
  // symmetric pair order shared with basis.cpp: (0,0),(1,1),(2,2),(0,1),(0,2),(1,2)
  a = s < 3 ? s : (s == 5 ? 1 : 0);
  b = s < 3 ? s : (s == 3 ? 1 : 2);
}

// Binary search of `row` in the sorted CSC column `col`; 0 when absent.
__device__ __forceinline__ double csc_value_at(const int64_t *__restrict__ col_ptr,
                                               const int *__restrict__ row_idx,
                                               const double *__restrict__ values, int row,
                                               int col) {
  const int64_t end = col_ptr[col + 1];
  int64_t lo = col_ptr[col], hi = end;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (row_idx[mid] < row) lo = mid + 1; else hi = mid;
  }
  return (lo < end && row_idx[lo] == row) ? values[lo] : 0.0;
}

// geo'_s for one cell: d(kappa det G_ab) and d(m det), G = J^-1 J^-T, with
// d det = det tr(J^-1 dJ) and d J^-1 = -J^-1 dJ J^-1.  Load samples are 0.
__global__ void lagrange_geometry_jvp_kernel(int n_cells, const int *__restrict__ cells,
                                             const double *__restrict__ verts,
                                             const double *__restrict__ verts_dot, double ca,
                                             double cb, double ca_dot, double cb_dot,
                                             double *__restrict__ geo, int stride, int *err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  double J[9], Jd[9], Ji[9], v0[3];
  tet_jacobian(cells, verts, c, J, v0);
  tet_jacobian(cells, verts_dot, c, Jd, v0);
  const double det = det3(J);
  double *g = geo + (size_t)stride * c;
  for (int i = 7; i < stride; ++i) g[i] = 0.0;
  if (!valid_jacobian(J, det)) {
    atomicCAS(err, 0, FFG_INVALID_INPUT);
    for (int i = 0; i < 7; ++i) g[i] = 0.0;
    return;
  }
  inv3(J, det, Ji);
  double T[9], Jid[9];  // T = J^-1 dJ, Jid = -T J^-1 (column-major)
#pragma unroll
  for (int col = 0; col < 3; ++col)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      T[r + 3 * col] = Ji[r] * Jd[3 * col] + Ji[r + 3] * Jd[3 * col + 1] + Ji[r + 6] * Jd[3 * col + 2];
#pragma unroll
  for (int col = 0; col < 3; ++col)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      Jid[r + 3 * col] =
          -(T[r] * Ji[3 * col] + T[r + 3] * Ji[3 * col + 1] + T[r + 6] * Ji[3 * col + 2]);
  const double det_dot = det * (T[0] + T[4] + T[8]);
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    int a, b;
    pair_of(s, a, b);
    double G = 0.0, Gd = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      G += Ji[a + 3 * k] * Ji[b + 3 * k];
      Gd += Jid[a + 3 * k] * Ji[b + 3 * k] + Ji[a + 3 * k] * Jid[b + 3 * k];
    }
    g[s] = ca_dot * det * G + ca * (det_dot * G + det * Gd);
  }
  g[6] = cb_dot * det + cb * det_dot;
}

// One warp per cell: Q_s = sum_ij Kbar_ij R^s_ij, then the cell's adjoints
// (12 vertex components, stiffness, mass) into cell_bar[14 c ...].
__global__ void lagrange_cell_vjp_kernel(int n_cells, const int *__restrict__ cells,
                                         const double *__restrict__ verts,
                                         const int *__restrict__ gd,
                                         const int *__restrict__ free_index, int nb,
                                         const int64_t *__restrict__ col_ptr,
                                         const int *__restrict__ row_idx,
                                         const double *__restrict__ values_bar,
                                         const double *__restrict__ ref, double ca, double cb,
                                         double *__restrict__ cell_bar, int *err) {
  const int c = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= n_cells) return;  // uniform across the warp
  const int *ge = gd + (size_t)nb * c;
  const int nn = nb * nb;
  double Q[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int idx = lane; idx < nn; idx += 32) {
    const int row = free_index[ge[idx % nb]], col = free_index[ge[idx / nb]];
    if (row < 0 || col < 0) continue;
    const double b = csc_value_at(col_ptr, row_idx, values_bar, row, col);
#pragma unroll
    for (int s = 0; s < 7; ++s) Q[s] += b * __ldg(ref + (size_t)s * nn + idx);
  }
#pragma unroll
  for (int s = 0; s < 7; ++s)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) Q[s] += __shfl_xor_sync(0xffffffffu, Q[s], off);
  if (lane != 0) return;
  double J[9], Ji[9], v0[3];
  tet_jacobian(cells, verts, c, J, v0);
  const double det = det3(J);
  double *out = cell_bar + (size_t)kCellBar * c;
  if (!valid_jacobian(J, det)) {
    atomicCAS(err, 0, FFG_INVALID_INPUT);
    for (int i = 0; i < kCellBar; ++i) out[i] = 0.0;
    return;
  }
  inv3(J, det, Ji);
  // L = sum_s geo_s Q_s.  geo_s = ca det G_s (s < 6), geo_6 = cb det.
  double gq = 0.0, Cm[9];
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    int a, b;
    pair_of(s, a, b);
    const double G = Ji[a] * Ji[b] + Ji[a + 3] * Ji[b + 3] + Ji[a + 6] * Ji[b + 6];
    gq += G * Q[s];
    // symmetric C with tr(C G) = sum_s ca det Q_s G_s
    const double w = ca * det * Q[s];
    if (a == b) {
      Cm[a + 3 * a] = w;
    } else {
      Cm[a + 3 * b] = 0.5 * w;
      Cm[b + 3 * a] = 0.5 * w;
    }
  }
  const double det_bar = ca * gq + cb * Q[6];
  // Jibar = 2 C J^-1 ; Jbar = -J^-T Jibar J^-T + det_bar det J^-T
  double Jib[9], A[9], Jb[9];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int a = 0; a < 3; ++a)
      Jib[a + 3 * k] = 2.0 * (Cm[a] * Ji[3 * k] + Cm[a + 3] * Ji[1 + 3 * k] + Cm[a + 6] * Ji[2 + 3 * k]);
  // J^-T(r, m) = Ji[m + 3 r]
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      A[r + 3 * k] = Ji[3 * r] * Jib[3 * k] + Ji[1 + 3 * r] * Jib[1 + 3 * k] + Ji[2 + 3 * r] * Jib[2 + 3 * k];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int r = 0; r < 3; ++r)
      Jb[r + 3 * k] = -(A[r] * Ji[k] + A[r + 3] * Ji[k + 3] + A[r + 6] * Ji[k + 6]) +
                      det_bar * det * Ji[k + 3 * r];
  // J(:, k) = v_{k+1} - v_0
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    out[r] = -(Jb[r] + Jb[r + 3] + Jb[r + 6]);
    out[3 + r] = Jb[r];
    out[6 + r] = Jb[r + 3];
    out[9 + r] = Jb[r + 6];
  }
  out[12] = det * gq;
  out[13] = det * Q[6];
}

struct NedVjpDims {
  int k, nb, fdc, edge_end;
  int oglobal;  // the nb x nb cotangent lives in `elem`, not in shared memory
};

// One CTA per cell (grid-stride).  The oriented cotangent Obar (the
// reference's dense_bar at the cell's global DoFs, :2222-2250) is gathered
// from the CSC, mapped back to the element basis as T Obar T^T (edge signs;
// per face (Obar T^T) then T (.) through the face block), contracted with
// the twelve reference tensors, and the cell's geometry adjoints follow from
// K = (c/det) sum_s C^s (J^T J)_s + m det sum_s V^s (J^-1 J^-T)_s.
__global__ void nedelec_cell_vjp_kernel(int n_cells, const int *__restrict__ cells,
                                        const double *__restrict__ verts,
                                        const int *__restrict__ gd,
                                        const int *__restrict__ free_index, NedVjpDims D,
                                        const int64_t *__restrict__ col_ptr,
                                        const int *__restrict__ row_idx,
                                        const double *__restrict__ values_bar,
                                        const double *__restrict__ ref,
                                        const int8_t *__restrict__ edge_sign,
                                        const uint8_t *__restrict__ face_perm,
                                        const double *__restrict__ face_blocks, double ca,
                                        double cb, double *__restrict__ elem,
                                        double *__restrict__ cell_bar, int *err) {
  extern __shared__ double sm[];
  const int nb = D.nb, fdc = D.fdc;
  const size_t nn = (size_t)nb * nb;
  double *O = D.oglobal ? nullptr : sm;
  double *tmp = D.oglobal ? sm : sm + nn;  // nb * fdc
  double *B = tmp + (size_t)nb * fdc;      // fdc * fdc
  __shared__ double part[12][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int c = blockIdx.x; c < n_cells; c += gridDim.x) {
    if (D.oglobal) O = elem + nn * c;
    const int *ge = gd + (size_t)nb * c;
    const int8_t *sg = edge_sign + 6 * (size_t)c;
    for (size_t idx = threadIdx.x; idx < nn; idx += blockDim.x) {
      const int i = (int)(idx % nb), j = (int)(idx / nb);
      const int row = free_index[ge[i]], col = free_index[ge[j]];
      double v = (row < 0 || col < 0) ? 0.0 : csc_value_at(col_ptr, row_idx, values_bar, row, col);
      if (i < D.edge_end && sg[i / D.k] == -1 && ((i % D.k) % 2) == 0) v = -v;
      if (j < D.edge_end && sg[j / D.k] == -1 && ((j % D.k) % 2) == 0) v = -v;
      O[idx] = v;
    }
    __syncthreads();
    // face blocks: T[st+m][st+r] = B[r*fdc+m], so (O T^T)[i][st+r] =
    // sum_m O[i][st+m] B[m*fdc+r] and (T O)[st+r][j] = sum_m B[m*fdc+r] O[st+m][j]
    for (int f = 0; f < 4 && fdc > 0; ++f) {
      const int st = D.edge_end + f * fdc;
      const double *Bg = face_blocks + (size_t)face_perm[4 * (size_t)c + f] * fdc * fdc;
      for (int q = threadIdx.x; q < fdc * fdc; q += blockDim.x) B[q] = Bg[q];
      __syncthreads();
      for (int q = threadIdx.x; q < nb * fdc; q += blockDim.x) {
        const int i = q % nb, r = q / nb;
        double acc = 0.0;
        for (int m = 0; m < fdc; ++m) acc += O[i + (size_t)nb * (st + m)] * B[m * fdc + r];
        tmp[q] = acc;
      }
      __syncthreads();
      for (int q = threadIdx.x; q < nb * fdc; q += blockDim.x)
        O[(q % nb) + (size_t)nb * (st + q / nb)] = tmp[q];
      __syncthreads();
      for (int q = threadIdx.x; q < nb * fdc; q += blockDim.x) {
        const int r = q % fdc, j = q / fdc;
        double acc = 0.0;
        for (int m = 0; m < fdc; ++m) acc += B[m * fdc + r] * O[(st + m) + (size_t)nb * j];
        tmp[q] = acc;
      }
      __syncthreads();
      for (int q = threadIdx.x; q < nb * fdc; q += blockDim.x)
        O[(st + q % fdc) + (size_t)nb * (q / fdc)] = tmp[q];
      __syncthreads();
    }
    double Q[12];
#pragma unroll
    for (int s = 0; s < 12; ++s) Q[s] = 0.0;
    for (size_t idx = threadIdx.x; idx < nn; idx += blockDim.x) {
      const double o = O[idx];
#pragma unroll
      for (int s = 0; s < 12; ++s) Q[s] += o * __ldg(ref + s * nn + idx);
    }
#pragma unroll
    for (int s = 0; s < 12; ++s) {
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) Q[s] += __shfl_xor_sync(0xffffffffu, Q[s], off);
      if (lane == 0) part[s][warp] = Q[s];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int s = 0; s < 12; ++s) {
        double a = 0.0;
        for (int w = 0; w < nwarps; ++w) a += part[s][w];
        Q[s] = a;
      }
      double J[9], Ji[9], v0[3];
      tet_jacobian(cells, verts, c, J, v0);
      const double det = det3(J);
      double *out = cell_bar + (size_t)kCellBar * c;
      if (!valid_jacobian(J, det)) {
        atomicCAS(err, 0, FFG_INVALID_INPUT);
        for (int i = 0; i < kCellBar; ++i) out[i] = 0.0;
      } else {
        inv3(J, det, Ji);
        double hq = 0.0, gq = 0.0, Dm[9], Cm[9];
        for (int s = 0; s < 6; ++s) {
          int a, b;
          pair_of(s, a, b);
          const double H = J[3 * a] * J[3 * b] + J[3 * a + 1] * J[3 * b + 1] + J[3 * a + 2] * J[3 * b + 2];
          const double G = Ji[a] * Ji[b] + Ji[a + 3] * Ji[b + 3] + Ji[a + 6] * Ji[b + 6];
          hq += H * Q[s];
          gq += G * Q[6 + s];
          const double wd = ca / det * Q[s], wc = cb * det * Q[6 + s];
          if (a == b) {
            Dm[a + 3 * a] = wd;
            Cm[a + 3 * a] = wc;
          } else {
            Dm[a + 3 * b] = Dm[b + 3 * a] = 0.5 * wd;
            Cm[a + 3 * b] = Cm[b + 3 * a] = 0.5 * wc;
          }
        }
        const double det_bar = -ca * hq / (det * det) + cb * gq;
        // Jbar = 2 J D - J^-T (2 C J^-1) J^-T + det_bar det J^-T
        double Jib[9], A[9], Jb[9];
        for (int k = 0; k < 3; ++k)
          for (int a = 0; a < 3; ++a)
            Jib[a + 3 * k] = 2.0 * (Cm[a] * Ji[3 * k] + Cm[a + 3] * Ji[1 + 3 * k] + Cm[a + 6] * Ji[2 + 3 * k]);
        for (int k = 0; k < 3; ++k)
          for (int r = 0; r < 3; ++r)
            A[r + 3 * k] = Ji[3 * r] * Jib[3 * k] + Ji[1 + 3 * r] * Jib[1 + 3 * k] + Ji[2 + 3 * r] * Jib[2 + 3 * k];
        for (int k = 0; k < 3; ++k)
          for (int r = 0; r < 3; ++r)
            Jb[r + 3 * k] = 2.0 * (J[r] * Dm[3 * k] + J[r + 3] * Dm[1 + 3 * k] + J[r + 6] * Dm[2 + 3 * k]) -
                            (A[r] * Ji[k] + A[r + 3] * Ji[k + 3] + A[r + 6] * Ji[k + 6]) +
                            det_bar * det * Ji[k + 3 * r];
        for (int r = 0; r < 3; ++r) {
          out[r] = -(Jb[r] + Jb[r + 3] + Jb[r + 6]);
          out[3 + r] = Jb[r];
          out[6 + r] = Jb[r + 3];
          out[9 + r] = Jb[r + 6];
        }
        out[12] = hq / det;
        out[13] = det * gq;
      }
    }
    __syncthreads();
  }
}

__global__ void iota_kernel(int64_t n, int *v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (int)i;
}

// Vertex v sums the adjoints of its (cell, node) incidences in ascending cell
// order: `keys` are the sorted vertex ids of the 4 n_cells incidences and
// `inc` their positions 4 c + node (stably sorted, so ascending per vertex).
__global__ void vertex_gather_kernel(int n_vertices, int64_t n_inc, const int *__restrict__ keys,
                                     const int *__restrict__ inc,
                                     const double *__restrict__ cell_bar,
                                     double *__restrict__ verts_bar) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n_vertices) return;
  int64_t lo = 0, hi = n_inc;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < v) lo = mid + 1; else hi = mid;
  }
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t p = lo; p < n_inc && keys[p] == v; ++p) {
    const int q = inc[p];
    const double *cb = cell_bar + (size_t)kCellBar * (q >> 2) + 3 * (q & 3);
    acc[0] += cb[0];
    acc[1] += cb[1];
    acc[2] += cb[2];
  }
  verts_bar[3 * (size_t)v] = acc[0];
  verts_bar[3 * (size_t)v + 1] = acc[1];
  verts_bar[3 * (size_t)v + 2] = acc[2];
}

// Fixed-order sum of the per-cell stiffness and mass adjoints (one CTA:
// contiguous chunks, then a shared-memory tree), reproducible run to run.
__global__ void coefficient_sum_kernel(int n_cells, const double *__restrict__ cell_bar,
                                       double *__restrict__ out) {
  __shared__ double sk[1024], sm[1024];
  const int t = threadIdx.x;
  const int chunk = (n_cells + blockDim.x - 1) / blockDim.x;
  const int lo = t * chunk, hi = min(n_cells, lo + chunk);
  double a = 0.0, b = 0.0;
  for (int c = lo; c < hi; ++c) {
    a += cell_bar[(size_t)kCellBar * c + 12];
    b += cell_bar[(size_t)kCellBar * c + 13];
  }
  sk[t] = a;
  sm[t] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (t < w) {
      sk[t] += sk[t + w];
      sm[t] += sm[t + w];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = sk[0];
    out[1] = sm[0];
  }
}

inline int blocks_for(int64_t n, int t) { return (int)((n + t - 1) / t); }

struct Scratch {
  void *p = nullptr;
  ~Scratch() {
    if (p) cudaFree(p);
  }
  int alloc(size_t bytes) {
    return cudaMalloc(&p, std::max<size_t>(bytes, 16)) == cudaSuccess ? FFG_OK : FFG_OUT_OF_MEMORY;
  }
};

}  // namespace

int launch_lagrange_geometry_jvp(const Topology &t, const DeviceTopology &dt,
                                 const double *vertices, const double *vertices_dot, double ca,
                                 double cb, double ca_dot, double cb_dot, double *geo, int stride,
                                 int *err, cudaStream_t s) {
  if (t.family != FFG_TETRA_LAGRANGE || stride < 7) return FFG_INVALID_INPUT;
  const int T = 128;
  lagrange_geometry_jvp_kernel<<<blocks_for(t.n_cells, T), T, 0, s>>>(
      t.n_cells, dt.cells, vertices, vertices_dot, ca, cb, ca_dot, cb_dot, geo, stride, err);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

namespace {

// Scratch of the reverse mode: per-cell adjoints and the sorted incidences.
struct VjpScratch {
  Scratch cell_bar, keys, inc, inc_in, temp;
  int alloc(int64_t nc) {
    int st;
    if ((st = cell_bar.alloc(sizeof(double) * kCellBar * nc))) return st;
    if ((st = keys.alloc(sizeof(int) * 4 * nc))) return st;
    if ((st = inc.alloc(sizeof(int) * 4 * nc))) return st;
    return inc_in.alloc(sizeof(int) * 4 * nc);
  }
};

// Vertex-owner gather of the per-cell adjoints and the coefficient sums.
int finish_vjp(const Topology &t, const DeviceTopology &dt, VjpScratch &w, double *vertices_bar,
               double *coef_bar, cudaStream_t s) {
  const int64_t n_inc = 4 * (int64_t)t.n_cells;
  iota_kernel<<<blocks_for(n_inc, 256), 256, 0, s>>>(n_inc, (int *)w.inc_in.p);
  int end_bit = 1;
  while (end_bit < 31 && (1LL << end_bit) < (int64_t)t.n_vertices) ++end_bit;
  size_t temp_bytes = 0;
  if (cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, dt.cells, (int *)w.keys.p,
                                      (const int *)w.inc_in.p, (int *)w.inc.p, n_inc, 0, end_bit,
                                      s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  int st;
  if ((st = w.temp.alloc(temp_bytes))) return st;
  if (cub::DeviceRadixSort::SortPairs(w.temp.p, temp_bytes, dt.cells, (int *)w.keys.p,
                                      (const int *)w.inc_in.p, (int *)w.inc.p, n_inc, 0, end_bit,
                                      s) != cudaSuccess)
    return FFG_CUDA_ERROR;
  vertex_gather_kernel<<<blocks_for(t.n_vertices, 128), 128, 0, s>>>(
      t.n_vertices, n_inc, (const int *)w.keys.p, (const int *)w.inc.p,
      (const double *)w.cell_bar.p, vertices_bar);
  coefficient_sum_kernel<<<1, 1024, 0, s>>>(t.n_cells, (const double *)w.cell_bar.p, coef_bar);
  if (cudaGetLastError() != cudaSuccess) return FFG_CUDA_ERROR;
  // the scratch buffers are released on return: let the stream pass them first
  return cudaStreamSynchronize(s) == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace

int lagrange_vjp(const Topology &t, const DeviceTopology &dt, const int64_t *col_ptr,
                 const int *row_idx, const double *vertices, const double *values_bar, double ca,
                 double cb, double *vertices_bar, double *coef_bar, int *err, cudaStream_t s) {
  if (t.family != FFG_TETRA_LAGRANGE) return FFG_INVALID_INPUT;
  VjpScratch w;
  int st;
  if ((st = w.alloc(t.n_cells))) return st;
  const int warps_per_block = 8;
  lagrange_cell_vjp_kernel<<<blocks_for(t.n_cells, warps_per_block), 32 * warps_per_block, 0, s>>>(
      t.n_cells, dt.cells, vertices, dt.gd, dt.free_index, t.nb, col_ptr, row_idx, values_bar,
      dt.ref, ca, cb, (double *)w.cell_bar.p, err);
  if (cudaGetLastError() != cudaSuccess) return FFG_CUDA_ERROR;
  return finish_vjp(t, dt, w, vertices_bar, coef_bar, s);
}

int nedelec_vjp(const Topology &t, const ElementTables &tab, const DeviceTopology &dt,
                const int64_t *col_ptr, const int *row_idx, const double *vertices,
                const double *values_bar, double ca, double cb, double *elem,
                double *vertices_bar, double *coef_bar, int *err, cudaStream_t s) {
  if (t.family != FFG_TETRA_NEDELEC || tab.n_terms != 12) return FFG_INVALID_INPUT;
  NedVjpDims D;
  D.k = t.degree;
  D.nb = t.nb;
  D.fdc = t.degree * (t.degree - 1);
  D.edge_end = 6 * t.degree;
  auto smem_for = [&](bool oglobal) {
    return sizeof(double) * ((oglobal ? 0 : (size_t)D.nb * D.nb) + (size_t)D.nb * D.fdc +
                             (size_t)D.fdc * D.fdc);
  };
  D.oglobal = smem_for(false) > 200 * 1024 ? 1 : 0;
  const size_t smem = smem_for(D.oglobal != 0);
  if (D.oglobal && !elem) return FFG_INVALID_INPUT;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(nedelec_cell_vjp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return FFG_CUDA_ERROR;
  VjpScratch w;
  int st;
  if ((st = w.alloc(t.n_cells))) return st;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::min<int64_t>(t.n_cells, (int64_t)sms * 8);
  nedelec_cell_vjp_kernel<<<grid, 256, smem, s>>>(
      t.n_cells, dt.cells, vertices, dt.gd, dt.free_index, D, col_ptr, row_idx, values_bar,
      dt.ref, dt.edge_sign, dt.face_perm, dt.face_blocks, ca, cb, elem, (double *)w.cell_bar.p,
      err);
  if (cudaGetLastError() != cudaSuccess) return FFG_CUDA_ERROR;
  return finish_vjp(t, dt, w, vertices_bar, coef_bar, s);
}

}  // namespace ffg
