// Assembly kernels (sm_100a): per-cell geometry (K1), Nedelec element
// matrices with orientation transform (K2), and the atomic-free,
// column-owner scatter into the constrained CSC (K3).
//
// K3 gives every CSC column (a free global DoF j) to one thread.  The thread
// walks the cells incident to j in ascending cell order, computes column l(j)
// of each element matrix and adds it into the column's slots through the
// precomputed slot map.  Every CSC value is therefore the sum of its element
// contributions in the reference's triplet order (cell-major, as
// assemble_*_csc emits them before csc_from_triplet), without atomics, and is
// bit-reproducible run to run.  The same pass accumulates the load, the
// Dirichlet lifting -A_fc g of sparse_direct_solve_constrained_real
// (src/solvers/fortfem_sparse_direct.f90:329-338, by symmetry of the element
// matrices) and the Jacobi diagonal of build_sparse_preconditioner
// (src/solvers/advanced_solvers.f90:1139-1154).
#include <cuda_runtime.h>

#include <algorithm>

#include "ffg_internal.h"
#include "tet_geometry.h"

namespace ffg {

namespace {

// symmetric pair order shared with basis.cpp: (0,0),(1,1),(2,2),(0,1),(0,2),(1,2)
__constant__ int kPa[6] = {0, 1, 2, 0, 0, 1};
__constant__ int kPb[6] = {0, 1, 2, 1, 2, 2};

// ------------------------------------------------------------ K1 geometry
// Lagrange: geo = [k det G_ab (6), m det, det f_q (n_q)], G = J^-1 J^-T.
__device__ __forceinline__ void lagrange_geometry_cell(int c, const int *__restrict__ cells,
                                                      const double *__restrict__ verts, double ca,
                                                      double cb, const double *__restrict__ cell_a,
                                                      const double *__restrict__ cell_b,
                                                      const double *__restrict__ samples, int nq,
                                                      double *__restrict__ geo, int stride,
                                                      int *err) {
  double J[9], Ji[9], v0[3];
  tet_jacobian(cells, verts, c, J, v0);
  const double det = det3(J);
  double *g = geo + (size_t)stride * c;
  if (!valid_jacobian(J, det)) {
    atomicCAS(err, 0, FFG_INVALID_INPUT);
    for (int i = 0; i < stride; ++i) g[i] = 0.0;
    return;
  }
  inv3(J, det, Ji);
  const double kappa = ca * (cell_a ? cell_a[c] : 1.0);
  const double mass = cb * (cell_b ? cell_b[c] : 1.0);
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    const int a = kPa[s], b = kPb[s];
    // (J^-1 J^-T)_ab = sum_k Ji(a,k) Ji(b,k), Ji column-major Ji[a + 3k]
    const double G = Ji[a] * Ji[b] + Ji[a + 3] * Ji[b + 3] + Ji[a + 6] * Ji[b + 6];
    g[s] = kappa * det * G;
  }
  g[6] = mass * det;
  for (int q = 0; q < nq; ++q) g[7 + q] = samples ? det * samples[(size_t)nq * c + q] : 0.0;
}

__global__ void lagrange_geometry_kernel(int n_cells, const int *__restrict__ cells,
                                         const double *__restrict__ verts, double ca, double cb,
                                         const double *__restrict__ cell_a,
                                         const double *__restrict__ cell_b,
                                         const double *__restrict__ samples, int nq,
                                         double *__restrict__ geo, int stride, int *err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n_cells)
    lagrange_geometry_cell(c, cells, verts, ca, cb, cell_a, cell_b, samples, nq, geo, stride, err);
}

// P1 triangles: closed-form local matrix of assemble_scalar_p1_matrix
// (src/fortfem_forms_simple.f90:1702-1717) and the load area/3 of
// assemble_scalar_p1_load (:1749-1758) with a per-cell source value.
__device__ __forceinline__ void p1_geometry_cell(int c, const int *__restrict__ tris,
                                                 const double *__restrict__ verts, double stiff,
                                                 double mass, const double *__restrict__ cell_a,
                                                 const double *__restrict__ cell_b,
                                                 const double *__restrict__ samples,
                                                 double *__restrict__ geo, int *err) {
  double x[3], y[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int v = tris[3 * (size_t)c + i];
    x[i] = verts[2 * (size_t)v];
    y[i] = verts[2 * (size_t)v + 1];
  }
  const double det = (x[1] - x[0]) * (y[2] - y[0]) - (x[2] - x[0]) * (y[1] - y[0]);
  double *g = geo + 10 * (size_t)c;
  if (fabs(det) <= 64.0 * kEps) {
    atomicCAS(err, 0, FFG_INVALID_INPUT);
    for (int i = 0; i < 10; ++i) g[i] = 0.0;
    return;
  }
  const double area = 0.5 * fabs(det);
  const double gx[3] = {(y[1] - y[2]) / det, (y[2] - y[0]) / det, (y[0] - y[1]) / det};
  const double gy[3] = {(x[2] - x[1]) / det, (x[0] - x[2]) / det, (x[1] - x[0]) / det};
  const double ks = stiff * (cell_a ? cell_a[c] : 1.0);
  const double km = mass * (cell_b ? cell_b[c] : 1.0);
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int a = 0; a < 3; ++a)
      g[a + 3 * b] = ks * area * (gx[a] * gx[b] + gy[a] * gy[b]) +
                     km * area * (a == b ? 2.0 : 1.0) / 12.0;
  g[9] = samples ? samples[c] * area / 3.0 : 0.0;
}

__global__ void p1_geometry_kernel(int n_cells, const int *__restrict__ tris,
                                   const double *__restrict__ verts, double stiff, double mass,
                                   const double *__restrict__ cell_a,
                                   const double *__restrict__ cell_b,
                                   const double *__restrict__ samples, double *__restrict__ geo,
                                   int *err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n_cells) p1_geometry_cell(c, tris, verts, stiff, mass, cell_a, cell_b, samples, geo, err);
}

// Arbitrary-order triangles: geo = [k |det| G_00, k |det| G_11, k |det| G_01,
// m |det|, |det| f_q (n_q)], G = J^-1 J^-T of the affine map (columns v1 - v0,
// v2 - v0); |det| as the P1 forms take the unsigned area.
__global__ void triangle_lagrange_geometry_kernel(int n_cells, const int *__restrict__ tris,
                                                  const double *__restrict__ verts, double ca,
                                                  double cb, const double *__restrict__ cell_a,
                                                  const double *__restrict__ cell_b,
                                                  const double *__restrict__ samples, int nq,
                                                  double *__restrict__ geo, int stride, int *err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  double x[3], y[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int v = tris[3 * (size_t)c + i];
    x[i] = verts[2 * (size_t)v];
    y[i] = verts[2 * (size_t)v + 1];
  }
  const double j00 = x[1] - x[0], j10 = y[1] - y[0], j01 = x[2] - x[0], j11 = y[2] - y[0];
  const double det = j00 * j11 - j01 * j10;
  const double m = fmax(fmax(fabs(j00), fabs(j10)), fmax(fabs(j01), fabs(j11)));
  const double sc = fmax(1.0, m);
  double *g = geo + (size_t)stride * c;
  if (!(fabs(det) > 64.0 * kEps * sc * sc)) {
    atomicCAS(err, 0, FFG_INVALID_INPUT);
    for (int i = 0; i < stride; ++i) g[i] = 0.0;
    return;
  }
  // J^-1 rows: (j11, -j01) / det and (-j10, j00) / det
  const double i00 = j11 / det, i01 = -j01 / det, i10 = -j10 / det, i11 = j00 / det;
  const double area = fabs(det);
  const double kappa = ca * (cell_a ? cell_a[c] : 1.0);
  const double mass = cb * (cell_b ? cell_b[c] : 1.0);
  g[0] = kappa * area * (i00 * i00 + i01 * i01);
  g[1] = kappa * area * (i10 * i10 + i11 * i11);
  g[2] = kappa * area * (i00 * i10 + i01 * i11);
  g[3] = mass * area;
  for (int q = 0; q < nq; ++q) g[4 + q] = samples ? area * samples[(size_t)nq * c + q] : 0.0;
}

// ----------------------------------------------------- K3 column-owner scatter
// SELL = false: values into the CSC value array (rhs in free-DoF order).
// SELL = true: values into the solver's slices (row iperm[j] of the SELL
// operator, which by symmetry is column j), with the FP32 copy, the Jacobi
// diagonal and the rhs in the SELL numbering.
template <int FAMILY, bool SELL>
__device__ __forceinline__ void column_body(int64_t j, const int64_t *__restrict__ col_ptr,
                              const int *__restrict__ row_idx, const int64_t *__restrict__ inc_ptr,
                              const int *__restrict__ inc_cell,
                              const uint8_t *__restrict__ inc_local,
                              const uint16_t *__restrict__ slot, const int *__restrict__ gd,
                              int nb, const double *__restrict__ geo, int stride,
                              const double *__restrict__ ref, const double *__restrict__ load_basis,
                              int nq, const double *__restrict__ elem,
                              const double *__restrict__ cell_rhs, const double *__restrict__ g,
                              const int *__restrict__ iperm, const int64_t *__restrict__ soff,
                              double *__restrict__ val64, float *__restrict__ val32,
                              double *__restrict__ dinv64, float *__restrict__ dinv32,
                              double *__restrict__ rhs, const float *__restrict__ elem32,
                              int ld32, int64_t cs32) {
  const int64_t start = col_ptr[j], end = col_ptr[j + 1];
  int64_t base, stride_out, out_row;
  if (SELL) {
    out_row = iperm[j];
    base = soff[out_row / kSliceRows] + out_row % kSliceRows;
    stride_out = kSliceRows;
  } else {
    out_row = j;
    base = start;
    stride_out = 1;
  }
  const int len = (int)(end - start);
  for (int k = 0; k < len; ++k) val64[base + stride_out * k] = 0.0;
  double b = 0.0, lift = 0.0;
  const size_t nn = (size_t)nb * nb;
  for (int64_t p = inc_ptr[j]; p < inc_ptr[j + 1]; ++p) {
    const int e = inc_cell[p];
    const int l = inc_local[p];
    const uint16_t *sl = slot + (size_t)p * nb;
    const int *ge = gd + (size_t)nb * e;
    // reference-tensor families: 7 weights (tetrahedra) or 4 (triangles)
    constexpr int NT = FAMILY == FFG_TRIANGLE_LAGRANGE ? 4 : 7;
    constexpr bool TENSORS = FAMILY == FFG_TETRA_LAGRANGE || FAMILY == FFG_TRIANGLE_LAGRANGE;
    double gco[NT];
    double F = 0.0;
    if (TENSORS) {
      const double *gg = geo + (size_t)stride * e;
#pragma unroll
      for (int s = 0; s < NT; ++s) gco[s] = gg[s];
      for (int q = 0; q < nq; ++q) F += gg[NT + q] * __ldg(load_basis + (size_t)q * nb + l);
    } else if (FAMILY == FFG_TRIANGLE_P1) {
      F = geo[10 * (size_t)e + 9];
    } else {
      F = cell_rhs[(size_t)nb * e + l];
    }
    for (int i = 0; i < nb; ++i) {
      double kil;
      if (TENSORS) {
        const size_t off = i + (size_t)nb * l;
        kil = 0.0;
#pragma unroll
        for (int s = 0; s < NT; ++s) kil += gco[s] * __ldg(ref + s * nn + off);
      } else if (FAMILY == FFG_TRIANGLE_P1) {
        kil = geo[10 * (size_t)e + i + 3 * l];
      } else if (elem32) {
        kil = (double)elem32[(size_t)cs32 * e + i + (size_t)ld32 * l];
      } else {
        kil = elem[nn * e + i + (size_t)nb * l];
      }
      const uint16_t s = sl[i];
      if (s == kConstrainedSlot) {
        if (g) lift += kil * g[ge[i]];
      } else {
        val64[base + stride_out * s] += kil;
      }
    }
    b += F;
  }
  rhs[out_row] = b - lift;
  if (SELL) {
    double d = 0.0;
    for (int k = 0; k < len; ++k) {
      const double v = val64[base + stride_out * k];
      val32[base + stride_out * k] = (float)v;
      if (row_idx[start + k] == (int)j) d = v;
    }
    const double di = (fabs(d) > 1.0e-14) ? 1.0 / d : 1.0;
    dinv64[out_row] = di;
    dinv32[out_row] = (float)di;
  }
}

template <int FAMILY, bool SELL>
__global__ void column_kernel(int64_t n_free, const int64_t *__restrict__ col_ptr,
                              const int *__restrict__ row_idx, const int64_t *__restrict__ inc_ptr,
                              const int *__restrict__ inc_cell,
                              const uint8_t *__restrict__ inc_local,
                              const uint16_t *__restrict__ slot, const int *__restrict__ gd,
                              int nb, const double *__restrict__ geo, int stride,
                              const double *__restrict__ ref, const double *__restrict__ load_basis,
                              int nq, const double *__restrict__ elem,
                              const double *__restrict__ cell_rhs, const double *__restrict__ g,
                              const int *__restrict__ iperm, const int64_t *__restrict__ soff,
                              double *__restrict__ val64, float *__restrict__ val32,
                              double *__restrict__ dinv64, float *__restrict__ dinv32,
                              double *__restrict__ rhs, const float *__restrict__ elem32,
                              int ld32, int64_t cs32) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n_free)
    column_body<FAMILY, SELL>(j, col_ptr, row_idx, inc_ptr, inc_cell, inc_local, slot, gd, nb, geo,
                              stride, ref, load_basis, nq, elem, cell_rhs, g, iperm, soff, val64,
                              val32, dinv64, dinv32, rhs, elem32, ld32, cs32);
}

// CSC columns of high-order elements (n_b >= 16), one warp per free column:
// the incidences go in ascending cell order as in column_kernel, and for each
// one the lanes take the element's local rows i (distinct rows land in
// distinct slots), adding into the column held in shared memory, so every
// entry receives its terms in the same order as in column_kernel; the
// element column, the slot row and the finished column are read and written
// contiguously.  The lifting is summed per lane and then across the warp in
// a fixed order.  Shared memory: max_len doubles per warp.
template <int FAMILY>
__global__ void csc_column_warp_kernel(int64_t n_free, int max_len,
                                       const int64_t *__restrict__ col_ptr,
                                       const int64_t *__restrict__ inc_ptr,
                                       const int *__restrict__ inc_cell,
                                       const uint8_t *__restrict__ inc_local,
                                       const uint16_t *__restrict__ slot,
                                       const int *__restrict__ gd, int nb,
                                       const double *__restrict__ geo, int stride,
                                       const double *__restrict__ ref,
                                       const double *__restrict__ load_basis, int nq,
                                       const double *__restrict__ elem,
                                       const double *__restrict__ cell_rhs,
                                       const double *__restrict__ g, double *__restrict__ val,
                                       double *__restrict__ rhs, const float *__restrict__ elem32,
                                       int ld32, int64_t cs32) {
  extern __shared__ double col_acc[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t j = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  if (j >= n_free) return;
  const int64_t start = col_ptr[j];
  const int len = (int)(col_ptr[j + 1] - start);
  double *A = col_acc + (size_t)warp * max_len;
  for (int k = lane; k < len; k += 32) A[k] = 0.0;
  __syncwarp();
  const size_t nn = (size_t)nb * nb;
  constexpr int NT = FAMILY == FFG_TRIANGLE_LAGRANGE ? 4 : 7;
  constexpr bool TENSORS = FAMILY == FFG_TETRA_LAGRANGE || FAMILY == FFG_TRIANGLE_LAGRANGE;
  double b = 0.0, lift = 0.0;
  for (int64_t p = inc_ptr[j]; p < inc_ptr[j + 1]; ++p) {
    const int e = inc_cell[p];
    const int l = inc_local[p];
    const uint16_t *sl = slot + (size_t)p * nb;
    const int *ge = gd + (size_t)nb * e;
    double gco[NT];
    double F = 0.0;
    if (TENSORS) {
      const double *gg = geo + (size_t)stride * e;
#pragma unroll
      for (int t = 0; t < NT; ++t) gco[t] = gg[t];
      for (int q = 0; q < nq; ++q) F += gg[NT + q] * __ldg(load_basis + (size_t)q * nb + l);
    } else {
      F = cell_rhs[(size_t)nb * e + l];
    }
    for (int i = lane; i < nb; i += 32) {
      double kil;
      if (TENSORS) {
        const size_t off = i + (size_t)nb * l;
        kil = 0.0;
#pragma unroll
        for (int t = 0; t < NT; ++t) kil += gco[t] * __ldg(ref + t * nn + off);
      } else if (elem32) {
        kil = (double)elem32[(size_t)cs32 * e + i + (size_t)ld32 * l];
      } else {
        kil = elem[nn * e + i + (size_t)nb * l];
      }
      const uint16_t sidx = sl[i];
      if (sidx == kConstrainedSlot) {
        if (g) lift += kil * g[ge[i]];
      } else {
        A[sidx] += kil;
      }
    }
    b += F;
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lift += __shfl_xor_sync(0xffffffffu, lift, o);
  for (int k = lane; k < len; k += 32) val[start + k] = A[k];
  if (lane == 0) rhs[j] = b - lift;
}

// SELL rows of Nedelec elements (16 <= n_b <= 128), one 256-thread CTA per
// half slice (16 rows, so that four CTAs share an SM and one's write-out
// overlaps the others' gathers): warp w gathers rows w and w + 8 of the half
// (free column j = perm[row]) with its lanes over the element's local rows
// i, as csc_column_warp_kernel does for a CSC column, into the half's image
// in shared memory (slot s of row r at s * 17 + r), every entry receiving
// its terms in ascending incidence order as in column_kernel; then the CTA
// writes the half's FP64 and FP32 values (128 contiguous bytes of FP64 per
// slot step) and each row's Jacobi diagonal and right-hand side.  Both rows'
// columns, incidence ranges and first 32 incidences are loaded before either
// is gathered; U incidences' element columns and slot rows (NI values per
// lane each) are loaded before any of them is added.
struct SliceArgs {
  const int2 *range;  // per SELL row: [p0, p1) of its column's incidences
  int nb, ld32;
  int64_t cs32;  // FP32 element matrices: elements per cell
  int64_t n;  // rows (free DoFs)
  const int *perm;
  const int64_t *soff, *col_ptr, *inc_ptr;
  const int *row_idx, *inc_cell, *gd;
  const uint8_t *inc_local;
  const uint16_t *slot;
  const double *elem, *cell_rhs, *g;
  const float *elem32;
  double *val64, *dinv64, *rhs;
  float *val32, *dinv32;
};
constexpr int kSliceHalf = kSliceRows / 2;      // rows of a CTA
constexpr int kSliceStride = kSliceHalf + 1;    // shared-memory row pitch of a half-slice image
constexpr int kSliceThreads = 256;
constexpr int kSliceRowsPerWarp = kSliceHalf / (kSliceThreads / 32);
static_assert(kSliceRowsPerWarp == 2, "two rows per warp");

// The incidences of one row: whether the row exists (j = 0, or -1 past the
// last row), its incidence range [p0, p1) and the first 32 incidences' cells
// and local indices, one per lane.
struct SliceRowHead {
  int j;
  int64_t p0, p1;
  int e, l;
};

__device__ __forceinline__ void slice_head(const SliceArgs &A, int64_t row, int lane,
                                           SliceRowHead &h) {
  h.j = row < A.n ? 0 : -1;
  const int2 rg = h.j >= 0 ? A.range[row] : make_int2(0, 0);
  h.p0 = rg.x;
  h.p1 = rg.y;
  h.e = 0;
  h.l = 0;
  if (h.p0 + lane < h.p1) {
    h.e = A.inc_cell[h.p0 + lane];
    h.l = A.inc_local[h.p0 + lane];
  }
}

// Incidence range of every SELL row's column (the slice gather's heads).
__global__ void inc_range_kernel(int64_t n, const int *perm, const int64_t *inc_ptr,
                                 int2 *range) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int j = perm[r];
  range[r] = make_int2((int)inc_ptr[j], (int)inc_ptr[j + 1]);
}

template <int NI, int U, bool F32>
__device__ __forceinline__ void slice_row(const SliceArgs &A, double *img, int r, int64_t row,
                                          int lane, SliceRowHead h) {
  const int nb = A.nb;
  double b = 0.0, lift = 0.0;
  const int64_t p0 = h.p0, p1 = h.p1;
  // local rows of this lane and whether they exist (nb <= 32 NI)
  bool has[NI];
#pragma unroll
  for (int c = 0; c < NI; ++c) has[c] = lane + 32 * c < nb;
  // element columns: FP64 nb x nb or FP32 with leading dimension ld32, per cell
  const int ld = F32 ? A.ld32 : nb;
  const size_t cell_stride = F32 ? (size_t)A.cs32 : (size_t)nb * nb;
  for (int64_t pb = p0; pb < p1; pb += 32) {
    const int cnt = (int)min((int64_t)32, p1 - pb);
    int my_e = h.e, my_l = h.l;
    if (pb != p0) {
      my_e = lane < cnt ? A.inc_cell[pb + lane] : 0;
      my_l = lane < cnt ? A.inc_local[pb + lane] : 0;
    }
    const double my_f = lane < cnt ? A.cell_rhs[(size_t)nb * my_e + my_l] : 0.0;
    // per lane: the offset of its incidence's element column
    const size_t my_col = (size_t)my_e * cell_stride + (size_t)ld * my_l;
    for (int u0 = 0; u0 < cnt; u0 += U) {
      double kil[U][NI];
      uint16_t sl[U][NI];
      int ev[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool live = u0 + u < cnt;
        const int uu = live ? u0 + u : u0;
        const size_t col = __shfl_sync(0xffffffffu, my_col, uu) + lane;
        ev[u] = __shfl_sync(0xffffffffu, my_e, uu);
        const uint16_t *slp = A.slot + (size_t)(pb + uu) * nb + lane;
#pragma unroll
        for (int c = 0; c < NI; ++c) {
          const bool in = has[c] && live;
          if (F32) kil[u][c] = in ? (double)A.elem32[col + 32 * c] : 0.0;
          else kil[u][c] = in ? A.elem[col + 32 * c] : 0.0;
          sl[u][c] = in ? slp[32 * c] : kConstrainedSlot;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int c = 0; c < NI; ++c) {
          if (sl[u][c] != kConstrainedSlot) {
            img[sl[u][c] * kSliceStride + r] += kil[u][c];
          } else if (A.g && has[c] && u0 + u < cnt) {
            lift += kil[u][c] * A.g[A.gd[(size_t)nb * ev[u] + lane + 32 * c]];
          }
        }
        __syncwarp();
      }
    }
    for (int u = 0; u < cnt; ++u) b += __shfl_sync(0xffffffffu, my_f, u);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lift += __shfl_xor_sync(0xffffffffu, lift, o);
  if (lane == 0) {
    // the diagonal's slot: local row l of any incidence (e, l) of column j
    // has global DoF j, so its slot entry is the diagonal
    const int dslot = p1 > p0 ? A.slot[(size_t)p0 * nb + h.l] : kConstrainedSlot;
    const double d = dslot != kConstrainedSlot ? img[dslot * kSliceStride + r] : 0.0;
    const double di = (fabs(d) > 1.0e-14) ? 1.0 / d : 1.0;
    A.dinv64[row] = di;
    A.dinv32[row] = (float)di;
    A.rhs[row] = b - lift;
  }
}

// Two rows of a warp gathered in lockstep (both with at most 32 incidences):
// batch u0 loads U incidences of each row before either is added, so both
// rows' element columns are in flight together; each row still receives its
// terms in ascending incidence order, into its own column of the image.
template <int NI, int U, bool F32>
__device__ __forceinline__ void slice_pair(const SliceArgs &A, double *img, const int (&r)[2],
                                           const int64_t (&row)[2], int lane,
                                           const SliceRowHead (&h)[2]) {
  const int nb = A.nb;
  const int ld = F32 ? A.ld32 : nb;
  const size_t cell_stride = F32 ? (size_t)A.cs32 : (size_t)nb * nb;
  bool has[NI];
#pragma unroll
  for (int c = 0; c < NI; ++c) has[c] = lane + 32 * c < nb;
  int cnt[2];
  size_t my_col[2];
  double my_f[2], b[2] = {0.0, 0.0}, lift[2] = {0.0, 0.0};
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    cnt[q] = h[q].j >= 0 ? (int)(h[q].p1 - h[q].p0) : 0;
    my_col[q] = (size_t)h[q].e * cell_stride + (size_t)ld * h[q].l;
    my_f[q] = lane < cnt[q] ? A.cell_rhs[(size_t)nb * h[q].e + h[q].l] : 0.0;
  }
  const int n_max = max(cnt[0], cnt[1]);
  for (int u0 = 0; u0 < n_max; u0 += U) {
    double kil[2][U][NI];
    uint16_t sl[2][U][NI];
    int ev[2][U];
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool live = u0 + u < cnt[q];
        const int uu = live ? u0 + u : 0;
        const size_t col = __shfl_sync(0xffffffffu, my_col[q], uu) + lane;
        ev[q][u] = __shfl_sync(0xffffffffu, h[q].e, uu);
        const uint16_t *slp = A.slot + (size_t)(h[q].p0 + uu) * nb + lane;
#pragma unroll
        for (int c = 0; c < NI; ++c) {
          const bool in = has[c] && live;
          if (F32) kil[q][u][c] = in ? (double)A.elem32[col + 32 * c] : 0.0;
          else kil[q][u][c] = in ? A.elem[col + 32 * c] : 0.0;
          sl[q][u][c] = in ? slp[32 * c] : kConstrainedSlot;
        }
      }
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int u = 0; u < U; ++u) {
#pragma unroll
        for (int c = 0; c < NI; ++c) {
          if (sl[q][u][c] != kConstrainedSlot) {
            img[sl[q][u][c] * kSliceStride + r[q]] += kil[q][u][c];
          } else if (A.g && has[c] && u0 + u < cnt[q]) {
            lift[q] += kil[q][u][c] * A.g[A.gd[(size_t)nb * ev[q][u] + lane + 32 * c]];
          }
        }
      }
    __syncwarp();
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    if (h[q].j < 0) continue;
    for (int u = 0; u < cnt[q]; ++u) b[q] += __shfl_sync(0xffffffffu, my_f[q], u);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lift[q] += __shfl_xor_sync(0xffffffffu, lift[q], o);
    if (lane == 0) {
      // the diagonal's slot: local row l of any incidence (e, l) of column j
      // has global DoF j, so its slot entry is the diagonal
      const int dslot = cnt[q] > 0 ? A.slot[(size_t)h[q].p0 * nb + h[q].l] : kConstrainedSlot;
      const double d = dslot != kConstrainedSlot ? img[dslot * kSliceStride + r[q]] : 0.0;
      const double di = (fabs(d) > 1.0e-14) ? 1.0 / d : 1.0;
      A.dinv64[row[q]] = di;
      A.dinv32[row[q]] = (float)di;
      A.rhs[row[q]] = b[q] - lift[q];
    }
  }
}

template <int NI, int U, bool F32>
__global__ void __launch_bounds__(kSliceThreads, 4) sell_slice_kernel(const __grid_constant__ SliceArgs A) {
  extern __shared__ double img[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kW = kSliceThreads / 32;
  const int64_t hs = blockIdx.x;
  const int64_t k = hs >> 1;
  const int half = (int)(hs & 1);
  const int64_t s0 = A.soff[k];
  const int width = (int)((A.soff[k + 1] - s0) / kSliceRows);
  const int64_t row0 = hs * kSliceHalf;
  // both rows' heads before the image is cleared, so their loads overlap it
  SliceRowHead h0, h1;
  slice_head(A, row0 + w, lane, h0);
  slice_head(A, row0 + w + kW, lane, h1);
  for (int q = threadIdx.x; q < width * kSliceStride; q += blockDim.x) img[q] = 0.0;
  __syncthreads();
  if (h0.p1 - h0.p0 <= 32 && h1.p1 - h1.p0 <= 32) {
    const SliceRowHead hh[2] = {h0, h1};
    const int rr[2] = {w, w + kW};
    const int64_t rows[2] = {row0 + w, row0 + w + kW};
    slice_pair<NI, U, F32>(A, img, rr, rows, lane, hh);
  } else {
    if (h0.j >= 0) slice_row<NI, U, F32>(A, img, w, row0 + w, lane, h0);
    if (h1.j >= 0) slice_row<NI, U, F32>(A, img, w + kW, row0 + w + kW, lane, h1);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < width * kSliceHalf; q += blockDim.x) {
    const int sl = q / kSliceHalf, r = q % kSliceHalf;
    const double v = img[sl * kSliceStride + r];
    const int64_t at = s0 + (int64_t)sl * kSliceRows + half * kSliceHalf + r;
    A.val64[at] = v;
    A.val32[at] = (float)v;
  }
}

inline int blocks_for(int64_t n, int t) { return (int)((n + t - 1) / t); }

// ------------------------------------------- batched assembly (serving)
// Independent systems of one family assembled by one launch per phase: a
// thread finds its system by binary search over the prefix sums of cells
// (geometry) or free columns (scatter) and runs the same per-cell / per-column
// body as the single-system kernels, so every system's values are the bits
// it gets alone.
__device__ __forceinline__ int batch_find(const int64_t *begin, int count, int64_t g) {
  int lo = 0, hi = count;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (begin[mid] <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void batch_prep_kernel(const __grid_constant__ AsmBatch B) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < B.count) *B.sys[s].err = 0;
}

template <int FAMILY>
__global__ void batch_geometry_kernel(const __grid_constant__ AsmBatch B) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= B.cell_begin[B.count]) return;
  const int s = batch_find(B.cell_begin, B.count, g);
  const AsmSys &S = B.sys[s];
  const int c = (int)(g - B.cell_begin[s]);
  if (FAMILY == FFG_TETRA_LAGRANGE)
    lagrange_geometry_cell(c, S.cells, S.verts, S.ca, S.cb, S.cell_a, S.cell_b, S.samples, S.nq,
                           S.geo, S.stride, S.err);
  else
    p1_geometry_cell(c, S.cells, S.verts, S.ca, S.cb, S.cell_a, S.cell_b, S.samples, S.geo, S.err);
}

// the SELL-layout scatter of every system, and x = 0 for its solve
template <int FAMILY>
__global__ void batch_column_kernel(const __grid_constant__ AsmBatch B) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= B.col_begin[B.count]) return;
  const int s = batch_find(B.col_begin, B.count, g);
  const AsmSys &S = B.sys[s];
  const int64_t j = g - B.col_begin[s];
  S.x[j] = 0.0;
  column_body<FAMILY, true>(j, S.col_ptr, S.row_idx, S.inc_ptr, S.inc_cell, S.inc_local, S.slot,
                            S.gd, S.nb, S.geo, S.stride, S.ref, S.load_basis, S.nq, nullptr,
                            nullptr, S.g, S.iperm, S.soff, S.val64, S.val32, S.dinv64, S.dinv32,
                            S.rhs, nullptr, 0, 0);
}

// every system's full solution: constrained DoFs from g (or 0), free DoFs
// from the solver's x (SELL order)
__global__ void batch_solution_kernel(const __grid_constant__ AsmBatch B) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= B.dof_begin[B.count]) return;
  const int s = batch_find(B.dof_begin, B.count, g);
  const AsmSys &S = B.sys[s];
  const int64_t d = g - B.dof_begin[s];
  const int f = S.free_index[d];
  S.solution[d] = f >= 0 ? S.x[S.iperm[f]] : (S.g ? S.g[d] : 0.0);
}

}  // namespace

int launch_batch_assembly(int family, int count, const AsmSys *sys, cudaStream_t s) {
  if (family != FFG_TETRA_LAGRANGE && family != FFG_TRIANGLE_P1) return FFG_INVALID_INPUT;
  for (int c0 = 0; c0 < count; c0 += kMaxAsmBatch) {
    AsmBatch B;
    B.count = std::min(kMaxAsmBatch, count - c0);
    B.cell_begin[0] = B.col_begin[0] = B.dof_begin[0] = 0;
    for (int i = 0; i < B.count; ++i) {
      B.sys[i] = sys[c0 + i];
      B.cell_begin[i + 1] = B.cell_begin[i] + B.sys[i].n_cells;
      B.col_begin[i + 1] = B.col_begin[i] + B.sys[i].n_free;
      B.dof_begin[i + 1] = B.dof_begin[i] + B.sys[i].n_dofs;
    }
    batch_prep_kernel<<<1, kMaxAsmBatch, 0, s>>>(B);
    const int64_t nc = B.cell_begin[B.count], nf = B.col_begin[B.count];
    if (family == FFG_TETRA_LAGRANGE) {
      if (nc) batch_geometry_kernel<FFG_TETRA_LAGRANGE><<<blocks_for(nc, 128), 128, 0, s>>>(B);
      if (nf) batch_column_kernel<FFG_TETRA_LAGRANGE><<<blocks_for(nf, 128), 128, 0, s>>>(B);
    } else {
      if (nc) batch_geometry_kernel<FFG_TRIANGLE_P1><<<blocks_for(nc, 128), 128, 0, s>>>(B);
      if (nf) batch_column_kernel<FFG_TRIANGLE_P1><<<blocks_for(nf, 128), 128, 0, s>>>(B);
    }
    if (cudaGetLastError() != cudaSuccess) return FFG_CUDA_ERROR;
  }
  return FFG_OK;
}

int launch_batch_solutions(int count, const AsmSys *sys, cudaStream_t s) {
  for (int c0 = 0; c0 < count; c0 += kMaxAsmBatch) {
    AsmBatch B;
    B.count = std::min(kMaxAsmBatch, count - c0);
    B.dof_begin[0] = 0;
    for (int i = 0; i < B.count; ++i) {
      B.sys[i] = sys[c0 + i];
      B.dof_begin[i + 1] = B.dof_begin[i] + B.sys[i].n_dofs;
    }
    const int64_t nd = B.dof_begin[B.count];
    if (nd) batch_solution_kernel<<<blocks_for(nd, 256), 256, 0, s>>>(B);
    if (cudaGetLastError() != cudaSuccess) return FFG_CUDA_ERROR;
  }
  return FFG_OK;
}

int launch_cell_geometry(const Topology &t, const ElementTables &tab, const DeviceTopology &dt,
                         const AssemblyInputs &in, double *geo, int stride, double *cell_rhs,
                         int *err, cudaStream_t s) {
  (void)cell_rhs;
  const int T = 128;
  if (t.family == FFG_TETRA_LAGRANGE) {
    lagrange_geometry_kernel<<<blocks_for(t.n_cells, T), T, 0, s>>>(
        t.n_cells, dt.cells, in.vertices, in.coef_a, in.coef_b, in.cell_a, in.cell_b, in.samples,
        tab.nq_load, geo, stride, err);
  } else if (t.family == FFG_TRIANGLE_LAGRANGE) {
    triangle_lagrange_geometry_kernel<<<blocks_for(t.n_cells, T), T, 0, s>>>(
        t.n_cells, dt.cells, in.vertices, in.coef_a, in.coef_b, in.cell_a, in.cell_b, in.samples,
        tab.nq_load, geo, stride, err);
  } else if (t.family == FFG_TRIANGLE_P1) {
    p1_geometry_kernel<<<blocks_for(t.n_cells, T), T, 0, s>>>(t.n_cells, dt.cells, in.vertices,
                                                             in.coef_a, in.coef_b, in.cell_a,
                                                             in.cell_b, in.samples, geo, err);
  }
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

int launch_nedelec(const Topology &t, const ElementTables &tab, const DeviceTopology &dt,
                   const AssemblyInputs &in, double *elem, double *cell_rhs, int *err,
                   cudaStream_t s, bool load_only) {
  (void)tab;
  if (!dt.ort) return FFG_INVALID_INPUT;
  return launch_nedelec_oriented(t, *dt.ort, dt, in, elem, cell_rhs, err, s, load_only);
}

int launch_columns(const Topology &t, const ElementTables &tab, const DeviceTopology &dt,
                   const AssemblyInputs &in, const double *geo, int stride,
                   const double *cell_rhs, const double *elem, const int64_t *col_ptr,
                   const int *row_idx, DeviceSell *sell, double *csc_val, double *rhs,
                   cudaStream_t s, const float *elem32, int ld32, int64_t cs32) {
  if (elem32 && cs32 <= 0) cs32 = (int64_t)ld32 * t.nb;
  const int T = (in.tune && in.tune->col_threads) ? in.tune->col_threads : 128;
  const int64_t F = t.n_free();
  if (F == 0) return FFG_OK;
  const int *iperm = sell ? sell->iperm : nullptr;
  const int64_t *soff = sell ? sell->soff : nullptr;
  double *v64 = sell ? sell->val64 : csc_val;
  float *v32 = sell ? sell->val32 : nullptr;
  double *d64 = sell ? sell->dinv64 : nullptr;
  float *d32 = sell ? sell->dinv32 : nullptr;
#define FFG_COLUMN_ARGS                                                                        \
  F, col_ptr, row_idx, dt.inc_ptr, dt.inc_cell, dt.inc_local, dt.slot, dt.gd, t.nb, geo, stride, \
      dt.ref, dt.load_basis, tab.nq_load, elem, cell_rhs, in.g, iperm, soff, v64, v32, d64, d32, rhs, \
      elem32, ld32, cs32
  // high-order CSC columns: one warp per column (48 KB of columns per block)
  constexpr int kColSmem = 48 * 1024;
  const int col_bytes = t.max_column * (int)sizeof(double);
  const bool by_warp = !sell && t.nb >= 16 && t.family != FFG_TRIANGLE_P1 && t.max_column > 0 &&
                       col_bytes <= kColSmem;
  const int wpb = by_warp ? std::max(1, std::min(8, kColSmem / col_bytes)) : 0;
  // Nedelec SELL rows: one CTA per slice while the slice image fits
  const size_t slice_smem = (size_t)t.max_column * kSliceStride * sizeof(double);
  // incidence ranges stored as int32 (every incidence index below 2^31)
  const int64_t n_inc = t.n_free() > 0 ? (int64_t)t.nb * t.n_cells : 0;
  if (sell && t.family == FFG_TETRA_NEDELEC && t.nb >= 16 && t.nb <= 128 && t.max_column > 0 &&
      slice_smem <= 200 * 1024 && sell->perm && n_inc < (int64_t)INT32_MAX) {
    if (!sell->inc_range) {
      if (cudaMalloc((void **)&sell->inc_range, sizeof(int2) * (size_t)F) != cudaSuccess)
        return FFG_OUT_OF_MEMORY;
      inc_range_kernel<<<blocks_for(F, 256), 256, 0, s>>>(F, sell->perm, dt.inc_ptr,
                                                         sell->inc_range);
    }
    SliceArgs A;
    A.range = sell->inc_range;
    A.nb = t.nb;
    A.ld32 = ld32;
    A.cs32 = cs32;
    A.n = F;
    A.perm = sell->perm;
    A.soff = sell->soff;
    A.col_ptr = col_ptr;
    A.inc_ptr = dt.inc_ptr;
    A.row_idx = row_idx;
    A.inc_cell = dt.inc_cell;
    A.gd = dt.gd;
    A.inc_local = dt.inc_local;
    A.slot = dt.slot;
    A.elem = elem;
    A.cell_rhs = cell_rhs;
    A.g = in.g;
    A.elem32 = elem32;
    A.val64 = sell->val64;
    A.dinv64 = sell->dinv64;
    A.rhs = rhs;
    A.val32 = sell->val32;
    A.dinv32 = sell->dinv32;
    const int ni = (t.nb + 31) / 32;
    auto go = [&](auto kern) -> int {
      if (slice_smem > 48 * 1024 &&
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)slice_smem) != cudaSuccess)
        return FFG_CUDA_ERROR;
      kern<<<(unsigned)(2 * sell->n_slices), kSliceThreads, slice_smem, s>>>(A);
      return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
    };
    // about eight loads of each kind in flight per lane
    if (elem32) {
      if (ni == 1) return go(sell_slice_kernel<1, 2, true>);
      if (ni == 2) return go(sell_slice_kernel<2, 1, true>);
      if (ni == 3) return go(sell_slice_kernel<3, 1, true>);
      return go(sell_slice_kernel<4, 1, true>);
    }
    if (ni == 1) return go(sell_slice_kernel<1, 2, false>);
    if (ni == 2) return go(sell_slice_kernel<2, 1, false>);
    if (ni == 3) return go(sell_slice_kernel<3, 1, false>);
    return go(sell_slice_kernel<4, 1, false>);
  }
#define FFG_LAUNCH(FAM)                                                                        \
  do {                                                                                         \
    if (sell)                                                                                  \
      column_kernel<FAM, true><<<blocks_for(F, T), T, 0, s>>>(FFG_COLUMN_ARGS);                \
    else if (by_warp && FAM != FFG_TRIANGLE_P1)                                                \
      csc_column_warp_kernel<FAM><<<(unsigned)((F + wpb - 1) / wpb), 32 * wpb,                 \
                                    (size_t)wpb * col_bytes, s>>>(                             \
          F, t.max_column, col_ptr, dt.inc_ptr, dt.inc_cell, dt.inc_local, dt.slot, dt.gd,      \
          t.nb, geo, stride, dt.ref, dt.load_basis, tab.nq_load, elem, cell_rhs, in.g, v64,    \
          rhs, elem32, ld32, cs32);                                                                  \
    else                                                                                       \
      column_kernel<FAM, false><<<blocks_for(F, T), T, 0, s>>>(FFG_COLUMN_ARGS);               \
  } while (0)
  if (t.family == FFG_TETRA_LAGRANGE)
    FFG_LAUNCH(FFG_TETRA_LAGRANGE);
  else if (t.family == FFG_TRIANGLE_P1)
    FFG_LAUNCH(FFG_TRIANGLE_P1);
  else if (t.family == FFG_TRIANGLE_LAGRANGE)
    FFG_LAUNCH(FFG_TRIANGLE_LAGRANGE);
  else
    FFG_LAUNCH(FFG_TETRA_NEDELEC);
#undef FFG_LAUNCH
#undef FFG_COLUMN_ARGS
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace ffg
