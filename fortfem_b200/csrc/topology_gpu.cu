// Device build of the Lagrange / P1 / Nedelec problem topology: the same arrays as the
// host build in topology.cpp (first-appearance DoF numbering, Dirichlet set,
// constrained CSC pattern, incidences, slot maps) and the solver's SELL layout
// of build_sell, made with sorts and scans instead of hash maps, so that a
// new mesh costs milliseconds instead of seconds.  Every output is integer and
// equal to the host build's, entry for entry.
//
// First appearance: the (key, position) pairs of all local DoFs are sorted by
// key with a stable radix sort, so inside a run of equal keys the positions
// stay in cell-major order and the run's first entry is the key's first
// appearance; flagging first appearances in position order and scanning the
// flags numbers the DoFs exactly as tetra_lagrange_global_dof_map.f90:13-99
// does with its search.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "ffg_internal.h"

namespace ffg {
namespace {

constexpr int kT = 256;
constexpr int kMaxLocalDofs = 216;  // Nedelec order 6 (Lagrange degree 4: 35)
inline unsigned nblk(int64_t n) { return (unsigned)((n + kT - 1) / kT); }

// Device buffer that frees itself.
template <class T>
struct Buf {
  T *p = nullptr;
  Buf() = default;
  Buf(const Buf &) = delete;
  ~Buf() {
    if (p) cudaFree(p);
  }
  bool alloc(size_t n) {
    if (p) cudaFree(p);
    p = nullptr;
    return cudaMalloc((void **)&p, sizeof(T) * std::max<size_t>(n, 1)) == cudaSuccess;
  }
  T *release() {
    T *q = p;
    p = nullptr;
    return q;
  }
};

struct Temp {
  Buf<unsigned char> b;
  size_t bytes = 0;
  bool ensure(size_t n) {
    if (n <= bytes) return true;
    bytes = n;
    return b.alloc(n);
  }
};

#define FFG_TRY(x)                      \
  do {                                  \
    if ((x) != cudaSuccess) {           \
      cudaGetLastError();               \
      return FFG_CUDA_ERROR;            \
    }                                   \
  } while (0)
#define FFG_ALLOC(buf, n)                                      \
  do {                                                         \
    if (!(buf).alloc(n)) {                                     \
      cudaGetLastError();                                      \
      return FFG_OUT_OF_MEMORY;                                \
    }                                                          \
  } while (0)

// stable sort of (key, value) pairs, 64-bit keys
int sort_pairs(Temp &tmp, const uint64_t *kin, uint64_t *kout, const int *vin, int *vout, int n,
               int end_bit = 64) {
  size_t need = 0;
  FFG_TRY(cub::DeviceRadixSort::SortPairs(nullptr, need, kin, kout, vin, vout, n, 0, end_bit));
  if (!tmp.ensure(need)) return FFG_OUT_OF_MEMORY;
  FFG_TRY(cub::DeviceRadixSort::SortPairs(tmp.b.p, need, kin, kout, vin, vout, n, 0, end_bit));
  return FFG_OK;
}

template <class T>
int exclusive_sum(Temp &tmp, const T *in, T *out, int n) {
  size_t need = 0;
  FFG_TRY(cub::DeviceScan::ExclusiveSum(nullptr, need, in, out, n));
  if (!tmp.ensure(need)) return FFG_OUT_OF_MEMORY;
  FFG_TRY(cub::DeviceScan::ExclusiveSum(tmp.b.p, need, in, out, n));
  return FFG_OK;
}

struct MaxOp {
  __device__ int operator()(int a, int b) const { return a > b ? a : b; }
};

int inclusive_max(Temp &tmp, const int *in, int *out, int n) {
  size_t need = 0;
  FFG_TRY(cub::DeviceScan::InclusiveScan(nullptr, need, in, out, MaxOp(), n));
  if (!tmp.ensure(need)) return FFG_OUT_OF_MEMORY;
  FFG_TRY(cub::DeviceScan::InclusiveScan(tmp.b.p, need, in, out, MaxOp(), n));
  return FFG_OK;
}

template <class T>
int read1(const T *p, T &out) {
  FFG_TRY(cudaMemcpy(&out, p, sizeof(T), cudaMemcpyDeviceToHost));
  return FFG_OK;
}

// ------------------------------------------------------------ numbering
// Key of local DoF l of cell c: its sub-simplex vertices with their barycentric
// weights, sorted by vertex, packed as in the host build (vertex+1 << 3 | weight).
__global__ void lagrange_keys_kernel(int64_t n, int nb, const int *cells, const int *idx,
                                     uint64_t *ka, uint64_t *kb, int *pos) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int c = (int)(q / nb), l = (int)(q % nb);
  int vv[4], ww[4], m = 0;
  for (int i = 0; i < 4; ++i) {
    const int w = idx[4 * l + i];
    if (w != 0) {
      vv[m] = cells[4 * (int64_t)c + i];
      ww[m] = w;
      ++m;
    }
  }
  for (int i = 1; i < m; ++i)  // insertion sort by vertex
    for (int j = i; j > 0 && vv[j - 1] > vv[j]; --j) {
      int t = vv[j]; vv[j] = vv[j - 1]; vv[j - 1] = t;
      t = ww[j]; ww[j] = ww[j - 1]; ww[j - 1] = t;
    }
  uint64_t a = 0, b = 0;
  for (int i = 0; i < m; ++i) {
    const uint64_t word = ((uint64_t)(vv[i] + 1) << 3) | (uint64_t)ww[i];
    if (i < 2) a |= word << (32 * i);
    else b |= word << (32 * (i - 2));
  }
  ka[q] = a;
  kb[q] = b;
  pos[q] = (int)q;
}

__global__ void gather_u64_kernel(int64_t n, const uint64_t *src, const int *at, uint64_t *dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[at[i]];
}

// run starts of equal (a, b) keys in sorted order (a gathered through `ord`)
__global__ void run_start_kernel(int64_t n, const uint64_t *ka, const uint64_t *kb_sorted,
                                 const int *ord, int *st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool start = i == 0 || kb_sorted[i] != kb_sorted[i - 1] || ka[ord[i]] != ka[ord[i - 1]];
  st[i] = start ? (int)i : 0;
}

__global__ void first_pos_kernel(int64_t n, const int *ord, const int *run, int *first) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) first[ord[i]] = ord[run[i]];
}

__global__ void first_flag_kernel(int64_t n, const int *first, int *flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = first[i] == (int)i ? 1 : 0;
}

__global__ void number_kernel(int64_t n, const int *first, const int *id, int *gd) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) gd[i] = id[first[i]];
}

// ------------------------------------------------------- Nedelec numbering
// Local edges and faces in the reference's order (tetra_edge_dof_map.f90:10-77,
// tetra_nedelec_global_dof_map.f90:15-105).
__constant__ int kNedEdges[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
__constant__ int kNedFaces[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

// (min, max) vertex key of local edge q = 6 c + le, and its orientation
// (+1 iff the first local vertex has the smaller global index)
__global__ void ned_edge_keys_kernel(int n_cells, const int *cells, uint64_t *key, int *pos,
                                     int8_t *sign) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 6 * (int64_t)n_cells) return;
  const int c = (int)(q / 6), le = (int)(q % 6);
  const int a = cells[4 * (int64_t)c + kNedEdges[le][0]];
  const int b = cells[4 * (int64_t)c + kNedEdges[le][1]];
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  key[q] = ((uint64_t)(uint32_t)lo << 32) | (uint32_t)hi;
  pos[q] = (int)q;
  sign[q] = a < b ? 1 : -1;
}

// sorted-vertex key of local face q = 4 c + lf and the permutation index of
// its local vertex order (ranks of the local vertices among the sorted ones,
// numbered 123, 132, 213, 231, 312, 321 -> 0..5)
__global__ void ned_face_keys_kernel(int n_cells, const int *cells, uint64_t *ka, uint64_t *kb,
                                     int *pos, uint8_t *perm) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 4 * (int64_t)n_cells) return;
  const int c = (int)(q / 4), lf = (int)(q % 4);
  int lv[3], f[3];
  for (int i = 0; i < 3; ++i) lv[i] = f[i] = cells[4 * (int64_t)c + kNedFaces[lf][i]];
  for (int i = 1; i < 3; ++i)
    for (int j = i; j > 0 && f[j - 1] > f[j]; --j) {
      const int t = f[j]; f[j] = f[j - 1]; f[j - 1] = t;
    }
  int r[3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      if (f[j] == lv[i]) r[i] = j + 1;
  const int code = 100 * r[0] + 10 * r[1] + r[2];
  perm[q] = code == 123 ? 0 : code == 132 ? 1 : code == 213 ? 2 : code == 231 ? 3 : code == 312 ? 4 : 5;
  ka[q] = ((uint64_t)(uint32_t)f[0] << 32) | (uint32_t)f[1];
  kb[q] = (uint64_t)(uint32_t)f[2];
  pos[q] = (int)q;
}

// first-appearance ids: id of the run's first position (ids in position order)
__global__ void run_start1_kernel(int64_t n, const uint64_t *ks, int *st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) st[i] = (i == 0 || ks[i] != ks[i - 1]) ? (int)i : 0;
}

__global__ void ned_gd_kernel(int n_cells, int k, int64_t edc, int64_t n_faces,
                              const int *edge_first, const int *edge_id, const int *face_first,
                              const int *face_id, int *gd) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  const int fdc = k * (k - 1), cdc = k * (k - 1) * (k - 2) / 2;
  const int nb = 6 * k + 4 * fdc + cdc;
  int *g = gd + (int64_t)nb * c;
  for (int e = 0; e < 6; ++e) {
    const int64_t ed = edge_id[edge_first[6 * (int64_t)c + e]];
    for (int m = 0; m < k; ++m) g[e * k + m] = (int)(ed * k + m);
  }
  for (int lf = 0; lf < 4; ++lf) {
    const int64_t fa = face_id[face_first[4 * (int64_t)c + lf]];
    for (int m = 0; m < fdc; ++m) g[6 * k + lf * fdc + m] = (int)(edc + fa * fdc + m);
  }
  for (int m = 0; m < cdc; ++m)
    g[6 * k + 4 * fdc + m] = (int)(edc + n_faces * fdc + (int64_t)c * cdc + m);
}

// incidence-one faces of a Nedelec mesh (build_zero_tangential_mask,
// fortfem_tetra_nedelec_solver_3d.f90:416-458): every DoF of the face's three
// edges and every face DoF
__global__ void ned_boundary_kernel(int64_t n, const uint64_t *ka, const uint64_t *kb,
                                    const int *ord, int k, const int *gd, uint8_t *con) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  auto same = [&](int64_t x, int64_t y) {
    return kb[x] == kb[y] && ka[ord[x]] == ka[ord[y]];
  };
  if ((i > 0 && same(i, i - 1)) || (i + 1 < n && same(i, i + 1))) return;
  const int q = ord[i], c = q / 4, lf = q % 4;
  const int fdc = k * (k - 1), cdc = k * (k - 1) * (k - 2) / 2;
  const int nb = 6 * k + 4 * fdc + cdc;
  const int *g = gd + (int64_t)nb * c;
  for (int le = 0; le < 6; ++le) {
    bool oa = false, ob = false;
    for (int j = 0; j < 3; ++j) {
      oa = oa || kNedFaces[lf][j] == kNedEdges[le][0];
      ob = ob || kNedFaces[lf][j] == kNedEdges[le][1];
    }
    if (oa && ob)
      for (int m = 0; m < k; ++m) con[g[le * k + m]] = 1;
  }
  for (int m = 0; m < fdc; ++m) con[g[6 * k + lf * fdc + m]] = 1;
}

// ---------------------------------------------------------- constraints
__global__ void tet_face_keys_kernel(int n_cells, const int *cells, uint64_t *ka, uint64_t *kb,
                                     int *val) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 4 * (int64_t)n_cells) return;
  const int c = (int)(q / 4), o = (int)(q % 4);
  int f[3], m = 0;
  for (int i = 0; i < 4; ++i)
    if (i != o) f[m++] = cells[4 * (int64_t)c + i];
  for (int i = 1; i < 3; ++i)
    for (int j = i; j > 0 && f[j - 1] > f[j]; --j) {
      int t = f[j]; f[j] = f[j - 1]; f[j - 1] = t;
    }
  ka[q] = ((uint64_t)(uint32_t)f[0] << 32) | (uint32_t)f[1];
  kb[q] = (uint64_t)(uint32_t)f[2];
  val[q] = (int)q;
}

__global__ void tri_edge_keys_kernel(int n_cells, const int *cells, uint64_t *key, int *val) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 3 * (int64_t)n_cells) return;
  const int c = (int)(q / 3), e = (int)(q % 3);
  int a = cells[3 * (int64_t)c + e], b = cells[3 * (int64_t)c + (e + 1) % 3];
  if (a > b) { int t = a; a = b; b = t; }
  key[q] = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
  val[q] = (int)q;
}

// incidence-one faces of a Lagrange mesh: constrain the DoFs on them
__global__ void lagrange_boundary_kernel(int64_t n, const uint64_t *ka, const uint64_t *kb,
                                         const int *ord, int nb, const int *idx, const int *gd,
                                         uint8_t *con) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  auto same = [&](int64_t x, int64_t y) {
    return kb[x] == kb[y] && ka[ord[x]] == ka[ord[y]];
  };
  if ((i > 0 && same(i, i - 1)) || (i + 1 < n && same(i, i + 1))) return;
  const int q = ord[i], c = q / 4, o = q % 4;
  for (int l = 0; l < nb; ++l)
    if (idx[4 * l + o] == 0) con[gd[(int64_t)nb * c + l]] = 1;
}

__global__ void p1_boundary_kernel(int64_t n, const uint64_t *key, uint8_t *con) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if ((i > 0 && key[i] == key[i - 1]) || (i + 1 < n && key[i] == key[i + 1])) return;
  con[key[i] >> 32] = 1;
  con[key[i] & 0xffffffffu] = 1;
}

__global__ void mask_kernel(int64_t n, const uint8_t *mask, uint8_t *con) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) con[i] = mask[i] ? 1 : 0;
}

__global__ void free_flag_kernel(int64_t n, const uint8_t *con, int *flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = con[i] ? 0 : 1;
}

__global__ void free_index_kernel(int64_t n, const uint8_t *con, const int *fi, int *free_index,
                                  int *free_dofs) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (con[i]) {
    free_index[i] = -1;
  } else {
    free_index[i] = fi[i];
    free_dofs[fi[i]] = (int)i;
  }
}

// ------------------------------------------------- incidences and pattern
__global__ void inc_flag_kernel(int64_t n, const int *gd, const int *free_index, int *flag) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) flag[q] = free_index[gd[q]] >= 0 ? 1 : 0;
}

__global__ void inc_pairs_kernel(int64_t n, int nb, const int *gd, const int *free_index,
                                 const int *at, uint64_t *key, int *val) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int f = free_index[gd[q]];
  if (f < 0) return;
  const int c = (int)(q / nb), l = (int)(q % nb);
  key[at[q]] = ((uint64_t)(uint32_t)f << 32) | (uint32_t)c;
  val[at[q]] = l;
}

__global__ void inc_unpack_kernel(int64_t n, const uint64_t *key, const int *val, int *cell,
                                  uint8_t *local, int *col, int64_t *ptr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int f = (int)(key[i] >> 32);
  cell[i] = (int)(key[i] & 0xffffffffu);
  local[i] = (uint8_t)val[i];
  col[i] = f;
  if (i + 1 == n || (int)(key[i + 1] >> 32) != f) ptr[f + 1] = i + 1;
  if (i == 0) ptr[0] = 0;
}

// number of coupled (free row, free column) pairs per cell
__global__ void cell_free_count_kernel(int n_cells, int nb, const int *gd, const int *free_index,
                                       int *cnt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  int m = 0;
  for (int l = 0; l < nb; ++l) m += free_index[gd[(int64_t)nb * c + l]] >= 0;
  cnt[c] = m * m;
}

__global__ void pattern_pairs_kernel(int n_cells, int nb, const int *gd, const int *free_index,
                                     const int *at, uint64_t *key) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  int f[kMaxLocalDofs], m = 0;  // Nedelec order 6: 216 local DoFs
  for (int l = 0; l < nb; ++l) {
    const int x = free_index[gd[(int64_t)nb * c + l]];
    if (x >= 0) f[m++] = x;
  }
  int64_t o = at[c];
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < m; ++i) key[o++] = ((uint64_t)(uint32_t)f[j] << 32) | (uint32_t)f[i];
}

__global__ void unique_flag_kernel(int64_t n, const uint64_t *key, int *flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

__global__ void pattern_unpack_kernel(int64_t n, const uint64_t *key, const int *flag,
                                      const int *at, int *row, int64_t *col_ptr) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  const int e = at[i];
  const int j = (int)(key[i] >> 32);
  row[e] = (int)(key[i] & 0xffffffffu);
  // the last unique entry of column j closes it
  int64_t k = i + 1;
  while (k < n && key[k] == key[i]) ++k;
  if (k == n || (int)(key[k] >> 32) != j) col_ptr[j + 1] = e + 1;
  if (e == 0) col_ptr[0] = 0;
}

__global__ void col_len_kernel(int64_t n, const int64_t *col_ptr, int *len) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) len[j] = (int)(col_ptr[j + 1] - col_ptr[j]);
}

__global__ void slot_kernel(int64_t n_inc, int nb, const int *inc_col, const int *inc_cell,
                            const int *gd, const int *free_index, const int64_t *col_ptr,
                            const int *row, uint16_t *slot) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_inc * nb) return;
  const int64_t p = q / nb;
  const int i = (int)(q % nb);
  const int f = free_index[gd[(int64_t)nb * inc_cell[p] + i]];
  if (f < 0) {
    slot[q] = kConstrainedSlot;
    return;
  }
  const int j = inc_col[p];
  int64_t lo = col_ptr[j], hi = col_ptr[j + 1];
  const int64_t base = lo;
  while (lo < hi) {  // lower_bound
    const int64_t mid = (lo + hi) / 2;
    if (row[mid] < f) lo = mid + 1;
    else hi = mid;
  }
  slot[q] = (uint16_t)(lo - base);
}

// ---------------------------------------------------------------- SELL
__global__ void sell_keys_kernel(int64_t n, const int *len, int sigma, uint64_t *key, int *val) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  key[r] = ((uint64_t)(r / sigma) << 32) | (uint64_t)(0xFFFFu - (unsigned)len[r]);
  val[r] = (int)r;
}

__global__ void iperm_kernel(int64_t n, const int *perm, int *iperm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) iperm[perm[i]] = (int)i;
}

__global__ void slice_width_kernel(int64_t n, int64_t n_slices, const int *perm, const int *len,
                                   int64_t *w) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slices) return;
  int mx = 0;
  for (int l = 0; l < kSliceRows; ++l) {
    const int64_t r = s * kSliceRows + l;
    if (r < n) mx = max(mx, len[perm[r]]);
  }
  w[s] = (int64_t)mx * kSliceRows;
}

__global__ void span_kernel(int64_t n, const int64_t *col_ptr, const int *row, const int *iperm,
                            int *lo, int *hi) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  int a = 0, b = 0;
  const int ir = iperm[r];
  for (int64_t e = col_ptr[r]; e < col_ptr[r + 1]; ++e) {
    const int d = iperm[row[e]] - ir;
    a = min(a, d);
    b = max(b, d);
  }
  lo[r] = a;
  hi[r] = b;
}

struct MinOp {
  __device__ int operator()(int a, int b) const { return a < b ? a : b; }
};

__global__ void sell_fill_kernel(int64_t n, int64_t n_slices, const int64_t *soff,
                                 const int *perm, const int *iperm, const int64_t *col_ptr,
                                 const int *row, int16_t *dcol, int *col) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_slices * kSliceRows) return;
  const int64_t s = r / kSliceRows;
  const int64_t width = (soff[s + 1] - soff[s]) / kSliceRows;
  const int64_t base = soff[s] + (r % kSliceRows);
  if (r >= n) {  // rows that only pad the last slice point at the last row
    for (int64_t k = 0; k < width; ++k) {
      if (dcol) dcol[base + k * kSliceRows] = (int16_t)((n - 1) - r);
      else col[base + k * kSliceRows] = (int)(n - 1);
    }
    return;
  }
  const int old = perm[r];
  int64_t k = 0;
  for (int64_t e = col_ptr[old]; e < col_ptr[old + 1]; ++e, ++k) {
    const int c = iperm[row[e]];
    if (dcol) dcol[base + k * kSliceRows] = (int16_t)(c - r);
    else col[base + k * kSliceRows] = c;
  }
  for (; k < width; ++k) {
    if (dcol) dcol[base + k * kSliceRows] = 0;
    else col[base + k * kSliceRows] = (int)r;
  }
}

}  // namespace

int build_topology_device(Topology &t, int mode, const uint8_t *mask, int grid,
                          DeviceTopology &dt, int64_t **csc_col_ptr, int **csc_row,
                          DeviceSell &S, std::string &msg) {
  const bool p1 = t.family == FFG_TRIANGLE_P1;
  const bool ned = t.family == FFG_TETRA_NEDELEC;
  if (!p1 && !ned && t.family != FFG_TETRA_LAGRANGE) {
    msg = "device topology: family";
    return FFG_INVALID_INPUT;
  }
  const int nc = t.n_cells;
  std::vector<int> idx;
  if (p1) {
    t.nb = 3;
  } else if (ned) {
    if (t.degree < 1 || t.degree > 6) { msg = "Nedelec order must be 1..6"; return FFG_INVALID_INPUT; }
    t.nb = nedelec_dof_count(t.degree);
  } else {
    if (t.degree < 1 || t.degree > 4) { msg = "Lagrange degree must be 1..4"; return FFG_INVALID_INPUT; }
    std::vector<double> nodes;
    lagrange_indices(t.degree, idx, nodes);
    t.nb = lagrange_dof_count(t.degree);
  }
  if (t.n_vertices >= (1 << 29)) { msg = "too many vertices"; return FFG_INVALID_INPUT; }
  const int nb = t.nb;
  const int64_t nl = (int64_t)nc * nb;
  if (nl >= (int64_t)1 << 31) { msg = "mesh too large for the device topology"; return FFG_INVALID_INPUT; }
  Temp tmp;
  Buf<int> cells, d_idx, gd;
  FFG_ALLOC(cells, (size_t)t.vpc * nc);
  FFG_TRY(cudaMemcpy(cells.p, t.cells.data(), sizeof(int) * t.cells.size(), cudaMemcpyHostToDevice));
  FFG_ALLOC(gd, (size_t)nl);
  int st;
  // Nedelec face keys stay for the boundary faces
  Buf<uint64_t> nfa, nfb_sorted;
  Buf<int> nford;
  Buf<int8_t> esign;
  Buf<uint8_t> fperm;
  // ---- DoF numbering
  if (p1) {
    FFG_TRY(cudaMemcpy(gd.p, cells.p, sizeof(int) * nl, cudaMemcpyDeviceToDevice));
    t.n_dofs = t.n_vertices;
  } else if (ned) {
    const int k = t.degree, fdc = k * (k - 1), cdc = k * (k - 1) * (k - 2) / 2;
    const int64_t nle = 6 * (int64_t)nc, nlf = 4 * (int64_t)nc;
    // edges by first appearance
    Buf<uint64_t> ek, eks;
    Buf<int> epos, eord, est, erun, efirst, eflag, eid;
    FFG_ALLOC(ek, nle); FFG_ALLOC(eks, nle); FFG_ALLOC(epos, nle); FFG_ALLOC(eord, nle);
    FFG_ALLOC(esign, nle);
    ned_edge_keys_kernel<<<nblk(nle), kT>>>(nc, cells.p, ek.p, epos.p, esign.p);
    if ((st = sort_pairs(tmp, ek.p, eks.p, epos.p, eord.p, (int)nle))) return st;
    FFG_ALLOC(est, nle); FFG_ALLOC(erun, nle);
    run_start1_kernel<<<nblk(nle), kT>>>(nle, eks.p, est.p);
    if ((st = inclusive_max(tmp, est.p, erun.p, (int)nle))) return st;
    FFG_ALLOC(efirst, nle); FFG_ALLOC(eflag, nle); FFG_ALLOC(eid, nle);
    first_pos_kernel<<<nblk(nle), kT>>>(nle, eord.p, erun.p, efirst.p);
    first_flag_kernel<<<nblk(nle), kT>>>(nle, efirst.p, eflag.p);
    if ((st = exclusive_sum(tmp, eflag.p, eid.p, (int)nle))) return st;
    int last_e = 0, last_ef = 0;
    if ((st = read1(eid.p + nle - 1, last_e)) || (st = read1(eflag.p + nle - 1, last_ef))) return st;
    const int64_t n_edges = (int64_t)last_e + last_ef;
    // faces by first appearance
    Buf<uint64_t> fkb, fk1;
    Buf<int> fpos, fo1, fst, frun, ffirst, fflag2, fid;
    FFG_ALLOC(nfa, nlf); FFG_ALLOC(fkb, nlf); FFG_ALLOC(fk1, nlf); FFG_ALLOC(nfb_sorted, nlf);
    FFG_ALLOC(fpos, nlf); FFG_ALLOC(fo1, nlf); FFG_ALLOC(nford, nlf); FFG_ALLOC(fperm, nlf);
    ned_face_keys_kernel<<<nblk(nlf), kT>>>(nc, cells.p, nfa.p, fkb.p, fpos.p, fperm.p);
    if ((st = sort_pairs(tmp, nfa.p, fk1.p, fpos.p, fo1.p, (int)nlf))) return st;
    gather_u64_kernel<<<nblk(nlf), kT>>>(nlf, fkb.p, fo1.p, fk1.p);
    if ((st = sort_pairs(tmp, fk1.p, nfb_sorted.p, fo1.p, nford.p, (int)nlf))) return st;
    FFG_ALLOC(fst, nlf); FFG_ALLOC(frun, nlf);
    run_start_kernel<<<nblk(nlf), kT>>>(nlf, nfa.p, nfb_sorted.p, nford.p, fst.p);
    if ((st = inclusive_max(tmp, fst.p, frun.p, (int)nlf))) return st;
    FFG_ALLOC(ffirst, nlf); FFG_ALLOC(fflag2, nlf); FFG_ALLOC(fid, nlf);
    first_pos_kernel<<<nblk(nlf), kT>>>(nlf, nford.p, frun.p, ffirst.p);
    first_flag_kernel<<<nblk(nlf), kT>>>(nlf, ffirst.p, fflag2.p);
    if ((st = exclusive_sum(tmp, fflag2.p, fid.p, (int)nlf))) return st;
    int last_f = 0, last_ff = 0;
    if ((st = read1(fid.p + nlf - 1, last_f)) || (st = read1(fflag2.p + nlf - 1, last_ff))) return st;
    const int64_t n_faces = (int64_t)last_f + last_ff;
    const int64_t edc = (int64_t)k * n_edges;
    const int64_t total = edc + n_faces * fdc + (int64_t)nc * cdc;
    if (total >= (1LL << 31)) { msg = "too many DoFs"; return FFG_INVALID_INPUT; }
    ned_gd_kernel<<<nblk(nc), kT>>>(nc, k, edc, n_faces, efirst.p, eid.p, ffirst.p, fid.p, gd.p);
    t.n_edges = (int)n_edges;
    t.n_faces = (int)n_faces;
    t.n_dofs = total;
  } else {
    FFG_ALLOC(d_idx, idx.size());
    FFG_TRY(cudaMemcpy(d_idx.p, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice));
    Buf<uint64_t> ka, kb, k1, k2;
    Buf<int> pos, o1, o2, runst, run, first, flag, id;
    FFG_ALLOC(ka, nl); FFG_ALLOC(kb, nl); FFG_ALLOC(k1, nl); FFG_ALLOC(k2, nl);
    FFG_ALLOC(pos, nl); FFG_ALLOC(o1, nl); FFG_ALLOC(o2, nl);
    lagrange_keys_kernel<<<nblk(nl), kT>>>(nl, nb, cells.p, d_idx.p, ka.p, kb.p, pos.p);
    if ((st = sort_pairs(tmp, ka.p, k1.p, pos.p, o1.p, (int)nl))) return st;
    gather_u64_kernel<<<nblk(nl), kT>>>(nl, kb.p, o1.p, k1.p);
    if ((st = sort_pairs(tmp, k1.p, k2.p, o1.p, o2.p, (int)nl))) return st;
    FFG_ALLOC(runst, nl); FFG_ALLOC(run, nl);
    run_start_kernel<<<nblk(nl), kT>>>(nl, ka.p, k2.p, o2.p, runst.p);
    if ((st = inclusive_max(tmp, runst.p, run.p, (int)nl))) return st;
    FFG_ALLOC(first, nl); FFG_ALLOC(flag, nl); FFG_ALLOC(id, nl);
    first_pos_kernel<<<nblk(nl), kT>>>(nl, o2.p, run.p, first.p);
    first_flag_kernel<<<nblk(nl), kT>>>(nl, first.p, flag.p);
    if ((st = exclusive_sum(tmp, flag.p, id.p, (int)nl))) return st;
    number_kernel<<<nblk(nl), kT>>>(nl, first.p, id.p, gd.p);
    int last_id = 0, last_flag = 0;
    if ((st = read1(id.p + nl - 1, last_id)) || (st = read1(flag.p + nl - 1, last_flag))) return st;
    t.n_dofs = last_id + last_flag;
  }
  const int64_t N = t.n_dofs;
  // ---- constraints
  Buf<uint8_t> con;
  FFG_ALLOC(con, (size_t)N);
  FFG_TRY(cudaMemset(con.p, 0, (size_t)N));
  if (mode == FFG_BOUNDARY_MASK) {
    if (!mask) { msg = "boundary mask missing"; return FFG_INVALID_INPUT; }
    Buf<uint8_t> m;
    FFG_ALLOC(m, (size_t)N);
    FFG_TRY(cudaMemcpy(m.p, mask, (size_t)N, cudaMemcpyHostToDevice));
    mask_kernel<<<nblk(N), kT>>>(N, m.p, con.p);
  } else if (mode == FFG_BOUNDARY_ALL) {
    if (ned) {
      ned_boundary_kernel<<<nblk(4 * (int64_t)nc), kT>>>(4 * (int64_t)nc, nfa.p, nfb_sorted.p,
                                                        nford.p, t.degree, gd.p, con.p);
    } else if (p1) {
      const int64_t ne = 3 * (int64_t)nc;
      Buf<uint64_t> k, ks;
      Buf<int> v, vs;
      FFG_ALLOC(k, ne); FFG_ALLOC(ks, ne); FFG_ALLOC(v, ne); FFG_ALLOC(vs, ne);
      tri_edge_keys_kernel<<<nblk(ne), kT>>>(nc, cells.p, k.p, v.p);
      if ((st = sort_pairs(tmp, k.p, ks.p, v.p, vs.p, (int)ne))) return st;
      p1_boundary_kernel<<<nblk(ne), kT>>>(ne, ks.p, con.p);
    } else {
      const int64_t nf = 4 * (int64_t)nc;
      Buf<uint64_t> ka, kb, k1, k2;
      Buf<int> v, o1, o2;
      FFG_ALLOC(ka, nf); FFG_ALLOC(kb, nf); FFG_ALLOC(k1, nf); FFG_ALLOC(k2, nf);
      FFG_ALLOC(v, nf); FFG_ALLOC(o1, nf); FFG_ALLOC(o2, nf);
      tet_face_keys_kernel<<<nblk(nf), kT>>>(nc, cells.p, ka.p, kb.p, v.p);
      if ((st = sort_pairs(tmp, ka.p, k1.p, v.p, o1.p, (int)nf))) return st;
      gather_u64_kernel<<<nblk(nf), kT>>>(nf, kb.p, o1.p, k1.p);
      if ((st = sort_pairs(tmp, k1.p, k2.p, o1.p, o2.p, (int)nf))) return st;
      lagrange_boundary_kernel<<<nblk(nf), kT>>>(nf, ka.p, k2.p, o2.p, nb, d_idx.p, gd.p, con.p);
    }
  } else if (mode != FFG_BOUNDARY_NONE) {
    msg = "bad boundary mode";
    return FFG_INVALID_INPUT;
  }
  // ---- free numbering
  Buf<int> fflag, fi, free_index, free_dofs;
  FFG_ALLOC(fflag, N); FFG_ALLOC(fi, N); FFG_ALLOC(free_index, N);
  free_flag_kernel<<<nblk(N), kT>>>(N, con.p, fflag.p);
  if ((st = exclusive_sum(tmp, fflag.p, fi.p, (int)N))) return st;
  int F = 0, lastf = 0;
  if ((st = read1(fi.p + N - 1, F)) || (st = read1(fflag.p + N - 1, lastf))) return st;
  F += lastf;
  FFG_ALLOC(free_dofs, F);
  free_index_kernel<<<nblk(N), kT>>>(N, con.p, fi.p, free_index.p, free_dofs.p);
  if (F == 0) { msg = "device topology: no free DoFs"; return FFG_INVALID_INPUT; }
  // ---- incidences (free column, cell ascending)
  Buf<int> iflag, iat;
  FFG_ALLOC(iflag, nl); FFG_ALLOC(iat, nl);
  inc_flag_kernel<<<nblk(nl), kT>>>(nl, gd.p, free_index.p, iflag.p);
  if ((st = exclusive_sum(tmp, iflag.p, iat.p, (int)nl))) return st;
  int n_inc = 0, lasti = 0;
  if ((st = read1(iat.p + nl - 1, n_inc)) || (st = read1(iflag.p + nl - 1, lasti))) return st;
  n_inc += lasti;
  Buf<uint64_t> ik, iks;
  Buf<int> iv, ivs, inc_cell, inc_col;
  Buf<uint8_t> inc_local;
  Buf<int64_t> inc_ptr;
  FFG_ALLOC(ik, n_inc); FFG_ALLOC(iks, n_inc); FFG_ALLOC(iv, n_inc); FFG_ALLOC(ivs, n_inc);
  inc_pairs_kernel<<<nblk(nl), kT>>>(nl, nb, gd.p, free_index.p, iat.p, ik.p, iv.p);
  if ((st = sort_pairs(tmp, ik.p, iks.p, iv.p, ivs.p, n_inc))) return st;
  FFG_ALLOC(inc_cell, n_inc); FFG_ALLOC(inc_col, n_inc); FFG_ALLOC(inc_local, n_inc);
  FFG_ALLOC(inc_ptr, (size_t)F + 1);
  inc_unpack_kernel<<<nblk(n_inc), kT>>>(n_inc, iks.p, ivs.p, inc_cell.p, inc_local.p, inc_col.p,
                                         inc_ptr.p);
  // ---- pattern of the constrained system
  Buf<int> ccnt, cat;
  FFG_ALLOC(ccnt, nc); FFG_ALLOC(cat, nc);
  cell_free_count_kernel<<<nblk(nc), kT>>>(nc, nb, gd.p, free_index.p, ccnt.p);
  if ((st = exclusive_sum(tmp, ccnt.p, cat.p, nc))) return st;
  int npairs = 0, lastc = 0;
  if ((st = read1(cat.p + nc - 1, npairs)) || (st = read1(ccnt.p + nc - 1, lastc))) return st;
  if ((int64_t)npairs + lastc >= ((int64_t)1 << 31)) { msg = "device topology: too many couplings"; return FFG_INVALID_INPUT; }
  npairs += lastc;
  Buf<int64_t> col_ptr;
  Buf<int> row;
  int64_t nnz = 0;
  {
    Buf<uint64_t> pk, pks;
    FFG_ALLOC(pk, npairs); FFG_ALLOC(pks, npairs);
    pattern_pairs_kernel<<<nblk(nc), kT>>>(nc, nb, gd.p, free_index.p, cat.p, pk.p);
    size_t need = 0;
    FFG_TRY(cub::DeviceRadixSort::SortKeys(nullptr, need, pk.p, pks.p, npairs));
    if (!tmp.ensure(need)) return FFG_OUT_OF_MEMORY;
    FFG_TRY(cub::DeviceRadixSort::SortKeys(tmp.b.p, need, pk.p, pks.p, npairs));
    Buf<int> uf, uat;
    FFG_ALLOC(uf, npairs); FFG_ALLOC(uat, npairs);
    unique_flag_kernel<<<nblk(npairs), kT>>>(npairs, pks.p, uf.p);
    if ((st = exclusive_sum(tmp, uf.p, uat.p, npairs))) return st;
    int lastu = 0, lasta = 0;
    if ((st = read1(uat.p + npairs - 1, lasta)) || (st = read1(uf.p + npairs - 1, lastu))) return st;
    nnz = (int64_t)lasta + lastu;
    FFG_ALLOC(row, nnz);
    FFG_ALLOC(col_ptr, (size_t)F + 1);
    pattern_unpack_kernel<<<nblk(npairs), kT>>>(npairs, pks.p, uf.p, uat.p, row.p, col_ptr.p);
  }
  Buf<int> clen;
  FFG_ALLOC(clen, F);
  col_len_kernel<<<nblk(F), kT>>>(F, col_ptr.p, clen.p);
  int maxc = 0;
  {
    Buf<int> mx;
    FFG_ALLOC(mx, 1);
    size_t need = 0;
    FFG_TRY(cub::DeviceReduce::Max(nullptr, need, clen.p, mx.p, F));
    if (!tmp.ensure(need)) return FFG_OUT_OF_MEMORY;
    FFG_TRY(cub::DeviceReduce::Max(tmp.b.p, need, clen.p, mx.p, F));
    if ((st = read1(mx.p, maxc))) return st;
  }
  if (maxc > kMaxColumnLength) { msg = "a CSC column exceeds 65534 entries"; return FFG_INVALID_INPUT; }
  // ---- slot maps
  Buf<uint16_t> slot;
  FFG_ALLOC(slot, (size_t)n_inc * nb);
  slot_kernel<<<nblk((int64_t)n_inc * nb), kT>>>(n_inc, nb, inc_col.p, inc_cell.p, gd.p,
                                                  free_index.p, col_ptr.p, row.p, slot.p);
  // ---- SELL-32-sigma layout (build_sell)
  free_sell(S);
  S.n = F;
  S.n_slices = (F + kSliceRows - 1) / kSliceRows;
  S.grid = grid;
  Buf<int> perm, iperm;
  {
    Buf<uint64_t> sk, sks;
    Buf<int> sv;
    FFG_ALLOC(sk, F); FFG_ALLOC(sks, F); FFG_ALLOC(sv, F); FFG_ALLOC(perm, F); FFG_ALLOC(iperm, F);
    sell_keys_kernel<<<nblk(F), kT>>>(F, clen.p, kSellSigma, sk.p, sv.p);
    if ((st = sort_pairs(tmp, sk.p, sks.p, sv.p, perm.p, F))) return st;
    iperm_kernel<<<nblk(F), kT>>>(F, perm.p, iperm.p);
  }
  Buf<int64_t> widths, soff;
  FFG_ALLOC(widths, (size_t)S.n_slices + 1); FFG_ALLOC(soff, (size_t)S.n_slices + 1);
  slice_width_kernel<<<nblk(S.n_slices), kT>>>(F, S.n_slices, perm.p, clen.p, widths.p);
  FFG_TRY(cudaMemset(widths.p + S.n_slices, 0, sizeof(int64_t)));
  if ((st = exclusive_sum(tmp, widths.p, soff.p, (int)S.n_slices + 1))) return st;
  if ((st = read1(soff.p + S.n_slices, S.padded))) return st;
  bool narrow;
  {
    Buf<int> lo, hi, r;
    FFG_ALLOC(lo, F); FFG_ALLOC(hi, F); FFG_ALLOC(r, 1);
    span_kernel<<<nblk(F), kT>>>(F, col_ptr.p, row.p, iperm.p, lo.p, hi.p);
    size_t need = 0;
    FFG_TRY(cub::DeviceReduce::Reduce(nullptr, need, lo.p, r.p, F, MinOp(), 0));
    if (!tmp.ensure(need)) return FFG_OUT_OF_MEMORY;
    FFG_TRY(cub::DeviceReduce::Reduce(tmp.b.p, need, lo.p, r.p, F, MinOp(), 0));
    int dmin = 0, dmax = 0;
    if ((st = read1(r.p, dmin))) return st;
    FFG_TRY(cub::DeviceReduce::Max(nullptr, need, hi.p, r.p, F));
    if (!tmp.ensure(need)) return FFG_OUT_OF_MEMORY;
    FFG_TRY(cub::DeviceReduce::Max(tmp.b.p, need, hi.p, r.p, F));
    if ((st = read1(r.p, dmax))) return st;
    narrow = dmin >= -32768 && dmax <= 32767;
  }
  const size_t P = (size_t)std::max<int64_t>(S.padded, 1);
  Buf<int16_t> dcol;
  Buf<int> colw;
  Buf<double> v64, d64;
  Buf<float> v32, d32;
  Buf<int> cta, wsl, wof;
  if (narrow) FFG_ALLOC(dcol, P);
  else FFG_ALLOC(colw, P);
  FFG_ALLOC(v64, P); FFG_ALLOC(v32, P); FFG_ALLOC(d64, F); FFG_ALLOC(d32, F);
  FFG_TRY(cudaMemset(v64.p, 0, sizeof(double) * P));
  FFG_TRY(cudaMemset(v32.p, 0, sizeof(float) * P));
  sell_fill_kernel<<<nblk(S.n_slices * kSliceRows), kT>>>(F, S.n_slices, soff.p, perm.p, iperm.p,
                                                           col_ptr.p, row.p, dcol.p, colw.p);
  // CTA partition and per-warp slice lists
  std::vector<int64_t> hsoff((size_t)S.n_slices + 1);
  FFG_TRY(cudaMemcpy(hsoff.data(), soff.p, sizeof(int64_t) * hsoff.size(), cudaMemcpyDeviceToHost));
  std::vector<int> cs, hws, hwo;
  sell_partition(hsoff.data(), S.n_slices, grid, cs, hws, hwo);
  FFG_ALLOC(cta, cs.size());
  FFG_ALLOC(wsl, std::max<size_t>(hws.size(), 1));
  FFG_ALLOC(wof, hwo.size());
  FFG_TRY(cudaMemcpy(cta.p, cs.data(), sizeof(int) * cs.size(), cudaMemcpyHostToDevice));
  if (!hws.empty())
    FFG_TRY(cudaMemcpy(wsl.p, hws.data(), sizeof(int) * hws.size(), cudaMemcpyHostToDevice));
  FFG_TRY(cudaMemcpy(wof.p, hwo.data(), sizeof(int) * hwo.size(), cudaMemcpyHostToDevice));
  FFG_TRY(cudaDeviceSynchronize());
  // ---- host copies the library reads later
  t.gd.resize((size_t)nl);
  t.constrained.resize((size_t)N);
  t.free_dofs.resize((size_t)F);
  t.col_ptr.resize((size_t)F + 1);
  t.row_idx.resize((size_t)nnz);
  FFG_TRY(cudaMemcpy(t.gd.data(), gd.p, sizeof(int) * nl, cudaMemcpyDeviceToHost));
  FFG_TRY(cudaMemcpy(t.constrained.data(), con.p, (size_t)N, cudaMemcpyDeviceToHost));
  FFG_TRY(cudaMemcpy(t.free_dofs.data(), free_dofs.p, sizeof(int) * F, cudaMemcpyDeviceToHost));
  FFG_TRY(cudaMemcpy(t.col_ptr.data(), col_ptr.p, sizeof(int64_t) * (F + 1), cudaMemcpyDeviceToHost));
  FFG_TRY(cudaMemcpy(t.row_idx.data(), row.p, sizeof(int) * nnz, cudaMemcpyDeviceToHost));
  t.max_column = maxc;
  if (ned) {
    t.edge_sign.resize(6 * (size_t)nc);
    t.face_perm.resize(4 * (size_t)nc);
    FFG_TRY(cudaMemcpy(t.edge_sign.data(), esign.p, 6 * (size_t)nc, cudaMemcpyDeviceToHost));
    FFG_TRY(cudaMemcpy(t.face_perm.data(), fperm.p, 4 * (size_t)nc, cudaMemcpyDeviceToHost));
    dt.edge_sign = esign.release();
    dt.face_perm = fperm.release();
  }
  // ---- hand the device arrays over
  dt.cells = cells.release();
  dt.gd = gd.release();
  dt.free_index = free_index.release();
  dt.inc_ptr = inc_ptr.release();
  dt.inc_cell = inc_cell.release();
  dt.inc_local = inc_local.release();
  dt.slot = slot.release();
  *csc_col_ptr = col_ptr.release();
  *csc_row = row.release();
  S.soff = soff.release();
  S.dcol = narrow ? dcol.release() : nullptr;
  S.col = narrow ? nullptr : colw.release();
  S.val64 = v64.release();
  S.val32 = v32.release();
  S.dinv64 = d64.release();
  S.dinv32 = d32.release();
  S.perm = perm.release();
  S.iperm = iperm.release();
  S.cta_slice = cta.release();
  S.wslice = wsl.release();
  S.woff = wof.release();
  return FFG_OK;
}

}  // namespace ffg
