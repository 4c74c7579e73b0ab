// Oriented reference tensors of the first-kind Nedelec element matrices and
// loads, and the FP64 contraction kernels that use them.
//
// The reference orients the local basis of every cell by a block-diagonal T
// (build_tetra_nedelec_basis_transform, tetra_nedelec_global_dof_map.f90:107-155,
// applied as T^T K T in assemble_arbitrary_order_curl_mass_csc,
// src/assembly/assembly_tetra_nedelec_3d.f90:2340-2342): -1 on the even
// moments of an edge whose first local vertex has the larger global index,
// one of six dense face blocks chosen by the order of the face's global
// vertex indices, identity on the cell moments.  Both choices depend only on
// the order of the cell's four global vertex indices, so every cell falls in
// one of 24 classes, and
//     K_cell = T^T (sum_s w_s R_s) T = sum_s w_s (T^T R_s T),
//     F_cell = T^T sum_q (det J^-1 f_q) . (w_q v(q)) = sum_{q,a} (det J^-1 f_q)_a (T^T w_q v_a(q))
// with the twelve reference tensors R_s of the curl + mass contraction and
// the weighted load basis tabulated once per class.  Cells listed class by
// class in tiles of 64 turn both into dense contractions: per tile one table,
// 64 rows of weights, and every output entry a short FMA chain with
// warp-uniform weights and lane-contiguous table rows and stores.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "ffg_internal.h"
#include "tet_geometry.h"

namespace ffg {

namespace {

constexpr int kOrtThreads = 256;   // eight warps, eight cells each
constexpr int kOrtChunk = 128;     // output entries per pass: four per lane


struct OrtArgs {
  int nb, nql;
  const int *cells;
  const double *verts;
  double ca, cb;
  const double *cell_a, *cell_b;
  const double *geo_in;     // caller weights (12 per cell) or null
  const double *verts_dot;  // tangent direction (forward mode) or null
  double ca_dot, cb_dot;
  const double *samples;    // 3 nql per cell or null
  const int *order;         // cells in class order
  const int4 *tiles;
  const double *ref;        // kOrtClasses x n_chunks x 12 x kOrtChunk (entries chunk-major)
  const double *load;       // kOrtClasses x load_stride: 3 nql x nb per class
  int64_t load_stride;      // 3 nql nb rounded up to an even count (16-byte aligned classes)
  int n_chunks;             // ceil(nb^2 / kOrtChunk)
  int parts, chunks_per_part;  // entry chunks of a tile split over `parts` CTAs
  double *elem, *cell_rhs;
  int *err;
};

// Geometry of cell c: det J and J^-1 (zero / identity for a degenerate
// cell, which is flagged), and the twelve contraction weights
// (c/det) (J^T J)_ab and m det (J^-1 J^-T)_ab, or their tangents along
// (verts_dot, ca_dot, cb_dot), or the caller's weights.
__device__ __forceinline__ void ort_geometry(const OrtArgs &A, int c, bool weights, double *w, double *Ji,
                             double &det_out) {
  double J[9], v0[3];
  tet_jacobian(A.cells, A.verts, c, J, v0);
  const double det = det3(J);
  const bool ok = valid_jacobian(J, det);
  if (!ok) atomicCAS(A.err, 0, FFG_INVALID_INPUT);
  inv3(J, ok ? det : 1.0, Ji);
  det_out = ok ? det : 0.0;
  if (!weights) return;
  const double cw = A.ca * (A.cell_a ? A.cell_a[c] : 1.0);
  const double mw = A.cb * (A.cell_b ? A.cell_b[c] : 1.0);
  // symmetric index pairs (a, b) of the six weights of each kind
  constexpr int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  if (A.geo_in) {
#pragma unroll
    for (int s = 0; s < 12; ++s) w[s] = ok ? A.geo_in[12 * (size_t)c + s] : 0.0;
  } else if (!A.verts_dot) {
#pragma unroll
    for (int s = 0; s < 6; ++s) {
      const int a = pa[s], b = pb[s];
      const double JtJ = J[3 * a] * J[3 * b] + J[3 * a + 1] * J[3 * b + 1] + J[3 * a + 2] * J[3 * b + 2];
      const double G = Ji[a] * Ji[b] + Ji[a + 3] * Ji[b + 3] + Ji[a + 6] * Ji[b + 6];
      w[s] = ok ? cw / det * JtJ : 0.0;
      w[6 + s] = ok ? mw * det * G : 0.0;
    }
  } else {
    // d(c/det J^T J) and d(m det J^-1 J^-T), with d det = det tr(J^-1 dJ)
    // and d J^-1 = -J^-1 dJ J^-1
    double Jd[9], T[9], Jid[9], w0[3];
    tet_jacobian(A.cells, A.verts_dot, c, Jd, w0);
#pragma unroll
    for (int col = 0; col < 3; ++col)
#pragma unroll
      for (int r = 0; r < 3; ++r)
        T[r + 3 * col] = Ji[r] * Jd[3 * col] + Ji[r + 3] * Jd[3 * col + 1] + Ji[r + 6] * Jd[3 * col + 2];
#pragma unroll
    for (int col = 0; col < 3; ++col)
#pragma unroll
      for (int r = 0; r < 3; ++r)
        Jid[r + 3 * col] = -(T[r] * Ji[3 * col] + T[r + 3] * Ji[3 * col + 1] + T[r + 6] * Ji[3 * col + 2]);
    const double dd = det * (T[0] + T[4] + T[8]);
    const double cwd = A.ca_dot * (A.cell_a ? A.cell_a[c] : 1.0);
    const double mwd = A.cb_dot * (A.cell_b ? A.cell_b[c] : 1.0);
#pragma unroll
    for (int s = 0; s < 6; ++s) {
      const int a = pa[s], b = pb[s];
      double JtJ = 0.0, dJtJ = 0.0, G = 0.0, dG = 0.0;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        JtJ += J[3 * a + r] * J[3 * b + r];
        dJtJ += Jd[3 * a + r] * J[3 * b + r] + J[3 * a + r] * Jd[3 * b + r];
        G += Ji[a + 3 * r] * Ji[b + 3 * r];
        dG += Jid[a + 3 * r] * Ji[b + 3 * r] + Ji[a + 3 * r] * Jid[b + 3 * r];
      }
      w[s] = ok ? cwd / det * JtJ - cw * dd / (det * det) * JtJ + cw / det * dJtJ : 0.0;
      w[6 + s] = ok ? mwd * det * G + mw * dd * G + mw * det * dG : 0.0;
    }
  }
}

// Element matrices of one tile: K[cell][i + nb l] = sum_s w_s R'_{s,class}[i + nb l].
// CTA (tile, part) runs the part's 128-entry chunks.  Warp w owns cells
// 8w .. 8w+7 of the tile, lane L entries L, L+32, L+64, L+96 of a chunk, so a
// store instruction writes 256 contiguous bytes of one cell's matrix.  The
// chunk's twelve table rows (12 KB, contiguous in the chunk-major table) are
// staged in shared memory, double-buffered: every thread holds its six
// values of the next chunk in registers while the current one is consumed.
constexpr int kOrtStage = 12 * kOrtChunk / kOrtThreads;  // table values per thread and chunk

__global__ void __launch_bounds__(kOrtThreads, 2) ort_matrix_kernel(const __grid_constant__ OrtArgs A) {
  __shared__ __align__(16) double W[12][kOrtTileCells];
  __shared__ __align__(16) double Rs[2][12 * kOrtChunk];
  __shared__ int cell_s[kOrtTileCells];
  const int4 tile = A.tiles[blockIdx.x / A.parts];
  const int part = blockIdx.x % A.parts;
  const int c0 = part * A.chunks_per_part, c1 = min(A.n_chunks, c0 + A.chunks_per_part);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (c0 >= c1) return;
  if (tid < kOrtTileCells) {
    double w[12], Ji[9], det;
    int c = -1;
    if (tid < tile.z) {
      c = A.order[tile.y + tid];
      ort_geometry(A, c, true, w, Ji, det);
    } else {
#pragma unroll
      for (int s = 0; s < 12; ++s) w[s] = 0.0;
    }
#pragma unroll
    for (int s = 0; s < 12; ++s) W[s][tid] = w[s];
    cell_s[tid] = c;
  }
  const int64_t nn = (int64_t)A.nb * A.nb;
  const double *R = A.ref + (size_t)tile.x * A.n_chunks * (12 * kOrtChunk);
  double pr[kOrtStage];
#pragma unroll
  for (int u = 0; u < kOrtStage; ++u)
    pr[u] = __ldg(R + (size_t)c0 * (12 * kOrtChunk) + tid + kOrtThreads * u);
  for (int ch = c0; ch < c1; ++ch) {
    double *buf = Rs[(ch - c0) & 1];
#pragma unroll
    for (int u = 0; u < kOrtStage; ++u) buf[tid + kOrtThreads * u] = pr[u];
    __syncthreads();  // this chunk staged (and, first time, the weights); the
                      // buffer written next was last read two chunks ago
    if (ch + 1 < c1) {
#pragma unroll
      for (int u = 0; u < kOrtStage; ++u)
        pr[u] = __ldg(R + (size_t)(ch + 1) * (12 * kOrtChunk) + tid + kOrtThreads * u);
    }
    double acc[8][4];
#pragma unroll
    for (int c = 0; c < 8; ++c)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[c][j] = 0.0;
#pragma unroll
    for (int s = 0; s < 12; ++s) {
      double r[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) r[j] = buf[s * kOrtChunk + lane + 32 * j];
      const double2 *w2p = reinterpret_cast<const double2 *>(&W[s][8 * warp]);
#pragma unroll
      for (int c2 = 0; c2 < 4; ++c2) {
        const double2 w2 = w2p[c2];  // the weights of two cells in one broadcast load
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[2 * c2][j] = fma(w2.x, r[j], acc[2 * c2][j]);
          acc[2 * c2 + 1][j] = fma(w2.y, r[j], acc[2 * c2 + 1][j]);
        }
      }
    }
    const int64_t base = (int64_t)ch * kOrtChunk;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int cell = cell_s[8 * warp + c];
      if (cell < 0) continue;
      double *out = A.elem + (size_t)cell * nn;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t idx = base + lane + 32 * j;
        if (idx < nn) out[idx] = acc[c][j];
      }
    }
  }
}

// Element loads of one tile: F[cell][i] = sum_{q,a} (det J^-1 f_q)_a L'_{class}[3q + a][i],
// a (64 cells) x (3 n_q) by (3 n_q) x (n_b) product per tile on the FP64
// tensor cores (mma.sync m8n8k4: warp w takes cells 8w .. 8w+7, NT tiles of 8
// entries per pass, 4 table rows per step), with Q points at a time: their
// 3 Q table rows (one contiguous block) come into shared memory by cp.async,
// double-buffered, and their sample factors det J^-1 f_q of the 64 cells are
// staged beside them; each thread fetches its samples of the next points
// into registers while the current ones are consumed.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait1() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

constexpr int kOrtLfPitch = kOrtTileCells + 2;  // even: 16-byte aligned rows of LF

template <int Q>
struct OrtLoadSmem {
  double Ji[9][kOrtTileCells];
  double det[kOrtTileCells];
  alignas(16) double LF[3 * Q][kOrtLfPitch];
  int cell[kOrtTileCells];
};

// D (8 x 8) += A (8 x 4) B (4 x 8) in FP64 on the tensor cores: lane L holds
// A[L / 4][L % 4], B[L % 4][L / 4] and D[L / 4][2 (L % 4) + {0, 1}].
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int NT, int Q>
__global__ void __launch_bounds__(kOrtThreads, 2) ort_load_kernel(const __grid_constant__ OrtArgs A) {
  extern __shared__ __align__(16) unsigned char ort_raw[];
  OrtLoadSmem<Q> &S = *reinterpret_cast<OrtLoadSmem<Q> *>(ort_raw);
  const int nb = A.nb, nql = A.nql;
  // two buffers of 3 Q table rows (an even count of doubles each)
  const int rows_cap = (3 * Q * nb + 1) & ~1;
  double *Lb = reinterpret_cast<double *>(ort_raw + sizeof(OrtLoadSmem<Q>));
  constexpr int kPairs = kOrtTileCells * Q / kOrtThreads;  // (cell, point) pairs per thread
  const int4 tile = A.tiles[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid < kOrtTileCells) {
    double Ji[9], det = 0.0;
    int c = -1;
    if (tid < tile.z) {
      c = A.order[tile.y + tid];
      ort_geometry(A, c, false, nullptr, Ji, det);
    } else {
#pragma unroll
      for (int i = 0; i < 9; ++i) Ji[i] = 0.0;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) S.Ji[i][tid] = Ji[i];
    S.det[tid] = det;
    S.cell[tid] = c;
  }
  __syncthreads();
  const double *L = A.load + (size_t)tile.x * A.load_stride;
  const int n_chunks = (nql + Q - 1) / Q;
  // the table rows of point chunk ci into buffer ci & 1 (16-byte pieces; the
  // table is padded so that a trailing odd double may be read)
  auto stage = [&](int ci) {
    if (ci < n_chunks) {
      const int q0 = ci * Q, nq = min(Q, nql - q0);
      const int pieces = (3 * nq * nb + 1) / 2;
      const double *src = L + (size_t)3 * q0 * nb;
      double *dst = Lb + (size_t)(ci & 1) * rows_cap;
      for (int i = tid; i < pieces; i += kOrtThreads) cp_async16(dst + 2 * i, src + 2 * i);
    }
    cp_async_commit();
  };
  double f[kPairs][3];
  // pair u of this thread: cell (tid + 256 u) / Q, point (tid + 256 u) % Q
  auto fetch = [&](int q0) {
#pragma unroll
    for (int u = 0; u < kPairs; ++u) {
      const int p = tid + kOrtThreads * u, c = p / Q, q = q0 + p % Q;
      const bool live = c < tile.z && q < nql;
      const double *sp = A.samples + 3 * ((size_t)nql * (live ? S.cell[c] : 0) + (live ? q : 0));
#pragma unroll
      for (int a = 0; a < 3; ++a) f[u][a] = live ? sp[a] : 0.0;
    }
  };
  // warp w: cells 8w .. 8w+7 (M), NT tiles of 8 entries (N) per pass, 4 table
  // rows (K) per step
  const int kr = lane & 3, cc = lane >> 2;
  for (int base = 0; base < nb; base += 8 * NT) {
    double acc[NT][2];
#pragma unroll
    for (int t = 0; t < NT; ++t) acc[t][0] = acc[t][1] = 0.0;
    __syncthreads();  // the previous pass has consumed both buffers
    stage(0);
    fetch(0);
    for (int ci = 0; ci < n_chunks; ++ci) {
      const int q0 = ci * Q, nq = min(Q, nql - q0);
      __syncthreads();  // chunk ci - 1 consumed: its buffer and LF may be rewritten
      stage(ci + 1);
#pragma unroll
      for (int u = 0; u < kPairs; ++u) {
        const int p = tid + kOrtThreads * u, c = p / Q, q = p % Q;
        const double d = S.det[c];
#pragma unroll
        for (int a = 0; a < 3; ++a)
          S.LF[3 * q + a][c] =
              d * (S.Ji[a][c] * f[u][0] + S.Ji[a + 3][c] * f[u][1] + S.Ji[a + 6][c] * f[u][2]);
      }
      cp_async_wait1();  // this thread's pieces of chunk ci have landed
      __syncthreads();   // everyone's pieces and factors are visible
      if (ci + 1 < n_chunks) fetch(q0 + Q);
      const double *rows = Lb + (size_t)(ci & 1) * rows_cap;
      const int nk = 3 * nq;
      for (int k0 = 0; k0 < nk; k0 += 4) {
        const int qa = k0 + kr;
        const bool kin = qa < nk;
        const double av = kin ? S.LF[qa][8 * warp + cc] : 0.0;
        const double *row = rows + (size_t)(kin ? qa : 0) * nb;
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          const int i = base + 8 * t + cc;
          const double bv = (kin && i < nb) ? row[i] : 0.0;
          dmma_8x8x4(acc[t][0], acc[t][1], av, bv);
        }
      }
    }
    const int cell = S.cell[8 * warp + cc];
    if (cell >= 0) {
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int i = base + 8 * t + 2 * kr;
        if (i < nb) A.cell_rhs[(size_t)nb * cell + i] = acc[t][0];
        if (i + 1 < nb) A.cell_rhs[(size_t)nb * cell + i + 1] = acc[t][1];
      }
    }
  }
  cp_async_wait_all();
}

// Entry tiles of 8 per pass of the load kernel: the fewest passes of at
// most 12 tiles, tiles spread evenly over them.
int load_tiles(int nb) {
  const int tiles = (nb + 7) / 8, passes = (tiles + 11) / 12;
  return (tiles + passes - 1) / passes;
}

// Ranks of the four vertices of class `cls` (inverse of class_of).
void class_ranks(int cls, int r[4]) {
  int avail[4] = {0, 1, 2, 3}, n = 4;
  const int digit[3] = {cls / 6, (cls / 2) % 3, cls % 2};
  for (int i = 0; i < 3; ++i) {
    r[i] = avail[digit[i]];
    for (int j = digit[i]; j + 1 < n; ++j) avail[j] = avail[j + 1];
    --n;
  }
  r[3] = avail[0];
}

// Column d of T: nonzeros T[start + m][d] = col[m] (a face block column) or
// the diagonal entry diag.
struct TCol {
  int start, size;
  const double *col;
  double diag;
};

TCol tcol(int k, int nb, const int8_t *sg, const uint8_t *fp, const double *face_blocks, int d) {
  const int fdc = k * (k - 1), edge_end = 6 * k, face_end = edge_end + 4 * fdc;
  (void)nb;
  if (d < edge_end) {
    const int e = d / k, m = d % k;
    return {d, 1, nullptr, (sg[e] == -1 && m % 2 == 0) ? -1.0 : 1.0};
  }
  if (d < face_end) {
    const int f = (d - edge_end) / fdc, r = (d - edge_end) % fdc;
    const int st = edge_end + f * fdc;
    return {st, fdc, face_blocks + (size_t)fp[f] * fdc * fdc + (size_t)fdc * r, 0.0};
  }
  return {d, 1, nullptr, 1.0};
}

}  // namespace

int ort_class(const int *v) {
  const int c0 = (v[1] < v[0]) + (v[2] < v[0]) + (v[3] < v[0]);
  const int c1 = (v[2] < v[1]) + (v[3] < v[1]);
  const int c2 = v[3] < v[2];
  return 6 * c0 + 2 * c1 + c2;
}

void ort_free(OrientedTables &o) {
  void *p[] = {o.ref, o.load, o.order_cells, o.tiles};
  for (void *q : p)
    if (q) cudaFree(q);
  o = OrientedTables();
}

int ort_build(const Topology &t, const ElementTables &tab, OrientedTables &o) {
  if (t.family != FFG_TETRA_NEDELEC || tab.n_terms != 12) return FFG_INVALID_INPUT;
  const int k = t.degree, nb = t.nb, nql = tab.nq_load;
  const size_t nn = (size_t)nb * nb;
  // classes and the stable class order of the cells
  std::vector<int> cls(t.n_cells), start(kOrtClasses + 1, 0), order(t.n_cells);
  int count[kOrtClasses] = {};
  for (int c = 0; c < t.n_cells; ++c) {
    cls[c] = ort_class(t.cells.data() + 4 * (size_t)c);
    ++count[cls[c]];
  }
  for (int q = 0; q < kOrtClasses; ++q) start[q + 1] = start[q] + count[q];
  {
    std::vector<int> at(start.begin(), start.end() - 1);
    for (int c = 0; c < t.n_cells; ++c) order[at[cls[c]]++] = c;
  }
  std::vector<int4> tiles;
  for (int q = 0; q < kOrtClasses; ++q)
    for (int f = 0; f < count[q]; f += kOrtTileCells)
      tiles.push_back(make_int4(q, start[q] + f, std::min(kOrtTileCells, count[q] - f), 0));
  // tables of the classes present
  // R' chunk-major: class, 128-entry chunk, term, entry of the chunk (zero
  // past nb^2), so that a chunk's twelve rows are one contiguous block
  const int n_chunks = (int)((nn + kOrtChunk - 1) / kOrtChunk);
  const size_t class_stride = (size_t)n_chunks * 12 * kOrtChunk;
  std::vector<double> ref((size_t)kOrtClasses * class_stride, 0.0);
  std::vector<double> Out(nn);
  const size_t load_stride = ((size_t)3 * nql * nb + 1) & ~(size_t)1;
  std::vector<double> load((size_t)kOrtClasses * load_stride, 0.0);
  std::vector<double> X(nn);
  std::vector<TCol> T(nb);
  for (int q = 0; q < kOrtClasses; ++q) {
    if (!count[q]) continue;
    int r[4];
    int8_t sg[6];
    uint8_t fp[4];
    class_ranks(q, r);
    nedelec_orientation(r, sg, fp);
    for (int d = 0; d < nb; ++d) T[d] = tcol(k, nb, sg, fp, tab.face_blocks.data(), d);
    for (int s = 0; s < 12; ++s) {
      const double *Rs = &tab.ref[(size_t)s * nn];
      // X = R_s T (column d of X from the nonzeros of column d of T)
      for (int d = 0; d < nb; ++d)
        for (int i = 0; i < nb; ++i) {
          double acc = 0.0;
          for (int m = 0; m < T[d].size; ++m)
            acc += Rs[i + (size_t)nb * (T[d].start + m)] * (T[d].col ? T[d].col[m] : T[d].diag);
          X[i + (size_t)nb * d] = acc;
        }
      // R' = T^T X
      for (int d = 0; d < nb; ++d)
        for (int j = 0; j < nb; ++j) {
          double acc = 0.0;
          for (int m = 0; m < T[d].size; ++m)
            acc += (T[d].col ? T[d].col[m] : T[d].diag) * X[(T[d].start + m) + (size_t)nb * j];
          Out[d + (size_t)nb * j] = acc;
        }
      for (size_t idx = 0; idx < nn; ++idx)
        ref[(size_t)q * class_stride + ((idx / kOrtChunk) * 12 + s) * kOrtChunk + idx % kOrtChunk] =
            Out[idx];
    }
    // L'[3p + a][i] = sum_m T[m][i] (w_p v_a(p))_m, load_basis ((p nb + m) 3 + a)
    double *Lq = &load[(size_t)q * load_stride];
    for (int p = 0; p < nql; ++p)
      for (int a = 0; a < 3; ++a)
        for (int i = 0; i < nb; ++i) {
          double acc = 0.0;
          for (int m = 0; m < T[i].size; ++m)
            acc += (T[i].col ? T[i].col[m] : T[i].diag) *
                   tab.load_basis[((size_t)p * nb + T[i].start + m) * 3 + a];
          Lq[(size_t)(3 * p + a) * nb + i] = acc;
        }
  }
  ort_free(o);
  auto up = [](auto **dst, const auto &v) -> int {
    using E = typename std::remove_reference<decltype(v[0])>::type;
    if (cudaMalloc((void **)dst, sizeof(E) * std::max<size_t>(v.size(), 1)) != cudaSuccess)
      return FFG_OUT_OF_MEMORY;
    if (!v.empty() &&
        cudaMemcpy(*dst, v.data(), sizeof(E) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return FFG_CUDA_ERROR;
    return FFG_OK;
  };
  int st;
  if ((st = up(&o.ref, ref)) || (st = up(&o.load, load)) || (st = up(&o.order_cells, order)) ||
      (st = up(&o.tiles, tiles))) {
    ort_free(o);
    return st;
  }
  o.order = k;
  o.nb = nb;
  o.nql = nql;
  o.n_chunks = n_chunks;
  o.load_stride = (int64_t)load_stride;
  o.n_tiles = (int)tiles.size();
  std::memcpy(o.class_count, count, sizeof(count));
  return FFG_OK;
}

// Oriented element matrices (unless load_only) and loads of every cell.
int launch_nedelec_oriented(const Topology &t, const OrientedTables &o, const DeviceTopology &dt,
                            const AssemblyInputs &in, double *elem, double *cell_rhs, int *err,
                            cudaStream_t s, bool load_only) {
  if (o.order != t.degree || o.nb != t.nb || !o.tiles) return FFG_INVALID_INPUT;
  if (o.n_tiles == 0) return FFG_OK;
  OrtArgs A;
  A.nb = o.nb;
  A.nql = o.nql;
  A.cells = dt.cells;
  A.verts = in.vertices;
  A.ca = in.coef_a;
  A.cb = in.coef_b;
  A.cell_a = in.cell_a;
  A.cell_b = in.cell_b;
  A.geo_in = in.geo_override;
  A.verts_dot = in.vertices_dot;
  A.ca_dot = in.coef_a_dot;
  A.cb_dot = in.coef_b_dot;
  A.samples = in.samples;
  A.order = o.order_cells;
  A.tiles = o.tiles;
  A.ref = o.ref;
  A.load = o.load;
  A.load_stride = o.load_stride;
  A.elem = elem;
  A.cell_rhs = cell_rhs;
  A.err = err;
  // enough CTAs for per_sm per SM (default 8): the entry chunks of a tile split over parts
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  A.n_chunks = o.n_chunks;
  const int per_sm = (in.tune && in.tune->ned_ctas_per_sm) ? in.tune->ned_ctas_per_sm : 8;
  A.parts = std::max(1, std::min(o.n_chunks, (per_sm * sms + o.n_tiles - 1) / o.n_tiles));
  A.chunks_per_part = (o.n_chunks + A.parts - 1) / A.parts;
  A.parts = (o.n_chunks + A.chunks_per_part - 1) / A.chunks_per_part;
  if (!load_only)
    ort_matrix_kernel<<<(unsigned)((int64_t)o.n_tiles * A.parts), kOrtThreads, 0, s>>>(A);
  if (in.samples) {
    auto go = [&](auto kern, int Q, size_t fixed) -> int {
      const size_t smem = fixed + 2 * sizeof(double) * (((size_t)3 * Q * o.nb + 1) & ~(size_t)1);
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
        return FFG_CUDA_ERROR;
      kern<<<o.n_tiles, kOrtThreads, smem, s>>>(A);
      return FFG_OK;
    };
    // Q = 16 points per stage up to order 4, 8 above (shared memory)
    const bool wide = o.nb > 84;
    const size_t f16 = sizeof(OrtLoadSmem<16>), f8 = sizeof(OrtLoadSmem<8>);
    int st;
    switch (load_tiles(o.nb)) {
      case 1: st = go(ort_load_kernel<1, 16>, 16, f16); break;
      case 3: st = go(ort_load_kernel<3, 16>, 16, f16); break;
      case 6: st = go(ort_load_kernel<6, 16>, 16, f16); break;
      case 7: st = wide ? go(ort_load_kernel<7, 8>, 8, f8) : go(ort_load_kernel<7, 16>, 16, f16); break;
      case 11: st = wide ? go(ort_load_kernel<11, 8>, 8, f8) : go(ort_load_kernel<11, 16>, 16, f16); break;
      default: st = wide ? go(ort_load_kernel<12, 8>, 8, f8) : go(ort_load_kernel<12, 16>, 16, f16); break;
    }
    if (st) return st;
  } else if (cudaMemsetAsync(cell_rhs, 0, sizeof(double) * t.nb * (size_t)t.n_cells, s) !=
             cudaSuccess) {
    return FFG_CUDA_ERROR;
  }
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace ffg
