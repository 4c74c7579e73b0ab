// 3xTF32 tensor-core contraction of the first-kind Nedelec curl + mass
// element matrices (orders 3 and 4), the tcgen05 path beside the FP64
// CUDA-core element kernel.
//
// The reference evaluates every element matrix by a quadrature loop
// (assemble_tetra_nedelec_curl_mass_element, src/assembly/assembly_tetra_nedelec_3d.f90:584-643,
// the double loop :632-640).  For affine cells the same matrix is the
// reference-tensor sum K~ = sum_t w_t R_t over twelve weights per cell
// (curl: (c/det) (J^T J)_ab, mass: m det (J^-1 J^-T)_ab), i.e. a GEMM
//     D[cell, entry] = W[cell, 0..11] . R[0..11, entry]
// with M = 128 cells per CTA (one TMEM lane per cell), N = element entries in
// tiles of at most 256 and K = 12 padded to 16.  Operands are split into
// TF32 hi/lo parts and three products (hi.hi + hi.lo + lo.hi) accumulate in
// FP32 in tensor memory (3xTF32), so the contraction keeps about 22 bits.
//
// The orientation transform T^T K~ T (assemble_arbitrary_order_curl_mass_csc,
// :2340-2342) is block diagonal: signs on the edge moments, one of six dense
// k(k-1) x k(k-1) blocks per face, identity on the cell moments.  The N
// dimension is therefore ordered by block pairs (I, J) and every block pair
// lies in one tile, so each epilogue thread (one cell) loads its K~[I, J] from
// tensor memory, forms T_I^T K~[I, J] T_J in registers (FP32) and writes the
// oriented block into the cell's element matrix (FP32, column-major with a
// leading dimension padded to a multiple of 4).
//
// Operand layout (shared memory, K-major, no swizzle): for R rows x 16 K
// values, the 16-byte chunk holding K values 4c..4c+3 of row r sits at
// byte c * R * 16 + r * 16, so eight rows form one 8 x 16-byte core matrix,
// core matrices of consecutive row groups are 128 bytes apart (stride byte
// offset) and the two chunks of one K = 8 step are R * 16 bytes apart
// (leading byte offset).  The B operand of every tile is prepared on the host
// in exactly this image (hi then lo) and brought in with one bulk copy
// (cp.async.bulk, no multicast), double-buffered against the epilogue.
//
// Every wait on an mbarrier is bounded (globaltimer); on expiry the kernel
// flags FFG_TIMEOUT, waits (bounded) for its own copies in flight, frees its
// tensor memory and returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "ffg_internal.h"
#include "tet_geometry.h"

namespace ffg {

namespace {

constexpr int kTcThreads = 128;  // one warpgroup: one thread (TMEM lane) per cell
constexpr int kTcCols = 256;     // tensor-memory columns of a CTA (one tile)
constexpr int kTcAlign = 16;     // TMEM column alignment of a block pair
constexpr unsigned long long kTcWaitNs = 2000000000ull;  // 2 s per wait

// block kinds of the orientation transform
constexpr int kEdge = 0, kFace = 1, kCell = 2;

__device__ __forceinline__ unsigned long long tc_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait for the phase with parity `parity` of `bar`.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  unsigned long long t0 = 0;
  for (uint32_t spin = 0;; ++spin) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((spin & 255u) == 0) {
      const unsigned long long t = tc_now();
      if (t0 == 0) t0 = t;
      else if (t - t0 > kTcWaitNs) return false;
    }
  }
}

// One untiled bulk copy global -> shared, completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major, no swizzle, version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: kind::tf32, A and B TF32 K-major, D FP32, M = 128.
__device__ __forceinline__ uint32_t tf32_idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

struct TcArgs {
  int n_cells;
  const int *cells;
  const double *verts;
  double ca, cb;
  const double *cell_a, *cell_b;
  const double *geo_in;  // caller weights (12 per cell) or null
  const int8_t *edge_sign;
  const uint8_t *face_perm;
  // plan
  int n_tiles;
  const int *tile_n;       // N of tile t (multiple of 16, <= 256)
  const int *tile_pair0;   // first pair of tile t; pairs of tile t: [pair0[t], pair0[t+1])
  const int *pair_code;    // (bi << 24) | (bj << 16) | tmem column
  const float *bimage;     // B operand images, tile t at bimage + 64 * boff[t]
  const int *boff;         // in units of 64 floats
  const float *face_t;     // 6 x fdc x fdc, column-major T_f per permutation
  float *elem;             // n_cells x nb x ld, column-major, leading dimension ld
  int ld;
  int *err;
};

template <int K>
struct Dims {
  static constexpr int fdc = K * (K - 1), nint = K * (K - 1) * (K - 2) / 2;
  static constexpr int edge_end = 6 * K, face_end = 6 * K + 4 * fdc, nb = face_end + nint;
  __device__ static constexpr int size(int b) { return b < 6 ? K : (b < 10 ? fdc : nint); }
  __device__ static constexpr int start(int b) {
    return b < 6 ? b * K : (b < 10 ? edge_end + (b - 6) * fdc : face_end);
  }
};

// T_I^T X T_J for one block pair of one cell.  X (NI x NJ, column-major) is
// read from tensor memory at column `col` of this warp's lanes; a dense block
// (faces) comes from the face table in shared memory, a diagonal one (edges:
// the reference's sign on even-indexed moments of reversed edges; cells: 1)
// from `dI` / `dJ`.
template <int NI, int NJ, bool DENSE_I, bool DENSE_J>
__device__ __forceinline__ void tc_pair(uint32_t taddr, const float *TI, const float *TJ,
                                        const float *dI, const float *dJ, float *out, int ld,
                                        bool store) {
  constexpr int NX = NI * NJ, NL = (NX + 15) / 16;
  float X[NL * 16];
#pragma unroll
  for (int c = 0; c < NL; ++c) tmem_ld16(taddr + 16 * c, X + 16 * c);
  tmem_wait_ld();
  // one output column at a time (not unrolled, so the T_I entries are read
  // per column instead of being held in registers beside X)
#pragma unroll 1
  for (int b = 0; b < NJ; ++b) {
    float z[NI];
#pragma unroll
    for (int a = 0; a < NI; ++a) {
      if (DENSE_J) {
        float s = 0.f;
#pragma unroll
        for (int m = 0; m < NJ; ++m) s = fmaf(X[a + NI * m], TJ[b * NJ + m], s);
        z[a] = s;
      } else {
        z[a] = X[a + NI * b] * dJ[b];
      }
    }
    float y[NI];
#pragma unroll
    for (int a2 = 0; a2 < NI; ++a2) {
      if (DENSE_I) {
        float s = 0.f;
#pragma unroll
        for (int a = 0; a < NI; ++a) s = fmaf(TI[a2 * NI + a], z[a], s);
        y[a2] = s;
      } else {
        y[a2] = dI[a2] * z[a2];
      }
    }
    if (store) {
      float *o = out + (size_t)ld * b;
#pragma unroll
      for (int a2 = 0; a2 < NI; ++a2) o[a2] = y[a2];
    }
  }
}

template <int K>
__device__ __forceinline__ void tc_epilogue_pair(int code, uint32_t tbase, const float *face_t,
                                                 const float (&esign)[6][K], const int *fp,
                                                 const float *ones, float *cell_out, int ld,
                                                 bool store) {
  using D = Dims<K>;
  const int bi = (code >> 24) & 0xFF, bj = (code >> 16) & 0xFF, col = code & 0xFFFF;
  const uint32_t taddr = tbase + (uint32_t)col;
  const int ki = bi < 6 ? kEdge : (bi < 10 ? kFace : kCell);
  const int kj = bj < 6 ? kEdge : (bj < 10 ? kFace : kCell);
  constexpr int F2 = D::fdc * D::fdc;
  const float *TI = ki == kFace ? face_t + fp[bi - 6] * F2 : nullptr;
  const float *TJ = kj == kFace ? face_t + fp[bj - 6] * F2 : nullptr;
  const float *dI = ki == kEdge ? esign[bi] : ones;
  const float *dJ = kj == kEdge ? esign[bj] : ones;
  float *out = cell_out + (size_t)ld * D::start(bj) + D::start(bi);
  constexpr int E = K, FD = D::fdc, C = D::nint;
  // the nine combinations of edge / face / cell blocks
  if (ki == kEdge && kj == kEdge) tc_pair<E, E, false, false>(taddr, TI, TJ, dI, dJ, out, ld, store);
  else if (ki == kEdge && kj == kFace) tc_pair<E, FD, false, true>(taddr, TI, TJ, dI, dJ, out, ld, store);
  else if (ki == kEdge && kj == kCell) tc_pair<E, C, false, false>(taddr, TI, TJ, dI, dJ, out, ld, store);
  else if (ki == kFace && kj == kEdge) tc_pair<FD, E, true, false>(taddr, TI, TJ, dI, dJ, out, ld, store);
  else if (ki == kFace && kj == kFace) tc_pair<FD, FD, true, true>(taddr, TI, TJ, dI, dJ, out, ld, store);
  else if (ki == kFace && kj == kCell) tc_pair<FD, C, true, false>(taddr, TI, TJ, dI, dJ, out, ld, store);
  else if (ki == kCell && kj == kEdge) tc_pair<C, E, false, false>(taddr, TI, TJ, dI, dJ, out, ld, store);
  else if (ki == kCell && kj == kFace) tc_pair<C, FD, false, true>(taddr, TI, TJ, dI, dJ, out, ld, store);
  else tc_pair<C, C, false, false>(taddr, TI, TJ, dI, dJ, out, ld, store);
}

constexpr int kAHalf = kTcThreads * 16 * 4;  // bytes of one A part (128 rows x 16 TF32)
constexpr int kBHalfMax = kTcCols * 16 * 4;  // bytes of one B part at N = 256

struct TcSmem {
  alignas(1024) unsigned char a[2 * kAHalf];         // A hi, A lo
  alignas(1024) unsigned char b[2][2 * kBHalfMax];   // two buffers of B hi + lo
  float face_t[6 * 144];
  uint64_t bbar[2];
  uint64_t mbar;
  uint32_t tmem;
  int abort;
};

template <int K>
__global__ void __launch_bounds__(kTcThreads, 2) nedelec_tc_kernel(TcArgs A) {
  using D = Dims<K>;
  extern __shared__ unsigned char tc_raw[];
  TcSmem &S = *reinterpret_cast<TcSmem *>(
      (unsigned char *)(((uintptr_t)tc_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5;
  constexpr int F2 = D::fdc * D::fdc;
  for (int i = tid; i < 6 * F2; i += kTcThreads) S.face_t[i] = A.face_t[i];
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&S.tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&S.bbar[0], 1);
    mbar_init(&S.bbar[1], 1);
    mbar_init(&S.mbar, 1);
    S.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem;
  const uint32_t tlane = tmem + ((uint32_t)(32 * warp) << 16);
  const float ones[12] = {1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f};

  const int n_groups = (A.n_cells + kTcThreads - 1) / kTcThreads;
  const int my_groups = blockIdx.x < n_groups ? (n_groups - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int total = my_groups * A.n_tiles;  // tiles this CTA runs
  uint32_t copies_issued = 0, copies_done = 0;
  auto issue_copy = [&](int u) {
    const int t = u % A.n_tiles, buf = u & 1;
    const uint32_t bytes = 128u * (uint32_t)A.tile_n[t];
    mbar_expect_tx(&S.bbar[buf], bytes);
    bulk_load(S.b[buf], A.bimage + 64 * (size_t)A.boff[t], bytes, &S.bbar[buf]);
  };
  if (tid == 0) {
    for (int u = 0; u < 2 && u < total; ++u) { issue_copy(u); ++copies_issued; }
  }
  int u = 0;
  bool aborted = false;
  for (int gi = 0; gi < my_groups && !aborted; ++gi) {
    const int g = blockIdx.x + gi * gridDim.x;
    const int c = g * kTcThreads + tid;
    const bool live = c < A.n_cells;
    // ---- weights of this cell (FP64 geometry), split into TF32 hi / lo
    double w[12];
    float esign[6][K];
    int fp[4] = {0, 0, 0, 0};
#pragma unroll
    for (int s = 0; s < 12; ++s) w[s] = 0.0;
#pragma unroll
    for (int e = 0; e < 6; ++e)
#pragma unroll
      for (int m = 0; m < K; ++m) esign[e][m] = 1.f;
    if (live) {
      double J[9], Ji[9], v0[3];
      tet_jacobian(A.cells, A.verts, c, J, v0);
      const double det = det3(J);
      const bool ok = valid_jacobian(J, det);
      if (!ok) atomicCAS(A.err, 0, FFG_INVALID_INPUT);
      if (ok) {
        inv3(J, det, Ji);
        if (A.geo_in) {
#pragma unroll
          for (int s = 0; s < 12; ++s) w[s] = A.geo_in[12 * (size_t)c + s];
        } else {
          const double cw = A.ca * (A.cell_a ? A.cell_a[c] : 1.0);
          const double mw = A.cb * (A.cell_b ? A.cell_b[c] : 1.0);
          const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
          for (int s = 0; s < 6; ++s) {
            const int a = pa[s], b = pb[s];
            const double JtJ =
                J[3 * a] * J[3 * b] + J[3 * a + 1] * J[3 * b + 1] + J[3 * a + 2] * J[3 * b + 2];
            const double G = Ji[a] * Ji[b] + Ji[a + 3] * Ji[b + 3] + Ji[a + 6] * Ji[b + 6];
            w[s] = cw / det * JtJ;
            w[6 + s] = mw * det * G;
          }
        }
      }
      const int8_t *sg = A.edge_sign + 6 * (size_t)c;
#pragma unroll
      for (int e = 0; e < 6; ++e)
#pragma unroll
        for (int m = 0; m < K; ++m) esign[e][m] = (sg[e] == -1 && (m % 2) == 0) ? -1.f : 1.f;
#pragma unroll
      for (int f = 0; f < 4; ++f) fp[f] = A.face_perm[4 * (size_t)c + f];
    }
    float *ahi = reinterpret_cast<float *>(S.a);
    float *alo = reinterpret_cast<float *>(S.a + kAHalf);
#pragma unroll
    for (int s = 0; s < 16; ++s) {
      const double x = s < 12 ? w[s] : 0.0;
      const float hi = tf32_round((float)x);
      const float lo = tf32_round((float)(x - (double)hi));
      // chunk s/4, row tid, element s%4
      ahi[(s >> 2) * (kTcThreads * 4) + tid * 4 + (s & 3)] = hi;
      alo[(s >> 2) * (kTcThreads * 4) + tid * 4 + (s & 3)] = lo;
    }
    fence_proxy_async();
    __syncthreads();
    float *cell_out = A.elem + (size_t)(live ? c : 0) * A.ld * D::nb;
    for (int t = 0; t < A.n_tiles; ++t, ++u) {
      const int n = A.tile_n[t], buf = u & 1;
      if (tid == 0) {
        if (!mbar_wait(&S.bbar[buf], (uint32_t)((u >> 1) & 1))) {
          atomicCAS(A.err, 0, FFG_TIMEOUT);
          S.abort = 1;
        } else {
          ++copies_done;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a0 = smem_u32(S.a), b0 = smem_u32(S.b[buf]);
          const uint32_t bhalf = 64u * (uint32_t)n;
          const uint32_t idesc = tf32_idesc(n);
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {
            const uint64_t ah = smem_desc(a0 + ks * 2 * (kTcThreads * 16), kTcThreads * 16, 128);
            const uint64_t al =
                smem_desc(a0 + kAHalf + ks * 2 * (kTcThreads * 16), kTcThreads * 16, 128);
            const uint64_t bh = smem_desc(b0 + ks * 2 * (16u * n), 16u * n, 128);
            const uint64_t bl = smem_desc(b0 + bhalf + ks * 2 * (16u * n), 16u * n, 128);
            mma_tf32(tmem, ah, bh, idesc, ks > 0 ? 1u : 0u);
            mma_tf32(tmem, ah, bl, idesc, 1u);
            mma_tf32(tmem, al, bh, idesc, 1u);
          }
          mma_commit(&S.mbar);
        }
      }
      __syncthreads();
      if (S.abort) { aborted = true; break; }
      if (!mbar_wait(&S.mbar, (uint32_t)(u & 1))) {
        atomicCAS(A.err, 0, FFG_TIMEOUT);
        S.abort = 1;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      __syncthreads();
      if (S.abort) { aborted = true; break; }
      // the MMAs of tile u have read B buffer `buf`: refill it with tile u + 2
      if (tid == 0 && u + 2 < total) { issue_copy(u + 2); ++copies_issued; }
      for (int p = A.tile_pair0[t]; p < A.tile_pair0[t + 1]; ++p)
        tc_epilogue_pair<K>(A.pair_code[p], tlane, S.face_t, esign, fp, ones, cell_out, A.ld,
                            live);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
    }
  }
  // copies still in flight complete before the CTA leaves (bounded)
  if (tid == 0) {
    while (copies_done < copies_issued) {
      const int v = (int)copies_done;  // tile index of the oldest copy not yet waited for
      if (!mbar_wait(&S.bbar[v & 1], (uint32_t)((v >> 1) & 1))) {
        atomicCAS(A.err, 0, FFG_TIMEOUT);
        break;
      }
      ++copies_done;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcCols)
                 : "memory");
  }
}

inline uint32_t host_tf32(float x) {
  // round to nearest, ties away from zero, to 10 stored mantissa bits
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) return u;
  u += 0x1000u;
  return u & 0xFFFFE000u;
}

inline float host_tf32f(double x) {
  const uint32_t u = host_tf32((float)x);
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

}  // namespace

size_t tc_smem_bytes() { return sizeof(TcSmem) + 1024; }

bool tc_supported_order(int k) { return k == 3 || k == 4; }

// Tile plan and B images of one order (host): block pairs in J-major order,
// each padded to a multiple of 16 TMEM columns, packed into tiles of at most
// 256 columns; the B image of a tile is its rows of the reference tensors
// (12 terms + 4 zero terms) split into TF32 hi / lo in the shared-memory
// layout the MMA reads.
int tc_build_plan(int k, const ElementTables &tab, TcPlan &plan) {
  if (!tc_supported_order(k) || tab.n_terms != 12) return FFG_INVALID_INPUT;
  const int nb = tab.nb, fdc = k * (k - 1), nint = k * (k - 1) * (k - 2) / 2;
  auto bsize = [&](int b) { return b < 6 ? k : (b < 10 ? fdc : nint); };
  auto bstart = [&](int b) { return b < 6 ? b * k : (b < 10 ? 6 * k + (b - 6) * fdc : 6 * k + 4 * fdc); };
  std::vector<int> tile_n, tile_pair0, pair_code, boff;
  std::vector<float> image;
  std::vector<int> rows_i, rows_j;  // entry (i, j) of every row of the current tile
  int cur = 0;
  auto flush = [&]() {
    if (cur == 0) return;
    const int n = cur;
    boff.push_back((int)(image.size() / 64));
    std::vector<float> hi((size_t)n * 16, 0.f), lo((size_t)n * 16, 0.f);
    for (int r = 0; r < n; ++r) {
      if (rows_i[r] < 0) continue;
      const size_t off = (size_t)rows_i[r] + (size_t)nb * rows_j[r];
      for (int s = 0; s < 12; ++s) {
        const double x = tab.ref[(size_t)s * nb * nb + off];
        const float h = host_tf32f(x);
        const float l = host_tf32f(x - (double)h);
        const size_t pos = (size_t)(s >> 2) * n * 4 + (size_t)r * 4 + (s & 3);
        hi[pos] = h;
        lo[pos] = l;
      }
    }
    image.insert(image.end(), hi.begin(), hi.end());
    image.insert(image.end(), lo.begin(), lo.end());
    tile_n.push_back(n);
    rows_i.clear();
    rows_j.clear();
    cur = 0;
  };
  for (int bj = 0; bj < 11; ++bj) {
    if (bsize(bj) == 0) continue;
    for (int bi = 0; bi < 11; ++bi) {
      if (bsize(bi) == 0) continue;
      const int ne = bsize(bi) * bsize(bj);
      const int padded = (ne + kTcAlign - 1) / kTcAlign * kTcAlign;
      if (padded > kTcCols) return FFG_INVALID_INPUT;
      if (cur + padded > kTcCols) flush();
      if (cur == 0) tile_pair0.push_back((int)pair_code.size());
      pair_code.push_back((bi << 24) | (bj << 16) | cur);
      for (int q = 0; q < padded; ++q) {
        if (q < ne) {
          rows_i.push_back(bstart(bi) + q % bsize(bi));
          rows_j.push_back(bstart(bj) + q / bsize(bi));
        } else {
          rows_i.push_back(-1);
          rows_j.push_back(-1);
        }
      }
      cur += padded;
    }
  }
  flush();
  tile_pair0.push_back((int)pair_code.size());
  std::vector<float> ft((size_t)6 * fdc * fdc);
  for (size_t i = 0; i < ft.size(); ++i) ft[i] = (float)tab.face_blocks[i];
  plan.order = k;
  plan.n_tiles = (int)tile_n.size();
  plan.ld = (nb + 3) / 4 * 4;
  auto up = [](auto **dst, const auto &v) -> int {
    using T = typename std::remove_reference<decltype(v[0])>::type;
    if (cudaMalloc((void **)dst, sizeof(T) * std::max<size_t>(v.size(), 1)) != cudaSuccess)
      return FFG_OUT_OF_MEMORY;
    if (cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return FFG_CUDA_ERROR;
    return FFG_OK;
  };
  int st;
  if ((st = up(&plan.tile_n, tile_n)) || (st = up(&plan.tile_pair0, tile_pair0)) ||
      (st = up(&plan.pair_code, pair_code)) || (st = up(&plan.boff, boff)) ||
      (st = up(&plan.bimage, image)) || (st = up(&plan.face_t, ft)))
    return st;
  plan.image_bytes = image.size() * sizeof(float);
  return FFG_OK;
}

void tc_free_plan(TcPlan &plan) {
  void *p[] = {plan.tile_n, plan.tile_pair0, plan.pair_code, plan.boff, plan.bimage, plan.face_t};
  for (void *q : p)
    if (q) cudaFree(q);
  plan = TcPlan();
}

int launch_nedelec_tc(const Topology &t, const DeviceTopology &dt, const AssemblyInputs &in,
                      const TcPlan &plan, float *elem, int *err, cudaStream_t s) {
  if (t.family != FFG_TETRA_NEDELEC || plan.order != t.degree || !plan.tile_n) return FFG_INVALID_INPUT;
  if (t.n_cells == 0) return FFG_OK;
  TcArgs A;
  A.n_cells = (int)t.n_cells;
  A.cells = dt.cells;
  A.verts = in.vertices;
  A.ca = in.coef_a;
  A.cb = in.coef_b;
  A.cell_a = in.cell_a;
  A.cell_b = in.cell_b;
  A.geo_in = in.geo_override;
  A.edge_sign = dt.edge_sign;
  A.face_perm = dt.face_perm;
  A.n_tiles = plan.n_tiles;
  A.tile_n = plan.tile_n;
  A.tile_pair0 = plan.tile_pair0;
  A.pair_code = plan.pair_code;
  A.bimage = plan.bimage;
  A.boff = plan.boff;
  A.face_t = plan.face_t;
  A.elem = elem;
  A.ld = plan.ld;
  A.err = err;
  const size_t smem = tc_smem_bytes();
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int groups = (int)((t.n_cells + kTcThreads - 1) / kTcThreads);
  const int per_sm = (in.tune && in.tune->tc_ctas_per_sm) ? in.tune->tc_ctas_per_sm : 2;
  const int grid = std::min(groups, per_sm * sms);
  cudaError_t e;
  if (t.degree == 3) {
    e = cudaFuncSetAttribute(nedelec_tc_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e == cudaSuccess) nedelec_tc_kernel<3><<<grid, kTcThreads, smem, s>>>(A);
  } else {
    e = cudaFuncSetAttribute(nedelec_tc_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e == cudaSuccess) nedelec_tc_kernel<4><<<grid, kTcThreads, smem, s>>>(A);
  }
  if (e != cudaSuccess) return FFG_CUDA_ERROR;
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace ffg
