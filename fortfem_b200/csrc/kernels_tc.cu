// 3xTF32 tensor-core contraction of the first-kind Nedelec curl + mass
// element matrices (orders 3 to 6), the tcgen05 path beside the FP64
// CUDA-core kernels of kernels_oriented.cu.
//
// The reference evaluates every element matrix by a quadrature loop
// (assemble_tetra_nedelec_curl_mass_element, src/assembly/assembly_tetra_nedelec_3d.f90:584-643,
// the double loop :632-640) and orients it as T^T K T
// (assemble_arbitrary_order_curl_mass_csc, :2340-2342).  For affine cells the
// oriented matrix is sum_s w_s (T^T R_s T) over twelve weights per cell, with
// T fixed by the order of the cell's four global vertex indices (24 classes;
// the oriented tensors are tabulated per class in kernels_oriented.cu).  For
// 128 cells of one class that is a GEMM
//     D[cell, entry] = W[cell, 0..11] . R'_class[0..11, entry]
// with M = 128 cells per CTA (one TMEM lane per cell), N = 128 entries per
// tile (one chunk of the FP64 table) and K = 12 padded to 16.  Operands are
// split into TF32 hi/lo parts and three products (hi.hi + hi.lo + lo.hi)
// accumulate in FP32 in tensor memory (3xTF32, about 22 bits kept).
//
// Operand layout (shared memory, K-major, no swizzle): for R rows x 16 K
// values, the 16-byte chunk holding K values 4c..4c+3 of row r sits at
// byte c * R * 16 + r * 16, so eight rows form one 8 x 16-byte core matrix,
// core matrices of consecutive row groups are 128 bytes apart (stride byte
// offset) and the two chunks of one K = 8 step are R * 16 bytes apart
// (leading byte offset).  The B operand of every (class, tile) is cut on the
// device from the FP64 table in exactly this image (hi then lo, 16 KB) and
// brought in with one bulk copy (cp.async.bulk, no multicast),
// double-buffered.  Two TMEM accumulators of 128 columns let the MMAs of the
// next tile run while the epilogue drains the current one: each warp loads
// 32 columns of its 32 cells (tcgen05.ld.32x32b.x32), transposes them through
// shared memory and stores every cell's 32 entries as one 128-byte row of
// the FP32 element matrices.
//
// Every wait on an mbarrier is bounded (globaltimer); on expiry the kernel
// flags FFG_TIMEOUT, waits (bounded) for its own copies and MMAs in flight,
// frees its tensor memory and returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "ffg_internal.h"
#include "tet_geometry.h"

namespace ffg {

namespace {

constexpr int kTcThreads = 128;  // cells per CTA: one TMEM lane each (M)
constexpr int kTcBlock = 256;    // two warpgroups: both drain the accumulators
constexpr int kTcN = 128;        // element entries per tile (N), one FP64 table chunk
constexpr int kTcCols = 2 * kTcN;  // tensor-memory columns of a CTA: two accumulators
constexpr unsigned long long kTcWaitNs = 2000000000ull;  // 2 s per wait
static_assert(kTcN == 128, "a tile is one 128-entry chunk of the oriented FP64 table");

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

// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
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
  int nb, n_chunks;
  int64_t nn;       // entries of an element matrix (nb^2)
  int64_t cstride;  // floats per cell in `elem` (nn rounded up to 32: 128-byte rows)
  const int *cells;
  const double *verts;
  double ca, cb;
  const double *cell_a, *cell_b;
  const double *geo_in;  // caller weights (12 per cell) or null
  const int *order;      // cells in class order
  const int4 *groups;    // {class, first position in order, count <= 128, 0}
  int n_groups;
  const float *bimage;   // per class and chunk: B hi then lo, 4096 floats
  float *elem;           // n_cells x nn, column-major nb x nb per cell
  int *err;
};

constexpr int kAHalf = kTcThreads * 16 * 4;  // bytes of one A part (128 rows x 16 TF32)
constexpr int kBHalf = kTcN * 16 * 4;        // bytes of one B part (128 rows x 16 TF32)
constexpr int kBImage = 2 * kBHalf;          // hi + lo of one tile
constexpr int kBFloats = kBImage / 4;

struct TcSmem {
  alignas(1024) unsigned char a[2 * kAHalf];   // A hi, A lo
  alignas(1024) unsigned char b[2][kBImage];   // two B buffers
  float stage[kTcBlock / 32][32][33];          // epilogue transpose, one per warp
  int cell[kTcThreads];                        // cell of each TMEM lane (-1: none)
  uint64_t bbar[2];                            // B copy of a buffer complete
  uint64_t mbar[2];                            // MMAs into an accumulator complete
  uint32_t tmem;
  int abort;
};

// Work unit u of a CTA: its group gi = u / n_chunks (global group
// blockIdx.x + gi * gridDim.x) and tile t = u % n_chunks.
__global__ void __launch_bounds__(kTcBlock, 2) nedelec_tc_kernel(const __grid_constant__ TcArgs A) {
  extern __shared__ unsigned char tc_raw[];
  TcSmem &S = *reinterpret_cast<TcSmem *>(
      (unsigned char *)(((uintptr_t)tc_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&S.tmem)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      mbar_init(&S.bbar[i], 1);
      mbar_init(&S.mbar[i], 1);
    }
    S.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem;
  // warp w drains TMEM lanes 32 (w % 4) .. +31 (its lane quarter), columns
  // 64 (w / 4) .. +63 of each accumulator
  const int quarter = warp & 3, half = warp >> 2;
  const uint32_t tlane = tmem + ((uint32_t)(32 * quarter) << 16);
  const int nch = A.n_chunks;
  const int my_groups =
      (int)blockIdx.x < A.n_groups ? (A.n_groups - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int total = my_groups * nch;
  // thread 0's accounting of copies and MMAs in flight
  int copies_issued = 0, copies_waited = 0, mma_issued = 0;
  auto unit_class = [&](int u) {
    return A.groups[blockIdx.x + (u / nch) * gridDim.x].x;
  };
  auto issue_copy = [&](int u) {
    const int buf = u & 1;
    const float *src = A.bimage + ((size_t)unit_class(u) * nch + u % nch) * kBFloats;
    mbar_expect_tx(&S.bbar[buf], (uint32_t)kBImage);
    bulk_load(S.b[buf], src, (uint32_t)kBImage, &S.bbar[buf]);
    ++copies_issued;
  };
  // thread 0: wait for the B tile of unit u and issue its MMAs into accumulator u & 1
  auto issue_mma = [&](int u) -> bool {
    const int buf = u & 1;
    if (!mbar_wait(&S.bbar[buf], (uint32_t)((u >> 1) & 1))) return false;
    ++copies_waited;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t a0 = smem_u32(S.a), b0 = smem_u32(S.b[buf]);
    const uint32_t idesc = tf32_idesc(kTcN);
    const uint32_t d = tmem + (uint32_t)(buf * kTcN);
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      const uint64_t ah = smem_desc(a0 + ks * 2 * (kTcThreads * 16), kTcThreads * 16, 128);
      const uint64_t al = smem_desc(a0 + kAHalf + ks * 2 * (kTcThreads * 16), kTcThreads * 16, 128);
      const uint64_t bh = smem_desc(b0 + ks * 2 * (kTcN * 16), kTcN * 16, 128);
      const uint64_t bl = smem_desc(b0 + kBHalf + ks * 2 * (kTcN * 16), kTcN * 16, 128);
      mma_tf32(d, ah, bh, idesc, ks > 0 ? 1u : 0u);
      mma_tf32(d, ah, bl, idesc, 1u);
      mma_tf32(d, al, bh, idesc, 1u);
    }
    mma_commit(&S.mbar[buf]);
    ++mma_issued;
    return true;
  };
  if (tid == 0) {
    for (int u = 0; u < 2 && u < total; ++u) issue_copy(u);
  }
  int u = 0, mma_waited = 0;
  for (int gi = 0; gi < my_groups; ++gi) {
    const int4 grp = A.groups[blockIdx.x + gi * gridDim.x];
    // ---- weights of this thread's cell (FP64 geometry), split into TF32 hi
    // / lo; every MMA of the previous group has completed (its last epilogue
    // waited for it), so A may be rewritten
    int cell = -1;
    double w[12];
#pragma unroll
    for (int s = 0; s < 12; ++s) w[s] = 0.0;
    if (tid < kTcThreads && tid < grp.z) {
      cell = A.order[grp.y + tid];
      double J[9], Ji[9], v0[3];
      tet_jacobian(A.cells, A.verts, cell, J, v0);
      const double det = det3(J);
      const bool ok = valid_jacobian(J, det);
      if (!ok) atomicCAS(A.err, 0, FFG_INVALID_INPUT);
      if (ok) {
        inv3(J, det, Ji);
        if (A.geo_in) {
#pragma unroll
          for (int s = 0; s < 12; ++s) w[s] = A.geo_in[12 * (size_t)cell + s];
        } else {
          const double cw = A.ca * (A.cell_a ? A.cell_a[cell] : 1.0);
          const double mw = A.cb * (A.cell_b ? A.cell_b[cell] : 1.0);
          constexpr int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
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
    }
    if (tid < kTcThreads) {
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
      S.cell[tid] = cell;
    }
    fence_proxy_async();
    __syncthreads();
    if (tid == 0 && !issue_mma(u)) {
      atomicCAS(A.err, 0, FFG_TIMEOUT);
      S.abort = 1;
    }
    __syncthreads();
    if (S.abort) break;
    for (int t = 0; t < nch; ++t, ++u) {
      // the next tile's MMAs go into the other accumulator, whose epilogue
      // ended before the last barrier
      if (tid == 0 && t + 1 < nch && !issue_mma(u + 1)) {
        atomicCAS(A.err, 0, FFG_TIMEOUT);
        S.abort = 1;
      }
      const int buf = u & 1;
      if (!mbar_wait(&S.mbar[buf], (uint32_t)((u >> 1) & 1))) {
        atomicCAS(A.err, 0, FFG_TIMEOUT);
        S.abort = 1;
      } else if (tid == 0) {
        mma_waited = u + 1;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      __syncthreads();
      if (S.abort) break;
      // the MMAs of unit u have read B buffer `buf`: refill it with unit u + 2
      if (tid == 0 && u + 2 < total) issue_copy(u + 2);
      const int64_t e0 = (int64_t)t * kTcN;
      const int my_cell = S.cell[32 * quarter + lane];
#pragma unroll 1
      for (int ch = 2 * half; ch < 2 * half + 2; ++ch) {
        float v[32];
        tmem_ld32(tlane + (uint32_t)(buf * kTcN + 32 * ch), v);
        tmem_wait_ld();
#pragma unroll
        for (int k = 0; k < 32; ++k) S.stage[warp][lane][k] = v[k];
        __syncwarp();
        const int64_t e = e0 + 32 * ch + lane;
        // one 128-byte, line-aligned row of a cell per store instruction
#pragma unroll 4
        for (int c = 0; c < 32; ++c) {
          const int cc = __shfl_sync(0xffffffffu, my_cell, c);
          if (cc >= 0 && e < A.nn) A.elem[(size_t)cc * A.cstride + e] = S.stage[warp][c][lane];
        }
        __syncwarp();
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (S.abort) break;
  }
  // copies and MMAs still in flight complete before the CTA leaves (bounded)
  if (tid == 0) {
    bool live = true;
    while (live && copies_waited < copies_issued) {
      const int v = copies_waited;
      live = mbar_wait(&S.bbar[v & 1], (uint32_t)((v >> 1) & 1));
      if (live) ++copies_waited;
    }
    while (live && mma_waited < mma_issued) {
      const int v = mma_waited;
      live = mbar_wait(&S.mbar[v & 1], (uint32_t)((v >> 1) & 1));
      if (live) ++mma_waited;
    }
    if (!live) atomicCAS(A.err, 0, FFG_TIMEOUT);
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

// B images of every (class, chunk) from the chunk-major FP64 table: row n
// of a tile is entry n of the chunk, its K values the twelve terms and four
// zeros, split into TF32 hi / lo in the K-major core-matrix layout (the
// same rounding as the device split of the weights).
__global__ void tc_image_kernel(const double *__restrict__ ref, int64_t units,
                                float *__restrict__ img) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= units * 16 * kTcN) return;
  const int64_t unit = i / (16 * kTcN);
  const int q = (int)(i % (16 * kTcN)), s = q / kTcN, n = q % kTcN;
  const double x = s < 12 ? ref[(unit * 12 + s) * kTcN + n] : 0.0;
  const float hi = tf32_round((float)x);
  const float lo = tf32_round((float)(x - (double)hi));
  float *o = img + unit * kBFloats;
  const int pos = (s >> 2) * (kTcN * 4) + n * 4 + (s & 3);
  o[pos] = hi;
  o[kBFloats / 2 + pos] = lo;
}

}  // namespace

size_t tc_smem_bytes() {
  // at least 80 KB, so that no more than two CTAs (2 x 256 TMEM columns) share an SM
  return std::max<size_t>(sizeof(TcSmem) + 1024, 80 * 1024);
}

bool tc_supported_order(int k) { return k >= 3 && k <= 6; }

int64_t tc_cell_stride(int nb) { return ((int64_t)nb * nb + 31) / 32 * 32; }

int tc_build_plan(const Topology &t, const OrientedTables &o, TcPlan &plan, cudaStream_t s) {
  if (!tc_supported_order(t.degree) || o.order != t.degree || !o.ref) return FFG_INVALID_INPUT;
  tc_free_plan(plan);
  std::vector<int4> groups;
  int first = 0;
  for (int q = 0; q < kOrtClasses; ++q) {
    for (int f = 0; f < o.class_count[q]; f += kTcThreads)
      groups.push_back(make_int4(q, first + f, std::min(kTcThreads, o.class_count[q] - f), 0));
    first += o.class_count[q];
  }
  const int64_t units = (int64_t)kOrtClasses * o.n_chunks;
  if (cudaMalloc((void **)&plan.bimage, (size_t)units * kBImage) != cudaSuccess ||
      cudaMalloc((void **)&plan.groups, sizeof(int4) * std::max<size_t>(groups.size(), 1)) !=
          cudaSuccess) {
    tc_free_plan(plan);
    return FFG_OUT_OF_MEMORY;
  }
  if (!groups.empty() && cudaMemcpy(plan.groups, groups.data(), sizeof(int4) * groups.size(),
                                    cudaMemcpyHostToDevice) != cudaSuccess) {
    tc_free_plan(plan);
    return FFG_CUDA_ERROR;
  }
  const int64_t n = units * 16 * kTcN;
  tc_image_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(o.ref, units, plan.bimage);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
    tc_free_plan(plan);
    return FFG_CUDA_ERROR;
  }
  plan.order = t.degree;
  plan.n_chunks = o.n_chunks;
  plan.n_groups = (int)groups.size();
  plan.image_bytes = (size_t)units * kBImage;
  return FFG_OK;
}

void tc_free_plan(TcPlan &plan) {
  if (plan.bimage) cudaFree(plan.bimage);
  if (plan.groups) cudaFree(plan.groups);
  plan = TcPlan();
}

int launch_nedelec_tc(const Topology &t, const DeviceTopology &dt, const AssemblyInputs &in,
                      const TcPlan &plan, float *elem, int *err, cudaStream_t s) {
  if (t.family != FFG_TETRA_NEDELEC || plan.order != t.degree || !plan.bimage || !dt.ort)
    return FFG_INVALID_INPUT;
  if (plan.n_groups == 0) return FFG_OK;
  TcArgs A;
  A.nb = t.nb;
  A.n_chunks = plan.n_chunks;
  A.nn = (int64_t)t.nb * t.nb;
  A.cstride = tc_cell_stride(t.nb);
  A.cells = dt.cells;
  A.verts = in.vertices;
  A.ca = in.coef_a;
  A.cb = in.coef_b;
  A.cell_a = in.cell_a;
  A.cell_b = in.cell_b;
  A.geo_in = in.geo_override;
  A.order = dt.ort->order_cells;
  A.groups = plan.groups;
  A.n_groups = plan.n_groups;
  A.bimage = plan.bimage;
  A.elem = elem;
  A.err = err;
  const size_t smem = tc_smem_bytes();
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int per_sm = (in.tune && in.tune->tc_ctas_per_sm) ? in.tune->tc_ctas_per_sm : 2;
  const int grid = std::min(plan.n_groups, per_sm * sms);
  if (cudaFuncSetAttribute(nedelec_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return FFG_CUDA_ERROR;
  nedelec_tc_kernel<<<grid, kTcBlock, smem, s>>>(A);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace ffg
