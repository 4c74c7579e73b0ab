// Persistent Jacobi-PCG (sm_100a) on a SELL-32-sigma operator.
//
// One cooperative launch runs the whole solve.  Every CTA owns a contiguous
// range of 32-row slices (balanced by stored entries plus a per-slice cost)
// and therefore a contiguous range of rows of the permuted system; its
// slices are dealt to its warps longest first (sell_partition).  In the SpMV
// a warp walks its slices: the bulk-copy engine streams each slice's values
// and 16-bit column offsets into shared memory, 10 columns at a time, and
// lane l accumulates row 32s+l in a fixed order.  Vector phases walk rows
// with all threads, coalesced.  Dot products are summed per thread in a
// fixed row order, reduced per CTA, written to a per-phase partial buffer and
// summed by every CTA in the same fixed order, so all CTAs take identical
// decisions and results are bit-reproducible for a given grid.  Grid
// barriers spin with a time bound and report FFG_TIMEOUT instead of hanging.
//
// FP64 mode restates pcg_solve_operator / pcg_iteration_loop
// (src/solvers/advanced_solvers.f90:831-925), two grid barriers an iteration:
//   A: p = z + beta p_old on the fly while gathering, q = A p, (p, q)
//   B: x += alpha p, r -= alpha q, z = D^-1 r, (r, r), (r, z)
// The (z, p) pair of every row is stored interleaved and double-buffered so
// the gather of iteration k never races with the writes of iteration k+1.
// It stops when the recursive residual ||r||_2 <= tol*||r_0||_2 (relative)
// or tol (absolute), or at breakdown (|p^T A p| < 1e-14 as the reference, or
// p^T A p <= 0 when selected); Jacobi z = D^-1 r with D^-1 = 1 where
// |a_ii| <= 1e-14.
// Mixed mode: the same CG recurrences in FP32 on a scaled residual with the
// solution accumulated in FP64, the SpMV gathering z alone (q = A p is
// carried as A z + beta q_old); whenever the FP32 residual has fallen by the
// reliable-update factor (or claims convergence) the true FP64 residual
// b - A x replaces it (the search direction is kept, rescaled), and the solve
// ends when ||b - A x||_2 <= tol*||b||_2.  A replacement is also forced when
// the FP32 residual grows tenfold past the last true residual (the search
// direction then restarts) or plateaus for four times the previous
// replacement interval.  If replacements stop reducing the true residual the
// solve continues in the FP64 loop from the current x; if the FP32 p^T A p is
// not positive (condition number beyond FP32 reach, as for curl-curl
// operators with a small mass term) the FP64 loop starts again from x = 0.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "ffg_internal.h"

namespace ffg {

namespace {

constexpr int kThreads = 1024;
constexpr int kWarps = kThreads / 32;
constexpr int kSlots = 4;
constexpr int kPartialBatch = 8;   // partial loads in flight per lane
constexpr int kResultDoubles = 16;
constexpr int kMinWindow = 256;  // iterations before a plateau forces a reliable update
constexpr unsigned long long kBarrierLimitNs = 4000000000ull;  // 4 s per barrier wait
// Staged SpMV: every warp streams its slices through kStages shared-memory
// buffers of kStageBytes (32 rows by as many columns as fit: values, then
// column indices).  Measured on the 48^3 P2 system (FP32 + int16): 2 x 10
// columns (120 KB per CTA) beats 2 x 6/8/12/14/16 and 3 x 8 (wider stages
// take L1 the gathers need).
constexpr int kStageBytes = 10 * 32 * (4 + 2);                 // 1920 B
constexpr int kStages = 2;                                   // chunks in flight per warp
constexpr int kStageSmem = kWarps * kStages * kStageBytes;   // 120 KB per CTA
constexpr unsigned long long kCopyLimitNs = 1000000000ull;   // 1 s per copy wait

struct PcgParams {
  int64_t n;
  const int64_t *soff;
  const int16_t *dcol;
  const int *col;
  const float *v32;
  const __half *v16;  // FFG_PRECISION_MIXED16: FP16 operator, row r scaled by rs[r]
  const float *rs;
  const double *v64;
  const float *d32;
  const double *d64;
  const int *cta_slice;
  const int *wslice, *woff;  // per-warp slice lists of the cooperative grid
  const double *b;
  double *x;
  double *r64;
  float *rf, *zf, *pf, *qf;  // mixed mode: r, z = D^-1 r, p, q = A p
  float *xf;                 // mixed mode: increment of x since it was last folded in
  float2 *zpf0, *zpf1;       // mixed mode after a switch to direct A p: (z, p) pairs
  double *rd, *qd;
  double2 *zpd0, *zpd1;
  double *partial;  // [2][kSlots][grid]
  unsigned int *bar;
  int *control;     // [0] error status
  double *result;   // kResultDoubles
  int precision, relative, max_it, max_updates, guard;
  double tol, delta;
  unsigned long long limit_ns;
  // CTAs that solve this system: blockIdx.x - cta0 in [0, ncta).  With one
  // CTA the system's slices are [0, n_slices) and barriers are CTA barriers.
  int cta0, ncta, n_slices;
  int staged;  // launched with kStageSmem bytes of dynamic shared memory
};

// Set when a warp's staged copy did not complete in time; every barrier
// checks it, so the solve ends on the next one.
__shared__ int g_abort;
// Per-warp mbarriers of the two staging buffers, initialised once per kernel
// (an mbarrier is not re-initialised while in use), and the parity each warp
// waits for next on each of them.
__shared__ unsigned long long g_mbar[kWarps][kStages];
__shared__ unsigned g_mparity[kWarps];

__device__ __forceinline__ int cta_of(const PcgParams &P) { return (int)blockIdx.x - P.cta0; }

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_volatile_int(const int *p) {
  return *reinterpret_cast<const volatile int *>(p);
}

// Bounded grid barrier.  Every CTA calls it the same number of times; the
// counter is reset by the host before launch.  Returns false on failure.
__device__ bool grid_barrier(const PcgParams &P, unsigned int &phase) {
  __shared__ int ok;
  __syncthreads();
  ++phase;
  if (g_abort) return false;
  if (P.ncta == 1) return true;
  if (threadIdx.x == 0) {
    // arrival with release semantics: the CTA's writes before the
    // __syncthreads above are ordered before it (bar.sync, then release)
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(P.bar) : "memory");
    const unsigned int target = phase * (unsigned int)P.ncta;
    const unsigned long long t0 = globaltimer();
    int good = 1;
    unsigned int spins = 0;
    while (true) {
      if ((int)(ld_acquire(P.bar) - target) >= 0) break;
      if (ld_volatile_int(P.control) != 0) { good = 0; break; }
      if ((++spins & 255u) == 0 && globaltimer() - t0 > kBarrierLimitNs) {
        atomicCAS(P.control, 0, FFG_TIMEOUT);
        good = 0;
        break;
      }
    }
    // the acquire load that saw the count orders the reads that follow
    ok = good && ld_volatile_int(P.control) == 0;
  }
  __syncthreads();
  return ok != 0;
}

// CTA-wide sums of nslot per-thread values into this phase's partial buffer.
__device__ void write_partials(const PcgParams &P, unsigned int phase, const double *v, int nslot) {
  __shared__ double red[kSlots][kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int s = 0; s < nslot; ++s) {
    double x = v[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[s][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < nslot) {
    double x = 0.0;
    for (int w = 0; w < kWarps; ++w) x += red[threadIdx.x][w];
    P.partial[((size_t)((phase + 1) & 1) * kSlots + threadIdx.x) * P.ncta + cta_of(P)] = x;
  }
}

// Sum the partials of the phase that just completed (identical on every CTA).
// Warp s reduces slot s; its loads are issued before the adds so they overlap,
// and the summation order is fixed (lane-strided, then a butterfly), so every
// CTA obtains the same bits.
__device__ void read_partials(const PcgParams &P, unsigned int phase, double *out, int nslot) {
  __shared__ double res[kSlots];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < nslot) {
    const int G = P.ncta;
    const double *src = P.partial + ((size_t)(phase & 1) * kSlots + warp) * G;
    double acc = 0.0;
    for (int b0 = 0; b0 < G; b0 += 32 * kPartialBatch) {
      double v[kPartialBatch];
#pragma unroll
      for (int j = 0; j < kPartialBatch; ++j) {
        const int b = b0 + lane + 32 * j;
        v[j] = b < G ? __ldcg(src + b) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < kPartialBatch; ++j) acc += v[j];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) res[warp] = acc;
  }
  __syncthreads();
  for (int s = 0; s < nslot; ++s) out[s] = res[s];
  __syncthreads();
}

// Slices [s0, s1) of the calling CTA.
__device__ __forceinline__ void slice_range(const PcgParams &P, int &s0, int &s1) {
  if (P.ncta == 1) {
    s0 = 0;
    s1 = P.n_slices;
  } else if (!P.cta_slice) {
    // a CTA group of a batch: equal slice counts
    s0 = (int)((int64_t)cta_of(P) * P.n_slices / P.ncta);
    s1 = (int)((int64_t)(cta_of(P) + 1) * P.n_slices / P.ncta);
  } else {
    s0 = P.cta_slice[cta_of(P)];
    s1 = P.cta_slice[cta_of(P) + 1];
  }
}

// The slices of one warp, in the order it takes them: the list dealt to it
// when the whole cooperative grid solves the system, otherwise every 32nd
// slice of the CTA's range.
struct WarpSlices {
  const int *list;
  int k0, n, first;
  __device__ __forceinline__ int at(int k) const { return list ? list[k0 + k] : first + k * kWarps; }
};

__device__ __forceinline__ WarpSlices warp_slices(const PcgParams &P, int warp) {
  WarpSlices w;
  if (P.wslice && P.ncta > 1) {
    const int i = cta_of(P) * kWarps + warp;
    w.list = P.wslice;
    w.k0 = P.woff[i];
    w.n = P.woff[i + 1] - w.k0;
    w.first = 0;
  } else {
    int s0, s1;
    slice_range(P, s0, s1);
    w.list = nullptr;
    w.k0 = 0;
    w.first = s0 + warp;
    w.n = w.first < s1 ? (s1 - w.first + kWarps - 1) / kWarps : 0;
  }
  return w;
}

// Asynchronous L2 prefetch of a byte range (16-byte aligned, size a nonzero
// multiple of 16): the warp's next slice streams into L2 while the current
// one is processed, so its loads meet L2 rather than HBM latency.
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Values and column indices of slice s.  Slice offsets are multiples of 32
// entries, so both ranges start 64-byte aligned and are multiples of 64 bytes.
template <typename V, bool NARROW>
__device__ __forceinline__ void prefetch_slice(const PcgParams &P, const V *val, int s) {
  const int64_t e0 = P.soff[s], e1 = P.soff[s + 1];
  if (e1 <= e0) return;
  prefetch_l2(val + e0, (unsigned)((e1 - e0) * sizeof(V)));
  if (NARROW) prefetch_l2(P.dcol + e0, (unsigned)((e1 - e0) * sizeof(int16_t)));
  else prefetch_l2(P.col + e0, (unsigned)((e1 - e0) * sizeof(int)));
}

// SELL SpMV over this CTA's slices: each warp walks its own slices
// (warp_slices) and prefetches its next slice into L2 while it sums the
// current one; lane l owns row 32s+l and accumulates it in a fixed order.
// Returns the thread's sum, in a fixed order, of what g.finish returns for
// its rows.
template <typename V, bool NARROW, class G>
__device__ __noinline__ double spmv_pairs(const PcgParams &P, const V *__restrict__ val,
                                          const G g) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSlices ws = warp_slices(P, warp);
  double dot = 0.0;
  if (lane == 0 && ws.n > 0) prefetch_slice<V, NARROW>(P, val, ws.at(0));
  for (int k = 0; k < ws.n; ++k) {
    const int s = ws.at(k);
    if (lane == 0 && k + 1 < ws.n) prefetch_slice<V, NARROW>(P, val, ws.at(k + 1));
    const int64_t base = P.soff[s] + lane;
    const int len = (int)((P.soff[s + 1] - P.soff[s]) / kSliceRows);
    const int row = s * kSliceRows + lane;
    typename G::Acc acc{};
#pragma unroll 8
    for (int j = 0; j < len; ++j) {
      const int64_t e = base + (int64_t)j * kSliceRows;
      const int c = NARROW ? row + (int)__ldcs(P.dcol + e) : __ldcs(P.col + e);
      g.accumulate(acc, __ldcs(val + e), c);
    }
    if (row < P.n) dot += g.finish(row, acc);
  }
  __syncthreads();
  return dot;
}

// ------------------------------------------------------ staged FP32 SpMV
__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *m) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(m)) : "memory");
}

// The operator is read once per iteration: its lines enter L2 as evict-first
// so that they do not push the iteration vectors out.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes,
                                          unsigned long long *m) {
  uint64_t policy;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(policy));
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(m)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ void mbar_expect(unsigned long long *m, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)),
               "r"(bytes)
               : "memory");
}

// Bounded wait on an mbarrier phase (1 s); on failure flags the solve and
// returns false.
__device__ bool mbar_wait(const PcgParams &P, unsigned long long *m, unsigned parity) {
  const unsigned a = smem_addr(m);
  unsigned long long t0 = 0;
  for (unsigned spin = 0;; ++spin) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((spin & 1023u) == 0) {
      const unsigned long long t = globaltimer();
      if (t0 == 0) t0 = t;
      else if (t - t0 > kCopyLimitNs) break;
    }
  }
  atomicCAS(P.control, 0, FFG_TIMEOUT);
  g_abort = 1;
  return false;
}

// Stage layout of one (value type, index type) pair: kStageBytes per stage
// holds COLS columns of 32 rows, values first.  FP32 + int16: 10 columns,
// FP32 + int32: 7, FP64 + int16: 6, FP64 + int32: 5.
template <typename V, bool NARROW>
struct StageShape {
  static constexpr int kEntry = (int)sizeof(V) + (NARROW ? 2 : 4);
  static constexpr int COLS = kStageBytes / (32 * kEntry);
  static constexpr int VAL = COLS * 32 * (int)sizeof(V);
};

// The chunk of `cols` columns starting at entry e0 into stage buffer `buf`
// (values, then indices).  Slice offsets are multiples of 32 entries and
// chunks multiples of COLS columns, so both sources are 64-byte aligned and
// both sizes multiples of 64.
template <typename V, bool NARROW>
__device__ __forceinline__ void issue_chunk(const PcgParams &P, const V *val, int64_t e0, int cols,
                                            unsigned char *buf, unsigned long long *m) {
  using SS = StageShape<V, NARROW>;
  const unsigned nv = (unsigned)cols * 32u * (unsigned)sizeof(V);
  const unsigned nc = (unsigned)cols * 32u * (NARROW ? 2u : 4u);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect(m, nv + nc);
  bulk_load(buf, val + e0, nv, m);
  if (NARROW) bulk_load(buf + SS::VAL, P.dcol + e0, nc, m);
  else bulk_load(buf + SS::VAL, P.col + e0, nc, m);
}

// One slice of a warp's list: its index, first entry and length in columns.
struct SliceRef {
  int s, len;
  int64_t e0;
};

// The SpMV of spmv_pairs (same slices per warp, same return value) with the
// operator streamed by the bulk-copy engine: warp w keeps one chunk of COLS
// columns in flight while it
// gathers and sums the other, so the bytes in flight per SM are set by shared
// memory rather than by registers.  The copies mark their L2 lines
// evict-first, which keeps the iteration vectors in L2.  Each row is still
// summed by one lane in column order.
template <typename V, bool NARROW, class G>
__device__ __noinline__ double spmv_staged(const PcgParams &P, const V *__restrict__ val,
                                           const G g) {
  using SS = StageShape<V, NARROW>;
  constexpr int COLS = SS::COLS;
  extern __shared__ __align__(1024) unsigned char stage_smem[];
  unsigned long long(&mbar)[kWarps][kStages] = g_mbar;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const WarpSlices ws = warp_slices(P, warp);
  unsigned char *wbuf = stage_smem + (size_t)warp * kStages * kStageBytes;
  // lane k holds slice k of the warp's list (read once per SpMV), so that the
  // copy of the next chunk never waits on a load of the slice offsets; a
  // list longer than 32 reads the rest from memory
  int my_s = 0, my_len = 0;
  int64_t my_e0 = 0;
  if (lane < ws.n) {
    my_s = ws.at(lane);
    my_e0 = P.soff[my_s];
    my_len = (int)((P.soff[my_s + 1] - my_e0) / kSliceRows);
  }
  auto slice = [&](int k) {  // k is warp-uniform
    SliceRef r;
    if (k < 32) {
      r.s = __shfl_sync(0xffffffffu, my_s, k);
      r.len = __shfl_sync(0xffffffffu, my_len, k);
      r.e0 = __shfl_sync(0xffffffffu, my_e0, k);
    } else {
      r.s = ws.at(k);
      r.e0 = P.soff[r.s];
      r.len = (int)((P.soff[r.s + 1] - r.e0) / kSliceRows);
    }
    return r;
  };
  // producer cursor: chunk pc of the warp's pk-th slice (pr) is copied next
  // (slices with no columns are skipped)
  int pk = 0, pc = 0;
  SliceRef pr{0, 0, 0};
  auto seek = [&]() {
    for (; pk < ws.n; ++pk) {
      pr = slice(pk);
      if (pr.len > 0) break;
    }
  };
  seek();
  auto advance = [&]() {
    if (++pc * COLS >= pr.len) {
      pc = 0;
      ++pk;
      seek();
    }
  };
  auto issue = [&](int st) {
    if (lane == 0)
      issue_chunk<V, NARROW>(P, val, pr.e0 + (int64_t)pc * COLS * 32, min(COLS, pr.len - pc * COLS),
                             wbuf + st * kStageBytes, &mbar[warp][st]);
  };
  unsigned pending = 0;  // stages with a copy issued and not yet waited for
  for (int k = 0; k < kStages && pk < ws.n; ++k) {
    issue(k);
    pending |= 1u << k;
    advance();
  }
  unsigned parity = g_mparity[warp], seq = 0;
  bool ok = true;
  double dot = 0.0;
  for (int ck = 0; ck < ws.n; ++ck) {
    const SliceRef cr = slice(ck);
    const int len = cr.len;
    const int row = cr.s * kSliceRows + lane;
    typename G::Acc acc{};
    for (int c = 0; c * COLS < len; ++c, ++seq) {
      const int st = (int)(seq % kStages);
      if (ok) {
        const bool got = mbar_wait(P, &mbar[warp][st], (parity >> st) & 1u);
        ok = __all_sync(0xffffffffu, got);
        if (ok) {
          pending &= ~(1u << st);
          parity ^= 1u << st;
        }
      }
      const int cols = min(COLS, len - c * COLS);
      const V *vb = reinterpret_cast<const V *>(wbuf + st * kStageBytes);
      const unsigned char *ib = wbuf + st * kStageBytes + SS::VAL;
      if (ok) {
#pragma unroll
        for (int j = 0; j < COLS; ++j) {
          if (j < cols) {
            const int cidx = NARROW ? row + (int)reinterpret_cast<const int16_t *>(ib)[j * 32 + lane]
                                    : reinterpret_cast<const int *>(ib)[j * 32 + lane];
            g.accumulate(acc, vb[j * 32 + lane], cidx);
          }
        }
      }
      __syncwarp();
      if (pk < ws.n) {
        if (ok) {
          issue(st);
          pending |= 1u << st;
        }
        advance();
      }
    }
    if (row < P.n && ok) dot += g.finish(row, acc);
  }
  // after a failed wait, give the copies still in flight (bounded) time to
  // land before the stage buffers are given up
  for (int st = 0; st < kStages; ++st)
    if (!ok && (pending >> st) & 1u) mbar_wait(P, &mbar[warp][st], (parity >> st) & 1u);
  __syncwarp();
  if (lane == 0) g_mparity[warp] = parity;
  __syncthreads();
  return dot;
}

template <class F>
__device__ __forceinline__ void for_rows(const PcgParams &P, F f) {
  int s0, s1;
  slice_range(P, s0, s1);
  const int64_t r0 = (int64_t)s0 * kSliceRows;
  const int64_t r1 = min((int64_t)s1 * kSliceRows, P.n);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) f((int)r);
}

// The same rows split evenly over the CTAs (32-row multiples).  The slice
// ranges balance stored entries, which suits the SpMV; a purely row-wise
// phase that follows a grid barrier balances better on equal row counts.
template <class F>
__device__ __forceinline__ void for_rows_even(const PcgParams &P, F f) {
  const int64_t per = ((P.n + (int64_t)P.ncta * kSliceRows - 1) / ((int64_t)P.ncta * kSliceRows)) *
                      kSliceRows;
  const int64_t r0 = (int64_t)cta_of(P) * per;
  const int64_t r1 = min(r0 + per, P.n);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) f((int)r);
}

// for_rows_even kRowBatch rows at a time: load(row, u) runs for the batch's
// rows before step(row, u) runs for any of them, so that their loads are in
// flight together; each thread still visits its rows in increasing order.
constexpr int kRowBatch = 4;
template <class L, class F>
__device__ __forceinline__ void for_rows_even_batched(const PcgParams &P, L load, F step) {
  const int64_t per = ((P.n + (int64_t)P.ncta * kSliceRows - 1) / ((int64_t)P.ncta * kSliceRows)) *
                      kSliceRows;
  const int64_t r0 = (int64_t)cta_of(P) * per;
  const int64_t r1 = min(r0 + per, P.n);
  for (int64_t b = r0 + threadIdx.x; b < r1; b += (int64_t)kRowBatch * kThreads) {
#pragma unroll
    for (int u = 0; u < kRowBatch; ++u) {
      const int64_t row = b + (int64_t)u * kThreads;
      if (row < r1) load((int)row, u);
    }
#pragma unroll
    for (int u = 0; u < kRowBatch; ++u) {
      const int64_t row = b + (int64_t)u * kThreads;
      if (row < r1) step((int)row, u);
    }
  }
}

__device__ __forceinline__ bool is_finite_d(double x) { return isfinite(x); }

struct Outcome {
  int iterations = 0, updates = 0, converged = 0, status = FFG_OK, stagnated = 0, aborted = 0;
  int restart = 0;  // the FP32 phase broke down: the FP64 loop starts again from x = 0
  double true_res = 0.0, final_res = 0.0, bnorm = 0.0;
};

// Device time of the phases seen by CTA 0 (the others are symmetric):
// SpMV work, wait at the following barrier, vector work, wait, and the
// residual-replacement phases.
struct Timing {
  unsigned long long a = 0, aw = 0, b = 0, bw = 0, u = 0;
};

__device__ __forceinline__ unsigned long long stamp(const PcgParams &P) {
  return (cta_of(P) == 0 && threadIdx.x == 0) ? globaltimer() : 0ull;
}

// Gather policies of the SpMV: accumulate(acc, a, c) adds the stored entry a
// of column c to the row's accumulator and finish(row, acc) stores the row's
// results with the row-wise updates that belong to them, returning the row's
// term of the phase's dot product.

// FP64 PCG: the operand p = z + beta p_old of column c is formed on the fly
// from the (z, p_old) pair; finish stores p and q = A p.
template <typename V, typename V2>
struct PairGather {
  const V2 *__restrict__ zc;
  V2 *__restrict__ zn;
  V *__restrict__ q;
  V beta;
  using Acc = V;
  __device__ __forceinline__ V column(int c) const {
    const V2 a = zc[c];
    return a.x + beta * a.y;
  }
  __device__ __forceinline__ void accumulate(Acc &acc, V v, int c) const { acc += v * column(c); }
  __device__ __forceinline__ double finish(int row, V acc) const {
    const V2 a = zc[row];
    const V pn = a.x + beta * a.y;
    zn[row].y = pn;
    q[row] = acc;
    return (double)pn * (double)acc;
  }
};

// Mixed mode: the SpMV gathers z alone and forms q = A p as A z + beta q_old
// (p = z + beta p_old), so a column costs 4 bytes of gather instead of the
// 8 of a (z, p) pair; finish stores p and q of the row.
struct ZGather {
  const float *__restrict__ z;
  float *__restrict__ p;
  float *__restrict__ q;
  float beta;
  using Acc = float;
  __device__ __forceinline__ void accumulate(Acc &acc, float v, int c) const { acc += v * z[c]; }
  __device__ __forceinline__ double finish(int row, float acc) const {
    const float pn = z[row] + beta * p[row];
    const float qn = acc + beta * q[row];
    p[row] = pn;
    q[row] = qn;
    return (double)pn * (double)qn;
  }
};

// The same two gathers on the FP16 operator: entries are FP16 bits of
// a_ij / s_i, so the row's sum is scaled by s_i before it is used.
struct ZGatherH {
  ZGather g;
  const float *__restrict__ rs;
  using Acc = float;
  __device__ __forceinline__ void accumulate(Acc &acc, __half v, int c) const {
    acc += __half2float(v) * g.z[c];
  }
  __device__ __forceinline__ double finish(int row, float acc) const {
    return g.finish(row, acc * rs[row]);
  }
};

struct PairGatherH {
  PairGather<float, float2> g;
  const float *__restrict__ rs;
  using Acc = float;
  __device__ __forceinline__ void accumulate(Acc &acc, __half v, int c) const {
    acc += __half2float(v) * g.column(c);
  }
  __device__ __forceinline__ double finish(int row, float acc) const {
    return g.finish(row, acc * rs[row]);
  }
};

// r64 = b - A x with the FP64 operator, returning the row's term of (r64, r64);
// with p given, also q = A p (FP64 products, stored in FP32) in the same pass.
struct ResidualGather {
  const double *__restrict__ x;
  const float *__restrict__ p;
  float *__restrict__ q;
  const double *__restrict__ b;
  double *__restrict__ r64;
  struct Acc {
    double x = 0.0, p = 0.0;
  };
  __device__ __forceinline__ void accumulate(Acc &acc, double v, int c) const {
    acc.x += v * x[c];
    if (p) acc.p += v * (double)p[c];
  }
  __device__ __forceinline__ double finish(int row, const Acc &acc) const {
    const double r = b[row] - acc.x;
    r64[row] = r;
    if (p) q[row] = (float)acc.p;
    return r * r;
  }
};

template <typename V, class G>
__device__ __forceinline__ double spmv(const PcgParams &P, const V *val, const G &g) {
  if (P.staged && P.dcol) return spmv_staged<V, true>(P, val, g);
  if (P.staged) return spmv_staged<V, false>(P, val, g);
  if (P.dcol) return spmv_pairs<V, true>(P, val, g);
  return spmv_pairs<V, false>(P, val, g);
}

// r64 = b - A x; returns the thread's share of (r64, r64) (and q = A p when p
// is given).
__device__ __forceinline__ double residual(const PcgParams &P, const float *p = nullptr,
                                           float *q = nullptr) {
  return spmv(P, P.v64, ResidualGather{P.x, p, q, P.b, P.r64});
}

// r64 = b - A x and the partial sums of (r64, r64) and (b, b), reduced.
__device__ bool residual_norms(const PcgParams &P, unsigned int &phase, double *red) {
  double part[kSlots];
  part[0] = residual(P);
  part[1] = 0.0;
  for_rows(P, [&](int row) {
    const double bb = P.b[row];
    part[1] += bb * bb;
  });
  write_partials(P, phase, part, 2);
  if (!grid_barrier(P, phase)) return false;
  read_partials(P, phase, red, 2);
  return true;
}

// FP64 Jacobi-PCG, the reference's recurrences.  `continuation` runs it after
// a stagnated mixed solve: its target is then the true residual tol*||b|| and
// its guard the SPD one.
__device__ __noinline__ void cg64(const PcgParams &P, unsigned int &phase,
                                  unsigned long long t_start, bool continuation, Outcome &o,
                                  Timing &tm) {
  const double *A = P.v64;
  const double *dinv = P.d64;
  double *r = P.rd;
  double *q = P.qd;
  double2 *zp[2] = {P.zpd0, P.zpd1};
  double part[kSlots], red[kSlots];
  unsigned long long t0, t1, t2;

  t0 = stamp(P);
  if (!residual_norms(P, phase, red)) { o.aborted = 1; return; }
  const double bnorm = sqrt(red[1]);
  const double rnorm = sqrt(red[0]);
  o.bnorm = bnorm;
  const double target = P.relative ? P.tol * (continuation ? bnorm : rnorm) : P.tol;
  double true_res = rnorm, last_true = rnorm;
  int stall = 0;
  // continuation: restarted cycles; a cycle ends when the recursive residual
  // reaches the target or after twice the first cycle's iterations
  int cycle_its = 0, first_cycle = 0;
  int converged = (rnorm <= target) ? 1 : 0;
  double rz = 0.0;
  if (!converged) {
    part[0] = 0.0;
    for_rows(P, [&](int row) {
      const double rr = P.r64[row];
      const double z = dinv[row] * rr;
      r[row] = rr;
      zp[0][row] = double2{z, 0.0};
      part[0] += rr * z;
    });
    write_partials(P, phase, part, 1);
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 1);
    rz = red[0];
  }
  tm.u += stamp(P) - t0;
  double beta = 0.0;
  int cur = 0;
  const int budget = P.max_it - o.iterations;
  for (int it = 1; !converged && it <= budget; ++it) {
    const double2 *zc = zp[cur];
    double2 *zn = zp[cur ^ 1];
    // A: p = z + beta p_old, q = A p, (p, q)
    t0 = stamp(P);
    part[0] = spmv(P, A, PairGather<double, double2>{zc, zn, q, beta});
    write_partials(P, phase, part, 1);
    t1 = stamp(P);
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 1);
    t2 = stamp(P);
    tm.a += t1 - t0;
    tm.aw += t2 - t1;
    const double pAp = red[0];
    const bool breakdown = (!continuation && P.guard == 0) ? (fabs(pAp) < 1.0e-14)
                                                           : !(pAp > 0.0 && is_finite_d(pAp));
    if (breakdown) break;
    const double alpha = rz / pAp;
    // B: x += alpha p, r -= alpha q, z = D^-1 r
    t0 = stamp(P);
    part[0] = part[1] = 0.0;
    part[2] = (cta_of(P) == 0 && threadIdx.x == 0 && globaltimer() - t_start > P.limit_ns) ? 1.0 : 0.0;
    {
      double2 a[kRowBatch] = {};
      double xv[kRowBatch] = {}, rv[kRowBatch] = {}, qv[kRowBatch] = {}, dv[kRowBatch] = {};
      for_rows_even_batched(
          P,
          [&](int row, int u) {
            a[u] = zn[row];
            xv[u] = P.x[row];
            rv[u] = r[row];
            qv[u] = q[row];
            dv[u] = dinv[row];
          },
          [&](int row, int u) {
            P.x[row] = xv[u] + alpha * a[u].y;
            const double rr = rv[u] - alpha * qv[u];
            r[row] = rr;
            const double z = dv[u] * rr;
            zn[row].x = z;
            part[0] += rr * rr;
            part[1] += rr * z;
          });
    }
    write_partials(P, phase, part, 3);
    t1 = stamp(P);
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 3);
    t2 = stamp(P);
    tm.b += t1 - t0;
    tm.bw += t2 - t1;
    ++o.iterations;
    double rz_new = red[1];
    const double est = sqrt(red[0]);
    true_res = est;
    if (red[2] != 0.0) { o.status = FFG_TIMEOUT; break; }
    if (est <= target && !continuation) { converged = 1; break; }
    ++cycle_its;
    bool restart = false;
    if (continuation &&
        (est <= target || (first_cycle > 0 && cycle_its >= 2 * first_cycle))) {
      // the continuation's target is the true residual: check b - A x and,
      // while it still falls, start a new CG cycle from it (the recursive
      // residual of a long FP64 run drifts from the true one, and a cycle
      // whose recursive residual cannot reach the target is cut off)
      t0 = stamp(P);
      if (first_cycle == 0) first_cycle = cycle_its;
      cycle_its = 0;
      restart = true;
      part[0] = residual(P);
      write_partials(P, phase, part, 1);
      if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
      read_partials(P, phase, red, 1);
      true_res = sqrt(red[0]);
      if (true_res <= target) { converged = 1; tm.u += stamp(P) - t0; break; }
      stall = (true_res > 0.5 * last_true) ? stall + 1 : 0;
      last_true = true_res;
      if (stall >= 2 || !is_finite_d(true_res)) { tm.u += stamp(P) - t0; break; }
      ++o.updates;
      part[0] = 0.0;
      for_rows(P, [&](int row) {
        const double rr2 = P.r64[row];
        r[row] = rr2;
        const double z = dinv[row] * rr2;
        double2 a = zn[row];
        a.x = z;
        zn[row] = a;
        part[0] += rr2 * z;
      });
      write_partials(P, phase, part, 1);
      if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
      read_partials(P, phase, red, 1);
      tm.u += stamp(P) - t0;
      rz_new = red[0];
    }
    beta = (rz != 0.0 && !restart) ? rz_new / rz : 0.0;
    rz = rz_new;
    cur ^= 1;
  }
  o.converged = converged;
  o.final_res = true_res;
  // true FP64 residual of the returned x
  t0 = stamp(P);
  part[0] = residual(P);
  write_partials(P, phase, part, 1);
  if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
  read_partials(P, phase, red, 1);
  tm.u += stamp(P) - t0;
  o.true_res = sqrt(red[0]);
}

// Mixed mode: x += the FP32 increment gathered since the last fold, for every
// row once, then a grid barrier so that x is whole before it is read.
__device__ bool fold_x(const PcgParams &P, unsigned int &phase) {
  for_rows_even(P, [&](int row) {
    P.x[row] += (double)P.xf[row];
    P.xf[row] = 0.f;
  });
  return grid_barrier(P, phase);
}

// Mixed mode: the PCG recurrences in FP32 on a scaled residual, the solution
// accumulated in FP64, two grid barriers an iteration:
//   A: w = A z (gathering z alone), p = z + beta p, q = w + beta q, (p, q)
//   B: dx += alpha p, r -= alpha q, z = D^-1 r, (r, r), (r, z)
// The step dx is accumulated in FP32 and added to the FP64 x before every
// true residual (iterative refinement: each interval between reliable updates
// solves for a correction whose own FP32 rounding the next interval removes).
// q is A p up to the rounding of its recurrence, and every reliable update
// recomputes it from p.  That rounding grows with the condition number: the
// first reliable update forced by a plateau, or one whose true residual has
// not halved (other than after a restart, which the non-monotone residual of
// CG makes routine early on), switches the solve for good to the direct
// form, in which A gathers (z, p_old) pairs and forms q = A (z + beta p_old)
// on the fly.
__device__ __noinline__ void cg_mixed(const PcgParams &P, unsigned int &phase,
                                      unsigned long long t_start, Outcome &o, Timing &tm) {
  const float *dinv = P.d32;
  float *r = P.rf, *z = P.zf, *p = P.pf, *q = P.qf;
  float2 *zp[2] = {P.zpf0, P.zpf1};
  double part[kSlots], red[kSlots];
  unsigned long long t0, t1, t2;

  t0 = stamp(P);
  if (!residual_norms(P, phase, red)) { o.aborted = 1; return; }
  const double bnorm = sqrt(red[1]);
  const double rnorm = sqrt(red[0]);
  o.bnorm = bnorm;
  double scale = rnorm > 0.0 ? rnorm : 1.0;
  const double target = P.relative ? P.tol * bnorm : P.tol;
  double true_res = rnorm, last_true = rnorm;
  int stall = 0, since = 0, window = kMinWindow;
  int converged = (rnorm <= target) ? 1 : 0;
  bool direct = false;
  int cur = 0;
  double rz = 0.0;
  if (!converged) {
    const double inv = 1.0 / scale;
    part[0] = 0.0;
    for_rows(P, [&](int row) {
      const float rr = (float)(P.r64[row] * inv);
      const float zz = dinv[row] * rr;
      r[row] = rr;
      z[row] = zz;
      p[row] = 0.f;
      q[row] = 0.f;
      P.xf[row] = 0.f;
      part[0] += (double)rr * (double)zz;
    });
    write_partials(P, phase, part, 1);
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 1);
    rz = red[0];
  }
  tm.u += stamp(P) - t0;
  double beta = 0.0;
  bool unfolded = false;  // xf holds a step not yet added to x
  const int budget = P.max_it - o.iterations;
  for (int it = 1; !converged && it <= budget; ++it) {
    // A: q = A p, p = z + beta p, (p, q)
    t0 = stamp(P);
    part[0] = 0.0;
    const float bt = (float)beta;
    float2 *zn = zp[cur ^ 1];
    if (P.v16)
      part[0] = direct ? spmv(P, P.v16, PairGatherH{{zp[cur], zn, q, bt}, P.rs})
                       : spmv(P, P.v16, ZGatherH{{z, p, q, bt}, P.rs});
    else
      part[0] = direct ? spmv(P, P.v32, PairGather<float, float2>{zp[cur], zn, q, bt})
                       : spmv(P, P.v32, ZGather{z, p, q, bt});
    write_partials(P, phase, part, 1);
    t1 = stamp(P);
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 1);
    t2 = stamp(P);
    tm.a += t1 - t0;
    tm.aw += t2 - t1;
    const double pAp = red[0];
    if (!(pAp > 0.0 && is_finite_d(pAp))) {
      // an FP32 p^T A p that is not positive (cancellation on a near-null
      // direction of the operator) ends the FP32 phase: the operator is
      // beyond FP32's reach, so the FP64 loop starts again from x = 0 (an x
      // built by FP32 steps on such an operator carries near-null error
      // components that FP64 CG reduces far more slowly than from zero)
      o.stagnated = 1;
      o.restart = 1;
      break;
    }
    const double alpha = rz / pAp;
    const float al = (float)alpha;
    const float xs = (float)(alpha * scale);
    // B: dx += alpha p, r -= alpha q, z = D^-1 r
    t0 = stamp(P);
    part[0] = part[1] = 0.0;
    part[2] = (cta_of(P) == 0 && threadIdx.x == 0 && globaltimer() - t_start > P.limit_ns) ? 1.0 : 0.0;
    {
      float xv[kRowBatch] = {}, pv[kRowBatch] = {}, rv[kRowBatch] = {}, qv[kRowBatch] = {},
            dv[kRowBatch] = {};
      auto step = [&](int row, int u) {
        P.xf[row] = xv[u] + xs * pv[u];
        const float rr = rv[u] - al * qv[u];
        r[row] = rr;
        const float zz = dv[u] * rr;
        if (direct) zn[row].x = zz;
        else z[row] = zz;
        part[0] += (double)rr * (double)rr;
        part[1] += (double)rr * (double)zz;
      };
      auto load = [&](int row, int u) {
        xv[u] = P.xf[row];
        rv[u] = r[row];
        qv[u] = q[row];
        dv[u] = dinv[row];
      };
      if (direct)
        for_rows_even_batched(P, [&](int row, int u) { load(row, u); pv[u] = zn[row].y; }, step);
      else
        for_rows_even_batched(P, [&](int row, int u) { load(row, u); pv[u] = p[row]; }, step);
    }
    write_partials(P, phase, part, 3);
    t1 = stamp(P);
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 3);
    t2 = stamp(P);
    tm.b += t1 - t0;
    tm.bw += t2 - t1;
    ++o.iterations;
    unfolded = true;
    if (direct) cur ^= 1;
    const double rr = red[0], rz_new = red[1];
    const double est = sqrt(rr) * scale;
    if (red[2] != 0.0) { o.status = FFG_TIMEOUT; true_res = est; break; }
    // reliable update: replace the recursive residual with b - A x in FP64
    // when it has fallen by delta, claims convergence, has grown tenfold
    // past the last true residual (the FP32 recurrence is diverging; the
    // search then restarts), or has not triggered within `window`
    // iterations (an FP32 plateau, judged by the stall test below)
    const bool grew = !(est < 10.0 * scale);
    const bool slow = o.iterations - since > window;
    if (!(est <= target || rr <= P.delta * P.delta || grew || slow)) {
      beta = rz_new / rz;
      rz = rz_new;
      continue;
    }
    if (o.updates >= P.max_updates) break;
    ++o.updates;
    t0 = stamp(P);
    if (!fold_x(P, phase)) { o.aborted = 1; return; }
    unfolded = false;
    // q = A p comes with the residual (used if the update goes on in the
    // recurrence form)
    part[0] = direct ? residual(P) : residual(P, p, q);
    write_partials(P, phase, part, 1);
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 1);
    true_res = sqrt(red[0]);
    if (true_res <= target) { converged = 1; tm.u += stamp(P) - t0; break; }
    if (!(true_res > 0.0) || !is_finite_d(true_res)) break;
    stall = (true_res > 0.5 * last_true) ? stall + 1 : 0;
    last_true = true_res;
    if (stall >= 2) { o.stagnated = 1; tm.u += stamp(P) - t0; break; }
    const bool to_direct = !direct && (slow || (stall > 0 && !grew));
    // r = (b - A x) / ||b - A x|| in the new units and z = D^-1 r; p keeps
    // the old units and the ratio goes into beta.  The recurrence form goes
    // on with q = A p from the residual pass; the direct form (or the switch
    // to it) stores (z, p).
    const double ratio = scale / true_res;
    const double inv = 1.0 / true_res;
    part[0] = 0.0;
    if (direct) {
      float2 *zc = zp[cur];
      for_rows(P, [&](int row) {
        const float rr2 = (float)(P.r64[row] * inv);
        const float zz = dinv[row] * rr2;
        r[row] = rr2;
        zc[row].x = zz;
        part[0] += (double)rr2 * (double)zz;
      });
    } else if (to_direct) {
      float2 *zc = zp[cur];
      for_rows(P, [&](int row) {
        const float rr2 = (float)(P.r64[row] * inv);
        const float zz = dinv[row] * rr2;
        r[row] = rr2;
        zc[row] = make_float2(zz, p[row]);
        part[0] += (double)rr2 * (double)zz;
      });
      direct = true;
    } else {
      for_rows(P, [&](int row) {
        const float rr2 = (float)(P.r64[row] * inv);
        const float zz = dinv[row] * rr2;
        r[row] = rr2;
        z[row] = zz;
        part[0] += (double)rr2 * (double)zz;
      });
    }
    write_partials(P, phase, part, 1);
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 1);
    tm.u += stamp(P) - t0;
    // p_new = z + beta' (ratio p): beta' against the old (r, z) in new units
    beta = grew ? 0.0 : red[0] / (rz * ratio);
    rz = red[0];
    scale = true_res;
    window = max(kMinWindow, 4 * (o.iterations - since));
    since = o.iterations;
  }
  if (unfolded && !fold_x(P, phase)) { o.aborted = 1; return; }
  o.converged = converged;
  o.final_res = true_res;
  if (converged) {
    o.true_res = true_res;
    return;
  }
  if (o.stagnated) return;  // the FP64 continuation measures its own residual
  // true FP64 residual of the returned x
  t0 = stamp(P);
  part[0] = residual(P);
  write_partials(P, phase, part, 1);
  if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
  read_partials(P, phase, red, 1);
  tm.u += stamp(P) - t0;
  o.true_res = sqrt(red[0]);
  o.final_res = o.true_res;
}

__device__ __forceinline__ void pcg_body(const PcgParams &P) {
  unsigned int phase = 0;
  if (threadIdx.x == 0) g_abort = 0;
  if (P.staged && (threadIdx.x & 31) == 0) {
    for (int st = 0; st < kStages; ++st) mbar_init(&g_mbar[threadIdx.x >> 5][st]);
    g_mparity[threadIdx.x >> 5] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // only block 0 judges the wall limit; its verdict travels through a partial slot
  const unsigned long long t_start = globaltimer();
  Outcome o;
  Timing tm;
  int continued = 0;
  if (P.precision == FFG_PRECISION_FP64) {
    cg64(P, phase, t_start, false, o, tm);
  } else {
    cg_mixed(P, phase, t_start, o, tm);
    if (!o.aborted && o.stagnated && !o.converged && o.status == FFG_OK) {
      continued = o.restart ? 2 : 1;
      if (o.restart) {
        for_rows_even(P, [&](int row) { P.x[row] = 0.0; });
        if (!grid_barrier(P, phase)) return;
      }
      cg64(P, phase, t_start, true, o, tm);
    }
  }
  if (o.aborted) return;
  if (cta_of(P) == 0 && threadIdx.x == 0) {
    P.result[0] = o.converged;
    P.result[1] = o.iterations;
    P.result[2] = o.updates;
    P.result[3] = o.final_res;
    P.result[4] = o.bnorm > 0.0 ? o.true_res / o.bnorm : o.true_res;
    P.result[5] = o.status;
    P.result[6] = o.bnorm;
    P.result[7] = continued;
    P.result[8] = 1e-9 * (double)tm.a;
    P.result[9] = 1e-9 * (double)tm.aw;
    P.result[10] = 1e-9 * (double)tm.b;
    P.result[11] = 1e-9 * (double)tm.bw;
    P.result[12] = 1e-9 * (double)tm.u;
  }
}

// One system solved by the whole cooperative grid.
__global__ void __launch_bounds__(kThreads, 1) pcg_kernel(PcgParams P) { pcg_body(P); }

// Up to kMaxBatch independent systems, one CTA each (no inter-CTA waits, so
// an ordinary launch; systems never share a CTA or a reduction, so every
// system's result is independent of what else is in the batch).
constexpr int kMaxBatch = 48;
struct PcgBatch {
  PcgParams sys[kMaxBatch];
};
__global__ void __launch_bounds__(kThreads, 1) pcg_batch_kernel(const __grid_constant__ PcgBatch B) {
  __shared__ PcgParams Ps;
  if (threadIdx.x == 0) {
    Ps = B.sys[blockIdx.x];
    Ps.cta0 = (int)blockIdx.x;
    Ps.ncta = 1;
  }
  __syncthreads();
  pcg_body(Ps);
}

// Up to kMaxGroups independent systems in one cooperative launch, system i
// on CTAs [first[i], first[i + 1]) with its own barrier counter, partial
// sums and control word.  The launch makes every CTA resident together, so
// a group's barrier waits only on CTAs that are running; the group size
// depends on the system alone (pcg_group_ctas), so its result does not
// depend on the other systems of the launch.
constexpr int kMaxGroups = 16;
constexpr int64_t kGroupRows = 16384;  // rows per CTA of a group
struct PcgGroups {
  PcgParams sys[kMaxGroups];
  int first[kMaxGroups + 1];
  int count;
};
__global__ void __launch_bounds__(kThreads, 1) pcg_group_kernel(const __grid_constant__ PcgGroups B) {
  __shared__ PcgParams Ps;
  if (threadIdx.x == 0) {
    int i = 0;
    while (i + 1 < B.count && B.first[i + 1] <= (int)blockIdx.x) ++i;
    Ps = B.sys[i];
    Ps.cta0 = B.first[i];
    Ps.ncta = B.first[i + 1] - B.first[i];
    // the operator's partition is for the whole grid: groups split evenly
    Ps.cta_slice = nullptr;
    Ps.wslice = nullptr;
    Ps.woff = nullptr;
  }
  __syncthreads();
  pcg_body(Ps);
}

// Drop-in FP64 CSR SpMV, one thread per row (spmv / csc_matvec semantics).
__global__ void csr_spmv64_kernel(int64_t n, const int64_t *rp, const int *ci, const double *v,
                                  const double *x, double *y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int64_t k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
  y[i] = s;
}

// FP32 copy of SELL values and the Jacobi inverse diagonal, from the CSR
// (old numbering) through the entry positions `pos`.
__global__ void sell_prepare_kernel(int64_t n, const int64_t *rp, const int *ci,
                                    const int64_t *pos, const int *iperm, const double *v64,
                                    float *v32, double *d64, float *d32, int jacobi) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double d = 0.0;
  for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
    const double a = v64[pos[k]];
    v32[pos[k]] = (float)a;
    if (ci[k] == (int)i) d = a;
  }
  // build_sparse_preconditioner("jacobi"), advanced_solvers.f90:1139-1154
  const double di = (jacobi && fabs(d) > 1.0e-14) ? 1.0 / d : 1.0;
  d64[iperm[i]] = di;
  d32[iperm[i]] = (float)di;
}

}  // namespace

namespace {
// Opt the PCG kernels into kStageSmem bytes of dynamic shared memory (once per
// device); false when the device refuses, in which case they run unstaged.
bool staged_smem_ready() {
  static std::mutex mu;
  static int state[64] = {0};  // 0 unknown, 1 ready, -1 refused
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return false;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (state[dev] == 0) {
    const bool ok =
        cudaFuncSetAttribute((const void *)pcg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kStageSmem) == cudaSuccess &&
        cudaFuncSetAttribute((const void *)pcg_batch_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kStageSmem) == cudaSuccess &&
        cudaFuncSetAttribute((const void *)pcg_group_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, kStageSmem) == cudaSuccess;
    if (!ok) cudaGetLastError();
    state[dev] = ok ? 1 : -1;
  }
  return state[dev] == 1;
}
}  // namespace

int pcg_grid_size(int *grid) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FFG_CUDA_ERROR;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return FFG_CUDA_ERROR;
  const size_t smem = staged_smem_ready() ? kStageSmem : 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel, kThreads, smem) !=
      cudaSuccess)
    return FFG_CUDA_ERROR;
  if (per_sm < 1) return FFG_CUDA_ERROR;
  *grid = sms;  // one 1024-thread CTA per SM
  return FFG_OK;
}

int upload_sell(const HostSell &h, int grid, DeviceSell &d) {
  free_sell(d);
  d.n = h.n;
  d.n_slices = h.n_slices;
  d.padded = h.padded;
  d.grid = grid;
  bool bad = false;
  auto A = [&](void **p, size_t bytes) {
    if (cudaMalloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) { bad = true; *p = nullptr; }
  };
  const size_t P = (size_t)std::max<int64_t>(h.padded, 1), N = (size_t)std::max<int64_t>(h.n, 1);
  A((void **)&d.soff, sizeof(int64_t) * h.soff.size());
  if (h.narrow) A((void **)&d.dcol, sizeof(int16_t) * P);
  else A((void **)&d.col, sizeof(int) * P);
  A((void **)&d.val64, sizeof(double) * P);
  A((void **)&d.val32, sizeof(float) * P);
  A((void **)&d.dinv64, sizeof(double) * N);
  A((void **)&d.dinv32, sizeof(float) * N);
  A((void **)&d.perm, sizeof(int) * N);
  A((void **)&d.iperm, sizeof(int) * N);
  std::vector<int> cs, wslice, woff;
  sell_partition(h.soff.data(), h.n_slices, grid, cs, wslice, woff);
  A((void **)&d.cta_slice, sizeof(int) * (grid + 1));
  A((void **)&d.wslice, sizeof(int) * wslice.size());
  A((void **)&d.woff, sizeof(int) * woff.size());
  if (bad) { cudaGetLastError(); free_sell(d); return FFG_OUT_OF_MEMORY; }
  bool ok = true;
  ok = ok && cudaMemcpy(d.soff, h.soff.data(), sizeof(int64_t) * h.soff.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  if (h.narrow)
    ok = ok && cudaMemcpy(d.dcol, h.dcol.data(), sizeof(int16_t) * h.padded, cudaMemcpyHostToDevice) == cudaSuccess;
  else
    ok = ok && cudaMemcpy(d.col, h.col.data(), sizeof(int) * h.padded, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemset(d.val64, 0, sizeof(double) * P) == cudaSuccess;
  ok = ok && cudaMemset(d.val32, 0, sizeof(float) * P) == cudaSuccess;
  ok = ok && cudaMemcpy(d.perm, h.perm.data(), sizeof(int) * h.n, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(d.iperm, h.iperm.data(), sizeof(int) * h.n, cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(d.cta_slice, cs.data(), sizeof(int) * (grid + 1), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!wslice.empty())
    ok = ok && cudaMemcpy(d.wslice, wslice.data(), sizeof(int) * wslice.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(d.woff, woff.data(), sizeof(int) * woff.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  return ok ? FFG_OK : FFG_CUDA_ERROR;
}

// A slice costs its stored entries plus kSliceCost for its row epilogue and
// copy waits.  CTAs take contiguous slice ranges of about equal cost; inside
// a CTA the slices are dealt longest first, each to the warp with the least
// cost so far (lowest warp on ties), and a warp takes its slices in the
// order dealt.  Dealing by cost rather than round robin matters because
// slices are sorted by length inside each sigma window, so every 32nd slice
// lands on a warp-dependent mix of long and short ones.
void sell_partition(const int64_t *soff, int64_t n_slices, int grid, std::vector<int> &cs,
                    std::vector<int> &wslice, std::vector<int> &woff, int slice_cost) {
  const int64_t kSliceCost = slice_cost;
  const int64_t ns = n_slices;
  auto cost = [&](int64_t s) { return soff[s + 1] - soff[s] + kSliceCost; };
  std::vector<int64_t> cum((size_t)ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s) cum[s + 1] = cum[s] + cost(s);
  cs.assign((size_t)grid + 1, 0);
  for (int b = 1; b < grid; ++b) {
    const int64_t target = (int64_t)((double)cum[ns] * b / grid);
    const int s = (int)(std::lower_bound(cum.begin(), cum.end(), target) - cum.begin());
    cs[b] = std::max(cs[b - 1], std::min<int>(s, (int)ns));
  }
  cs[grid] = (int)ns;
  wslice.clear();
  wslice.reserve((size_t)ns);
  woff.assign((size_t)grid * kWarps + 1, 0);
  std::vector<std::vector<int>> lists(kWarps);
  std::vector<int> order;
  for (int b = 0; b < grid; ++b) {
    order.resize((size_t)(cs[b + 1] - cs[b]));
    for (size_t i = 0; i < order.size(); ++i) order[i] = cs[b] + (int)i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return cost(x) > cost(y); });
    std::vector<int64_t> load(kWarps, 0);
    for (int s : order) {
      const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      lists[w].push_back(s);
      load[w] += cost(s);
    }
    for (int w = 0; w < kWarps; ++w) {
      woff[(size_t)b * kWarps + w] = (int)wslice.size();
      wslice.insert(wslice.end(), lists[w].begin(), lists[w].end());
      lists[w].clear();
    }
  }
  woff[(size_t)grid * kWarps] = (int)wslice.size();
}

namespace {
// val16 = FP16(val32 / s_r) with s_r the row's largest |val32| (1 for an
// empty row); one thread per row walks the row's entries in its slice.
__global__ void sell_half_kernel(int64_t n, const int64_t *__restrict__ soff,
                                 const float *__restrict__ v32, __half *__restrict__ v16,
                                 float *__restrict__ rs) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t s = r / kSliceRows, e0 = soff[s] + r % kSliceRows;
  const int width = (int)((soff[s + 1] - soff[s]) / kSliceRows);
  float m = 0.f;
  for (int k = 0; k < width; ++k) m = fmaxf(m, fabsf(v32[e0 + (int64_t)k * kSliceRows]));
  const float sc = m > 0.f ? m : 1.f;
  const float inv = 1.f / sc;
  for (int k = 0; k < width; ++k) {
    const int64_t e = e0 + (int64_t)k * kSliceRows;
    v16[e] = __float2half_rn(v32[e] * inv);
  }
  rs[r] = sc;
}

// padding rows of the last slice: zero values, unit scale
__global__ void sell_half_pad_kernel(int64_t n, int64_t n_slices, const int64_t *__restrict__ soff,
                                     __half *__restrict__ v16) {
  const int64_t r = n + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_slices * kSliceRows) return;
  const int64_t s = r / kSliceRows, e0 = soff[s] + r % kSliceRows;
  const int width = (int)((soff[s + 1] - soff[s]) / kSliceRows);
  for (int k = 0; k < width; ++k) v16[e0 + (int64_t)k * kSliceRows] = __float2half_rn(0.f);
}
}  // namespace

int sell_half(DeviceSell &d, cudaStream_t s) {
  if (d.n <= 0) return FFG_OK;
  const size_t P = (size_t)std::max<int64_t>(d.padded, 1);
  if (!d.val16 && cudaMalloc((void **)&d.val16, sizeof(uint16_t) * P) != cudaSuccess) {
    cudaGetLastError();
    return FFG_OUT_OF_MEMORY;
  }
  if (!d.rscale && cudaMalloc((void **)&d.rscale, sizeof(float) * (size_t)d.n) != cudaSuccess) {
    cudaGetLastError();
    return FFG_OUT_OF_MEMORY;
  }
  __half *v16 = reinterpret_cast<__half *>(d.val16);
  sell_half_kernel<<<(unsigned)((d.n + 255) / 256), 256, 0, s>>>(d.n, d.soff, d.val32, v16,
                                                                  d.rscale);
  const int64_t pad = d.n_slices * kSliceRows - d.n;
  if (pad > 0)
    sell_half_pad_kernel<<<(unsigned)((pad + 255) / 256), 256, 0, s>>>(d.n, d.n_slices, d.soff,
                                                                      v16);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

int sell_repartition(DeviceSell &d, int slice_cost) {
  if (d.grid <= 0 || !d.soff || !d.cta_slice || !d.woff) return FFG_INVALID_INPUT;
  std::vector<int64_t> soff((size_t)d.n_slices + 1);
  if (cudaMemcpy(soff.data(), d.soff, sizeof(int64_t) * soff.size(), cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return FFG_CUDA_ERROR;
  std::vector<int> cs, ws, wo;
  sell_partition(soff.data(), d.n_slices, d.grid, cs, ws, wo, slice_cost);
  bool ok = cudaMemcpy(d.cta_slice, cs.data(), sizeof(int) * cs.size(), cudaMemcpyHostToDevice) ==
            cudaSuccess;
  if (!ws.empty())
    ok = ok && cudaMemcpy(d.wslice, ws.data(), sizeof(int) * ws.size(), cudaMemcpyHostToDevice) ==
                   cudaSuccess;
  ok = ok && cudaMemcpy(d.woff, wo.data(), sizeof(int) * wo.size(), cudaMemcpyHostToDevice) ==
                 cudaSuccess;
  return ok ? FFG_OK : FFG_CUDA_ERROR;
}

void free_sell(DeviceSell &d) {
  void *ptrs[] = {d.soff, d.dcol, d.col, d.val64, d.val32, d.val16, d.rscale, d.dinv64, d.dinv32,
                  d.perm, d.iperm,
                  d.cta_slice, d.wslice, d.woff, d.inc_range};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  d = DeviceSell();
}

int solve_work_alloc(SolveWork &w, int64_t n, int grid) {
  solve_work_free(w);
  w.n = n;
  w.grid = grid;
  const size_t N = (size_t)std::max<int64_t>(n, 1);
  bool bad = false;
  auto A = [&](void **p, size_t bytes) {
    if (cudaMalloc(p, bytes) != cudaSuccess) { bad = true; *p = nullptr; }
  };
  A((void **)&w.r64, N * sizeof(double));
  A((void **)&w.rd, N * sizeof(double));
  A((void **)&w.qd, N * sizeof(double));
  A((void **)&w.zpd0, N * sizeof(double2));
  A((void **)&w.zpd1, N * sizeof(double2));
  A((void **)&w.rf, N * sizeof(float));
  A((void **)&w.zf, N * sizeof(float));
  A((void **)&w.pf, N * sizeof(float));
  A((void **)&w.qf, N * sizeof(float));
  A((void **)&w.xf, N * sizeof(float));
  A((void **)&w.zpf0, N * sizeof(float2));
  A((void **)&w.zpf1, N * sizeof(float2));
  A((void **)&w.partial, 2 * kSlots * (size_t)grid * sizeof(double));
  A((void **)&w.barrier, 64);
  A((void **)&w.control, 64);
  A((void **)&w.result, kResultDoubles * sizeof(double));
  if (!bad && (cudaMallocHost((void **)&w.result_host, kResultDoubles * sizeof(double)) != cudaSuccess ||
               cudaMallocHost((void **)&w.control_host, 2 * sizeof(int)) != cudaSuccess))
    bad = true;
  if (!bad) {
    std::memset(w.result_host, 0, kResultDoubles * sizeof(double));
    w.control_host[0] = w.control_host[1] = 0;
    if (cudaMemset(w.control, 0, 64) != cudaSuccess || cudaMemset(w.barrier, 0, 64) != cudaSuccess)
      bad = true;
  }
  if (bad) {
    solve_work_free(w);
    cudaGetLastError();
    return FFG_OUT_OF_MEMORY;
  }
  return FFG_OK;
}

void solve_work_free(SolveWork &w) {
  void *ptrs[] = {w.r64, w.rd, w.qd, w.zpd0, w.zpd1, w.rf, w.zf, w.pf, w.qf, w.xf, w.zpf0, w.zpf1,
                  w.partial,
                  w.barrier, w.control, w.result};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (w.result_host) cudaFreeHost(w.result_host);
  if (w.control_host) cudaFreeHost(w.control_host);
  w = SolveWork();
}

namespace {
PcgParams make_params(const DeviceSell &A, const double *b, double *x,
                      const ffg_solver_options &opts, const SolveWork &w) {
  PcgParams P;
  P.n = A.n;
  P.soff = A.soff;
  P.dcol = A.dcol;
  P.col = A.col;
  P.v32 = A.val32;
  P.v16 = opts.precision == FFG_PRECISION_MIXED16 ? reinterpret_cast<const __half *>(A.val16)
                                                  : nullptr;
  P.rs = A.rscale;
  P.v64 = A.val64;
  P.d32 = A.dinv32;
  P.d64 = A.dinv64;
  P.cta_slice = A.cta_slice;
  P.wslice = A.wslice;
  P.woff = A.woff;
  P.b = b;
  P.x = x;
  P.r64 = w.r64;
  P.rf = w.rf; P.zf = w.zf; P.pf = w.pf; P.qf = w.qf; P.xf = w.xf;
  P.zpf0 = w.zpf0; P.zpf1 = w.zpf1;
  P.rd = w.rd; P.qd = w.qd; P.zpd0 = w.zpd0; P.zpd1 = w.zpd1;
  P.partial = w.partial;
  P.bar = w.barrier;
  P.control = w.control;
  P.result = w.result;
  P.precision = opts.precision;
  P.relative = opts.tolerance_type == 0;
  P.max_it = opts.max_iterations;
  P.max_updates = opts.max_refinements;
  P.tol = opts.tolerance;
  P.delta = opts.inner_tolerance;
  P.guard = opts.breakdown_guard;
  // clamped to a million seconds so that the conversion stays in range
  const double limit = fmin(opts.timeout_seconds > 0 ? opts.timeout_seconds : 60.0, 1.0e6);
  P.limit_ns = (unsigned long long)(limit * 1e9);
  P.cta0 = 0;
  P.ncta = A.grid;
  P.n_slices = (int)A.n_slices;
  P.staged = 0;
  return P;
}
}  // namespace

int pcg_launch(const DeviceSell &A, const double *b, double *x, const ffg_solver_options &opts,
               SolveWork &w, cudaStream_t stream, std::string &msg) {
  if (w.n != A.n || w.grid <= 0 || A.grid != w.grid) {
    msg = "solver workspace mismatch";
    return FFG_INVALID_INPUT;
  }
  PcgParams P = make_params(A, b, x, opts, w);
  P.staged = staged_smem_ready() ? 1 : 0;
  if (cudaMemsetAsync(w.barrier, 0, 64, stream) != cudaSuccess) return FFG_CUDA_ERROR;
  if (cudaMemsetAsync(w.control, 0, 64, stream) != cudaSuccess) return FFG_CUDA_ERROR;
  if (cudaMemsetAsync(w.result, 0, kResultDoubles * sizeof(double), stream) != cudaSuccess)
    return FFG_CUDA_ERROR;
  void *args[] = {&P};
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)pcg_kernel, dim3(w.grid),
                                              dim3(kThreads), args,
                                              P.staged ? kStageSmem : 0, stream);
  if (e != cudaSuccess) {
    msg = std::string("cooperative launch failed: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return FFG_CUDA_ERROR;
  }
  if (cudaMemcpyAsync(w.result_host, w.result, kResultDoubles * sizeof(double),
                      cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaMemcpyAsync(w.control_host, w.control, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess)
    return FFG_CUDA_ERROR;
  return FFG_OK;
}

int pcg_launch_batch(int count, const DeviceSell *const *A, const double *const *b,
                     double *const *x, const ffg_solver_options &opts, SolveWork *const *w,
                     cudaStream_t stream, std::string &msg) {
  for (int i = 0; i < count; ++i)
    if (w[i]->n != A[i]->n || A[i]->n < 1) {
      msg = "solver workspace mismatch";
      return FFG_INVALID_INPUT;
    }
  static_assert(sizeof(PcgBatch) <= 32000, "kernel parameter block too large");
  const int staged = staged_smem_ready() ? 1 : 0;
  PcgBatch B;
  for (int c0 = 0; c0 < count; c0 += kMaxBatch) {
    const int m = std::min(kMaxBatch, count - c0);
    for (int i = 0; i < m; ++i) {
      B.sys[i] = make_params(*A[c0 + i], b[c0 + i], x[c0 + i], opts, *w[c0 + i]);
      B.sys[i].staged = staged;
      w[c0 + i]->control_host[0] = 0;
    }
    pcg_batch_kernel<<<m, kThreads, staged ? kStageSmem : 0, stream>>>(B);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      msg = std::string("batch launch failed: ") + cudaGetErrorString(e);
      return FFG_CUDA_ERROR;
    }
    for (int i = 0; i < m; ++i)
      if (cudaMemcpyAsync(w[c0 + i]->result_host, w[c0 + i]->result,
                          kResultDoubles * sizeof(double), cudaMemcpyDeviceToHost,
                          stream) != cudaSuccess)
        return FFG_CUDA_ERROR;
  }
  return FFG_OK;
}

int pcg_group_ctas(int64_t n, int grid) {
  const int64_t g = (n + kGroupRows - 1) / kGroupRows;
  return (int)std::max<int64_t>(2, std::min<int64_t>(g, grid));
}

int pcg_launch_groups(int count, const DeviceSell *const *A, const double *const *b,
                      double *const *x, const ffg_solver_options &opts, SolveWork *const *w,
                      cudaStream_t stream, std::string &msg) {
  static_assert(sizeof(PcgGroups) <= 32000, "kernel parameter block too large");
  int grid = 0;
  int st = pcg_grid_size(&grid);
  if (st) return st;
  for (int i = 0; i < count; ++i)
    if (w[i]->n != A[i]->n || A[i]->n < 1 || w[i]->grid < pcg_group_ctas(A[i]->n, grid)) {
      msg = "solver workspace mismatch";
      return FFG_INVALID_INPUT;
    }
  const int staged = staged_smem_ready() ? 1 : 0;
  // consecutive systems fill a launch while their groups fit the grid
  for (int i0 = 0; i0 < count;) {
    PcgGroups B;
    B.count = 0;
    B.first[0] = 0;
    int i = i0;
    while (i < count && B.count < kMaxGroups) {
      const int g = pcg_group_ctas(A[i]->n, grid);
      if (B.count > 0 && B.first[B.count] + g > grid) break;
      B.sys[B.count] = make_params(*A[i], b[i], x[i], opts, *w[i]);
      B.sys[B.count].staged = staged;
      B.first[B.count + 1] = B.first[B.count] + g;
      ++B.count;
      w[i]->control_host[0] = 0;
      if (cudaMemsetAsync(w[i]->barrier, 0, 64, stream) != cudaSuccess ||
          cudaMemsetAsync(w[i]->control, 0, 64, stream) != cudaSuccess ||
          cudaMemsetAsync(w[i]->result, 0, kResultDoubles * sizeof(double), stream) !=
              cudaSuccess)
        return FFG_CUDA_ERROR;
      ++i;
    }
    void *args[] = {&B};
    const cudaError_t e = cudaLaunchCooperativeKernel(
        (const void *)pcg_group_kernel, dim3(B.first[B.count]), dim3(kThreads), args,
        staged ? kStageSmem : 0, stream);
    if (e != cudaSuccess) {
      msg = std::string("cooperative group launch failed: ") + cudaGetErrorString(e);
      cudaGetLastError();
      return FFG_CUDA_ERROR;
    }
    for (int k = i0; k < i; ++k)
      if (cudaMemcpyAsync(w[k]->result_host, w[k]->result, kResultDoubles * sizeof(double),
                          cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
          cudaMemcpyAsync(w[k]->control_host, w[k]->control, 2 * sizeof(int),
                          cudaMemcpyDeviceToHost, stream) != cudaSuccess)
        return FFG_CUDA_ERROR;
    i0 = i;
  }
  return FFG_OK;
}

int pcg_collect(SolveWork &w, ffg_solver_stats *stats, std::string &msg) {
  const double *res = w.result_host;
  if (w.control_host[0] != 0) {
    msg = "grid barrier timed out";
    if (stats) stats->status = w.control_host[0];
    return w.control_host[0];
  }
  if (stats) {
    stats->converged = (int)res[0];
    stats->iterations = (int)res[1];
    stats->refinements = (int)res[2];
    stats->final_residual = res[3];
    stats->true_relative_residual = res[4];
    stats->status = (int)res[5];
    if (stats->status == FFG_OK && !stats->converged) stats->status = FFG_NOT_CONVERGED;
  }
  for (int i = 0; i < 6; ++i) w.phase_seconds[i] = res[7 + i];
  return FFG_OK;
}

int pcg_solve(const DeviceSell &A, const double *b, double *x, const ffg_solver_options &opts,
              SolveWork &w, ffg_solver_stats *stats, cudaStream_t stream, std::string &msg) {
  int st = pcg_launch(A, b, x, opts, w, stream, msg);
  if (st) return st;
  if (cudaStreamSynchronize(stream) != cudaSuccess) return FFG_CUDA_ERROR;
  return pcg_collect(w, stats, msg);
}

int csr_spmv64(int64_t n, const int64_t *rp, const int *ci, const double *v, const double *x,
               double *y, cudaStream_t stream) {
  if (n <= 0) return FFG_OK;
  csr_spmv64_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(n, rp, ci, v, x, y);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

int sell_prepare(DeviceSell &A, const int64_t *rp, const int *ci, const int64_t *pos, bool jacobi,
                 cudaStream_t s) {
  if (A.n <= 0) return FFG_OK;
  sell_prepare_kernel<<<(unsigned)((A.n + 255) / 256), 256, 0, s>>>(
      A.n, rp, ci, pos, A.iperm, A.val64, A.val32, A.dinv64, A.dinv32, jacobi ? 1 : 0);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace ffg
