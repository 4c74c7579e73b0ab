// Persistent Jacobi-PCG (sm_100a).
//
// One cooperative launch runs the whole solve.  CTAs own fixed row tiles of
// the CSR matrix (the constrained CSC of a symmetric operator read as CSR).
// Each SpMV streams the CTA's tiles with 16-byte loads into shared memory and
// sums every row in a fixed order.  Dot products are reduced per CTA, written
// to a per-phase partial buffer and summed by every CTA in the same fixed
// order, so all CTAs take identical decisions and results are
// bit-reproducible for a given grid.  Grid barriers spin with a time bound and
// report FFG_TIMEOUT instead of hanging.
//
// Iteration (two grid barriers):
//   A: p = z + beta p_old on the fly while gathering, q = A p, (p, q)
//   B: x += alpha p (FP64), r -= alpha q, z = D^-1 r, (r, r), (r, z)
// The (z, p) pair of every row is stored interleaved and double-buffered so
// the gather of iteration k never races with the writes of iteration k+1.
//
// FP64 mode restates pcg_solve_operator / pcg_iteration_loop
// (src/solvers/advanced_solvers.f90:831-925): stop when the recursive residual
// ||r||_2 <= tol*||r_0||_2 (relative) or tol (absolute), or at breakdown
// (|p^T A p| < 1e-14 as the reference, or p^T A p <= 0 when selected);
// Jacobi z = D^-1 r with D^-1 = 1 where |a_ii| <= 1e-14.
// Mixed mode: the same CG recurrences in FP32 on a scaled residual with the
// solution accumulated in FP64; whenever the FP32 residual has fallen by
// `reliable_delta` (or claims convergence) the true FP64 residual b - A x
// replaces it (reliable updates: the search direction is kept, rescaled), and
// the solve ends when ||b - A x||_2 <= tol*||b||_2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "ffg_internal.h"

namespace ffg {

namespace {

constexpr int kThreads = 512;
constexpr int kTileNnz = 4096;
constexpr int kSlots = 4;
constexpr int kPartialBatch = 8;   // partial loads in flight per lane
constexpr int kResultDoubles = 16;
constexpr unsigned long long kBarrierLimitNs = 4000000000ull;  // 4 s per barrier wait

struct PcgParams {
  int64_t n;
  const int64_t *rp;
  const int *col;
  const float *v32;
  const double *v64;
  const float *d32;
  const double *d64;
  const int *tile_row;
  int n_tiles;
  const double *b;
  double *x;
  double *r64;
  float *rf, *qf;
  float2 *zpf0, *zpf1;
  double *rd, *qd;
  double2 *zpd0, *zpd1;
  double *partial;  // [2][kSlots][grid]
  unsigned int *bar;
  int *control;     // [0] error status
  double *result;   // 8 doubles
  int precision, relative, max_it, max_updates, guard;
  double tol, delta;
  unsigned long long limit_ns;
};

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
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(P.bar, 1u);
    const unsigned int target = phase * gridDim.x;
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
      __nanosleep(20);
    }
    __threadfence();
    ok = good && ld_volatile_int(P.control) == 0;
  }
  __syncthreads();
  return ok != 0;
}

// CTA-wide sums of nslot per-thread values into this phase's partial buffer.
__device__ void write_partials(const PcgParams &P, unsigned int phase, const double *v, int nslot) {
  __shared__ double red[kSlots][kThreads / 32];
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
    for (int w = 0; w < kThreads / 32; ++w) x += red[threadIdx.x][w];
    P.partial[((size_t)((phase + 1) & 1) * kSlots + threadIdx.x) * gridDim.x + blockIdx.x] = x;
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
    const int G = (int)gridDim.x;
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

// ---------------------------------------------------------------- tile staging
// The (column, value) stream of a tile is copied global -> shared by the bulk
// async-copy engine (cp.async.bulk, completion on an mbarrier), double
// buffered so that the next tile streams while the current one is gathered
// and summed.  Ranges are widened to 16-byte boundaries (the matrix arrays are
// padded) and the extra entries are ignored.
constexpr int kTileCap = kTileNnz + 8;
struct __align__(16) TileBuf {
  int col[kTileCap];
  double val[kTileCap];  // FP32 tiles use the first half as float[]
};
struct StageSmem {
  TileBuf buf[2];
  unsigned long long mbar[2];
};

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *m) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(m)) : "memory");
}

// The matrix is streamed once per SpMV: evict it first from L2 so that the
// solver vectors (a few MB, reused every phase) stay resident.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes,
                                          unsigned long long *m) {
  unsigned long long policy;
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

// Bounded wait on an mbarrier phase; returns false (and flags the solve) if
// the copy did not complete within the limit.
__device__ __forceinline__ bool mbar_wait(unsigned long long *m, unsigned parity, int *control) {
  const unsigned a = smem_addr(m);
  for (unsigned spin = 0; spin < (1u << 26); ++spin) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  atomicCAS(control, 0, FFG_TIMEOUT);
  return false;
}

template <typename VT>
__device__ __forceinline__ void issue_tile(const PcgParams &P, const VT *val, int t, TileBuf &b,
                                           unsigned long long *m) {
  const int r0 = P.tile_row[t], r1 = P.tile_row[t + 1];
  const int64_t a0 = P.rp[r0] & ~(int64_t)3;
  const int64_t a1 = (P.rp[r1] + 3) & ~(int64_t)3;
  const unsigned n = (unsigned)(a1 - a0);
  const unsigned cb = n * 4u, vb = n * (unsigned)sizeof(VT);
  mbar_expect(m, cb + vb);
  bulk_load(b.col, P.col + a0, cb, m);
  bulk_load(b.val, val + a0, vb, m);
}

// Tile SpMV: for every row r of this CTA's tiles, epi(r, sum_k A_rk gather(c_k)).
// Rows are summed by groups of 4 lanes in a fixed order (lane-strided partial
// sums, then a butterfly); lane 0 of the group applies the epilogue.
template <typename VT, typename AT, class G, class Epi>
__device__ __forceinline__ void spmv_tiles(const PcgParams &P, const VT *__restrict__ val,
                                           StageSmem &S, unsigned &parity_bits, G gather,
                                           Epi epi) {
  const int first = blockIdx.x;
  if (first >= P.n_tiles) return;
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    issue_tile<VT>(P, val, first, S.buf[0], &S.mbar[0]);
  }
  int slot = 0;
  for (int t = first; t < P.n_tiles; t += gridDim.x, slot ^= 1) {
    const int nt = t + gridDim.x;
    if (threadIdx.x == 0 && nt < P.n_tiles) {
      // the other buffer was last read before the trailing __syncthreads of the
      // previous tile; order those generic accesses before the async copy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue_tile<VT>(P, val, nt, S.buf[slot ^ 1], &S.mbar[slot ^ 1]);
    }
    TileBuf &B = S.buf[slot];
    const bool arrived = mbar_wait(&S.mbar[slot], (parity_bits >> slot) & 1u, P.control);
    parity_bits ^= (1u << slot);
    // a copy that never completed leaves the buffer undefined: its column
    // indices are not dereferenced (the solve already reports FFG_TIMEOUT)
    if (!__syncthreads_and(arrived)) continue;
    const int r0 = P.tile_row[t], r1 = P.tile_row[t + 1];
    const int64_t e0 = P.rp[r0], e1 = P.rp[r1];
    const int64_t a0 = e0 & ~(int64_t)3;
    const int lo = (int)(e0 - a0), hi = (int)(e1 - a0);
    const VT *sv = reinterpret_cast<const VT *>(B.val);
    AT *prod = reinterpret_cast<AT *>(B.val);
#pragma unroll 4
    for (int k = lo + threadIdx.x; k < hi; k += kThreads) {
      const AT a = (AT)sv[k];
      prod[k] = a * gather(B.col[k]);
    }
    __syncthreads();
    const int g = threadIdx.x >> 2, j = threadIdx.x & 3;
    for (int base = r0; base < r1; base += kThreads / 4) {
      const int row = base + g;
      AT s = 0;
      if (row < r1) {
        const int k0 = (int)(P.rp[row] - a0), k1 = (int)(P.rp[row + 1] - a0);
        for (int k = k0 + j; k < k1; k += 4) s += prod[k];
      }
      s += __shfl_xor_sync(0xffffffffu, s, 1);
      s += __shfl_xor_sync(0xffffffffu, s, 2);
      if (row < r1 && j == 0) epi(row, s);
    }
    __syncthreads();
  }
}

template <class F>
__device__ __forceinline__ void for_rows(const PcgParams &P, F f) {
  for (int t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
    const int r0 = P.tile_row[t], r1 = P.tile_row[t + 1];
    for (int r = r0 + threadIdx.x; r < r1; r += kThreads) f(r);
  }
}

__device__ __forceinline__ bool is_finite_d(double x) { return isfinite(x); }

template <typename V>
struct VecOf;
template <>
struct VecOf<float> {
  using V2 = float2;
};
template <>
struct VecOf<double> {
  using V2 = double2;
};

struct Outcome {
  int iterations = 0, updates = 0, converged = 0, status = FFG_OK, stagnated = 0, aborted = 0;
  double true_res = 0.0, final_res = 0.0, bnorm = 0.0;
};

// Device time of the phases seen by CTA 0 (the others are symmetric):
// SpMV work, wait at the following barrier, vector work, wait, and the
// reliable-update phases.
struct Timing {
  unsigned long long a = 0, aw = 0, b = 0, bw = 0, u = 0;
};

__device__ __forceinline__ unsigned long long stamp() {
  return (blockIdx.x == 0 && threadIdx.x == 0) ? globaltimer() : 0ull;
}

// The CG loop in value type V (float: mixed mode, double: FP64 mode).
// `continuation` runs the FP64 loop after a stagnated mixed solve: its target
// is the true residual tol*||b|| and its guard is the SPD one.
template <typename V>
__device__ __noinline__ void cg(const PcgParams &P, StageSmem &S, unsigned int &phase, unsigned &parity_bits,
                   unsigned long long t_start, bool continuation, Outcome &o, Timing &tm) {
  using V2 = typename VecOf<V>::V2;
  constexpr bool kMixed = sizeof(V) == 4;
  const V *A = kMixed ? (const V *)P.v32 : (const V *)P.v64;
  const V *dinv = kMixed ? (const V *)P.d32 : (const V *)P.d64;
  V *r = kMixed ? (V *)P.rf : (V *)P.rd;
  V *q = kMixed ? (V *)P.qf : (V *)P.qd;
  V2 *zp[2] = {kMixed ? (V2 *)P.zpf0 : (V2 *)P.zpd0, kMixed ? (V2 *)P.zpf1 : (V2 *)P.zpd1};
  double part[kSlots], red[kSlots];
  const bool true_target = kMixed || continuation;
  unsigned long long t0, t1, t2;

  // r64 = b - A x, ||r64||, ||b||
  t0 = stamp();
  part[0] = part[1] = 0.0;
  spmv_tiles<double, double>(P, P.v64, S, parity_bits, [&](int c) { return P.x[c]; },
                             [&](int row, double s) {
                               const double bb = P.b[row];
                               const double rr = bb - s;
                               P.r64[row] = rr;
                               part[0] += rr * rr;
                               part[1] += bb * bb;
                             });
  write_partials(P, phase, part, 2);
  if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
  read_partials(P, phase, red, 2);
  const double bnorm = sqrt(red[1]);
  const double rnorm = sqrt(red[0]);
  o.bnorm = bnorm;
  double scale = kMixed ? (rnorm > 0.0 ? rnorm : 1.0) : 1.0;
  const double target = P.relative ? P.tol * (true_target ? bnorm : rnorm) : P.tol;
  double true_res = rnorm, last_true = rnorm;
  int stall = 0;
  int converged = (rnorm <= target) ? 1 : 0;
  double rz = 0.0;
  if (!converged) {
    const double inv = 1.0 / scale;
    part[0] = 0.0;
    for_rows(P, [&](int row) {
      const V rr = (V)(P.r64[row] * inv);
      const V z = dinv[row] * rr;
      r[row] = rr;
      zp[0][row] = V2{z, (V)0};
      part[0] += (double)rr * (double)z;
    });
    write_partials(P, phase, part, 1);
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 1);
    rz = red[0];
  }
  tm.u += stamp() - t0;
  double beta = 0.0, rr_last = 1.0;
  int cur = 0;
  const int budget = P.max_it - o.iterations;
  for (int it = 1; !converged && it <= budget; ++it) {
    const V2 *zc = zp[cur];
    V2 *zn = zp[cur ^ 1];
    const V bt = (V)beta;
    // A: p = z + beta p_old, q = A p, (p, q)
    t0 = stamp();
    part[0] = 0.0;
    spmv_tiles<V, V>(P, A, S, parity_bits,
                     [&](int c) {
                       const V2 a = zc[c];
                       return a.x + bt * a.y;
                     },
                     [&](int row, V s) {
                       const V2 a = zc[row];
                       const V pn = a.x + bt * a.y;
                       zn[row].y = pn;
                       q[row] = s;
                       part[0] += (double)pn * (double)s;
                     });
    write_partials(P, phase, part, 1);
    t1 = stamp();
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 1);
    t2 = stamp();
    tm.a += t1 - t0;
    tm.aw += t2 - t1;
    const double pAp = red[0];
    const bool breakdown = (!kMixed && !continuation && P.guard == 0)
                               ? (fabs(pAp) < 1.0e-14)
                               : !(pAp > 0.0 && is_finite_d(pAp));
    if (breakdown) break;
    const double alpha = rz / pAp;
    const V al = (V)alpha;
    const double xs = alpha * scale;
    // B: x += alpha p (FP64), r -= alpha q, z = D^-1 r
    t0 = stamp();
    part[0] = part[1] = 0.0;
    part[2] = (blockIdx.x == 0 && threadIdx.x == 0 && globaltimer() - t_start > P.limit_ns) ? 1.0 : 0.0;
    for_rows(P, [&](int row) {
      const V pn = zn[row].y;
      P.x[row] = P.x[row] + xs * (double)pn;
      const V rr = r[row] - al * q[row];
      r[row] = rr;
      const V z = dinv[row] * rr;
      zn[row].x = z;
      part[0] += (double)rr * (double)rr;
      part[1] += (double)rr * (double)z;
    });
    write_partials(P, phase, part, 3);
    t1 = stamp();
    if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
    read_partials(P, phase, red, 3);
    t2 = stamp();
    tm.b += t1 - t0;
    tm.bw += t2 - t1;
    ++o.iterations;
    double rr = red[0], rz_new = red[1];
    const double est = sqrt(rr) * scale;
    if (red[2] != 0.0) { o.status = FFG_TIMEOUT; true_res = est; break; }
    if (!kMixed) {
      true_res = est;
      if (est <= target) { converged = 1; break; }
    } else if (est <= target || rr <= P.delta * P.delta * rr_last) {
      // reliable update: replace the recursive residual with b - A x in FP64
      if (o.updates >= P.max_updates) break;
      ++o.updates;
      t0 = stamp();
      part[0] = 0.0;
      spmv_tiles<double, double>(P, P.v64, S, parity_bits, [&](int c) { return P.x[c]; },
                                 [&](int row, double s) {
                                   const double v = P.b[row] - s;
                                   P.r64[row] = v;
                                   part[0] += v * v;
                                 });
      write_partials(P, phase, part, 1);
      if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
      read_partials(P, phase, red, 1);
      true_res = sqrt(red[0]);
      if (true_res <= target) { converged = 1; tm.u += stamp() - t0; break; }
      if (!(true_res > 0.0) || !is_finite_d(true_res)) break;
      // FP32 recurrences that no longer reduce the true residual (condition
      // number beyond FP32 reach) hand the solve to the FP64 loop
      stall = (true_res > 0.5 * last_true) ? stall + 1 : 0;
      last_true = true_res;
      if (stall >= 2) { o.stagnated = 1; tm.u += stamp() - t0; break; }
      const double ratio = scale / true_res;  // old units -> new units
      const V rt = (V)ratio;
      const double inv = 1.0 / true_res;
      part[0] = 0.0;
      for_rows(P, [&](int row) {
        const V rr2 = (V)(P.r64[row] * inv);
        r[row] = rr2;
        const V z = dinv[row] * rr2;
        V2 a = zn[row];
        a.x = z;
        a.y = a.y * rt;
        zn[row] = a;
        part[0] += (double)rr2 * (double)z;
      });
      write_partials(P, phase, part, 1);
      if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
      read_partials(P, phase, red, 1);
      tm.u += stamp() - t0;
      rz = rz * ratio * ratio;
      rz_new = red[0];
      scale = true_res;
      rr_last = 1.0;
    }
    beta = rz_new / rz;
    rz = rz_new;
    cur ^= 1;
  }
  o.converged = converged;
  o.final_res = true_res;
  if (kMixed && converged) {
    o.true_res = true_res;
    return;
  }
  if (kMixed && o.stagnated) return;  // the FP64 continuation measures its own residual
  // true FP64 residual of the returned x
  t0 = stamp();
  part[0] = 0.0;
  spmv_tiles<double, double>(P, P.v64, S, parity_bits, [&](int c) { return P.x[c]; },
                             [&](int row, double s) {
                               const double v = P.b[row] - s;
                               part[0] += v * v;
                             });
  write_partials(P, phase, part, 1);
  if (!grid_barrier(P, phase)) { o.aborted = 1; return; }
  read_partials(P, phase, red, 1);
  tm.u += stamp() - t0;
  o.true_res = sqrt(red[0]);
  if (kMixed) o.final_res = o.true_res;
}

__global__ void __launch_bounds__(kThreads, 2) pcg_kernel(PcgParams P) {
  extern __shared__ __align__(128) unsigned char dyn[];
  StageSmem &S = *reinterpret_cast<StageSmem *>(dyn);
  if (threadIdx.x == 0) {
    mbar_init(&S.mbar[0]);
    mbar_init(&S.mbar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned int phase = 0;
  unsigned parity_bits = 0;
  // only block 0 judges the wall limit; its verdict travels through a partial slot
  const unsigned long long t_start = globaltimer();
  Outcome o;
  Timing tm;
  int continued = 0;
  if (P.precision == FFG_PRECISION_FP64) {
    cg<double>(P, S, phase, parity_bits, t_start, false, o, tm);
  } else {
    cg<float>(P, S, phase, parity_bits, t_start, false, o, tm);
    if (!o.aborted && o.stagnated && !o.converged && o.status == FFG_OK) {
      continued = 1;
      cg<double>(P, S, phase, parity_bits, t_start, true, o, tm);
    }
  }
  if (o.aborted) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
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

// Standalone FP64 tile SpMV (one CTA per tile).
__global__ void __launch_bounds__(kThreads) spmv64_kernel(int64_t n, const int64_t *rp,
                                                          const int *col, const double *val,
                                                          const int *tile_row, int n_tiles,
                                                          const double *x, double *y) {
  __shared__ double sm[kTileNnz];
  const int t = blockIdx.x;
  if (t >= n_tiles) return;
  const int r0 = tile_row[t], r1 = tile_row[t + 1];
  const int64_t e0 = rp[r0];
  const int E = (int)(rp[r1] - e0);
  for (int k = threadIdx.x; k < E; k += kThreads) sm[k] = val[e0 + k] * x[col[e0 + k]];
  __syncthreads();
  for (int r = r0 + threadIdx.x; r < r1; r += kThreads) {
    const int k0 = (int)(rp[r] - e0), k1 = (int)(rp[r + 1] - e0);
    double s = 0.0;
    for (int k = k0; k < k1; ++k) s += sm[k];
    y[r] = s;
  }
}

}  // namespace

int tile_capacity() { return kTileNnz; }
int matrix_padding() { return 8; }

int pcg_grid_size(int *grid) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FFG_CUDA_ERROR;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (cudaFuncSetAttribute(pcg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(StageSmem)) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel, kThreads,
                                                    sizeof(StageSmem)) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (per_sm < 1) return FFG_CUDA_ERROR;
  *grid = sms * std::min(per_sm, 2);
  return FFG_OK;
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
  A((void **)&w.qf, N * sizeof(float));
  A((void **)&w.zpf0, N * sizeof(float2));
  A((void **)&w.zpf1, N * sizeof(float2));
  A((void **)&w.partial, 2 * kSlots * (size_t)grid * sizeof(double));
  A((void **)&w.barrier, 64);
  A((void **)&w.control, 64);
  A((void **)&w.result, kResultDoubles * sizeof(double));
  if (bad) {
    solve_work_free(w);
    cudaGetLastError();
    return FFG_OUT_OF_MEMORY;
  }
  return FFG_OK;
}

void solve_work_free(SolveWork &w) {
  void *ptrs[] = {w.r64, w.rd, w.qd, w.zpd0, w.zpd1, w.rf, w.qf, w.zpf0, w.zpf1, w.partial,
                  w.barrier, w.control, w.result};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  w = SolveWork();
}

int pcg_solve(const DeviceCsr &A, const double *b, double *x, const ffg_solver_options &opts,
              SolveWork &w, ffg_solver_stats *stats, cudaStream_t stream, std::string &msg) {
  if (w.n != A.n || w.grid <= 0) { msg = "solver workspace mismatch"; return FFG_INVALID_INPUT; }
  PcgParams P;
  P.n = A.n;
  P.rp = A.row_ptr;
  P.col = A.col;
  P.v32 = A.val32;
  P.v64 = A.val64;
  P.d32 = A.dinv32;
  P.d64 = A.dinv64;
  P.tile_row = A.tile_row;
  P.n_tiles = A.n_tiles;
  P.b = b;
  P.x = x;
  P.r64 = w.r64;
  P.rf = w.rf; P.qf = w.qf; P.zpf0 = w.zpf0; P.zpf1 = w.zpf1;
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
  const double limit = opts.timeout_seconds > 0 ? opts.timeout_seconds : 60.0;
  P.limit_ns = (unsigned long long)(limit * 1e9);
  if (cudaMemsetAsync(w.barrier, 0, 64, stream) != cudaSuccess) return FFG_CUDA_ERROR;
  if (cudaMemsetAsync(w.control, 0, 64, stream) != cudaSuccess) return FFG_CUDA_ERROR;
  void *args[] = {&P};
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)pcg_kernel, dim3(w.grid),
                                              dim3(kThreads), args, sizeof(StageSmem), stream);
  if (e != cudaSuccess) {
    msg = std::string("cooperative launch failed: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return FFG_CUDA_ERROR;
  }
  double res[kResultDoubles];
  int ctrl[2];
  if (cudaMemcpyAsync(res, w.result, sizeof(res), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (cudaMemcpyAsync(ctrl, w.control, sizeof(ctrl), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (cudaStreamSynchronize(stream) != cudaSuccess) return FFG_CUDA_ERROR;
  if (ctrl[0] != 0) {
    msg = "grid barrier timed out";
    if (stats) stats->status = ctrl[0];
    return ctrl[0];
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

int spmv64(const DeviceCsr &A, const double *x, double *y, cudaStream_t stream) {
  if (A.n_tiles == 0) return FFG_OK;
  spmv64_kernel<<<A.n_tiles, kThreads, 0, stream>>>(A.n, A.row_ptr, A.col, A.val64, A.tile_row,
                                                    A.n_tiles, x, y);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace ffg
