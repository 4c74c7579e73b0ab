// Persistent Jacobi-PCG (sm_100a).
//
// One cooperative launch runs the whole solve.  CTAs own fixed row tiles of
// the CSR matrix (the constrained CSC of a symmetric operator read as CSR);
// each SpMV streams the CTA's tiles with coalesced loads into shared memory
// and sums every row in a fixed order.  Dot products are reduced per CTA,
// written to a per-phase partial buffer and summed by every CTA in the same
// fixed order, so all CTAs take identical decisions and results are
// bit-reproducible for a given grid.  Grid barriers spin with a bound and
// report FFG_TIMEOUT instead of hanging.
//
// FP64 mode restates pcg_solve_operator / pcg_iteration_loop
// (src/solvers/advanced_solvers.f90:831-925): stop when the recursive residual
// ||r||_2 <= tol*||r_0||_2 (relative) or tol (absolute), or when
// |p^T A p| < 1e-14; Jacobi z = D^-1 r with D^-1 = 1 where |a_ii| <= 1e-14.
// Mixed mode: inner FP32 PCG on the scaled residual, outer FP64 iterative
// refinement on the true residual b - A x until ||b - A x|| <= tol*||b||.
#include <cuda_runtime.h>

#include <cstdio>

#include "ffg_internal.h"

namespace ffg {

namespace {

constexpr int kThreads = 256;
constexpr int kTileNnz = 4096;
constexpr int kSlots = 4;
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
  float *xf, *rf, *zf, *pf, *apf;
  double *pd, *apd, *zd;
  double *partial;  // [2][kSlots][grid]
  unsigned int *bar;
  int *control;     // [0] error status
  double *result;   // 8 doubles
  int precision, relative, max_it, max_ref, guard;
  double tol, inner_tol;
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
      __nanosleep(32);
    }
    __threadfence();
    ok = good && ld_volatile_int(P.control) == 0;
  }
  __syncthreads();
  return ok != 0;
}

// CTA-wide sum of per-thread values for kSlots slots, written to the partial
// buffer of this phase parity.
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
__device__ void read_partials(const PcgParams &P, unsigned int phase, double *out, int nslot) {
  __shared__ double res[kSlots];
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    for (int s = 0; s < nslot; ++s) {
      const double *src = P.partial + ((size_t)(phase & 1) * kSlots + s) * gridDim.x;
      double x = 0.0;
      for (int b = lane; b < (int)gridDim.x; b += 32) x += __ldcg(src + b);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) res[s] = x;
    }
  }
  __syncthreads();
  for (int s = 0; s < nslot; ++s) out[s] = res[s];
  __syncthreads();
}

// Tile SpMV: for every row r of this CTA's tiles, epi(r, sum_k A_rk x_k).
template <typename VT, typename AT, typename XT, class Epi>
__device__ __forceinline__ void spmv_tiles(const PcgParams &P, const VT *__restrict__ val,
                                           const XT *x, AT *smem, Epi epi) {
  for (int t = blockIdx.x; t < P.n_tiles; t += gridDim.x) {
    const int r0 = P.tile_row[t], r1 = P.tile_row[t + 1];
    const int64_t e0 = P.rp[r0];
    const int E = (int)(P.rp[r1] - e0);
    const VT *vv = val + e0;
    const int *cc = P.col + e0;
#pragma unroll 4
    for (int k = threadIdx.x; k < E; k += kThreads) {
      const VT a = __ldcs(vv + k);
      const int c = __ldcs(cc + k);
      smem[k] = (AT)a * (AT)x[c];
    }
    __syncthreads();
    for (int r = r0 + threadIdx.x; r < r1; r += kThreads) {
      const int k0 = (int)(P.rp[r] - e0), k1 = (int)(P.rp[r + 1] - e0);
      AT s = 0;
      for (int k = k0; k < k1; ++k) s += smem[k];
      epi(r, s);
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

__global__ void __launch_bounds__(kThreads, 2) pcg_kernel(PcgParams P) {
  __shared__ __align__(16) double smem_d[kTileNnz];
  float *smem_f = reinterpret_cast<float *>(smem_d);
  unsigned int phase = 0;
  // only block 0 judges the wall limit; its verdict travels through a partial slot
  const unsigned long long t_start = globaltimer();
  double part[kSlots];
  double red[kSlots];
  int iterations = 0, refinements = 0, converged = 0, status = FFG_OK;
  double final_res = 0.0, true_rel = 0.0;

  // ||b||
  part[0] = 0.0;
  for_rows(P, [&](int r) { const double v = P.b[r]; part[0] += v * v; });
  write_partials(P, phase, part, 1);
  if (!grid_barrier(P, phase)) return;
  read_partials(P, phase, red, 1);
  const double bnorm = sqrt(red[0]);

  if (P.precision == FFG_PRECISION_FP64) {
    // r = b - A x ; z = D^-1 r ; p = z
    part[0] = part[1] = part[2] = 0.0;
    spmv_tiles<double, double, double>(P, P.v64, P.x, smem_d, [&](int r, double s) {
      const double rr = P.b[r] - s;
      const double z = P.d64[r] * rr;
      P.r64[r] = rr;
      P.zd[r] = z;
      P.pd[r] = z;
      part[0] += rr * rr;
      part[1] += rr * z;
    });
    write_partials(P, phase, part, 2);
    if (!grid_barrier(P, phase)) return;
    read_partials(P, phase, red, 2);
    const double initial = sqrt(red[0]);
    double res = initial, rz_old = red[1];
    const double tol = P.relative ? P.tol * initial : P.tol;
    for (int it = 1; it <= P.max_it; ++it) {
      part[0] = 0.0;
      spmv_tiles<double, double, double>(P, P.v64, P.pd, smem_d, [&](int r, double s) {
        P.apd[r] = s;
        part[0] += P.pd[r] * s;
      });
      write_partials(P, phase, part, 1);
      if (!grid_barrier(P, phase)) return;
      read_partials(P, phase, red, 1);
      const double pAp = red[0];
      if (P.guard == 0 ? fabs(pAp) < 1.0e-14 : !(pAp > 0.0 && is_finite_d(pAp))) break;
      const double alpha = rz_old / pAp;
      part[0] = part[1] = 0.0;
      part[2] = (blockIdx.x == 0 && threadIdx.x == 0 && globaltimer() - t_start > P.limit_ns) ? 1.0 : 0.0;
      for_rows(P, [&](int r) {
        P.x[r] = P.x[r] + alpha * P.pd[r];
        const double rr = P.r64[r] - alpha * P.apd[r];
        P.r64[r] = rr;
        const double z = P.d64[r] * rr;
        P.zd[r] = z;
        part[0] += rr * rr;
        part[1] += rr * z;
      });
      write_partials(P, phase, part, 3);
      if (!grid_barrier(P, phase)) return;
      read_partials(P, phase, red, 3);
      res = sqrt(red[0]);
      iterations = it;
      if (res <= tol) { converged = 1; break; }
      if (red[2] != 0.0) { status = FFG_TIMEOUT; break; }
      const double beta = red[1] / rz_old;
      rz_old = red[1];
      for_rows(P, [&](int r) { P.pd[r] = P.zd[r] + beta * P.pd[r]; });
      if (!grid_barrier(P, phase)) return;
    }
    if (!converged && res <= tol) converged = 1;
    final_res = res;
  } else {
    // mixed precision: outer FP64 refinement, inner FP32 PCG
    const double target = P.relative ? P.tol * bnorm : P.tol;
    int total_it = 0;
    double rnorm = 0.0;
    for (int outer = 0;; ++outer) {
      part[0] = 0.0;
      spmv_tiles<double, double, double>(P, P.v64, P.x, smem_d, [&](int r, double s) {
        const double rr = P.b[r] - s;
        P.r64[r] = rr;
        part[0] += rr * rr;
      });
      part[1] = (blockIdx.x == 0 && threadIdx.x == 0 && globaltimer() - t_start > P.limit_ns) ? 1.0 : 0.0;
      write_partials(P, phase, part, 2);
      if (!grid_barrier(P, phase)) return;
      read_partials(P, phase, red, 2);
      rnorm = sqrt(red[0]);
      final_res = rnorm;
      if (rnorm <= target) { converged = 1; break; }
      if (outer >= P.max_ref || total_it >= P.max_it) break;
      if (red[1] != 0.0) { status = FFG_TIMEOUT; break; }
      if (!is_finite_d(rnorm)) break;
      const double scale = 1.0 / rnorm;
      part[0] = part[1] = 0.0;
      for_rows(P, [&](int r) {
        const float rr = (float)(P.r64[r] * scale);
        const float z = P.d32[r] * rr;
        P.rf[r] = rr;
        P.xf[r] = 0.0f;
        P.zf[r] = z;
        P.pf[r] = z;
        part[0] += (double)rr * (double)z;
        part[1] += (double)rr * (double)rr;
      });
      write_partials(P, phase, part, 2);
      if (!grid_barrier(P, phase)) return;
      read_partials(P, phase, red, 2);
      double rz = red[0];
      const double rr0 = red[1];
      const double inner_target = P.inner_tol * P.inner_tol * rr0;
      while (total_it < P.max_it) {
        part[0] = 0.0;
        spmv_tiles<float, float, float>(P, P.v32, P.pf, smem_f, [&](int r, float s) {
          P.apf[r] = s;
          part[0] += (double)P.pf[r] * (double)s;
        });
        write_partials(P, phase, part, 1);
        if (!grid_barrier(P, phase)) return;
        read_partials(P, phase, red, 1);
        const double pAp = red[0];
        if (!(pAp > 0.0) || !is_finite_d(pAp)) break;
        const float alpha = (float)(rz / pAp);
        part[0] = part[1] = 0.0;
        part[2] = (blockIdx.x == 0 && threadIdx.x == 0 && globaltimer() - t_start > P.limit_ns) ? 1.0 : 0.0;
        for_rows(P, [&](int r) {
          P.xf[r] = P.xf[r] + alpha * P.pf[r];
          const float rr = P.rf[r] - alpha * P.apf[r];
          P.rf[r] = rr;
          const float z = P.d32[r] * rr;
          P.zf[r] = z;
          part[0] += (double)rr * (double)z;
          part[1] += (double)rr * (double)rr;
        });
        write_partials(P, phase, part, 3);
        if (!grid_barrier(P, phase)) return;
        read_partials(P, phase, red, 3);
        ++total_it;
        if (red[1] <= inner_target || red[2] != 0.0) break;
        const float beta = (float)(red[0] / rz);
        rz = red[0];
        for_rows(P, [&](int r) { P.pf[r] = P.zf[r] + beta * P.pf[r]; });
        if (!grid_barrier(P, phase)) return;
      }
      for_rows(P, [&](int r) { P.x[r] = P.x[r] + rnorm * (double)P.xf[r]; });
      if (!grid_barrier(P, phase)) return;
      refinements = outer + 1;
    }
    iterations = total_it;
    true_rel = bnorm > 0.0 ? rnorm / bnorm : rnorm;
  }

  if (P.precision == FFG_PRECISION_FP64) {
    // true FP64 residual of the returned x
    part[0] = 0.0;
    spmv_tiles<double, double, double>(P, P.v64, P.x, smem_d, [&](int r, double s) {
      const double rr = P.b[r] - s;
      part[0] += rr * rr;
    });
    write_partials(P, phase, part, 1);
    if (!grid_barrier(P, phase)) return;
    read_partials(P, phase, red, 1);
    true_rel = bnorm > 0.0 ? sqrt(red[0]) / bnorm : sqrt(red[0]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.result[0] = converged;
    P.result[1] = iterations;
    P.result[2] = refinements;
    P.result[3] = final_res;
    P.result[4] = true_rel;
    P.result[5] = status;
    P.result[6] = bnorm;
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

int pcg_grid_size(int *grid) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FFG_CUDA_ERROR;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return FFG_CUDA_ERROR;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel, kThreads, 0) !=
      cudaSuccess)
    return FFG_CUDA_ERROR;
  if (per_sm < 1) return FFG_CUDA_ERROR;
  *grid = sms * per_sm;
  return FFG_OK;
}

int solve_work_alloc(SolveWork &w, int64_t n, int grid) {
  solve_work_free(w);
  w.n = n;
  w.grid = grid;
  const size_t N = (size_t)std::max<int64_t>(n, 1);
  cudaError_t e = cudaSuccess;
  e = (cudaError_t)(e | cudaMalloc(&w.r64, N * sizeof(double)));
  e = (cudaError_t)(e | cudaMalloc(&w.pd, N * sizeof(double)));
  e = (cudaError_t)(e | cudaMalloc(&w.apd, N * sizeof(double)));
  e = (cudaError_t)(e | cudaMalloc(&w.zd, N * sizeof(double)));
  e = (cudaError_t)(e | cudaMalloc(&w.xf, N * sizeof(float)));
  e = (cudaError_t)(e | cudaMalloc(&w.rf, N * sizeof(float)));
  e = (cudaError_t)(e | cudaMalloc(&w.zf, N * sizeof(float)));
  e = (cudaError_t)(e | cudaMalloc(&w.pf, N * sizeof(float)));
  e = (cudaError_t)(e | cudaMalloc(&w.apf, N * sizeof(float)));
  e = (cudaError_t)(e | cudaMalloc(&w.partial, 2 * kSlots * (size_t)grid * sizeof(double)));
  e = (cudaError_t)(e | cudaMalloc(&w.barrier, 64));
  e = (cudaError_t)(e | cudaMalloc(&w.control, 64));
  e = (cudaError_t)(e | cudaMalloc(&w.result, 8 * sizeof(double)));
  if (e != cudaSuccess) {
    solve_work_free(w);
    cudaGetLastError();
    return FFG_OUT_OF_MEMORY;
  }
  return FFG_OK;
}

void solve_work_free(SolveWork &w) {
  void *ptrs[] = {w.r64, w.pd, w.apd, w.zd, w.xf, w.rf, w.zf, w.pf, w.apf, w.partial,
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
  P.xf = w.xf; P.rf = w.rf; P.zf = w.zf; P.pf = w.pf; P.apf = w.apf;
  P.pd = w.pd; P.apd = w.apd; P.zd = w.zd;
  P.partial = w.partial;
  P.bar = w.barrier;
  P.control = w.control;
  P.result = w.result;
  P.precision = opts.precision;
  P.relative = opts.tolerance_type == 0;
  P.max_it = opts.max_iterations;
  P.max_ref = opts.max_refinements;
  P.tol = opts.tolerance;
  P.inner_tol = opts.inner_tolerance;
  P.guard = opts.breakdown_guard;
  const double limit = opts.timeout_seconds > 0 ? opts.timeout_seconds : 60.0;
  P.limit_ns = (unsigned long long)(limit * 1e9);
  if (cudaMemsetAsync(w.barrier, 0, 64, stream) != cudaSuccess) return FFG_CUDA_ERROR;
  if (cudaMemsetAsync(w.control, 0, 64, stream) != cudaSuccess) return FFG_CUDA_ERROR;
  void *args[] = {&P};
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)pcg_kernel, dim3(w.grid), dim3(kThreads),
                                              args, 0, stream);
  if (e != cudaSuccess) {
    msg = std::string("cooperative launch failed: ") + cudaGetErrorString(e);
    return FFG_CUDA_ERROR;
  }
  double res[8];
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
  return FFG_OK;
}

int spmv64(const DeviceCsr &A, const double *x, double *y, cudaStream_t stream) {
  if (A.n_tiles == 0) return FFG_OK;
  spmv64_kernel<<<A.n_tiles, kThreads, 0, stream>>>(A.n, A.row_ptr, A.col, A.val64, A.tile_row,
                                                    A.n_tiles, x, y);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

int tile_capacity() { return kTileNnz; }

}  // namespace ffg
