// Allocation-free Jacobi-PCG for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc or cudaFree: codes
// that claim all of a GPU's memory at start-up for their own arena (a Fortran
// or MPI application that hands out pieces of one block, so any further
// allocation fails), and time-stepping loops that share the GPU with work on
// other streams, where cudaFree would synchronise the whole device at every
// solve.  For them ffg_solve_csr_device_noalloc solves an SPD system held in
// caller-owned device memory with the FP64 Jacobi-PCG of solve_sparse,
// keeping every work vector in one file-scope device array of fixed size.
//
// The array is found once per device: the first call made with a device
// current looks up its address there (cudaGetSymbolAddress) and caches it, so
// that first call should come before any stream capture.  The array is shared
// by all calls on a device and keeps the last call's contents; the kernel
// writes every value before it reads it.  Calls whose kernels overlap on the
// same GPU race on the array, so callers serialise them (one stream, or
// events).  Every GPU the library runs on holds the array (about 2.6 MB)
// until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "ffg_internal.h"

namespace ffg {
namespace {

constexpr int kNoAllocMaxRows = FFG_NOALLOC_MAX_ROWS;  // largest system the array holds
constexpr int kNoAllocThreads = 1024;   // one CTA solves the whole system
constexpr int kNoAllocWarps = kNoAllocThreads / 32;
constexpr int kNoAllocResult = 8;  // converged, iterations, res, true res, timeout, seconds, bad input
// layout (doubles): r, z, p, q, D^-1 (kNoAllocMaxRows each), then the result block
constexpr size_t kNoAllocDoubles = 5 * (size_t)kNoAllocMaxRows + kNoAllocResult;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// CTA-wide sum in a fixed order (warp butterflies, then warps in order).
__device__ double cta_sum(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < kNoAllocWarps; ++w) t += red[w];
  __syncthreads();
  return t;
}

// y = A x for a CSR matrix: one warp per row, lanes over the row's entries,
// summed in a fixed order.
__device__ void csr_apply(int n, const int64_t *rp, const int *ci, const double *v,
                          const double *x, double *y) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = warp; i < n; i += kNoAllocWarps) {
    double s = 0.0;
    for (int64_t k = rp[i] + lane; k < rp[i + 1]; k += 32) s += v[k] * x[ci[k]];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[i] = s;
  }
  __syncthreads();
}

// pcg_solve_operator / pcg_iteration_loop (src/solvers/advanced_solvers.f90:831-925)
// in one CTA; jacobi diagonal as build_sparse_preconditioner (:1139-1154).
__global__ void __launch_bounds__(kNoAllocThreads, 1)
    noalloc_pcg_kernel(int n, int64_t nnz, const int64_t *rp, const int *ci, const double *v,
                       const double *b, double *x, double *scratch, int jacobi, int relative,
                       double tol, int max_it, int guard, unsigned long long limit_ns) {
  __shared__ double red[kNoAllocWarps];
  __shared__ int stop;
  double *r = scratch, *z = r + kNoAllocMaxRows, *p = z + kNoAllocMaxRows;
  double *q = p + kNoAllocMaxRows, *dinv = q + kNoAllocMaxRows;
  double *result = dinv + kNoAllocMaxRows;
  const unsigned long long t0 = now_ns();
  // The CSR arrays come from the caller: check them before any indexed access
  // (row_ptr starts at 0, ends at nnz and never decreases; every column index
  // is a row of the system), so that a malformed matrix is reported, not read
  // out of bounds.  The column indices are read only once row_ptr has passed.
  int bad = 0;
  if (threadIdx.x == 0) bad = (rp[0] != 0 || rp[n] != nnz) ? 1 : 0;
  for (int i = threadIdx.x; i < n; i += kNoAllocThreads) bad |= rp[i] > rp[i + 1] ? 1 : 0;
  if (__syncthreads_or(bad) == 0) {
    for (int64_t k = threadIdx.x; k < nnz; k += kNoAllocThreads)
      bad |= (ci[k] < 0 || ci[k] >= n) ? 1 : 0;
    bad = __syncthreads_or(bad);
  } else {
    bad = 1;
  }
  if (bad) {
    if (threadIdx.x == 0) {
      for (int i = 0; i < 6; ++i) result[i] = 0.0;
      result[6] = 1.0;
    }
    return;
  }
  for (int i = threadIdx.x; i < n; i += kNoAllocThreads) {
    double d = 0.0;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) { d = v[k]; break; }
    dinv[i] = (jacobi && fabs(d) > 1.0e-14) ? 1.0 / d : 1.0;
  }
  __syncthreads();
  csr_apply(n, rp, ci, v, x, q);  // q = A x0
  double rr = 0.0, rz = 0.0;
  for (int i = threadIdx.x; i < n; i += kNoAllocThreads) {
    const double ri = b[i] - q[i];
    const double zi = dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    rr += ri * ri;
    rz += ri * zi;
  }
  const double initial = sqrt(cta_sum(rr, red));
  double rz_old = cta_sum(rz, red);
  const double target = relative ? tol * initial : tol;
  double res = initial;
  int iterations = 0, converged = res <= target ? 1 : 0, timed_out = 0;
  for (int it = 1; !converged && it <= max_it; ++it) {
    csr_apply(n, rp, ci, v, p, q);
    double pq = 0.0;
    for (int i = threadIdx.x; i < n; i += kNoAllocThreads) pq += p[i] * q[i];
    const double pAp = cta_sum(pq, red);
    if (guard == 0 ? fabs(pAp) < 1.0e-14 : !(pAp > 0.0 && isfinite(pAp))) break;
    const double alpha = rz_old / pAp;
    double s_rr = 0.0, s_rz = 0.0;
    for (int i = threadIdx.x; i < n; i += kNoAllocThreads) {
      x[i] = x[i] + alpha * p[i];
      const double ri = r[i] - alpha * q[i];
      const double zi = dinv[i] * ri;
      r[i] = ri;
      z[i] = zi;
      s_rr += ri * ri;
      s_rz += ri * zi;
    }
    res = sqrt(cta_sum(s_rr, red));
    const double rz_new = cta_sum(s_rz, red);
    iterations = it;
    if (res <= target) { converged = 1; break; }
    if (threadIdx.x == 0) stop = (now_ns() - t0 > limit_ns) ? 1 : 0;
    __syncthreads();
    if (stop) { timed_out = 1; break; }
    const double beta = rz_new / rz_old;
    for (int i = threadIdx.x; i < n; i += kNoAllocThreads) p[i] = z[i] + beta * p[i];
    rz_old = rz_new;
    __syncthreads();
  }
  // true residual of the returned x
  __syncthreads();
  csr_apply(n, rp, ci, v, x, q);
  double tr = 0.0, bb = 0.0;
  for (int i = threadIdx.x; i < n; i += kNoAllocThreads) {
    const double d = b[i] - q[i];
    tr += d * d;
    bb += b[i] * b[i];
  }
  const double true_res = sqrt(cta_sum(tr, red));
  const double bnorm = sqrt(cta_sum(bb, red));
  if (threadIdx.x == 0) {
    result[0] = converged;
    result[1] = iterations;
    result[2] = res;
    result[3] = bnorm > 0.0 ? true_res / bnorm : true_res;
    result[4] = timed_out;
    result[5] = 1e-9 * (double)(now_ns() - t0);
    result[6] = 0.0;
  }
}

std::mutex g_noalloc_mutex;
constexpr int kMaxDevices = 64;
double *g_noalloc_address[kMaxDevices] = {nullptr};

// Device address of the scratch array for the current device.  In host code
// the symbol g_noalloc_scratch is only a host-side stand-in; the device
// address is obtained once per device (with that device current) and cached.
int noalloc_scratch_address(double **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return FFG_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_address[dev]) {
    double *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      cudaGetLastError();
      return FFG_CUDA_ERROR;
    }
    g_noalloc_address[dev] = ptr;
  }
  *out = g_noalloc_address[dev];
  return FFG_OK;
}

}  // namespace
}  // namespace ffg

using namespace ffg;

extern "C" void ffg_solve_csr_device_noalloc(int n, int64_t nnz, const int64_t *row_ptr,
                                             const int *col_ind, const double *values,
                                             const double *b, double *x,
                                             const ffg_solver_options *opts,
                                             ffg_solver_stats *stats, void *stream, int *status) {
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (n < 1 || nnz < 0 || !row_ptr || !col_ind || !values || !b || !x) {
    *status = FFG_INVALID_INPUT;
    return;
  }
  if (n > kNoAllocMaxRows) {
    std::fprintf(stderr,
                 "ffg_solve_csr_device_noalloc: %d rows exceed the %d-row scratch array\n", n,
                 kNoAllocMaxRows);
    *status = FFG_CAPACITY;
    return;
  }
  // solver_options_t fields as ffg_solve_sparse reads them; precision is ignored
  // (always FP64) and so are the mixed-mode fields
  ffg_solver_options o;
  ffg_default_options(&o);
  if (opts) {
    if (opts->version != FFG_OPTIONS_VERSION || opts->tolerance < 0 ||
        opts->max_iterations < 0) {
      *status = FFG_INVALID_INPUT;
      return;
    }
    o = *opts;
  }
  // wall limit in ns; clamped to a million seconds so that the conversion
  // below stays inside the range of unsigned long long
  const double limit = std::fmin(o.timeout_seconds > 0 ? o.timeout_seconds : 60.0, 1.0e6);
  double *scratch = nullptr;
  int st = noalloc_scratch_address(&scratch);
  if (st) { *status = st; return; }
  cudaStream_t s = (cudaStream_t)stream;
  noalloc_pcg_kernel<<<1, kNoAllocThreads, 0, s>>>(n, nnz, row_ptr, col_ind, values, b, x, scratch,
                                                   o.preconditioner != 0, o.tolerance_type == 0,
                                                   o.tolerance, o.max_iterations, o.breakdown_guard,
                                                   (unsigned long long)(limit * 1e9));
  if (cudaGetLastError() != cudaSuccess) { *status = FFG_CUDA_ERROR; return; }
  double res[kNoAllocResult];
  const double *dres = scratch + 5 * (size_t)kNoAllocMaxRows;
  if (cudaMemcpyAsync(res, dres, sizeof(double) * 7, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    *status = FFG_CUDA_ERROR;
    return;
  }
  if (res[6] != 0.0) {
    std::fprintf(stderr,
                 "ffg_solve_csr_device_noalloc: malformed CSR matrix (row_ptr must run from 0 "
                 "to nnz without decreasing, column indices must lie in [0, n))\n");
    if (stats) stats->status = FFG_INVALID_INPUT;
    *status = FFG_INVALID_INPUT;
    return;
  }
  if (stats) {
    stats->converged = (int)res[0];
    stats->iterations = (int)res[1];
    stats->final_residual = res[2];
    stats->true_relative_residual = res[3];
    stats->solve_seconds = res[5];
    stats->status = res[4] != 0.0 ? FFG_TIMEOUT : (res[0] != 0.0 ? FFG_OK : FFG_NOT_CONVERGED);
  }
  *status = res[4] != 0.0 ? FFG_TIMEOUT : (res[0] != 0.0 ? FFG_OK : FFG_NOT_CONVERGED);
}
