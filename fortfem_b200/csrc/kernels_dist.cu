// Kernels of the row-block (sharded) Jacobi-PCG of one system over several
// GPUs: the operator SpMV on a problem's SELL layout, fused vector updates
// with dot products over the rows a rank owns, and the halo gather/scatter.
// The iteration loop, the halo exchange and the scalar all-reduces run on
// the host (fortfem_b200/sharding.py) between these launches.
//
// Dot products are deterministic: a fixed grid of kDotBlocks blocks writes
// per-block partials in a fixed order and one block sums them in order.
#include <cuda_runtime.h>

#include "ffg_internal.h"

namespace ffg {

namespace {

constexpr int kDotBlocks = 256;
constexpr int kDotThreads = 256;

__device__ __forceinline__ double block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  __syncthreads();
  return s;  // valid on thread 0
}

// y = A x on the SELL layout (FP64 values), one warp per 32-row slice.
template <bool NARROW>
__global__ void sell_spmv64_kernel(int64_t n, int64_t n_slices, const int64_t *__restrict__ soff,
                                   const int16_t *__restrict__ dcol, const int *__restrict__ col,
                                   const double *__restrict__ val, const double *__restrict__ x,
                                   double *__restrict__ y) {
  const int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (s >= n_slices) return;
  const int64_t row = s * 32 + lane;
  const int64_t base = soff[s] + lane;
  const int len = (int)((soff[s + 1] - soff[s]) / 32);
  double acc = 0.0;
  for (int j = 0; j < len; ++j) {
    const int64_t k = base + (int64_t)j * 32;
    const int64_t c = NARROW ? row + dcol[k] : col[k];
    acc += val[k] * x[c];
  }
  if (row < n) y[row] = acc;
}

// x += alpha p, r -= alpha q, z = D^-1 r on owned rows; partials of
// (r, r) and (r, z) over owned rows.
__global__ void update_kernel(int64_t n, const uint8_t *__restrict__ owned, double alpha,
                              const double *__restrict__ p, const double *__restrict__ q,
                              const double *__restrict__ dinv, double *__restrict__ x,
                              double *__restrict__ r, double *__restrict__ z,
                              double *__restrict__ partial) {
  __shared__ double red[kDotThreads / 32];
  double rr = 0.0, rz = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!owned[i]) continue;
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * q[i];
    const double zi = dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    rr += ri * ri;
    rz += ri * zi;
  }
  const double a = block_sum(rr, red), b = block_sum(rz, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = a;
    partial[kDotBlocks + blockIdx.x] = b;
  }
}

// r = b - Ax, z = D^-1 r, p = z on owned rows; partials of (r, r), (r, z), (b, b).
__global__ void start_kernel(int64_t n, const uint8_t *__restrict__ owned,
                             const double *__restrict__ b, const double *__restrict__ ax,
                             const double *__restrict__ dinv, double *__restrict__ r,
                             double *__restrict__ z, double *__restrict__ p,
                             double *__restrict__ partial) {
  __shared__ double red[kDotThreads / 32];
  double rr = 0.0, rz = 0.0, bb = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!owned[i]) continue;
    const double ri = b[i] - ax[i];
    const double zi = dinv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    rr += ri * ri;
    rz += ri * zi;
    bb += b[i] * b[i];
  }
  const double s0 = block_sum(rr, red), s1 = block_sum(rz, red), s2 = block_sum(bb, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = s0;
    partial[kDotBlocks + blockIdx.x] = s1;
    partial[2 * kDotBlocks + blockIdx.x] = s2;
  }
}

__global__ void dot_kernel(int64_t n, const uint8_t *__restrict__ owned,
                           const double *__restrict__ a, const double *__restrict__ b,
                           double *__restrict__ partial) {
  __shared__ double red[kDotThreads / 32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (owned[i]) s += a[i] * b[i];
  const double t = block_sum(s, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// Single-reduction PCG (Chronopoulos-Gear): partials of (r, z), (w, z) and
// (r, r) over owned rows, w = A z.
__global__ void cgs_dots_kernel(int64_t n, const uint8_t *__restrict__ owned,
                                const double *__restrict__ r, const double *__restrict__ z,
                                const double *__restrict__ w, double *__restrict__ partial) {
  __shared__ double red[kDotThreads / 32];
  double rz = 0.0, wz = 0.0, rr = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!owned[i]) continue;
    rz += r[i] * z[i];
    wz += w[i] * z[i];
    rr += r[i] * r[i];
  }
  const double a = block_sum(rz, red), b = block_sum(wz, red), c = block_sum(rr, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = a;
    partial[kDotBlocks + blockIdx.x] = b;
    partial[2 * kDotBlocks + blockIdx.x] = c;
  }
}

// p = z + beta p, s = w + beta s (s = A p by recurrence), x += alpha p,
// r -= alpha s, z = D^-1 r on owned rows.
__global__ void cgs_update_kernel(int64_t n, const uint8_t *__restrict__ owned, double alpha,
                                  double beta, const double *__restrict__ w,
                                  const double *__restrict__ dinv, double *__restrict__ p,
                                  double *__restrict__ s, double *__restrict__ x,
                                  double *__restrict__ r, double *__restrict__ z) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !owned[i]) return;
  const double pi = z[i] + beta * p[i];
  const double si = w[i] + beta * s[i];
  p[i] = pi;
  s[i] = si;
  x[i] += alpha * pi;
  const double ri = r[i] - alpha * si;
  r[i] = ri;
  z[i] = dinv[i] * ri;
}

// out[k] = sum of the kDotBlocks partials of slot k, in block order.
__global__ void finish_kernel(int nslot, const double *__restrict__ partial,
                              double *__restrict__ out) {
  if (threadIdx.x < nslot) {
    double s = 0.0;
    for (int b = 0; b < kDotBlocks; ++b) s += partial[threadIdx.x * kDotBlocks + b];
    out[threadIdx.x] = s;
  }
}

__global__ void direction_kernel(int64_t n, const uint8_t *__restrict__ owned, double beta,
                                 const double *__restrict__ z, double *__restrict__ p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && owned[i]) p[i] = z[i] + beta * p[i];
}

__global__ void gather_kernel(int64_t m, const int *__restrict__ idx,
                              const double *__restrict__ src, double *__restrict__ dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) dst[i] = src[idx[i]];
}

__global__ void scatter_kernel(int64_t m, const int *__restrict__ idx,
                               const double *__restrict__ src, double *__restrict__ dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) dst[idx[i]] = src[i];
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

inline int launched() { return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR; }

}  // namespace

int sell_spmv64(const DeviceSell &A, const double *x, double *y, cudaStream_t s) {
  if (A.n_slices == 0) return FFG_OK;
  const unsigned grid = blocks_for(A.n_slices * 32, 256);
  if (A.dcol)
    sell_spmv64_kernel<true><<<grid, 256, 0, s>>>(A.n, A.n_slices, A.soff, A.dcol, A.col,
                                                  A.val64, x, y);
  else
    sell_spmv64_kernel<false><<<grid, 256, 0, s>>>(A.n, A.n_slices, A.soff, A.dcol, A.col,
                                                   A.val64, x, y);
  return launched();
}

}  // namespace ffg

extern "C" {

using namespace ffg;

void ffg_dist_start(int64_t n, const uint8_t *owned, const double *b, const double *ax,
                    const double *dinv, double *r, double *z, double *p, double *work,
                    double *dots, void *stream, int *status) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || !work || !dots) { *status = FFG_INVALID_INPUT; return; }
  start_kernel<<<kDotBlocks, kDotThreads, 0, s>>>(n, owned, b, ax, dinv, r, z, p, work);
  finish_kernel<<<1, 32, 0, s>>>(3, work, dots);
  *status = launched();
}

void ffg_dist_update(int64_t n, const uint8_t *owned, double alpha, const double *p,
                     const double *q, const double *dinv, double *x, double *r, double *z,
                     double *work, double *dots, void *stream, int *status) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || !work || !dots) { *status = FFG_INVALID_INPUT; return; }
  update_kernel<<<kDotBlocks, kDotThreads, 0, s>>>(n, owned, alpha, p, q, dinv, x, r, z, work);
  finish_kernel<<<1, 32, 0, s>>>(2, work, dots);
  *status = launched();
}

void ffg_dist_dot(int64_t n, const uint8_t *owned, const double *a, const double *b,
                  double *work, double *dot, void *stream, int *status) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || !work || !dot) { *status = FFG_INVALID_INPUT; return; }
  dot_kernel<<<kDotBlocks, kDotThreads, 0, s>>>(n, owned, a, b, work);
  finish_kernel<<<1, 32, 0, s>>>(1, work, dot);
  *status = launched();
}

void ffg_dist_cgs_dots(int64_t n, const uint8_t *owned, const double *r, const double *z,
                       const double *w, double *work, double *dots, void *stream, int *status) {
  cudaStream_t s = (cudaStream_t)stream;
  if (n < 0 || !work || !dots) { *status = FFG_INVALID_INPUT; return; }
  cgs_dots_kernel<<<kDotBlocks, kDotThreads, 0, s>>>(n, owned, r, z, w, work);
  finish_kernel<<<1, 32, 0, s>>>(3, work, dots);
  *status = launched();
}

void ffg_dist_cgs_update(int64_t n, const uint8_t *owned, double alpha, double beta,
                         const double *w, const double *dinv, double *p, double *s, double *x,
                         double *r, double *z, void *stream, int *status) {
  if (n < 0) { *status = FFG_INVALID_INPUT; return; }
  if (n > 0)
    cgs_update_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        n, owned, alpha, beta, w, dinv, p, s, x, r, z);
  *status = launched();
}

void ffg_dist_direction(int64_t n, const uint8_t *owned, double beta, const double *z, double *p,
                        void *stream, int *status) {
  if (n < 0) { *status = FFG_INVALID_INPUT; return; }
  if (n > 0)
    direction_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, owned, beta, z, p);
  *status = launched();
}

void ffg_dist_gather(int64_t m, const int *idx, const double *src, double *dst, void *stream,
                     int *status) {
  if (m < 0) { *status = FFG_INVALID_INPUT; return; }
  if (m > 0) gather_kernel<<<blocks_for(m, 256), 256, 0, (cudaStream_t)stream>>>(m, idx, src, dst);
  *status = launched();
}

void ffg_dist_scatter(int64_t m, const int *idx, const double *src, double *dst, void *stream,
                      int *status) {
  if (m < 0) { *status = FFG_INVALID_INPUT; return; }
  if (m > 0) scatter_kernel<<<blocks_for(m, 256), 256, 0, (cudaStream_t)stream>>>(m, idx, src, dst);
  *status = launched();
}

}  // extern "C"
