// Complex PML forms of the first-kind Nedelec curl-curl operator
// (assemble_tetra_nedelec_pml_csc, src/assembly/assembly_tetra_nedelec_3d.f90:1613-1685,
// element :826-887; assemble_tetra_nedelec_curvilinear_pml_csc :1372-1444,
// element :1092-1153).
//
// The element matrix is sum_q w det (curl_i . Cc curl_j - k^2 v_i . Cm v_j)
// with complex symmetric per-cell tensors Cc, Cm.  With curl_i = J c_i / det
// and v_i = J^-T r_i this is the real Nedelec contraction with complex
// weights:
//   curl pair (a,b):  (1/det) (J^T Cc J)_ab,
//   mass pair (a,b):  -k^2 det (J^-1 Cm J^-T)_ab,
// so the complex matrix is the real element kernel run once on the real
// parts of the weights and once on the imaginary parts (the orientation
// transform is real), each gathered into the CSC by the primal column kernel.
#include <cuda_runtime.h>

#include <cfloat>

#include "ffg_internal.h"
#include "tet_geometry.h"

namespace ffg {

namespace {

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx cscale(double s, cplx a) { return {s * a.re, s * a.im}; }
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
__device__ __forceinline__ double cabs(cplx a) { return hypot(a.re, a.im); }
__device__ __forceinline__ bool cfinite(cplx a) { return isfinite(a.re) && isfinite(a.im); }

// cartesian_curl_curl_pml_coefficients (src/boundary/cartesian_helmholtz_pml.f90:94-108):
// Cm = diag(s2 s3 / s1, s1 s3 / s2, s1 s2 / s3), Cc = Cm^-1 (elementwise).
__device__ bool cartesian_tensors(const cplx *s, cplx *Cc, cplx *Cm) {
  for (int a = 0; a < 3; ++a)
    if (cabs(s[a]) <= DBL_MIN) return false;
  for (int i = 0; i < 9; ++i) Cc[i] = Cm[i] = {0.0, 0.0};
  Cm[0] = cdiv(cmul(s[1], s[2]), s[0]);
  Cm[4] = cdiv(cmul(s[0], s[2]), s[1]);
  Cm[8] = cdiv(cmul(s[0], s[1]), s[2]);
  for (int a = 0; a < 3; ++a) Cc[4 * a] = cdiv({1.0, 0.0}, Cm[4 * a]);
  return true;
}

// curvilinear_curl_curl_pml_coefficients (src/boundary/curvilinear_helmholtz_pml.f90:113-131)
// with inverse_and_determinant (:202-216): Cc = S^T S / det S, Cm = det S S^-1 S^-T.
__device__ bool curvilinear_tensors(const cplx *S, cplx *Cc, cplx *Cm) {
  auto m = [&](int r, int c) { return S[r + 3 * c]; };
  const cplx det =
      cadd(csub(cmul(m(0, 0), csub(cmul(m(1, 1), m(2, 2)), cmul(m(1, 2), m(2, 1)))),
                cmul(m(0, 1), csub(cmul(m(1, 0), m(2, 2)), cmul(m(1, 2), m(2, 0))))),
           cmul(m(0, 2), csub(cmul(m(1, 0), m(2, 1)), cmul(m(1, 1), m(2, 0)))));
  double mx = 0.0;
  for (int i = 0; i < 9; ++i) {
    if (!cfinite(S[i])) return false;
    mx = fmax(mx, cabs(S[i]));
  }
  if (!cfinite(det)) return false;
  const double sc = fmax(1.0, mx);
  if (cabs(det) <= 64.0 * kEps * sc * sc * sc) return false;
  cplx inv[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
      // inverse = transpose(cofactor) / det
      inv[c + 3 * r] = cdiv(csub(cmul(m(r1, c1), m(r2, c2)), cmul(m(r1, c2), m(r2, c1))), det);
    }
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      cplx a = {0.0, 0.0}, b = {0.0, 0.0};
      for (int q = 0; q < 3; ++q) {
        a = cadd(a, cmul(S[q + 3 * r], S[q + 3 * c]));
        b = cadd(b, cmul(inv[r + 3 * q], inv[c + 3 * q]));
      }
      Cc[r + 3 * c] = cdiv(a, det);
      Cm[r + 3 * c] = cmul(det, b);
    }
  return true;
}

__global__ void pml_weights_kernel(int n_cells, const int *__restrict__ cells,
                                   const double *__restrict__ verts,
                                   const double *__restrict__ stretch, int curvilinear,
                                   double wave, double *__restrict__ geo_re,
                                   double *__restrict__ geo_im, int *err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  double *gr = geo_re + 12 * (size_t)c, *gi = geo_im + 12 * (size_t)c;
  for (int s = 0; s < 12; ++s) gr[s] = gi[s] = 0.0;
  double J[9], Ji[9], v0[3];
  tet_jacobian(cells, verts, c, J, v0);
  const double det = det3(J);
  if (!valid_jacobian(J, det)) {
    atomicCAS(err, 0, FFG_INVALID_INPUT);
    return;
  }
  inv3(J, det, Ji);
  const int sw = curvilinear ? 9 : 3;
  cplx S[9], Cc[9], Cm[9];
  for (int i = 0; i < sw; ++i)
    S[i] = {stretch[2 * (sw * (size_t)c + i)], stretch[2 * (sw * (size_t)c + i) + 1]};
  if (!(curvilinear ? curvilinear_tensors(S, Cc, Cm) : cartesian_tensors(S, Cc, Cm))) {
    atomicCAS(err, 0, FFG_INVALID_INPUT);
    return;
  }
  // symmetric pair order shared with basis.cpp: (0,0),(1,1),(2,2),(0,1),(0,2),(1,2)
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  const double k2 = wave * wave;
  for (int s = 0; s < 6; ++s) {
    const int a = pa[s], b = pb[s];
    cplx curl = {0.0, 0.0}, mass = {0.0, 0.0};
    for (int r = 0; r < 3; ++r)
      for (int e = 0; e < 3; ++e) {
        // (J^T Cc J)_ab = sum J(r,a) Cc(r,e) J(e,b); (J^-1 Cm J^-T)_ab = sum Ji(a,r) Cm(r,e) Ji(b,e)
        curl = cadd(curl, cscale(J[r + 3 * a] * J[e + 3 * b], Cc[r + 3 * e]));
        mass = cadd(mass, cscale(Ji[a + 3 * r] * Ji[b + 3 * e], Cm[r + 3 * e]));
      }
    gr[s] = curl.re / det;
    gi[s] = curl.im / det;
    gr[6 + s] = -k2 * det * mass.re;
    gi[6 + s] = -k2 * det * mass.im;
  }
}

__global__ void interleave_kernel(int64_t n, const double *__restrict__ re,
                                  const double *__restrict__ im, double *__restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) reinterpret_cast<double2 *>(out)[i] = make_double2(re[i], im[i]);
}

inline int blocks_for(int64_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

int launch_pml_weights(const Topology &t, const DeviceTopology &dt, const double *vertices,
                       const double *stretch, bool curvilinear, double wave_number,
                       double *geo_re, double *geo_im, int *err, cudaStream_t s) {
  if (t.family != FFG_TETRA_NEDELEC || !(wave_number > 0.0)) return FFG_INVALID_INPUT;
  pml_weights_kernel<<<blocks_for(t.n_cells, 128), 128, 0, s>>>(
      t.n_cells, dt.cells, vertices, stretch, curvilinear ? 1 : 0, wave_number, geo_re, geo_im,
      err);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

int launch_interleave(int64_t n, const double *re, const double *im, double *values,
                      cudaStream_t s) {
  if (n <= 0) return FFG_OK;
  interleave_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, re, im, values);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace ffg
