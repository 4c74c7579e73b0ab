// Device helpers of the tetrahedral geometry shared by the assembly kernels:
// the affine map's Jacobian J (columns v1-v0, v2-v0, v3-v0, column-major
// J[r + 3c]), its determinant and inverse by cofactors, and the reference's
// degenerate-cell test.
#pragma once

#include <cuda_runtime.h>

namespace ffg {
namespace {

constexpr double kEps = 2.220446049250313e-16;

__device__ __forceinline__ double det3(const double *J) {
  return J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
         J[6] * (J[1] * J[5] - J[4] * J[2]);
}

__device__ __forceinline__ void inv3(const double *J, double det, double *Ji) {
  const double r = 1.0 / det;
  Ji[0] = (J[4] * J[8] - J[7] * J[5]) * r;
  Ji[3] = -(J[3] * J[8] - J[6] * J[5]) * r;
  Ji[6] = (J[3] * J[7] - J[6] * J[4]) * r;
  Ji[1] = -(J[1] * J[8] - J[7] * J[2]) * r;
  Ji[4] = (J[0] * J[8] - J[6] * J[2]) * r;
  Ji[7] = -(J[0] * J[7] - J[6] * J[1]) * r;
  Ji[2] = (J[1] * J[5] - J[4] * J[2]) * r;
  Ji[5] = -(J[0] * J[5] - J[3] * J[2]) * r;
  Ji[8] = (J[0] * J[4] - J[3] * J[1]) * r;
}

// valid_jacobian (assembly_tetra_lagrange_arbitrary_order_3d.f90:65-66, 796-802)
__device__ __forceinline__ bool valid_jacobian(const double *J, double det) {
  double m = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) m = fmax(m, fabs(J[i]));
  const double s = fmax(1.0, m);
  return det > 64.0 * kEps * s * s * s;
}

__device__ __forceinline__ void tet_jacobian(const int *cells, const double *verts, int c,
                                             double *J, double *v0) {
  const int4 t = *reinterpret_cast<const int4 *>(cells + 4 * (size_t)c);
  const double *p0 = verts + 3 * (size_t)t.x;
  const double *p1 = verts + 3 * (size_t)t.y;
  const double *p2 = verts + 3 * (size_t)t.z;
  const double *p3 = verts + 3 * (size_t)t.w;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const double a = p0[r];
    v0[r] = a;
    J[r] = p1[r] - a;
    J[r + 3] = p2[r] - a;
    J[r + 6] = p3[r] - a;
  }
}

}  // namespace
}  // namespace ffg
