// Tensor-weighted first-kind Nedelec curl-curl + mass
// (assemble_tetra_nedelec_weighted_csc, src/assembly/assembly_tetra_nedelec_3d.f90:1870-2000,
// elements :2406-2514).
//
// The element matrix is sum_q det w_q (curl_i . M curl_j + m v_i . v_j).  With
// a cellwise-constant symmetric tensor M and curl_i = J c_i / det,
// v_i = J^-T r_i this is the Nedelec reference-tensor contraction with the
// twelve weights
//   curl pair (a,b):  (1/det) (J^T M J)_ab,
//   mass pair (a,b):  m det (J^-1 J^-T)_ab,
// which this kernel writes per cell; the Nedelec element kernel then runs on
// them (caller weights) with the usual orientation transform, and the column
// kernel gathers the result.  The scalar curl / mass coefficients and their
// per-cell factors multiply the tensor and the mass term.
#include <cuda_runtime.h>

#include "ffg_internal.h"
#include "tet_geometry.h"

namespace ffg {

namespace {

__global__ void weighted_weights_kernel(int n_cells, const int *__restrict__ cells,
                                        const double *__restrict__ verts, double ca, double cb,
                                        const double *__restrict__ cell_a,
                                        const double *__restrict__ cell_b,
                                        const double *__restrict__ tensor,
                                        double *__restrict__ geo, int *err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  double *g = geo + 12 * (size_t)c;
  double J[9], Ji[9], v0[3];
  tet_jacobian(cells, verts, c, J, v0);
  const double det = det3(J);
  if (!valid_jacobian(J, det)) {
    // the element kernel reports the cell; its weights stay finite
    for (int s = 0; s < 12; ++s) g[s] = 0.0;
    atomicCAS(err, 0, FFG_INVALID_INPUT);
    return;
  }
  inv3(J, det, Ji);
  const double cw = ca * (cell_a ? cell_a[c] : 1.0);
  const double mw = cb * (cell_b ? cell_b[c] : 1.0);
  const double *M = tensor + 9 * (size_t)c;  // column-major M(r, e) = M[r + 3e]
  // symmetric pair order shared with basis.cpp: (0,0),(1,1),(2,2),(0,1),(0,2),(1,2)
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  for (int s = 0; s < 6; ++s) {
    const int a = pa[s], b = pb[s];
    double curl = 0.0, mass = 0.0;
    for (int r = 0; r < 3; ++r) {
      // (J^T M J)_ab = sum_re J(r,a) M(r,e) J(e,b); (J^-1 J^-T)_ab = sum_r Ji(a,r) Ji(b,r)
      const double ma = J[r + 3 * a];
      for (int e = 0; e < 3; ++e) curl += ma * M[r + 3 * e] * J[e + 3 * b];
      mass += Ji[a + 3 * r] * Ji[b + 3 * r];
    }
    g[s] = cw * curl / det;
    g[6 + s] = mw * det * mass;
  }
}

}  // namespace

int launch_weighted_weights(const Topology &t, const DeviceTopology &dt, const AssemblyInputs &in,
                            const double *tensor, double *geo, int *err, cudaStream_t s) {
  if (t.family != FFG_TETRA_NEDELEC || !tensor || !geo || !in.vertices) return FFG_INVALID_INPUT;
  if (t.n_cells == 0) return FFG_OK;
  weighted_weights_kernel<<<(unsigned)((t.n_cells + 127) / 128), 128, 0, s>>>(
      (int)t.n_cells, dt.cells, in.vertices, in.coef_a, in.coef_b, in.cell_a, in.cell_b, tensor,
      geo, err);
  return cudaGetLastError() == cudaSuccess ? FFG_OK : FFG_CUDA_ERROR;
}

}  // namespace ffg
