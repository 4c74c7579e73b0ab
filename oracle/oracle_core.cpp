// fortfem hot-path ORACLE (test infrastructure only; see oracle.h).
//
// FP64 CPU restatement of quadrature, meshes, tetrahedral Lagrange assembly,
// P1 triangle forms, triplet->CSC, constrained reduction and Jacobi-PCG.
// Loop orders and summation orders follow the cited reference routines so the
// results reproduce the reference's arithmetic up to the unpinned rounding of
// its third-party det3/inv3/gauss_legendre_ab helpers.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <unordered_map>
#include <vector>

namespace {

const double kEps = 2.220446049250313e-16;  // epsilon(1.0_dp)

// fortnum det3 / inv3 restated by cofactor expansion (fortnum @3920109d, called
// at src/assembly/assembly_tetra_lagrange_arbitrary_order_3d.f90:64,67).
// J is column-major: J[r + 3*c].
double det3(const double *J) {
  return J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
         J[6] * (J[1] * J[5] - J[4] * J[2]);
}

void inv3(const double *J, double det, double *Ji) {
  // inverse = adjugate / det, column-major.
  Ji[0] = (J[4] * J[8] - J[7] * J[5]) / det;
  Ji[3] = -(J[3] * J[8] - J[6] * J[5]) / det;
  Ji[6] = (J[3] * J[7] - J[6] * J[4]) / det;
  Ji[1] = -(J[1] * J[8] - J[7] * J[2]) / det;
  Ji[4] = (J[0] * J[8] - J[6] * J[2]) / det;
  Ji[7] = -(J[0] * J[7] - J[6] * J[1]) / det;
  Ji[2] = (J[1] * J[5] - J[4] * J[2]) / det;
  Ji[5] = -(J[0] * J[5] - J[3] * J[2]) / det;
  Ji[8] = (J[0] * J[4] - J[3] * J[1]) / det;
}

void tetra_jacobian(const double *v, double *J) {
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) J[r + 3 * c] = v[r + 3 * (c + 1)] - v[r];
}

// valid_jacobian, assembly_tetra_lagrange_arbitrary_order_3d.f90:65-66,796-802
bool valid_jacobian(const double *J, double det) {
  double m = 0.0;
  for (int i = 0; i < 9; ++i) m = std::max(m, std::fabs(J[i]));
  double s = std::max(1.0, m);
  return det > 64.0 * kEps * s * s * s;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- quadrature
// Gauss-Legendre on [a,b] by Newton iteration on the three-term recurrence
// (restates fortnum gauss_legendre_ab, called at tetra_duffy_quadrature.f90:27-28).
int or_gauss_legendre(int n, double a, double b, double *nodes, double *weights) {
  if (n < 1) return 1;
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < n; ++i) {
    double x = std::cos(pi * (i + 0.75) / (n + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      double pn = (n == 1) ? x : p1;
      double pnm1 = (n == 1) ? 1.0 : p0;
      dp = n * (x * pn - pnm1) / (x * x - 1.0);
      double dx = pn / dp;
      x -= dx;
      if (std::fabs(dx) < 1e-17) break;
    }
    {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      double pn = (n == 1) ? x : p1;
      double pnm1 = (n == 1) ? 1.0 : p0;
      dp = n * (x * pn - pnm1) / (x * x - 1.0);
    }
    double w = 2.0 / ((1.0 - x * x) * dp * dp);
    // ascending order on [a, b]
    int j = n - 1 - i;
    nodes[j] = 0.5 * (b - a) * x + 0.5 * (b + a);
    weights[j] = 0.5 * (b - a) * w;
  }
  return 0;
}

int or_tetra_duffy_count(int q) {
  if (q < 0) return 0;
  int m = (q + 4) / 2;
  return m * m * m;
}

// src/quadrature/tetra_duffy_quadrature.f90:12-51
int or_tetra_duffy(int q, double *x, double *y, double *z, double *w) {
  if (q < 0) return 1;
  int m = (q + 4) / 2;
  std::vector<double> t(m), tw(m);
  or_gauss_legendre(m, 0.0, 1.0, t.data(), tw.data());
  int p = 0;
  for (int a = 0; a < m; ++a) {
    double c1 = 1.0 - t[a];
    for (int b = 0; b < m; ++b) {
      double c2 = 1.0 - t[b];
      for (int c = 0; c < m; ++c) {
        x[p] = t[a];
        y[p] = c1 * t[b];
        z[p] = c1 * c2 * t[c];
        w[p] = tw[a] * tw[b] * tw[c] * (c1 * c1) * c2;
        ++p;
      }
    }
  }
  return 0;
}

int or_triangle_duffy_count(int q) {
  if (q < 0) return 0;
  int m = (q + 3) / 2;
  return m * m;
}

// src/quadrature/triangle_duffy_quadrature.f90:12-45
int or_triangle_duffy(int q, double *x, double *y, double *w) {
  if (q < 0) return 1;
  int m = (q + 3) / 2;
  std::vector<double> t(m), tw(m);
  or_gauss_legendre(m, 0.0, 1.0, t.data(), tw.data());
  int p = 0;
  for (int a = 0; a < m; ++a)
    for (int b = 0; b < m; ++b) {
      x[p] = t[a];
      y[p] = (1.0 - t[a]) * t[b];
      w[p] = tw[a] * tw[b] * (1.0 - t[a]);
      ++p;
    }
  return 0;
}

// tetra_degree_two_quadrature, src/assembly/assembly_tetra_nedelec_3d.f90:2570-2581
void or_tetra_degree_two_rule(double *pts, double *wts) {
  const double a = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0;
  const double b = (5.0 - std::sqrt(5.0)) / 20.0;
  const double P[12] = {b, b, b, a, b, b, b, a, b, b, b, a};
  std::memcpy(pts, P, sizeof(P));
  for (int i = 0; i < 4; ++i) wts[i] = 1.0 / 24.0;
}

// -------------------------------------------------------------------- meshes
// src/mesh/structured_tetra_box_mesh.f90:12-94 (vertex_index :72-76,
// add_brick_tetrahedra :78-94, orientation swap :56-68).
int or_structured_tetra_box_mesh(const double *bounds, const int *counts, double *vertices,
                                 int *tets) {
  for (int d = 0; d < 3; ++d) {
    if (counts[d] < 1) return 1;
    if (bounds[3 + d] <= bounds[d]) return 1;
  }
  const int nx = counts[0], ny = counts[1], nz = counts[2];
  auto vid = [&](int i, int j, int k) { return i + (nx + 1) * (j + (ny + 1) * k); };
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        int v = vid(i, j, k);
        const int ijk[3] = {i, j, k};
        for (int d = 0; d < 3; ++d) {
          double c = (double)ijk[d] / (double)counts[d];
          vertices[3 * v + d] = bounds[d] + c * (bounds[3 + d] - bounds[d]);
        }
      }
  static const int local[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7},
                                  {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};
  int cell = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        int brick[8] = {vid(i, j, k),         vid(i + 1, j, k),         vid(i, j + 1, k),
                        vid(i + 1, j + 1, k), vid(i, j, k + 1),         vid(i + 1, j, k + 1),
                        vid(i, j + 1, k + 1), vid(i + 1, j + 1, k + 1)};
        for (int c = 0; c < 6; ++c, ++cell)
          for (int n = 0; n < 4; ++n) tets[4 * cell + n] = brick[local[c][n]];
      }
  for (int c = 0; c < cell; ++c) {
    double v[12];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = vertices[3 * tets[4 * c + n] + d];
    double J[9];
    tetra_jacobian(v, J);
    if (det3(J) < 0.0) std::swap(tets[4 * c + 2], tets[4 * c + 3]);
  }
  return 0;
}

// create_rectangular, src/mesh/mesh_2d.f90:90-148 (n vertices per side on
// [0,1]^2, unit_square_mesh at src/fortfem_api_mesh.f90:128-139).
int or_unit_square_mesh(int n, double *vertices, int *tris) {
  if (n < 2) return 1;
  double dx = 1.0 / (double)(n - 1);
  int k = 0;
  for (int j = 1; j <= n; ++j)
    for (int i = 1; i <= n; ++i, ++k) {
      vertices[2 * k] = 0.0 + (i - 1) * dx;
      vertices[2 * k + 1] = 0.0 + (j - 1) * dx;
    }
  k = 0;
  for (int j = 1; j <= n - 1; ++j)
    for (int i = 1; i <= n - 1; ++i) {
      int v1 = (j - 1) * n + i, v2 = (j - 1) * n + i + 1, v3 = j * n + i + 1, v4 = j * n + i;
      tris[3 * k] = v1 - 1; tris[3 * k + 1] = v2 - 1; tris[3 * k + 2] = v3 - 1; ++k;
      tris[3 * k] = v1 - 1; tris[3 * k + 1] = v3 - 1; tris[3 * k + 2] = v4 - 1; ++k;
    }
  return 0;
}

// find_boundary, src/mesh/mesh_2d.f90:560-603: an edge with exactly one
// incident triangle is a boundary edge; both its vertices are boundary vertices.
int or_square_boundary_vertices(int nv, int nt, const int *tris, uint8_t *is_boundary) {
  std::unordered_map<uint64_t, int> count;
  count.reserve((size_t)nt * 3);
  for (int t = 0; t < nt; ++t)
    for (int e = 0; e < 3; ++e) {
      uint32_t a = tris[3 * t + e], b = tris[3 * t + (e + 1) % 3];
      if (a > b) std::swap(a, b);
      count[((uint64_t)a << 32) | b] += 1;
    }
  std::memset(is_boundary, 0, nv);
  for (auto &kv : count)
    if (kv.second == 1) {
      is_boundary[kv.first >> 32] = 1;
      is_boundary[kv.first & 0xffffffffu] = 1;
    }
  return 0;
}

// ------------------------------------------------------- tetrahedral Lagrange
int or_lagrange_dof_count(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }

// initialize_tetra_lagrange, src/elements/tetra_lagrange_arbitrary_order.f90:29-66
int or_lagrange_barycentric_indices(int p, int *idx, double *nodes) {
  if (p < 0) return 1;
  if (p == 0) {
    for (int i = 0; i < 4; ++i) idx[i] = 0;
    if (nodes) nodes[0] = nodes[1] = nodes[2] = 0.25;
    return 0;
  }
  int dof = 0;
  for (int a = 0; a <= p; ++a)
    for (int b = 0; b <= p - a; ++b)
      for (int c = 0; c <= p - a - b; ++c, ++dof) {
        int d = p - a - b - c;
        idx[4 * dof] = a; idx[4 * dof + 1] = b; idx[4 * dof + 2] = c; idx[4 * dof + 3] = d;
        if (nodes) {
          nodes[3 * dof] = (double)b / p;
          nodes[3 * dof + 1] = (double)c / p;
          nodes[3 * dof + 2] = (double)d / p;
        }
      }
  return 0;
}

static double factorial_d(int n) {
  double v = 1.0;
  for (int f = 2; f <= n; ++f) v *= (double)f;
  return v;
}

// cardinal_factor, tetra_lagrange_arbitrary_order.f90:207-249 (value and first
// derivative).
static void cardinal_factor(int index, int degree, double lambda, double *value, double *deriv) {
  double v = 1.0;
  for (int f = 0; f <= index - 1; ++f) v = v * ((double)degree * lambda - (double)f);
  v = v / factorial_d(index);
  double d = 0.0;
  for (int df = 0; df <= index - 1; ++df) {
    double term = (double)degree;
    for (int f = 0; f <= index - 1; ++f)
      if (f != df) term = term * ((double)degree * lambda - (double)f);
    d = d + term;
  }
  d = d / factorial_d(index);
  *value = v;
  *deriv = d;
}

// evaluate_tetra_lagrange, tetra_lagrange_arbitrary_order.f90:68-116
int or_lagrange_evaluate(int p, const double *pt, double *values, double *gradients) {
  int nb = or_lagrange_dof_count(p);
  std::vector<int> idx(4 * nb);
  or_lagrange_barycentric_indices(p, idx.data(), nullptr);
  double bary[4] = {1.0 - (pt[0] + pt[1] + pt[2]), pt[0], pt[1], pt[2]};
  for (int i = 0; i < 4; ++i)
    if (bary[i] < -64.0 * kEps) return 1;
  for (int b = 0; b < nb; ++b) {
    double fac[4], der[4];
    for (int c = 0; c < 4; ++c) cardinal_factor(idx[4 * b + c], p, bary[c], &fac[c], &der[c]);
    double prod = 1.0;
    for (int c = 0; c < 4; ++c) prod *= fac[c];
    values[b] = prod;
    double ld[4];
    for (int c = 0; c < 4; ++c) {
      ld[c] = der[c];
      for (int o = 0; o < 4; ++o)
        if (o != c) ld[c] = ld[c] * fac[o];
    }
    for (int d = 0; d < 3; ++d) gradients[3 * b + d] = ld[d + 1] - ld[0];
  }
  return 0;
}

namespace {
struct LagKey {
  int v[4];
  int w[4];
  bool operator==(const LagKey &o) const {
    return std::memcmp(v, o.v, sizeof(v)) == 0 && std::memcmp(w, o.w, sizeof(w)) == 0;
  }
};
struct LagKeyHash {
  size_t operator()(const LagKey &k) const {
    uint64_t h = 1469598103934665603ull;
    for (int i = 0; i < 4; ++i) {
      h = (h ^ (uint64_t)(uint32_t)k.v[i]) * 1099511628211ull;
      h = (h ^ (uint64_t)(uint32_t)k.w[i]) * 1099511628211ull;
    }
    return (size_t)h;
  }
};

// sort_key, tetra_lagrange_global_dof_map.f90:81-99.  Vertices here are
// one-based (as in the reference) so that 0 keeps meaning "empty slot".
void sort_key(int *v, int *w) {
  for (int a = 0; a < 3; ++a)
    for (int b = a + 1; b < 4; ++b) {
      if (v[b] == 0) continue;
      if (v[a] != 0 && v[a] <= v[b]) continue;
      std::swap(v[a], v[b]);
      std::swap(w[a], w[b]);
    }
}

bool distinct_vertices(const int *t) {
  for (int a = 0; a < 4; ++a)
    for (int b = a + 1; b < 4; ++b)
      if (t[a] == t[b]) return false;
  return true;
}

LagKey make_key(const int *tet, const int *idx) {
  LagKey k;
  std::memset(&k, 0, sizeof(k));
  int e = 0;
  for (int c = 0; c < 4; ++c) {
    if (idx[c] == 0) continue;
    k.v[e] = tet[c] + 1;
    k.w[e] = idx[c];
    ++e;
  }
  sort_key(k.v, k.w);
  return k;
}
}  // namespace

// build_tetra_lagrange_dof_map, src/elements/tetra_lagrange_global_dof_map.f90:13-79,
// restated literally including its linear search over existing keys (:62-68).
int or_lagrange_dof_map_faithful(int p, int nt, const int *tets, int *gd, int *n_global) {
  if (p < 1 || p > 4) return 1;
  for (int c = 0; c < nt; ++c) {
    for (int i = 0; i < 4; ++i)
      if (tets[4 * c + i] < 0) return 1;
    if (!distinct_vertices(tets + 4 * c)) return 1;
  }
  int nb = or_lagrange_dof_count(p);
  std::vector<int> idx(4 * nb);
  or_lagrange_barycentric_indices(p, idx.data(), nullptr);
  std::vector<LagKey> keys;
  for (int c = 0; c < nt; ++c)
    for (int l = 0; l < nb; ++l) {
      LagKey k = make_key(tets + 4 * c, idx.data() + 4 * l);
      int found = -1;
      for (size_t e = 0; e < keys.size(); ++e)
        if (keys[e] == k) { found = (int)e; break; }
      if (found < 0) { keys.push_back(k); found = (int)keys.size() - 1; }
      gd[(size_t)nb * c + l] = found;
    }
  *n_global = (int)keys.size();
  return 0;
}

// Same numbering (first appearance in cell-major, local-DoF order) with a hash
// map in place of the linear search; proven identical by the tests.
int or_lagrange_dof_map(int p, int nt, const int *tets, int *gd, int *n_global) {
  if (p < 1 || p > 4) return 1;
  for (int c = 0; c < nt; ++c) {
    for (int i = 0; i < 4; ++i)
      if (tets[4 * c + i] < 0) return 1;
    if (!distinct_vertices(tets + 4 * c)) return 1;
  }
  int nb = or_lagrange_dof_count(p);
  std::vector<int> idx(4 * nb);
  or_lagrange_barycentric_indices(p, idx.data(), nullptr);
  std::unordered_map<LagKey, int, LagKeyHash> map;
  map.reserve((size_t)nt * nb / 2 + 16);
  int next = 0;
  for (int c = 0; c < nt; ++c)
    for (int l = 0; l < nb; ++l) {
      LagKey k = make_key(tets + 4 * c, idx.data() + 4 * l);
      auto it = map.find(k);
      int id;
      if (it == map.end()) { id = next++; map.emplace(k, id); } else id = it->second;
      gd[(size_t)nb * c + l] = id;
    }
  *n_global = next;
  return 0;
}

namespace {
struct Rule {
  std::vector<double> x, y, z, w;
};
bool make_rule(int rule, int q, Rule &r) {
  if (rule == 1) {
    double P[12], W[4];
    or_tetra_degree_two_rule(P, W);
    for (int i = 0; i < 4; ++i) {
      r.x.push_back(P[3 * i]); r.y.push_back(P[3 * i + 1]); r.z.push_back(P[3 * i + 2]);
      r.w.push_back(W[i]);
    }
    return true;
  }
  if (rule != 0 || q < 0) return false;
  int n = or_tetra_duffy_count(q);
  r.x.resize(n); r.y.resize(n); r.z.resize(n); r.w.resize(n);
  or_tetra_duffy(q, r.x.data(), r.y.data(), r.z.data(), r.w.data());
  return true;
}
}  // namespace

// assemble_tetra_lagrange_stiffness_element,
// src/assembly/assembly_tetra_lagrange_arbitrary_order_3d.f90:40-105
int or_lagrange_element(const double *v, int p, int rule, int q, double stiff, double mass,
                        double *M) {
  if (p < 1 || p > 4) return 1;
  double J[9], Ji[9];
  tetra_jacobian(v, J);
  double det = det3(J);
  if (!valid_jacobian(J, det)) return 1;
  inv3(J, det, Ji);
  Rule R;
  if (!make_rule(rule, q, R)) return 1;
  int nb = or_lagrange_dof_count(p);
  std::vector<double> val(nb), grad(3 * nb);
  std::fill(M, M + (size_t)nb * nb, 0.0);
  for (size_t pt = 0; pt < R.w.size(); ++pt) {
    double P[3] = {R.x[pt], R.y[pt], R.z[pt]};
    if (or_lagrange_evaluate(p, P, val.data(), grad.data())) return 1;
    double pw = det * R.w[pt];
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row) {
        double pr[3], pc[3];
        for (int i = 0; i < 3; ++i) {
          // matmul(transpose(inverse_jacobian), g): sum_k Ji(k,i) g(k)
          double s = 0.0, t = 0.0;
          for (int k = 0; k < 3; ++k) {
            s += Ji[k + 3 * i] * grad[3 * row + k];
            t += Ji[k + 3 * i] * grad[3 * col + k];
          }
          pr[i] = s;
          pc[i] = t;
        }
        double dotg = 0.0;
        for (int i = 0; i < 3; ++i) dotg += pr[i] * pc[i];
        M[row + (size_t)nb * col] += pw * (stiff * dotg + mass * val[row] * val[col]);
      }
  }
  return 0;
}

// -------------------------------------------------------------- triplet->CSC
// fortsparse csc_from_triplet (fortsparse @3c19c978, not vendored): sums
// duplicates; rows ascending within each column (the row order is not pinned by
// any reference test and is fixed here as ascending).  Duplicates are summed in
// triplet order.
int or_csc_from_triplet(int n_rows, int n_cols, int64_t nt, const int *rows, const int *cols,
                        const double *vals, int64_t cap, int64_t *nnz, int64_t *col_ptr,
                        int *row_idx, double *out) {
  std::vector<int64_t> start(n_cols + 1, 0);
  for (int64_t t = 0; t < nt; ++t) {
    if (cols[t] < 0 || cols[t] >= n_cols || rows[t] < 0 || rows[t] >= n_rows) return 1;
    start[cols[t] + 1]++;
  }
  for (int c = 0; c < n_cols; ++c) start[c + 1] += start[c];
  std::vector<int64_t> order(nt);
  {
    std::vector<int64_t> pos(start.begin(), start.end() - 1);
    for (int64_t t = 0; t < nt; ++t) order[pos[cols[t]]++] = t;
  }
  // first pass: count unique rows per column
  int64_t total = 0;
  std::vector<int64_t> cnt(n_cols, 0);
  std::vector<int> tmp;
  for (int c = 0; c < n_cols; ++c) {
    tmp.clear();
    for (int64_t k = start[c]; k < start[c + 1]; ++k) tmp.push_back(rows[order[k]]);
    std::sort(tmp.begin(), tmp.end());
    int64_t u = std::unique(tmp.begin(), tmp.end()) - tmp.begin();
    cnt[c] = u;
    total += u;
  }
  *nnz = total;
  if (total > cap || !col_ptr) return -2;
  col_ptr[0] = 0;
  for (int c = 0; c < n_cols; ++c) col_ptr[c + 1] = col_ptr[c] + cnt[c];
  std::vector<std::pair<int, int64_t>> ent;
  for (int c = 0; c < n_cols; ++c) {
    ent.clear();
    for (int64_t k = start[c]; k < start[c + 1]; ++k) ent.emplace_back(rows[order[k]], order[k]);
    std::stable_sort(ent.begin(), ent.end(),
                     [](const std::pair<int, int64_t> &a, const std::pair<int, int64_t> &b) {
                       return a.first < b.first;
                     });
    int64_t o = col_ptr[c] - 1;
    int last = -1;
    for (auto &e : ent) {
      if (e.first != last) {
        ++o;
        row_idx[o] = e.first;
        out[o] = vals[e.second];
        last = e.first;
      } else {
        out[o] = out[o] + vals[e.second];
      }
    }
  }
  return 0;
}

// fortsparse csc_matvec (called from spmv, src/solvers/fortfem_sparse_matrix.f90:46-58)
void or_csc_matvec(int n, const int64_t *cp, const int *ri, const double *v, const double *x,
                   double *y) {
  for (int i = 0; i < n; ++i) y[i] = 0.0;
  for (int c = 0; c < n; ++c) {
    double xc = x[c];
    for (int64_t k = cp[c]; k < cp[c + 1]; ++k) y[ri[k]] += v[k] * xc;
  }
}

int64_t or_lagrange_csc_nnz(int p, int nt, const int *tets) {
  int nb = or_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  if (or_lagrange_dof_map(p, nt, tets, gd.data(), &ng)) return -1;
  std::vector<uint64_t> keys;
  keys.reserve((size_t)nt * nb * nb);
  for (int c = 0; c < nt; ++c)
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i)
        keys.push_back(((uint64_t)gd[(size_t)nb * c + j] << 32) | (uint32_t)gd[(size_t)nb * c + i]);
  std::sort(keys.begin(), keys.end());
  return std::unique(keys.begin(), keys.end()) - keys.begin();
}

// assemble_tetra_lagrange_stiffness_csc, assembly_tetra_lagrange_arbitrary_order_3d.f90:276-334.
// Optional per-cell coefficient arrays multiply the scalar coefficients
// cellwise, as fortfem's own cell-coefficient assembler does
// (src/fortfem_forms_simple.f90:979-1045).
int or_lagrange_csc(int nv, const double *verts, int nt, const int *tets, int p, int rule, int q,
                    double stiff, double mass, const double *cs, const double *cm, int64_t cap,
                    int *n_dofs, int64_t *nnz, int64_t *col_ptr, int *row_idx, double *values) {
  if (nt < 1) return 1;
  for (int64_t i = 0; i < 4LL * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  int nb = or_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  if (or_lagrange_dof_map(p, nt, tets, gd.data(), &ng)) return 1;
  *n_dofs = ng;
  int64_t ntrip = (int64_t)nt * nb * nb;
  std::vector<int> rows(ntrip), cols(ntrip);
  std::vector<double> tv(ntrip);
  std::vector<double> M((size_t)nb * nb);
  int64_t e = 0;
  for (int c = 0; c < nt; ++c) {
    double v[12];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * c + n] + d];
    double ks = cs ? stiff * cs[c] : stiff;
    double km = cm ? mass * cm[c] : mass;
    if (or_lagrange_element(v, p, rule, q, ks, km, M.data())) return 1;
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row, ++e) {
        rows[e] = gd[(size_t)nb * c + row];
        cols[e] = gd[(size_t)nb * c + col];
        tv[e] = M[row + (size_t)nb * col];
      }
  }
  return or_csc_from_triplet(ng, ng, ntrip, rows.data(), cols.data(), tv.data(), cap, nnz, col_ptr,
                             row_idx, values);
}

// ------------------------------------------------- forward / reverse mode
// fortnum det3_jvp / inv3_jvp / det3_vjp / inv3_vjp (not vendored) restated
// from their definitions: d(det J) = det tr(J^-1 dJ), d(J^-1) = -J^-1 dJ J^-1,
// and the adjoints Jbar += detbar det J^-T, Jbar = -J^-T Jibar J^-T.
namespace {
static void mat3_mul(const double *A, const double *B, double *C) {  // column-major C = A B
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += A[r + 3 * k] * B[k + 3 * c];
      C[r + 3 * c] = s;
    }
}
}  // namespace

// assemble_tetra_lagrange_stiffness_element_jvp,
// assembly_tetra_lagrange_arbitrary_order_3d.f90:107-180: the same point loop
// as the primal element, differentiated term by term.
int or_lagrange_element_jvp(const double *v, int p, int rule, int q, double stiff, double mass,
                            const double *vdot, double stiff_dot, double mass_dot, double *Md) {
  if (p < 1 || p > 4) return 1;
  double J[9], Jd[9], Ji[9], Jid[9], T[9];
  tetra_jacobian(v, J);
  tetra_jacobian(vdot, Jd);
  const double det = det3(J);
  if (!valid_jacobian(J, det)) return 1;
  inv3(J, det, Ji);
  mat3_mul(Ji, Jd, T);
  const double det_dot = det * (T[0] + T[4] + T[8]);
  double U[9];
  mat3_mul(T, Ji, U);
  for (int i = 0; i < 9; ++i) Jid[i] = -U[i];
  Rule R;
  if (!make_rule(rule, q, R)) return 1;
  const int nb = or_lagrange_dof_count(p);
  std::vector<double> val(nb), grad(3 * nb), pg(3 * nb), pgd(3 * nb);
  std::fill(Md, Md + (size_t)nb * nb, 0.0);
  for (size_t pt = 0; pt < R.w.size(); ++pt) {
    double P[3] = {R.x[pt], R.y[pt], R.z[pt]};
    if (or_lagrange_evaluate(p, P, val.data(), grad.data())) return 1;
    for (int d = 0; d < nb; ++d)
      for (int i = 0; i < 3; ++i) {
        double s = 0.0, t = 0.0;
        for (int k = 0; k < 3; ++k) {
          s += Ji[k + 3 * i] * grad[3 * d + k];
          t += Jid[k + 3 * i] * grad[3 * d + k];
        }
        pg[3 * d + i] = s;
        pgd[3 * d + i] = t;
      }
    const double w = R.w[pt];
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row) {
        double ge = 0.0, gd = 0.0;
        for (int i = 0; i < 3; ++i) {
          ge += pg[3 * row + i] * pg[3 * col + i];
          gd += pgd[3 * row + i] * pg[3 * col + i] + pg[3 * row + i] * pgd[3 * col + i];
        }
        const double me = val[row] * val[col];
        Md[row + (size_t)nb * col] +=
            w * (det_dot * (stiff * ge + mass * me) +
                 det * (stiff_dot * ge + stiff * gd + mass_dot * me));
      }
  }
  return 0;
}

// assemble_tetra_lagrange_stiffness_element_vjp, same file :182-274.
int or_lagrange_element_vjp(const double *v, int p, int rule, int q, double stiff, double mass,
                            const double *Mb, double *vbar, double *stiff_bar, double *mass_bar) {
  for (int i = 0; i < 12; ++i) vbar[i] = 0.0;
  *stiff_bar = 0.0;
  *mass_bar = 0.0;
  if (p < 1 || p > 4) return 1;
  const int nb = or_lagrange_dof_count(p);
  double J[9], Ji[9];
  tetra_jacobian(v, J);
  const double det = det3(J);
  if (!valid_jacobian(J, det)) return 1;
  inv3(J, det, Ji);
  Rule R;
  if (!make_rule(rule, q, R)) return 1;
  std::vector<double> val(nb), grad(3 * nb), pg(3 * nb), pgb(3 * nb);
  double det_bar = 0.0, Jib[9] = {0};
  for (size_t pt = 0; pt < R.w.size(); ++pt) {
    double P[3] = {R.x[pt], R.y[pt], R.z[pt]};
    if (or_lagrange_evaluate(p, P, val.data(), grad.data())) return 1;
    for (int d = 0; d < nb; ++d)
      for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += Ji[k + 3 * i] * grad[3 * d + k];
        pg[3 * d + i] = s;
      }
    std::fill(pgb.begin(), pgb.end(), 0.0);
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row) {
        const double seed = R.w[pt] * Mb[row + (size_t)nb * col];
        double ge = 0.0;
        for (int i = 0; i < 3; ++i) ge += pg[3 * row + i] * pg[3 * col + i];
        const double me = val[row] * val[col];
        det_bar += seed * (stiff * ge + mass * me);
        *stiff_bar += seed * det * ge;
        *mass_bar += seed * det * me;
        for (int i = 0; i < 3; ++i) {
          pgb[3 * row + i] += seed * det * stiff * pg[3 * col + i];
          pgb[3 * col + i] += seed * det * stiff * pg[3 * row + i];
        }
      }
    // inverse_jacobian_bar += matmul(gradients, transpose(physical_gradients_bar))
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) {
        double s = 0.0;
        for (int d = 0; d < nb; ++d) s += grad[3 * d + r] * pgb[3 * d + c];
        Jib[r + 3 * c] += s;
      }
  }
  // Jbar = -J^-T Jib J^-T + det_bar det J^-T
  double JiT[9], A[9], B[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) JiT[r + 3 * c] = Ji[c + 3 * r];
  mat3_mul(JiT, Jib, A);
  mat3_mul(A, JiT, B);
  double Jb[9];
  for (int i = 0; i < 9; ++i) Jb[i] = -B[i] + det_bar * det * JiT[i];
  // tetra_jacobian_vjp: J(:,c) = v(:,c+1) - v(:,0)
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      vbar[r + 3 * (c + 1)] += Jb[r + 3 * c];
      vbar[r] -= Jb[r + 3 * c];
    }
  return 0;
}

// assemble_tetra_lagrange_stiffness_csc_jvp, same file :336-391: element
// tangents scattered through csc_from_triplet, so the pattern is the primal's.
int or_lagrange_csc_jvp(int nv, const double *verts, int nt, const int *tets, int p, int rule,
                        int q, double stiff, double mass, const double *vdot, double stiff_dot,
                        double mass_dot, int64_t cap, int *n_dofs, int64_t *nnz, int64_t *col_ptr,
                        int *row_idx, double *values) {
  if (nt < 1) return 1;
  for (int64_t i = 0; i < 4LL * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  const int nb = or_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  if (or_lagrange_dof_map(p, nt, tets, gd.data(), &ng)) return 1;
  *n_dofs = ng;
  const int64_t ntrip = (int64_t)nt * nb * nb;
  std::vector<int> rows(ntrip), cols(ntrip);
  std::vector<double> tv(ntrip), M((size_t)nb * nb);
  int64_t e = 0;
  for (int c = 0; c < nt; ++c) {
    double v[12], vd[12];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) {
        v[3 * n + d] = verts[3 * tets[4 * c + n] + d];
        vd[3 * n + d] = vdot[3 * tets[4 * c + n] + d];
      }
    if (or_lagrange_element_jvp(v, p, rule, q, stiff, mass, vd, stiff_dot, mass_dot, M.data()))
      return 1;
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row, ++e) {
        rows[e] = gd[(size_t)nb * c + row];
        cols[e] = gd[(size_t)nb * c + col];
        tv[e] = M[row + (size_t)nb * col];
      }
  }
  return or_csc_from_triplet(ng, ng, ntrip, rows.data(), cols.data(), tv.data(), cap, nnz, col_ptr,
                             row_idx, values);
}

// assemble_tetra_lagrange_stiffness_csc_vjp, same file :393-471, with
// csc_value_bar_at (:836-851) reading each element entry's cotangent from the
// merged pattern; vertex and coefficient adjoints accumulate in cell order.
int or_lagrange_csc_vjp(int nv, const double *verts, int nt, const int *tets, int p, int rule,
                        int q, double stiff, double mass, int64_t nnz, const double *values_bar,
                        double *verts_bar, double *stiff_bar, double *mass_bar) {
  for (int64_t i = 0; i < 3LL * nv; ++i) verts_bar[i] = 0.0;
  *stiff_bar = 0.0;
  *mass_bar = 0.0;
  if (nt < 1) return 1;
  for (int64_t i = 0; i < 4LL * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  const int64_t pat = or_lagrange_csc_nnz(p, nt, tets);
  if (pat < 0 || pat != nnz) return 1;
  int ng = 0, nd = 0;
  const int nb = or_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  if (or_lagrange_dof_map(p, nt, tets, gd.data(), &ng)) return 1;
  std::vector<int64_t> cp(ng + 1);
  std::vector<int> ri(nnz);
  std::vector<double> vals(nnz);
  int64_t got = 0;
  if (or_lagrange_csc(nv, verts, nt, tets, p, rule, q, stiff, mass, nullptr, nullptr, nnz, &nd,
                      &got, cp.data(), ri.data(), vals.data()))
    return 1;
  std::vector<double> Mb((size_t)nb * nb);
  for (int c = 0; c < nt; ++c) {
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row) {
        const int gr = gd[(size_t)nb * c + row], gc = gd[(size_t)nb * c + col];
        double b = 0.0;
        for (int64_t k = cp[gc]; k < cp[gc + 1]; ++k)
          if (ri[k] == gr) { b = values_bar[k]; break; }
        Mb[row + (size_t)nb * col] = b;
      }
    double v[12], vb[12], sb = 0.0, mb = 0.0;
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * c + n] + d];
    if (or_lagrange_element_vjp(v, p, rule, q, stiff, mass, Mb.data(), vb, &sb, &mb)) return 1;
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) verts_bar[3 * tets[4 * c + n] + d] += vb[3 * n + d];
    *stiff_bar += sb;
    *mass_bar += mb;
  }
  return 0;
}

// assemble_tetra_lagrange_scalar_load_samples,
// assembly_tetra_lagrange_arbitrary_order_3d.f90:473-528.  rhs has n_dofs entries.
int or_lagrange_load_samples(int nv, const double *verts, int nt, const int *tets, int p, int rule,
                             int q, const double *src, double *rhs) {
  int nb = or_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  if (or_lagrange_dof_map(p, nt, tets, gd.data(), &ng)) return 1;
  Rule R;
  if (!make_rule(rule, q, R)) return 1;
  int nq = (int)R.w.size();
  std::vector<double> val((size_t)nb * nq), grad(3 * (size_t)nb);
  for (int pt = 0; pt < nq; ++pt) {
    double P[3] = {R.x[pt], R.y[pt], R.z[pt]};
    if (or_lagrange_evaluate(p, P, val.data() + (size_t)nb * pt, grad.data())) return 1;
  }
  for (int i = 0; i < ng; ++i) rhs[i] = 0.0;
  for (int c = 0; c < nt; ++c) {
    double v[12], J[9];
    for (int n = 0; n < 4; ++n) {
      if (tets[4 * c + n] < 0 || tets[4 * c + n] >= nv) return 1;
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * c + n] + d];
    }
    tetra_jacobian(v, J);
    double det = det3(J);
    if (!valid_jacobian(J, det)) return 1;
    for (int pt = 0; pt < nq; ++pt)
      for (int d = 0; d < nb; ++d) {
        int g = gd[(size_t)nb * c + d];
        rhs[g] = rhs[g] + det * R.w[pt] * src[(size_t)nq * c + pt] * val[(size_t)nb * pt + d];
      }
  }
  return 0;
}

// Physical quadrature points vertices(:,1) + J*xi (assembly_..._3d.f90:757-758), used
// to sample source functions for the sampled-load entry.
int or_lagrange_quadrature_points(int nv, const double *verts, int nt, const int *tets, int rule,
                                  int q, double *out) {
  Rule R;
  if (!make_rule(rule, q, R)) return 1;
  int nq = (int)R.w.size();
  for (int c = 0; c < nt; ++c) {
    double v[12], J[9];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * c + n] + d];
    tetra_jacobian(v, J);
    for (int pt = 0; pt < nq; ++pt) {
      double xi[3] = {R.x[pt], R.y[pt], R.z[pt]};
      for (int r = 0; r < 3; ++r) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += J[r + 3 * k] * xi[k];
        out[3 * ((size_t)nq * c + pt) + r] = v[r] + s;
      }
    }
  }
  return 0;
}

namespace {
// Face incidence by hash (the reference counts by an O(T^2) scan; the result
// is the same set of incidence-one faces).
uint64_t face_key(int a, int b, int c) {
  int t[3] = {a, b, c};
  std::sort(t, t + 3);
  return ((uint64_t)(uint32_t)t[0] << 42) ^ ((uint64_t)(uint32_t)t[1] << 21) ^ (uint64_t)(uint32_t)t[2];
}
}  // namespace

static int lagrange_dirichlet_impl(int p, int nv, const double *verts, int nt, const int *tets,
                                   uint8_t *constrained, double *node_points, bool faithful) {
  int nb = or_lagrange_dof_count(p);
  std::vector<int> idx(4 * nb);
  std::vector<double> nodes(3 * nb);
  or_lagrange_barycentric_indices(p, idx.data(), nodes.data());
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  int st = faithful ? or_lagrange_dof_map_faithful(p, nt, tets, gd.data(), &ng)
                    : or_lagrange_dof_map(p, nt, tets, gd.data(), &ng);
  if (st) return 1;
  std::memset(constrained, 0, ng);
  if (node_points)
    for (int i = 0; i < 3 * ng; ++i) node_points[i] = 0.0;
  std::unordered_map<uint64_t, int> inc;
  if (!faithful) {
    inc.reserve((size_t)nt * 4);
    for (int c = 0; c < nt; ++c)
      for (int o = 0; o < 4; ++o) {
        int f[3], k = 0;
        for (int n = 0; n < 4; ++n)
          if (n != o) f[k++] = tets[4 * c + n];
        inc[face_key(f[0], f[1], f[2])] += 1;
      }
  }
  for (int c = 0; c < nt; ++c) {
    double v[12], J[9];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * c + n] + d];
    tetra_jacobian(v, J);
    for (int o = 0; o < 4; ++o) {
      int f[3], k = 0;
      for (int n = 0; n < 4; ++n)
        if (n != o) f[k++] = tets[4 * c + n];
      int incidence = 0;
      if (faithful) {
        // fortfem_tetra_lagrange_solver_3d.f90:587-597, O(T^2)
        for (int oc = 0; oc < nt; ++oc) {
          bool all = true;
          for (int a = 0; a < 3; ++a) {
            bool any = false;
            for (int n = 0; n < 4; ++n) any = any || tets[4 * oc + n] == f[a];
            all = all && any;
          }
          if (all) ++incidence;
        }
      } else {
        incidence = inc[face_key(f[0], f[1], f[2])];
      }
      if (incidence != 1) continue;
      for (int d = 0; d < nb; ++d) {
        if (idx[4 * d + o] != 0) continue;
        int g = gd[(size_t)nb * c + d];
        constrained[g] = 1;
        if (node_points)
          for (int r = 0; r < 3; ++r) {
            double s = 0.0;
            for (int kk = 0; kk < 3; ++kk) s += J[r + 3 * kk] * nodes[3 * d + kk];
            node_points[3 * g + r] = v[r] + s;
          }
      }
    }
  }
  return 0;
}

// build_dirichlet_data, src/solvers/fortfem_tetra_lagrange_solver_3d.f90:551-610
int or_lagrange_dirichlet_faithful(int p, int nv, const double *verts, int nt, const int *tets,
                                   uint8_t *constrained, double *node_points) {
  return lagrange_dirichlet_impl(p, nv, verts, nt, tets, constrained, node_points, true);
}
int or_lagrange_dirichlet(int p, int nv, const double *verts, int nt, const int *tets,
                          uint8_t *constrained, double *node_points) {
  return lagrange_dirichlet_impl(p, nv, verts, nt, tets, constrained, node_points, false);
}

// ---------------------------------------------------------- solution probes
// evaluate_tetra_lagrange_solution, src/solvers/fortfem_tetra_lagrange_solver_3d.f90:131-150:
// initialize_tetra_lagrange_solution_evaluator (:437-489: every cell valid,
// solution sized to the DoF map) then evaluate_tetra_lagrange_solution_prepared
// (:491-528: value = sum u_i phi_i, gradient = J^-T sum u_i grad phi_i).
int or_lagrange_evaluate_solution(int nv, const double *verts, int nt, const int *tets, int p,
                                  int n_dofs, const double *u, int cell, const double *xi,
                                  double *value, double *grad) {
  *value = 0.0;
  grad[0] = grad[1] = grad[2] = 0.0;
  if (nt < 1 || p < 1 || p > 4) return 1;
  for (int64_t i = 0; i < 4LL * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  const int nb = or_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  if (or_lagrange_dof_map(p, nt, tets, gd.data(), &ng)) return 1;
  for (int c = 0; c < nt; ++c) {
    double v[12], J[9];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * c + n] + d];
    tetra_jacobian(v, J);
    if (!valid_jacobian(J, det3(J))) return 1;
  }
  if (cell < 0 || cell >= nt || n_dofs != ng) return 1;
  // evaluate_tetra_lagrange rejects barycentric coordinates below -64 eps (:88-89)
  const double bary[4] = {1.0 - (xi[0] + xi[1] + xi[2]), xi[0], xi[1], xi[2]};
  for (double b : bary)
    if (b < -64.0 * kEps) return 1;
  std::vector<double> val(nb), g(3 * nb);
  if (or_lagrange_evaluate(p, xi, val.data(), g.data())) return 1;
  double v[12], J[9], Ji[9];
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * cell + n] + d];
  tetra_jacobian(v, J);
  inv3(J, det3(J), Ji);
  double rg[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < nb; ++d) {
    const double ud = u[gd[(size_t)nb * cell + d]];
    *value += ud * val[d];
    for (int a = 0; a < 3; ++a) rg[a] += ud * g[3 * d + a];
  }
  // matmul(transpose(inverse_jacobian), reference_gradient)
  for (int i = 0; i < 3; ++i) grad[i] = Ji[3 * i] * rg[0] + Ji[3 * i + 1] * rg[1] + Ji[3 * i + 2] * rg[2];
  return 0;
}

// evaluate_tetra_lagrange_solution_at_point, same file :305-325, with
// invert_tetra_affine_map (src/geometry/tetra_affine_map.f90:15-33).
int or_lagrange_evaluate_solution_at_point(int nv, const double *verts, int nt, const int *tets,
                                           int p, int n_dofs, const double *u, int cell,
                                           const double *point, double *value, double *grad) {
  *value = 0.0;
  grad[0] = grad[1] = grad[2] = 0.0;
  if (cell < 0 || cell >= nt) return 1;
  for (int n = 0; n < 4; ++n)
    if (tets[4 * cell + n] < 0 || tets[4 * cell + n] >= nv) return 1;
  double v[12], J[9], Ji[9];
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * cell + n] + d];
  tetra_jacobian(v, J);
  const double det = det3(J);
  if (!valid_jacobian(J, det)) return 1;
  inv3(J, det, Ji);
  double xi[3];
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s += Ji[i + 3 * k] * (point[k] - v[k]);
    xi[i] = s;
  }
  return or_lagrange_evaluate_solution(nv, verts, nt, tets, p, n_dofs, u, cell, xi, value, grad);
}

// Point probe over all cells for a Lagrange solution, the loop of
// evaluate_box_solution_order (src/solvers/fortfem_magnetic_box_3d.f90:269-343)
// with the scalar basis: every cell with det > 0 whose reference coordinates
// of the point are >= -1e-12 with sum <= 1 + 1e-12 contributes (value,
// gradient); mode 0 averages them in cell order, mode 1 takes the first.
// *count is the number of contributing cells (0: none; -1: a contributing
// cell rejected by the basis evaluation's -64 eps test).
int or_lagrange_probe(int nv, const double *verts, int nt, const int *tets, int p, int n_dofs,
                      const double *u, const double *point, int mode, double *value,
                      double *grad, int *count) {
  *value = 0.0;
  grad[0] = grad[1] = grad[2] = 0.0;
  *count = 0;
  const int nb = or_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  if (or_lagrange_dof_map(p, nt, tets, gd.data(), &ng) || n_dofs != ng) return 1;
  std::vector<double> val(nb), g(3 * nb);
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  int found = 0;
  for (int c = 0; c < nt; ++c) {
    double v[12], J[9], Ji[9];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * c + n] + d];
    tetra_jacobian(v, J);
    const double det = det3(J);
    if (det <= 0.0) continue;
    inv3(J, det, Ji);
    double xi[3];
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += Ji[i + 3 * k] * (point[k] - v[k]);
      xi[i] = s;
    }
    if (xi[0] < -1.0e-12 || xi[1] < -1.0e-12 || xi[2] < -1.0e-12) continue;
    if (xi[0] + xi[1] + xi[2] > 1.0 + 1.0e-12) continue;
    if (1.0 - (xi[0] + xi[1] + xi[2]) < -64.0 * kEps || xi[0] < -64.0 * kEps ||
        xi[1] < -64.0 * kEps || xi[2] < -64.0 * kEps) {
      *count = -1;
      return 1;
    }
    or_lagrange_evaluate(p, xi, val.data(), g.data());
    double val_c = 0.0, rg[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < nb; ++d) {
      const double ud = u[gd[(size_t)nb * c + d]];
      val_c += ud * val[d];
      for (int a = 0; a < 3; ++a) rg[a] += ud * g[3 * d + a];
    }
    acc[0] += val_c;
    for (int i = 0; i < 3; ++i)
      acc[1 + i] += Ji[3 * i] * rg[0] + Ji[3 * i + 1] * rg[1] + Ji[3 * i + 2] * rg[2];
    ++found;
    if (mode == 1) break;
  }
  *count = found;
  if (found < 1) return 1;
  *value = acc[0] / found;
  for (int i = 0; i < 3; ++i) grad[i] = acc[1 + i] / found;
  return 0;
}

// --------------------------------------------------------------- P1 triangles
// assemble_scalar_p1_matrix, src/fortfem_forms_simple.f90:1678-1728 (dense).
static int p1_local(const double *verts, const int *tri, double mass, double stiff, double *local) {
  double x[3], y[3];
  for (int i = 0; i < 3; ++i) { x[i] = verts[2 * tri[i]]; y[i] = verts[2 * tri[i] + 1]; }
  double det = (x[1] - x[0]) * (y[2] - y[0]) - (x[2] - x[0]) * (y[1] - y[0]);
  if (std::fabs(det) <= 64.0 * kEps) return 1;
  double area = 0.5 * std::fabs(det);
  double g[2][3] = {{(y[1] - y[2]) / det, (y[2] - y[0]) / det, (y[0] - y[1]) / det},
                    {(x[2] - x[1]) / det, (x[0] - x[2]) / det, (x[1] - x[0]) / det}};
  for (int b = 0; b < 3; ++b)
    for (int a = 0; a < 3; ++a) {
      double gg = g[0][a] * g[0][b] + g[1][a] * g[1][b];
      double m = (a == b) ? 2.0 : 1.0;
      local[a + 3 * b] = stiff * area * gg + mass * area * m / 12.0;
    }
  return 0;
}

int or_p1_dense_matrix(int nv, const double *verts, int nt, const int *tris, double mass,
                       double stiff, double *A) {
  for (size_t i = 0; i < (size_t)nv * nv; ++i) A[i] = 0.0;
  for (int t = 0; t < nt; ++t) {
    double L[9];
    if (p1_local(verts, tris + 3 * t, mass, stiff, L)) return 3;
    for (int b = 0; b < 3; ++b)
      for (int a = 0; a < 3; ++a)
        A[tris[3 * t + a] + (size_t)nv * tris[3 * t + b]] += L[a + 3 * b];
  }
  return 0;
}

// assemble_scalar_p1_load, src/fortfem_forms_simple.f90:1730-1761
int or_p1_load(int nv, const double *verts, int nt, const int *tris, double load, double *vec) {
  for (int i = 0; i < nv; ++i) vec[i] = 0.0;
  for (int t = 0; t < nt; ++t) {
    double x[3], y[3];
    for (int i = 0; i < 3; ++i) { x[i] = verts[2 * tris[3 * t + i]]; y[i] = verts[2 * tris[3 * t + i] + 1]; }
    double det = (x[1] - x[0]) * (y[2] - y[0]) - (x[2] - x[0]) * (y[1] - y[0]);
    if (std::fabs(det) <= 64.0 * kEps) return 3;
    double area = 0.5 * std::fabs(det);
    for (int b = 0; b < 3; ++b) vec[tris[3 * t + b]] += load * area / 3.0;
  }
  return 0;
}

// The same element formulas scattered into CSC through triplets (the dense
// reference cannot hold large meshes); per-cell coefficient optional.
int or_p1_csc(int nv, const double *verts, int nt, const int *tris, double mass, double stiff,
              const double *cs, int64_t cap, int64_t *nnz, int64_t *col_ptr, int *row_idx,
              double *values) {
  int64_t ntrip = 9LL * nt;
  std::vector<int> rows(ntrip), cols(ntrip);
  std::vector<double> tv(ntrip);
  int64_t e = 0;
  for (int t = 0; t < nt; ++t) {
    double L[9];
    if (p1_local(verts, tris + 3 * t, mass, cs ? stiff * cs[t] : stiff, L)) return 3;
    for (int b = 0; b < 3; ++b)
      for (int a = 0; a < 3; ++a, ++e) {
        rows[e] = tris[3 * t + a];
        cols[e] = tris[3 * t + b];
        tv[e] = L[a + 3 * b];
      }
  }
  return or_csc_from_triplet(nv, nv, ntrip, rows.data(), cols.data(), tv.data(), cap, nnz, col_ptr,
                             row_idx, values);
}

// Dirichlet elimination of solve_compiled_p1_problem,
// src/solvers/fortfem_solvers_laplacian.f90:88-97.
int or_p1_dirichlet_eliminate_dense(int n, double *A, double *rhs, const uint8_t *bnd, double g) {
  for (int d = 0; d < n; ++d) {
    if (!bnd[d]) continue;
    for (int i = 0; i < n; ++i) rhs[i] = rhs[i] - A[i + (size_t)n * d] * g;
    for (int i = 0; i < n; ++i) A[i + (size_t)n * d] = 0.0;
    for (int j = 0; j < n; ++j) A[d + (size_t)n * j] = 0.0;
    A[d + (size_t)n * d] = 1.0;
    rhs[d] = g;
  }
  return 0;
}

// ------------------------------------------------------ reduction and solvers
// sparse_direct_solve_constrained_real (reduction part),
// src/solvers/fortfem_sparse_direct.f90:264-344.
int or_reduce_constrained(int n, const int64_t *cp, const int *ri, const double *v,
                          const double *rhs, const uint8_t *con, const double *cval, int *n_free,
                          int64_t *nnz_r, int64_t *rcp, int *rri, double *rv, double *rrhs,
                          int *free_dofs) {
  std::vector<int> free_index(n, -1);
  int nf = 0;
  for (int c = 0; c < n; ++c)
    if (!con[c]) { free_index[c] = nf; if (free_dofs) free_dofs[nf] = c; ++nf; }
  *n_free = nf;
  int64_t e = 0;
  if (rcp) rcp[0] = 0;
  int f = 0;
  for (int c = 0; c < n; ++c) {
    if (con[c]) continue;
    for (int64_t k = cp[c]; k < cp[c + 1]; ++k) {
      int r = ri[k];
      if (con[r]) continue;
      if (rri) { rri[e] = free_index[r]; rv[e] = v[k]; }
      ++e;
    }
    ++f;
    if (rcp) rcp[f] = e;
  }
  *nnz_r = e;
  if (rrhs) {
    for (int c = 0; c < n; ++c)
      if (!con[c]) rrhs[free_index[c]] = rhs[c];
    for (int c = 0; c < n; ++c) {
      if (!con[c]) continue;
      for (int64_t k = cp[c]; k < cp[c + 1]; ++k) {
        int r = ri[k];
        if (con[r]) continue;
        rrhs[free_index[r]] = rrhs[free_index[r]] - v[k] * (cval ? cval[c] : 0.0);
      }
    }
  }
  return 0;
}

}  // extern "C"

namespace {
// guard = 0: the reference's absolute breakdown test |p^T A p| < 1e-14
// (advanced_solvers.f90:897); guard = 1: stop only on p^T A p <= 0 or a
// non-finite value (SPD breakdown), which lets scale-free tolerances be reached
// on systems whose p^T A p falls below 1e-14 before convergence.
template <class MatVec>
int pcg_core(int n, MatVec matvec, const std::vector<double> &diag, const double *b, double *x,
             double tol_in, int relative, int maxit, int guard, double *stats) {
  // pcg_solve_operator / initialize_pcg_state / pcg_iteration_loop,
  // src/solvers/advanced_solvers.f90:831-925; tolerance :1063-1073.
  std::vector<double> r(n), z(n), p(n), Ap(n), Ax(n);
  matvec(x, Ax.data());
  double rr = 0.0;
  for (int i = 0; i < n; ++i) { r[i] = b[i] - Ax[i]; }
  for (int i = 0; i < n; ++i) rr += r[i] * r[i];
  double initial = std::sqrt(rr), res = initial;
  for (int i = 0; i < n; ++i) z[i] = diag[i] * r[i];
  p = z;
  double rz_old = 0.0;
  for (int i = 0; i < n; ++i) rz_old += r[i] * z[i];
  double tol = relative ? tol_in * initial : tol_in;
  int converged = 0, iters = 0;
  for (int it = 1; it <= maxit; ++it) {
    matvec(p.data(), Ap.data());
    double pAp = 0.0;
    for (int i = 0; i < n; ++i) pAp += p[i] * Ap[i];
    if (guard == 0 ? std::fabs(pAp) < 1.0e-14 : !(pAp > 0.0 && std::isfinite(pAp))) break;
    double alpha = rz_old / pAp;
    for (int i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
    for (int i = 0; i < n; ++i) r[i] = r[i] - alpha * Ap[i];
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += r[i] * r[i];
    res = std::sqrt(s);
    if (res <= tol) { converged = 1; iters = it; break; }
    for (int i = 0; i < n; ++i) z[i] = diag[i] * r[i];
    double rz_new = 0.0;
    for (int i = 0; i < n; ++i) rz_new += r[i] * z[i];
    double beta = rz_new / rz_old;
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rz_old = rz_new;
    iters = it;
  }
  if (!converged && res <= tol) converged = 1;  // finalize_solver_status :1075-1086
  if (stats) { stats[0] = iters; stats[1] = converged; stats[2] = res; stats[3] = initial; }
  return 0;
}
}  // namespace

extern "C" {

// solve_sparse(method="pcg"), src/solvers/advanced_solvers.f90:135-195, with the
// Jacobi diagonal found by a column search as build_sparse_preconditioner does
// (:1139-1154).
int or_pcg_sparse(int n, const int64_t *cp, const int *ri, const double *v, const double *b,
                  double *x, double tol, int relative, int maxit, int jacobi, int guard,
                  double *stats) {
  std::vector<double> diag(n, 1.0);
  if (jacobi)
    for (int i = 0; i < n; ++i) {
      double a = 0.0;
      for (int64_t k = cp[i]; k < cp[i + 1]; ++k)
        if (ri[k] == i) { a = v[k]; break; }
      diag[i] = (std::fabs(a) > 1.0e-14) ? 1.0 / a : 1.0;
    }
  auto mv = [&](const double *in, double *out) { or_csc_matvec(n, cp, ri, v, in, out); };
  return pcg_core(n, mv, diag, b, x, tol, relative, maxit, guard, stats);
}

// pcg_solve (dense), src/solvers/advanced_solvers.f90:800-829; Jacobi :1101-1109.
int or_pcg_dense(int n, const double *A, const double *b, double *x, double tol, int relative,
                 int maxit, int jacobi, int guard, double *stats) {
  std::vector<double> diag(n, 1.0);
  if (jacobi)
    for (int i = 0; i < n; ++i) {
      double a = A[i + (size_t)n * i];
      diag[i] = (std::fabs(a) > 1.0e-14) ? 1.0 / a : 1.0;
    }
  auto mv = [&](const double *in, double *out) {
    for (int i = 0; i < n; ++i) out[i] = 0.0;
    for (int j = 0; j < n; ++j) {
      double xj = in[j];
      const double *col = A + (size_t)n * j;
      for (int i = 0; i < n; ++i) out[i] += col[i] * xj;
    }
  };
  return pcg_core(n, mv, diag, b, x, tol, relative, maxit, guard, stats);
}

}  // extern "C"
