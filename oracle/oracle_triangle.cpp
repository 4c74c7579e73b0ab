// fortfem hot-path ORACLE (test infrastructure only; see oracle.h).
//
// FP64 CPU restatement of the arbitrary-order triangle Lagrange basis
// (src/elements/triangle_lagrange_arbitrary_order.f90:29-127, 143-198: the
// Bernstein polynomials of the barycentric powers, made nodal by the inverse
// of their Vandermonde matrix at the equispaced nodes) and of the element
// and CSC assembly of kappa grad u . grad v + m u v with it.  The reference
// has the basis but no triangle assembly routine; the element follows the
// pattern of its tetrahedral Lagrange element (assembly_tetra_lagrange_
// arbitrary_order_3d.f90:40-105) with |det J| as the area factor (the P1
// forms of src/fortfem_forms_simple.f90:1702-1717 use the unsigned area), and
// the DoF numbering is the first-appearance rule of the tetrahedral map
// (tetra_lagrange_global_dof_map.f90:13-99) on triangles.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

namespace {
const double kEps = 2.220446049250313e-16;

double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}
double factorial(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= (double)i;
  return r;
}

// barycentric powers (first = 1 - x - y, second = x, third = y) and nodes,
// initialize_triangle_lagrange_basis :52-68
void powers_and_nodes(int p, std::vector<int> &pw, std::vector<double> &nodes) {
  pw.clear();
  nodes.clear();
  if (p == 0) {
    pw = {0, 0, 0};
    nodes = {1.0 / 3.0, 1.0 / 3.0};
    return;
  }
  for (int a = 0; a <= p; ++a)
    for (int b = 0; b <= p - a; ++b) {
      const int c = p - a - b;
      pw.insert(pw.end(), {a, b, c});
      nodes.insert(nodes.end(), {(double)b / p, (double)c / p});
    }
}

// evaluate_bernstein_polynomials :143-176 with power_derivative :178-198
void bernstein(int p, const std::vector<int> &pw, double x, double y, double *val, double *grad) {
  const int n = (int)pw.size() / 3;
  const double bary[3] = {1.0 - x - y, x, y};
  for (int d = 0; d < n; ++d) {
    const int e[3] = {pw[3 * d], pw[3 * d + 1], pw[3 * d + 2]};
    const double coef = factorial(p) / (factorial(e[0]) * factorial(e[1]) * factorial(e[2]));
    val[d] = coef * ipow(bary[0], e[0]) * ipow(bary[1], e[1]) * ipow(bary[2], e[2]);
    double der[3];
    for (int k = 0; k < 3; ++k) {
      if (e[k] == 0) { der[k] = 0.0; continue; }
      int r[3] = {e[0], e[1], e[2]};
      r[k] -= 1;
      der[k] = (double)e[k] * ipow(bary[0], r[0]) * ipow(bary[1], r[1]) * ipow(bary[2], r[2]);
    }
    grad[2 * d] = coef * (-der[0] + der[1]);
    grad[2 * d + 1] = coef * (-der[0] + der[2]);
  }
}

// inverse of the Vandermonde matrix (dense_solve of fortnum, not vendored,
// restated as Gauss-Jordan elimination with partial pivoting); C[m + n*b]
bool nodal_coefficients(int p, std::vector<double> &C) {
  std::vector<int> pw;
  std::vector<double> nodes;
  powers_and_nodes(p, pw, nodes);
  const int n = (int)pw.size() / 3;
  std::vector<double> V((size_t)n * n), g(2 * n), row(n);
  for (int d = 0; d < n; ++d) {
    bernstein(p, pw, nodes[2 * d], nodes[2 * d + 1], row.data(), g.data());
    for (int m = 0; m < n; ++m) V[d + (size_t)n * m] = row[m];  // V(d, m)
  }
  C.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) C[i + (size_t)n * i] = 1.0;
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (std::fabs(V[r + (size_t)n * col]) > std::fabs(V[piv + (size_t)n * col])) piv = r;
    if (std::fabs(V[piv + (size_t)n * col]) == 0.0) return false;
    if (piv != col)
      for (int k = 0; k < n; ++k) {
        std::swap(V[col + (size_t)n * k], V[piv + (size_t)n * k]);
        std::swap(C[col + (size_t)n * k], C[piv + (size_t)n * k]);
      }
    const double inv = 1.0 / V[col + (size_t)n * col];
    for (int k = 0; k < n; ++k) {
      V[col + (size_t)n * k] *= inv;
      C[col + (size_t)n * k] *= inv;
    }
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      const double f = V[r + (size_t)n * col];
      if (f == 0.0) continue;
      for (int k = 0; k < n; ++k) {
        V[r + (size_t)n * k] -= f * V[col + (size_t)n * k];
        C[r + (size_t)n * k] -= f * C[col + (size_t)n * k];
      }
    }
  }
  return true;
}

struct TriRule {
  std::vector<double> x, y, w;
};
void triangle_rule(int q, TriRule &R) {
  const int n = or_triangle_duffy_count(q);
  R.x.resize(n);
  R.y.resize(n);
  R.w.resize(n);
  or_triangle_duffy(q, R.x.data(), R.y.data(), R.w.data());
}

bool tri_geometry(const double *v, double *J, double *det) {
  J[0] = v[2] - v[0];  // column-major 2x2: J(:,0) = v1 - v0, J(:,1) = v2 - v0
  J[1] = v[3] - v[1];
  J[2] = v[4] - v[0];
  J[3] = v[5] - v[1];
  *det = J[0] * J[3] - J[2] * J[1];
  double m = 0.0;
  for (int i = 0; i < 4; ++i) m = std::max(m, std::fabs(J[i]));
  const double s = std::max(1.0, m);
  return std::fabs(*det) > 64.0 * kEps * s * s;
}
}  // namespace

extern "C" {

int or_triangle_lagrange_dof_count(int p) { return (p + 1) * (p + 2) / 2; }

int or_triangle_lagrange_nodes(int p, double *nodes, int *powers) {
  if (p < 0) return 1;
  std::vector<int> pw;
  std::vector<double> nd;
  powers_and_nodes(p, pw, nd);
  std::copy(nd.begin(), nd.end(), nodes);
  if (powers) std::copy(pw.begin(), pw.end(), powers);
  return 0;
}

// evaluate_triangle_lagrange_basis :90-127; gradients (2, n_b)
int or_triangle_lagrange_evaluate(int p, double x, double y, double *values, double *gradients) {
  if (p < 0) return 1;
  const double tol = 64.0 * kEps;
  if (x < -tol || y < -tol || x + y > 1.0 + tol) return 1;
  std::vector<int> pw;
  std::vector<double> nodes, C;
  powers_and_nodes(p, pw, nodes);
  if (!nodal_coefficients(p, C)) return 2;
  const int n = (int)pw.size() / 3;
  std::vector<double> bv(n), bg(2 * n);
  bernstein(p, pw, x, y, bv.data(), bg.data());
  for (int b = 0; b < n; ++b) {
    double v = 0.0, gx = 0.0, gy = 0.0;
    for (int m = 0; m < n; ++m) {
      const double c = C[m + (size_t)n * b];
      v += c * bv[m];
      gx += c * bg[2 * m];
      gy += c * bg[2 * m + 1];
    }
    values[b] = v;
    gradients[2 * b] = gx;
    gradients[2 * b + 1] = gy;
  }
  return 0;
}

// First-appearance numbering: a local DoF is keyed by its (vertex, power)
// pairs with nonzero power, sorted by vertex.
int or_triangle_lagrange_dof_map(int p, int nt, const int *tris, int *gd, int *n_global) {
  if (p < 1) return 1;
  std::vector<int> pw;
  std::vector<double> nodes;
  powers_and_nodes(p, pw, nodes);
  const int nb = (int)pw.size() / 3;
  std::map<std::vector<int>, int> seen;
  int next = 0;
  for (int c = 0; c < nt; ++c) {
    const int *v = tris + 3 * c;
    if (v[0] == v[1] || v[0] == v[2] || v[1] == v[2]) return 1;
    for (int l = 0; l < nb; ++l) {
      std::vector<std::pair<int, int>> kv;
      for (int i = 0; i < 3; ++i)
        if (pw[3 * l + i] != 0) kv.push_back({v[i], pw[3 * l + i]});
      std::sort(kv.begin(), kv.end());
      std::vector<int> key;
      for (auto &e : kv) key.insert(key.end(), {e.first, e.second});
      auto it = seen.emplace(key, next);
      if (it.second) ++next;
      gd[(size_t)nb * c + l] = it.first->second;
    }
  }
  *n_global = next;
  return 0;
}

// Element matrix, column-major n_b x n_b; q = quadrature degree of the
// triangle Duffy rule (src/quadrature/triangle_duffy_quadrature.f90:12-45).
int or_triangle_lagrange_element(const double *v, int p, int q, double stiff, double mass,
                                 double *M) {
  if (p < 1 || q < 0) return 1;
  double J[4], det;
  if (!tri_geometry(v, J, &det)) return 1;
  const double Ji[4] = {J[3] / det, -J[1] / det, -J[2] / det, J[0] / det};  // column-major
  TriRule R;
  triangle_rule(q, R);
  const int nb = or_triangle_lagrange_dof_count(p);
  std::vector<double> val(nb), grad(2 * nb), pg(2 * nb);
  std::fill(M, M + (size_t)nb * nb, 0.0);
  const double area = std::fabs(det);
  for (size_t pt = 0; pt < R.w.size(); ++pt) {
    if (or_triangle_lagrange_evaluate(p, R.x[pt], R.y[pt], val.data(), grad.data())) return 1;
    for (int d = 0; d < nb; ++d)
      for (int i = 0; i < 2; ++i)  // J^-T grad: sum_k Ji(k, i) g(k)
        pg[2 * d + i] = Ji[2 * i] * grad[2 * d] + Ji[2 * i + 1] * grad[2 * d + 1];
    const double pw = area * R.w[pt];
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row)
        M[row + (size_t)nb * col] +=
            pw * (stiff * (pg[2 * row] * pg[2 * col] + pg[2 * row + 1] * pg[2 * col + 1]) +
                  mass * val[row] * val[col]);
  }
  return 0;
}

int64_t or_triangle_lagrange_csc_nnz(int p, int nt, const int *tris) {
  const int nb = or_triangle_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  if (or_triangle_lagrange_dof_map(p, nt, tris, gd.data(), &ng)) return -1;
  std::vector<uint64_t> keys;
  for (int c = 0; c < nt; ++c)
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i)
        keys.push_back(((uint64_t)gd[(size_t)nb * c + j] << 32) | (uint32_t)gd[(size_t)nb * c + i]);
  std::sort(keys.begin(), keys.end());
  return std::unique(keys.begin(), keys.end()) - keys.begin();
}

int or_triangle_lagrange_csc(int nv, const double *verts, int nt, const int *tris, int p, int q,
                             double stiff, double mass, const double *cs, const double *cm,
                             int64_t cap, int *n_dofs, int64_t *nnz, int64_t *col_ptr,
                             int *row_idx, double *values) {
  if (nt < 1) return 1;
  for (int i = 0; i < 3 * nt; ++i)
    if (tris[i] < 0 || tris[i] >= nv) return 1;
  const int nb = or_triangle_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  if (or_triangle_lagrange_dof_map(p, nt, tris, gd.data(), &ng)) return 1;
  *n_dofs = ng;
  const int64_t ntrip = (int64_t)nt * nb * nb;
  std::vector<int> rows(ntrip), cols(ntrip);
  std::vector<double> tv(ntrip), M((size_t)nb * nb);
  int64_t e = 0;
  for (int c = 0; c < nt; ++c) {
    double v[6];
    for (int n = 0; n < 3; ++n)
      for (int d = 0; d < 2; ++d) v[2 * n + d] = verts[2 * tris[3 * c + n] + d];
    const double ks = cs ? stiff * cs[c] : stiff, km = cm ? mass * cm[c] : mass;
    if (or_triangle_lagrange_element(v, p, q, ks, km, M.data())) return 1;
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

// Load with per-point source samples (n_q per cell, cell-major) at the rule's
// points; rhs has n_dofs entries.
int or_triangle_lagrange_load_samples(int nv, const double *verts, int nt, const int *tris, int p,
                                      int q, const double *samples, double *rhs) {
  const int nb = or_triangle_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt);
  int ng = 0;
  if (or_triangle_lagrange_dof_map(p, nt, tris, gd.data(), &ng)) return 1;
  TriRule R;
  triangle_rule(q, R);
  const int nq = (int)R.w.size();
  std::fill(rhs, rhs + ng, 0.0);
  std::vector<double> val(nb), grad(2 * nb);
  for (int c = 0; c < nt; ++c) {
    double v[6], J[4], det;
    for (int n = 0; n < 3; ++n)
      for (int d = 0; d < 2; ++d) v[2 * n + d] = verts[2 * tris[3 * c + n] + d];
    if (!tri_geometry(v, J, &det)) return 1;
    for (int pt = 0; pt < nq; ++pt) {
      or_triangle_lagrange_evaluate(p, R.x[pt], R.y[pt], val.data(), grad.data());
      const double f = samples[(size_t)nq * c + pt] * std::fabs(det) * R.w[pt];
      for (int i = 0; i < nb; ++i) rhs[gd[(size_t)nb * c + i]] += f * val[i];
    }
  }
  (void)nv;
  return 0;
}

// Physical points of the rule (2 x n_q x T) and of every DoF (2 x n_dofs).
int or_triangle_lagrange_points(int nv, const double *verts, int nt, const int *tris, int p, int q,
                                double *sample_points, double *dof_points) {
  const int nb = or_triangle_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt), pw;
  std::vector<double> nodes;
  int ng = 0;
  if (or_triangle_lagrange_dof_map(p, nt, tris, gd.data(), &ng)) return 1;
  powers_and_nodes(p, pw, nodes);
  TriRule R;
  triangle_rule(q, R);
  const int nq = (int)R.w.size();
  for (int c = 0; c < nt; ++c) {
    const double *a = verts + 2 * tris[3 * c], *b = verts + 2 * tris[3 * c + 1],
                 *d = verts + 2 * tris[3 * c + 2];
    if (sample_points)
      for (int pt = 0; pt < nq; ++pt)
        for (int k = 0; k < 2; ++k)
          sample_points[2 * ((size_t)nq * c + pt) + k] =
              a[k] + (b[k] - a[k]) * R.x[pt] + (d[k] - a[k]) * R.y[pt];
    if (dof_points)
      for (int l = 0; l < nb; ++l)
        for (int k = 0; k < 2; ++k)
          dof_points[2 * (size_t)gd[(size_t)nb * c + l] + k] =
              a[k] + (b[k] - a[k]) * nodes[2 * l] + (d[k] - a[k]) * nodes[2 * l + 1];
  }
  (void)nv;
  return 0;
}

// DoFs on boundary edges (edges of one triangle).
int or_triangle_lagrange_boundary(int p, int nt, const int *tris, uint8_t *constrained) {
  const int nb = or_triangle_lagrange_dof_count(p);
  std::vector<int> gd((size_t)nb * nt), pw;
  std::vector<double> nodes;
  int ng = 0;
  if (or_triangle_lagrange_dof_map(p, nt, tris, gd.data(), &ng)) return 1;
  powers_and_nodes(p, pw, nodes);
  std::map<std::pair<int, int>, int> cnt;
  for (int c = 0; c < nt; ++c)
    for (int o = 0; o < 3; ++o) {
      int a = tris[3 * c + (o + 1) % 3], b = tris[3 * c + (o + 2) % 3];
      cnt[{std::min(a, b), std::max(a, b)}]++;
    }
  std::fill(constrained, constrained + ng, 0);
  for (int c = 0; c < nt; ++c)
    for (int o = 0; o < 3; ++o) {
      int a = tris[3 * c + (o + 1) % 3], b = tris[3 * c + (o + 2) % 3];
      if (cnt[{std::min(a, b), std::max(a, b)}] != 1) continue;
      for (int l = 0; l < nb; ++l)
        if (pw[3 * l + o] == 0) constrained[gd[(size_t)nb * c + l]] = 1;
    }
  return 0;
}

}  // extern "C"
