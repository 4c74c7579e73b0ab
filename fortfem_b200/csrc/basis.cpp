// Reference-element data of the assembly path: quadrature rules, Lagrange and
// first-kind Nedelec bases, and the reference tensors the per-cell
// contraction uses.
//
// With affine cells and cellwise-constant coefficients every element matrix of
// the reference is a linear combination of a few reference-element matrices:
//   Lagrange (assemble_tetra_lagrange_stiffness_element,
//     src/assembly/assembly_tetra_lagrange_arbitrary_order_3d.f90:40-105):
//     K = k det sum_ab (J^-1 J^-T)_ab R^ab + m det R^mass,
//     R^ab_ij = sum_q w_q dphi_i/dxi_a dphi_j/dxi_b;
//   Nedelec (assemble_tetra_nedelec_curl_mass_element,
//     src/assembly/assembly_tetra_nedelec_3d.f90:584-643, covariant Piola map
//     src/elements/tetra_piola_maps.f90:18-57):
//     K = (c/det) sum_ab (J^T J)_ab C^ab + m det sum_ab (J^-1 J^-T)_ab V^ab.
// The reference tensors are built here from the same quadrature rule and the
// same basis values as the qp-wise reference loop, so the two agree to
// rounding.  Symmetric pairs are folded: for a != b the stored tensor is
// R^ab + R^ba and the geometric factor is the (a,b) entry once.
#include <cmath>
#include <cstring>

#include "ffg_internal.h"
#include "nedelec_tables.inc"

namespace ffg {

void gauss_legendre01(int n, double *x, double *w) {
  // Newton on the Legendre three-term recurrence; nodes ascending on [0,1].
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < n; ++i) {
    double t = std::cos(pi * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = t;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (t * p1 - p0) / (t * t - 1.0);
      double dx = p1 / dp;
      t -= dx;
      if (std::fabs(dx) < 1e-17) break;
    }
    double p0 = 1.0, p1 = t;
    for (int k = 2; k <= n; ++k) {
      double p2 = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    dp = n * (t * p1 - p0) / (t * t - 1.0);
    int j = n - 1 - i;
    x[j] = 0.5 * t + 0.5;
    w[j] = 0.5 * 2.0 / ((1.0 - t * t) * dp * dp);
  }
}

// tetra_duffy_quadrature (src/quadrature/tetra_duffy_quadrature.f90:12-51) or the
// 4-point degree-two rule (assembly_tetra_nedelec_3d.f90:2570-2581).
bool make_rule(int rule, int degree, Rule &r) {
  r = Rule();
  if (rule == FFG_RULE_DEGREE_TWO) {
    const double a = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0;
    const double b = (5.0 - std::sqrt(5.0)) / 20.0;
    const double P[4][3] = {{b, b, b}, {a, b, b}, {b, a, b}, {b, b, a}};
    for (auto &p : P) {
      r.x.push_back(p[0]); r.y.push_back(p[1]); r.z.push_back(p[2]); r.w.push_back(1.0 / 24.0);
    }
    return true;
  }
  if (rule != FFG_RULE_DUFFY || degree < 0) return false;
  int m = (degree + 4) / 2;
  std::vector<double> t(m), tw(m);
  gauss_legendre01(m, t.data(), tw.data());
  for (int a = 0; a < m; ++a)
    for (int b = 0; b < m; ++b)
      for (int c = 0; c < m; ++c) {
        double c1 = 1.0 - t[a], c2 = 1.0 - t[b];
        r.x.push_back(t[a]);
        r.y.push_back(c1 * t[b]);
        r.z.push_back(c1 * c2 * t[c]);
        r.w.push_back(tw[a] * tw[b] * tw[c] * (c1 * c1) * c2);
      }
  return true;
}

int lagrange_dof_count(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }

// DoF ordering of initialize_tetra_lagrange (tetra_lagrange_arbitrary_order.f90:29-66)
void lagrange_indices(int p, std::vector<int> &idx, std::vector<double> &nodes) {
  idx.clear();
  nodes.clear();
  for (int a = 0; a <= p; ++a)
    for (int b = 0; b <= p - a; ++b)
      for (int c = 0; c <= p - a - b; ++c) {
        int d = p - a - b - c;
        idx.insert(idx.end(), {a, b, c, d});
        nodes.insert(nodes.end(), {(double)b / p, (double)c / p, (double)d / p});
      }
}

// evaluate_tetra_lagrange with cardinal_factor (tetra_lagrange_arbitrary_order.f90:68-116,207-249)
void lagrange_eval(int p, const std::vector<int> &idx, const double *pt, double *val,
                   double *grad) {
  int nb = lagrange_dof_count(p);
  double bary[4] = {1.0 - (pt[0] + pt[1] + pt[2]), pt[0], pt[1], pt[2]};
  for (int l = 0; l < nb; ++l) {
    double f[4], d[4];
    for (int c = 0; c < 4; ++c) {
      int n = idx[4 * l + c];
      double fact = 1.0, v = 1.0, dv = 0.0;
      for (int q = 2; q <= n; ++q) fact *= q;
      for (int q = 0; q < n; ++q) v *= (p * bary[c] - q);
      for (int dq = 0; dq < n; ++dq) {
        double term = p;
        for (int q = 0; q < n; ++q)
          if (q != dq) term *= (p * bary[c] - q);
        dv += term;
      }
      f[c] = v / fact;
      d[c] = dv / fact;
    }
    val[l] = f[0] * f[1] * f[2] * f[3];
    double ld[4];
    for (int c = 0; c < 4; ++c) {
      ld[c] = d[c];
      for (int o = 0; o < 4; ++o)
        if (o != c) ld[c] *= f[o];
    }
    for (int a = 0; a < 3; ++a) grad[3 * l + a] = ld[a + 1] - ld[0];
  }
}

int triangle_lagrange_dof_count(int p) { return (p + 1) * (p + 2) / 2; }

// Barycentric powers (first = 1 - x - y, second = x, third = y) and nodes in
// the order of initialize_triangle_lagrange_basis
// (src/elements/triangle_lagrange_arbitrary_order.f90:52-68).
void triangle_lagrange_indices(int p, std::vector<int> &pw, std::vector<double> &nodes) {
  pw.clear();
  nodes.clear();
  for (int a = 0; a <= p; ++a)
    for (int b = 0; b <= p - a; ++b) {
      const int c = p - a - b;
      pw.insert(pw.end(), {a, b, c});
      nodes.insert(nodes.end(), {(double)b / p, (double)c / p});
    }
}

namespace {
double factorial(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= (double)i;
  return r;
}
double ipow_n(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}
// Bernstein polynomials of the barycentric powers and their (x, y) gradients
// (evaluate_bernstein_polynomials, triangle_lagrange_arbitrary_order.f90:143-198).
void triangle_bernstein(int p, const std::vector<int> &pw, double x, double y, double *val,
                        double *grad) {
  const int n = (int)pw.size() / 3;
  const double bary[3] = {1.0 - x - y, x, y};
  for (int d = 0; d < n; ++d) {
    const int e[3] = {pw[3 * d], pw[3 * d + 1], pw[3 * d + 2]};
    const double coef = factorial(p) / (factorial(e[0]) * factorial(e[1]) * factorial(e[2]));
    val[d] = coef * ipow_n(bary[0], e[0]) * ipow_n(bary[1], e[1]) * ipow_n(bary[2], e[2]);
    double der[3];
    for (int k = 0; k < 3; ++k) {
      if (e[k] == 0) { der[k] = 0.0; continue; }
      int r[3] = {e[0], e[1], e[2]};
      r[k] -= 1;
      der[k] = (double)e[k] * ipow_n(bary[0], r[0]) * ipow_n(bary[1], r[1]) * ipow_n(bary[2], r[2]);
    }
    grad[2 * d] = coef * (-der[0] + der[1]);
    grad[2 * d + 1] = coef * (-der[0] + der[2]);
  }
}
}  // namespace

// The nodal basis is the Bernstein basis times the inverse of its Vandermonde
// matrix at the nodes (triangle_lagrange_arbitrary_order.f90:70-88; the
// reference inverts with fortnum's dense_solve, here Gauss-Jordan with
// partial pivoting).  C[m + n b] is the weight of Bernstein polynomial m in
// basis function b.
bool triangle_lagrange_coefficients(int p, std::vector<double> &C) {
  std::vector<int> pw;
  std::vector<double> nodes;
  triangle_lagrange_indices(p, pw, nodes);
  const int n = (int)pw.size() / 3;
  std::vector<double> V((size_t)n * n), row(n), g(2 * (size_t)n);
  for (int d = 0; d < n; ++d) {
    triangle_bernstein(p, pw, nodes[2 * d], nodes[2 * d + 1], row.data(), g.data());
    for (int m = 0; m < n; ++m) V[d + (size_t)n * m] = row[m];
  }
  C.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) C[i + (size_t)n * i] = 1.0;
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (std::fabs(V[r + (size_t)n * col]) > std::fabs(V[piv + (size_t)n * col])) piv = r;
    if (V[piv + (size_t)n * col] == 0.0) return false;
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

// Values and (x, y) gradients of the nodal triangle basis at (x, y).
void triangle_lagrange_eval(int p, const std::vector<int> &pw, const std::vector<double> &C,
                            double x, double y, double *val, double *grad) {
  const int n = (int)pw.size() / 3;
  std::vector<double> bv(n), bg(2 * (size_t)n);
  triangle_bernstein(p, pw, x, y, bv.data(), bg.data());
  for (int b = 0; b < n; ++b) {
    double v = 0.0, gx = 0.0, gy = 0.0;
    for (int m = 0; m < n; ++m) {
      const double c = C[m + (size_t)n * b];
      v += c * bv[m];
      gx += c * bg[2 * m];
      gy += c * bg[2 * m + 1];
    }
    val[b] = v;
    grad[2 * b] = gx;
    grad[2 * b + 1] = gy;
  }
}

// triangle_duffy_quadrature (src/quadrature/triangle_duffy_quadrature.f90:12-45):
// (q + 3) / 2 Gauss points per direction, x = t_a, y = (1 - t_a) t_b.
void triangle_rule(int q, std::vector<double> &x, std::vector<double> &y, std::vector<double> &w) {
  const int m = (q + 3) / 2;
  std::vector<double> t(m), tw(m);
  gauss_legendre01(m, t.data(), tw.data());
  x.clear(); y.clear(); w.clear();
  for (int a = 0; a < m; ++a)
    for (int b = 0; b < m; ++b) {
      x.push_back(t[a]);
      y.push_back((1.0 - t[a]) * t[b]);
      w.push_back(tw[a] * tw[b] * (1.0 - t[a]));
    }
}

int nedelec_dof_count(int k) { return k * (k + 2) * (k + 3) / 2; }

static double ipow(double x, int n) {
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

// Candidate monomial space of evaluate_runtime_candidates (order <= 5; order 6
// uses the same construction, see gen_nedelec_tables.py;
// tetra_nedelec_arbitrary_order.f90:318-396) times the exact dual-basis
// coefficients (evaluate_tetra_nedelec_first_kind, :75-106).
void nedelec_candidate_terms(int k, std::vector<int> &terms) {
  terms.clear();
  auto add = [&](int c0, int s0, int a0, int b0, int z0, int c1, int s1, int a1, int b1, int z1) {
    terms.insert(terms.end(), {c0, s0, a0, b0, z0, c1, s1, a1, b1, z1});
  };
  for (int comp = 0; comp < 3; ++comp)
    for (int d = 0; d < k; ++d)
      for (int a = 0; a <= d; ++a)
        for (int b = 0; b <= d - a; ++b) add(comp, 1, a, b, d - a - b, -1, 0, 0, 0, 0);
  const int d = k - 1;
  for (int fam = 0; fam < 2; ++fam)
    for (int a = 0; a <= d; ++a)
      for (int b = 0; b <= d - a; ++b) {
        const int c = d - a - b;
        if (fam == 0)
          add(0, -1, a, b + 1, c, 1, 1, a + 1, b, c);
        else
          add(0, -1, a, b, c + 1, 2, 1, a + 1, b, c);
      }
  for (int b = 0; b <= d; ++b) {
    const int c = d - b;
    add(1, -1, 0, b, c + 1, 2, 1, 0, b + 1, c);
  }
}

const double *nedelec_coefficients(int k) {
  return (k >= 1 && k <= FFG_NEDELEC_TABLE_MAX_ORDER) ? kNedelecCoefficientTables[k] : nullptr;
}

bool nedelec_eval(int k, const double *pt, double *val, double *curl) {
  if (k < 1 || k > FFG_NEDELEC_TABLE_MAX_ORDER) return false;
  const int n = nedelec_dof_count(k);
  std::vector<int> terms;
  nedelec_candidate_terms(k, terms);
  std::vector<double> cv(3 * n, 0.0), cc(3 * n, 0.0);
  for (int cand = 0; cand < n; ++cand)
    for (int t = 0; t < 2; ++t) {
      const int *tm = &terms[10 * (size_t)cand + 5 * t];
      const int comp = tm[0];
      if (comp < 0) continue;
      const double coef = tm[1];
      const int pw[3] = {tm[2], tm[3], tm[4]};
      cv[3 * cand + comp] += coef * ipow(pt[0], pw[0]) * ipow(pt[1], pw[1]) * ipow(pt[2], pw[2]);
      double der[3];
      for (int dd = 0; dd < 3; ++dd) {
        if (pw[dd] == 0) { der[dd] = 0.0; continue; }
        int r[3] = {pw[0], pw[1], pw[2]};
        r[dd] -= 1;
        der[dd] = coef * pw[dd] * ipow(pt[0], r[0]) * ipow(pt[1], r[1]) * ipow(pt[2], r[2]);
      }
      double *cu = &cc[3 * cand];
      if (comp == 0) { cu[1] += der[2]; cu[2] -= der[1]; }
      if (comp == 1) { cu[0] -= der[2]; cu[2] += der[0]; }
      if (comp == 2) { cu[0] += der[1]; cu[1] -= der[0]; }
    }
  const double *C = kNedelecCoefficientTables[k];
  for (int bf = 0; bf < n; ++bf)
    for (int a = 0; a < 3; ++a) {
      double s = 0.0, t = 0.0;
      for (int c = 0; c < n; ++c) {
        s += cv[3 * c + a] * C[c + (size_t)n * bf];
        t += cc[3 * c + a] * C[c + (size_t)n * bf];
      }
      val[3 * bf + a] = s;
      curl[3 * bf + a] = t;
    }
  return true;
}

const double *face_transform_table(int k, int p) { return kFaceTransformTable(k, p); }

static const int kPairA[6] = {0, 1, 2, 0, 0, 1};
static const int kPairB[6] = {0, 1, 2, 1, 2, 2};

int build_tables(const Topology &t, int rule, int qdeg, ElementTables &tab, std::string &msg) {
  tab = ElementTables();
  tab.nb = t.nb;
  const int nb = t.nb;
  if (t.family == FFG_TRIANGLE_P1) {
    tab.n_terms = 0;
    tab.nq_load = 1;
    return FFG_OK;
  }
  if (t.family == FFG_TRIANGLE_LAGRANGE) {
    // K = sum_ab kappa |det| (J^-1 J^-T)_ab R^ab + m |det| R^mass, pairs
    // (0,0), (1,1), (0,1); one Duffy rule of degree qdeg for matrix and load
    if (qdeg < 0) { msg = "bad quadrature degree"; return FFG_INVALID_INPUT; }
    std::vector<int> pw;
    std::vector<double> nodes, C, qx, qy, qw;
    triangle_lagrange_indices(t.degree, pw, nodes);
    if (!triangle_lagrange_coefficients(t.degree, C)) {
      msg = "singular triangle Vandermonde matrix";
      return FFG_INVALID_INPUT;
    }
    triangle_rule(qdeg, qx, qy, qw);
    const int nq = (int)qw.size();
    std::vector<double> val((size_t)nq * nb), grad((size_t)nq * nb * 2);
    for (int q = 0; q < nq; ++q)
      triangle_lagrange_eval(t.degree, pw, C, qx[q], qy[q], &val[(size_t)q * nb],
                             &grad[(size_t)q * nb * 2]);
    const int pa[3] = {0, 1, 0}, pb[3] = {0, 1, 1};
    tab.n_terms = 4;
    tab.ref.assign((size_t)4 * nb * nb, 0.0);
    for (int s = 0; s < 3; ++s) {
      const int a = pa[s], b = pb[s];
      double *M = &tab.ref[(size_t)s * nb * nb];
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) {
          double acc = 0.0;
          for (int q = 0; q < nq; ++q) {
            const double *g = &grad[(size_t)q * nb * 2];
            double v = g[2 * i + a] * g[2 * j + b];
            if (a != b) v += g[2 * i + b] * g[2 * j + a];
            acc += qw[q] * v;
          }
          M[i + (size_t)nb * j] = acc;
        }
    }
    double *Mm = &tab.ref[(size_t)3 * nb * nb];
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        double acc = 0.0;
        for (int q = 0; q < nq; ++q) acc += qw[q] * val[(size_t)q * nb + i] * val[(size_t)q * nb + j];
        Mm[i + (size_t)nb * j] = acc;
      }
    tab.nq_load = nq;
    tab.load_basis.assign((size_t)nq * nb, 0.0);
    tab.load_xi.assign((size_t)nq * 3, 0.0);
    for (int q = 0; q < nq; ++q) {
      for (int i = 0; i < nb; ++i) tab.load_basis[(size_t)q * nb + i] = qw[q] * val[(size_t)q * nb + i];
      tab.load_xi[3 * q] = qx[q];
      tab.load_xi[3 * q + 1] = qy[q];
    }
    return FFG_OK;
  }
  if (t.family == FFG_TETRA_LAGRANGE) {
    Rule R;
    if (!make_rule(rule, qdeg, R)) { msg = "bad quadrature rule"; return FFG_INVALID_INPUT; }
    std::vector<int> idx;
    std::vector<double> nodes;
    lagrange_indices(t.degree, idx, nodes);
    const int nq = R.size();
    std::vector<double> val((size_t)nq * nb), grad((size_t)nq * nb * 3);
    for (int q = 0; q < nq; ++q) {
      double P[3] = {R.x[q], R.y[q], R.z[q]};
      lagrange_eval(t.degree, idx, P, &val[(size_t)q * nb], &grad[(size_t)q * nb * 3]);
    }
    tab.n_terms = 7;
    tab.ref.assign((size_t)7 * nb * nb, 0.0);
    for (int s = 0; s < 6; ++s) {
      int a = kPairA[s], b = kPairB[s];
      double *M = &tab.ref[(size_t)s * nb * nb];
      for (int j = 0; j < nb; ++j)
        for (int i = 0; i < nb; ++i) {
          double acc = 0.0;
          for (int q = 0; q < nq; ++q) {
            const double *g = &grad[(size_t)q * nb * 3];
            double v = g[3 * i + a] * g[3 * j + b];
            if (a != b) v += g[3 * i + b] * g[3 * j + a];
            acc += R.w[q] * v;
          }
          M[i + (size_t)nb * j] = acc;
        }
    }
    double *Mm = &tab.ref[(size_t)6 * nb * nb];
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        double acc = 0.0;
        for (int q = 0; q < nq; ++q) acc += R.w[q] * val[(size_t)q * nb + i] * val[(size_t)q * nb + j];
        Mm[i + (size_t)nb * j] = acc;
      }
    tab.nq_load = nq;
    tab.load_basis.assign((size_t)nq * nb, 0.0);
    tab.load_xi.assign((size_t)nq * 3, 0.0);
    for (int q = 0; q < nq; ++q) {
      for (int i = 0; i < nb; ++i) tab.load_basis[(size_t)q * nb + i] = R.w[q] * val[(size_t)q * nb + i];
      tab.load_xi[3 * q] = R.x[q]; tab.load_xi[3 * q + 1] = R.y[q]; tab.load_xi[3 * q + 2] = R.z[q];
    }
    return FFG_OK;
  }
  // Nedelec
  const int k = t.degree;
  Rule R, RL;
  // matrix: order 1 -> 4-point rule (assemble_tetra_nedelec_element :2357-2404),
  // order >= 2 -> Duffy 2k (assemble_arbitrary_order_curl_mass_csc :2331-2333);
  // load: order 1 -> 4-point rule (:2516-2553), order >= 2 -> Duffy 2k+2 (:547)
  make_rule(k == 1 ? FFG_RULE_DEGREE_TWO : FFG_RULE_DUFFY, 2 * k, R);
  make_rule(k == 1 ? FFG_RULE_DEGREE_TWO : FFG_RULE_DUFFY, 2 * k + 2, RL);
  const int nq = R.size();
  std::vector<double> v((size_t)nq * nb * 3), c((size_t)nq * nb * 3);
  for (int q = 0; q < nq; ++q) {
    double P[3] = {R.x[q], R.y[q], R.z[q]};
    if (!nedelec_eval(k, P, &v[(size_t)q * nb * 3], &c[(size_t)q * nb * 3])) {
      msg = "Nedelec order not tabulated";
      return FFG_INVALID_INPUT;
    }
  }
  tab.n_terms = 12;
  tab.ref.assign((size_t)12 * nb * nb, 0.0);
  for (int s = 0; s < 12; ++s) {
    const std::vector<double> &B = (s < 6) ? c : v;
    int a = kPairA[s % 6], b = kPairB[s % 6];
    double *M = &tab.ref[(size_t)s * nb * nb];
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        double acc = 0.0;
        for (int q = 0; q < nq; ++q) {
          const double *g = &B[(size_t)q * nb * 3];
          double x = g[3 * i + a] * g[3 * j + b];
          if (a != b) x += g[3 * i + b] * g[3 * j + a];
          acc += R.w[q] * x;
        }
        M[i + (size_t)nb * j] = acc;
      }
  }
  const int nql = RL.size();
  tab.nq_load = nql;
  tab.load_basis.assign((size_t)nql * nb * 3, 0.0);
  tab.load_xi.assign((size_t)nql * 3, 0.0);
  std::vector<double> lv((size_t)nb * 3), lc((size_t)nb * 3);
  for (int q = 0; q < nql; ++q) {
    double P[3] = {RL.x[q], RL.y[q], RL.z[q]};
    nedelec_eval(k, P, lv.data(), lc.data());
    for (int i = 0; i < nb * 3; ++i) tab.load_basis[(size_t)q * nb * 3 + i] = RL.w[q] * lv[i];
    tab.load_xi[3 * q] = RL.x[q]; tab.load_xi[3 * q + 1] = RL.y[q]; tab.load_xi[3 * q + 2] = RL.z[q];
  }
  const int fdc = k * (k - 1);
  if (fdc > 0) {
    tab.face_blocks.assign((size_t)6 * fdc * fdc, 0.0);
    for (int p = 0; p < 6; ++p)
      std::memcpy(&tab.face_blocks[(size_t)p * fdc * fdc], face_transform_table(k, p),
                  sizeof(double) * fdc * fdc);
  }
  return FFG_OK;
}

int geo_stride_for(const Topology &t, const ElementTables &tab) {
  switch (t.family) {
    case FFG_TETRA_LAGRANGE: return 7 + tab.nq_load;
    case FFG_TETRA_NEDELEC: return 12;
    case FFG_TRIANGLE_P1: return 10;
    case FFG_TRIANGLE_LAGRANGE: return 4 + tab.nq_load;
  }
  return 0;
}

}  // namespace ffg
