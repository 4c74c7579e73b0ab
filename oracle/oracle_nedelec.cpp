// fortfem hot-path ORACLE (test infrastructure only; see oracle.h).
//
// FP64 CPU restatement of first-kind tetrahedral Nedelec assembly: candidate
// evaluation x dual-basis coefficients, covariant Piola map, edge/face DoF
// numbering, orientation transforms, curl-mass element and CSC, sampled loads
// and the zero-tangential (PEC) mask.  The exact coefficient and face tables
// are the repository's generated data (fortfem_b200/csrc/nedelec_tables.inc),
// which the tests pin against the reference's own generated tables.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../fortfem_b200/csrc/nedelec_tables.inc"

namespace {
const double kEps = 2.220446049250313e-16;

double det3(const double *J) {
  return J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
         J[6] * (J[1] * J[5] - J[4] * J[2]);
}
void inv3(const double *J, double det, double *Ji) {
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
// tetra_geometry, src/assembly/assembly_tetra_nedelec_3d.f90:2555-2568
bool tetra_geometry(const double *v, double *J, double *det) {
  tetra_jacobian(v, J);
  *det = det3(J);
  double m = 0.0;
  for (int i = 0; i < 9; ++i) m = std::max(m, std::fabs(J[i]));
  double s = std::max(1.0, m);
  return *det > 64.0 * kEps * s * s * s;
}

double ipow(double x, int n) {
  // Fortran x**n for small non-negative integer n
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

struct Term {
  int comp;
  double coef;
  int pw[3];
};

// Candidate list of evaluate_runtime_candidates for order <= 5,
// src/elements/tetra_nedelec_arbitrary_order.f90:318-396.
std::vector<std::vector<Term>> candidate_terms(int k) {
  std::vector<std::vector<Term>> c;
  for (int comp = 0; comp < 3; ++comp)
    for (int d = 0; d <= k - 1; ++d)
      for (int a = 0; a <= d; ++a)
        for (int b = 0; b <= d - a; ++b) c.push_back({{comp, 1.0, {a, b, d - a - b}}});
  int d = k - 1;
  for (int fam = 4; fam <= 5; ++fam)
    for (int a = 0; a <= d; ++a)
      for (int b = 0; b <= d - a; ++b) {
        int cc = d - a - b;
        if (fam == 4)
          c.push_back({{0, -1.0, {a, b + 1, cc}}, {1, 1.0, {a + 1, b, cc}}});
        else
          c.push_back({{0, -1.0, {a, b, cc + 1}}, {2, 1.0, {a + 1, b, cc}}});
      }
  for (int b = 0; b <= d; ++b) {
    int cc = d - b;
    c.push_back({{1, -1.0, {0, b, cc + 1}}, {2, 1.0, {0, b + 1, cc}}});
  }
  return c;
}

// add_candidate_term, tetra_nedelec_arbitrary_order.f90:710-737
void candidates(int k, const double *p, double *vals, double *curls) {
  auto terms = candidate_terms(k);
  int n = (int)terms.size();
  std::fill(vals, vals + 3 * n, 0.0);
  std::fill(curls, curls + 3 * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (auto &t : terms[i]) {
      double value = t.coef * ipow(p[0], t.pw[0]) * ipow(p[1], t.pw[1]) * ipow(p[2], t.pw[2]);
      double der[3];
      for (int dir = 0; dir < 3; ++dir) {
        if (t.pw[dir] == 0) { der[dir] = 0.0; continue; }
        int red[3] = {t.pw[0], t.pw[1], t.pw[2]};
        red[dir] -= 1;
        der[dir] = t.coef * ((double)t.pw[dir] *
                             (ipow(p[0], red[0]) * ipow(p[1], red[1]) * ipow(p[2], red[2])));
      }
      vals[3 * i + t.comp] += value;
      double *cu = curls + 3 * i;
      switch (t.comp) {
        case 0: cu[1] += der[2]; cu[2] -= der[1]; break;
        case 1: cu[0] -= der[2]; cu[2] += der[0]; break;
        case 2: cu[0] += der[1]; cu[1] -= der[0]; break;
      }
    }
}

int face_perm_index(const int *perm) {
  int code = 100 * perm[0] + 10 * perm[1] + perm[2];
  switch (code) {
    case 123: return 0;
    case 132: return 1;
    case 213: return 2;
    case 231: return 3;
    case 312: return 4;
    case 321: return 5;
  }
  return -1;
}

struct RuleN {
  std::vector<double> x, y, z, w;
};
bool make_rule(int rule, int q, RuleN &r) {
  if (rule == 1) {
    double P[12], W[4];
    or_tetra_degree_two_rule(P, W);
    for (int i = 0; i < 4; ++i) {
      r.x.push_back(P[3 * i]); r.y.push_back(P[3 * i + 1]); r.z.push_back(P[3 * i + 2]);
      r.w.push_back(W[i]);
    }
    return true;
  }
  if (q < 0) return false;
  int n = or_tetra_duffy_count(q);
  r.x.resize(n); r.y.resize(n); r.z.resize(n); r.w.resize(n);
  or_tetra_duffy(q, r.x.data(), r.y.data(), r.z.data(), r.w.data());
  return true;
}

// map_tetra_nedelec_covariant, src/elements/tetra_piola_maps.f90:18-57
void covariant(const double *J, double det, const double *Ji, int n, const double *rv,
               const double *rc, double *pv, double *pc) {
  for (int b = 0; b < n; ++b)
    for (int i = 0; i < 3; ++i) {
      double s = 0.0, t = 0.0;
      for (int k = 0; k < 3; ++k) {
        s += Ji[k + 3 * i] * rv[3 * b + k];  // transpose(Ji) * v
        t += J[i + 3 * k] * rc[3 * b + k];   // J * c
      }
      pv[3 * b + i] = s;
      pc[3 * b + i] = t / det;
    }
}
}  // namespace

extern "C" {

int or_nedelec_dof_count(int k) { return k * (k + 2) * (k + 3) / 2; }

// evaluate_tetra_nedelec_first_kind, tetra_nedelec_arbitrary_order.f90:75-106
int or_nedelec_evaluate(int k, const double *p, double *vals, double *curls) {
  if (k < 1 || k > FFG_NEDELEC_TABLE_MAX_ORDER) return 1;
  double tol = 64.0 * kEps;
  if (p[0] < -tol || p[1] < -tol || p[2] < -tol) return 1;
  if (p[0] + p[1] + p[2] > 1.0 + tol) return 1;
  int n = or_nedelec_dof_count(k);
  std::vector<double> cv(3 * n), cc(3 * n);
  candidates(k, p, cv.data(), cc.data());
  const double *C = kNedelecCoefficientTables[k];
  for (int b = 0; b < n; ++b)
    for (int i = 0; i < 3; ++i) {
      double s = 0.0, t = 0.0;
      for (int c = 0; c < n; ++c) {
        s += cv[3 * c + i] * C[c + (size_t)n * b];
        t += cc[3 * c + i] * C[c + (size_t)n * b];
      }
      vals[3 * b + i] = s;
      curls[3 * b + i] = t;
    }
  return 0;
}

// evaluate_tetra_nedelec_first_order, src/elements/tetra_nedelec_first_order.f90:11-51
int or_whitney_evaluate(const double *p, double *vals, double *curls) {
  double tol = 64.0 * kEps;
  double lam[4] = {1.0 - p[0] - p[1] - p[2], p[0], p[1], p[2]};
  for (int i = 0; i < 4; ++i)
    if (lam[i] < -tol || lam[i] > 1.0 + tol) return 1;
  const double g[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const int ev[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  for (int e = 0; e < 6; ++e) {
    int a = ev[e][0], b = ev[e][1];
    for (int i = 0; i < 3; ++i) vals[3 * e + i] = lam[a] * g[b][i] - lam[b] * g[a][i];
    curls[3 * e + 0] = 2.0 * (g[a][1] * g[b][2] - g[a][2] * g[b][1]);
    curls[3 * e + 1] = 2.0 * (g[a][2] * g[b][0] - g[a][0] * g[b][2]);
    curls[3 * e + 2] = 2.0 * (g[a][0] * g[b][1] - g[a][1] * g[b][0]);
  }
  return 0;
}

static const int kLocalEdges[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
static const int kLocalFaces[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

static bool distinct4(const int *t) {
  for (int a = 0; a < 4; ++a)
    for (int b = a + 1; b < 4; ++b)
      if (t[a] == t[b]) return false;
  return true;
}

// build_tetra_edge_dof_map, src/elements/tetra_edge_dof_map.f90:10-77 (literal,
// linear search :54-60).  edges: 2 x E (zero-based vertex ids).
int or_edge_dof_map_faithful(int nt, const int *tets, int *edges, int *gd, int *orient,
                             int *n_edges) {
  if (nt < 1) return 1;
  for (int i = 0; i < 4 * nt; ++i)
    if (tets[i] < 0) return 1;
  std::vector<std::pair<int, int>> ed;
  for (int t = 0; t < nt; ++t) {
    if (!distinct4(tets + 4 * t)) return 1;
    for (int le = 0; le < 6; ++le) {
      int fv = tets[4 * t + kLocalEdges[le][0]], sv = tets[4 * t + kLocalEdges[le][1]];
      int a = std::min(fv, sv), b = std::max(fv, sv);
      int found = -1;
      for (size_t e = 0; e < ed.size(); ++e)
        if (ed[e].first == a && ed[e].second == b) { found = (int)e; break; }
      if (found < 0) { ed.emplace_back(a, b); found = (int)ed.size() - 1; }
      gd[6 * t + le] = found;
      orient[6 * t + le] = (fv < sv) ? 1 : -1;
    }
  }
  *n_edges = (int)ed.size();
  if (edges)
    for (size_t e = 0; e < ed.size(); ++e) { edges[2 * e] = ed[e].first; edges[2 * e + 1] = ed[e].second; }
  return 0;
}

int or_edge_dof_map(int nt, const int *tets, int *edges, int *gd, int *orient, int *n_edges) {
  if (nt < 1) return 1;
  for (int i = 0; i < 4 * nt; ++i)
    if (tets[i] < 0) return 1;
  std::unordered_map<uint64_t, int> map;
  map.reserve((size_t)nt * 2);
  std::vector<std::pair<int, int>> ed;
  for (int t = 0; t < nt; ++t) {
    if (!distinct4(tets + 4 * t)) return 1;
    for (int le = 0; le < 6; ++le) {
      int fv = tets[4 * t + kLocalEdges[le][0]], sv = tets[4 * t + kLocalEdges[le][1]];
      int a = std::min(fv, sv), b = std::max(fv, sv);
      uint64_t key = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
      auto it = map.find(key);
      int id;
      if (it == map.end()) { id = (int)ed.size(); ed.emplace_back(a, b); map.emplace(key, id); }
      else id = it->second;
      gd[6 * t + le] = id;
      orient[6 * t + le] = (fv < sv) ? 1 : -1;
    }
  }
  *n_edges = (int)ed.size();
  if (edges)
    for (size_t e = 0; e < ed.size(); ++e) { edges[2 * e] = ed[e].first; edges[2 * e + 1] = ed[e].second; }
  return 0;
}

// build_tetra_nedelec_dof_map, src/elements/tetra_nedelec_global_dof_map.f90:15-105.
// Output arrays: edges 2 x E, faces 3 x F (sorted vertex triples), global_dofs
// n_b x T, edge_orientations 6 x T, face_permutations 3 x 4 x T (1-based
// positions as in the reference).  Pass null output pointers to query counts.
int or_nedelec_dof_map(int k, int nt, const int *tets, int faithful, int *edges, int *n_edges,
                       int *faces, int *n_faces, int *gd, int *eo, int *fp, int *n_global) {
  if (k < 1) return 1;
  std::vector<int> egd(6 * (size_t)nt), eor(6 * (size_t)nt);
  int ne = 0;
  std::vector<int> edv(2 * (size_t)nt * 6);
  int st = faithful ? or_edge_dof_map_faithful(nt, tets, edv.data(), egd.data(), eor.data(), &ne)
                    : or_edge_dof_map(nt, tets, edv.data(), egd.data(), eor.data(), &ne);
  if (st) return st;
  int nb = or_nedelec_dof_count(k);
  int fdc = k * (k - 1), cdc = k * (k - 1) * (k - 2) / 2;
  int64_t edc = (int64_t)k * ne;
  std::vector<std::array<int, 3>> fl;
  std::unordered_map<uint64_t, int> fmap;
  if (!faithful) fmap.reserve((size_t)nt * 3);
  std::vector<int> tgd(gd ? 0 : (size_t)nb * nt);
  int *G = gd ? gd : tgd.data();
  for (int t = 0; t < nt; ++t)
    for (int e = 0; e < 6; ++e)
      for (int m = 0; m < k; ++m) G[(size_t)nb * t + e * k + m] = (int)((int64_t)egd[6 * t + e] * k + m);
  std::vector<int> face_of(4 * (size_t)nt);
  for (int t = 0; t < nt; ++t)
    for (int lf = 0; lf < 4; ++lf) {
      int lv[3], cv[3];
      for (int i = 0; i < 3; ++i) lv[i] = cv[i] = tets[4 * t + kLocalFaces[lf][i]];
      std::sort(cv, cv + 3);  // sort_three
      int found = -1;
      if (faithful) {
        for (size_t f = 0; f < fl.size(); ++f)
          if (fl[f][0] == cv[0] && fl[f][1] == cv[1] && fl[f][2] == cv[2]) { found = (int)f; break; }
      } else {
        uint64_t key = ((uint64_t)(uint32_t)cv[0] << 42) ^ ((uint64_t)(uint32_t)cv[1] << 21) ^
                       (uint64_t)(uint32_t)cv[2];
        auto it = fmap.find(key);
        if (it != fmap.end()) found = it->second;
        else { fmap.emplace(key, (int)fl.size()); }
      }
      if (found < 0) { fl.push_back({cv[0], cv[1], cv[2]}); found = (int)fl.size() - 1; }
      face_of[4 * t + lf] = found;
      if (fp)
        for (int i = 0; i < 3; ++i) {
          int pos = 0;
          for (int j = 0; j < 3; ++j)
            if (cv[j] == lv[i]) { pos = j + 1; break; }
          fp[(size_t)12 * t + 3 * lf + i] = pos;
        }
      int fs = 6 * k + lf * fdc;
      for (int m = 0; m < fdc; ++m)
        G[(size_t)nb * t + fs + m] = (int)(edc + (int64_t)found * fdc + m);
    }
  int nf = (int)fl.size();
  int cs = 6 * k + 4 * fdc;
  for (int t = 0; t < nt; ++t)
    for (int m = 0; m < cdc; ++m)
      G[(size_t)nb * t + cs + m] = (int)(edc + (int64_t)nf * fdc + (int64_t)t * cdc + m);
  if (n_edges) *n_edges = ne;
  if (n_faces) *n_faces = nf;
  if (n_global) *n_global = (int)(edc + (int64_t)nf * fdc + (int64_t)nt * cdc);
  if (edges) std::memcpy(edges, edv.data(), sizeof(int) * 2 * ne);
  if (faces)
    for (int f = 0; f < nf; ++f)
      for (int i = 0; i < 3; ++i) faces[3 * f + i] = fl[f][i];
  if (eo) std::memcpy(eo, eor.data(), sizeof(int) * 6 * (size_t)nt);
  return 0;
}

// build_tetra_face_basis_to_local_matrix, tetra_face_moment_transforms.f90:23-52
// (generated tables for the orders the repository tabulates).
int or_face_basis_to_local(int k, const int *perm, double *T) {
  int m = k * (k - 1);
  int pi = face_perm_index(perm);
  if (pi < 0 || k < 2 || k > FFG_NEDELEC_TABLE_MAX_ORDER) return 1;
  std::memcpy(T, kFaceTransformTable(k, pi), sizeof(double) * m * m);
  return 0;
}

// build_tetra_nedelec_basis_transform, tetra_nedelec_global_dof_map.f90:107-155
int or_nedelec_transform(int k, const int *eo, const int *fp, double *T) {
  int n = or_nedelec_dof_count(k);
  std::fill(T, T + (size_t)n * n, 0.0);
  for (int d = 0; d < n; ++d) T[d + (size_t)n * d] = 1.0;
  for (int e = 0; e < 6; ++e) {
    if (eo[e] == 1) continue;
    if (eo[e] != -1) return 1;
    for (int m = 0; m < k; m += 2) {
      int s = e * k + m;
      T[s + (size_t)n * s] = -1.0;
    }
  }
  int fdc = k * (k - 1);
  if (fdc == 0) return 0;
  std::vector<double> F((size_t)fdc * fdc);
  for (int f = 0; f < 4; ++f) {
    int s = 6 * k + f * fdc;
    if (or_face_basis_to_local(k, fp + 3 * f, F.data())) return 1;
    for (int c = 0; c < fdc; ++c)
      for (int r = 0; r < fdc; ++r) T[(s + r) + (size_t)n * (s + c)] = F[r + (size_t)fdc * c];
  }
  return 0;
}

// assemble_tetra_nedelec_curl_mass_element, src/assembly/assembly_tetra_nedelec_3d.f90:584-643
int or_nedelec_element(const double *v, int k, int q, double cw, double mw, double *M) {
  if (k < 1 || q < 0) return 1;
  double J[9], Ji[9], det;
  if (!tetra_geometry(v, J, &det)) return 1;
  inv3(J, det, Ji);
  RuleN R;
  make_rule(0, q, R);
  int n = or_nedelec_dof_count(k);
  std::vector<double> rv(3 * n), rc(3 * n), pv(3 * n), pc(3 * n);
  std::fill(M, M + (size_t)n * n, 0.0);
  for (size_t pt = 0; pt < R.w.size(); ++pt) {
    double P[3] = {R.x[pt], R.y[pt], R.z[pt]};
    if (or_nedelec_evaluate(k, P, rv.data(), rc.data())) return 1;
    covariant(J, det, Ji, n, rv.data(), rc.data(), pv.data(), pc.data());
    double pw = det * R.w[pt];
    for (int col = 0; col < n; ++col)
      for (int row = 0; row < n; ++row) {
        double dc = 0.0, dv = 0.0;
        for (int i = 0; i < 3; ++i) dc += pc[3 * row + i] * pc[3 * col + i];
        for (int i = 0; i < 3; ++i) dv += pv[3 * row + i] * pv[3 * col + i];
        M[row + (size_t)n * col] += pw * (cw * dc + mw * dv);
      }
  }
  return 0;
}

// assemble_tetra_nedelec_element (order 1, 4-point rule), assembly_tetra_nedelec_3d.f90:2357-2404
int or_nedelec_whitney_element(const double *v, double cw, double mw, double *M) {
  double J[9], Ji[9], det;
  if (!tetra_geometry(v, J, &det)) return 1;
  inv3(J, det, Ji);
  double P[12], W[4];
  or_tetra_degree_two_rule(P, W);
  double rv[18], rc[18], pv[18], pc[18];
  std::fill(M, M + 36, 0.0);
  for (int pt = 0; pt < 4; ++pt) {
    if (or_whitney_evaluate(P + 3 * pt, rv, rc)) return 1;
    covariant(J, det, Ji, 6, rv, rc, pv, pc);
    for (int col = 0; col < 6; ++col)
      for (int row = 0; row < 6; ++row) {
        double dc = 0.0, dv = 0.0;
        for (int i = 0; i < 3; ++i) dc += pc[3 * row + i] * pc[3 * col + i];
        for (int i = 0; i < 3; ++i) dv += pv[3 * row + i] * pv[3 * col + i];
        M[row + 6 * col] += det * (1.0 / 24.0) * (cw * dc + mw * dv);
      }
  }
  return 0;
}

int64_t or_nedelec_csc_nnz(int k, int nt, const int *tets) {
  int nb = or_nedelec_dof_count(k), ng = 0;
  std::vector<int> gd((size_t)nb * nt);
  if (or_nedelec_dof_map(k, nt, tets, 0, nullptr, nullptr, nullptr, nullptr, gd.data(), nullptr,
                         nullptr, &ng))
    return -1;
  std::vector<uint64_t> keys;
  keys.reserve((size_t)nt * nb * nb);
  for (int t = 0; t < nt; ++t)
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i)
        keys.push_back(((uint64_t)gd[(size_t)nb * t + j] << 32) | (uint32_t)gd[(size_t)nb * t + i]);
  std::sort(keys.begin(), keys.end());
  return std::unique(keys.begin(), keys.end()) - keys.begin();
}

// assemble_tetra_nedelec_curl_mass_csc (order 1: :2042-2112 with s_i s_j; order >= 2:
// assemble_arbitrary_order_curl_mass_csc :2289-2355 with T^T K T and q = 2k).
// Optional per-cell arrays scale the curl / mass coefficients cellwise.
int or_nedelec_csc(int nv, const double *verts, int nt, const int *tets, int k, double cw,
                   double mw, const double *ccurl, const double *cmass, int64_t cap, int *n_dofs,
                   int64_t *nnz, int64_t *col_ptr, int *row_idx, double *values) {
  if (k < 1 || nt < 1) return 1;
  for (int i = 0; i < 4 * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  int nb = or_nedelec_dof_count(k), ng = 0;
  std::vector<int> gd((size_t)nb * nt), eo(6 * (size_t)nt), fp(12 * (size_t)nt);
  if (or_nedelec_dof_map(k, nt, tets, 0, nullptr, nullptr, nullptr, nullptr, gd.data(), eo.data(),
                         fp.data(), &ng))
    return 1;
  *n_dofs = ng;
  int64_t ntrip = (int64_t)nt * nb * nb;
  std::vector<int> rows(ntrip), cols(ntrip);
  std::vector<double> tv(ntrip), K((size_t)nb * nb), T((size_t)nb * nb), KT((size_t)nb * nb),
      O((size_t)nb * nb);
  int64_t e = 0;
  for (int t = 0; t < nt; ++t) {
    double v[12];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * t + n] + d];
    double c = ccurl ? cw * ccurl[t] : cw, m = cmass ? mw * cmass[t] : mw;
    if (k == 1) {
      if (or_nedelec_whitney_element(v, c, m, K.data())) return 1;
      for (int col = 0; col < 6; ++col)
        for (int row = 0; row < 6; ++row, ++e) {
          rows[e] = gd[(size_t)nb * t + row];
          cols[e] = gd[(size_t)nb * t + col];
          tv[e] = (double)(eo[6 * t + row] * eo[6 * t + col]) * K[row + 6 * col];
        }
      continue;
    }
    if (or_nedelec_element(v, k, 2 * k, c, m, K.data())) return 1;
    if (or_nedelec_transform(k, eo.data() + 6 * t, fp.data() + 12 * t, T.data())) return 1;
    // oriented = matmul(transpose(T), matmul(K, T))
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        double s = 0.0;
        for (int l = 0; l < nb; ++l) s += K[i + (size_t)nb * l] * T[l + (size_t)nb * j];
        KT[i + (size_t)nb * j] = s;
      }
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        double s = 0.0;
        for (int l = 0; l < nb; ++l) s += T[l + (size_t)nb * i] * KT[l + (size_t)nb * j];
        O[i + (size_t)nb * j] = s;
      }
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row, ++e) {
        rows[e] = gd[(size_t)nb * t + row];
        cols[e] = gd[(size_t)nb * t + col];
        tv[e] = O[row + (size_t)nb * col];
      }
  }
  return or_csc_from_triplet(ng, ng, ntrip, rows.data(), cols.data(), tv.data(), cap, nnz, col_ptr,
                             row_idx, values);
}

// assemble_tetra_nedelec_weighted_element (order 1, the 4-point rule,
// assembly_tetra_nedelec_3d.f90:2406-2450) and
// assemble_tetra_nedelec_weighted_element_order (Duffy rule of degree 2k+2,
// :2452-2514): K_ij = sum_q det w_q (curl_i . M(x_q) curl_j + m v_i . v_j).
// The tensor callback is a per-cell constant here (`tensor`, column-major
// 3 x 3), i.e. a callback that returns the same M at every point of the cell.
int or_nedelec_weighted_element(const double *v, int k, const double *tensor, double mw,
                                double *M) {
  if (k < 1) return 1;
  double J[9], Ji[9], det;
  if (!tetra_geometry(v, J, &det)) return 1;
  inv3(J, det, Ji);
  std::vector<double> px, py, pz, pw;
  if (k == 1) {
    double P[12], W[4];
    or_tetra_degree_two_rule(P, W);
    for (int q = 0; q < 4; ++q) {
      px.push_back(P[3 * q]); py.push_back(P[3 * q + 1]); pz.push_back(P[3 * q + 2]);
      pw.push_back(W[q]);
    }
  } else {
    RuleN R;
    make_rule(0, 2 * k + 2, R);
    px = R.x; py = R.y; pz = R.z; pw = R.w;
  }
  const int n = or_nedelec_dof_count(k);
  std::vector<double> rv(3 * n), rc(3 * n), pv(3 * n), pc(3 * n);
  std::fill(M, M + (size_t)n * n, 0.0);
  for (size_t pt = 0; pt < pw.size(); ++pt) {
    const double P[3] = {px[pt], py[pt], pz[pt]};
    if (k == 1 ? or_whitney_evaluate(P, rv.data(), rc.data())
               : or_nedelec_evaluate(k, P, rv.data(), rc.data()))
      return 1;
    covariant(J, det, Ji, n, rv.data(), rc.data(), pv.data(), pc.data());
    const double w = det * pw[pt];
    for (int col = 0; col < n; ++col) {
      double mc[3];
      for (int i = 0; i < 3; ++i)
        mc[i] = tensor[i] * pc[3 * col] + tensor[i + 3] * pc[3 * col + 1] +
                tensor[i + 6] * pc[3 * col + 2];
      for (int row = 0; row < n; ++row) {
        double dc = 0.0, dv = 0.0;
        for (int i = 0; i < 3; ++i) dc += pc[3 * row + i] * mc[i];
        for (int i = 0; i < 3; ++i) dv += pv[3 * row + i] * pv[3 * col + i];
        M[row + (size_t)n * col] += w * (dc + mw * dv);
      }
    }
  }
  return 0;
}

// assemble_tetra_nedelec_weighted_csc / assemble_arbitrary_order_weighted_csc
// (assembly_tetra_nedelec_3d.f90:1870-1931,1933-2000): order 1 with the edge
// sign products, order >= 2 with T^T K T; triplets j-outer / i-inner into
// csc_from_triplet.  `tensors` holds one column-major 3 x 3 tensor per cell.
int or_nedelec_weighted_csc(int nv, const double *verts, int nt, const int *tets, int k,
                            const double *tensors, double mw, int64_t cap, int *n_dofs,
                            int64_t *nnz, int64_t *col_ptr, int *row_idx, double *values) {
  if (k < 1 || nt < 1 || !tensors) return 1;
  for (int i = 0; i < 4 * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  int nb = or_nedelec_dof_count(k), ng = 0;
  std::vector<int> gd((size_t)nb * nt), eo(6 * (size_t)nt), fp(12 * (size_t)nt);
  if (or_nedelec_dof_map(k, nt, tets, 0, nullptr, nullptr, nullptr, nullptr, gd.data(), eo.data(),
                         fp.data(), &ng))
    return 1;
  *n_dofs = ng;
  int64_t ntrip = (int64_t)nt * nb * nb;
  std::vector<int> rows(ntrip), cols(ntrip);
  std::vector<double> tv(ntrip), K((size_t)nb * nb), T((size_t)nb * nb), KT((size_t)nb * nb),
      O((size_t)nb * nb);
  int64_t e = 0;
  for (int t = 0; t < nt; ++t) {
    double v[12];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * t + n] + d];
    if (or_nedelec_weighted_element(v, k, tensors + 9 * (size_t)t, mw, K.data())) return 1;
    if (k == 1) {
      for (int col = 0; col < 6; ++col)
        for (int row = 0; row < 6; ++row, ++e) {
          rows[e] = gd[(size_t)nb * t + row];
          cols[e] = gd[(size_t)nb * t + col];
          tv[e] = (double)(eo[6 * t + row] * eo[6 * t + col]) * K[row + 6 * col];
        }
      continue;
    }
    if (or_nedelec_transform(k, eo.data() + 6 * t, fp.data() + 12 * t, T.data())) return 1;
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        double s = 0.0;
        for (int l = 0; l < nb; ++l) s += K[i + (size_t)nb * l] * T[l + (size_t)nb * j];
        KT[i + (size_t)nb * j] = s;
      }
    for (int j = 0; j < nb; ++j)
      for (int i = 0; i < nb; ++i) {
        double s = 0.0;
        for (int l = 0; l < nb; ++l) s += T[l + (size_t)nb * i] * KT[l + (size_t)nb * j];
        O[i + (size_t)nb * j] = s;
      }
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row, ++e) {
        rows[e] = gd[(size_t)nb * t + row];
        cols[e] = gd[(size_t)nb * t + col];
        tv[e] = O[row + (size_t)nb * col];
      }
  }
  return or_csc_from_triplet(ng, ng, ntrip, rows.data(), cols.data(), tv.data(), cap, nnz, col_ptr,
                             row_idx, values);
}

// ------------------------------------------------- forward / reverse mode
namespace {
static void mat3_mul(const double *A, const double *B, double *C) {  // column-major C = A B
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += A[r + 3 * k] * B[k + 3 * c];
      C[r + 3 * c] = s;
    }
}

// oriented = T^T M T (forward) or T M T^T (reverse), n x n column-major
static void sandwich(int n, const double *T, const double *M, bool forward, double *out) {
  std::vector<double> X((size_t)n * n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int l = 0; l < n; ++l)
        s += M[i + (size_t)n * l] * (forward ? T[l + (size_t)n * j] : T[j + (size_t)n * l]);
      X[i + (size_t)n * j] = s;
    }
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int l = 0; l < n; ++l)
        s += (forward ? T[l + (size_t)n * i] : T[i + (size_t)n * l]) * X[l + (size_t)n * j];
      out[i + (size_t)n * j] = s;
    }
}
}  // namespace

// assemble_tetra_nedelec_curl_mass_element_jvp, assembly_tetra_nedelec_3d.f90:645-719,
// with map_tetra_nedelec_covariant_jvp (src/elements/tetra_piola_maps.f90:59-105)
// at zero reference tangents: values' = dJ^-T v, curls' = dJ c / det - J c ddet / det^2.
int or_nedelec_element_jvp(const double *v, int k, int q, double cw, double mw, const double *vdot,
                           double cw_dot, double mw_dot, double *Md) {
  if (k < 1 || q < 0) return 1;
  double J[9], Jd[9], Ji[9], Jid[9], T[9], U[9], det;
  if (!tetra_geometry(v, J, &det)) return 1;
  tetra_jacobian(vdot, Jd);
  inv3(J, det, Ji);
  mat3_mul(Ji, Jd, T);
  const double det_dot = det * (T[0] + T[4] + T[8]);
  mat3_mul(T, Ji, U);
  for (int i = 0; i < 9; ++i) Jid[i] = -U[i];
  RuleN R;
  make_rule(0, q, R);
  const int n = or_nedelec_dof_count(k);
  std::vector<double> rv(3 * n), rc(3 * n), pv(3 * n), pc(3 * n), pvd(3 * n), pcd(3 * n);
  std::fill(Md, Md + (size_t)n * n, 0.0);
  for (size_t pt = 0; pt < R.w.size(); ++pt) {
    double P[3] = {R.x[pt], R.y[pt], R.z[pt]};
    if (or_nedelec_evaluate(k, P, rv.data(), rc.data())) return 1;
    covariant(J, det, Ji, n, rv.data(), rc.data(), pv.data(), pc.data());
    for (int b = 0; b < n; ++b)
      for (int i = 0; i < 3; ++i) {
        double s = 0.0, jc = 0.0, jdc = 0.0;
        for (int m = 0; m < 3; ++m) {
          s += Jid[m + 3 * i] * rv[3 * b + m];
          jc += J[i + 3 * m] * rc[3 * b + m];
          jdc += Jd[i + 3 * m] * rc[3 * b + m];
        }
        pvd[3 * b + i] = s;
        pcd[3 * b + i] = jdc / det - jc * det_dot / (det * det);
      }
    const double w = R.w[pt];
    for (int col = 0; col < n; ++col)
      for (int row = 0; row < n; ++row) {
        double ce = 0.0, me = 0.0, cd = 0.0, md = 0.0;
        for (int i = 0; i < 3; ++i) {
          ce += pc[3 * row + i] * pc[3 * col + i];
          me += pv[3 * row + i] * pv[3 * col + i];
          cd += pcd[3 * row + i] * pc[3 * col + i] + pc[3 * row + i] * pcd[3 * col + i];
          md += pvd[3 * row + i] * pv[3 * col + i] + pv[3 * row + i] * pvd[3 * col + i];
        }
        Md[row + (size_t)n * col] +=
            w * (det_dot * (cw * ce + mw * me) +
                 det * (cw_dot * ce + cw * cd + mw_dot * me + mw * md));
      }
  }
  return 0;
}

// assemble_tetra_nedelec_curl_mass_element_vjp, same file :721-806, with
// map_tetra_nedelec_covariant_vjp (tetra_piola_maps.f90:107-167) per point.
int or_nedelec_element_vjp(const double *v, int k, int q, double cw, double mw, const double *Mb,
                           double *vbar, double *cw_bar, double *mw_bar) {
  for (int i = 0; i < 12; ++i) vbar[i] = 0.0;
  *cw_bar = 0.0;
  *mw_bar = 0.0;
  if (k < 1 || q < 0) return 1;
  double J[9], Ji[9], det;
  if (!tetra_geometry(v, J, &det)) return 1;
  inv3(J, det, Ji);
  RuleN R;
  make_rule(0, q, R);
  const int n = or_nedelec_dof_count(k);
  std::vector<double> rv(3 * n), rc(3 * n), pv(3 * n), pc(3 * n), vb(3 * n), cb(3 * n);
  double Jb[9] = {0}, det_bar = 0.0;
  double JiT[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) JiT[r + 3 * c] = Ji[c + 3 * r];
  for (size_t pt = 0; pt < R.w.size(); ++pt) {
    double P[3] = {R.x[pt], R.y[pt], R.z[pt]};
    if (or_nedelec_evaluate(k, P, rv.data(), rc.data())) return 1;
    covariant(J, det, Ji, n, rv.data(), rc.data(), pv.data(), pc.data());
    std::fill(vb.begin(), vb.end(), 0.0);
    std::fill(cb.begin(), cb.end(), 0.0);
    for (int col = 0; col < n; ++col)
      for (int row = 0; row < n; ++row) {
        const double seed = R.w[pt] * Mb[row + (size_t)n * col];
        double ce = 0.0, me = 0.0;
        for (int i = 0; i < 3; ++i) {
          ce += pc[3 * row + i] * pc[3 * col + i];
          me += pv[3 * row + i] * pv[3 * col + i];
        }
        det_bar += seed * (cw * ce + mw * me);
        *cw_bar += seed * det * ce;
        *mw_bar += seed * det * me;
        for (int i = 0; i < 3; ++i) {
          cb[3 * row + i] += seed * det * cw * pc[3 * col + i];
          cb[3 * col + i] += seed * det * cw * pc[3 * row + i];
          vb[3 * row + i] += seed * det * mw * pv[3 * col + i];
          vb[3 * col + i] += seed * det * mw * pv[3 * row + i];
        }
      }
    // map_tetra_nedelec_covariant_vjp: values = J^-T rv, curls = J rc / det
    double Jib[9], A[9], B[9];
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) {
        double s = 0.0;
        for (int b = 0; b < n; ++b) s += rv[3 * b + r] * vb[3 * b + c];
        Jib[r + 3 * c] = s;
      }
    mat3_mul(JiT, Jib, A);
    mat3_mul(A, JiT, B);
    double local[9], db = 0.0;
    for (int c = 0; c < 3; ++c)
      for (int r = 0; r < 3; ++r) {
        double s = 0.0;
        for (int b = 0; b < n; ++b) s += (cb[3 * b + r] / det) * rc[3 * b + c];
        local[r + 3 * c] = -B[r + 3 * c] + s;
      }
    for (int b = 0; b < n; ++b)
      for (int i = 0; i < 3; ++i) {
        double mc = 0.0;
        for (int m = 0; m < 3; ++m) mc += J[i + 3 * m] * rc[3 * b + m];
        db += cb[3 * b + i] * mc;
      }
    db = -db / (det * det);
    for (int i = 0; i < 9; ++i) Jb[i] += local[i] + db * det * JiT[i];
  }
  for (int i = 0; i < 9; ++i) Jb[i] += det_bar * det * JiT[i];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) {
      vbar[r + 3 * (c + 1)] += Jb[r + 3 * c];
      vbar[r] -= Jb[r + 3 * c];
    }
  return 0;
}

// assemble_tetra_nedelec_curl_mass_csc_jvp, same file :2114-2181: the element
// tangent at quadrature degree 2k+2, oriented T^T K' T, through csc_from_triplet.
int or_nedelec_csc_jvp(int nv, const double *verts, int nt, const int *tets, int k, double cw,
                       double mw, const double *vdot, double cw_dot, double mw_dot, int64_t cap,
                       int *n_dofs, int64_t *nnz, int64_t *col_ptr, int *row_idx,
                       double *values) {
  if (k < 1 || nt < 1) return 1;
  for (int i = 0; i < 4 * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  const int nb = or_nedelec_dof_count(k);
  int ng = 0;
  std::vector<int> gd((size_t)nb * nt), eo(6 * (size_t)nt), fp(12 * (size_t)nt);
  if (or_nedelec_dof_map(k, nt, tets, 0, nullptr, nullptr, nullptr, nullptr, gd.data(), eo.data(),
                         fp.data(), &ng))
    return 1;
  *n_dofs = ng;
  const int64_t ntrip = (int64_t)nt * nb * nb;
  std::vector<int> rows(ntrip), cols(ntrip);
  std::vector<double> tv(ntrip), K((size_t)nb * nb), T((size_t)nb * nb), O((size_t)nb * nb);
  int64_t e = 0;
  for (int t = 0; t < nt; ++t) {
    double v[12], vd[12];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) {
        v[3 * n + d] = verts[3 * tets[4 * t + n] + d];
        vd[3 * n + d] = vdot[3 * tets[4 * t + n] + d];
      }
    if (or_nedelec_element_jvp(v, k, 2 * k + 2, cw, mw, vd, cw_dot, mw_dot, K.data())) return 1;
    if (or_nedelec_transform(k, eo.data() + 6 * t, fp.data() + 12 * t, T.data())) return 1;
    sandwich(nb, T.data(), K.data(), true, O.data());
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row, ++e) {
        rows[e] = gd[(size_t)nb * t + row];
        cols[e] = gd[(size_t)nb * t + col];
        tv[e] = O[row + (size_t)nb * col];
      }
  }
  return or_csc_from_triplet(ng, ng, ntrip, rows.data(), cols.data(), tv.data(), cap, nnz, col_ptr,
                             row_idx, values);
}

// assemble_tetra_nedelec_curl_mass_csc_vjp, same file :2183-2287: the oriented
// cotangent read from the merged pattern, T Obar T^T, element VJP at 2k+2.
int or_nedelec_csc_vjp(int nv, const double *verts, int nt, const int *tets, int k, double cw,
                       double mw, int64_t nnz, const double *values_bar, double *verts_bar,
                       double *cw_bar, double *mw_bar) {
  for (int64_t i = 0; i < 3LL * nv; ++i) verts_bar[i] = 0.0;
  *cw_bar = 0.0;
  *mw_bar = 0.0;
  if (k < 1 || nt < 1) return 1;
  for (int i = 0; i < 4 * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  const int64_t pat = or_nedelec_csc_nnz(k, nt, tets);
  if (pat < 0 || pat != nnz) return 1;
  const int nb = or_nedelec_dof_count(k);
  int ng = 0, nd = 0;
  std::vector<int> gd((size_t)nb * nt), eo(6 * (size_t)nt), fp(12 * (size_t)nt);
  if (or_nedelec_dof_map(k, nt, tets, 0, nullptr, nullptr, nullptr, nullptr, gd.data(), eo.data(),
                         fp.data(), &ng))
    return 1;
  std::vector<int64_t> cp(ng + 1);
  std::vector<int> ri(nnz);
  std::vector<double> vals(nnz);
  int64_t got = 0;
  if (or_nedelec_csc(nv, verts, nt, tets, k, cw, mw, nullptr, nullptr, nnz, &nd, &got, cp.data(),
                     ri.data(), vals.data()))
    return 1;
  std::vector<double> Ob((size_t)nb * nb), T((size_t)nb * nb), Eb((size_t)nb * nb);
  for (int t = 0; t < nt; ++t) {
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row) {
        const int gr = gd[(size_t)nb * t + row], gc = gd[(size_t)nb * t + col];
        double b = 0.0;
        for (int64_t x = cp[gc]; x < cp[gc + 1]; ++x)
          if (ri[x] == gr) { b = values_bar[x]; break; }
        Ob[row + (size_t)nb * col] = b;
      }
    if (or_nedelec_transform(k, eo.data() + 6 * t, fp.data() + 12 * t, T.data())) return 1;
    sandwich(nb, T.data(), Ob.data(), false, Eb.data());
    double v[12], vb[12], cb = 0.0, mb = 0.0;
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * t + n] + d];
    if (or_nedelec_element_vjp(v, k, 2 * k + 2, cw, mw, Eb.data(), vb, &cb, &mb)) return 1;
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) verts_bar[3 * tets[4 * t + n] + d] += vb[3 * n + d];
    *cw_bar += cb;
    *mw_bar += mb;
  }
  return 0;
}

// ---------------------------------------------------------- solution probes
namespace {
// The oriented field of a solution on one cell at reference point xi: local
// DoFs T u(gd), basis values / curls, covariant map (the body of
// evaluate_box_solution_order, fortfem_magnetic_box_3d.f90:313-334).
int nedelec_cell_field(int k, const double *J, double det, const double *Ji, const int *gd,
                       const int *eo, const int *fp, const double *u, const double *xi,
                       double *value, double *curl) {
  const int n = or_nedelec_dof_count(k);
  std::vector<double> T((size_t)n * n), ld(n), rv(3 * n), rc(3 * n), pv(3 * n), pc(3 * n);
  if (or_nedelec_transform(k, eo, fp, T.data())) return 1;
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += T[i + (size_t)n * j] * u[gd[j]];
    ld[i] = s;
  }
  if (or_nedelec_evaluate(k, xi, rv.data(), rc.data())) return 1;
  covariant(J, det, Ji, n, rv.data(), rc.data(), pv.data(), pc.data());
  for (int a = 0; a < 3; ++a) {
    double s = 0.0, t = 0.0;
    for (int i = 0; i < n; ++i) {
      s += pv[3 * i + a] * ld[i];
      t += pc[3 * i + a] * ld[i];
    }
    value[a] = s;
    curl[a] = t;
  }
  return 0;
}
}  // namespace

// Field and curl of a Nedelec solution at a reference point of one cell (the
// per-cell evaluation of evaluate_box_solution_order); the cell must pass
// tetra_geometry's test.
int or_nedelec_evaluate_solution(int nv, const double *verts, int nt, const int *tets, int k,
                                 int n_dofs, const double *u, int cell, const double *xi,
                                 double *value, double *curl) {
  for (int a = 0; a < 3; ++a) value[a] = curl[a] = 0.0;
  if (k < 1 || nt < 1 || cell < 0 || cell >= nt) return 1;
  for (int i = 0; i < 4 * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  const int nb = or_nedelec_dof_count(k);
  int ng = 0;
  std::vector<int> gd((size_t)nb * nt), eo(6 * (size_t)nt), fp(12 * (size_t)nt);
  if (or_nedelec_dof_map(k, nt, tets, 0, nullptr, nullptr, nullptr, nullptr, gd.data(), eo.data(),
                         fp.data(), &ng))
    return 1;
  if (n_dofs != ng) return 1;
  double v[12], J[9], Ji[9], det;
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * cell + n] + d];
  if (!tetra_geometry(v, J, &det)) return 1;
  inv3(J, det, Ji);
  return nedelec_cell_field(k, J, det, Ji, gd.data() + (size_t)nb * cell, eo.data() + 6 * cell,
                            fp.data() + 12 * cell, u, xi, value, curl);
}

// evaluate_box_solution_order, src/solvers/fortfem_magnetic_box_3d.f90:269-343
// (mode 0: the average over every containing cell, in cell order) and
// probe_box_az / probe_box_curl, :345-440 (mode 1: the first containing
// cell).  A cell contains the point when det > 0 and its reference
// coordinates are >= -1e-12 with sum <= 1 + 1e-12.  *count = number of
// contributing cells; -1 when evaluate_tetra_nedelec_first_kind rejects the
// point on a containing cell (its -64 eps test), which fails the probe.
int or_nedelec_probe(int nv, const double *verts, int nt, const int *tets, int k, int n_dofs,
                     const double *u, const double *point, int mode, double *value, double *curl,
                     int *count) {
  for (int a = 0; a < 3; ++a) value[a] = curl[a] = 0.0;
  *count = 0;
  if (k < 1 || nt < 1) return 1;
  const int nb = or_nedelec_dof_count(k);
  int ng = 0;
  std::vector<int> gd((size_t)nb * nt), eo(6 * (size_t)nt), fp(12 * (size_t)nt);
  if (or_nedelec_dof_map(k, nt, tets, 0, nullptr, nullptr, nullptr, nullptr, gd.data(), eo.data(),
                         fp.data(), &ng))
    return 1;
  if (n_dofs != ng) return 1;
  double acc_v[3] = {0.0, 0.0, 0.0}, acc_c[3] = {0.0, 0.0, 0.0};
  int found = 0;
  const double tol = 64.0 * kEps;
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
      for (int q = 0; q < 3; ++q) s += Ji[i + 3 * q] * (point[q] - v[q]);
      xi[i] = s;
    }
    if (xi[0] < -1.0e-12 || xi[1] < -1.0e-12 || xi[2] < -1.0e-12) continue;
    if (xi[0] + xi[1] + xi[2] > 1.0 + 1.0e-12) continue;
    if (xi[0] < -tol || xi[1] < -tol || xi[2] < -tol || xi[0] + xi[1] + xi[2] > 1.0 + tol) {
      *count = -1;
      return 1;
    }
    double fv[3], fc[3];
    if (nedelec_cell_field(k, J, det, Ji, gd.data() + (size_t)nb * c, eo.data() + 6 * c,
                           fp.data() + 12 * c, u, xi, fv, fc))
      return 1;
    for (int a = 0; a < 3; ++a) {
      acc_v[a] += fv[a];
      acc_c[a] += fc[a];
    }
    ++found;
    if (mode == 1) break;
  }
  *count = found;
  if (found < 1) return 1;
  for (int a = 0; a < 3; ++a) {
    value[a] = acc_v[a] / found;
    curl[a] = acc_c[a] / found;
  }
  return 0;
}

// ---------------------------------------------------------- complex PML
namespace {
using cplx = std::complex<double>;

// cartesian_curl_curl_pml_coefficients (src/boundary/cartesian_helmholtz_pml.f90:94-108)
// through cartesian_scalar_helmholtz_pml_coefficients (:30-48): mass = the H1
// tensor diag(s2 s3/s1, s1 s3/s2, s1 s2/s3), curl = its inverse.
bool cartesian_pml(const cplx *s, cplx *cc, cplx *mc) {
  for (int a = 0; a < 3; ++a)
    if (std::abs(s[a]) <= DBL_MIN) return false;
  mc[0] = s[1] * s[2] / s[0];
  mc[1] = s[0] * s[2] / s[1];
  mc[2] = s[0] * s[1] / s[2];
  for (int a = 0; a < 3; ++a) cc[a] = 1.0 / mc[a];
  return true;
}

// curvilinear_curl_curl_pml_coefficients (src/boundary/curvilinear_helmholtz_pml.f90:113-131)
// with inverse_and_determinant (:202-216): curl = S^T S / det S, mass = det S S^-1 S^-T.
// S, cc, mc column-major 3x3.
bool curvilinear_pml(const cplx *S, cplx *cc, cplx *mc) {
  auto m = [&](int r, int c) { return S[r + 3 * c]; };
  const cplx det = m(0, 0) * (m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1)) -
                   m(0, 1) * (m(1, 0) * m(2, 2) - m(1, 2) * m(2, 0)) +
                   m(0, 2) * (m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0));
  double mx = 0.0;
  for (int i = 0; i < 9; ++i) {
    if (!std::isfinite(S[i].real()) || !std::isfinite(S[i].imag())) return false;
    mx = std::max(mx, std::abs(S[i]));
  }
  if (!std::isfinite(det.real()) || !std::isfinite(det.imag())) return false;
  const double sc = std::max(1.0, mx);
  if (std::abs(det) <= 64.0 * kEps * sc * sc * sc) return false;
  cplx cof[9], inv[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
      cof[r + 3 * c] = m(r1, c1) * m(r2, c2) - m(r1, c2) * m(r2, c1);
    }
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) inv[r + 3 * c] = cof[c + 3 * r] / det;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      cplx a = 0.0, b = 0.0;
      for (int q = 0; q < 3; ++q) {
        a += S[q + 3 * r] * S[q + 3 * c];      // (S^T S)(r, c)
        b += inv[r + 3 * q] * inv[c + 3 * q];  // (S^-1 S^-T)(r, c)
      }
      cc[r + 3 * c] = a / det;
      mc[r + 3 * c] = det * b;
    }
  return true;
}

// The element loops of assemble_tetra_nedelec_pml_element (assembly_tetra_nedelec_3d.f90:826-887,
// diagonal tensors) and assemble_tetra_nedelec_curvilinear_pml_element (:1092-1153,
// full tensors): K += det w (curl_i . Cc curl_j - k^2 v_i . Cm v_j).
int pml_element(const double *v, int k, int q, const cplx *cc, const cplx *mc, bool full,
                double wave, cplx *M) {
  double J[9], Ji[9], det;
  if (!tetra_geometry(v, J, &det)) return 1;
  inv3(J, det, Ji);
  RuleN R;
  make_rule(0, q, R);
  const int n = or_nedelec_dof_count(k);
  std::vector<double> rv(3 * n), rc(3 * n), pv(3 * n), pc(3 * n);
  std::fill(M, M + (size_t)n * n, cplx(0.0, 0.0));
  auto apply = [&](const cplx *C, const double *x, cplx *y) {
    for (int a = 0; a < 3; ++a) {
      if (!full) { y[a] = C[a] * x[a]; continue; }
      y[a] = C[a] * x[0] + C[a + 3] * x[1] + C[a + 6] * x[2];
    }
  };
  for (size_t pt = 0; pt < R.w.size(); ++pt) {
    double P[3] = {R.x[pt], R.y[pt], R.z[pt]};
    if (or_nedelec_evaluate(k, P, rv.data(), rc.data())) return 1;
    covariant(J, det, Ji, n, rv.data(), rc.data(), pv.data(), pc.data());
    const double pw = det * R.w[pt];
    for (int col = 0; col < n; ++col) {
      cplx ccj[3], mcj[3];
      apply(cc, &pc[3 * col], ccj);
      apply(mc, &pv[3 * col], mcj);
      for (int row = 0; row < n; ++row) {
        cplx a = 0.0, b = 0.0;
        for (int i = 0; i < 3; ++i) {
          a += pc[3 * row + i] * ccj[i];
          b += pv[3 * row + i] * mcj[i];
        }
        M[row + (size_t)n * col] += pw * (a - wave * wave * b);
      }
    }
  }
  return 0;
}

// assemble_tetra_nedelec_pml_csc (:1613-1685) / _curvilinear_pml_csc (:1372-1444):
// element at quadrature degree 2k+2, oriented T^T K T, csc_from_triplet on the
// real and imaginary parts (the same triplet order for both).
int pml_csc(int nv, const double *verts, int nt, const int *tets, int k, const double *stretch,
            bool full, double wave, int64_t cap, int *n_dofs, int64_t *nnz, int64_t *col_ptr,
            int *row_idx, double *values) {
  if (k < 1 || nt < 1 || !(wave > 0.0)) return 1;
  for (int i = 0; i < 4 * nt; ++i)
    if (tets[i] < 0 || tets[i] >= nv) return 1;
  const int nb = or_nedelec_dof_count(k);
  int ng = 0;
  std::vector<int> gd((size_t)nb * nt), eo(6 * (size_t)nt), fp(12 * (size_t)nt);
  if (or_nedelec_dof_map(k, nt, tets, 0, nullptr, nullptr, nullptr, nullptr, gd.data(), eo.data(),
                         fp.data(), &ng))
    return 1;
  *n_dofs = ng;
  const int64_t ntrip = (int64_t)nt * nb * nb;
  std::vector<int> rows(ntrip), cols(ntrip);
  std::vector<double> tre(ntrip), tim(ntrip), T((size_t)nb * nb), X((size_t)nb * nb);
  std::vector<cplx> K((size_t)nb * nb);
  const int sw = full ? 9 : 3;
  int64_t e = 0;
  for (int t = 0; t < nt; ++t) {
    double v[12];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * t + n] + d];
    cplx S[9], cc[9], mc[9];
    for (int i = 0; i < sw; ++i)
      S[i] = cplx(stretch[2 * (sw * (size_t)t + i)], stretch[2 * (sw * (size_t)t + i) + 1]);
    if (!(full ? curvilinear_pml(S, cc, mc) : cartesian_pml(S, cc, mc))) return 1;
    if (pml_element(v, k, 2 * k + 2, cc, mc, full, wave, K.data())) return 1;
    if (or_nedelec_transform(k, eo.data() + 6 * t, fp.data() + 12 * t, T.data())) return 1;
    std::vector<double> Kr((size_t)nb * nb), Kim((size_t)nb * nb), Or((size_t)nb * nb),
        Oi((size_t)nb * nb);
    for (size_t i = 0; i < K.size(); ++i) {
      Kr[i] = K[i].real();
      Kim[i] = K[i].imag();
    }
    sandwich(nb, T.data(), Kr.data(), true, Or.data());
    sandwich(nb, T.data(), Kim.data(), true, Oi.data());
    for (int col = 0; col < nb; ++col)
      for (int row = 0; row < nb; ++row, ++e) {
        rows[e] = gd[(size_t)nb * t + row];
        cols[e] = gd[(size_t)nb * t + col];
        tre[e] = Or[row + (size_t)nb * col];
        tim[e] = Oi[row + (size_t)nb * col];
      }
  }
  std::vector<double> vre, vim;
  int64_t z = 0;
  int st = or_csc_from_triplet(ng, ng, ntrip, rows.data(), cols.data(), tre.data(), 0, &z, nullptr,
                               nullptr, nullptr);
  *nnz = z;
  if (z > cap || !col_ptr) return -2;
  vre.resize(z);
  vim.resize(z);
  st = or_csc_from_triplet(ng, ng, ntrip, rows.data(), cols.data(), tre.data(), cap, nnz, col_ptr,
                           row_idx, vre.data());
  if (st) return st;
  st = or_csc_from_triplet(ng, ng, ntrip, rows.data(), cols.data(), tim.data(), cap, nnz, col_ptr,
                           row_idx, vim.data());
  if (st) return st;
  for (int64_t i = 0; i < z; ++i) {
    values[2 * i] = vre[i];
    values[2 * i + 1] = vim[i];
  }
  return 0;
}
}  // namespace

int or_nedelec_pml_element(const double *v, int k, int q, const double *stretch, double wave,
                           double *M) {
  if (k < 1 || q < 0 || !(wave > 0.0)) return 1;
  cplx S[3], cc[3], mc[3];
  for (int a = 0; a < 3; ++a) S[a] = cplx(stretch[2 * a], stretch[2 * a + 1]);
  if (!cartesian_pml(S, cc, mc)) return 1;
  return pml_element(v, k, q, cc, mc, false, wave, reinterpret_cast<cplx *>(M));
}

int or_nedelec_curvilinear_pml_element(const double *v, int k, int q, const double *stretch,
                                       double wave, double *M) {
  if (k < 1 || q < 0 || !(wave > 0.0)) return 1;
  cplx S[9], cc[9], mc[9];
  for (int a = 0; a < 9; ++a) S[a] = cplx(stretch[2 * a], stretch[2 * a + 1]);
  if (!curvilinear_pml(S, cc, mc)) return 1;
  return pml_element(v, k, q, cc, mc, true, wave, reinterpret_cast<cplx *>(M));
}

int or_nedelec_pml_csc(int nv, const double *verts, int nt, const int *tets, int k,
                       const double *stretch, double wave, int64_t cap, int *n_dofs, int64_t *nnz,
                       int64_t *col_ptr, int *row_idx, double *values) {
  return pml_csc(nv, verts, nt, tets, k, stretch, false, wave, cap, n_dofs, nnz, col_ptr, row_idx,
                 values);
}

int or_nedelec_curvilinear_pml_csc(int nv, const double *verts, int nt, const int *tets, int k,
                                   const double *stretch, double wave, int64_t cap, int *n_dofs,
                                   int64_t *nnz, int64_t *col_ptr, int *row_idx, double *values) {
  return pml_csc(nv, verts, nt, tets, k, stretch, true, wave, cap, n_dofs, nnz, col_ptr, row_idx,
                 values);
}

static int nedelec_load_rule(int k, RuleN &R) {
  // order 1: the 4-point rule (assemble_tetra_nedelec_load_element :2516-2553);
  // order >= 2: Duffy with q = 2k+2 (assemble_tetra_nedelec_load_element_order :547)
  return make_rule(k == 1 ? 1 : 0, 2 * k + 2, R) ? 0 : 1;
}

int or_nedelec_load_points(int nv, const double *verts, int nt, const int *tets, int k,
                           double *out) {
  RuleN R;
  if (nedelec_load_rule(k, R)) return 1;
  int nq = (int)R.w.size();
  for (int t = 0; t < nt; ++t) {
    double v[12], J[9];
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * t + n] + d];
    tetra_jacobian(v, J);
    for (int pt = 0; pt < nq; ++pt) {
      double xi[3] = {R.x[pt], R.y[pt], R.z[pt]};
      for (int r = 0; r < 3; ++r) {
        double s = v[r];
        for (int c = 0; c < 3; ++c) s = s + J[r + 3 * c] * xi[c];
        out[3 * ((size_t)nq * t + pt) + r] = s;
      }
    }
  }
  return 0;
}

// Vector load with per-quadrature-point source samples: order 1 as
// assemble_tetra_nedelec_vector_load (:2002-2040, signs), order >= 2 as
// assemble_tetra_nedelec_vector_load_order (:71-127, T^T b_e).  rhs has n_dofs entries.
int or_nedelec_load_samples(int nv, const double *verts, int nt, const int *tets, int k,
                            const double *src, double *rhs) {
  int nb = or_nedelec_dof_count(k), ng = 0;
  std::vector<int> gd((size_t)nb * nt), eo(6 * (size_t)nt), fp(12 * (size_t)nt);
  if (or_nedelec_dof_map(k, nt, tets, 0, nullptr, nullptr, nullptr, nullptr, gd.data(), eo.data(),
                         fp.data(), &ng))
    return 1;
  RuleN R;
  if (nedelec_load_rule(k, R)) return 1;
  int nq = (int)R.w.size();
  for (int i = 0; i < ng; ++i) rhs[i] = 0.0;
  std::vector<double> rv(3 * (size_t)nb * nq), rc(3 * (size_t)nb * nq), pv(3 * nb), pc(3 * nb),
      ev(nb), T((size_t)nb * nb);
  for (int pt = 0; pt < nq; ++pt) {
    double P[3] = {R.x[pt], R.y[pt], R.z[pt]};
    int st = (k == 1) ? or_whitney_evaluate(P, rv.data() + 3 * (size_t)nb * pt,
                                            rc.data() + 3 * (size_t)nb * pt)
                      : or_nedelec_evaluate(k, P, rv.data() + 3 * (size_t)nb * pt,
                                            rc.data() + 3 * (size_t)nb * pt);
    if (st) return 1;
  }
  for (int t = 0; t < nt; ++t) {
    double v[12], J[9], Ji[9], det;
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) v[3 * n + d] = verts[3 * tets[4 * t + n] + d];
    if (!tetra_geometry(v, J, &det)) return 1;
    inv3(J, det, Ji);
    std::fill(ev.begin(), ev.end(), 0.0);
    for (int pt = 0; pt < nq; ++pt) {
      covariant(J, det, Ji, nb, rv.data() + 3 * (size_t)nb * pt, rc.data() + 3 * (size_t)nb * pt,
                pv.data(), pc.data());
      const double *s = src + 3 * ((size_t)nq * t + pt);
      for (int d = 0; d < nb; ++d) {
        double dt = 0.0;
        for (int i = 0; i < 3; ++i) dt += s[i] * pv[3 * d + i];
        ev[d] = ev[d] + det * R.w[pt] * dt;
      }
    }
    if (k == 1) {
      for (int d = 0; d < 6; ++d) {
        int g = gd[(size_t)nb * t + d];
        rhs[g] = rhs[g] + (double)eo[6 * t + d] * ev[d];
      }
      continue;
    }
    if (or_nedelec_transform(k, eo.data() + 6 * t, fp.data() + 12 * t, T.data())) return 1;
    for (int d = 0; d < nb; ++d) {
      double s = 0.0;
      for (int l = 0; l < nb; ++l) s += T[l + (size_t)nb * d] * ev[l];
      int g = gd[(size_t)nb * t + d];
      rhs[g] = rhs[g] + s;
    }
  }
  return 0;
}

// build_zero_tangential_mask, src/solvers/fortfem_tetra_nedelec_solver_3d.f90:416-458.
// faithful = 1 runs the reference's O(F*T) incidence and O(F*E) edge scans.
int or_pec_mask(int k, int nt, const int *tets, int faithful, uint8_t *con) {
  int ne = 0, nf = 0, ng = 0;
  if (or_nedelec_dof_map(k, nt, tets, faithful, nullptr, &ne, nullptr, &nf, nullptr, nullptr,
                         nullptr, &ng))
    return 1;
  std::vector<int> edges(2 * (size_t)ne), faces(3 * (size_t)nf);
  or_nedelec_dof_map(k, nt, tets, faithful, edges.data(), &ne, faces.data(), &nf, nullptr, nullptr,
                     nullptr, &ng);
  std::memset(con, 0, ng);
  int64_t edc = (int64_t)k * ne;
  int fdc = k * (k - 1);
  std::vector<int> inc(nf, 0);
  std::unordered_map<uint64_t, int> emap;
  if (faithful) {
    for (int f = 0; f < nf; ++f)
      for (int t = 0; t < nt; ++t) {
        bool all = true;
        for (int a = 0; a < 3; ++a) {
          bool any = false;
          for (int n = 0; n < 4; ++n) any = any || tets[4 * t + n] == faces[3 * f + a];
          all = all && any;
        }
        if (all) inc[f]++;
      }
  } else {
    std::unordered_map<uint64_t, int> fmap;
    for (int f = 0; f < nf; ++f)
      fmap[((uint64_t)(uint32_t)faces[3 * f] << 42) ^ ((uint64_t)(uint32_t)faces[3 * f + 1] << 21) ^
           (uint64_t)(uint32_t)faces[3 * f + 2]] = f;
    for (int t = 0; t < nt; ++t)
      for (int lf = 0; lf < 4; ++lf) {
        int cv[3];
        for (int i = 0; i < 3; ++i) cv[i] = tets[4 * t + kLocalFaces[lf][i]];
        std::sort(cv, cv + 3);
        inc[fmap[((uint64_t)(uint32_t)cv[0] << 42) ^ ((uint64_t)(uint32_t)cv[1] << 21) ^
                 (uint64_t)(uint32_t)cv[2]]]++;
      }
    for (int e = 0; e < ne; ++e)
      emap[((uint64_t)(uint32_t)edges[2 * e] << 32) | (uint32_t)edges[2 * e + 1]] = e;
  }
  for (int f = 0; f < nf; ++f) {
    if (inc[f] != 1) continue;
    const int *fv = faces.data() + 3 * f;
    if (faithful) {
      for (int e = 0; e < ne; ++e) {
        bool a = fv[0] == edges[2 * e] || fv[1] == edges[2 * e] || fv[2] == edges[2 * e];
        bool b = fv[0] == edges[2 * e + 1] || fv[1] == edges[2 * e + 1] || fv[2] == edges[2 * e + 1];
        if (a && b)
          for (int m = 0; m < k; ++m) con[(int64_t)e * k + m] = 1;
      }
    } else {
      const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
      for (auto &pr : pairs) {
        int a = std::min(fv[pr[0]], fv[pr[1]]), b = std::max(fv[pr[0]], fv[pr[1]]);
        int e = emap[((uint64_t)(uint32_t)a << 32) | (uint32_t)b];
        for (int m = 0; m < k; ++m) con[(int64_t)e * k + m] = 1;
      }
    }
    for (int m = 0; m < fdc; ++m) con[edc + (int64_t)f * fdc + m] = 1;
  }
  return 0;
}

}  // extern "C"
