// Host-side topology of the assembly path: DoF numbering in the reference's
// first-appearance order, constrained sets, the constrained CSC pattern and
// the element-to-CSC slot map used by the atomic-free column assembly.
//
// Numbering rules restated (hash maps replace the reference's linear searches,
// which give the same first-appearance order):
//   Lagrange  build_tetra_lagrange_dof_map  src/elements/tetra_lagrange_global_dof_map.f90:13-99
//   edges     build_tetra_edge_dof_map      src/elements/tetra_edge_dof_map.f90:10-77
//   Nedelec   build_tetra_nedelec_dof_map   src/elements/tetra_nedelec_global_dof_map.f90:15-105
//   P1        vertex numbering of create_rectangular, src/mesh/mesh_2d.f90:90-148
// Constraints:
//   Lagrange  build_dirichlet_data          src/solvers/fortfem_tetra_lagrange_solver_3d.f90:551-610
//   Nedelec   build_zero_tangential_mask    src/solvers/fortfem_tetra_nedelec_solver_3d.f90:416-458
//   P1        find_boundary                 src/mesh/mesh_2d.f90:560-603
#include <algorithm>
#include <cstring>
#include <unordered_map>

#include "ffg_internal.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace ffg {

namespace {

struct Key128 {
  uint64_t a, b;
  bool operator==(const Key128 &o) const { return a == o.a && b == o.b; }
};
struct Key128Hash {
  size_t operator()(const Key128 &k) const {
    uint64_t h = k.a * 0x9E3779B97F4A7C15ull;
    h ^= (k.b + 0x632BE59BD9B4E019ull) * 0xC2B2AE3D27D4EB4Full;
    h ^= h >> 29;
    return (size_t)h;
  }
};
struct U64Hash {
  size_t operator()(uint64_t x) const {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    return (size_t)x;
  }
};

uint64_t edge_key(int a, int b) {
  if (a > b) std::swap(a, b);
  return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
}
Key128 face_key(int a, int b, int c) {
  int t[3] = {a, b, c};
  std::sort(t, t + 3);
  return {((uint64_t)(uint32_t)t[0] << 32) | (uint32_t)t[1], (uint64_t)(uint32_t)t[2]};
}

const int kLocalEdges[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
const int kLocalFaces[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

int perm_index(const int p[3]) {
  switch (100 * p[0] + 10 * p[1] + p[2]) {
    case 123: return 0;
    case 132: return 1;
    case 213: return 2;
    case 231: return 3;
    case 312: return 4;
    case 321: return 5;
  }
  return -1;
}

bool check_cells(const Topology &t, std::string &msg) {
  if (t.n_cells < 1) { msg = "no cells"; return false; }
  for (int c = 0; c < t.n_cells; ++c) {
    const int *v = t.cells.data() + (size_t)t.vpc * c;
    for (int i = 0; i < t.vpc; ++i) {
      if (v[i] < 0 || v[i] >= t.n_vertices) { msg = "cell vertex out of range"; return false; }
      for (int j = i + 1; j < t.vpc; ++j)
        if (v[i] == v[j]) { msg = "cell with repeated vertices"; return false; }
    }
  }
  return true;
}

int build_lagrange(Topology &t, std::string &msg) {
  const int p = t.degree;
  if (p < 1 || p > 4) { msg = "Lagrange degree must be 1..4"; return FFG_INVALID_INPUT; }
  std::vector<int> idx;
  std::vector<double> nodes;
  lagrange_indices(p, idx, nodes);
  t.nb = lagrange_dof_count(p);
  t.gd.assign((size_t)t.nb * t.n_cells, 0);
  // key: the DoF's sub-simplex vertices with their barycentric weights, sorted
  // by vertex (sort_key, tetra_lagrange_global_dof_map.f90:81-99).  Weights
  // are <= 4, so 3 bits each; vertex ids use 29 bits each (n < 2^29).
  if (t.n_vertices >= (1 << 29)) { msg = "too many vertices"; return FFG_INVALID_INPUT; }
  std::unordered_map<Key128, int, Key128Hash> map;
  map.reserve((size_t)t.n_cells * t.nb / 3 + 64);
  int next = 0;
  for (int c = 0; c < t.n_cells; ++c) {
    const int *v = t.cells.data() + 4 * (size_t)c;
    for (int l = 0; l < t.nb; ++l) {
      std::pair<int, int> kv[4];
      int n = 0;
      for (int i = 0; i < 4; ++i)
        if (idx[4 * l + i] != 0) kv[n++] = {v[i], idx[4 * l + i]};
      std::sort(kv, kv + n);
      uint64_t a = 0, b = 0;
      for (int i = 0; i < n; ++i) {
        uint64_t word = ((uint64_t)(kv[i].first + 1) << 3) | (uint64_t)kv[i].second;  // 32 bits
        if (i < 2) a |= word << (32 * i); else b |= word << (32 * (i - 2));
      }
      auto it = map.emplace(Key128{a, b}, next);
      if (it.second) ++next;
      t.gd[(size_t)t.nb * c + l] = it.first->second;
    }
  }
  t.n_dofs = next;
  return FFG_OK;
}

// Arbitrary-order triangles: the first-appearance rule of the tetrahedral
// map on triangles (a local DoF is keyed by its (vertex, power) pairs of
// nonzero power, sorted by vertex).
int build_triangle_lagrange(Topology &t, std::string &msg) {
  const int p = t.degree;
  if (p < 1 || p > 6) { msg = "triangle Lagrange degree must be 1..6"; return FFG_INVALID_INPUT; }
  std::vector<int> pw;
  std::vector<double> nodes;
  triangle_lagrange_indices(p, pw, nodes);
  t.nb = triangle_lagrange_dof_count(p);
  t.gd.assign((size_t)t.nb * t.n_cells, 0);
  if (t.n_vertices >= (1 << 29)) { msg = "too many vertices"; return FFG_INVALID_INPUT; }
  std::unordered_map<Key128, int, Key128Hash> map;
  map.reserve((size_t)t.n_cells * t.nb / 2 + 64);
  int next = 0;
  for (int c = 0; c < t.n_cells; ++c) {
    const int *v = t.cells.data() + 3 * (size_t)c;
    for (int l = 0; l < t.nb; ++l) {
      std::pair<int, int> kv[3];
      int n = 0;
      for (int i = 0; i < 3; ++i)
        if (pw[3 * l + i] != 0) kv[n++] = {v[i], pw[3 * l + i]};
      std::sort(kv, kv + n);
      uint64_t a = 0, b = 0;
      for (int i = 0; i < n; ++i) {
        uint64_t word = ((uint64_t)(kv[i].first + 1) << 3) | (uint64_t)kv[i].second;
        if (i < 2) a |= word << (32 * i); else b |= word;
      }
      auto it = map.emplace(Key128{a, b}, next);
      if (it.second) ++next;
      t.gd[(size_t)t.nb * c + l] = it.first->second;
    }
  }
  t.n_dofs = next;
  return FFG_OK;
}

int build_nedelec(Topology &t, std::string &msg) {
  const int k = t.degree;
  if (k < 1 || k > 6) { msg = "Nedelec order must be 1..6"; return FFG_INVALID_INPUT; }
  t.nb = nedelec_dof_count(k);
  const int fdc = k * (k - 1), cdc = k * (k - 1) * (k - 2) / 2;
  t.gd.assign((size_t)t.nb * t.n_cells, 0);
  t.edge_sign.assign(6 * (size_t)t.n_cells, 1);
  t.face_perm.assign(4 * (size_t)t.n_cells, 0);
  std::vector<int> cell_edge(6 * (size_t)t.n_cells), cell_face(4 * (size_t)t.n_cells);
  std::unordered_map<uint64_t, int, U64Hash> emap;
  emap.reserve((size_t)t.n_cells * 2 + 64);
  int ne = 0;
  for (int c = 0; c < t.n_cells; ++c) {
    const int *v = t.cells.data() + 4 * (size_t)c;
    nedelec_orientation(v, &t.edge_sign[6 * (size_t)c], &t.face_perm[4 * (size_t)c]);
    for (int le = 0; le < 6; ++le) {
      int a = v[kLocalEdges[le][0]], b = v[kLocalEdges[le][1]];
      auto it = emap.emplace(edge_key(a, b), ne);
      if (it.second) ++ne;
      cell_edge[6 * (size_t)c + le] = it.first->second;
    }
  }
  std::unordered_map<Key128, int, Key128Hash> fmap;
  fmap.reserve((size_t)t.n_cells * 2 + 64);
  int nf = 0;
  if (fdc > 0 || true) {
    for (int c = 0; c < t.n_cells; ++c) {
      const int *v = t.cells.data() + 4 * (size_t)c;
      for (int lf = 0; lf < 4; ++lf) {
        auto it = fmap.emplace(
            face_key(v[kLocalFaces[lf][0]], v[kLocalFaces[lf][1]], v[kLocalFaces[lf][2]]), nf);
        if (it.second) ++nf;
        cell_face[4 * (size_t)c + lf] = it.first->second;
      }
    }
  }
  t.n_edges = ne;
  t.n_faces = nf;
  const int64_t edc = (int64_t)k * ne;
  const int64_t total = edc + (int64_t)nf * fdc + (int64_t)t.n_cells * cdc;
  if (total >= (1LL << 31)) { msg = "too many DoFs"; return FFG_INVALID_INPUT; }
  for (int c = 0; c < t.n_cells; ++c) {
    int *g = t.gd.data() + (size_t)t.nb * c;
    for (int e = 0; e < 6; ++e)
      for (int m = 0; m < k; ++m) g[e * k + m] = (int)((int64_t)cell_edge[6 * (size_t)c + e] * k + m);
    for (int lf = 0; lf < 4; ++lf)
      for (int m = 0; m < fdc; ++m)
        g[6 * k + lf * fdc + m] = (int)(edc + (int64_t)cell_face[4 * (size_t)c + lf] * fdc + m);
    for (int m = 0; m < cdc; ++m)
      g[6 * k + 4 * fdc + m] = (int)(edc + (int64_t)nf * fdc + (int64_t)c * cdc + m);
  }
  t.n_dofs = total;
  return FFG_OK;
}

}  // namespace

// Orientation of a Nedelec cell from its global vertex indices (the
// reference's convention, tetra_edge_dof_map.f90:54-60 and
// tetra_nedelec_global_dof_map.f90:68-74): edge le is reversed (-1) when its
// first local vertex has the larger index; face lf gets the index 0..5 of the
// permutation taking its local vertex order to ascending index order (ranks
// 123, 132, 213, 231, 312, 321).
void nedelec_orientation(const int *v, int8_t *sign, uint8_t *perm) {
  for (int le = 0; le < 6; ++le)
    sign[le] = v[kLocalEdges[le][0]] < v[kLocalEdges[le][1]] ? 1 : -1;
  for (int lf = 0; lf < 4; ++lf) {
    const int lv[3] = {v[kLocalFaces[lf][0]], v[kLocalFaces[lf][1]], v[kLocalFaces[lf][2]]};
    int cv[3] = {lv[0], lv[1], lv[2]};
    std::sort(cv, cv + 3);
    int p[3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        if (cv[j] == lv[i]) p[i] = j + 1;
    perm[lf] = (uint8_t)perm_index(p);
  }
}

bool validate_cells(const Topology &t, std::string &msg) { return check_cells(t, msg); }

int build_dofs(Topology &t, std::string &msg) {
  if (!check_cells(t, msg)) return FFG_INVALID_INPUT;
  switch (t.family) {
    case FFG_TETRA_LAGRANGE:
      if (t.vpc != 4) return FFG_INVALID_INPUT;
      return build_lagrange(t, msg);
    case FFG_TETRA_NEDELEC:
      if (t.vpc != 4) return FFG_INVALID_INPUT;
      return build_nedelec(t, msg);
    case FFG_TRIANGLE_LAGRANGE:
      if (t.vpc != 3) return FFG_INVALID_INPUT;
      return build_triangle_lagrange(t, msg);
    case FFG_TRIANGLE_P1:
      if (t.vpc != 3 || t.degree != 1) { msg = "P1 triangles only"; return FFG_INVALID_INPUT; }
      t.nb = 3;
      t.gd = t.cells;
      t.n_dofs = t.n_vertices;
      return FFG_OK;
  }
  msg = "unknown family";
  return FFG_INVALID_INPUT;
}

int build_constraints(Topology &t, int mode, const uint8_t *mask, std::string &msg) {
  t.constrained.assign((size_t)t.n_dofs, 0);
  if (mode == FFG_BOUNDARY_NONE) return FFG_OK;
  if (mode == FFG_BOUNDARY_MASK) {
    if (!mask) { msg = "boundary mask missing"; return FFG_INVALID_INPUT; }
    for (int64_t i = 0; i < t.n_dofs; ++i) t.constrained[i] = mask[i] ? 1 : 0;
    return FFG_OK;
  }
  if (mode != FFG_BOUNDARY_ALL) { msg = "bad boundary mode"; return FFG_INVALID_INPUT; }
  if (t.family == FFG_TRIANGLE_P1) {
    std::unordered_map<uint64_t, int, U64Hash> cnt;
    cnt.reserve((size_t)t.n_cells * 2);
    for (int c = 0; c < t.n_cells; ++c)
      for (int e = 0; e < 3; ++e) cnt[edge_key(t.cells[3 * c + e], t.cells[3 * c + (e + 1) % 3])]++;
    for (auto &kv : cnt)
      if (kv.second == 1) {
        t.constrained[kv.first >> 32] = 1;
        t.constrained[kv.first & 0xffffffffu] = 1;
      }
    return FFG_OK;
  }
  if (t.family == FFG_TRIANGLE_LAGRANGE) {
    // every DoF on an edge of one triangle (the opposite vertex's power is 0)
    std::unordered_map<uint64_t, int, U64Hash> cnt;
    cnt.reserve((size_t)t.n_cells * 2);
    for (int c = 0; c < t.n_cells; ++c)
      for (int e = 0; e < 3; ++e) cnt[edge_key(t.cells[3 * c + e], t.cells[3 * c + (e + 1) % 3])]++;
    std::vector<int> pw;
    std::vector<double> nodes;
    triangle_lagrange_indices(t.degree, pw, nodes);
    for (int c = 0; c < t.n_cells; ++c) {
      const int *v = t.cells.data() + 3 * (size_t)c;
      for (int o = 0; o < 3; ++o) {
        if (cnt[edge_key(v[(o + 1) % 3], v[(o + 2) % 3])] != 1) continue;
        for (int l = 0; l < t.nb; ++l)
          if (pw[3 * l + o] == 0) t.constrained[t.gd[(size_t)t.nb * c + l]] = 1;
      }
    }
    return FFG_OK;
  }
  // incidence-one faces
  std::unordered_map<Key128, int, Key128Hash> inc;
  inc.reserve((size_t)t.n_cells * 2 + 64);
  for (int c = 0; c < t.n_cells; ++c) {
    const int *v = t.cells.data() + 4 * (size_t)c;
    for (int lf = 0; lf < 4; ++lf)
      inc[face_key(v[kLocalFaces[lf][0]], v[kLocalFaces[lf][1]], v[kLocalFaces[lf][2]])]++;
  }
  if (t.family == FFG_TETRA_LAGRANGE) {
    std::vector<int> idx;
    std::vector<double> nodes;
    lagrange_indices(t.degree, idx, nodes);
    for (int c = 0; c < t.n_cells; ++c) {
      const int *v = t.cells.data() + 4 * (size_t)c;
      for (int o = 0; o < 4; ++o) {
        int f[3], n = 0;
        for (int i = 0; i < 4; ++i)
          if (i != o) f[n++] = v[i];
        if (inc[face_key(f[0], f[1], f[2])] != 1) continue;
        for (int l = 0; l < t.nb; ++l)
          if (idx[4 * l + o] == 0) t.constrained[t.gd[(size_t)t.nb * c + l]] = 1;
      }
    }
    return FFG_OK;
  }
  // Nedelec: all edge DoFs of the boundary face's edges and all its face DoFs
  const int k = t.degree, fdc = k * (k - 1);
  for (int c = 0; c < t.n_cells; ++c) {
    const int *v = t.cells.data() + 4 * (size_t)c;
    const int *g = t.gd.data() + (size_t)t.nb * c;
    for (int lf = 0; lf < 4; ++lf) {
      if (inc[face_key(v[kLocalFaces[lf][0]], v[kLocalFaces[lf][1]], v[kLocalFaces[lf][2]])] != 1)
        continue;
      for (int le = 0; le < 6; ++le) {
        int a = kLocalEdges[le][0], b = kLocalEdges[le][1];
        bool on = false, onb = false;
        for (int i = 0; i < 3; ++i) {
          on = on || kLocalFaces[lf][i] == a;
          onb = onb || kLocalFaces[lf][i] == b;
        }
        if (on && onb)
          for (int m = 0; m < k; ++m) t.constrained[g[le * k + m]] = 1;
      }
      for (int m = 0; m < fdc; ++m) t.constrained[g[6 * k + lf * fdc + m]] = 1;
    }
  }
  return FFG_OK;
}

int build_pattern(Topology &t, std::string &msg) {
  const int64_t N = t.n_dofs;
  t.free_index.assign((size_t)N, -1);
  t.free_dofs.clear();
  for (int64_t i = 0; i < N; ++i)
    if (!t.constrained[i]) {
      t.free_index[i] = (int)t.free_dofs.size();
      t.free_dofs.push_back((int)i);
    }
  const int64_t F = (int64_t)t.free_dofs.size();
  const int nb = t.nb;
  // incidence: counting sort of (cell, local) pairs by free column, cells ascending
  t.inc_ptr.assign((size_t)F + 1, 0);
  for (int c = 0; c < t.n_cells; ++c)
    for (int l = 0; l < nb; ++l) {
      int f = t.free_index[t.gd[(size_t)nb * c + l]];
      if (f >= 0) t.inc_ptr[f + 1]++;
    }
  for (int64_t j = 0; j < F; ++j) t.inc_ptr[j + 1] += t.inc_ptr[j];
  const int64_t n_inc = t.inc_ptr[F];
  t.inc_cell.assign((size_t)n_inc, 0);
  t.inc_local.assign((size_t)n_inc, 0);
  {
    std::vector<int64_t> pos(t.inc_ptr.begin(), t.inc_ptr.end() - 1);
    for (int c = 0; c < t.n_cells; ++c)
      for (int l = 0; l < nb; ++l) {
        int f = t.free_index[t.gd[(size_t)nb * c + l]];
        if (f < 0) continue;
        int64_t p = pos[f]++;
        t.inc_cell[p] = c;
        t.inc_local[p] = (uint8_t)l;
      }
  }
  // column lengths (unique free rows over incident cells), then rows and slots
  std::vector<int64_t> len((size_t)F, 0);
  int bad = 0;
#pragma omp parallel
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 1024)
    for (int64_t j = 0; j < F; ++j) {
      buf.clear();
      for (int64_t p = t.inc_ptr[j]; p < t.inc_ptr[j + 1]; ++p) {
        const int *g = t.gd.data() + (size_t)nb * t.inc_cell[p];
        for (int i = 0; i < nb; ++i) {
          int f = t.free_index[g[i]];
          if (f >= 0) buf.push_back(f);
        }
      }
      std::sort(buf.begin(), buf.end());
      len[j] = std::unique(buf.begin(), buf.end()) - buf.begin();
      if (len[j] > kMaxColumnLength) bad = 1;
    }
  }
  if (bad) { msg = "a CSC column exceeds 65534 entries"; return FFG_INVALID_INPUT; }
  t.col_ptr.assign((size_t)F + 1, 0);
  for (int64_t j = 0; j < F; ++j) t.col_ptr[j + 1] = t.col_ptr[j] + len[j];
  t.row_idx.assign((size_t)t.col_ptr[F], 0);
  t.slot.assign((size_t)n_inc * nb, kConstrainedSlot);
  int maxc = 0;
#pragma omp parallel reduction(max : maxc)
  {
    std::vector<int> buf;
#pragma omp for schedule(dynamic, 1024)
    for (int64_t j = 0; j < F; ++j) {
      buf.clear();
      for (int64_t p = t.inc_ptr[j]; p < t.inc_ptr[j + 1]; ++p) {
        const int *g = t.gd.data() + (size_t)nb * t.inc_cell[p];
        for (int i = 0; i < nb; ++i) {
          int f = t.free_index[g[i]];
          if (f >= 0) buf.push_back(f);
        }
      }
      std::sort(buf.begin(), buf.end());
      buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
      std::copy(buf.begin(), buf.end(), t.row_idx.begin() + t.col_ptr[j]);
      maxc = std::max(maxc, (int)buf.size());
      for (int64_t p = t.inc_ptr[j]; p < t.inc_ptr[j + 1]; ++p) {
        const int *g = t.gd.data() + (size_t)nb * t.inc_cell[p];
        for (int i = 0; i < nb; ++i) {
          int f = t.free_index[g[i]];
          if (f < 0) continue;
          auto it = std::lower_bound(buf.begin(), buf.end(), f);
          t.slot[(size_t)p * nb + i] = (uint16_t)(it - buf.begin());
        }
      }
    }
  }
  t.max_column = maxc;
  return FFG_OK;
}

// SELL-32-sigma layout of a CSR operator.  Rows are stably sorted by length
// (longest first) inside windows of `sigma` rows, which keeps the padding of
// each 32-row slice small while moving no row further than sigma; entries of
// a row keep their CSR order.  Padding entries carry a zero value and point at
// a valid column (the row itself, or the last row for the rows that only pad
// the final slice).
void build_sell(const std::vector<int64_t> &rp, const std::vector<int> &ci, int sigma,
                HostSell &out) {
  const int64_t n = (int64_t)rp.size() - 1;
  out = HostSell();
  out.n = n;
  std::vector<int> order((size_t)n);
  for (int64_t i = 0; i < n; ++i) order[i] = (int)i;
  auto len = [&](int r) { return rp[r + 1] - rp[r]; };
  for (int64_t w0 = 0; w0 < n; w0 += sigma) {
    const int64_t w1 = std::min<int64_t>(n, w0 + sigma);
    std::stable_sort(order.begin() + w0, order.begin() + w1,
                     [&](int p, int q) { return len(p) > len(q); });
  }
  out.perm = order;
  out.iperm.assign((size_t)n, 0);
  for (int64_t i = 0; i < n; ++i) out.iperm[order[i]] = (int)i;
  out.n_slices = (n + kSliceRows - 1) / kSliceRows;
  out.soff.assign((size_t)out.n_slices + 1, 0);
  for (int64_t s = 0; s < out.n_slices; ++s) {
    int64_t mx = 0;
    for (int l = 0; l < kSliceRows; ++l) {
      const int64_t r = s * kSliceRows + l;
      if (r < n) mx = std::max(mx, len(order[r]));
    }
    out.soff[s + 1] = out.soff[s] + mx * kSliceRows;
  }
  out.padded = out.soff[out.n_slices];
  // narrow if every |column - row| (new numbering) fits int16
  bool narrow = true;
  for (int64_t i = 0; i < n && narrow; ++i) {
    const int64_t r = out.iperm[i];
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      const int64_t d = (int64_t)out.iperm[ci[k]] - r;
      if (d < -32768 || d > 32767) { narrow = false; break; }
    }
  }
  out.narrow = narrow;
  if (narrow) out.dcol.assign((size_t)out.padded, 0);
  else out.col.assign((size_t)out.padded, 0);
  out.pos.assign(rp.back(), 0);
  for (int64_t s = 0; s < out.n_slices; ++s)
    for (int l = 0; l < kSliceRows; ++l) {
      const int64_t r = s * kSliceRows + l;
      const int64_t slen = (out.soff[s + 1] - out.soff[s]) / kSliceRows;
      const int64_t base = out.soff[s] + l;
      if (r >= n) {
        // padding row: every entry points at the last row with a zero value
        for (int64_t k = 0; k < slen; ++k) {
          if (narrow) out.dcol[base + k * kSliceRows] = (int16_t)((n - 1) - r);
          else out.col[base + k * kSliceRows] = (int)(n - 1);
        }
        continue;
      }
      const int old = order[r];
      int64_t k = 0;
      for (int64_t e = rp[old]; e < rp[old + 1]; ++e, ++k) {
        const int64_t p = base + k * kSliceRows;
        out.pos[e] = p;
        const int c = out.iperm[ci[e]];
        if (narrow) out.dcol[p] = (int16_t)(c - r);
        else out.col[p] = c;
      }
      for (; k < slen; ++k) {
        if (narrow) out.dcol[base + k * kSliceRows] = 0;
        else out.col[base + k * kSliceRows] = (int)r;
      }
    }
}

}  // namespace ffg
