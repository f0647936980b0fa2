// ============================================================================
// embed_oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// FP64 CPU restatement of the reference's embedded-quadrature construction:
// classification of background cells against an embedded volumetric mesh,
// cut-cell quadrature in the background element's reference coordinates, and
// moment-fitting quadrature simplification.  Used only by tests/ and by
// bench.py's CPU leg, as the reference the CUDA path in
// higher_order_embedded_fem_b200/csrc/embed.cu is compared with; the product
// never links it.
//
// Reference (fenris):
//   embed_mesh_3d_with_opts / embed_in_cell      src/embedding/embedding3d.rs:57-196
//   compute_element_embedded_quadrature          src/embedding/embedding3d.rs:233-289
//   PolyMesh3d::intersect_half_space             src/geometry/polymesh.rs:629-808
//   PolyMesh3d::triangulate (Max 2000)           src/geometry/polymesh.rs:402-507
//   PolyMesh::keep_cells                         src/geometry/polymesh.rs:509-571
//   PolyMesh::from(&Mesh)                        src/mesh_convert.rs:578-637
//   Tet4Mesh::try_from(&PolyMesh3d)              src/mesh_convert.rs:639-705
//   compute_polyhedron_volume_from_faces         src/geometry/mod.rs:1002-1032
//   LineSegment3d::closest_point_to_plane        src/geometry/mod.rs:741-774
//   map_physical_coordinates (Newton, 1e-12 d)   src/element.rs:2203-2275
//   build_moment_fitting_system / optimize_quadrature
//                                                src/embedding/quadrature_reduction.rs:35-190
// The reference solves the simplification as a linear feasibility problem
// with OR-Tools GLOP (lp-bfp crate, absent here): any basic feasible point of
// {w >= 0, P w = P w0} is a valid answer, and GLOP's is not reproducible.
// This restatement finds one by Caratheodory elimination (repeatedly moving
// along a null vector of r + 1 support columns of P until a weight reaches
// zero), which keeps every moment and ends with at most r points.
// ============================================================================
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace embed_oracle {

using i64 = int64_t;
using V3 = std::array<double, 3>;

static V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
static double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static V3 cross(const V3& a, const V3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
static double norm(const V3& a) { return std::sqrt(dot(a, a)); }

// Polygon area vector: fan from vertex 0, sum of 0.5 ab x ac (geometry/mod.rs:811-828).
static V3 area_vector(const std::vector<V3>& poly) {
  V3 s{0, 0, 0};
  for (size_t i = 1; i + 1 < poly.size(); ++i) {
    V3 c = cross(sub(poly[i], poly[0]), sub(poly[i + 1], poly[0]));
    for (int k = 0; k < 3; ++k) s[k] += c[k] * 0.5;
  }
  return s;
}

// compute_polyhedron_volume_from_faces (geometry/mod.rs:1002-1032).
static double polyhedron_volume(const std::vector<std::vector<V3>>& faces) {
  double vol = 0.0;
  for (const auto& f : faces) {
    if (f.size() > 2) {
      V3 a = area_vector(f);
      double area = norm(a);
      if (area > 0.0) {
        V3 n{a[0] / area, a[1] / area, a[2] / area};
        vol += dot(n, f[0]) * area;
      }
    }
  }
  return std::fabs(vol) / 3.0;
}

// Tetrahedron faces tri(0,1,2), tri(0,3,1), tri(1,3,2), tri(0,2,3) (geometry/mod.rs:1086-1097).
static double tet_volume(const V3 x[4]) {
  static const int F[4][3] = {{0, 1, 2}, {0, 3, 1}, {1, 3, 2}, {0, 2, 3}};
  std::vector<std::vector<V3>> faces;
  for (auto& f : F) faces.push_back({x[f[0]], x[f[1]], x[f[2]]});
  return polyhedron_volume(faces);
}

// Hexahedron faces quad(0,1,2,3), (4,5,1,0), (5,6,2,1), (6,7,3,2), (0,3,7,4),
// (4,7,6,5), each with an inward normal (geometry/mod.rs:597-622).
static const int HEX_FACES[6][4] = {{0, 1, 2, 3}, {4, 5, 1, 0}, {5, 6, 2, 1}, {6, 7, 3, 2}, {0, 3, 7, 4}, {4, 7, 6, 5}};

struct PolyMesh {
  std::vector<V3> vertices;
  std::vector<std::vector<int>> faces;
  std::vector<std::vector<int>> cells;
};

// PolyMesh::from(&Tet4Mesh): faces deduplicated by vertex set, each kept with
// the vertex order of its first occurrence (mesh_convert.rs:578-637); Tet4
// face order (connectivity.rs:489-499).
static PolyMesh polymesh_from_tets(const double* X, i64 nv, const i64* tets, i64 nt) {
  static const int TF[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {0, 3, 2}};
  PolyMesh m;
  m.vertices.resize(nv);
  for (i64 i = 0; i < nv; ++i) m.vertices[i] = {X[3 * i], X[3 * i + 1], X[3 * i + 2]};
  std::map<std::array<i64, 3>, int> index;
  for (i64 t = 0; t < nt; ++t) {
    std::vector<int> cell;
    for (auto& f : TF) {
      std::array<i64, 3> v{tets[4 * t + f[0]], tets[4 * t + f[1]], tets[4 * t + f[2]]};
      std::array<i64, 3> key = v;
      std::sort(key.begin(), key.end());
      auto it = index.find(key);
      int fi;
      if (it == index.end()) {
        fi = (int)m.faces.size();
        m.faces.push_back({(int)v[0], (int)v[1], (int)v[2]});
        index.emplace(key, fi);
      } else {
        fi = it->second;
      }
      cell.push_back(fi);
    }
    m.cells.push_back(cell);
  }
  return m;
}

// keep_cells: the listed cells, with faces and vertices renumbered in their
// original relative order (polymesh.rs:509-571).
static PolyMesh keep_cells(const PolyMesh& m, const std::vector<int>& cells) {
  std::set<int> fset, vset;
  for (int c : cells)
    for (int f : m.cells[c]) {
      fset.insert(f);
      for (int v : m.faces[f]) vset.insert(v);
    }
  std::map<int, int> fmap, vmap;
  PolyMesh r;
  for (int v : vset) {
    vmap[v] = (int)r.vertices.size();
    r.vertices.push_back(m.vertices[v]);
  }
  for (int f : fset) {
    fmap[f] = (int)r.faces.size();
    std::vector<int> fv;
    for (int v : m.faces[f]) fv.push_back(vmap[v]);
    r.faces.push_back(fv);
  }
  for (int c : cells) {
    std::vector<int> cf;
    for (int f : m.cells[c]) cf.push_back(fmap[f]);
    r.cells.push_back(cf);
  }
  return r;
}

// closest_point_to_plane on the segment a -> b (geometry/mod.rs:741-774).
static V3 segment_plane_point(const V3& a, const V3& b, const V3& x0, const V3& n) {
  V3 d = sub(b, a), y = sub(x0, a);
  double nTd = dot(n, d), nTy = dot(n, y);
  double t;
  if (std::signbit(nTd) == std::signbit(nTy)) {
    t = std::fabs(nTy) >= std::fabs(nTd) ? 1.0 : nTy / nTd;
  } else {
    t = 0.0;
  }
  V3 r;
  for (int k = 0; k < 3; ++k) r[k] = a[k] * (1.0 - t) + b[k] * t;
  return r;
}

using Edge = std::pair<int, int>;  // undirected, first <= second; (a, a) = original vertex a
static Edge edge(int a, int b) { return a <= b ? Edge{a, b} : Edge{b, a}; }

// PolyMesh3d::intersect_half_space (polymesh.rs:640-808): keeps the part of
// every cell on the side n.(x - x0) >= 0.
static PolyMesh intersect_half_space(const PolyMesh& m, const V3& x0, const V3& n) {
  const int nv = (int)m.vertices.size();
  std::vector<char> inside(nv);
  for (int v = 0; v < nv; ++v) inside[v] = dot(n, sub(m.vertices[v], x0)) >= 0.0;
  enum { IN, OUT, CUT };
  std::vector<std::vector<Edge>> nf;
  std::vector<int> cls;
  for (const auto& f : m.faces) {
    std::vector<Edge> out;
    int c = IN;
    const int k = (int)f.size();
    for (int i = 0; i < k; ++i) {
      int a = f[i], b = f[(i + 1) % k];
      if (inside[a]) out.push_back(Edge{a, a});
      if (inside[a] != inside[b]) {
        out.push_back(edge(a, b));
        c = CUT;
      }
    }
    if (out.empty()) c = OUT;
    nf.push_back(out);
    cls.push_back(c);
  }
  auto is_cut_vertex = [](const Edge& e) { return e.first != e.second; };
  std::vector<std::vector<int>> ncells;
  for (const auto& cf : m.cells) {
    std::vector<int> cellf;
    std::vector<std::pair<Edge, Edge>> iedges;
    for (int fi : cf) {
      if (cls[fi] == IN) cellf.push_back(fi);
      else if (cls[fi] == CUT) {
        cellf.push_back(fi);
        const auto& fv = nf[fi];
        const int k = (int)fv.size();
        for (int i = 0; i < k; ++i) {
          const Edge& a = fv[i];
          const Edge& b = fv[(i + 1) % k];
          if (is_cut_vertex(a) && is_cut_vertex(b)) iedges.push_back({a, b});
        }
      }
    }
    // string the intersection edges into new faces
    while (!iedges.empty()) {
      auto start = iedges.back();
      iedges.pop_back();
      std::vector<Edge> face{start.first};
      Edge next = start.second;
      for (;;) {
        size_t pos = iedges.size();
        for (size_t i = 0; i < iedges.size(); ++i)
          if (iedges[i].first == next || iedges[i].second == next) { pos = i; break; }
        if (pos == iedges.size()) break;
        auto e = iedges[pos];
        iedges[pos] = iedges.back();  // swap_remove
        iedges.pop_back();
        if (e.first == next) {
          face.push_back(e.first);
          next = e.second;
        } else {
          face.push_back(e.second);
          next = e.first;
        }
      }
      cellf.push_back((int)nf.size());
      nf.push_back(face);
    }
    ncells.push_back(cellf);
  }
  // vertex labels by first appearance over all faces (generate_edge_repr_vertex_labels)
  std::map<Edge, int> label;
  for (const auto& f : nf)
    for (const Edge& e : f)
      if (!label.count(e)) {
        int l = (int)label.size();
        label.emplace(e, l);
      }
  PolyMesh r;
  r.vertices.resize(label.size());
  for (const auto& kv : label) {
    const Edge& e = kv.first;
    if (e.first == e.second) r.vertices[kv.second] = m.vertices[e.first];
    else r.vertices[kv.second] = segment_plane_point(m.vertices[e.first], m.vertices[e.second], x0, n);
  }
  // faces: drop empty ones, renumber in order
  std::vector<int> fmap(nf.size(), -1);
  for (size_t i = 0; i < nf.size(); ++i) {
    if (nf[i].empty()) continue;
    fmap[i] = (int)r.faces.size();
    std::vector<int> fv;
    for (const Edge& e : nf[i]) fv.push_back(label[e]);
    r.faces.push_back(fv);
  }
  for (const auto& c : ncells) {
    if (c.empty()) continue;
    std::vector<int> cf;
    for (int f : c) cf.push_back(fmap[f]);
    r.cells.push_back(cf);
  }
  return r;
}

// triangulate (Max 2000) + Tet4Mesh::try_from: the tetrahedra of every cell,
// each as 4 vertex indices (base a, b, c oriented towards the apex, apex).
static std::vector<std::array<int, 4>> tetrahedralize(const PolyMesh& m) {
  // fan triangulation of every face from its smallest vertex index
  std::vector<std::vector<std::array<int, 3>>> tri(m.faces.size());
  for (size_t fi = 0; fi < m.faces.size(); ++fi) {
    const auto& f = m.faces[fi];
    if (f.size() < 3) throw std::runtime_error("face with less than 3 vertices");
    const int k = (int)f.size();
    int mi = (int)(std::min_element(f.begin(), f.end()) - f.begin());
    for (int i = 0; i + 2 < k; ++i) tri[fi].push_back({f[mi], f[(i + 1 + mi) % k], f[(i + 2 + mi) % k]});
  }
  std::vector<std::array<int, 4>> tets;
  for (const auto& cell : m.cells) {
    if (cell.empty()) continue;
    int v = INT32_MAX;
    for (int fi : cell)
      for (int x : m.faces[fi]) v = std::min(v, x);
    for (int fi : cell) {
      const auto& fv = m.faces[fi];
      if (std::find(fv.begin(), fv.end(), v) != fv.end()) continue;
      for (const auto& t : tri[fi]) {
        std::array<int, 3> base{t[0], t[1], t[2]};
        // Triangle::point_orientation of the apex (geometry/mod.rs:372-389)
        V3 a = m.vertices[base[0]], b = m.vertices[base[1]], c = m.vertices[base[2]];
        V3 nrm = cross(sub(b, a), sub(c, a));
        double nn = norm(nrm);
        V3 nu{nrm[0] / nn, nrm[1] / nn, nrm[2] / nn};
        double d = dot(nu, sub(m.vertices[v], a));
        if (d < 0.0) std::swap(base[0], base[1]);
        tets.push_back({base[0], base[1], base[2], v});
      }
    }
  }
  return tets;
}

// ---- background element (Hex27 / Hex8 geometry = the 8 corners) ------------
static const double HEX8_ALPHA[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                        {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
static void hex8_map(const V3 X[8], const V3& xi, V3& x, double J[9]) {
  x = {0, 0, 0};
  for (int k = 0; k < 9; ++k) J[k] = 0.0;
  for (int I = 0; I < 8; ++I) {
    const double* a = HEX8_ALPHA[I];
    double p0 = (1.0 + a[0] * xi[0]) / 2.0, p1 = (1.0 + a[1] * xi[1]) / 2.0, p2 = (1.0 + a[2] * xi[2]) / 2.0;
    double N = p0 * p1 * p2;
    double g[3] = {a[0] / 2.0 * p1 * p2, p0 * a[1] / 2.0 * p2, p0 * p1 * a[2] / 2.0};
    for (int i = 0; i < 3; ++i) {
      x[i] += X[I][i] * N;
      for (int j = 0; j < 3; ++j) J[3 * i + j] += X[I][i] * g[j];
    }
  }
}
static double det3(const double J[9]) {
  return J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) + J[2] * (J[3] * J[7] - J[4] * J[6]);
}
// 3x3 solve by Gaussian elimination with full pivoting
static bool solve3(const double J[9], const double b[3], double x[3]) {
  double A[3][4];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) A[i][j] = J[3 * i + j];
    A[i][3] = b[i];
  }
  int col[3] = {0, 1, 2};
  for (int k = 0; k < 3; ++k) {
    int pi = k, pj = k;
    for (int i = k; i < 3; ++i)
      for (int j = k; j < 3; ++j)
        if (std::fabs(A[i][j]) > std::fabs(A[pi][pj])) { pi = i; pj = j; }
    if (A[pi][pj] == 0.0) return false;
    for (int j = 0; j < 4; ++j) std::swap(A[k][j], A[pi][j]);
    for (int i = 0; i < 3; ++i) std::swap(A[i][k], A[i][pj]);
    std::swap(col[k], col[pj]);
    for (int i = k + 1; i < 3; ++i) {
      double f = A[i][k] / A[k][k];
      for (int j = k; j < 4; ++j) A[i][j] -= f * A[k][j];
    }
  }
  double y[3];
  for (int k = 2; k >= 0; --k) {
    double s = A[k][3];
    for (int j = k + 1; j < 3; ++j) s -= A[k][j] * y[j];
    y[k] = s / A[k][k];
  }
  for (int k = 0; k < 3; ++k) x[col[k]] = y[k];
  return true;
}
// map_physical_coordinates: Newton from xi = 0, ||T(xi) - x|| <= 1e-12 diameter, <= 20 iterations.
static bool hex_inverse(const V3 X[8], const V3& x, V3& xi) {
  double diam = 0.0;
  for (int i = 0; i < 8; ++i)
    for (int j = i + 1; j < 8; ++j) diam = std::max(diam, norm(sub(X[i], X[j])));
  const double tol = 1e-12 * diam;
  xi = {0, 0, 0};
  V3 y;
  double J[9];
  hex8_map(X, xi, y, J);
  V3 f = sub(y, x);
  for (int it = 0;; ++it) {
    if (!(norm(f) > tol)) return true;
    if (it == 20) return false;
    double d[3];
    if (!solve3(J, f.data(), d)) return false;
    for (int k = 0; k < 3; ++k) xi[k] -= d[k];
    hex8_map(X, xi, y, J);
    f = sub(y, x);
  }
}

struct Result {
  std::vector<int> cls;          // per background cell: 0 exterior, 1 interior, 2 interface
  std::vector<double> cut_volume;
  std::vector<PolyMesh> cut;     // per background cell (interface cells only filled)
};

static bool aabb_overlap(const double a[6], const double b[6]) {
  for (int k = 0; k < 3; ++k)
    if (!(a[k] <= b[3 + k] && b[k] <= a[3 + k])) return false;
  return true;
}

static void hex_corners(const double* X, const i64* conn, int npc, i64 c, V3 H[8]) {
  for (int I = 0; I < 8; ++I) {
    i64 v = conn[npc * c + I];
    H[I] = {X[3 * v], X[3 * v + 1], X[3 * v + 2]};
  }
}

// embed_mesh_3d_with_opts: classify every background cell (embedding3d.rs:57-196).
static Result embed(const double* bgX, const i64* bg_conn, i64 nbc, int npc, const double* eX, i64 nev, const i64* tets,
                    i64 nt, double lower, double upper, bool keep_cut) {
  PolyMesh em = polymesh_from_tets(eX, nev, tets, nt);
  std::vector<std::array<double, 6>> tb(nt);
  for (i64 t = 0; t < nt; ++t) {
    double* b = tb[t].data();
    for (int k = 0; k < 3; ++k) { b[k] = INFINITY; b[3 + k] = -INFINITY; }
    for (int f : em.cells[t])
      for (int v : em.faces[f])
        for (int k = 0; k < 3; ++k) {
          b[k] = std::min(b[k], em.vertices[v][k]);
          b[3 + k] = std::max(b[3 + k], em.vertices[v][k]);
        }
  }
  Result r;
  r.cls.assign(nbc, 0);
  r.cut_volume.assign(nbc, 0.0);
  if (keep_cut) r.cut.resize(nbc);
#pragma omp parallel for schedule(dynamic, 4)
  for (i64 c = 0; c < nbc; ++c) {
    V3 H[8];
    hex_corners(bgX, bg_conn, npc, c, H);
    double cb[6];
    for (int k = 0; k < 3; ++k) { cb[k] = INFINITY; cb[3 + k] = -INFINITY; }
    for (auto& h : H)
      for (int k = 0; k < 3; ++k) { cb[k] = std::min(cb[k], h[k]); cb[3 + k] = std::max(cb[3 + k], h[k]); }
    std::vector<int> cand;
    for (i64 t = 0; t < nt; ++t)
      if (aabb_overlap(cb, tb[t].data())) cand.push_back((int)t);
    PolyMesh reg = keep_cells(em, cand);
    for (auto& hf : HEX_FACES) {
      std::vector<V3> q{H[hf[0]], H[hf[1]], H[hf[2]], H[hf[3]]};
      V3 a = area_vector(q);
      double an = norm(a);
      V3 n{a[0] / an, a[1] / an, a[2] / an};
      reg = intersect_half_space(reg, q[0], n);
    }
    int cls = 0;
    double vol = 0.0;
    if (!reg.cells.empty()) {
      std::vector<std::vector<V3>> hfaces;
      for (auto& hf : HEX_FACES) hfaces.push_back({H[hf[0]], H[hf[1]], H[hf[2]], H[hf[3]]});
      const double bgv = polyhedron_volume(hfaces);
      for (const auto& t : tetrahedralize(reg)) {
        V3 x[4] = {reg.vertices[t[0]], reg.vertices[t[1]], reg.vertices[t[2]], reg.vertices[t[3]]};
        vol += tet_volume(x);
      }
      cls = vol < lower * bgv ? 0 : (vol < upper * bgv ? 2 : 1);
    }
    r.cls[c] = cls;
    r.cut_volume[c] = vol;
    if (keep_cut && cls == 2) r.cut[c] = std::move(reg);
  }
  return r;
}

// compute_element_embedded_quadrature (embedding3d.rs:233-289): the tet rule
// on every tetrahedron of the cut polyhedron, mapped to the background
// element's reference coordinates; optional stabilization appended.
static void cell_quadrature(const PolyMesh& cut, const V3 H[8], const double* tw, const double* tp, int nq,
                            double stab_factor, const double* sw, const double* sp, int nsq, std::vector<double>& w,
                            std::vector<double>& p) {
  for (const auto& t : tetrahedralize(cut)) {
    V3 X[4] = {cut.vertices[t[0]], cut.vertices[t[1]], cut.vertices[t[2]], cut.vertices[t[3]]};
    // Tet4 element: N = [-(xi+eta+zeta+1)/2, (xi+1)/2, (eta+1)/2, (zeta+1)/2] (element.rs:978-1028)
    double Jt[9];
    for (int i = 0; i < 3; ++i) {
      Jt[3 * i + 0] = -0.5 * X[0][i] + 0.5 * X[1][i];
      Jt[3 * i + 1] = -0.5 * X[0][i] + 0.5 * X[2][i];
      Jt[3 * i + 2] = -0.5 * X[0][i] + 0.5 * X[3][i];
    }
    const double dJt = std::fabs(det3(Jt));
    for (int q = 0; q < nq; ++q) {
      const double* xi = tp + 3 * q;
      double N[4] = {-0.5 * xi[0] - 0.5 * xi[1] - 0.5 * xi[2] - 0.5, 0.5 * xi[0] + 0.5, 0.5 * xi[1] + 0.5,
                     0.5 * xi[2] + 0.5};
      V3 x{0, 0, 0};
      for (int I = 0; I < 4; ++I)
        for (int i = 0; i < 3; ++i) x[i] += X[I][i] * N[I];
      V3 xb;
      if (!hex_inverse(H, x, xb)) throw std::runtime_error("inverse map did not converge");
      V3 y;
      double Jb[9];
      hex8_map(H, xb, y, Jb);
      w.push_back(tw[q] * dJt / std::fabs(det3(Jb)));
      p.insert(p.end(), xb.begin(), xb.end());
    }
  }
  for (int q = 0; q < nsq; ++q) {
    w.push_back(stab_factor * sw[q]);
    p.insert(p.end(), sp + 3 * q, sp + 3 * q + 3);
  }
}

// ---- simplification -------------------------------------------------------
static double chebyshev(double x, int n) {
  if (n == 0) return 1.0;
  if (n == 1) return x;
  return 2.0 * x * chebyshev(x, n - 1) - chebyshev(x, n - 2);
}

// Moment matrix P (r x n, row-major): Chebyshev tensor products of total
// degree <= strength on the points' bounding box (quadrature_reduction.rs:35-105).
static int moment_matrix(const double* p, int n, int strength, std::vector<double>& P) {
  double lo[3], hi[3];
  for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[3 * i + k]); hi[k] = std::max(hi[k], p[3 * i + k]); }
  double al[3], be[3];
  for (int k = 0; k < 3; ++k) {
    double c = (lo[k] + hi[k]) / 2.0, l = (hi[k] - lo[k]) / 2.0;
    al[k] = l != 0.0 ? 1.0 / l : 0.0;
    be[k] = 1.0 - al[k] * (c + l);
  }
  P.clear();
  int r = 0;
  for (int a = 0; a <= strength; ++a)
    for (int b = 0; b <= strength; ++b)
      for (int c = 0; c <= strength; ++c) {
        if (a + b + c > strength) continue;
        for (int i = 0; i < n; ++i)
          P.push_back(chebyshev(al[0] * p[3 * i] + be[0], a) * chebyshev(al[1] * p[3 * i + 1] + be[1], b) *
                      chebyshev(al[2] * p[3 * i + 2] + be[2], c));
        ++r;
      }
  return r;
}

// Null vector of the r x (r + 1) matrix A (row-major): Gaussian elimination
// with partial pivoting; the last free column gets 1.
static void null_vector(std::vector<double> A, int r, std::vector<double>& z) {
  const int m = r + 1;
  std::vector<int> pivcol;
  int row = 0;
  double scale = 0.0;
  for (double v : A) scale = std::max(scale, std::fabs(v));
  const double eps = 1e-13 * scale;
  std::vector<char> is_piv(m, 0);
  for (int c = 0; c < m && row < r; ++c) {
    int pr = row;
    for (int i = row + 1; i < r; ++i)
      if (std::fabs(A[i * m + c]) > std::fabs(A[pr * m + c])) pr = i;
    if (std::fabs(A[pr * m + c]) <= eps) continue;
    if (pr != row)
      for (int j = 0; j < m; ++j) std::swap(A[row * m + j], A[pr * m + j]);
    for (int i = row + 1; i < r; ++i) {
      const double f = A[i * m + c] / A[row * m + c];
      for (int j = c; j < m; ++j) A[i * m + j] -= f * A[row * m + j];
    }
    pivcol.push_back(c);
    is_piv[c] = 1;
    ++row;
  }
  int free_col = m - 1;
  while (free_col >= 0 && is_piv[free_col]) --free_col;
  z.assign(m, 0.0);
  z[free_col] = 1.0;
  for (int k = (int)pivcol.size() - 1; k >= 0; --k) {
    const int c = pivcol[k];
    double s = 0.0;
    for (int j = c + 1; j < m; ++j) s += A[k * m + j] * z[j];
    z[c] = -s / A[k * m + c];
  }
}

// optimize_quadrature: rules with at most r points are returned unchanged.
static void simplify(const double* w0, const double* p, int n, int strength, std::vector<double>& w_out,
                     std::vector<double>& p_out) {
  std::vector<double> P;
  const int r = moment_matrix(p, n, strength, P);
  w_out.clear();
  p_out.clear();
  if (n <= r) {
    w_out.assign(w0, w0 + n);
    p_out.assign(p, p + 3 * n);
    return;
  }
  std::vector<double> w(w0, w0 + n);
  std::vector<int> S;
  for (int i = 0; i < n; ++i)
    if (w[i] > 0.0) S.push_back(i);
  std::vector<double> A((size_t)r * (r + 1)), z;
  while ((int)S.size() > r) {
    for (int i = 0; i < r; ++i)
      for (int j = 0; j <= r; ++j) A[(size_t)i * (r + 1) + j] = P[(size_t)i * n + S[j]];
    null_vector(A, r, z);
    bool pos = false;
    for (int j = 0; j <= r; ++j) pos = pos || z[j] > 0.0;
    if (!pos)
      for (double& v : z) v = -v;
    int arg = -1;
    double t = INFINITY;
    for (int j = 0; j <= r; ++j)
      if (z[j] > 0.0 && w[S[j]] / z[j] < t) { t = w[S[j]] / z[j]; arg = j; }
    for (int j = 0; j <= r; ++j) {
      double v = w[S[j]] - t * z[j];
      w[S[j]] = (j == arg || v < 0.0) ? 0.0 : v;
    }
    std::vector<int> S2;
    for (int i : S)
      if (w[i] > 0.0) S2.push_back(i);
    S.swap(S2);
  }
  for (int i : S) {
    w_out.push_back(w[i]);
    p_out.insert(p_out.end(), p + 3 * i, p + 3 * i + 3);
  }
}

}  // namespace embed_oracle

using namespace embed_oracle;

namespace {
thread_local std::string g_embed_error;
struct EmbedHandle {
  Result r;
  const double* bgX = nullptr;  // not owned; only used during quadrature
  std::vector<double> bg;
  std::vector<i64> conn;
  int npc = 8;
  std::vector<i64> offsets;
  std::vector<double> w, p;
};
}  // namespace

extern "C" {

const char* oracle_embed_last_error() { return g_embed_error.c_str(); }

// Classifies the background cells; keeps the cut polyhedra of interface cells.
void* oracle_embed_create(const double* bgX, i64 nbv, const i64* bg_conn, i64 nbc, int npc, const double* eX, i64 nev,
                          const i64* tets, i64 nt, double lower, double upper) {
  try {
    auto* h = new EmbedHandle();
    h->r = embed(bgX, bg_conn, nbc, npc, eX, nev, tets, nt, lower, upper, true);
    h->bg.assign(bgX, bgX + 3 * nbv);
    h->conn.assign(bg_conn, bg_conn + (size_t)npc * nbc);
    h->npc = npc;
    return h;
  } catch (const std::exception& ex) {
    g_embed_error = ex.what();
    return nullptr;
  }
}
void oracle_embed_destroy(void* h) { delete (EmbedHandle*)h; }
// cls per cell (0 exterior, 1 interior, 2 interface) and cut volume per cell
void oracle_embed_cells(void* hp, int* cls, double* vol) {
  auto* h = (EmbedHandle*)hp;
  for (size_t c = 0; c < h->r.cls.size(); ++c) {
    cls[c] = h->r.cls[c];
    if (vol) vol[c] = h->r.cut_volume[c];
  }
}
// Builds the interface quadratures (interface cells in cell order); returns the total point count.
i64 oracle_embed_quadrature(void* hp, const double* tw, const double* tp, int nq, double stab_factor, const double* sw,
                            const double* sp, int nsq) {
  auto* h = (EmbedHandle*)hp;
  try {
    std::vector<i64> cells;
    for (size_t c = 0; c < h->r.cls.size(); ++c)
      if (h->r.cls[c] == 2) cells.push_back((i64)c);
    std::vector<std::vector<double>> W(cells.size()), Pp(cells.size());
#pragma omp parallel for schedule(dynamic, 4)
    for (size_t k = 0; k < cells.size(); ++k) {
      V3 H[8];
      hex_corners(h->bg.data(), h->conn.data(), h->npc, cells[k], H);
      cell_quadrature(h->r.cut[cells[k]], H, tw, tp, nq, stab_factor, sw, sp, nsq, W[k], Pp[k]);
    }
    h->offsets.assign(1, 0);
    h->w.clear();
    h->p.clear();
    for (size_t k = 0; k < cells.size(); ++k) {
      h->w.insert(h->w.end(), W[k].begin(), W[k].end());
      h->p.insert(h->p.end(), Pp[k].begin(), Pp[k].end());
      h->offsets.push_back((i64)h->w.size());
    }
    return (i64)h->w.size();
  } catch (const std::exception& ex) {
    g_embed_error = ex.what();
    return -1;
  }
}
void oracle_embed_copy_quadrature(void* hp, i64* offsets, double* w, double* p) {
  auto* h = (EmbedHandle*)hp;
  std::copy(h->offsets.begin(), h->offsets.end(), offsets);
  std::copy(h->w.begin(), h->w.end(), w);
  std::copy(h->p.begin(), h->p.end(), p);
}

// Simplifies nrules rules (offsets nrules + 1); the output uses the same
// offsets layout and fits in buffers of the input's size.
int oracle_quadrature_simplify(i64 nrules, const i64* offsets, const double* w, const double* p, int strength,
                               i64* out_offsets, double* out_w, double* out_p) {
  std::vector<std::vector<double>> W(nrules), Pp(nrules);
#pragma omp parallel for schedule(dynamic, 4)
  for (i64 k = 0; k < nrules; ++k)
    simplify(w + offsets[k], p + 3 * offsets[k], (int)(offsets[k + 1] - offsets[k]), strength, W[k], Pp[k]);
  out_offsets[0] = 0;
  for (i64 k = 0; k < nrules; ++k) {
    std::copy(W[k].begin(), W[k].end(), out_w + out_offsets[k]);
    std::copy(Pp[k].begin(), Pp[k].end(), out_p + 3 * out_offsets[k]);
    out_offsets[k + 1] = out_offsets[k] + (i64)W[k].size();
  }
  return 0;
}

// Moment matrix of one rule (r x n row-major into P, r returned; P may be null to query r).
int oracle_moment_matrix(const double* p, int n, int strength, double* P) {
  std::vector<double> M;
  int r = moment_matrix(p, n, strength, M);
  if (P) std::copy(M.begin(), M.end(), P);
  return r;
}

}  // extern "C"
