// Synthetic scene construction (host).  Input building only: the meshes the
// reference would feed its hot path, built the way the reference builds them.
//
//  create_rectangular_uniform_hex_mesh   fenris/src/geometry/procedural.rs:191-250
//  PolyMesh3d::from(&HexMesh)            fenris/src/mesh_convert.rs:577-637
//  PolyMesh3d::triangulate (Max 2000)    fenris/src/geometry/polymesh.rs:402-500
//  PolyMesh::dedup_faces                 fenris/src/geometry/polymesh.rs:249-287
//  Tet4Mesh::try_from(&PolyMesh3d)       fenris/src/mesh_convert.rs:639-727
//  Tet10 / Hex27 refinement (FromTemp)   fenris/src/mesh_convert.rs:41-75,163-244,296-406
//  Mesh::keep_cells                      fenris/src/mesh.rs:321-366
//  quadrature tables                     fenris/src/quadrature.rs:698-781,1136-1220
// Node numbering (and hence the CSR pattern and the coloring) follows from
// these steps, so they are reproduced step by step; hash maps replace the
// reference's HashMap / FxHashMap only for lookups (labels are assigned in
// first-appearance order either way).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "scene.h"

namespace hoefem {

// ---- quadrature tables (fenris/src/quadrature.rs) ---------------------------
// tet_quadrature_strength_5: 14 points on the [-1,1]^3 corner simplex.
static const double TET5_W[14] = {
    0.15025056762402113439891420311104844508, 0.15025056762402113439891420311104844508,
    0.15025056762402113439891420311104844508, 0.15025056762402113439891420311104844508,
    0.097990724155149266058280273981770004697, 0.097990724155149266058280273981770004697,
    0.097990724155149266058280273981770004697, 0.097990724155149266058280273981770004697,
    0.05672802770277528858409257082700992237, 0.05672802770277528858409257082700992237,
    0.05672802770277528858409257082700992237, 0.05672802770277528858409257082700992237,
    0.05672802770277528858409257082700992237, 0.05672802770277528858409257082700992237};
static const double T5A = -0.37822816147339878040530853247308433401, T5B = -0.86531551557980365878407440258074699796;
static const double T5C = -0.81452949937821754719535217252593878951, T5D = 0.44358849813465264158605651757781636853;
static const double T5E = -0.90899259174870070101623894744132112187, T5F = -0.091007408251299298983761052558678878131;
static const double TET5_P[14][3] = {{T5A, T5A, T5B}, {T5A, T5B, T5A}, {T5B, T5A, T5A}, {T5A, T5A, T5A},
                                     {T5C, T5C, T5D}, {T5C, T5D, T5C}, {T5D, T5C, T5C}, {T5C, T5C, T5C},
                                     {T5E, T5F, T5F}, {T5F, T5E, T5F}, {T5E, T5E, T5F}, {T5E, T5F, T5E},
                                     {T5F, T5E, T5E}, {T5F, T5F, T5E}};
// hex_quadrature_strength_5: 14 points on [-1,1]^3.
static const double H5W1 = 0.88642659279778393351800554016620498615, H5W2 = 0.33518005540166204986149584487534626039;
static const double H5A = 0.79582242575422146326454882047613584616, H5B = 0.75878691063932814626903427811226742764;
static const double HEX5_W[14] = {H5W1, H5W1, H5W1, H5W1, H5W1, H5W1, H5W2, H5W2, H5W2, H5W2, H5W2, H5W2, H5W2, H5W2};
static const double HEX5_P[14][3] = {{-H5A, 0, 0},      {0, 0, H5A},      {0, H5A, 0},     {0, 0, -H5A},
                                     {H5A, 0, 0},       {0, -H5A, 0},     {H5B, -H5B, -H5B}, {-H5B, H5B, H5B},
                                     {-H5B, H5B, -H5B}, {-H5B, -H5B, -H5B}, {-H5B, -H5B, H5B}, {H5B, H5B, -H5B},
                                     {H5B, H5B, H5B},   {H5B, -H5B, H5B}};

// tet_quadrature_strength_1 / _2 / _3 (quadrature.rs:570-696): 1, 4 and 8
// points on the same simplex (embedded cut-cell quadrature).
static const double T2A = -0.72360679774997896964091736687312762354, T2B = 0.17082039324993690892275210061938287063;
static const double T3A = -0.34367339496723662642072827083693243093, T3B = -0.9689798150982901207378151874892027072;
static const double T3C = -0.78390550020314279176487322158837338344, T3D = 0.35171650060942837529461966476512015033;
static const double T3W1 = 0.18162379004944980942342872025562069427, T3W2 = 0.15170954328388352390990461307771263906;
static const double TET1_P[1][3] = {{-0.5, -0.5, -0.5}};
static const double TET2_P[4][3] = {{T2A, T2A, T2B}, {T2A, T2B, T2A}, {T2B, T2A, T2A}, {T2A, T2A, T2A}};
static const double TET3_W[8] = {T3W1, T3W1, T3W1, T3W1, T3W2, T3W2, T3W2, T3W2};
static const double TET3_P[8][3] = {{T3A, T3A, T3B}, {T3A, T3B, T3A}, {T3B, T3A, T3A}, {T3A, T3A, T3A},
                                    {T3C, T3C, T3D}, {T3C, T3D, T3C}, {T3D, T3C, T3C}, {T3C, T3C, T3C}};

// Tet rule of the given strength (1, 2, 3, 5); false for other strengths.
bool tet_quadrature(int strength, std::vector<double>& w, std::vector<double>& p) {
  p.clear();
  switch (strength) {
    case 1:
      w.assign(1, 4.0 / 3.0);
      p.assign(&TET1_P[0][0], &TET1_P[0][0] + 3);
      return true;
    case 2:
      w.assign(4, 0.33333333333333333333333333333333333333);
      for (auto& x : TET2_P) p.insert(p.end(), x, x + 3);
      return true;
    case 3:
      w.assign(TET3_W, TET3_W + 8);
      for (auto& x : TET3_P) p.insert(p.end(), x, x + 3);
      return true;
    case 5:
      w.assign(TET5_W, TET5_W + 14);
      for (auto& x : TET5_P) p.insert(p.end(), x, x + 3);
      return true;
    default:
      return false;
  }
}

void tet_quadrature_5(std::vector<double>& w, std::vector<double>& p) {
  w.assign(TET5_W, TET5_W + 14);
  p.clear();
  for (auto& x : TET5_P) p.insert(p.end(), x, x + 3);
}
void hex_quadrature_5(std::vector<double>& w, std::vector<double>& p) {
  w.assign(HEX5_W, HEX5_W + 14);
  p.clear();
  for (auto& x : HEX5_P) p.insert(p.end(), x, x + 3);
}

// ---- seeded random numbers ----------------------------------------------------
uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uniform01(uint64_t& s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }
void random_normal(uint64_t seed, int64_t n, double sigma, double* out) {
  uint64_t s = seed;
  const double two_pi = 6.283185307179586476925286766559;
  for (int64_t i = 0; i < n; i += 2) {
    double u1 = 1.0 - uniform01(s);  // (0, 1]
    double u2 = uniform01(s);
    double r = std::sqrt(-2.0 * std::log(u1));
    out[i] = sigma * r * std::cos(two_pi * u2);
    if (i + 1 < n) out[i + 1] = sigma * r * std::sin(two_pi * u2);
  }
}

// ---- meshes --------------------------------------------------------------------
namespace {

template <int N>
struct ArrHash {
  size_t operator()(const std::array<int64_t, N>& a) const {
    uint64_t h = 1469598103934665603ull;
    for (int64_t x : a) {
      h ^= (uint64_t)x + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
      h *= 1099511628211ull;
    }
    return (size_t)h;
  }
};

struct Cells {
  std::vector<double> X;
  std::vector<int64_t> C;  // flat
  int nn = 0;
};

Cells hex_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cpu) {
  Cells m;
  m.nn = 8;
  if (cpu == 0 || ux == 0 || uy == 0) return m;
  const double h = unit / (double)cpu;
  const int64_t nx = ux * cpu, ny = uy * cpu, nz = uz * cpu;
  const int64_t vx = nx + 1, vy = ny + 1, vz = nz + 1;
  auto idx = [&](int64_t i, int64_t j, int64_t k) { return vx * vy * k + vx * j + i; };
  m.X.reserve(3 * vx * vy * vz);
  for (int64_t k = 0; k < vz; ++k)
    for (int64_t j = 0; j < vy; ++j)
      for (int64_t i = 0; i < vx; ++i) {
        m.X.push_back((double)i * h);
        m.X.push_back((double)j * h);
        m.X.push_back((double)k * h);
      }
  for (int64_t k = 0; k < nz; ++k)
    for (int64_t j = 0; j < ny; ++j)
      for (int64_t i = 0; i < nx; ++i) {
        const int64_t c[8] = {idx(i, j, k),     idx(i + 1, j, k),     idx(i + 1, j + 1, k),     idx(i, j + 1, k),
                              idx(i, j, k + 1), idx(i + 1, j, k + 1), idx(i + 1, j + 1, k + 1), idx(i, j + 1, k + 1)};
        m.C.insert(m.C.end(), c, c + 8);
      }
  return m;
}

// Hex -> PolyMesh faces (shared faces stored once, first orientation kept) ->
// Max triangulation -> dedup -> Tet4 with the apex on the non-negative side.
Cells tet4_from_hex(const Cells& hx) {
  static const int HF[6][4] = {{3, 2, 1, 0}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {4, 7, 3, 0}, {5, 6, 7, 4}};
  const int64_t ncell = (int64_t)hx.C.size() / 8;
  std::vector<std::array<int64_t, 4>> faces;
  std::vector<std::array<int64_t, 6>> cells(ncell);
  {
    std::unordered_map<std::array<int64_t, 4>, int64_t, ArrHash<4>> map;
    map.reserve(ncell * 4);
    for (int64_t c = 0; c < ncell; ++c)
      for (int f = 0; f < 6; ++f) {
        std::array<int64_t, 4> face = {hx.C[8 * c + HF[f][0]], hx.C[8 * c + HF[f][1]], hx.C[8 * c + HF[f][2]],
                                       hx.C[8 * c + HF[f][3]]};
        auto key = face;
        std::sort(key.begin(), key.end());
        auto it = map.find(key);
        int64_t fi;
        if (it != map.end()) fi = it->second;
        else {
          fi = (int64_t)faces.size();
          faces.push_back(face);
          map.emplace(key, fi);
        }
        cells[c][f] = fi;
      }
  }
  // triangulate faces from their smallest vertex
  std::vector<std::array<int64_t, 3>> tri;
  std::vector<std::array<int64_t, 2>> fmap(faces.size());
  for (size_t f = 0; f < faces.size(); ++f) {
    const auto& fc = faces[f];
    int mi = 0;
    for (int i = 1; i < 4; ++i)
      if (fc[i] < fc[mi]) mi = i;
    for (int i = 0; i < 2; ++i) {
      fmap[f][i] = (int64_t)tri.size();
      tri.push_back({fc[mi], fc[(i + 1 + mi) % 4], fc[(i + 2 + mi) % 4]});
    }
  }
  // tetrahedra: the cell's smallest vertex joined to the triangles of the faces
  // that do not contain it.  The base triangle is the triangulated original
  // face (dedup keeps the first copy, i.e. that triangle); the apex is v.
  Cells t;
  t.nn = 4;
  t.X = hx.X;
  for (int64_t c = 0; c < ncell; ++c) {
    int64_t v = -1;
    for (int f = 0; f < 6; ++f)
      for (int64_t x : faces[cells[c][f]])
        if (v < 0 || x < v) v = x;
    for (int f = 0; f < 6; ++f) {
      const auto& of = faces[cells[c][f]];
      if (std::find(of.begin(), of.end(), v) != of.end()) continue;
      for (int k = 0; k < 2; ++k) {
        auto b = tri[fmap[cells[c][f]][k]];
        const double* a0 = &t.X[3 * b[0]];
        const double* a1 = &t.X[3 * b[1]];
        const double* a2 = &t.X[3 * b[2]];
        const double* p = &t.X[3 * v];
        double ab[3] = {a1[0] - a0[0], a1[1] - a0[1], a1[2] - a0[2]};
        double ac[3] = {a2[0] - a0[0], a2[1] - a0[1], a2[2] - a0[2]};
        double nrm[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
        double len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        double d = (nrm[0] / len) * (p[0] - a0[0]) + (nrm[1] / len) * (p[1] - a0[1]) + (nrm[2] / len) * (p[2] - a0[2]);
        if (d < 0.0) std::swap(b[0], b[1]);
        t.C.insert(t.C.end(), {b[0], b[1], b[2], v});
      }
    }
  }
  return t;
}

// FromTemp refinement: nodes labelled in first-appearance order keyed by the
// sorted parent vertex set.
Cells refine(const Cells& m, int target) {
  static const int TE[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {2, 3}, {1, 3}};
  static const int HE[12][2] = {{0, 1}, {0, 3}, {0, 4}, {1, 2}, {1, 5}, {2, 3},
                                {2, 6}, {3, 7}, {4, 5}, {4, 7}, {5, 6}, {6, 7}};
  static const int HFN[6][4] = {{0, 1, 2, 3}, {0, 1, 4, 5}, {0, 3, 4, 7}, {1, 2, 5, 6}, {2, 3, 6, 7}, {4, 5, 6, 7}};
  static const double HFX[6][3] = {{0, 0, -1}, {0, -1, 0}, {-1, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  static const double HA[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                  {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  Cells out;
  out.nn = target == HOEFEM_ELEM_TET10 ? 10 : 27;
  const int64_t ncell = (int64_t)m.C.size() / m.nn;
  std::unordered_map<std::array<int64_t, 8>, int64_t, ArrHash<8>> label;
  label.reserve(ncell * (target == HOEFEM_ELEM_TET10 ? 3 : 8));
  out.C.reserve(ncell * out.nn);
  auto hex8_map = [&](const int64_t* c, const double* xi, double* x) {
    for (int d = 0; d < 3; ++d) x[d] = 0.0;
    for (int I = 0; I < 8; ++I) {
      double N = (1.0 + HA[I][0] * xi[0]) / 2.0 * ((1.0 + HA[I][1] * xi[1]) / 2.0) * ((1.0 + HA[I][2] * xi[2]) / 2.0);
      for (int d = 0; d < 3; ++d) x[d] += m.X[3 * c[I] + d] * N;
    }
  };
  for (int64_t e = 0; e < ncell; ++e) {
    const int64_t* c = &m.C[e * m.nn];
    std::vector<std::array<int64_t, 8>> par;
    std::vector<std::array<double, 3>> pos;
    auto key = [](std::initializer_list<int64_t> l) {
      std::array<int64_t, 8> k;
      k.fill(-1);
      int i = 0;
      for (int64_t x : l) k[i++] = x;
      std::sort(k.begin(), k.begin() + i);
      return k;
    };
    auto P = [&](int64_t i) { return std::array<double, 3>{m.X[3 * i], m.X[3 * i + 1], m.X[3 * i + 2]}; };
    for (int I = 0; I < m.nn; ++I) {
      par.push_back(key({c[I]}));
      pos.push_back(P(c[I]));
    }
    auto edge = [&](int a, int b) {
      par.push_back(key({c[a], c[b]}));
      auto pa = P(c[a]), pb = P(c[b]);
      pos.push_back({pa[0] * 0.5 + pb[0] * 0.5, pa[1] * 0.5 + pb[1] * 0.5, pa[2] * 0.5 + pb[2] * 0.5});
    };
    if (target == HOEFEM_ELEM_TET10) {
      for (auto& ed : TE) edge(ed[0], ed[1]);
    } else {
      for (auto& ed : HE) edge(ed[0], ed[1]);
      for (int f = 0; f < 6; ++f) {
        par.push_back(key({c[HFN[f][0]], c[HFN[f][1]], c[HFN[f][2]], c[HFN[f][3]]}));
        std::array<double, 3> x;
        hex8_map(c, HFX[f], x.data());
        pos.push_back(x);
      }
      par.push_back(key({c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]}));
      const double zero[3] = {0, 0, 0};
      std::array<double, 3> x;
      hex8_map(c, zero, x.data());
      pos.push_back(x);
    }
    for (size_t k = 0; k < par.size(); ++k) {
      auto it = label.find(par[k]);
      if (it != label.end()) out.C.push_back(it->second);
      else {
        int64_t l = (int64_t)(out.X.size() / 3);
        label.emplace(par[k], l);
        out.X.insert(out.X.end(), pos[k].begin(), pos[k].end());
        out.C.push_back(l);
      }
    }
  }
  return out;
}

Cells keep_cells(const Cells& m, const std::vector<int64_t>& cells) {
  const int64_t nv = (int64_t)m.X.size() / 3;
  std::vector<char> keep(nv, 0);
  for (int64_t c : cells)
    for (int I = 0; I < m.nn; ++I) keep[m.C[c * m.nn + I]] = 1;
  std::vector<int64_t> lab(nv, -1);
  Cells out;
  out.nn = m.nn;
  int64_t next = 0;
  for (int64_t i = 0; i < nv; ++i)
    if (keep[i]) {
      lab[i] = next++;
      out.X.insert(out.X.end(), m.X.begin() + 3 * i, m.X.begin() + 3 * i + 3);
    }
  for (int64_t c : cells)
    for (int I = 0; I < m.nn; ++I) out.C.push_back(lab[m.C[c * m.nn + I]]);
  return out;
}

double hex8_detj(const double* Xc /* 8 x 3 */, const double* xi) {
  static const double HA[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                  {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  double J[9] = {0};
  for (int c = 0; c < 8; ++c) {
    double l0 = (1.0 + HA[c][0] * xi[0]) / 2.0, l1 = (1.0 + HA[c][1] * xi[1]) / 2.0, l2 = (1.0 + HA[c][2] * xi[2]) / 2.0;
    double g[3] = {HA[c][0] / 2.0 * l1 * l2, l0 * HA[c][1] / 2.0 * l2, l0 * l1 * HA[c][2] / 2.0};
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) J[3 * i + j] += Xc[3 * c + i] * g[j];
  }
  return J[0] * (J[4] * J[8] - J[7] * J[5]) - J[1] * (J[3] * J[8] - J[6] * J[5]) + J[2] * (J[3] * J[7] - J[6] * J[4]);
}

}  // namespace

Scene* scene_tet10_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cpu) {
  Cells hx = hex_box(unit, ux, uy, uz, cpu);
  Cells t4 = tet4_from_hex(hx);
  Cells t10 = refine(t4, HOEFEM_ELEM_TET10);
  Scene* s = new Scene();
  s->X = std::move(t10.X);
  s->cell_size = unit / (double)cpu;
  SceneBlock b;
  b.kind = HOEFEM_ELEM_TET10;
  b.nn = 10;
  b.conn = std::move(t10.C);
  b.uniform = true;
  tet_quadrature_5(b.qw, b.qp);
  s->blocks.push_back(std::move(b));
  return s;
}

Scene* scene_hex27_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cpu) {
  Cells hx = hex_box(unit, ux, uy, uz, cpu);
  Cells h27 = refine(hx, HOEFEM_ELEM_HEX27);
  Scene* s = new Scene();
  s->X = std::move(h27.X);
  s->cell_size = unit / (double)cpu;
  SceneBlock b;
  b.kind = HOEFEM_ELEM_HEX27;
  b.nn = 27;
  b.conn = std::move(h27.C);
  b.uniform = true;
  hex_quadrature_5(b.qw, b.qp);
  s->blocks.push_back(std::move(b));
  return s;
}

Scene* scene_embedded_cylinder(int64_t n, double r_in, double r_out, int qmin, int qmax, uint64_t seed) {
  Cells hx = hex_box(1.0, 1, 1, 1, n);
  Cells h27 = refine(hx, HOEFEM_ELEM_HEX27);
  const int64_t ncell = (int64_t)hx.C.size() / 8;
  const int S = 8;  // sub-cell samples per axis for the volume fraction
  std::vector<double> phi(ncell);
  std::vector<int64_t> interior, interface;
  for (int64_t c = 0; c < ncell; ++c) {
    const int64_t* v = &hx.C[8 * c];
    double lo[3], hi[3];
    for (int d = 0; d < 3; ++d) { lo[d] = hx.X[3 * v[0] + d]; hi[d] = hx.X[3 * v[6] + d]; }
    int inside = 0;
    for (int a = 0; a < S; ++a)
      for (int b = 0; b < S; ++b)
        for (int k = 0; k < S; ++k) {
          double x = lo[0] + (hi[0] - lo[0]) * (a + 0.5) / S;
          double y = lo[1] + (hi[1] - lo[1]) * (b + 0.5) / S;
          (void)k;
          double r = std::sqrt((x - 0.5) * (x - 0.5) + (y - 0.5) * (y - 0.5));
          if (r >= r_in && r <= r_out) ++inside;
        }
    phi[c] = (double)inside / (double)(S * S * S);
    // thresholds of the reference's cut-cell classification (embedding3d.rs:129-143)
    if (phi[c] >= 0.999) interior.push_back(c);
    else if (phi[c] >= 1e-4) interface.push_back(c);
  }
  std::vector<int64_t> keep = interior;
  keep.insert(keep.end(), interface.begin(), interface.end());
  Cells km = keep_cells(h27, keep);
  Scene* s = new Scene();
  s->X = std::move(km.X);
  s->cell_size = 1.0 / (double)n;
  const int64_t ni = (int64_t)interior.size();
  SceneBlock bi, bf;
  bi.kind = bf.kind = HOEFEM_ELEM_HEX27;
  bi.nn = bf.nn = 27;
  bi.conn.assign(km.C.begin(), km.C.begin() + 27 * ni);
  bf.conn.assign(km.C.begin() + 27 * ni, km.C.end());
  bi.uniform = true;
  hex_quadrature_5(bi.qw, bi.qp);
  bf.uniform = false;
  uint64_t st = seed;
  bf.qoff.push_back(0);
  for (size_t k = 0; k < interface.size(); ++k) {
    int Q = qmin + (int)(splitmix64(st) % (uint64_t)(qmax - qmin + 1));
    double f = phi[interface[k]];
    std::vector<double> e(Q);
    double tot = 0.0;
    for (int q = 0; q < Q; ++q) {
      for (int d = 0; d < 3; ++d) bf.qp.push_back(2.0 * uniform01(st) - 1.0);
      e[q] = -std::log(1.0 - uniform01(st));
      tot += e[q];
    }
    for (int q = 0; q < Q; ++q) bf.qw.push_back(e[q] / tot * 8.0 * f);
    bf.qoff.push_back(bf.qoff.back() + Q);
  }
  s->blocks.push_back(std::move(bi));
  s->blocks.push_back(std::move(bf));
  return s;
}

void scene_volume_fractions(const Scene& s, double* out) {
  HOEFEM_REQUIRE(s.blocks.size() == 2, HOEFEM_ERR_INVALID_ARGUMENT, "scene has no interface block");
  const SceneBlock& b = s.blocks[1];
  const int64_t ne = (int64_t)b.conn.size() / 27;
  const double g = 1.0 / std::sqrt(3.0);
  for (int64_t e = 0; e < ne; ++e) {
    double Xc[24];
    for (int I = 0; I < 8; ++I)
      for (int d = 0; d < 3; ++d) Xc[3 * I + d] = s.X[3 * b.conn[27 * e + I] + d];
    double emb = 0.0;
    for (int64_t q = b.qoff[e]; q < b.qoff[e + 1]; ++q) emb += b.qw[q] * hex8_detj(Xc, &b.qp[3 * q]);
    double vol = 0.0;
    for (int a = 0; a < 8; ++a) {
      double xi[3] = {(a & 1) ? g : -g, (a & 2) ? g : -g, (a & 4) ? g : -g};
      vol += std::fabs(hex8_detj(Xc, xi));
    }
    out[e] = emb / vol;
  }
}

}  // namespace hoefem
