// ============================================================================
// hoefem_oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// FP64 CPU restatement of the reference's per-step hot path
// (InteractiveComputerGraphics/higher_order_embedded_fem): the CUDA library's
// results are compared with it, and it is the timed CPU baseline.  Nothing in the
// product (higher_order_embedded_fem_b200/) links or calls this file; only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
//
// The reference is Rust and cannot be built in this environment (no rustc,
// no MKL, no OR-Tools), so every function below is a restatement of the cited
// Rust source, pinned by the reference's own unit-test vectors (tests/golden).
// Threading mirrors rayon/paradis: colors run sequentially, the elements of a
// color run in parallel (OpenMP), so every CSR value / force entry receives
// its contributions in the same color order as the reference.
// ============================================================================
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <numeric>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

using i64 = int64_t;

// ---------------------------------------------------------------------------
// Small dense helpers (3x3 row-major: m[3*i+j] = M(i, j))
// ---------------------------------------------------------------------------
struct M3 {
  double m[9];
  double& operator()(int i, int j) { return m[3 * i + j]; }
  double operator()(int i, int j) const { return m[3 * i + j]; }
};

static M3 zero3() { M3 r; std::memset(r.m, 0, sizeof(r.m)); return r; }
static M3 eye3() { M3 r = zero3(); r(0, 0) = r(1, 1) = r(2, 2) = 1.0; return r; }
static M3 transpose(const M3& a) {
  M3 r;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r(i, j) = a(j, i);
  return r;
}
static M3 mul(const M3& a, const M3& b) {
  M3 r = zero3();
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += a(i, k) * b(k, j);
      r(i, j) = s;
    }
  return r;
}
static M3 add(const M3& a, const M3& b) { M3 r; for (int i = 0; i < 9; ++i) r.m[i] = a.m[i] + b.m[i]; return r; }
static M3 scale(const M3& a, double s) { M3 r; for (int i = 0; i < 9; ++i) r.m[i] = a.m[i] * s; return r; }
static double trace(const M3& a) { return a(0, 0) + a(1, 1) + a(2, 2); }
// nalgebra 0.21 3x3 determinant (cofactor expansion along the first row).
static double det3(const M3& m) {
  double m12_m23 = m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2);
  double m11_m23 = m(1, 0) * m(2, 2) - m(2, 0) * m(1, 2);
  double m11_m22 = m(1, 0) * m(2, 1) - m(2, 0) * m(1, 1);
  return m(0, 0) * m12_m23 - m(0, 1) * m11_m23 + m(0, 2) * m11_m22;
}
// Adjugate / det; returns false when det == 0 (nalgebra `try_inverse`).
static bool inv3(const M3& m, M3& out) {
  double d = det3(m);
  if (d == 0.0) return false;
  out(0, 0) = (m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2)) / d;
  out(0, 1) = -(m(0, 1) * m(2, 2) - m(2, 1) * m(0, 2)) / d;
  out(0, 2) = (m(0, 1) * m(1, 2) - m(1, 1) * m(0, 2)) / d;
  out(1, 0) = -(m(1, 0) * m(2, 2) - m(2, 0) * m(1, 2)) / d;
  out(1, 1) = (m(0, 0) * m(2, 2) - m(2, 0) * m(0, 2)) / d;
  out(1, 2) = -(m(0, 0) * m(1, 2) - m(1, 0) * m(0, 2)) / d;
  out(2, 0) = (m(1, 0) * m(2, 1) - m(2, 0) * m(1, 1)) / d;
  out(2, 1) = -(m(0, 0) * m(2, 1) - m(2, 0) * m(0, 1)) / d;
  out(2, 2) = (m(0, 0) * m(1, 1) - m(1, 0) * m(0, 1)) / d;
  return true;
}

// ---------------------------------------------------------------------------
// Materials — fenris/src/solid/materials.rs
// ---------------------------------------------------------------------------
enum MaterialKind { MAT_STVK = 0, MAT_SNH = 1, MAT_LINEAR = 2 };

struct Lame { double mu, lambda; };

// LameParameters::from(YoungPoisson), materials.rs:27-38.  The factor 0.5 on
// lambda (4x too small vs. the textbook formula) is the reference's documented
// erratum and is reproduced on purpose.
static Lame lame_from_young_poisson(double young, double poisson) {
  double mu = 0.5 * young / (1.0 + poisson);
  double lambda = 0.5 * mu * poisson / (1.0 - 2.0 * poisson);
  return {mu, lambda};
}

// reparametrize_lame_for_stable_neo_hookean, materials.rs:242-253 (d = 3).
static Lame snh_reparam(const Lame& l) {
  const double d = 3.0;
  return {(d + 1.0) / d * l.mu, l.lambda + (1.0 - 2.0 / (d * (d + 1.0))) * l.mu};
}

struct Material {
  int kind;
  Lame lame;
};

// StVK energy / stress / pair contraction, materials.rs:177-219.
static double stvk_energy(const Lame& l, const M3& F) {
  M3 E = scale(add(mul(transpose(F), F), scale(eye3(), -1.0)), 0.5);
  double tr = trace(E), fro = 0.0;
  for (double x : E.m) fro += x * x;
  return l.mu * fro + 0.5 * l.lambda * tr * tr;
}
static M3 stvk_stress(const Lame& l, const M3& F) {
  M3 E = scale(add(mul(transpose(F), F), scale(eye3(), -1.0)), 0.5);
  M3 S = add(scale(E, 2.0 * l.mu), scale(eye3(), l.lambda * trace(E)));
  return mul(F, S);
}
static M3 stvk_contract(const Lame& l, const M3& F, const double* a, const double* b) {
  M3 B;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) B(i, j) = a[i] * b[j];
  M3 E = scale(add(mul(transpose(F), F), scale(eye3(), -1.0)), 0.5);
  double EdotB = 0.0;
  for (int i = 0; i < 9; ++i) EdotB += E.m[i] * B.m[i];
  M3 first = scale(eye3(), EdotB * 2.0 * l.mu + l.lambda * trace(E) * trace(B));
  M3 inner = add(add(scale(transpose(B), l.mu), scale(B, l.lambda)), scale(eye3(), l.mu * trace(B)));
  return add(first, mul(mul(F, inner), transpose(F)));
}

// Linear elastic (used by the reference's CG FEM test), materials.rs:55-160.
static M3 linear_stress(const Lame& l, const M3& F) {
  M3 eps = scale(add(add(F, transpose(F)), scale(eye3(), -2.0)), 0.5);
  return add(scale(eps, 2.0 * l.mu), scale(eye3(), l.lambda * trace(eps)));
}
static M3 linear_contract(const Lame& l, const M3& /*F*/, const double* a, const double* b) {
  M3 B;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) B(i, j) = a[i] * b[j];
  M3 r = add(scale(eye3(), l.mu * trace(B)), add(scale(transpose(B), l.mu), scale(B, l.lambda)));
  return r;
}

// Stable Neo-Hookean, materials.rs:269-346.
static double snh_energy(const Lame& lame, const M3& F) {
  const double d = 3.0;
  Lame r = snh_reparam(lame);
  double a = r.mu / r.lambda * (d / (d + 1.0));
  double alpha = 1.0 + a;
  double IC = trace(mul(transpose(F), F));
  double J = det3(F);
  double Jm = J - alpha;
  // The reference evaluates this expression with the *un-reparametrised* mu and
  // lambda (materials.rs:295-296); kept as is.
  return 0.5 * lame.mu * (IC - d) + 0.5 * lame.lambda * ((Jm * Jm) - (a * a)) -
         0.5 * lame.mu * std::log((IC + 1.0) / (d + 1.0));
}
static bool snh_stress(const Lame& lame, const M3& F, M3& P) {
  const double d = 3.0;
  Lame r = snh_reparam(lame);
  double alpha = 1.0 + r.mu / r.lambda * (d / (d + 1.0));
  double IC = trace(mul(transpose(F), F));
  double J = det3(F);
  M3 Finv;
  if (!inv3(F, Finv)) return false;
  M3 dJdF = scale(transpose(Finv), J);
  P = add(scale(F, r.mu * (1.0 - 1.0 / (IC + 1.0))), scale(dJdF, r.lambda * (J - alpha)));
  return true;
}
static bool snh_contract(const Lame& lame, const M3& F, const double* a, const double* b, M3& out) {
  const double d = 3.0;
  M3 B;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) B(i, j) = a[i] * b[j];
  Lame r = snh_reparam(lame);
  double alpha = 1.0 + r.mu / r.lambda * (d / (d + 1.0));
  double IC = trace(mul(transpose(F), F));
  double J = det3(F);
  double beta = IC + 1.0, beta2 = beta * beta;
  double G = 1.0 - 1.0 / beta;
  double H = (J - alpha) * J;
  M3 Finv;
  if (!inv3(F, Finv)) return false;
  M3 FinvT = transpose(Finv);
  M3 Q = add(scale(mul(mul(F, B), transpose(F)), 2.0 / beta2), scale(eye3(), G * trace(B)));
  M3 R = add(scale(mul(mul(FinvT, B), Finv), (2.0 * J - alpha) * J),
             scale(mul(mul(FinvT, transpose(B)), Finv), -H));
  out = add(scale(Q, r.mu), scale(R, r.lambda));
  return true;
}

// vectorize (column-major, materials.rs:745-761): v[3*j + i] = M(i, j).
static void vectorize(const M3& m, double* v) {
  for (int j = 0; j < 3; ++j) for (int i = 0; i < 3; ++i) v[3 * j + i] = m(i, j);
}
// cross_product_matrix (fenris/src/util.rs): [v]_x
static M3 cross_mat(const double* v) {
  M3 r = zero3();
  r(0, 1) = -v[2]; r(0, 2) = v[1];
  r(1, 0) = v[2];  r(1, 2) = -v[0];
  r(2, 0) = -v[1]; r(2, 1) = v[0];
  return r;
}

// build_stable_neohookean_dp_df + add_volume_hessian_3d, materials.rs:504-557,763-776.
// C is 9x9 row-major: C[9*row + col], row = 3k+i, col = 3l+j.
static bool snh_dp_df(const Lame& reparam, const M3& F, double* C) {
  const double d = 3.0;
  double mu = reparam.mu, lambda = reparam.lambda;
  double alpha = 1.0 + mu / lambda * (d / (d + 1.0));
  double IC = trace(mul(transpose(F), F));
  double J = det3(F);
  double beta = IC + 1.0, beta2 = beta * beta;
  M3 Finv;
  if (!inv3(F, Finv)) return false;
  M3 dJdF = scale(transpose(Finv), J);
  double f[9], g[9];
  vectorize(F, f);
  vectorize(dJdF, g);
  for (int i = 0; i < 81; ++i) C[i] = 0.0;
  for (int i = 0; i < 9; ++i) C[9 * i + i] = mu * (1.0 - 1.0 / beta);
  double cf = mu * 2.0 / beta2;
  for (int i = 0; i < 9; ++i) for (int j = 0; j < 9; ++j) C[9 * i + j] += cf * f[i] * f[j];
  for (int i = 0; i < 9; ++i) for (int j = 0; j < 9; ++j) C[9 * i + j] += lambda * g[i] * g[j];
  double s = lambda * (J - alpha);
  double c0[3] = {F(0, 0), F(1, 0), F(2, 0)}, c1[3] = {F(0, 1), F(1, 1), F(2, 1)}, c2[3] = {F(0, 2), F(1, 2), F(2, 2)};
  M3 f0 = scale(cross_mat(c0), s), f1 = scale(cross_mat(c1), s), f2 = scale(cross_mat(c2), s);
  auto addblk = [&](int r0, int c0_, const M3& m, double sg) {
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) C[9 * (r0 + i) + (c0_ + j)] += sg * m(i, j);
  };
  addblk(3, 0, f2, 1.0);
  addblk(6, 0, f1, -1.0);
  addblk(0, 3, f2, -1.0);
  addblk(6, 3, f0, 1.0);
  addblk(0, 6, f1, 1.0);
  addblk(3, 6, f0, -1.0);
  return true;
}

// contract_stiffness_tensor, materials.rs:689-743: adds, J outer / I >= J inner,
// mirrored transposed into the (J, I) block.  out is (3n x 3n) row-major.
static void contract_stiffness_tensor(double* out, int n, const double* C, const double* a /* 3 x n row-major a[k*n+I] */) {
  const int dim = 3 * n;
  for (int J = 0; J < n; ++J) {
    for (int I = J; I < n; ++I) {
      double r[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int l = 0; l < 3; ++l)
        for (int k = 0; k < 3; ++k)
          for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i)
              r[i][j] += C[9 * (3 * k + i) + (3 * l + j)] * a[k * n + I] * a[l * n + J];
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) out[(3 * I + i) * dim + 3 * J + j] += r[i][j];
      if (I != J)
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) out[(3 * J + j) * dim + 3 * I + i] += r[i][j];
    }
  }
}

static bool material_stress(const Material& m, const M3& F, M3& P) {
  switch (m.kind) {
    case MAT_STVK: P = stvk_stress(m.lame, F); return true;
    case MAT_SNH: return snh_stress(m.lame, F, P);
    case MAT_LINEAR: P = linear_stress(m.lame, F); return true;
  }
  return false;
}

static double material_energy(const Material& m, const M3& F) {
  switch (m.kind) {
    case MAT_STVK: return stvk_energy(m.lame, F);
    case MAT_SNH: return snh_energy(m.lame, F);
    default: return 0.0;
  }
}

static bool material_contract_pair(const Material& m, const M3& F, const double* a, const double* b, M3& out) {
  switch (m.kind) {
    case MAT_STVK: out = stvk_contract(m.lame, F, a, b); return true;
    case MAT_SNH: return snh_contract(m.lame, F, a, b, out);
    case MAT_LINEAR: out = linear_contract(m.lame, F, a, b); return true;
  }
  return false;
}

// contract_multiple_stress_tensors_into: SNH uses the dp/df path
// (materials.rs:348-376); StVK / linear use the trait default pairwise loop
// (fenris/src/solid/mod.rs:56-86).  Adds into out.
static bool material_contract_multiple(const Material& m, double* out, const M3& F, const double* a, int n) {
  if (m.kind == MAT_SNH) {
    double C[81];
    if (!snh_dp_df(snh_reparam(m.lame), F, C)) return false;
    contract_stiffness_tensor(out, n, C, a);
    return true;
  }
  const int dim = 3 * n;
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      double ai[3] = {a[0 * n + i], a[1 * n + i], a[2 * n + i]};
      double aj[3] = {a[0 * n + j], a[1 * n + j], a[2 * n + j]};
      M3 c;
      if (!material_contract_pair(m, F, ai, aj, c)) return false;
      for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) out[(3 * i + r) * dim + 3 * j + s] += c(r, s);
      if (i != j)
        for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) out[(3 * j + r) * dim + 3 * i + s] += c(s, r);
    }
  return true;
}

// ---------------------------------------------------------------------------
// Reference elements — fenris/src/element.rs
// ---------------------------------------------------------------------------
enum ElementKind { ELEM_TET4 = 0, ELEM_TET10 = 1, ELEM_HEX8 = 2, ELEM_HEX27 = 3 };

static int element_nodes(int kind) {
  switch (kind) {
    case ELEM_TET4: return 4;
    case ELEM_TET10: return 10;
    case ELEM_HEX8: return 8;
    case ELEM_HEX27: return 27;
  }
  return 0;
}

// Tet4 on the [-1,1]^3 corner simplex, element.rs:978-1003.
static void tet4_basis(const double* xi, double* N) {
  N[0] = -0.5 * xi[0] - 0.5 * xi[1] - 0.5 * xi[2] - 0.5;
  N[1] = 0.5 * xi[0] + 0.5;
  N[2] = 0.5 * xi[1] + 0.5;
  N[3] = 0.5 * xi[2] + 0.5;
}
static void tet4_grad(double* g /* 3 x 4 */) {
  const double G[3][4] = {{-0.5, 0.5, 0.0, 0.0}, {-0.5, 0.0, 0.5, 0.0}, {-0.5, 0.0, 0.0, 0.5}};
  for (int k = 0; k < 3; ++k) for (int I = 0; I < 4; ++I) g[k * 4 + I] = G[k][I];
}
// Tet10 as products of Tet4 functions, element.rs:1896-1948.
static const int TET10_EDGES[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {2, 3}, {1, 3}};
static void tet10_basis(const double* xi, double* N) {
  double p[4];
  tet4_basis(xi, p);
  for (int i = 0; i < 4; ++i) N[i] = p[i] * (2.0 * p[i] - 1.0);
  for (int e = 0; e < 6; ++e) N[4 + e] = 4.0 * p[TET10_EDGES[e][0]] * p[TET10_EDGES[e][1]];
}
static void tet10_grad(const double* xi, double* g /* 3 x 10 */) {
  double p[4], g4[12];
  tet4_basis(xi, p);
  tet4_grad(g4);
  for (int k = 0; k < 3; ++k) {
    for (int i = 0; i < 4; ++i) g[k * 10 + i] = g4[k * 4 + i] * (4.0 * p[i] - 1.0);
    for (int e = 0; e < 6; ++e) {
      int a = TET10_EDGES[e][0], b = TET10_EDGES[e][1];
      g[k * 10 + 4 + e] = g4[k * 4 + a] * (4.0 * p[b]) + g4[k * 4 + b] * (4.0 * p[a]);
    }
  }
}
// Hex8 / Hex27 tensor-product bases, element.rs:1035-1195,1244-1423.
static const double HEX8_ALPHA[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                        {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
static const double HEX27_ALPHA[27][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
    {0, -1, -1},  {-1, 0, -1}, {-1, -1, 0}, {1, 0, -1}, {1, -1, 0}, {0, 1, -1}, {1, 1, 0}, {-1, 1, 0},
    {0, -1, 1},   {-1, 0, 1},  {1, 0, 1},   {0, 1, 1},  {0, 0, -1}, {0, -1, 0}, {-1, 0, 0}, {1, 0, 0},
    {0, 1, 0},    {0, 0, 1},   {0, 0, 0}};
static inline double phi_lin(double a, double x) { return (1.0 + a * x) / 2.0; }
static inline double phi_lin_grad(double a) { return a / 2.0; }
static inline double phi_quad(double a, double x) {
  double a2 = a * a, x2 = x * x;
  return (3.0 / 2.0 * a2 - 1.0) * x2 + 0.5 * a * x + 1.0 - a2;
}
static inline double phi_quad_grad(double a, double x) {
  double a2 = a * a;
  return 2.0 * (3.0 / 2.0 * a2 - 1.0) * x + 0.5 * a;
}
static void hex8_basis(const double* xi, double* N) {
  for (int I = 0; I < 8; ++I)
    N[I] = phi_lin(HEX8_ALPHA[I][0], xi[0]) * phi_lin(HEX8_ALPHA[I][1], xi[1]) * phi_lin(HEX8_ALPHA[I][2], xi[2]);
}
static void hex8_grad(const double* xi, double* g /* 3 x 8 */) {
  for (int I = 0; I < 8; ++I) {
    const double* a = HEX8_ALPHA[I];
    g[0 * 8 + I] = phi_lin_grad(a[0]) * phi_lin(a[1], xi[1]) * phi_lin(a[2], xi[2]);
    g[1 * 8 + I] = phi_lin(a[0], xi[0]) * phi_lin_grad(a[1]) * phi_lin(a[2], xi[2]);
    g[2 * 8 + I] = phi_lin(a[0], xi[0]) * phi_lin(a[1], xi[1]) * phi_lin_grad(a[2]);
  }
}
static void hex27_basis(const double* xi, double* N) {
  for (int I = 0; I < 27; ++I)
    N[I] = phi_quad(HEX27_ALPHA[I][0], xi[0]) * phi_quad(HEX27_ALPHA[I][1], xi[1]) * phi_quad(HEX27_ALPHA[I][2], xi[2]);
}
static void hex27_grad(const double* xi, double* g /* 3 x 27 */) {
  for (int I = 0; I < 27; ++I) {
    const double* a = HEX27_ALPHA[I];
    g[0 * 27 + I] = phi_quad_grad(a[0], xi[0]) * phi_quad(a[1], xi[1]) * phi_quad(a[2], xi[2]);
    g[1 * 27 + I] = phi_quad(a[0], xi[0]) * phi_quad_grad(a[1], xi[1]) * phi_quad(a[2], xi[2]);
    g[2 * 27 + I] = phi_quad(a[0], xi[0]) * phi_quad(a[1], xi[1]) * phi_quad_grad(a[2], xi[2]);
  }
}

static void element_basis(int kind, const double* xi, double* N) {
  switch (kind) {
    case ELEM_TET4: tet4_basis(xi, N); break;
    case ELEM_TET10: tet10_basis(xi, N); break;
    case ELEM_HEX8: hex8_basis(xi, N); break;
    case ELEM_HEX27: hex27_basis(xi, N); break;
  }
}
static void element_grad(int kind, const double* xi, double* g) {
  switch (kind) {
    case ELEM_TET4: tet4_grad(g); break;
    case ELEM_TET10: tet10_grad(xi, g); break;
    case ELEM_HEX8: hex8_grad(xi, g); break;
    case ELEM_HEX27: hex27_grad(xi, g); break;
  }
}

// reference_jacobian: J = X * G^T over the linear geometry nodes (Tet10 ->
// Tet4 corners, element.rs:1951-1955; Hex27 -> Hex8 corners, element.rs:1406-1408).
static M3 element_jacobian(int kind, const double* X /* n x 3 */, const double* xi) {
  double g[3 * 8];
  int ng;
  if (kind == ELEM_TET4 || kind == ELEM_TET10) { tet4_grad(g); ng = 4; }
  else { hex8_grad(xi, g); ng = 8; }
  M3 J = zero3();
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int I = 0; I < ng; ++I) s += X[3 * I + i] * g[j * ng + I];
      J(i, j) = s;
    }
  return J;
}
static void element_map(int kind, const double* X, const double* xi, double* x) {
  double N[8];
  int ng;
  if (kind == ELEM_TET4 || kind == ELEM_TET10) { tet4_basis(xi, N); ng = 4; }
  else { hex8_basis(xi, N); ng = 8; }
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int I = 0; I < ng; ++I) s += X[3 * I + i] * N[I];
    x[i] = s;
  }
}

// ---------------------------------------------------------------------------
// Element-level assembly — fenris/src/assembly.rs:618-797
// ---------------------------------------------------------------------------
struct Quad {
  const double* w;  // nq
  const double* p;  // nq x 3
  int nq;
};

// assemble_generalized_element_elliptic_term with MaterialEllipticOperator
// (g = -P^T), assembly.rs:673-711 + solid/assembly.rs:34-40.  fe is 3 x n.
static bool element_force(int kind, const double* X, const double* ue /* 3 x n */, const Quad& q,
                          const Material& mat, double* fe) {
  const int n = element_nodes(kind);
  for (int i = 0; i < 3 * n; ++i) fe[i] = 0.0;
  double G[3 * 27];
  for (int iq = 0; iq < q.nq; ++iq) {
    const double* xi = q.p + 3 * iq;
    double w = q.w[iq];
    element_grad(kind, xi, G);
    M3 J = element_jacobian(kind, X, xi);
    double Jdet = det3(J);
    M3 Jinv;
    if (!inv3(J, Jinv)) return false;
    // u_grad = (u * (G^T * J_inv))^T : u_grad(k, c) = sum_I (sum_m G(m,I) Jinv(m,k)) u(c,I)
    M3 ugrad = zero3();
    for (int k = 0; k < 3; ++k)
      for (int c = 0; c < 3; ++c) {
        double s = 0.0;
        for (int I = 0; I < n; ++I) {
          double gk = 0.0;
          for (int m = 0; m < 3; ++m) gk += G[m * n + I] * Jinv(m, k);
          s += ue[c * n + I] * gk;
        }
        ugrad(k, c) = s;
      }
    M3 F = add(transpose(ugrad), eye3());
    M3 P;
    if (!material_stress(mat, F, P)) return false;
    // f_e += (g^T * J_inv^T * G) * w * |detJ|, with g^T = -P
    M3 A = mul(scale(P, -1.0), transpose(Jinv));
    for (int i = 0; i < 3; ++i)
      for (int I = 0; I < n; ++I) {
        double s = 0.0;
        for (int m = 0; m < 3; ++m) s += A(i, m) * G[m * n + I];
        fe[i * n + I] += s * w * std::fabs(Jdet);
      }
  }
  return true;
}

// assemble_generalized_element_stiffness, assembly.rs:746-797.  Ke is 3n x 3n.
static bool element_stiffness(int kind, const double* X, const double* ue, const Quad& q, const Material& mat,
                              double* Ke) {
  const int n = element_nodes(kind);
  const int dim = 3 * n;
  for (int i = 0; i < dim * dim; ++i) Ke[i] = 0.0;
  double Gref[3 * 27], G[3 * 27];
  for (int iq = 0; iq < q.nq; ++iq) {
    const double* xi = q.p + 3 * iq;
    double w = q.w[iq];
    M3 J = element_jacobian(kind, X, xi);
    double Jdet = det3(J);
    M3 Jinv;
    if (!inv3(J, Jinv)) return false;
    M3 JinvT = transpose(Jinv);
    element_grad(kind, xi, Gref);
    for (int k = 0; k < 3; ++k)
      for (int I = 0; I < n; ++I) {
        double s = 0.0;
        for (int m = 0; m < 3; ++m) s += JinvT(k, m) * Gref[m * n + I];
        G[k * n + I] = s;
      }
    // u_grad = G * u^T
    M3 ugrad = zero3();
    for (int k = 0; k < 3; ++k)
      for (int c = 0; c < 3; ++c) {
        double s = 0.0;
        for (int I = 0; I < n; ++I) s += G[k * n + I] * ue[c * n + I];
        ugrad(k, c) = s;
      }
    double sc = std::sqrt(w * std::fabs(Jdet));
    for (int i = 0; i < 3 * n; ++i) G[i] *= sc;
    M3 F = add(transpose(ugrad), eye3());
    if (!material_contract_multiple(mat, Ke, F, G, n)) return false;
  }
  return true;
}

// assemble_generalized_element_mass, assembly.rs:624-671 (solution dim 3).
static void element_mass(int kind, const double* X, const Quad& q, double density, double* Me) {
  const int n = element_nodes(kind);
  const int dim = 3 * n;
  std::vector<double> ms(n * n, 0.0);
  double N[27];
  for (int iq = 0; iq < q.nq; ++iq) {
    const double* xi = q.p + 3 * iq;
    double w = q.w[iq];
    double Jdet = det3(element_jacobian(kind, X, xi));
    element_basis(kind, xi, N);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) ms[i * n + j] += density * std::fabs(Jdet) * w * N[i] * N[j];
  }
  for (int i = 0; i < dim * dim; ++i) Me[i] = 0.0;
  for (int c = 0; c < 3; ++c)
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) Me[(3 * i + c) * dim + 3 * j + c] = ms[i * n + j];
}

// ---------------------------------------------------------------------------
// Sparsity pattern — CsrParAssembler::assemble_pattern, assembly.rs:177-249
// ---------------------------------------------------------------------------
struct Pattern {
  i64 nrows = 0;
  std::vector<i64> row_offsets;
  std::vector<i64> col_indices;
};

static Pattern assemble_pattern(const std::vector<std::vector<i64>>& elems, int sdim, i64 num_nodes) {
  std::vector<std::pair<i64, i64>> coords;
  size_t total = 0;
  for (auto& e : elems) total += (size_t)(sdim * e.size()) * (sdim * e.size());
  coords.reserve(total);
  for (auto& e : elems)
    for (i64 ni : e)
      for (i64 nj : e)
        for (int i = 0; i < sdim; ++i)
          for (int j = 0; j < sdim; ++j) coords.emplace_back(sdim * ni + i, sdim * nj + j);
  std::sort(coords.begin(), coords.end());
  Pattern p;
  p.nrows = sdim * num_nodes;
  p.row_offsets.push_back(0);
  i64 current_row = 0;
  bool has_prev = false;
  i64 prev_col = 0;
  for (auto& c : coords) {
    if (c.first >= p.nrows) throw std::runtime_error("Coordinates must be in bounds");
    while (c.first > current_row) {
      p.row_offsets.push_back((i64)p.col_indices.size());
      current_row += 1;
      has_prev = false;
    }
    if (!has_prev || c.second != prev_col) {
      p.col_indices.push_back(c.second);
      prev_col = c.second;
      has_prev = true;
    }
  }
  for (i64 r = current_row; r < p.nrows; ++r) p.row_offsets.push_back((i64)p.col_indices.size());
  return p;
}

// ---------------------------------------------------------------------------
// Greedy coloring — paradis/src/coloring.rs:48-72 (first fit over existing
// colors in creation order, disjointness on the node sets).
// ---------------------------------------------------------------------------
static std::vector<std::vector<i64>> greedy_coloring(const std::vector<std::vector<i64>>& subsets) {
  std::vector<std::vector<i64>> labels;
  std::vector<std::set<i64>> indices;
  std::set<i64> ws;
  for (size_t label = 0; label < subsets.size(); ++label) {
    ws.clear();
    for (i64 idx : subsets[label]) ws.insert(idx);
    bool placed = false;
    for (size_t c = 0; c < labels.size() && !placed; ++c) {
      bool disjoint = true;
      for (i64 idx : ws)
        if (indices[c].count(idx)) { disjoint = false; break; }
      if (disjoint) {
        labels[c].push_back((i64)label);
        for (i64 idx : ws) indices[c].insert(idx);
        placed = true;
      }
    }
    if (!placed) {
      labels.push_back({(i64)label});
      indices.emplace_back(ws.begin(), ws.end());
    }
  }
  return labels;
}

// ---------------------------------------------------------------------------
// CSR helpers — fenris/src/sparse.rs
// ---------------------------------------------------------------------------
struct Csr {
  const Pattern* pat = nullptr;
  std::vector<double> v;
};

// CsrRow::get (binary search), sparse.rs:457-470.
static bool csr_get(const Pattern& p, const double* v, i64 row, i64 col, double& out) {
  const i64* b = p.col_indices.data() + p.row_offsets[row];
  const i64* e = p.col_indices.data() + p.row_offsets[row + 1];
  const i64* it = std::lower_bound(b, e, col);
  if (it == e || *it != col) return false;
  out = v[p.row_offsets[row] + (it - p.col_indices.data() - p.row_offsets[row])];
  return true;
}

// spmv_csr (y = beta*y + alpha*A x), sparse.rs:1164-1199; row-parallel.
static void spmv(double beta, double* y, double alpha, const Pattern& p, const double* v, const double* x) {
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < p.nrows; ++i) {
    double s = 0.0;
    for (i64 k = p.row_offsets[i]; k < p.row_offsets[i + 1]; ++k) s += v[k] * x[p.col_indices[k]];
    y[i] = beta * y[i];
    y[i] += alpha * s;
  }
}

// add_element_row_to_csr_row, assembly.rs:1042-1075 — forward linear search.
static void add_element_row(const Pattern& p, double* v, i64 row, const i64* nodes, const int* perm, int n, int sdim,
                            const double* local_row) {
  i64 k = p.row_offsets[row], kend = p.row_offsets[row + 1];
  for (int pi = 0; pi < n; ++pi) {
    int ln = perm[pi];
    i64 gn = nodes[ln];
    for (int i = 0; i < sdim; ++i) {
      i64 gcol = sdim * gn + i;
      while (k < kend && p.col_indices[k] != gcol) ++k;
      if (k == kend) throw std::runtime_error("Could not find column index associated with node in CSR row");
      v[k] += local_row[sdim * ln + i];
      ++k;
    }
  }
}

// ---------------------------------------------------------------------------
// Model: element blocks with colors — fenris/src/model.rs:32-117,
// fenris/src/embedding/mod.rs:39-59,243-283.
// ---------------------------------------------------------------------------
struct QuadTable {
  // Either uniform (offsets empty: every element uses rule [0, nq_uniform)) or
  // per element (offsets has E+1 entries into w / p).
  std::vector<i64> offsets;
  std::vector<double> w, p;
  Quad rule(i64 e) const {
    if (offsets.empty()) return {w.data(), p.data(), (int)w.size()};
    i64 b = offsets[e], en = offsets[e + 1];
    return {w.data() + b, p.data() + 3 * b, (int)(en - b)};
  }
};

struct Block {
  int kind;
  std::vector<std::vector<i64>> conn;
  QuadTable quad;
  std::vector<std::vector<i64>> colors;
};

struct Model {
  std::vector<double> X;  // N x 3
  i64 num_nodes = 0;
  std::vector<Block> blocks;
  Pattern pattern;  // shared pattern of mass / stiffness / Jacobian
};

static void gather_element(const Model& m, const Block& b, i64 e, const double* u, double* Xe, double* ue) {
  const auto& c = b.conn[e];
  const int n = (int)c.size();
  for (int I = 0; I < n; ++I)
    for (int k = 0; k < 3; ++k) {
      Xe[3 * I + k] = m.X[3 * c[I] + k];
      if (u) ue[k * n + I] = u[3 * c[I] + k];
    }
}

// assemble_generalized_elliptic_term_into_par (assembly.rs:915-966) over each
// block in order (embedding/mod.rs:516-554).  Adds into f.
static bool assemble_forces(const Model& m, const Material& mat, const double* u, double* f) {
  bool ok = true;
  for (const Block& b : m.blocks) {
    const int n = element_nodes(b.kind);
    for (const auto& color : b.colors) {
#pragma omp parallel for schedule(dynamic, 16)
      for (i64 ci = 0; ci < (i64)color.size(); ++ci) {
        i64 e = color[ci];
        double Xe[27 * 3], ue[3 * 27], fe[3 * 27];
        gather_element(m, b, e, u, Xe, ue);
        if (!element_force(b.kind, Xe, ue, b.quad.rule(e), mat, fe)) {
#pragma omp atomic write
          ok = false;
          continue;
        }
        const auto& c = b.conn[e];
        for (int I = 0; I < n; ++I)
          for (int i = 0; i < 3; ++i) f[3 * c[I] + i] += fe[i * n + I];
      }
      if (!ok) return false;
    }
  }
  return ok;
}

// CsrParAssembler::assemble_into_csr with the generalized stiffness element
// assembler (assembly.rs:252-314,362-401).  Adds into v (pattern m.pattern).
static bool assemble_stiffness(const Model& m, const Material& mat, const double* u, double* v) {
  bool ok = true;
  for (const Block& b : m.blocks) {
    const int n = element_nodes(b.kind);
    for (const auto& color : b.colors) {
#pragma omp parallel for schedule(dynamic, 4)
      for (i64 ci = 0; ci < (i64)color.size(); ++ci) {
        i64 e = color[ci];
        double Xe[27 * 3], ue[3 * 27];
        std::vector<double> Ke(9 * n * n);
        gather_element(m, b, e, u, Xe, ue);
        if (!element_stiffness(b.kind, Xe, ue, b.quad.rule(e), mat, Ke.data())) {
#pragma omp atomic write
          ok = false;
          continue;
        }
        const auto& c = b.conn[e];
        int perm[27];
        std::iota(perm, perm + n, 0);
        std::sort(perm, perm + n, [&](int a, int bb) { return c[a] < c[bb]; });
        for (int I = 0; I < n; ++I)
          for (int i = 0; i < 3; ++i)
            add_element_row(m.pattern, v, 3 * c[I] + i, c.data(), perm, n, 3, Ke.data() + (3 * I + i) * 3 * n);
      }
      if (!ok) return false;
    }
  }
  return ok;
}

// Mass matrix values on the model pattern (assemble_mass(density).to_csr(Add),
// fe_model.rs:489-515).  Element order, sequential.
static void assemble_mass(const Model& m, double density, double* v) {
  for (const Block& b : m.blocks) {
    const int n = element_nodes(b.kind);
    std::vector<double> Me(9 * n * n);
    for (i64 e = 0; e < (i64)b.conn.size(); ++e) {
      double Xe[27 * 3];
      gather_element(m, b, e, nullptr, Xe, nullptr);
      element_mass(b.kind, Xe, b.quad.rule(e), density, Me.data());
      const auto& c = b.conn[e];
      int perm[27];
      std::iota(perm, perm + n, 0);
      std::sort(perm, perm + n, [&](int a, int bb) { return c[a] < c[bb]; });
      for (int I = 0; I < n; ++I)
        for (int i = 0; i < 3; ++i)
          add_element_row(m.pattern, v, 3 * c[I] + i, c.data(), perm, n, 3, Me.data() + (3 * I + i) * 3 * n);
    }
  }
}

// apply_homogeneous_dirichlet_bc_csr, assembly.rs:799-869 (solution dim d).
static void dirichlet_csr(const Pattern& p, double* v, const i64* nodes, i64 nn, int d) {
  double sc = 1.0;
  for (i64 i = 0; i < p.nrows; ++i) {
    double x;
    if (!csr_get(p, v, i, i, x)) x = 0.0;
    if (x != 0.0) { sc = std::fabs(x); break; }
  }
  std::vector<char> member(p.nrows, 0), visit(p.nrows, 0);
  for (i64 a = 0; a < nn; ++a)
    for (int i = 0; i < d; ++i) {
      i64 r = d * nodes[a] + i;
      member[r] = 1;
      for (i64 k = p.row_offsets[r]; k < p.row_offsets[r + 1]; ++k) {
        i64 c = p.col_indices[k];
        if (c == r) v[k] = sc;
        else { v[k] = 0.0; visit[c] = 1; }
      }
    }
  for (i64 r = 0; r < p.nrows; ++r)
    if (visit[r] && !member[r])
      for (i64 k = p.row_offsets[r]; k < p.row_offsets[r + 1]; ++k)
        if (member[p.col_indices[k]]) v[k] = 0.0;
}

// ---------------------------------------------------------------------------
// Symmetric eigen-decomposition (cyclic Jacobi) and the Schwarz block inverse.
// The reference calls LAPACK dsyev through nalgebra-lapack/MKL
// (schwarz_precond.rs:329-342); eigenpairs are not unique, so parity is taken
// on the recomposed block, which this solver computes to ~1e-15 relative.
// ---------------------------------------------------------------------------
static void jacobi_eigen(int n, std::vector<double>& A /* n x n, destroyed */, std::vector<double>& V,
                         std::vector<double>& lam) {
  V.assign(n * n, 0.0);
  for (int i = 0; i < n; ++i) V[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double x = A[i * n + j] * A[i * n + j];
        tot += x;
        if (i != j) off += x;
      }
    if (off <= 1e-32 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = A[p * n + q];
        if (apq == 0.0) continue;
        double app = A[p * n + p], aqq = A[q * n + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * vkq;
          V[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  lam.resize(n);
  for (int i = 0; i < n; ++i) lam[i] = A[i * n + i];
}

// invert_element_block, schwarz_precond.rs:329-342.
static void invert_block(int n, std::vector<double>& A, std::vector<double>& out) {
  std::vector<double> V, lam;
  jacobi_eigen(n, A, V, lam);
  double amax = 0.0;
  for (double l : lam) amax = std::max(amax, std::fabs(l));
  double lower = 1e-12 * amax;
  for (double& l : lam) l = (std::fabs(l) >= lower) ? 1.0 / std::fabs(l) : 1.0 / lower;
  out.assign(n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < n; ++k) s += V[i * n + k] * lam[k] * V[j * n + k];
      out[i * n + j] = s;
    }
}

// DefaultSemidefiniteProjection (fenris/src/assembly.rs:549-564): symmetric
// eigen-decomposition, negative eigenvalues set to zero, recomposed.
static void psd_project(int n, double* Ke) {
  std::vector<double> A(Ke, Ke + n * n), V, lam;
  jacobi_eigen(n, A, V, lam);
  for (double& l : lam) l = std::max(0.0, l);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int k = 0; k < n; ++k) s += V[i * n + k] * lam[k] * V[j * n + k];
      Ke[i * n + j] = s;
    }
}

// assemble_transformed_stiffness_into_par with DefaultSemidefiniteProjection
// (system_assembly.rs:107-142 with projected = true): every element matrix is
// projected before the colored scatter.  Adds into v.
static bool assemble_stiffness_projected(const Model& m, const Material& mat, const double* u, double* v) {
  bool ok = true;
  for (const Block& b : m.blocks) {
    const int n = element_nodes(b.kind);
    for (const auto& color : b.colors) {
#pragma omp parallel for schedule(dynamic, 4)
      for (i64 ci = 0; ci < (i64)color.size(); ++ci) {
        i64 e = color[ci];
        double Xe[27 * 3], ue[3 * 27];
        std::vector<double> Ke(9 * n * n);
        gather_element(m, b, e, u, Xe, ue);
        if (!element_stiffness(b.kind, Xe, ue, b.quad.rule(e), mat, Ke.data())) {
#pragma omp atomic write
          ok = false;
          continue;
        }
        psd_project(3 * n, Ke.data());
        const auto& c = b.conn[e];
        int perm[27];
        std::iota(perm, perm + n, 0);
        std::sort(perm, perm + n, [&](int a, int bb) { return c[a] < c[bb]; });
        for (int I = 0; I < n; ++I)
          for (int i = 0; i < 3; ++i)
            add_element_row(m.pattern, v, 3 * c[I] + i, c.data(), perm, n, 3, Ke.data() + (3 * I + i) * 3 * n);
      }
      if (!ok) return false;
    }
  }
  return ok;
}

struct Schwarz {
  std::vector<std::vector<i64>> subdomains;  // node lists
  std::vector<i64> untreated;                // sorted node indices
  std::vector<std::vector<i64>> colors;
  Pattern pattern;
  std::vector<double> v;
};

// build_preconditioner_pattern, schwarz_precond.rs:134-169 (COO -> CSR).
static Pattern schwarz_pattern(i64 num_nodes, const std::vector<std::vector<i64>>& subs, const std::vector<i64>& untreated,
                               int sdim) {
  std::vector<std::pair<i64, i64>> coords;
  for (auto& s : subs)
    for (i64 a : s)
      for (i64 b : s)
        for (int i = 0; i < sdim; ++i)
          for (int j = 0; j < sdim; ++j) coords.emplace_back(sdim * a + i, sdim * b + j);
  for (i64 a : untreated)
    for (int i = 0; i < sdim; ++i) coords.emplace_back(sdim * a + i, sdim * a + i);
  std::sort(coords.begin(), coords.end());
  coords.erase(std::unique(coords.begin(), coords.end()), coords.end());
  Pattern p;
  p.nrows = sdim * num_nodes;
  p.row_offsets.assign(p.nrows + 1, 0);
  for (auto& c : coords) p.row_offsets[c.first + 1]++;
  for (i64 r = 0; r < p.nrows; ++r) p.row_offsets[r + 1] += p.row_offsets[r];
  p.col_indices.reserve(coords.size());
  for (auto& c : coords) p.col_indices.push_back(c.second);
  return p;
}

// build_schwarz_preconditioner_into, schwarz_precond.rs:171-216,250-327.
static bool schwarz_update(Schwarz& S, const Pattern& jp, const double* jv) {
  std::fill(S.v.begin(), S.v.end(), 0.0);
  bool ok = true;
  for (const auto& color : S.colors) {
#pragma omp parallel for schedule(dynamic, 1)
    for (i64 ci = 0; ci < (i64)color.size(); ++ci) {
      const auto& nodes = S.subdomains[color[ci]];
      const int n = (int)nodes.size();
      const int dim = 3 * n;
      std::vector<double> blk(dim * dim), inv;
      for (int I = 0; I < n; ++I)
        for (int i = 0; i < 3; ++i)
          for (int J = 0; J < n; ++J)
            for (int j = 0; j < 3; ++j) {
              double x;
              if (!csr_get(jp, jv, 3 * nodes[I] + i, 3 * nodes[J] + j, x)) {
#pragma omp atomic write
                ok = false;
                x = 0.0;
              }
              blk[(3 * I + i) * dim + 3 * J + j] = x;
            }
      invert_block(dim, blk, inv);
      int perm[27];
      std::iota(perm, perm + n, 0);
      std::sort(perm, perm + n, [&](int a, int b) { return nodes[a] < nodes[b]; });
      for (int I = 0; I < n; ++I)
        for (int i = 0; i < 3; ++i)
          add_element_row(S.pattern, S.v.data(), 3 * nodes[I] + i, nodes.data(), perm, n, 3, inv.data() + (3 * I + i) * dim);
    }
  }
  if (!ok) return false;
  for (i64 a : S.untreated)
    for (int i = 0; i < 3; ++i) {
      i64 r = 3 * a + i;
      double x;
      if (!csr_get(jp, jv, r, r, x)) x = 0.0;
      if (x == 0.0) return false;
      S.v[S.pattern.row_offsets[r]] = 1.0 / x;
    }
  return true;
}

// ---------------------------------------------------------------------------
// Preconditioned CG — fenris/src/cg.rs:376-482 with RelativeResidualCriterion.
// ---------------------------------------------------------------------------
enum CgStatus { CG_OK = 0, CG_INDEFINITE_OPERATOR = 1, CG_INDEFINITE_PRECOND = 2, CG_MAX_ITER = 3, CG_PRECOND_ERROR = 4 };

using LinOp = std::function<bool(double* y, const double* x)>;

static double dot(const double* a, const double* b, i64 n) {
  double s = 0.0;
  for (i64 i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

static int cg_solve(i64 n, const LinOp& A, const LinOp* P, const double* b, double* x, double tol, i64 max_iter,
                    i64* iters) {
  std::vector<double> r(n), z(n), p(n), Ap(n);
  *iters = 0;
  A(r.data(), x);
  for (i64 i = 0; i < n; ++i) r[i] = b[i] - r[i];
  if (P) { if (!(*P)(z.data(), r.data())) return CG_PRECOND_ERROR; }
  else z = r;
  p = z;
  double zTr = dot(z.data(), r.data(), n);
  double bnorm = std::sqrt(dot(b, b, n));
  if (bnorm == 0.0) { std::fill(x, x + n, 0.0); return CG_OK; }
  for (;;) {
    double rn = std::sqrt(dot(r.data(), r.data(), n));
    if (rn <= tol * bnorm) break;
    if (max_iter >= 0 && *iters >= max_iter) return CG_MAX_ITER;
    A(Ap.data(), p.data());
    double pAp = dot(p.data(), Ap.data(), n);
    if (pAp <= 0.0) return CG_INDEFINITE_OPERATOR;
    if (zTr <= 0.0) return CG_INDEFINITE_PRECOND;
    double alpha = zTr / pAp;
    for (i64 i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
    for (i64 i = 0; i < n; ++i) r[i] = r[i] - alpha * Ap[i];
    *iters += 1;
    if (P) { if (!(*P)(z.data(), r.data())) return CG_PRECOND_ERROR; }
    else z = r;
    double zTr_next = dot(z.data(), r.data(), n);
    double beta = zTr_next / zTr;
    for (i64 i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    zTr = zTr_next;
  }
  return CG_OK;
}

// ---------------------------------------------------------------------------
// Newton-CG backward Euler — simulation_toolbox/src/fem/newton_cg.rs:146-802,
// hamilton2/src/integrators/euler.rs:76-199, hamilton2/src/newton.rs:76-248,
// simulation_toolbox/src/fem/system_assembly.rs:78-235.
// ---------------------------------------------------------------------------
enum PrecondKind { PRECOND_DIAGONAL = 0, PRECOND_SCHWARZ = 1 };

enum StepStatus {
  STEP_OK = 0,
  STEP_NEWTON_MAX_ITER = 10,
  STEP_LINE_SEARCH_FAILED = 11,
  STEP_JACOBIAN_ERROR = 12,
  STEP_ASSEMBLY_ERROR = 13,
  STEP_SUBSTEP_FAILED = 14,
};

struct Scene {
  Model model;
  Material mat;
  double density = 1000.0;
  double gravity = -9.81;  // scalar gravity on the last component
  bool gravity_enabled = true;
  std::vector<i64> bc_nodes;
  std::vector<char> bc_dof;
  std::vector<double> mass;  // on model.pattern, Dirichlet applied
  double representative_force = 0.0;
  std::vector<double> g_force;
  int precond = PRECOND_DIAGONAL;
  Schwarz schwarz;
  double cg_tol = 1e-5;
  i64 cg_max_iter = 500;
  i64 newton_max_iter = 100;
  double newton_tol_factor = 1e-5;
  // damping D = gamma M + alpha K_proj(u), recomputed at the start of every
  // (sub)step (compute_damping_matrix_into, system_assembly.rs:145-193)
  bool has_mass_damping = false, has_stiffness_damping = false;
  double mass_damping = 0.0, stiffness_damping = 0.0;
  bool has_damping = false;
  std::vector<double> damping;
  // statistics of the last step
  std::vector<i64> cg_iters;
  std::vector<int> cg_status;
  i64 newton_iters = 0;
  i64 ls_backtracks = 0;  // line-search reductions of alpha below 1 in the last step (all attempts)
  i64 num_substeps = 1;
  double last_residual = 0.0;
};

static void apply_bc_unknowns(const Scene& s, double* u, double* v) {
  for (i64 a : s.bc_nodes)
    for (int i = 0; i < 3; ++i) { u[3 * a + i] = 0.0; v[3 * a + i] = 0.0; }
}

// compute_representative_force, fe_model.rs:423-431.
static double representative_force(const Pattern& p, const double* mass) {
  std::vector<double> a(p.nrows, std::sqrt((10.0 * 10.0) / 3.0)), y(p.nrows, 0.0);
  spmv(0.0, y.data(), 1.0, p, mass, a.data());
  return std::sqrt(dot(y.data(), y.data(), p.nrows));
}

static void scene_setup(Scene& s) {
  const Pattern& p = s.model.pattern;
  s.mass.assign(p.col_indices.size(), 0.0);
  assemble_mass(s.model, s.density, s.mass.data());
  dirichlet_csr(p, s.mass.data(), s.bc_nodes.data(), (i64)s.bc_nodes.size(), 3);
  s.representative_force = representative_force(p, s.mass.data());
  s.bc_dof.assign(p.nrows, 0);
  for (i64 a : s.bc_nodes) for (int i = 0; i < 3; ++i) s.bc_dof[3 * a + i] = 1;
  // gravity force M g (compute_gravity_density, system_assembly.rs:30-75)
  std::vector<double> gd(p.nrows, 0.0);
  if (s.gravity_enabled)
    for (i64 i = 0; i < p.nrows; ++i) if (i % 3 == 2) gd[i] = s.gravity;
  s.g_force.assign(p.nrows, 0.0);
  spmv(0.0, s.g_force.data(), 1.0, p, s.mass.data(), gd.data());
  if (s.precond == PRECOND_SCHWARZ) {
    s.schwarz.pattern = schwarz_pattern(s.model.num_nodes, s.schwarz.subdomains, s.schwarz.untreated, 3);
    s.schwarz.v.assign(s.schwarz.pattern.col_indices.size(), 0.0);
    s.schwarz.colors = greedy_coloring(s.schwarz.subdomains);
  }
}

// NewtonCgDynamicSystem::eval_f (newton_cg.rs:441-478):
//   f = M g + f_int(u) - D v, Dirichlet rows zeroed.
static bool eval_f(Scene& s, const double* u_in, const double* v_in, double* f) {
  const i64 n = s.model.pattern.nrows;
  std::vector<double> u(u_in, u_in + n), v(v_in, v_in + n);
  std::copy(s.g_force.begin(), s.g_force.end(), f);
  apply_bc_unknowns(s, u.data(), v.data());
  if (!assemble_forces(s.model, s.mat, u.data(), f)) return false;
  if (s.has_damping) spmv(1.0, f, -1.0, s.model.pattern, s.damping.data(), v.data());
  for (i64 i = 0; i < n; ++i) if (s.bc_dof[i]) f[i] = 0.0;
  return true;
}

// compute_damping_matrix_into (system_assembly.rs:145-193): K projected at u
// (no boundary conditions applied to u or D), then D = 0 + alpha K + gamma M
// in the order of compute_jacobian_combination_into (stiffness, then mass).
static bool compute_damping(Scene& s, const double* u) {
  s.has_damping = s.has_mass_damping || s.has_stiffness_damping;
  if (!s.has_damping) return true;
  const Pattern& p = s.model.pattern;
  std::vector<double> K(p.col_indices.size(), 0.0);
  if (s.has_stiffness_damping && !assemble_stiffness_projected(s.model, s.mat, u, K.data())) return false;
  s.damping.assign(p.col_indices.size(), 0.0);
  if (s.has_stiffness_damping)
    for (size_t k = 0; k < K.size(); ++k) s.damping[k] += s.stiffness_damping * K[k];
  if (s.has_mass_damping)
    for (size_t k = 0; k < K.size(); ++k) s.damping[k] += s.mass_damping * s.mass[k];
  return true;
}

// BackwardEulerImplicitFunction::eval_into (euler.rs:97-114):
//   F(w) = M w - dt f(t+dt, u_p + dt w, v_n + w)
static bool eval_F(Scene& s, const std::vector<double>& up, const std::vector<double>& vn, double dt, const double* w,
                   double* F) {
  const i64 n = s.model.pattern.nrows;
  std::vector<double> u(n), v(n);
  for (i64 i = 0; i < n; ++i) { u[i] = up[i] + w[i] * dt; v[i] = vn[i] + w[i]; }
  if (!eval_f(s, u.data(), v.data(), F)) return false;
  for (i64 i = 0; i < n; ++i) F[i] *= dt * -1.0;
  spmv(1.0, F, 1.0, s.model.pattern, s.mass.data(), w);
  return true;
}

// solve_jacobian_combination (newton_cg.rs:680-802) for J = M + dt D + dt^2 K.
static int solve_jacobian(Scene& s, const std::vector<double>& up, const std::vector<double>& vn, double dt,
                          const double* w, const double* rhs, double* sol) {
  const Pattern& p = s.model.pattern;
  const i64 n = p.nrows;
  std::vector<double> u(n), v(n);
  for (i64 i = 0; i < n; ++i) { u[i] = up[i] + w[i] * dt; v[i] = vn[i] + w[i]; }
  apply_bc_unknowns(s, u.data(), v.data());
  std::vector<double> K(p.col_indices.size(), 0.0);
  if (!assemble_stiffness(s.model, s.mat, u.data(), K.data())) return STEP_ASSEMBLY_ERROR;
  // J = gamma M - beta D - alpha K with alpha = -dt^2, beta = -dt, gamma = 1
  // (euler.rs:136), accumulated in the order stiffness, damping, mass
  std::vector<double> J(p.col_indices.size(), 0.0);
  double ck = -(-dt * dt);
  for (size_t k = 0; k < J.size(); ++k) J[k] += ck * K[k];
  if (s.has_damping) {
    double cd = -(-dt);
    for (size_t k = 0; k < J.size(); ++k) J[k] += cd * s.damping[k];
  }
  for (size_t k = 0; k < J.size(); ++k) J[k] += 1.0 * s.mass[k];
  dirichlet_csr(p, J.data(), s.bc_nodes.data(), (i64)s.bc_nodes.size(), 3);
  LinOp A = [&](double* y, const double* x) { spmv(0.0, y, 1.0, p, J.data(), x); return true; };
  LinOp P;
  std::vector<double> diag;
  if (s.precond == PRECOND_SCHWARZ) {
    if (!schwarz_update(s.schwarz, p, J.data())) return STEP_JACOBIAN_ERROR;
    P = [&](double* y, const double* x) {
      spmv(0.0, y, 1.0, s.schwarz.pattern, s.schwarz.v.data(), x);
      return true;
    };
  } else {
    diag.resize(n);
    for (i64 i = 0; i < n; ++i) {
      double x;
      if (!csr_get(p, J.data(), i, i, x)) x = 0.0;
      if (x == 0.0) return STEP_JACOBIAN_ERROR;
      diag[i] = 1.0 / x;
    }
    P = [&](double* y, const double* x) {
      for (i64 i = 0; i < n; ++i) y[i] = diag[i] * x[i];
      return true;
    };
  }
  std::fill(sol, sol + n, 0.0);
  i64 it = 0;
  int st = cg_solve(n, A, &P, rhs, sol, s.cg_tol, s.cg_max_iter, &it);
  s.cg_iters.push_back(it);
  s.cg_status.push_back(st);
  if (st == CG_OK || st == CG_MAX_ITER || st == CG_INDEFINITE_OPERATOR) return STEP_OK;
  return STEP_JACOBIAN_ERROR;
}

// backward_euler_step (euler.rs:155-199) + newton_line_search with
// BacktrackingLineSearch (newton.rs:76-131,171-248).
static int backward_euler_step(Scene& s, double* u, double* v, double t0, double dt) {
  (void)t0;
  const i64 n = s.model.pattern.nrows;
  std::vector<double> vn(v, v + n), up(n);
  for (i64 i = 0; i < n; ++i) up[i] = u[i] + v[i] * dt;
  std::vector<double> w(n, 0.0), F(n), mdx(n);
  double tol = dt * (s.newton_tol_factor * s.representative_force);
  if (!eval_F(s, up, vn, dt, w.data(), F.data())) return STEP_ASSEMBLY_ERROR;
  i64 iter = 0;
  while (std::sqrt(dot(F.data(), F.data(), n)) > tol) {
    if (iter == s.newton_max_iter) return STEP_NEWTON_MAX_ITER;
    int st = solve_jacobian(s, up, vn, dt, w.data(), F.data(), mdx.data());
    if (st != STEP_OK) return st;
    for (i64 i = 0; i < n; ++i) mdx[i] *= -1.0;
    // line search
    const double c = 1e-4, alpha_min = 1e-6;
    double g0 = 0.5 * dot(F.data(), F.data(), n);
    double alpha_prev = 0.0, alpha = 1.0;
    int k = 1;
    const double initial[4] = {0.0, 1.0, 0.75, 0.5};
    double tail = 0.25;
    for (;;) {
      double da = alpha - alpha_prev;
      for (i64 i = 0; i < n; ++i) w[i] = da * mdx[i] + 1.0 * w[i];
      if (!eval_F(s, up, vn, dt, w.data(), F.data())) return STEP_ASSEMBLY_ERROR;
      double g = 0.5 * dot(F.data(), F.data(), n);
      if (g <= (1.0 - c * alpha) * g0) break;
      if (alpha < alpha_min) return STEP_LINE_SEARCH_FAILED;
      alpha_prev = alpha;
      ++s.ls_backtracks;
      ++k;
      if (k < 4) alpha = initial[k];
      else { alpha = tail; tail *= 0.25; }
    }
    ++iter;
  }
  s.newton_iters = iter;
  s.last_residual = std::sqrt(dot(F.data(), F.data(), n));
  for (i64 i = 0; i < n; ++i) v[i] += w[i];
  for (i64 i = 0; i < n; ++i) u[i] += v[i] * dt;
  return STEP_OK;
}

// integrate_model + integrate_model_with_substeps (newton_cg.rs:146-295).
static int integrate(Scene& s, double* u, double* v, double t, double dt) {
  const i64 n = s.model.pattern.nrows;
  s.cg_iters.clear();
  s.cg_status.clear();
  s.ls_backtracks = 0;
  apply_bc_unknowns(s, u, v);
  const i64 max_substeps = 1000, factor = 5;
  std::vector<double> us(u, u + n), vs(v, v + n);
  i64 num = 1;
  double sdt = dt / (double)num;
  for (;;) {
    bool failed = false;
    for (i64 k = 0; k < num; ++k) {
      double st = t + (double)k * sdt;
      // integrate_model: damping from the substep's initial state, then the step
      int r = compute_damping(s, us.data()) ? backward_euler_step(s, us.data(), vs.data(), st, sdt)
                                            : STEP_ASSEMBLY_ERROR;
      if (r == STEP_OK) apply_bc_unknowns(s, us.data(), vs.data());
      else { failed = true; break; }
    }
    if (!failed) break;
    num *= factor;
    if (num >= max_substeps) return STEP_SUBSTEP_FAILED;
    sdt = dt / (double)num;
    std::copy(u, u + n, us.begin());
    std::copy(v, v + n, vs.begin());
  }
  s.num_substeps = num;
  std::copy(us.begin(), us.end(), u);
  std::copy(vs.begin(), vs.end(), v);
  return STEP_OK;
}

// ---------------------------------------------------------------------------
// Mesh pipeline (input construction) — literal restatement of
// fenris/src/geometry/procedural.rs:191-250, polymesh.rs:402-500 (Max 2000
// triangulation) + dedup_faces (249-287), mesh_convert.rs:577-727 (PolyMesh
// from mesh, Tet4 from PolyMesh), mesh_convert.rs:41-75,163-244,296-406
// (FromTemp refinement to Tet10 / Hex27), mesh.rs:321-366 (keep_cells).
// ---------------------------------------------------------------------------
struct Mesh {
  std::vector<double> X;           // N x 3
  std::vector<std::vector<i64>> C;  // cells
};

static Mesh rect_hex_mesh(double unit, i64 ux, i64 uy, i64 uz, i64 cpu) {
  Mesh m;
  if (cpu == 0 || ux == 0 || uy == 0) return m;
  double h = unit / (double)cpu;
  i64 nx = ux * cpu, ny = uy * cpu, nz = uz * cpu;
  i64 vx = nx + 1, vy = ny + 1, vz = nz + 1;
  auto idx = [&](i64 i, i64 j, i64 k) { return vx * vy * k + vx * j + i; };
  for (i64 k = 0; k < vz; ++k)
    for (i64 j = 0; j < vy; ++j)
      for (i64 i = 0; i < vx; ++i) {
        m.X.push_back((double)i * h);
        m.X.push_back((double)j * h);
        m.X.push_back((double)k * h);
      }
  for (i64 k = 0; k < nz; ++k)
    for (i64 j = 0; j < ny; ++j)
      for (i64 i = 0; i < nx; ++i)
        m.C.push_back({idx(i, j, k), idx(i + 1, j, k), idx(i + 1, j + 1, k), idx(i, j + 1, k), idx(i, j, k + 1),
                       idx(i + 1, j, k + 1), idx(i + 1, j + 1, k + 1), idx(i, j + 1, k + 1)});
  return m;
}

struct PolyMesh {
  std::vector<double> X;
  std::vector<std::vector<i64>> faces;
  std::vector<std::vector<i64>> cells;
};

static PolyMesh polymesh_from_hex(const Mesh& m) {
  static const int HF[6][4] = {{3, 2, 1, 0}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {4, 7, 3, 0}, {5, 6, 7, 4}};
  PolyMesh pm;
  pm.X = m.X;
  std::map<std::vector<i64>, i64> cmap;
  for (auto& c : m.C) {
    std::vector<i64> cell;
    for (int f = 0; f < 6; ++f) {
      std::vector<i64> face = {c[HF[f][0]], c[HF[f][1]], c[HF[f][2]], c[HF[f][3]]};
      std::vector<i64> key = face;
      std::sort(key.begin(), key.end());
      auto it = cmap.find(key);
      i64 fi;
      if (it != cmap.end()) fi = it->second;
      else { fi = (i64)pm.faces.size(); pm.faces.push_back(face); cmap.emplace(key, fi); }
      cell.push_back(fi);
    }
    pm.cells.push_back(cell);
  }
  return pm;
}

static void dedup_faces(PolyMesh& pm) {
  std::map<std::vector<i64>, i64> cmap;
  std::vector<std::vector<i64>> nf;
  std::vector<i64> relabel;
  for (auto& f : pm.faces) {
    std::vector<i64> key = f;
    std::sort(key.begin(), key.end());
    auto it = cmap.find(key);
    if (it != cmap.end()) relabel.push_back(it->second);
    else { i64 ni = (i64)nf.size(); cmap.emplace(key, ni); nf.push_back(f); relabel.push_back(ni); }
  }
  pm.faces = nf;
  for (auto& c : pm.cells) for (auto& fi : c) fi = relabel[fi];
}

static PolyMesh triangulate(const PolyMesh& pm) {
  std::vector<std::vector<i64>> tf;
  std::vector<std::vector<i64>> fmap;
  for (auto& face : pm.faces) {
    if (face.size() < 3) throw std::runtime_error("face with less than 3 vertices");
    size_t mi = 0;
    for (size_t i = 1; i < face.size(); ++i) if (face[i] < face[mi]) mi = i;
    std::vector<i64> arr;
    for (size_t i = 0; i + 2 < face.size(); ++i) {
      arr.push_back((i64)tf.size());
      tf.push_back({face[mi], face[(i + 1 + mi) % face.size()], face[(i + 2 + mi) % face.size()]});
    }
    fmap.push_back(arr);
  }
  std::vector<std::vector<i64>> tets;
  for (auto& cell : pm.cells) {
    if (cell.empty()) continue;
    i64 v = -1;
    for (i64 fi : cell) for (i64 x : pm.faces[fi]) if (v < 0 || x < v) v = x;
    for (i64 fi : cell) {
      const auto& of = pm.faces[fi];
      if (std::find(of.begin(), of.end(), v) != of.end()) continue;
      for (i64 ti : fmap[fi]) {
        i64 a = tf[ti][0], b = tf[ti][1], c = tf[ti][2];
        i64 abv = (i64)tf.size();
        tf.push_back({a, b, v});
        tf.push_back({b, c, v});
        tf.push_back({c, a, v});
        tets.push_back({ti, abv, abv + 1, abv + 2});
      }
    }
  }
  PolyMesh out;
  out.X = pm.X;
  out.faces = tf;
  out.cells = tets;
  dedup_faces(out);
  return out;
}

static Mesh tet4_from_polymesh(const PolyMesh& pm) {
  Mesh m;
  m.X = pm.X;
  for (auto& cell : pm.cells) {
    if (cell.size() != 4) throw std::runtime_error("non-tetrahedral cell");
    i64 base[3] = {pm.faces[cell[0]][0], pm.faces[cell[0]][1], pm.faces[cell[0]][2]};
    i64 apex = -1;
    for (i64 x : pm.faces[cell[1]])
      if (x != base[0] && x != base[1] && x != base[2]) { apex = x; break; }
    if (apex < 0) throw std::runtime_error("degenerate cell");
    const double* a = &pm.X[3 * base[0]];
    const double* b = &pm.X[3 * base[1]];
    const double* c = &pm.X[3 * base[2]];
    const double* p = &pm.X[3 * apex];
    double ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    double ac[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    double nrm[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
    double len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
    double d = (nrm[0] / len) * (p[0] - a[0]) + (nrm[1] / len) * (p[1] - a[1]) + (nrm[2] / len) * (p[2] - a[2]);
    if (d < 0.0) std::swap(base[0], base[1]);
    m.C.push_back({base[0], base[1], base[2], apex});
  }
  return m;
}

// FromTemp::from (mesh_convert.rs:296-406): label refined nodes in first-
// appearance order, keyed by (child index, sorted parents).
static Mesh refine(const Mesh& m, int target) {
  Mesh out;
  std::map<std::vector<i64>, i64> label;
  for (auto& c : m.C) {
    std::vector<std::vector<i64>> parents;
    std::vector<std::array<double, 3>> pos;
    auto P = [&](i64 i) { return std::array<double, 3>{m.X[3 * i], m.X[3 * i + 1], m.X[3 * i + 2]}; };
    for (i64 v : c) { parents.push_back({v}); pos.push_back(P(v)); }
    auto edge = [&](int a, int b) {
      std::vector<i64> par = {c[a], c[b]};
      std::sort(par.begin(), par.end());
      parents.push_back(par);
      auto pa = P(c[a]), pb = P(c[b]);
      pos.push_back({pa[0] * 0.5 + pb[0] * 0.5, pa[1] * 0.5 + pb[1] * 0.5, pa[2] * 0.5 + pb[2] * 0.5});
    };
    if (target == ELEM_TET10) {
      for (auto& e : TET10_EDGES) edge(e[0], e[1]);
    } else {
      static const int HE[12][2] = {{0, 1}, {0, 3}, {0, 4}, {1, 2}, {1, 5}, {2, 3},
                                    {2, 6}, {3, 7}, {4, 5}, {4, 7}, {5, 6}, {6, 7}};
      for (auto& e : HE) edge(e[0], e[1]);
      double Xe[24];
      for (int I = 0; I < 8; ++I) for (int k = 0; k < 3; ++k) Xe[3 * I + k] = m.X[3 * c[I] + k];
      static const int HFN[6][4] = {{0, 1, 2, 3}, {0, 1, 4, 5}, {0, 3, 4, 7}, {1, 2, 5, 6}, {2, 3, 6, 7}, {4, 5, 6, 7}};
      static const double HFX[6][3] = {{0, 0, -1}, {0, -1, 0}, {-1, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
      for (int f = 0; f < 6; ++f) {
        std::vector<i64> par;
        for (int k = 0; k < 4; ++k) par.push_back(c[HFN[f][k]]);
        std::sort(par.begin(), par.end());
        parents.push_back(par);
        std::array<double, 3> x;
        element_map(ELEM_HEX8, Xe, HFX[f], x.data());
        pos.push_back(x);
      }
      std::vector<i64> par(c.begin(), c.end());
      std::sort(par.begin(), par.end());
      parents.push_back(par);
      const double zero[3] = {0, 0, 0};
      std::array<double, 3> x;
      element_map(ELEM_HEX8, Xe, zero, x.data());
      pos.push_back(x);
    }
    std::vector<i64> nc;
    for (size_t k = 0; k < parents.size(); ++k) {
      auto it = label.find(parents[k]);
      if (it != label.end()) nc.push_back(it->second);
      else {
        i64 l = (i64)(out.X.size() / 3);
        label.emplace(parents[k], l);
        for (int d = 0; d < 3; ++d) out.X.push_back(pos[k][d]);
        nc.push_back(l);
      }
    }
    out.C.push_back(nc);
  }
  return out;
}

static Mesh keep_cells(const Mesh& m, const std::vector<i64>& cells) {
  i64 nv = (i64)(m.X.size() / 3);
  std::vector<char> keep(nv, 0);
  for (i64 c : cells) for (i64 v : m.C[c]) keep[v] = 1;
  std::vector<i64> lab(nv, -1);
  Mesh out;
  i64 next = 0;
  for (i64 i = 0; i < nv; ++i)
    if (keep[i]) {
      lab[i] = next++;
      for (int d = 0; d < 3; ++d) out.X.push_back(m.X[3 * i + d]);
    }
  for (i64 c : cells) {
    std::vector<i64> nc;
    for (i64 v : m.C[c]) nc.push_back(lab[v]);
    out.C.push_back(nc);
  }
  return out;
}

}  // namespace oracle

// ============================================================================
// extern "C" surface for the Python test harness (ctypes).
// ============================================================================
using namespace oracle;

namespace {
thread_local std::string g_last_error;
struct MeshResult {
  Mesh mesh;
};
}  // namespace

extern "C" {

const char* oracle_last_error() { return g_last_error.c_str(); }

int oracle_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void oracle_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

void oracle_lame_from_young_poisson(double young, double poisson, double* mu, double* lambda) {
  Lame l = lame_from_young_poisson(young, poisson);
  *mu = l.mu;
  *lambda = l.lambda;
}

// F, P: 3x3 row-major.
int oracle_material_stress(int kind, double mu, double lambda, const double* F, double* P) {
  Material m{kind, {mu, lambda}};
  M3 f, p;
  std::memcpy(f.m, F, sizeof(f.m));
  if (!material_stress(m, f, p)) return 1;
  std::memcpy(P, p.m, sizeof(p.m));
  return 0;
}
double oracle_material_energy(int kind, double mu, double lambda, const double* F) {
  Material m{kind, {mu, lambda}};
  M3 f;
  std::memcpy(f.m, F, sizeof(f.m));
  return material_energy(m, f);
}
int oracle_material_contract(int kind, double mu, double lambda, const double* F, const double* a, const double* b,
                             double* out) {
  Material m{kind, {mu, lambda}};
  M3 f, o;
  std::memcpy(f.m, F, sizeof(f.m));
  if (!material_contract_pair(m, f, a, b, o)) return 1;
  std::memcpy(out, o.m, sizeof(o.m));
  return 0;
}
// a: 3 x n row-major; out (3n x 3n) is ADDED into.
int oracle_material_contract_multiple(int kind, double mu, double lambda, const double* F, const double* a, int n,
                                      double* out) {
  Material m{kind, {mu, lambda}};
  M3 f;
  std::memcpy(f.m, F, sizeof(f.m));
  return material_contract_multiple(m, out, f, a, n) ? 0 : 1;
}
// dp/df of SNH from un-reparametrised Lame parameters; C 9x9 row-major.
int oracle_snh_dp_df(double mu, double lambda, const double* F, double* C) {
  M3 f;
  std::memcpy(f.m, F, sizeof(f.m));
  return snh_dp_df(snh_reparam({mu, lambda}), f, C) ? 0 : 1;
}

void oracle_element_basis(int kind, const double* xi, double* N) { element_basis(kind, xi, N); }
void oracle_element_gradients(int kind, const double* xi, double* g) { element_grad(kind, xi, g); }

int oracle_element_force(int kind, const double* X, const double* ue, const double* qw, const double* qp, int nq,
                         int mat_kind, double mu, double lambda, double* fe) {
  Material m{mat_kind, {mu, lambda}};
  return element_force(kind, X, ue, Quad{qw, qp, nq}, m, fe) ? 0 : 1;
}
int oracle_element_stiffness(int kind, const double* X, const double* ue, const double* qw, const double* qp, int nq,
                             int mat_kind, double mu, double lambda, double* Ke) {
  Material m{mat_kind, {mu, lambda}};
  return element_stiffness(kind, X, ue, Quad{qw, qp, nq}, m, Ke) ? 0 : 1;
}
void oracle_element_mass(int kind, const double* X, const double* qw, const double* qp, int nq, double density,
                         double* Me) {
  element_mass(kind, X, Quad{qw, qp, nq}, density, Me);
}

// Pattern from ragged element node lists (offsets E+1, nodes).
void* oracle_pattern_create(const int64_t* offsets, const int64_t* nodes, int64_t ne, int sdim, int64_t num_nodes) {
  try {
    std::vector<std::vector<i64>> elems(ne);
    for (i64 e = 0; e < ne; ++e) elems[e].assign(nodes + offsets[e], nodes + offsets[e + 1]);
    return new Pattern(assemble_pattern(elems, sdim, num_nodes));
  } catch (std::exception& ex) {
    g_last_error = ex.what();
    return nullptr;
  }
}
int64_t oracle_pattern_nnz(void* p) { return (int64_t)((Pattern*)p)->col_indices.size(); }
int64_t oracle_pattern_nrows(void* p) { return ((Pattern*)p)->nrows; }
void oracle_pattern_copy(void* p, int64_t* row_offsets, int64_t* cols) {
  Pattern* pp = (Pattern*)p;
  std::memcpy(row_offsets, pp->row_offsets.data(), sizeof(i64) * pp->row_offsets.size());
  if (!pp->col_indices.empty()) std::memcpy(cols, pp->col_indices.data(), sizeof(i64) * pp->col_indices.size());
}
void oracle_pattern_destroy(void* p) { delete (Pattern*)p; }

// Coloring of ragged subsets; color_offsets (ncolors+1) and labels (ne).
int64_t oracle_greedy_coloring(const int64_t* offsets, const int64_t* nodes, int64_t ne, int64_t* color_offsets,
                               int64_t* labels) {
  std::vector<std::vector<i64>> subs(ne);
  for (i64 e = 0; e < ne; ++e) subs[e].assign(nodes + offsets[e], nodes + offsets[e + 1]);
  auto colors = greedy_coloring(subs);
  i64 k = 0;
  color_offsets[0] = 0;
  for (size_t c = 0; c < colors.size(); ++c) {
    for (i64 l : colors[c]) labels[k++] = l;
    color_offsets[c + 1] = k;
  }
  return (int64_t)colors.size();
}

// Dirichlet on an explicit CSR (values modified in place).
void oracle_dirichlet_csr(int64_t nrows, const int64_t* row_offsets, const int64_t* cols, double* v,
                          const int64_t* nodes, int64_t nn, int d) {
  Pattern p;
  p.nrows = nrows;
  p.row_offsets.assign(row_offsets, row_offsets + nrows + 1);
  p.col_indices.assign(cols, cols + row_offsets[nrows]);
  dirichlet_csr(p, v, nodes, nn, d);
}

// Dense-operator CG for the reference's CG unit tests.  A, P row-major n x n
// (P may be null = identity).
int oracle_cg_dense(int64_t n, const double* A, const double* P, const double* b, double* x, double tol,
                    int64_t max_iter, int64_t* iters) {
  LinOp op = [&](double* y, const double* xx) {
    for (i64 i = 0; i < n; ++i) { double s = 0; for (i64 j = 0; j < n; ++j) s += A[i * n + j] * xx[j]; y[i] = s; }
    return true;
  };
  LinOp pop = [&](double* y, const double* xx) {
    for (i64 i = 0; i < n; ++i) { double s = 0; for (i64 j = 0; j < n; ++j) s += P[i * n + j] * xx[j]; y[i] = s; }
    return true;
  };
  return cg_solve(n, op, P ? &pop : nullptr, b, x, tol, max_iter, iters);
}

// Block inverse used by the Schwarz preconditioner (n x n row-major).
void oracle_invert_block(int n, const double* A, double* out) {
  std::vector<double> a(A, A + n * n), o;
  invert_block(n, a, o);
  std::memcpy(out, o.data(), sizeof(double) * n * n);
}

// ---- meshes ---------------------------------------------------------------
void* oracle_mesh_hex_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cpu) {
  auto* r = new MeshResult();
  r->mesh = rect_hex_mesh(unit, ux, uy, uz, cpu);
  return r;
}
// Max triangulation -> Tet4 -> Tet10 (or Tet4 if tet10 == 0).
void* oracle_mesh_tets_from_hex(void* hex, int tet10) {
  try {
    auto* h = (MeshResult*)hex;
    PolyMesh pm = polymesh_from_hex(h->mesh);
    PolyMesh tri = triangulate(pm);
    Mesh t4 = tet4_from_polymesh(tri);
    auto* r = new MeshResult();
    r->mesh = tet10 ? refine(t4, ELEM_TET10) : t4;
    return r;
  } catch (std::exception& ex) {
    g_last_error = ex.what();
    return nullptr;
  }
}
void* oracle_mesh_hex27_from_hex(void* hex) {
  auto* h = (MeshResult*)hex;
  auto* r = new MeshResult();
  r->mesh = refine(h->mesh, ELEM_HEX27);
  return r;
}
void* oracle_mesh_keep_cells(void* mesh, const int64_t* cells, int64_t nc) {
  auto* h = (MeshResult*)mesh;
  auto* r = new MeshResult();
  r->mesh = keep_cells(h->mesh, std::vector<i64>(cells, cells + nc));
  return r;
}
int64_t oracle_mesh_num_vertices(void* m) { return (int64_t)(((MeshResult*)m)->mesh.X.size() / 3); }
int64_t oracle_mesh_num_cells(void* m) { return (int64_t)((MeshResult*)m)->mesh.C.size(); }
int oracle_mesh_cell_size(void* m) {
  auto& C = ((MeshResult*)m)->mesh.C;
  return C.empty() ? 0 : (int)C[0].size();
}
void oracle_mesh_copy(void* m, double* X, int64_t* C) {
  auto& mm = ((MeshResult*)m)->mesh;
  std::memcpy(X, mm.X.data(), sizeof(double) * mm.X.size());
  i64 k = 0;
  for (auto& c : mm.C) for (i64 v : c) C[k++] = v;
}
void oracle_mesh_destroy(void* m) { delete (MeshResult*)m; }

// ---- scenes (model + material + BCs + integrator settings) -----------------
// Blocks are added in order; a block's quadrature is uniform when qoff == null.
void* oracle_scene_create(const double* X, int64_t num_nodes) {
  auto* s = new Scene();
  s->model.X.assign(X, X + 3 * num_nodes);
  s->model.num_nodes = num_nodes;
  return s;
}
int oracle_scene_add_block(void* sp, int kind, const int64_t* conn, int64_t ne, const int64_t* qoff, const double* qw,
                           const double* qp, int64_t nq_total) {
  auto* s = (Scene*)sp;
  Block b;
  b.kind = kind;
  int n = element_nodes(kind);
  b.conn.resize(ne);
  for (i64 e = 0; e < ne; ++e) b.conn[e].assign(conn + e * n, conn + (e + 1) * n);
  if (qoff) b.quad.offsets.assign(qoff, qoff + ne + 1);
  b.quad.w.assign(qw, qw + nq_total);
  b.quad.p.assign(qp, qp + 3 * nq_total);
  b.colors = greedy_coloring(b.conn);
  s->model.blocks.push_back(std::move(b));
  return 0;
}
// Colors across all blocks: returns number of colors of block `bi`.
int64_t oracle_scene_block_colors(void* sp, int bi, int64_t* color_offsets, int64_t* labels) {
  auto& b = ((Scene*)sp)->model.blocks[bi];
  if (color_offsets) {
    i64 k = 0;
    color_offsets[0] = 0;
    for (size_t c = 0; c < b.colors.size(); ++c) {
      for (i64 l : b.colors[c]) labels[k++] = l;
      color_offsets[c + 1] = k;
    }
  }
  return (int64_t)b.colors.size();
}
// Builds the shared pattern; must be called after all blocks are added.
int oracle_scene_finalize_pattern(void* sp) {
  auto* s = (Scene*)sp;
  std::vector<std::vector<i64>> all;
  for (auto& b : s->model.blocks) for (auto& c : b.conn) all.push_back(c);
  try {
    s->model.pattern = assemble_pattern(all, 3, s->model.num_nodes);
  } catch (std::exception& ex) {
    g_last_error = ex.what();
    return 1;
  }
  return 0;
}
int64_t oracle_scene_nnz(void* sp) { return (int64_t)((Scene*)sp)->model.pattern.col_indices.size(); }
void oracle_scene_pattern(void* sp, int64_t* ro, int64_t* ci) {
  auto& p = ((Scene*)sp)->model.pattern;
  std::memcpy(ro, p.row_offsets.data(), sizeof(i64) * p.row_offsets.size());
  std::memcpy(ci, p.col_indices.data(), sizeof(i64) * p.col_indices.size());
}
void oracle_scene_set_material(void* sp, int kind, double mu, double lambda, double density) {
  auto* s = (Scene*)sp;
  s->mat = {kind, {mu, lambda}};
  s->density = density;
}
int oracle_scene_assemble_forces(void* sp, const double* u, double* f) {
  auto* s = (Scene*)sp;
  return assemble_forces(s->model, s->mat, u, f) ? 0 : 1;
}
int oracle_scene_assemble_stiffness(void* sp, const double* u, double* v) {
  auto* s = (Scene*)sp;
  try {
    return assemble_stiffness(s->model, s->mat, u, v) ? 0 : 1;
  } catch (std::exception& ex) {
    g_last_error = ex.what();
    return 2;
  }
}
void oracle_scene_assemble_mass(void* sp, double density, double* v) {
  auto* s = (Scene*)sp;
  assemble_mass(s->model, density, v);
}
// Integrator configuration.  bc nodes sorted; schwarz subdomains ragged.
void oracle_scene_set_bc(void* sp, const int64_t* nodes, int64_t nn) {
  auto* s = (Scene*)sp;
  s->bc_nodes.assign(nodes, nodes + nn);
}
void oracle_scene_set_gravity(void* sp, int enabled, double g) {
  auto* s = (Scene*)sp;
  s->gravity_enabled = enabled != 0;
  s->gravity = g;
}
void oracle_scene_set_damping(void* sp, int has_mass, double mass_coeff, int has_stiffness, double stiffness_coeff) {
  auto* s = (Scene*)sp;
  s->has_mass_damping = has_mass != 0;
  s->mass_damping = mass_coeff;
  s->has_stiffness_damping = has_stiffness != 0;
  s->stiffness_damping = stiffness_coeff;
}
// Damping matrix at state u (after set_damping and setup); returns 0 on success.
int oracle_scene_damping(void* sp, const double* u, double* out) {
  auto* s = (Scene*)sp;
  if (!compute_damping(*s, u)) return 1;
  if (s->has_damping) std::copy(s->damping.begin(), s->damping.end(), out);
  return 0;
}
int oracle_scene_assemble_stiffness_projected(void* sp, const double* u, double* v) {
  auto* s = (Scene*)sp;
  return assemble_stiffness_projected(s->model, s->mat, u, v) ? 0 : 1;
}
void oracle_scene_set_solver(void* sp, double cg_tol, int64_t cg_max_iter, int64_t newton_max_iter) {
  auto* s = (Scene*)sp;
  s->cg_tol = cg_tol;
  s->cg_max_iter = cg_max_iter;
  s->newton_max_iter = newton_max_iter;
}
void oracle_scene_set_schwarz(void* sp, const int64_t* offsets, const int64_t* nodes, int64_t ns,
                              const int64_t* untreated, int64_t nu) {
  auto* s = (Scene*)sp;
  s->precond = PRECOND_SCHWARZ;
  s->schwarz.subdomains.resize(ns);
  for (i64 k = 0; k < ns; ++k) s->schwarz.subdomains[k].assign(nodes + offsets[k], nodes + offsets[k + 1]);
  s->schwarz.untreated.assign(untreated, untreated + nu);
}
int oracle_scene_setup(void* sp) {
  auto* s = (Scene*)sp;
  try {
    scene_setup(*s);
  } catch (std::exception& ex) {
    g_last_error = ex.what();
    return 1;
  }
  return 0;
}
void oracle_scene_mass(void* sp, double* v) {
  auto* s = (Scene*)sp;
  std::memcpy(v, s->mass.data(), sizeof(double) * s->mass.size());
}
double oracle_scene_representative_force(void* sp) { return ((Scene*)sp)->representative_force; }
int64_t oracle_scene_schwarz_nnz(void* sp) { return (int64_t)((Scene*)sp)->schwarz.pattern.col_indices.size(); }
void oracle_scene_schwarz_pattern(void* sp, int64_t* ro, int64_t* ci) {
  auto& p = ((Scene*)sp)->schwarz.pattern;
  std::memcpy(ro, p.row_offsets.data(), sizeof(i64) * p.row_offsets.size());
  std::memcpy(ci, p.col_indices.data(), sizeof(i64) * p.col_indices.size());
}
// Schwarz update for a given system matrix (values on the model pattern).
int oracle_scene_schwarz_update(void* sp, const double* jv, double* pv) {
  auto* s = (Scene*)sp;
  if (!schwarz_update(s->schwarz, s->model.pattern, jv)) return 1;
  std::memcpy(pv, s->schwarz.v.data(), sizeof(double) * s->schwarz.v.size());
  return 0;
}
// J = dt^2 K + M with Dirichlet (compute_jacobian_combination_into).
void oracle_scene_jacobian(void* sp, const double* K, double dt, double* J) {
  auto* s = (Scene*)sp;
  const auto& p = s->model.pattern;
  size_t nnz = p.col_indices.size();
  double ck = -(-dt * dt);
  for (size_t k = 0; k < nnz; ++k) J[k] = 0.0;
  for (size_t k = 0; k < nnz; ++k) J[k] += ck * K[k];
  for (size_t k = 0; k < nnz; ++k) J[k] += 1.0 * s->mass[k];
  dirichlet_csr(p, J, s->bc_nodes.data(), (i64)s->bc_nodes.size(), 3);
}
// CG on the scene pattern with the scene's preconditioner (already updated
// when Schwarz).  Returns the CG status.
int oracle_scene_cg(void* sp, const double* J, const double* b, double* x, double tol, int64_t max_iter,
                    int64_t* iters) {
  auto* s = (Scene*)sp;
  const auto& p = s->model.pattern;
  const i64 n = p.nrows;
  LinOp A = [&](double* y, const double* xx) { spmv(0.0, y, 1.0, p, J, xx); return true; };
  std::vector<double> diag;
  LinOp P;
  if (s->precond == PRECOND_SCHWARZ) {
    P = [&](double* y, const double* xx) { spmv(0.0, y, 1.0, s->schwarz.pattern, s->schwarz.v.data(), xx); return true; };
  } else {
    diag.resize(n);
    for (i64 i = 0; i < n; ++i) {
      double d;
      if (!csr_get(p, J, i, i, d)) d = 0.0;
      diag[i] = 1.0 / d;
    }
    P = [&](double* y, const double* xx) { for (i64 i = 0; i < n; ++i) y[i] = diag[i] * xx[i]; return true; };
  }
  return cg_solve(n, A, &P, b, x, tol, max_iter, iters);
}
int oracle_scene_eval_f(void* sp, const double* u, const double* v, double* f) {
  return eval_f(*(Scene*)sp, u, v, f) ? 0 : 1;
}
// One NewtonCgIntegrator3d step (with substepping).  u, v updated in place.
int oracle_scene_step(void* sp, double* u, double* v, double t, double dt) {
  auto* s = (Scene*)sp;
  try {
    return integrate(*s, u, v, t, dt);
  } catch (std::exception& ex) {
    g_last_error = ex.what();
    return 99;
  }
}
int64_t oracle_scene_last_newton_iters(void* sp) { return ((Scene*)sp)->newton_iters; }
int64_t oracle_scene_last_num_cg(void* sp) { return (int64_t)((Scene*)sp)->cg_iters.size(); }
void oracle_scene_last_cg(void* sp, int64_t* iters, int32_t* status) {
  auto* s = (Scene*)sp;
  for (size_t k = 0; k < s->cg_iters.size(); ++k) {
    iters[k] = s->cg_iters[k];
    status[k] = s->cg_status[k];
  }
}
int64_t oracle_scene_last_substeps(void* sp) { return ((Scene*)sp)->num_substeps; }
int64_t oracle_scene_last_ls_backtracks(void* sp) { return ((Scene*)sp)->ls_backtracks; }
double oracle_scene_last_residual(void* sp) { return ((Scene*)sp)->last_residual; }
void oracle_scene_destroy(void* sp) { delete (Scene*)sp; }

}  // extern "C"
