// Embedded quadrature construction on the device: classification of the
// background cells of a hexahedral mesh against an embedded Tet4 mesh, the
// cut-cell quadrature of every interface cell in its background element's
// reference coordinates, and moment-preserving quadrature simplification.
//
// Reference (fenris):
//   embed_mesh_3d_with_opts / embed_in_cell      src/embedding/embedding3d.rs:57-196
//   compute_element_embedded_quadrature          src/embedding/embedding3d.rs:233-289
//   PolyMesh3d::intersect_half_space             src/geometry/polymesh.rs:629-808
//   PolyMesh3d::triangulate (Max 2000)           src/geometry/polymesh.rs:402-507
//   Tet4Mesh::try_from(&PolyMesh3d)              src/mesh_convert.rs:639-705
//   compute_polyhedron_volume_from_faces         src/geometry/mod.rs:1002-1032
//   map_physical_coordinates                     src/element.rs:2203-2275
//   optimize_quadrature / simplify_quadrature    src/embedding/quadrature_reduction.rs:35-260
//
// Decomposition.  The reference intersects, per background cell, the region
// of the embedded mesh whose cells' bounding boxes meet the cell's box with
// the cell's six face half-spaces, one embedded cell after another in the
// same mesh.  Every embedded cell is clipped independently of the others
// there (a face is classified from its own vertices; a new cap face belongs
// to one cell), so here every (background cell, embedded tet) pair is one
// thread: the tet is clipped by the six half-spaces in registers / local
// memory, the result split into tetrahedra, and their volumes summed in pair
// order.  Vertex labels, which pick the triangulation's apex and fan origins,
// follow the reference's first-appearance rule over the pair's own faces (the
// tet's faces in Tet4 face order, its vertices initially in ascending global
// index); the reference applies it over the whole region, with faces shared
// between cells, so the two triangulations of a cut polyhedron may differ
// while every integral of a polynomial up to the rule's strength agrees.
//
// Simplification.  The reference finds a basic feasible point of
// {w >= 0 : P w = P w0} with the OR-Tools GLOP solver (P: Chebyshev tensor
// moments up to the strength on the points' bounding box).  Here Caratheodory
// elimination does it: while more than r points carry weight, the null vector
// of r + 1 of their moment columns moves the weights until one reaches zero.
// Every moment is kept and at most r points remain (see k_simplify for the
// parallel form).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <memory>
#include <vector>

#include "internal.h"
#include "scene.h"

namespace hoefem {

namespace {

constexpr int EMV = 32;   // vertices of a clipped tet
constexpr int EMF = 16;   // faces
constexpr int EMFV = 16;  // vertices per face
constexpr int ERR_CAPACITY = 1, ERR_INVERSE = 2, ERR_DEGENERATE = 4;

__constant__ int c_hex_faces[6][4] = {{0, 1, 2, 3}, {4, 5, 1, 0}, {5, 6, 2, 1}, {6, 7, 3, 2}, {0, 3, 7, 4}, {4, 7, 6, 5}};
__constant__ double c_hex_alpha[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                         {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

struct P3 {
  double x, y, z;
};
__device__ __forceinline__ P3 mk(double a, double b, double c) { return P3{a, b, c}; }
__device__ __forceinline__ P3 sub(P3 a, P3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double dot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ P3 cross(P3 a, P3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double nrm(P3 a) { return sqrt(dot(a, a)); }

// Polygon area vector: fan from the first vertex, sum of (ab x ac) / 2.
__device__ P3 area_vec(const P3* v, int k) {
  P3 s = mk(0, 0, 0);
  for (int i = 1; i + 1 < k; ++i) {
    P3 c = cross(sub(v[i], v[0]), sub(v[i + 1], v[0]));
    s.x += c.x * 0.5;
    s.y += c.y * 0.5;
    s.z += c.z * 0.5;
  }
  return s;
}
// one face's term of the polyhedron volume: (n . x0) area
__device__ double volume_term(const P3* v, int k) {
  if (k <= 2) return 0.0;
  P3 a = area_vec(v, k);
  double ar = nrm(a);
  if (!(ar > 0.0)) return 0.0;
  return dot(mk(a.x / ar, a.y / ar, a.z / ar), v[0]) * ar;
}
// Tetrahedron volume from its faces (0,1,2), (0,3,1), (1,3,2), (0,2,3).
__device__ double tet_volume(P3 a, P3 b, P3 c, P3 d) {
  P3 f[3];
  double s = 0.0;
  f[0] = a; f[1] = b; f[2] = c; s += volume_term(f, 3);
  f[0] = a; f[1] = d; f[2] = b; s += volume_term(f, 3);
  f[0] = b; f[1] = d; f[2] = c; s += volume_term(f, 3);
  f[0] = a; f[1] = c; f[2] = d; s += volume_term(f, 3);
  return fabs(s) / 3.0;
}

struct Hex {
  P3 X[8];
};
__device__ Hex load_hex(const double* __restrict__ corners, long long c) {
  Hex h;
  for (int I = 0; I < 8; ++I) {
    const double* p = corners + (size_t)24 * c + 3 * I;
    h.X[I] = mk(p[0], p[1], p[2]);
  }
  return h;
}
// inward half-space of face f: point, unit normal
__device__ void hex_half_space(const Hex& h, int f, P3& x0, P3& n) {
  P3 q[4];
  for (int k = 0; k < 4; ++k) q[k] = h.X[c_hex_faces[f][k]];
  P3 a = area_vec(q, 4);
  double an = nrm(a);
  n = mk(a.x / an, a.y / an, a.z / an);
  x0 = q[0];
}

// ---- the clipped polyhedron of one (cell, tet) pair ---------------------------
struct Poly {
  int nv, nf;
  P3 X[EMV];
  unsigned char fn[EMF];
  unsigned char fv[EMF][EMFV];
};

__device__ __forceinline__ unsigned short rep(int a, int b) {
  return a <= b ? (unsigned short)((a << 8) | b) : (unsigned short)((b << 8) | a);
}

// Closest point to the plane on the segment a -> b.
__device__ P3 seg_plane(P3 a, P3 b, P3 x0, P3 n) {
  P3 d = sub(b, a), y = sub(x0, a);
  double nTd = dot(n, d), nTy = dot(n, y);
  double t;
  if (signbit(nTd) == signbit(nTy)) t = fabs(nTy) >= fabs(nTd) ? 1.0 : nTy / nTd;
  else t = 0.0;
  return mk(a.x * (1.0 - t) + b.x * t, a.y * (1.0 - t) + b.y * t, a.z * (1.0 - t) + b.z * t);
}

// Keeps the part with n.(x - x0) >= 0.  Returns false on a capacity overflow.
__device__ bool clip(Poly& P, P3 x0, P3 n) {
  bool in[EMV];
  for (int v = 0; v < P.nv; ++v) in[v] = dot(n, sub(P.X[v], x0)) >= 0.0;
  unsigned short R[EMF][EMFV];
  unsigned char rn[EMF];
  int nr = 0;
  unsigned short ie[EMF][2];  // intersection edges (pairs of cut vertices)
  int nie = 0;
  for (int f = 0; f < P.nf; ++f) {
    const int k = P.fn[f];
    int m = 0;
    bool cut = false;
    for (int i = 0; i < k; ++i) {
      const int a = P.fv[f][i], b = P.fv[f][(i + 1) % k];
      if (in[a]) {
        if (m == EMFV) return false;
        R[nr][m++] = rep(a, a);
      }
      if (in[a] != in[b]) {
        if (m == EMFV) return false;
        R[nr][m++] = rep(a, b);
        cut = true;
      }
    }
    rn[nr] = (unsigned char)m;
    if (cut) {
      for (int i = 0; i < m; ++i) {
        const unsigned short ra = R[nr][i], rb = R[nr][(i + 1) % m];
        if ((ra >> 8) != (ra & 255) && (rb >> 8) != (rb & 255)) {
          if (nie == EMF) return false;
          ie[nie][0] = ra;
          ie[nie][1] = rb;
          ++nie;
        }
      }
    }
    ++nr;
  }
  // string the intersection edges into cap faces (last edge first, then the
  // first edge that continues the chain, removed by swapping in the last)
  while (nie > 0) {
    if (nr == EMF) return false;
    --nie;
    const unsigned short sa = ie[nie][0];
    unsigned short next = ie[nie][1];
    int m = 0;
    R[nr][m++] = sa;
    for (;;) {
      int pos = -1;
      for (int i = 0; i < nie; ++i)
        if (ie[i][0] == next || ie[i][1] == next) { pos = i; break; }
      if (pos < 0) break;
      const unsigned short ea = ie[pos][0], eb = ie[pos][1];
      ie[pos][0] = ie[nie - 1][0];
      ie[pos][1] = ie[nie - 1][1];
      --nie;
      if (m == EMFV) return false;
      if (ea == next) {
        R[nr][m++] = ea;
        next = eb;
      } else {
        R[nr][m++] = eb;
        next = ea;
      }
    }
    rn[nr++] = (unsigned char)m;
  }
  // labels by first appearance; new coordinates
  unsigned short lab[EMV];
  int nl = 0;
  P3 Y[EMV];
  unsigned char newf[EMF][EMFV];
  unsigned char newn[EMF];
  int nf = 0;
  for (int f = 0; f < nr; ++f) {
    if (rn[f] == 0) continue;
    for (int i = 0; i < rn[f]; ++i) {
      const unsigned short r = R[f][i];
      int l = -1;
      for (int j = 0; j < nl; ++j)
        if (lab[j] == r) { l = j; break; }
      if (l < 0) {
        if (nl == EMV) return false;
        l = nl++;
        lab[l] = r;
        const int a = r >> 8, b = r & 255;
        Y[l] = (a == b) ? P.X[a] : seg_plane(P.X[a], P.X[b], x0, n);
      }
      newf[nf][i] = (unsigned char)l;
    }
    newn[nf] = rn[f];
    ++nf;
  }
  P.nv = nl;
  for (int v = 0; v < nl; ++v) P.X[v] = Y[v];
  P.nf = nf;
  for (int f = 0; f < nf; ++f) {
    P.fn[f] = newn[f];
    for (int i = 0; i < newn[f]; ++i) P.fv[f][i] = newf[f][i];
  }
  return true;
}

// Clips tet t of the embedded mesh by cell c's six half-spaces.
__device__ bool clip_pair(const Hex& h, const double* __restrict__ eX, const int* __restrict__ tet_faces, long long t,
                          Poly& P) {
  // vertices in ascending global index, faces in the embedded mesh's order
  const int* tf = tet_faces + (size_t)12 * t;
  int g[4];
  int ng = 0;
  for (int k = 0; k < 12; ++k) {
    bool seen = false;
    for (int j = 0; j < ng; ++j) seen = seen || g[j] == tf[k];
    if (!seen && ng < 4) g[ng++] = tf[k];
  }
  for (int i = 1; i < ng; ++i)
    for (int j = i; j > 0 && g[j - 1] > g[j]; --j) {
      int tmp = g[j];
      g[j] = g[j - 1];
      g[j - 1] = tmp;
    }
  P.nv = ng;
  for (int i = 0; i < ng; ++i) P.X[i] = mk(eX[3 * (size_t)g[i]], eX[3 * (size_t)g[i] + 1], eX[3 * (size_t)g[i] + 2]);
  P.nf = 4;
  for (int f = 0; f < 4; ++f) {
    P.fn[f] = 3;
    for (int i = 0; i < 3; ++i) {
      int l = 0;
      while (l < ng && g[l] != tf[3 * f + i]) ++l;
      P.fv[f][i] = (unsigned char)l;
    }
  }
  for (int f = 0; f < 6; ++f) {
    P3 x0, n;
    hex_half_space(h, f, x0, n);
    if (!clip(P, x0, n)) return false;
    if (P.nf == 0) break;
  }
  return true;
}

// Visits the tetrahedra of the clipped polyhedron: apex = the vertex with the
// smallest label, every face without it fanned from its smallest label, the
// base oriented towards the apex.  visit(a, b, c, d) gets the 4 corners.
template <class F>
__device__ void for_each_tet(const Poly& P, F&& visit) {
  if (P.nf == 0) return;
  int v = 255;
  for (int f = 0; f < P.nf; ++f)
    for (int i = 0; i < P.fn[f]; ++i) v = min(v, (int)P.fv[f][i]);
  for (int f = 0; f < P.nf; ++f) {
    const int k = P.fn[f];
    bool has = false;
    int mi = 0;
    for (int i = 0; i < k; ++i) {
      has = has || P.fv[f][i] == v;
      if (P.fv[f][i] < P.fv[f][mi]) mi = i;
    }
    if (has) continue;
    for (int i = 0; i + 2 < k; ++i) {
      int a = P.fv[f][mi], b = P.fv[f][(i + 1 + mi) % k], c = P.fv[f][(i + 2 + mi) % k];
      P3 nn = cross(sub(P.X[b], P.X[a]), sub(P.X[c], P.X[a]));
      double l = nrm(nn);
      P3 nu = mk(nn.x / l, nn.y / l, nn.z / l);
      if (dot(nu, sub(P.X[v], P.X[a])) < 0.0) {
        int tmp = a;
        a = b;
        b = tmp;
      }
      visit(P.X[a], P.X[b], P.X[c], P.X[v]);
    }
  }
}

// Trilinear map of the background cell (Hex27 geometry = its 8 corners).
__device__ void hex_map(const Hex& h, P3 xi, P3& x, double J[9]) {
  x = mk(0, 0, 0);
  for (int k = 0; k < 9; ++k) J[k] = 0.0;
  for (int I = 0; I < 8; ++I) {
    const double a0 = c_hex_alpha[I][0], a1 = c_hex_alpha[I][1], a2 = c_hex_alpha[I][2];
    const double p0 = (1.0 + a0 * xi.x) / 2.0, p1 = (1.0 + a1 * xi.y) / 2.0, p2 = (1.0 + a2 * xi.z) / 2.0;
    const double N = p0 * p1 * p2;
    const double g[3] = {a0 / 2.0 * p1 * p2, p0 * a1 / 2.0 * p2, p0 * p1 * a2 / 2.0};
    const double X[3] = {h.X[I].x, h.X[I].y, h.X[I].z};
    x.x += X[0] * N;
    x.y += X[1] * N;
    x.z += X[2] * N;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) J[3 * i + j] += X[i] * g[j];
  }
}
__device__ double det3(const double J[9]) {
  return J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) + J[2] * (J[3] * J[7] - J[4] * J[6]);
}
// J d = b by elimination with full pivoting
__device__ bool solve3(const double J[9], const double b[3], double d[3]) {
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
        if (fabs(A[i][j]) > fabs(A[pi][pj])) { pi = i; pj = j; }
    if (A[pi][pj] == 0.0) return false;
    for (int j = 0; j < 4; ++j) { double t = A[k][j]; A[k][j] = A[pi][j]; A[pi][j] = t; }
    for (int i = 0; i < 3; ++i) { double t = A[i][k]; A[i][k] = A[i][pj]; A[i][pj] = t; }
    int tc = col[k]; col[k] = col[pj]; col[pj] = tc;
    for (int i = k + 1; i < 3; ++i) {
      const double f = A[i][k] / A[k][k];
      for (int j = k; j < 4; ++j) A[i][j] -= f * A[k][j];
    }
  }
  double y[3];
  for (int k = 2; k >= 0; --k) {
    double s = A[k][3];
    for (int j = k + 1; j < 3; ++j) s -= A[k][j] * y[j];
    y[k] = s / A[k][k];
  }
  for (int k = 0; k < 3; ++k) d[col[k]] = y[k];
  return true;
}
// Newton from xi = 0 until |T(xi) - x| <= 1e-12 diameter, at most 20 steps.
__device__ bool hex_inverse(const Hex& h, P3 x, P3& xi) {
  double diam = 0.0;
  for (int i = 0; i < 8; ++i)
    for (int j = i + 1; j < 8; ++j) diam = fmax(diam, nrm(sub(h.X[i], h.X[j])));
  const double tol = 1e-12 * diam;
  xi = mk(0, 0, 0);
  P3 y;
  double J[9];
  hex_map(h, xi, y, J);
  P3 f = sub(y, x);
  for (int it = 0;; ++it) {
    if (!(nrm(f) > tol)) return true;
    if (it == 20) return false;
    double b[3] = {f.x, f.y, f.z}, d[3];
    if (!solve3(J, b, d)) return false;
    xi = mk(xi.x - d[0], xi.y - d[1], xi.z - d[2]);
    hex_map(h, xi, y, J);
    f = sub(y, x);
  }
}

// ---- kernels -------------------------------------------------------------------
// Candidate tets of every cell (bounding boxes meet, closed intervals), in
// ascending tet order: count pass (out == nullptr) or fill pass.
__global__ void __launch_bounds__(256) k_embed_candidates(long long nbc, const double* __restrict__ cbox,
                                                          long long nt, const double* __restrict__ tbox,
                                                          const long long* __restrict__ off, long long* __restrict__ count,
                                                          int* __restrict__ out) {
  __shared__ int s_w[8];
  __shared__ long long s_base;
  const long long c = blockIdx.x;
  if (c >= nbc) return;
  double cb[6];
  for (int k = 0; k < 6; ++k) cb[k] = cbox[6 * c + k];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_base = out ? off[c] : 0;
  __syncthreads();
  for (long long t0 = 0; t0 < nt; t0 += blockDim.x) {
    const long long t = t0 + threadIdx.x;
    bool hit = false;
    if (t < nt) {
      const double* tb = tbox + 6 * t;
      hit = cb[0] <= tb[3] && tb[0] <= cb[3] && cb[1] <= tb[4] && tb[1] <= cb[4] && cb[2] <= tb[5] && tb[2] <= cb[5];
    }
    const unsigned bal = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) s_w[w] = __popc(bal);
    __syncthreads();
    int before = 0, total = 0;
    for (int k = 0; k < 8; ++k) {
      if (k < w) before += s_w[k];
      total += s_w[k];
    }
    if (hit && out) out[s_base + before + __popc(bal & ((1u << lane) - 1u))] = (int)t;
    __syncthreads();
    if (threadIdx.x == 0) s_base += total;
    __syncthreads();
  }
  if (!out && threadIdx.x == 0) count[c] = s_base;
}

// Pass 1: cut volume and tetrahedron count of every pair.
__global__ void __launch_bounds__(128) k_embed_clip_count(long long npairs, const int* __restrict__ pcell,
                                                          const int* __restrict__ ptet, const double* __restrict__ corners,
                                                          const double* __restrict__ eX, const int* __restrict__ tet_faces,
                                                          double* __restrict__ vol, int* __restrict__ ntet, int* err) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  const Hex h = load_hex(corners, pcell[k]);
  Poly P;
  if (!clip_pair(h, eX, tet_faces, ptet[k], P)) {
    atomicOr(err, ERR_CAPACITY);
    vol[k] = 0.0;
    ntet[k] = 0;
    return;
  }
  double v = 0.0;
  int nt = 0;
  for_each_tet(P, [&](P3 a, P3 b, P3 c, P3 d) {
    v += tet_volume(a, b, c, d);
    ++nt;
  });
  vol[k] = v;
  ntet[k] = nt;
}

// Classification by the summed cut volume (pairs of a cell summed in order).
__global__ void k_embed_classify(long long nbc, const long long* __restrict__ off, const double* __restrict__ vol,
                                 const double* __restrict__ corners, double lower, double upper,
                                 int* __restrict__ cls, double* __restrict__ cut) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= nbc) return;
  double v = 0.0;
  bool any = false;
  for (long long k = off[c]; k < off[c + 1]; ++k) {
    v += vol[k];
    any = any || vol[k] != 0.0;
  }
  // the reference's volume of the hexahedron from its six faces
  const Hex h = load_hex(corners, c);
  double s = 0.0;
  for (int f = 0; f < 6; ++f) {
    P3 q[4];
    for (int j = 0; j < 4; ++j) q[j] = h.X[c_hex_faces[f][j]];
    s += volume_term(q, 4);
  }
  const double bgv = fabs(s) / 3.0;
  (void)any;
  cut[c] = v;
  cls[c] = v < lower * bgv ? 0 : (v < upper * bgv ? 2 : 1);
}

// Pass 2: the tet rule on every tetrahedron of the listed pairs, mapped to the
// background cell's reference coordinates.
__global__ void __launch_bounds__(128) k_embed_clip_write(long long nlist, const long long* __restrict__ list,
                                                          const int* __restrict__ pcell, const int* __restrict__ ptet,
                                                          const double* __restrict__ corners,
                                                          const double* __restrict__ eX,
                                                          const int* __restrict__ tet_faces,
                                                          const long long* __restrict__ qoff, int nq,
                                                          const double* __restrict__ tw, const double* __restrict__ tp,
                                                          double* __restrict__ w, double* __restrict__ p, int* err) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= nlist) return;
  const long long k = list[j];
  const Hex h = load_hex(corners, pcell[k]);
  Poly P;
  if (!clip_pair(h, eX, tet_faces, ptet[k], P)) {
    atomicOr(err, ERR_CAPACITY);
    return;
  }
  long long o = qoff[j];
  for_each_tet(P, [&](P3 a, P3 b, P3 c, P3 d) {
    // Tet4: N = [-(xi + eta + zeta + 1) / 2, (xi + 1) / 2, (eta + 1) / 2, (zeta + 1) / 2]
    double Jt[9] = {-0.5 * a.x + 0.5 * b.x, -0.5 * a.x + 0.5 * c.x, -0.5 * a.x + 0.5 * d.x,
                    -0.5 * a.y + 0.5 * b.y, -0.5 * a.y + 0.5 * c.y, -0.5 * a.y + 0.5 * d.y,
                    -0.5 * a.z + 0.5 * b.z, -0.5 * a.z + 0.5 * c.z, -0.5 * a.z + 0.5 * d.z};
    const double dJt = fabs(det3(Jt));
    for (int q = 0; q < nq; ++q) {
      const double* xi = tp + 3 * q;
      const double N0 = -0.5 * xi[0] - 0.5 * xi[1] - 0.5 * xi[2] - 0.5, N1 = 0.5 * xi[0] + 0.5,
                   N2 = 0.5 * xi[1] + 0.5, N3 = 0.5 * xi[2] + 0.5;
      P3 x = mk(a.x * N0 + b.x * N1 + c.x * N2 + d.x * N3, a.y * N0 + b.y * N1 + c.y * N2 + d.y * N3,
                a.z * N0 + b.z * N1 + c.z * N2 + d.z * N3);
      P3 xb;
      if (!hex_inverse(h, x, xb)) {
        atomicOr(err, ERR_INVERSE);
        xb = mk(0, 0, 0);
      }
      P3 y;
      double Jb[9];
      hex_map(h, xb, y, Jb);
      w[o] = tw[q] * dJt / fabs(det3(Jb));
      p[3 * o] = xb.x;
      p[3 * o + 1] = xb.y;
      p[3 * o + 2] = xb.z;
      ++o;
    }
  });
}

// Stabilization points (factor x the uncut rule) at the end of every interface rule.
__global__ void k_embed_stab(long long ncell, const long long* __restrict__ soff, int ns, double factor,
                             const double* __restrict__ sw, const double* __restrict__ sp, double* __restrict__ w,
                             double* __restrict__ p) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= ncell * ns) return;
  const long long c = j / ns;
  const int q = (int)(j - c * ns);
  const long long o = soff[c] + q;
  w[o] = factor * sw[q];
  for (int k = 0; k < 3; ++k) p[3 * o + k] = sp[3 * q + k];
}

// ---- simplification ------------------------------------------------------------
// Any subset of a rule's points can be reduced on its own: keeping the subset's
// moments keeps the rule's.  So one CTA per rule reduces groups of 2r
// consecutive points to at most r points each (one warp per group), then
// merges neighbouring groups pairwise (2r -> r) until one group is left.  A
// reduction step takes the first r + 1 points of a group's list, computes a
// null vector of their r x (r + 1) moment block (Gaussian elimination with
// partial pivoting in the warp's shared memory; the block is evaluated from
// the points on the fly), moves the weights along it until one reaches zero,
// and drops that point.
constexpr int SIMP_RMAX = 56;  // strength 5

__device__ __forceinline__ double cheb(double x, int n) {
  double t0 = 1.0, t1 = x;
  if (n == 0) return t0;
  for (int k = 2; k <= n; ++k) {
    const double t2 = __dsub_rn(__dmul_rn(__dmul_rn(2.0, x), t1), t0);
    t0 = t1;
    t1 = t2;
  }
  return t1;
}

__device__ double block_reduce_max(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = sh[0];
  for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = fmax(r, sh[k]);
  __syncthreads();
  return r;
}
__device__ double block_reduce_min(double v, double* sh) { return -block_reduce_max(-v, sh); }

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// (value, index) reductions: the largest (smallest) value, ties to the smaller index
__device__ __forceinline__ void warp_argmax(double& v, int& i) {
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
  }
}
__device__ __forceinline__ void warp_argmin(double& v, int& i) {
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (ov < v || (ov == v && oi < i)) { v = ov; i = oi; }
  }
}

struct SimpCta {
  unsigned char mono[SIMP_RMAX][3];  // (a, b, c) of every moment row
  double al[3], be[3];               // Chebyshev scaling of the rule's bounding box
  double sh[32];
};

// Reduces the warp's list L (nL sorted point indices with positive weight) to
// at most r points; returns the new length.  A: r x (r + 1), z, pv: m entries.
__device__ int warp_reduce_list(const SimpCta& C, int r, int strength, const double* __restrict__ pp,
                                double* __restrict__ w, int* L, int nL, double* A, double* z, int* pv, int* err) {
  const int lane = threadIdx.x & 31;
  const int m = r + 1;
  while (nL > r) {
    // moment block of the first m points, element by element
    for (int t = lane; t < r * m; t += 32) {
      const int i = t / m, j = t - i * m;
      const double* x = pp + 3 * (size_t)L[j];
      A[t] = __dmul_rn(__dmul_rn(cheb(C.al[0] * x[0] + C.be[0], C.mono[i][0]), cheb(C.al[1] * x[1] + C.be[1], C.mono[i][1])),
                       cheb(C.al[2] * x[2] + C.be[2], C.mono[i][2]));
    }
    __syncwarp();
    double amax = 0.0;
    for (int t = lane; t < r * m; t += 32) amax = fmax(amax, fabs(A[t]));
    const double eps = 1e-13 * warp_max(amax);
    int row = 0, npiv = 0;
    unsigned long long pivmask = 0ull;
    for (int c = 0; c < m && row < r; ++c) {
      double best = -1.0;
      int bi = r;
      for (int i = row + lane; i < r; i += 32) {
        const double v = fabs(A[i * m + c]);
        if (v > best) { best = v; bi = i; }
      }
      warp_argmax(best, bi);
      if (!(best > eps)) continue;
      if (bi != row)
        for (int j = lane; j < m; j += 32) {
          const double t = A[row * m + j];
          A[row * m + j] = A[bi * m + j];
          A[bi * m + j] = t;
        }
      __syncwarp();
      // row factors (into z, free until the back substitution), then the
      // update element by element over all lanes
      for (int i = row + 1 + lane; i < r; i += 32) z[i] = A[i * m + c] / A[row * m + c];
      __syncwarp();
      const int nrow = r - row - 1, ncol = m - c;
      for (int t = lane; t < nrow * ncol; t += 32) {
        const int i = row + 1 + t / ncol, j = c + t % ncol;
        A[i * m + j] = __dsub_rn(A[i * m + j], __dmul_rn(z[i], A[row * m + j]));
      }
      __syncwarp();
      if (lane == 0) pv[npiv] = c;
      ++npiv;
      pivmask |= 1ull << c;
      ++row;
    }
    __syncwarp();
    const unsigned long long freemask = ~pivmask & ((m == 64) ? ~0ull : ((1ull << m) - 1ull));
    if (freemask == 0ull) {  // (cannot happen with m = r + 1 columns)
      if (lane == 0) atomicOr(err, ERR_DEGENERATE);
      return nL;
    }
    const int fc = 63 - __clzll((long long)freemask);
    for (int j = lane; j < m; j += 32) z[j] = (j == fc) ? 1.0 : 0.0;
    __syncwarp();
    for (int k = npiv - 1; k >= 0; --k) {
      const int c = pv[k];
      double s = 0.0;
      for (int j = c + 1 + lane; j < m; j += 32) s = __dadd_rn(s, __dmul_rn(A[k * m + j], z[j]));
      s = warp_sum(s);
      if (lane == 0) z[c] = -s / A[k * m + c];
      __syncwarp();
    }
    // direction: flipped when no component is positive
    bool pos = false;
    for (int j = lane; j < m; j += 32) pos = pos || z[j] > 0.0;
    const bool flip = !__any_sync(0xffffffffu, pos);
    double tmin = INFINITY;
    int arg = m;
    for (int j = lane; j < m; j += 32) {
      const double zj = flip ? -z[j] : z[j];
      if (zj > 0.0) {
        const double q = w[L[j]] / zj;
        if (q < tmin) { tmin = q; arg = j; }
      }
    }
    warp_argmin(tmin, arg);
    for (int j = lane; j < m; j += 32) {
      const double zj = flip ? -z[j] : z[j];
      const double v = __dsub_rn(w[L[j]], __dmul_rn(tmin, zj));
      w[L[j]] = (j == arg || v < 0.0) ? 0.0 : v;
    }
    __syncwarp();
    // drop the points whose weight reached zero (order kept)
    int out = 0;
    for (int base = 0; base < nL; base += 32) {
      const int j = base + lane;
      const int idx = j < nL ? L[j] : -1;
      const bool keep = j < nL && w[idx] > 0.0;
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      __syncwarp();
      if (keep) L[out + __popc(bal & ((1u << lane) - 1u))] = idx;
      out += __popc(bal);
      __syncwarp();
    }
    nL = out;
  }
  return nL;
}

// One CTA per rule (warps = blockDim.x / 32).  grp: per-rule scratch of n
// ints (group lists, stride 2r), gcnt: group lengths (n entries per rule).
__global__ void __launch_bounds__(256, 4) k_simplify(const long long* __restrict__ off, const double* __restrict__ p, double* __restrict__ wk,
                           int strength, int r, int* __restrict__ grp, int* __restrict__ gcnt,
                           int* __restrict__ keep, int* __restrict__ nkeep, int* err) {
  extern __shared__ double smem[];
  __shared__ SimpCta C;
  const long long o = off[blockIdx.x];
  const int n = (int)(off[blockIdx.x + 1] - o);
  const double* pp = p + 3 * o;
  double* w = wk + o;
  int* kp = keep + o;
  if (n <= r) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) kp[i] = i;
    if (threadIdx.x == 0) nkeep[blockIdx.x] = n;
    return;
  }
  if (threadIdx.x == 0) {
    int row = 0;
    for (int a = 0; a <= strength; ++a)
      for (int b = 0; b <= strength; ++b)
        for (int c = 0; c <= strength; ++c)
          if (a + b + c <= strength && row < SIMP_RMAX) {
            C.mono[row][0] = (unsigned char)a;
            C.mono[row][1] = (unsigned char)b;
            C.mono[row][2] = (unsigned char)c;
            ++row;
          }
  }
  for (int d = 0; d < 3; ++d) {
    double lo = INFINITY, hi = -INFINITY;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      lo = fmin(lo, pp[3 * i + d]);
      hi = fmax(hi, pp[3 * i + d]);
    }
    lo = block_reduce_min(lo, C.sh);
    hi = block_reduce_max(hi, C.sh);
    if (threadIdx.x == 0) {
      const double c = (lo + hi) / 2.0, l = (hi - lo) / 2.0;
      C.al[d] = l != 0.0 ? 1.0 / l : 0.0;
      C.be[d] = 1.0 - C.al[d] * (c + l);
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int m = r + 1, G = 2 * r;
  // per-warp shared memory: A (r x m), z (m), L (2r ints), pv (m ints)
  const size_t per = (size_t)r * m + m + (size_t)(G + m + 1) / 2 + 1;
  double* A = smem + per * wid;
  double* z = A + (size_t)r * m;
  int* L = (int*)(z + m);
  int* pv = L + G;
  int* glist = grp + o;
  int* gc = gcnt + o;
  const int ng = (n + G - 1) / G;
  // level 0: groups of G consecutive points
  for (int g = wid; g < ng; g += nw) {
    const int lo = g * G, hi = min(lo + G, n);
    int nL = 0;
    for (int base = lo; base < hi; base += 32) {
      const int i = base + lane;
      const bool pos = i < hi && w[i] > 0.0;
      const unsigned bal = __ballot_sync(0xffffffffu, pos);
      if (pos) L[nL + __popc(bal & ((1u << lane) - 1u))] = i;
      nL += __popc(bal);
    }
    __syncwarp();
    nL = warp_reduce_list(C, r, strength, pp, w, L, nL, A, z, pv, err);
    for (int j = lane; j < nL; j += 32) glist[(size_t)g * G + j] = L[j];
    if (lane == 0) gc[g] = nL;
    __syncwarp();
  }
  __syncthreads();
  // pairwise merges
  for (int s = 1; s < ng; s *= 2) {
    for (int g = 2 * s * wid; g < ng; g += 2 * s * nw) {
      int nL = gc[g];
      for (int j = lane; j < nL; j += 32) L[j] = glist[(size_t)g * G + j];
      if (g + s < ng) {
        const int n2 = gc[g + s];
        if (nL + n2 > G) {  // (a reduction left more than r points: cannot happen)
          if (lane == 0) atomicOr(err, ERR_DEGENERATE);
          continue;
        }
        for (int j = lane; j < n2; j += 32) L[nL + j] = glist[(size_t)(g + s) * G + j];
        nL += n2;
      }
      __syncwarp();
      nL = warp_reduce_list(C, r, strength, pp, w, L, nL, A, z, pv, err);
      for (int j = lane; j < nL; j += 32) glist[(size_t)g * G + j] = L[j];
      if (lane == 0) gc[g] = nL;
      __syncwarp();
    }
    __syncthreads();
  }
  for (int j = threadIdx.x; j < gc[0]; j += blockDim.x) kp[j] = glist[j];
  if (threadIdx.x == 0) nkeep[blockIdx.x] = gc[0];
}

// The kept points of every rule, compacted to the output offsets.
__global__ void k_simplify_gather(const long long* __restrict__ off, const long long* __restrict__ outoff,
                                  const int* __restrict__ keep, const double* __restrict__ w,
                                  const double* __restrict__ p, double* __restrict__ ow, double* __restrict__ op) {
  const long long o = off[blockIdx.x], q = outoff[blockIdx.x];
  const int nk = (int)(outoff[blockIdx.x + 1] - q);
  for (int j = threadIdx.x; j < nk; j += blockDim.x) {
    const long long i = o + keep[o + j];
    ow[q + j] = w[i];
    for (int d = 0; d < 3; ++d) op[3 * (q + j) + d] = p[3 * i + d];
  }
}

}  // namespace

// ---- host side -------------------------------------------------------------------

struct Embedding {
  int device = 0;
  cudaStream_t stream = nullptr;
  i64 nbc = 0, nt = 0, npairs = 0;
  std::vector<i64> off;        // pairs of cell c: [off[c], off[c+1])
  std::vector<int> cls;
  std::vector<double> cut;
  DBuf<double> d_corners, d_eX;
  DBuf<int> d_tet_faces, d_pcell, d_ptet;
  std::vector<int> ntet;
  // last quadrature (device resident until copied out)
  std::vector<i64> q_off;
  DBuf<double> q_w, q_p;
  i64 q_total = 0;
  ~Embedding() {
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {
void check_err(DBuf<int>& err, cudaStream_t s) {
  int e = 0;
  HOEFEM_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  HOEFEM_REQUIRE(!(e & ERR_CAPACITY), HOEFEM_ERR_INVALID_ARGUMENT,
                 "a clipped embedded cell exceeds the local polyhedron capacity (degenerate input?)");
  HOEFEM_REQUIRE(!(e & ERR_INVERSE), HOEFEM_ERR_SINGULAR, "background element map could not be inverted");
  HOEFEM_REQUIRE(!(e & ERR_DEGENERATE), HOEFEM_ERR_SINGULAR, "quadrature simplification found no null vector");
}
void require_device() {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    throw Error(HOEFEM_ERR_NO_DEVICE, "no CUDA device available");
  }
}
}  // namespace

Embedding* embedding_create(const double* bgX, i64 nbv, const i64* bg_conn, i64 nbc, int npc, const double* eX,
                            i64 nev, const i64* tets, i64 nt, double lower, double upper) {
  HOEFEM_REQUIRE(npc == 8 || npc == 27, HOEFEM_ERR_INVALID_ARGUMENT, "background cells need 8 or 27 nodes");
  HOEFEM_REQUIRE(nbc > 0 && nt >= 0 && nev >= 0 && nbv > 0, HOEFEM_ERR_INVALID_ARGUMENT, "empty mesh");
  HOEFEM_REQUIRE(nbc < (i64)INT32_MAX && nt < (i64)INT32_MAX && nev < (i64)INT32_MAX, HOEFEM_ERR_INVALID_ARGUMENT,
                 "mesh too large");
  auto E = std::make_unique<Embedding>();
  E->nbc = nbc;
  E->nt = nt;
  // background corners and boxes
  std::vector<double> corners((size_t)24 * nbc), cbox((size_t)6 * nbc);
  for (i64 c = 0; c < nbc; ++c) {
    double* b = &cbox[6 * c];
    for (int k = 0; k < 3; ++k) { b[k] = INFINITY; b[3 + k] = -INFINITY; }
    for (int I = 0; I < 8; ++I) {
      const i64 v = bg_conn[(size_t)npc * c + I];
      HOEFEM_REQUIRE(v >= 0 && v < nbv, HOEFEM_ERR_INVALID_ARGUMENT, "background connectivity out of range");
      for (int k = 0; k < 3; ++k) {
        const double x = bgX[3 * v + k];
        corners[24 * c + 3 * I + k] = x;
        b[k] = std::min(b[k], x);
        b[3 + k] = std::max(b[3 + k], x);
      }
    }
  }
  // every tet's faces in Tet4 face order (0,2,1), (0,1,3), (1,2,3), (0,3,2);
  // bounding boxes
  static const int TF[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {0, 3, 2}};
  std::vector<int> tet_faces((size_t)12 * std::max<i64>(nt, 1));
  std::vector<double> tbox((size_t)6 * std::max<i64>(nt, 1));
  for (i64 t = 0; t < nt; ++t) {
    const i64* v = tets + 4 * t;
    for (int i = 0; i < 4; ++i) {
      HOEFEM_REQUIRE(v[i] >= 0 && v[i] < nev, HOEFEM_ERR_INVALID_ARGUMENT, "tet connectivity out of range");
      for (int j = 0; j < i; ++j)
        HOEFEM_REQUIRE(v[i] != v[j], HOEFEM_ERR_INVALID_ARGUMENT, "tet with repeated vertices");
    }
    for (int f = 0; f < 4; ++f)
      for (int i = 0; i < 3; ++i) tet_faces[12 * t + 3 * f + i] = (int)v[TF[f][i]];
    double* b = &tbox[6 * t];
    for (int k = 0; k < 3; ++k) {
      b[k] = INFINITY;
      b[3 + k] = -INFINITY;
      for (int i = 0; i < 4; ++i) {
        const double x = eX[3 * v[i] + k];
        b[k] = std::min(b[k], x);
        b[3 + k] = std::max(b[3 + k], x);
      }
    }
  }
  require_device();
  HOEFEM_CUDA(cudaGetDevice(&E->device));
  HOEFEM_CUDA(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking));
  cudaStream_t s = E->stream;
  E->d_corners.upload(corners, s);
  if (nev) E->d_eX.upload(eX, (size_t)3 * nev, s);
  else E->d_eX.alloc(3);
  E->d_tet_faces.upload(tet_faces, s);
  DBuf<double> d_cbox, d_tbox;
  d_cbox.upload(cbox, s);
  d_tbox.upload(tbox, s);
  // candidate pairs
  DBuf<long long> d_count, d_off;
  d_count.alloc(nbc);
  (note_launch(), k_embed_candidates<<<(unsigned)nbc, 256, 0, s>>>(nbc, d_cbox.p, nt, d_tbox.p, nullptr, d_count.p,
                                                                   nullptr));
  HOEFEM_CUDA(cudaGetLastError());
  std::vector<long long> cnt(nbc);
  HOEFEM_CUDA(cudaMemcpyAsync(cnt.data(), d_count.p, sizeof(long long) * nbc, cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  E->off.assign(nbc + 1, 0);
  for (i64 c = 0; c < nbc; ++c) E->off[c + 1] = E->off[c] + cnt[c];
  E->npairs = E->off[nbc];
  HOEFEM_REQUIRE(E->npairs < (i64)INT32_MAX, HOEFEM_ERR_INVALID_ARGUMENT, "too many (cell, tet) pairs");
  std::vector<long long> offl(E->off.begin(), E->off.end());
  d_off.upload(offl, s);
  E->d_ptet.alloc(E->npairs);
  (note_launch(), k_embed_candidates<<<(unsigned)nbc, 256, 0, s>>>(nbc, d_cbox.p, nt, d_tbox.p, d_off.p, nullptr,
                                                                   E->d_ptet.p));
  std::vector<int> pcell(E->npairs);
  for (i64 c = 0; c < nbc; ++c)
    for (i64 k = E->off[c]; k < E->off[c + 1]; ++k) pcell[k] = (int)c;
  E->d_pcell.upload(pcell, s);
  // pass 1 + classification
  DBuf<double> d_vol, d_cut;
  DBuf<int> d_ntet, d_cls, d_err;
  d_vol.alloc(E->npairs);
  d_ntet.alloc(E->npairs);
  d_cls.alloc(nbc);
  d_cut.alloc(nbc);
  d_err.alloc(1);
  d_err.zero(s);
  if (E->npairs > 0)
    (note_launch(), k_embed_clip_count<<<(unsigned)((E->npairs + 127) / 128), 128, 0, s>>>(
                        E->npairs, E->d_pcell.p, E->d_ptet.p, E->d_corners.p, E->d_eX.p, E->d_tet_faces.p, d_vol.p,
                        d_ntet.p, d_err.p));
  (note_launch(), k_embed_classify<<<(unsigned)((nbc + 127) / 128), 128, 0, s>>>(nbc, d_off.p, d_vol.p, E->d_corners.p,
                                                                               lower, upper, d_cls.p, d_cut.p));
  HOEFEM_CUDA(cudaGetLastError());
  E->cls.resize(nbc);
  E->cut.resize(nbc);
  E->ntet.resize(E->npairs);
  HOEFEM_CUDA(cudaMemcpyAsync(E->cls.data(), d_cls.p, sizeof(int) * nbc, cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaMemcpyAsync(E->cut.data(), d_cut.p, sizeof(double) * nbc, cudaMemcpyDeviceToHost, s));
  if (E->npairs)
    HOEFEM_CUDA(cudaMemcpyAsync(E->ntet.data(), d_ntet.p, sizeof(int) * E->npairs, cudaMemcpyDeviceToHost, s));
  check_err(d_err, s);
  return E.release();
}

void embedding_destroy(Embedding* e) { delete e; }

void embedding_cells(const Embedding& e, i64* ne, i64* ni, i64* nf, int* cls, double* cut) {
  i64 c0 = 0, c1 = 0, c2 = 0;
  for (int c : e.cls) (c == 0 ? c0 : c == 1 ? c1 : c2) += 1;
  if (ne) *ne = c0;
  if (ni) *ni = c1;
  if (nf) *nf = c2;
  if (cls) std::copy(e.cls.begin(), e.cls.end(), cls);
  if (cut) std::copy(e.cut.begin(), e.cut.end(), cut);
}

i64 embedding_quadrature(Embedding& e, const double* tw, const double* tp, i64 nq, double stab_factor,
                         const double* sw, const double* sp, i64 ns) {
  HOEFEM_REQUIRE(nq > 0 && tw && tp, HOEFEM_ERR_INVALID_ARGUMENT, "empty tet quadrature");
  HOEFEM_REQUIRE(ns >= 0 && (ns == 0 || (sw && sp)), HOEFEM_ERR_INVALID_ARGUMENT, "bad stabilization quadrature");
  HOEFEM_CUDA(cudaSetDevice(e.device));
  cudaStream_t s = e.stream;
  // interface cells in cell order; their pairs; offsets
  std::vector<long long> list, qoff, soff;
  e.q_off.assign(1, 0);
  i64 total = 0;
  for (i64 c = 0; c < e.nbc; ++c) {
    if (e.cls[c] != 2) continue;
    for (i64 k = e.off[c]; k < e.off[c + 1]; ++k) {
      if (e.ntet[k] == 0) continue;
      list.push_back(k);
      qoff.push_back(total);
      total += (i64)e.ntet[k] * nq;
    }
    soff.push_back(total);
    total += ns;
    e.q_off.push_back(total);
  }
  const i64 ncell = (i64)e.q_off.size() - 1;
  DBuf<long long> d_list, d_qoff, d_soff;
  DBuf<double> d_tw, d_tp, d_sw, d_sp;
  DBuf<double>& d_w = e.q_w;
  DBuf<double>& d_p = e.q_p;
  DBuf<int> d_err;
  d_list.upload(list, s);
  d_qoff.upload(qoff, s);
  d_soff.upload(soff, s);
  d_tw.upload(tw, nq, s);
  d_tp.upload(tp, 3 * nq, s);
  if (ns) {
    d_sw.upload(sw, ns, s);
    d_sp.upload(sp, 3 * ns, s);
  }
  d_w.alloc(total);
  d_p.alloc(3 * total);
  d_err.alloc(1);
  d_err.zero(s);
  const i64 nl = (i64)list.size();
  if (nl)
    (note_launch(), k_embed_clip_write<<<(unsigned)((nl + 127) / 128), 128, 0, s>>>(
                        nl, d_list.p, e.d_pcell.p, e.d_ptet.p, e.d_corners.p, e.d_eX.p, e.d_tet_faces.p, d_qoff.p,
                        (int)nq, d_tw.p, d_tp.p, d_w.p, d_p.p, d_err.p));
  if (ns && ncell)
    (note_launch(), k_embed_stab<<<(unsigned)((ncell * ns + 255) / 256), 256, 0, s>>>(ncell, d_soff.p, (int)ns,
                                                                                      stab_factor, d_sw.p, d_sp.p,
                                                                                      d_w.p, d_p.p));
  HOEFEM_CUDA(cudaGetLastError());
  check_err(d_err, s);
  e.q_total = total;
  return total;
}

void embedding_copy_quadrature(const Embedding& e, i64* off, double* w, double* p) {
  HOEFEM_REQUIRE(!e.q_off.empty(), HOEFEM_ERR_INVALID_ARGUMENT, "no interface quadrature has been built");
  HOEFEM_CUDA(cudaSetDevice(e.device));
  std::copy(e.q_off.begin(), e.q_off.end(), off);
  if (e.q_total) {
    HOEFEM_CUDA(cudaMemcpyAsync(w, e.q_w.p, sizeof(double) * e.q_total, cudaMemcpyDeviceToHost, e.stream));
    HOEFEM_CUDA(cudaMemcpyAsync(p, e.q_p.p, sizeof(double) * 3 * e.q_total, cudaMemcpyDeviceToHost, e.stream));
  }
  HOEFEM_CUDA(cudaStreamSynchronize(e.stream));
}

int polynomial_space_dim(int strength) {
  int r = 0;
  for (int a = 0; a <= strength; ++a)
    for (int b = 0; b <= strength; ++b)
      for (int c = 0; c <= strength; ++c)
        if (a + b + c <= strength) ++r;
  return r;
}

void quadrature_simplify(i64 nrules, const i64* off, const double* w, const double* p, int strength, i64* out_off,
                         double* out_w, double* out_p) {
  HOEFEM_REQUIRE(strength >= 0 && strength <= 5, HOEFEM_ERR_INVALID_ARGUMENT, "strength must be in [0, 5]");
  HOEFEM_REQUIRE(nrules >= 0 && off && off[0] == 0, HOEFEM_ERR_INVALID_ARGUMENT, "bad rule offsets");
  for (i64 k = 0; k < nrules; ++k)
    HOEFEM_REQUIRE(off[k + 1] >= off[k], HOEFEM_ERR_INVALID_ARGUMENT, "rule offsets must not decrease");
  out_off[0] = 0;
  if (nrules == 0) return;
  require_device();
  const i64 total = off[nrules];
  const int r = polynomial_space_dim(strength);
  cudaStream_t s;
  HOEFEM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{s};
  std::vector<long long> offl(off, off + nrules + 1);
  DBuf<long long> d_off;
  DBuf<double> d_p, d_w;
  DBuf<int> d_keep, d_nkeep, d_err, d_grp, d_gcnt;
  d_off.upload(offl, s);
  d_p.upload(p, 3 * total, s);
  d_w.upload(w, total, s);
  d_keep.alloc(total);
  d_nkeep.alloc(nrules);
  d_grp.alloc(total);
  d_gcnt.alloc(total);
  d_err.alloc(1);
  d_err.zero(s);
  // warps per CTA from the per-warp shared memory (A, z, list, pivots)
  const int m = r + 1, G = 2 * r;
  const size_t per = (size_t)r * m + m + (size_t)(G + m + 1) / 2 + 1;
  const int nw = (int)std::max<size_t>(1, std::min<size_t>(8, (200 * 1024) / (per * sizeof(double))));
  const size_t smem = (size_t)nw * per * sizeof(double);
  HOEFEM_CUDA(cudaFuncSetAttribute(k_simplify, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  (note_launch(), k_simplify<<<(unsigned)nrules, 32 * nw, smem, s>>>(d_off.p, d_p.p, d_w.p, strength, r, d_grp.p,
                                                                      d_gcnt.p, d_keep.p, d_nkeep.p, d_err.p));
  HOEFEM_CUDA(cudaGetLastError());
  std::vector<int> nkeep(nrules);
  HOEFEM_CUDA(cudaMemcpyAsync(nkeep.data(), d_nkeep.p, sizeof(int) * nrules, cudaMemcpyDeviceToHost, s));
  check_err(d_err, s);
  std::vector<long long> oo(nrules + 1, 0);
  for (i64 k = 0; k < nrules; ++k) oo[k + 1] = oo[k] + nkeep[k];
  const i64 kept = oo[nrules];
  DBuf<long long> d_oo;
  DBuf<double> d_ow, d_op;
  d_oo.upload(oo, s);
  d_ow.alloc(kept);
  d_op.alloc(3 * kept);
  (note_launch(), k_simplify_gather<<<(unsigned)nrules, 128, 0, s>>>(d_off.p, d_oo.p, d_keep.p, d_w.p, d_p.p, d_ow.p,
                                                                      d_op.p));
  HOEFEM_CUDA(cudaGetLastError());
  if (kept) {
    HOEFEM_CUDA(cudaMemcpyAsync(out_w, d_ow.p, sizeof(double) * kept, cudaMemcpyDeviceToHost, s));
    HOEFEM_CUDA(cudaMemcpyAsync(out_p, d_op.p, sizeof(double) * 3 * kept, cudaMemcpyDeviceToHost, s));
  }
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  for (i64 k = 0; k <= nrules; ++k) out_off[k] = oo[k];
}

}  // namespace hoefem
