// Element kernels: hyperelastic internal force, tangent stiffness fused with
// the colored CSR scatter, and the consistent mass matrix (FP64).
//
// Reference: fenris/src/assembly.rs:618-797 (element mass / elliptic term /
// stiffness), :252-314 + :1042-1075 (colored CSR scatter), :915-966 (colored
// force scatter); materials in fenris/src/solid/materials.rs.
//
// Layout: connectivity is SoA (conn[I * ne + e]) so that the lanes that own
// the nodes of one element read it with one transaction per node.  Forces:
// one warp per Tet10 element with a lane per quadrature point (affine
// geometry), eight warps per Hex27 element over its points.  Stiffness: 64
// threads per Tet10 element (4 per CTA; the per-point phase one lane per
// point), 384 per Hex27 element.  Per quadrature point the kernel builds the
// per-node vectors a_I = sqrt(w |det J|) J^-T grad N_I, b_I = F a_I and
// c_I = Cof(F) a_I (SNH) or S a_I (StVK); the stiffness block of a node pair
// is then a closed-form rank-structured expression of those vectors (the
// contraction sum_kl C[3k+i,3l+j] a_I[k] a_J[l] of materials.rs:689-743
// evaluated without forming the 9x9 tensor), accumulated in registers over
// the quadrature points.  The element matrix is scattered straight into the
// CSR values with the precomputed element-to-nnz map; colors are launched in
// sequence so no two concurrent elements touch the same node (no atomics,
// and every CSR entry receives its contributions in color order).
#include <cuda_runtime.h>

#include "element_math.cuh"
#include "internal.h"

namespace hoefem {

namespace {

constexpr int TPB = 128;


// ============================================================================
// Internal force: warp per element (nodes <= 32), per-color launch.
// f_e(:, I) += -(P J^-T grad N_I) w |det J|  (assembly.rs:695-708)
// ============================================================================
template <int NN>
__global__ void __launch_bounds__(TPB) k_forces(const BlockDev b, const int* __restrict__ elems, int count,
                                                const double* __restrict__ X, const double* __restrict__ u,
                                                double* __restrict__ f, MatDev mat, int* err,
                                                double* __restrict__ fst = nullptr) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * (TPB / 32) + warp;
  __shared__ double s_corner[TPB / 32][24];
  if (idx >= count) return;
  const int e = elems[idx];
  if (b.scene_active && !b.scene_active[b.escene[e]]) return;
  const bool own = lane < NN;
  int g = own ? b.conn[lane * b.ne + e] : 0;
  double Xl[3] = {0, 0, 0}, ul[3] = {0, 0, 0};
  if (own) {
#pragma unroll
    for (int k = 0; k < 3; ++k) { Xl[k] = X[3 * g + k]; ul[k] = u[3 * g + k]; }
  }
  constexpr int NC = (NN == 10) ? 4 : 8;
  if (lane < NC) {
#pragma unroll
    for (int k = 0; k < 3; ++k) s_corner[warp][3 * lane + k] = Xl[k];
  }
  __syncwarp();
  double J[9], Ji[9], detJ = 0.0;
  if (NN == 10) {
    tet4_jacobian(s_corner[warp], J);
    detJ = inv3(J, Ji);
  }
  double fl[3] = {0, 0, 0};
  int q0, nq;
  quad_rule(b, e, q0, nq);
  bool ok = true;
  for (int q = 0; q < nq; ++q) {
    const double xi[3] = {b.qp[3 * (q0 + q)], b.qp[3 * (q0 + q) + 1], b.qp[3 * (q0 + q) + 2]};
    const double w = b.qw[q0 + q];
    if (NN == 27) {
      hex8_jacobian(s_corner[warp], xi, J);
      detJ = inv3(J, Ji);
    }
    if (detJ == 0.0) { ok = false; break; }
    double gr[3] = {0, 0, 0}, G[3] = {0, 0, 0};
    if (own) {
      if (NN == 10) tet10_grad(lane, xi, gr); else hex27_grad(lane, xi, gr);
      // G = J^-T gr
#pragma unroll
      for (int k = 0; k < 3; ++k) G[k] = Ji[k] * gr[0] + Ji[3 + k] * gr[1] + Ji[6 + k] * gr[2];
    }
    // F(c,k) = delta + sum_I u_I[c] G_I[k]
    double F[9];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < 3; ++k) F[3 * c + k] = warp_sum(ul[c] * G[k]) + (c == k ? 1.0 : 0.0);
    QpState<double> st;
    const double emu = b.emat ? b.emat[2 * e] : mat.mu, elam = b.emat ? b.emat[2 * e + 1] : mat.lambda;
    if (!material_state(mat.kind, F, emu, elam, st, true)) { ok = false; break; }
    if (own) {
      double sc = w * fabs(detJ);
#pragma unroll
      for (int i = 0; i < 3; ++i)
        fl[i] += -(st.P[3 * i] * G[0] + st.P[3 * i + 1] * G[1] + st.P[3 * i + 2] * G[2]) * sc;
    }
  }
  if (!ok) {
    if (lane == 0) set_error(err, HOEFEM_ERR_SINGULAR);
    return;
  }
  if (own) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (fst) fst[((size_t)e * NN + lane) * 3 + i] = fl[i];
      else f[3 * g + i] += fl[i];
    }
  }
}

// ============================================================================
// Internal force, Tet10 (affine geometry, uniform rule of <= 32 points): warp
// per element, lane q evaluates quadrature point q (F from all 10 nodes, the
// stress once) and writes its contribution to every node into shared memory;
// the node lanes then add the points' contributions in point order, as the
// sequential loop of the reference does.
// ============================================================================
constexpr int T10_FSTRIDE = 31;  // doubles per point row (30 used; odd stride)

__global__ void __launch_bounds__(TPB) k_forces_tet10(const BlockDev b, const int* __restrict__ elems, int count,
                                                      const double* __restrict__ X, const double* __restrict__ u,
                                                      double* __restrict__ f, MatDev mat, int* err,
                                                      double* __restrict__ fst = nullptr) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * (TPB / 32) + warp;
  __shared__ double s_corner[TPB / 32][12];
  __shared__ double s_u[TPB / 32][30];
  __shared__ double s_f[TPB / 32][32 * T10_FSTRIDE];
  if (idx >= count) return;
  const int e = elems[idx];
  if (b.scene_active && !b.scene_active[b.escene[e]]) return;
  int g = 0;
  if (lane < 10) {
    g = b.conn[lane * b.ne + e];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double x = X[3 * g + k];
      s_u[warp][3 * lane + k] = u[3 * g + k];
      if (lane < 4) s_corner[warp][3 * lane + k] = x;
    }
  }
  __syncwarp();
  double J[9], Ji[9];
  tet4_jacobian(s_corner[warp], J);
  const double detJ = inv3(J, Ji);
  const int nq = b.nq;
  bool ok = detJ != 0.0;
  if (ok && lane < nq) {
    const double xi[3] = {b.qp[3 * lane], b.qp[3 * lane + 1], b.qp[3 * lane + 2]};
    double F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int I = 0; I < 10; ++I) {
      double gr[3], G[3];
      tet10_grad(I, xi, gr);
#pragma unroll
      for (int k = 0; k < 3; ++k) G[k] = Ji[k] * gr[0] + Ji[3 + k] * gr[1] + Ji[6 + k] * gr[2];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 3; ++k) F[3 * c + k] += s_u[warp][3 * I + c] * G[k];
    }
    F[0] += 1.0;
    F[4] += 1.0;
    F[8] += 1.0;
    QpState<double> st;
    const double emu = b.emat ? b.emat[2 * e] : mat.mu, elam = b.emat ? b.emat[2 * e + 1] : mat.lambda;
    ok = material_state(mat.kind, F, emu, elam, st, true);
    if (ok) {
      const double sc = b.qw[lane] * fabs(detJ);
      double* out = s_f[warp] + lane * T10_FSTRIDE;
#pragma unroll
      for (int I = 0; I < 10; ++I) {
        double gr[3], G[3];
        tet10_grad(I, xi, gr);
#pragma unroll
        for (int k = 0; k < 3; ++k) G[k] = Ji[k] * gr[0] + Ji[3 + k] * gr[1] + Ji[6 + k] * gr[2];
#pragma unroll
        for (int i = 0; i < 3; ++i)
          out[3 * I + i] = -(st.P[3 * i] * G[0] + st.P[3 * i + 1] * G[1] + st.P[3 * i + 2] * G[2]) * sc;
      }
    }
  }
  ok = __all_sync(0xffffffffu, ok);
  __syncwarp();
  if (!ok) {
    if (lane == 0) set_error(err, HOEFEM_ERR_SINGULAR);
    return;
  }
  if (lane < 10) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double acc = 0.0;
      for (int q = 0; q < nq; ++q) acc += s_f[warp][q * T10_FSTRIDE + 3 * lane + i];
      if (fst) fst[((size_t)e * 10 + lane) * 3 + i] = acc;
      else f[3 * g + i] += acc;
    }
  }
}

// ============================================================================
// Internal force, Hex27: FW warps per element (one CTA), warp w takes the
// quadrature points w, w + FW, ...; the per-warp node forces are summed in
// shared memory in warp order (deterministic) and scattered once.  A color
// of a few hundred elements then fills the GPU with FW times more warps.
// ============================================================================
constexpr int FW = 8;

__global__ void __launch_bounds__(32 * FW, 2) k_forces_hex27(const BlockDev b, const int* __restrict__ elems, int count,
                                                         const double* __restrict__ X, const double* __restrict__ u,
                                                         double* __restrict__ f, MatDev mat, int* err,
                                                         double* __restrict__ fst = nullptr) {
  constexpr int NN = 27;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ double s_corner[24];
  __shared__ double s_f[FW][NN][3];
  __shared__ int s_ok;
  const int e = elems[blockIdx.x];
  if (b.scene_active && !b.scene_active[b.escene[e]]) return;  // uniform over the CTA
  const bool own = lane < NN;
  const int g = own ? b.conn[lane * b.ne + e] : 0;
  double ul[3] = {0, 0, 0};
  if (own) {
#pragma unroll
    for (int k = 0; k < 3; ++k) ul[k] = u[3 * g + k];
    if (warp == 0 && lane < 8) {
#pragma unroll
      for (int k = 0; k < 3; ++k) s_corner[3 * lane + k] = X[3 * g + k];
    }
  }
  if (threadIdx.x == 0) s_ok = 1;
  __syncthreads();
  int q0, nq;
  quad_rule(b, e, q0, nq);
  const double emu = b.emat ? b.emat[2 * e] : mat.mu, elam = b.emat ? b.emat[2 * e + 1] : mat.lambda;
  double fl[3] = {0, 0, 0};
  for (int q = warp; q < nq; q += FW) {
    const double xi[3] = {b.qp[3 * (q0 + q)], b.qp[3 * (q0 + q) + 1], b.qp[3 * (q0 + q) + 2]};
    const double w = b.qw[q0 + q];
    double J[9], Ji[9];
    hex8_jacobian(s_corner, xi, J);
    const double detJ = inv3(J, Ji);
    double gr[3] = {0, 0, 0}, G[3] = {0, 0, 0};
    if (own) {
      hex27_grad(lane, xi, gr);
#pragma unroll
      for (int k = 0; k < 3; ++k) G[k] = Ji[k] * gr[0] + Ji[3 + k] * gr[1] + Ji[6 + k] * gr[2];
    }
    double F[9];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < 3; ++k) F[3 * c + k] = warp_sum(ul[c] * G[k]) + (c == k ? 1.0 : 0.0);
    QpState<double> st;
    if (detJ == 0.0 || !material_state(mat.kind, F, emu, elam, st, true)) {
      if (lane == 0) s_ok = 0;
      break;
    }
    if (own) {
      const double sc = w * fabs(detJ);
#pragma unroll
      for (int i = 0; i < 3; ++i)
        fl[i] += -(st.P[3 * i] * G[0] + st.P[3 * i + 1] * G[1] + st.P[3 * i + 2] * G[2]) * sc;
    }
  }
  if (own) {
#pragma unroll
    for (int i = 0; i < 3; ++i) s_f[warp][lane][i] = fl[i];
  }
  __syncthreads();
  if (!s_ok) {
    if (threadIdx.x == 0) set_error(err, HOEFEM_ERR_SINGULAR);
    return;
  }
  if (threadIdx.x < 3 * NN) {
    const int I = threadIdx.x / 3, i = threadIdx.x % 3;
    double acc = 0.0;
#pragma unroll
    for (int w = 0; w < FW; ++w) acc += s_f[w][I][i];
    if (fst) {
      fst[((size_t)e * NN + I) * 3 + i] = acc;
    } else {
      const int gI = b.conn[I * b.ne + e];
      f[3 * gI + i] += acc;
    }
  }
}

// ============================================================================
// Stiffness + scatter.  TPE threads (TPE / 32 warps) own one element, EPC
// elements per CTA.  The quadrature points are processed in tiles of QT:
//  phase A: warp w of the element takes points w, w + TPE/32, ... of the
//    tile; its lanes (one per node) build J, grad N, F (warp sums), the
//    material state and the per-node vectors a, F a, M1 a into shared memory;
//  phase B: every thread accumulates its node pair(s) over the tile's points
//    from shared memory, with no barrier between points.
// Two barriers per tile (one tile for all standard rules), against two per
// point with a single node-building warp.
// ============================================================================
template <int NN>
struct PairTable {
  static constexpr int NP = NN * (NN + 1) / 2;
};
__constant__ unsigned char c_pairs10[55][2];
__constant__ unsigned char c_pairs27[378][2];

template <int NN>
__device__ __forceinline__ void pair_of(int p, int& I, int& J) {
  if (NN == 10) { I = c_pairs10[p][0]; J = c_pairs10[p][1]; }
  else { I = c_pairs27[p][0]; J = c_pairs27[p][1]; }
}

template <int NN>
struct StiffCfg {
  static constexpr int TPE = NN == 10 ? 64 : 384;  // threads per element
  static constexpr int EPC = NN == 10 ? 4 : 1;     // elements per CTA
  static constexpr int QT = NN == 10 ? 14 : 27;    // quadrature points per tile
  static constexpr int TPB = TPE * EPC;
};

template <int NN, class R>
constexpr size_t stiffness_smem() {
  using C = StiffCfg<NN>;
  return sizeof(R) * (size_t)C::EPC * C::QT * NN * 9 + sizeof(QpPair<R>) * (size_t)C::EPC * C::QT;
}

template <int NN, class R>
__global__ void __launch_bounds__(StiffCfg<NN>::TPB, 2) k_stiffness(const BlockDev b, const int* __restrict__ elems,
                                                                    int count, const double* __restrict__ X,
                                                                    const double* __restrict__ u,
                                                                    const int* __restrict__ adj_off,
                                                                    const long long* __restrict__ base,
                                                                    double* __restrict__ vals, MatDev mat, int* err,
                                                                    double* __restrict__ stage,
                                                                    R* __restrict__ pblk = nullptr) {
  using C = StiffCfg<NN>;
  constexpr int TPE = C::TPE, EPC = C::EPC, QT = C::QT, WPE = TPE / 32;
  constexpr int NP = PairTable<NN>::NP;
  constexpr int PPT = (NP + TPE - 1) / TPE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R(*s_vec)[QT][NN][9] = reinterpret_cast<R(*)[QT][NN][9]>(smem_raw);
  QpPair<R>(*s_qp)[QT] =
      reinterpret_cast<QpPair<R>(*)[QT]>(smem_raw + sizeof(R) * (size_t)EPC * QT * NN * 9);
  __shared__ R s_corner[EPC][24];
  __shared__ R s_u[EPC][NN == 10 ? 30 : 1];  // Tet10: node displacements for the point lanes
  __shared__ int s_g[EPC][NN];
  __shared__ int s_ok[EPC];
  __shared__ int s_nq[EPC];
  const int grp = threadIdx.x / TPE, t = threadIdx.x % TPE;
  const int lane = threadIdx.x & 31, wl = t >> 5;
  const int idx = blockIdx.x * EPC + grp;
  const int e = idx < count ? elems[idx] : 0;
  const bool active = idx < count && (!b.scene_active || b.scene_active[b.escene[e]]);
  if (active && t < NN) {
    const int g = b.conn[t * b.ne + e];
    s_g[grp][t] = g;
    constexpr int NC = (NN == 10) ? 4 : 8;
    if (t < NC) {
#pragma unroll
      for (int k = 0; k < 3; ++k) s_corner[grp][3 * t + k] = (R)X[3 * g + k];
    }
  }
  int q0 = 0, nq = 0;
  if (active) quad_rule(b, e, q0, nq);
  if (t == 0) {
    s_ok[grp] = 1;
    s_nq[grp] = nq;
  }
  __syncthreads();
  int nq_max = 0;
#pragma unroll
  for (int k = 0; k < EPC; ++k) nq_max = max(nq_max, s_nq[k]);
  const R mu = (R)(b.emat ? b.emat[2 * e] : mat.mu), lam = (R)(b.emat ? b.emat[2 * e + 1] : mat.lambda);
  // the lane's node data, kept in registers across tiles
  const bool own = active && lane < NN;
  R ul[3] = {0, 0, 0};
  if (own) {
    const int g = s_g[grp][lane];
#pragma unroll
    for (int k = 0; k < 3; ++k) ul[k] = (R)u[3 * g + k];
    if constexpr (NN == 10) {
      if (wl == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k) s_u[grp][3 * lane + k] = ul[k];
    }
  }
  if constexpr (NN == 10) __syncthreads();
  R acc[PPT][9];
#pragma unroll
  for (int k = 0; k < PPT; ++k)
#pragma unroll
    for (int m = 0; m < 9; ++m) acc[k][m] = 0;
  for (int qt = 0; qt < nq_max; qt += QT) {
    // ---- phase A: per-point data of this tile ----
    if constexpr (NN == 10) {
      // affine geometry: lane ql of the element's first warp takes point ql
      // (the material state once per point, F from all 10 nodes)
      const int ql = lane;
      if (wl == 0 && ql < QT && qt + ql < nq) {
        const int q = q0 + qt + ql;
        const R xi[3] = {(R)b.qp[3 * q], (R)b.qp[3 * q + 1], (R)b.qp[3 * q + 2]};
        const R w = (R)b.qw[q];
        R J[9], Ji[9];
        tet4_jacobian(s_corner[grp], J);
        const R detJ = inv3(J, Ji);
        R F[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int I = 0; I < 10; ++I) {
          R gr[3], G[3];
          tet10_grad(I, xi, gr);
#pragma unroll
          for (int k = 0; k < 3; ++k) G[k] = Ji[k] * gr[0] + Ji[3 + k] * gr[1] + Ji[6 + k] * gr[2];
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 3; ++k) F[3 * c + k] += s_u[grp][3 * I + c] * G[k];
        }
        F[0] += R(1);
        F[4] += R(1);
        F[8] += R(1);
        QpState<R> st;
        const bool okq = (detJ != R(0)) && material_state(mat.kind, F, mu, lam, st, false);
        if (!okq) {
          s_ok[grp] = 0;
        } else {
          const R sc = sqrt(w * fabs(detJ));
#pragma unroll
          for (int I = 0; I < 10; ++I) {
            R gr[3];
            tet10_grad(I, xi, gr);
            const R a[3] = {(Ji[0] * gr[0] + Ji[3] * gr[1] + Ji[6] * gr[2]) * sc,
                            (Ji[1] * gr[0] + Ji[4] * gr[1] + Ji[7] * gr[2]) * sc,
                            (Ji[2] * gr[0] + Ji[5] * gr[1] + Ji[8] * gr[2]) * sc};
            R* v = s_vec[grp][ql][I];
            v[0] = a[0]; v[1] = a[1]; v[2] = a[2];
            mat3vec(st.F, a, v + 3);
            mat3vec(st.M1, a, v + 6);
          }
          qp_pair_from(mat.kind, st, s_qp[grp][ql]);
        }
      }
    } else
    for (int ql = wl; ql < QT && qt + ql < nq; ql += WPE) {
      const int q = q0 + qt + ql;
      const R xi[3] = {(R)b.qp[3 * q], (R)b.qp[3 * q + 1], (R)b.qp[3 * q + 2]};
      const R w = (R)b.qw[q];
      R J[9], Ji[9];
      if (NN == 10) tet4_jacobian(s_corner[grp], J);
      else hex8_jacobian(s_corner[grp], xi, J);
      const R detJ = inv3(J, Ji);
      R gr[3] = {0, 0, 0}, G[3] = {0, 0, 0};
      if (lane < NN) {
        if (NN == 10) tet10_grad(lane, xi, gr); else hex27_grad(lane, xi, gr);
#pragma unroll
        for (int k = 0; k < 3; ++k) G[k] = Ji[k] * gr[0] + Ji[3 + k] * gr[1] + Ji[6 + k] * gr[2];
      }
      R F[9];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 3; ++k) F[3 * c + k] = warp_sum(ul[c] * G[k]) + (c == k ? R(1) : R(0));
      QpState<R> st;
      const bool okq = (detJ != R(0)) && material_state(mat.kind, F, mu, lam, st, false);
      if (!okq) {
        if (lane == 0) s_ok[grp] = 0;
      } else {
        if (lane < NN) {
          const R sc = sqrt(w * fabs(detJ));
          const R a[3] = {G[0] * sc, G[1] * sc, G[2] * sc};
          R* v = s_vec[grp][ql][lane];
          v[0] = a[0]; v[1] = a[1]; v[2] = a[2];
          mat3vec(st.F, a, v + 3);
          mat3vec(st.M1, a, v + 6);
        }
        if (lane == 0) qp_pair_from(mat.kind, st, s_qp[grp][ql]);
      }
    }
    __syncthreads();
    // ---- phase B: node pairs over the tile's points ----
    const int nql = min(QT, nq - qt);
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      const int p = t + k * TPE;
      if (p < NP && active) {
        int I, Jn;
        pair_of<NN>(p, I, Jn);
        for (int ql = 0; ql < nql; ++ql) pair_block(mat.kind, s_qp[grp][ql], s_vec[grp][ql][I], s_vec[grp][ql][Jn], acc[k]);
      }
    }
    __syncthreads();
  }
  if (!active) return;
  if (!s_ok[grp]) {
    if (t == 0) set_error(err, HOEFEM_ERR_SINGULAR);
    return;
  }
  if (pblk) {
    // the element's node-pair blocks, pblk[(e NP + p) 9 + 3 i + j], for the
    // gather into the CSR values
    R* o = pblk + (size_t)e * NP * 9;
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      const int p = t + k * TPE;
      if (p < NP) {
#pragma unroll
        for (int ab = 0; ab < 9; ++ab) o[(size_t)p * 9 + ab] = acc[k][ab];
      }
    }
    return;
  }
  if (stage) {
    // dense element matrix (row-major 3NN x 3NN) instead of the scatter
    constexpr int D = 3 * NN;
    double* ke = stage + (size_t)e * D * D;
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      int p = t + k * TPE;
      if (p < NP) {
        int I, Jn;
        pair_of<NN>(p, I, Jn);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            ke[(3 * I + i) * D + 3 * Jn + j] = (double)acc[k][3 * i + j];
            if (I != Jn) ke[(3 * Jn + j) * D + 3 * I + i] = (double)acc[k][3 * i + j];
          }
      }
    }
    return;
  }
  const int* em = b.emap + (size_t)e * NN * NN;
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    int p = t + k * TPE;
    if (p < NP) {
      int I, Jn;
      pair_of<NN>(p, I, Jn);
      int gI = s_g[grp][I], gJ = s_g[grp][Jn];
      int rlI = 3 * (adj_off[gI + 1] - adj_off[gI]);
      long long bIJ = base[gI] + em[I * NN + Jn];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) vals[bIJ + i * rlI + j] += (double)acc[k][3 * i + j];
      if (I != Jn) {
        int rlJ = 3 * (adj_off[gJ + 1] - adj_off[gJ]);
        long long bJI = base[gJ] + em[Jn * NN + I];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) vals[bJI + j * rlJ + i] += (double)acc[k][3 * i + j];
      }
    }
  }
}

// ============================================================================
// Mass: warp per element, scalar mass m_IJ = sum rho |det J| w phi_I phi_J
// replicated on the three components (assembly.rs:624-671).
// ============================================================================
template <int NN>
__global__ void __launch_bounds__(TPB) k_mass(const BlockDev b, const int* __restrict__ elems, int count,
                                              const double* __restrict__ X, const int* __restrict__ adj_off,
                                              const long long* __restrict__ nbase, double* __restrict__ vals,
                                              double density, int* err) {
  constexpr int NE = NN * NN;
  constexpr int EPT = (NE + 31) / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * (TPB / 32) + warp;
  __shared__ double s_corner[TPB / 32][24];
  __shared__ double s_phi[TPB / 32][32];
  __shared__ int s_g[TPB / 32][32];
  if (idx >= count) return;
  const int e = elems[idx];
  int g = lane < NN ? b.conn[lane * b.ne + e] : 0;
  s_g[warp][lane] = g;
  constexpr int NC = (NN == 10) ? 4 : 8;
  if (lane < NC)
    for (int k = 0; k < 3; ++k) s_corner[warp][3 * lane + k] = X[3 * g + k];
  __syncwarp();
  double acc[EPT];
#pragma unroll
  for (int k = 0; k < EPT; ++k) acc[k] = 0.0;
  double J[9];
  int q0, nq;
  quad_rule(b, e, q0, nq);
  for (int q = 0; q < nq; ++q) {
    const double xi[3] = {b.qp[3 * (q0 + q)], b.qp[3 * (q0 + q) + 1], b.qp[3 * (q0 + q) + 2]};
    const double w = b.qw[q0 + q];
    if (NN == 10) tet4_jacobian(s_corner[warp], J); else hex8_jacobian(s_corner[warp], xi, J);
    double dJ = det3(J);
    if (lane < NN) s_phi[warp][lane] = (NN == 10) ? tet10_phi(lane, xi) : hex27_phi(lane, xi);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < EPT; ++k) {
      int p = lane + 32 * k;
      if (p < NE) {
        int I = p / NN, Jn = p % NN;
        acc[k] += density * fabs(dJ) * w * s_phi[warp][I] * s_phi[warp][Jn];
      }
    }
    __syncwarp();
  }
  const int* em = b.emap + (size_t)e * NE;
#pragma unroll
  for (int k = 0; k < EPT; ++k) {
    int p = lane + 32 * k;
    if (p < NE) {
      int I = p / NN, Jn = p % NN;
      int gI = s_g[warp][I];
      int rl = 3 * (adj_off[gI + 1] - adj_off[gI]);
      long long base = nbase[gI] + em[p];
#pragma unroll
      for (int c = 0; c < 3; ++c) vals[base + c * rl + c] += acc[k];
    }
  }
  (void)err;
}

bool g_pairs_ready = false;
void init_pairs() {
  if (g_pairs_ready) return;
  unsigned char p10[55][2], p27[378][2];
  int k = 0;
  for (int J = 0; J < 10; ++J)
    for (int I = J; I < 10; ++I) { p10[k][0] = (unsigned char)I; p10[k][1] = (unsigned char)J; ++k; }
  k = 0;
  for (int J = 0; J < 27; ++J)
    for (int I = J; I < 27; ++I) { p27[k][0] = (unsigned char)I; p27[k][1] = (unsigned char)J; ++k; }
  HOEFEM_CUDA(cudaMemcpyToSymbol(c_pairs10, p10, sizeof(p10)));
  HOEFEM_CUDA(cudaMemcpyToSymbol(c_pairs27, p27, sizeof(p27)));
  g_pairs_ready = true;
}

template <class F>
void for_each_color(const Block& blk, F&& fn) {
  const int nc = (int)blk.color_off.size() - 1;
  for (int c = 0; c < nc; ++c) {
    int begin = (int)blk.color_off[c];
    int cnt = (int)(blk.color_off[c + 1] - begin);
    if (cnt > 0) fn(blk.d_color_elems.p + begin, cnt);
  }
}

}  // namespace

void launch_forces(const Model& m, const MatDev& mat, const double* u, double* f, cudaStream_t s) {
  for (const Block* bp : m.blocks) {
    BlockDev bd = bp->dev();
    auto launch = [&](const int* elems, int cnt, double* fst) {
      int grid = (cnt + TPB / 32 - 1) / (TPB / 32);
      if (bp->kind == HOEFEM_ELEM_TET10 && bd.uniform && bd.nq <= 32)
        (note_launch(), k_forces_tet10<<<grid, TPB, 0, s>>>(bd, elems, cnt, m.d_X.p, u, f, mat, m.d_err.p, fst));
      else if (bp->kind == HOEFEM_ELEM_TET10)
        (note_launch(), k_forces<10><<<grid, TPB, 0, s>>>(bd, elems, cnt, m.d_X.p, u, f, mat, m.d_err.p, fst));
      else
        (note_launch(), k_forces_hex27<<<cnt, 32 * FW, 0, s>>>(bd, elems, cnt, m.d_X.p, u, f, mat, m.d_err.p, fst));
    };
    if (stiffness_pairs_eligible(m, *bp)) {
      // every element in one launch into per-element node forces, then the
      // per-node gather (element order)
      double* fst = forces_stage_buffer(m, *bp, s);
      if (bp->ne > 0) launch(bp->d_color_elems.p, (int)bp->ne, fst);
      HOEFEM_CUDA(cudaGetLastError());
      forces_gather(m, *bp, f, s);
    } else {
      for_each_color(*bp, [&](const int* elems, int cnt) { launch(elems, cnt, nullptr); });
    }
  }
  HOEFEM_CUDA(cudaGetLastError());
}

template <int NN, class R>
void launch_stiffness_kind(const Model& m, const Block& blk, const MatDev& mat, const double* u, double* vals,
                           cudaStream_t s, double* stage = nullptr, R* pblk = nullptr) {
  using C = StiffCfg<NN>;
  constexpr size_t smem = stiffness_smem<NN, R>();
  static bool attr_set[64] = {};
  int dev = 0;
  HOEFEM_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    HOEFEM_CUDA(cudaFuncSetAttribute(k_stiffness<NN, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set[dev] = true;
  }
  BlockDev bd = blk.dev();
  if (stage || pblk) {
    // all elements at once (no scatter, no coloring needed)
    const int cnt = (int)blk.ne;
    if (cnt > 0)
      (note_launch(), k_stiffness<NN, R><<<(cnt + C::EPC - 1) / C::EPC, C::TPB, smem, s>>>(
                          bd, blk.d_color_elems.p, cnt, m.d_X.p, u, m.d_adj_off.p, m.d_base.p, vals, mat, m.d_err.p,
                          stage, pblk));
    return;
  }
  for_each_color(blk, [&](const int* elems, int cnt) {
    const int grid = (cnt + C::EPC - 1) / C::EPC;
    (note_launch(), k_stiffness<NN, R><<<grid, C::TPB, smem, s>>>(bd, elems, cnt, m.d_X.p, u, m.d_adj_off.p,
                                                                   m.d_base.p, vals, mat, m.d_err.p, nullptr));
  });
}

// Dense FP64 element matrices of one block into stage (element e at
// e * (3 nn)^2), no scatter.
void launch_stiffness_staged(const Model& m, const Block& blk, const MatDev& mat, const double* u, double* stage,
                             cudaStream_t s) {
  init_pairs();
  if (blk.kind == HOEFEM_ELEM_TET10) launch_stiffness_kind<10, double>(m, blk, mat, u, nullptr, s, stage);
  else launch_stiffness_kind<27, double>(m, blk, mat, u, nullptr, s, stage);
  HOEFEM_CUDA(cudaGetLastError());
}

void launch_stiffness(const Model& m, const MatDev& mat, const double* u, double* vals, cudaStream_t s,
                      int precision, bool assign) {
  init_pairs();
  const bool f32 = precision == PRECISION_FP32;
  // a single block whose gather writes every entry stores instead of adding
  const bool one = m.blocks.size() == 1;
  const bool gathered = one && ((f32 && stiffness_tc_eligible(m, *m.blocks[0])) || stiffness_pairs_eligible(m, *m.blocks[0]));
  if (assign && !gathered) HOEFEM_CUDA(cudaMemsetAsync(vals, 0, sizeof(double) * (size_t)m.nnz, s));
  const bool store = assign && gathered;
  for (const Block* bp : m.blocks) {
    if (f32 && stiffness_tc_eligible(m, *bp)) {
      launch_stiffness_tc(m, *bp, mat, u, vals, s, store);
      continue;
    }
    if (stiffness_pairs_eligible(m, *bp)) {
      // every element of the block in one launch, node-pair blocks staged,
      // then the gather into the CSR values
      void* pb = stiffness_pair_buffer(m, *bp, f32, s);
      if (bp->kind == HOEFEM_ELEM_TET10) {
        if (f32) launch_stiffness_kind<10, float>(m, *bp, mat, u, nullptr, s, nullptr, (float*)pb);
        else launch_stiffness_kind<10, double>(m, *bp, mat, u, nullptr, s, nullptr, (double*)pb);
      } else {
        if (f32) launch_stiffness_kind<27, float>(m, *bp, mat, u, nullptr, s, nullptr, (float*)pb);
        else launch_stiffness_kind<27, double>(m, *bp, mat, u, nullptr, s, nullptr, (double*)pb);
      }
      HOEFEM_CUDA(cudaGetLastError());
      stiffness_gather_pairs(m, *bp, f32, vals, store, s);
      continue;
    }
    if (bp->kind == HOEFEM_ELEM_TET10) {
      if (f32) launch_stiffness_kind<10, float>(m, *bp, mat, u, vals, s);
      else launch_stiffness_kind<10, double>(m, *bp, mat, u, vals, s);
    } else {
      if (f32) launch_stiffness_kind<27, float>(m, *bp, mat, u, vals, s);
      else launch_stiffness_kind<27, double>(m, *bp, mat, u, vals, s);
    }
  }
  HOEFEM_CUDA(cudaGetLastError());
}

void launch_mass(const Model& m, double density, double* vals, cudaStream_t s) {
  for (const Block* bp : m.blocks) {
    BlockDev bd = bp->dev();
    for_each_color(*bp, [&](const int* elems, int cnt) {
      int grid = (cnt + TPB / 32 - 1) / (TPB / 32);
      if (bp->kind == HOEFEM_ELEM_TET10)
        (note_launch(), k_mass<10><<<grid, TPB, 0, s>>>(bd, elems, cnt, m.d_X.p, m.d_adj_off.p, m.d_base.p, vals, density,
                                                         m.d_err.p));
      else
        (note_launch(), k_mass<27><<<grid, TPB, 0, s>>>(bd, elems, cnt, m.d_X.p, m.d_adj_off.p, m.d_base.p, vals, density,
                                                         m.d_err.p));
    });
  }
  HOEFEM_CUDA(cudaGetLastError());
}

}  // namespace hoefem
