// Device math shared by the element kernels: reference Tet10 / Hex27 shape
// function gradients, the Hex8 / Tet4 geometry Jacobians, the materials
// (stable Neo-Hookean, St. Venant-Kirchhoff) and the node-pair stiffness
// block of one quadrature point.
//
// Reference: fenris/src/element.rs (Tet10 1921-1947, Hex27 basis),
// fenris/src/solid/materials.rs (stress and its contraction 689-743).
#pragma once

#include <cuda_runtime.h>

#include "internal.h"

namespace hoefem {
namespace {

__constant__ signed char c_hex27_alpha[27][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
    {0, -1, -1},  {-1, 0, -1}, {-1, -1, 0}, {1, 0, -1}, {1, -1, 0}, {0, 1, -1}, {1, 1, 0}, {-1, 1, 0},
    {0, -1, 1},   {-1, 0, 1},  {1, 0, 1},   {0, 1, 1},  {0, 0, -1}, {0, -1, 0}, {-1, 0, 0}, {1, 0, 0},
    {0, 1, 0},    {0, 0, 1},   {0, 0, 0}};
__constant__ signed char c_tet10_edge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {2, 3}, {1, 3}};

template <class R>
__device__ __forceinline__ R warp_sum(R v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void set_error(int* err, int code) { atomicCAS(err, 0, code); }

// ---- reference elements ----------------------------------------------------
template <class R>
__device__ __forceinline__ void tet4_psi(const R* xi, R* p) {
  p[0] = -R(0.5) * xi[0] - R(0.5) * xi[1] - R(0.5) * xi[2] - R(0.5);
  p[1] = R(0.5) * xi[0] + R(0.5);
  p[2] = R(0.5) * xi[1] + R(0.5);
  p[3] = R(0.5) * xi[2] + R(0.5);
}
// gradient of Tet4 basis function I (constant): column I of [[-.5,.5,0,0],[-.5,0,.5,0],[-.5,0,0,.5]]
template <class R>
__device__ __forceinline__ void tet4_g(int I, R* g) {
  g[0] = (I == 0) ? -R(0.5) : (I == 1 ? R(0.5) : R(0.0));
  g[1] = (I == 0) ? -R(0.5) : (I == 2 ? R(0.5) : R(0.0));
  g[2] = (I == 0) ? -R(0.5) : (I == 3 ? R(0.5) : R(0.0));
}
// Tet10 reference gradient of node I (element.rs:1921-1947)
template <class R>
__device__ __forceinline__ void tet10_grad(int I, const R* xi, R* g) {
  R p[4];
  tet4_psi(xi, p);
  if (I < 4) {
    R gi[3];
    tet4_g(I, gi);
    R f = R(4.0) * p[I] - R(1.0);
    g[0] = gi[0] * f; g[1] = gi[1] * f; g[2] = gi[2] * f;
  } else {
    int a = c_tet10_edge[I - 4][0], b = c_tet10_edge[I - 4][1];
    R ga[3], gb[3];
    tet4_g(a, ga);
    tet4_g(b, gb);
    R fb = R(4.0) * p[b], fa = R(4.0) * p[a];
    g[0] = ga[0] * fb + gb[0] * fa;
    g[1] = ga[1] * fb + gb[1] * fa;
    g[2] = ga[2] * fb + gb[2] * fa;
  }
}
template <class R>
__device__ __forceinline__ R tet10_phi(int I, const R* xi) {
  R p[4];
  tet4_psi(xi, p);
  if (I < 4) return p[I] * (R(2.0) * p[I] - R(1.0));
  return R(4.0) * p[c_tet10_edge[I - 4][0]] * p[c_tet10_edge[I - 4][1]];
}
template <class R>
__device__ __forceinline__ R phi_q(R a, R x) {
  R a2 = a * a, x2 = x * x;
  return (R(3.0) / R(2.0) * a2 - R(1.0)) * x2 + R(0.5) * a * x + R(1.0) - a2;
}
template <class R>
__device__ __forceinline__ R dphi_q(R a, R x) {
  R a2 = a * a;
  return R(2.0) * (R(3.0) / R(2.0) * a2 - R(1.0)) * x + R(0.5) * a;
}
template <class R>
__device__ __forceinline__ void hex27_grad(int I, const R* xi, R* g) {
  R a0 = c_hex27_alpha[I][0], a1 = c_hex27_alpha[I][1], a2 = c_hex27_alpha[I][2];
  R p0 = phi_q(a0, xi[0]), p1 = phi_q(a1, xi[1]), p2 = phi_q(a2, xi[2]);
  g[0] = dphi_q(a0, xi[0]) * p1 * p2;
  g[1] = p0 * dphi_q(a1, xi[1]) * p2;
  g[2] = p0 * p1 * dphi_q(a2, xi[2]);
}
template <class R>
__device__ __forceinline__ R hex27_phi(int I, const R* xi) {
  return phi_q((R)c_hex27_alpha[I][0], xi[0]) * phi_q((R)c_hex27_alpha[I][1], xi[1]) *
         phi_q((R)c_hex27_alpha[I][2], xi[2]);
}
// Jacobian of the trilinear Hex8 geometry from the 8 corners (smem, xyz per corner).
template <class R>
__device__ __forceinline__ void hex8_jacobian(const R* Xc, const R* xi, R* J) {
#pragma unroll
  for (int k = 0; k < 9; ++k) J[k] = R(0.0);
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    R a0 = c_hex27_alpha[c][0], a1 = c_hex27_alpha[c][1], a2 = c_hex27_alpha[c][2];
    R l0 = (R(1.0) + a0 * xi[0]) / R(2.0), l1 = (R(1.0) + a1 * xi[1]) / R(2.0), l2 = (R(1.0) + a2 * xi[2]) / R(2.0);
    R g0 = a0 / R(2.0) * l1 * l2, g1 = l0 * a1 / R(2.0) * l2, g2 = l0 * l1 * a2 / R(2.0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      R x = Xc[3 * c + i];
      J[3 * i + 0] += x * g0;
      J[3 * i + 1] += x * g1;
      J[3 * i + 2] += x * g2;
    }
  }
}
// Jacobian of the affine Tet4 geometry: J(:,j) = R(0.5) (X_{j+1} - X_0)
template <class R>
__device__ __forceinline__ void tet4_jacobian(const R* Xc, R* J) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) J[3 * i + j] = -R(0.5) * Xc[i] + R(0.5) * Xc[3 * (j + 1) + i];
}

template <class R>
__device__ __forceinline__ R det3(const R* m) {
  return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[1] * (m[3] * m[8] - m[6] * m[5]) + m[2] * (m[3] * m[7] - m[6] * m[4]);
}
// inverse (row-major), returns det; out undefined when det == 0
template <class R>
__device__ __forceinline__ R inv3(const R* m, R* o) {
  R d = det3(m);
  o[0] = (m[4] * m[8] - m[7] * m[5]) / d;
  o[1] = -(m[1] * m[8] - m[7] * m[2]) / d;
  o[2] = (m[1] * m[5] - m[4] * m[2]) / d;
  o[3] = -(m[3] * m[8] - m[6] * m[5]) / d;
  o[4] = (m[0] * m[8] - m[6] * m[2]) / d;
  o[5] = -(m[0] * m[5] - m[3] * m[2]) / d;
  o[6] = (m[3] * m[7] - m[6] * m[4]) / d;
  o[7] = -(m[0] * m[7] - m[6] * m[1]) / d;
  o[8] = (m[0] * m[4] - m[3] * m[1]) / d;
  return d;
}

// ---- materials (materials.rs) -----------------------------------------------
// Per quadrature point state.  M1 / M2 are the two matrices the pair
// contraction needs: SNH: M1 = Cof(F) = J F^-T, StVK: M1 = S, M2 = F F^T.
template <class R>
struct QpState {
  R F[9];
  R M1[9];
  R M2[9];
  R s1, s2, s3, s4;
  R P[9];
};

template <class R>
__device__ __forceinline__ bool snh_state(const R* F, R mu0, R lam0, QpState<R>& q, bool need_stress) {
  const R d = R(3.0);
  R mu = (d + R(1.0)) / d * mu0;
  R lam = lam0 + (R(1.0) - R(2.0) / (d * (d + R(1.0)))) * mu0;
  R alpha = R(1.0) + mu / lam * (d / (d + R(1.0)));
  R IC = R(0.0);
#pragma unroll
  for (int k = 0; k < 9; ++k) IC += F[k] * F[k];
  R Fi[9];
  R J = inv3(F, Fi);
  if (J == R(0.0)) return false;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) q.M1[3 * i + j] = Fi[3 * j + i] * J;  // dJ/dF = F^-T J
  R beta = IC + R(1.0);
  q.s1 = mu * (R(1.0) - R(1.0) / beta);
  q.s2 = mu * R(2.0) / (beta * beta);
  q.s3 = lam * (J - alpha);
  q.s4 = lam;
  if (need_stress) {
    R cf = mu * (R(1.0) - R(1.0) / (IC + R(1.0))), cj = lam * (J - alpha);
#pragma unroll
    for (int k = 0; k < 9; ++k) q.P[k] = F[k] * cf + q.M1[k] * cj;
  }
  return true;
}

template <class R>
__device__ __forceinline__ void stvk_state(const R* F, R mu, R lam, QpState<R>& q, bool need_stress) {
  R E[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      R s = F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j];  // (F^T F)(i,j)
      E[3 * i + j] = (s - (i == j ? R(1.0) : R(0.0))) * R(0.5);
    }
  R tr = E[0] + E[4] + E[8];
#pragma unroll
  for (int k = 0; k < 9; ++k) q.M1[k] = E[k] * R(2.0) * mu + ((k % 4 == 0) ? lam * tr : R(0.0));
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) q.M2[3 * i + j] = F[3 * i] * F[3 * j] + F[3 * i + 1] * F[3 * j + 1] + F[3 * i + 2] * F[3 * j + 2];
  q.s1 = mu;
  q.s4 = lam;
  if (need_stress) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        q.P[3 * i + j] = F[3 * i] * q.M1[j] + F[3 * i + 1] * q.M1[3 + j] + F[3 * i + 2] * q.M1[6 + j];
  }
}

template <class R>
__device__ __forceinline__ bool material_state(int kind, const R* F, R mu, R lam, QpState<R>& q,
                                               bool need_stress) {
#pragma unroll
  for (int k = 0; k < 9; ++k) q.F[k] = F[k];
  if (kind == HOEFEM_MAT_SNH) return snh_state(F, mu, lam, q, need_stress);
  stvk_state(F, mu, lam, q, need_stress);
  return true;
}

template <class R>
__device__ __forceinline__ void mat3vec(const R* M, const R* a, R* o) {
  o[0] = M[0] * a[0] + M[1] * a[1] + M[2] * a[2];
  o[1] = M[3] * a[0] + M[4] * a[1] + M[5] * a[2];
  o[2] = M[6] * a[0] + M[7] * a[1] + M[8] * a[2];
}

// Per quadrature point data the pair contraction needs (13 values): T = F
// (SNH, cross term) or F F^T (StVK), and four scalars (SNH: s1, s2, s3 =
// lam (J - alpha), s4 = lam; StVK: s1 = mu, s4 = lam).
template <class R>
struct QpPair {
  R T[9];
  R s1, s2, s3, s4;
};

template <class R>
__device__ __forceinline__ void qp_pair_from(int kind, const QpState<R>& q, QpPair<R>& o) {
#pragma unroll
  for (int k = 0; k < 9; ++k) o.T[k] = (kind == HOEFEM_MAT_SNH) ? q.F[k] : q.M2[k];
  o.s1 = q.s1;
  o.s2 = q.s2;
  o.s3 = q.s3;
  o.s4 = q.s4;
}

// Stiffness block of node pair (I row, J column), added into acc (3x3 row-major).
// Per-node vectors: v[0..2] = a, v[3..5] = F a, v[6..8] = M1 a.
//  SNH : s1 (aI.aJ) I + s2 (F aI)(F aJ)^T + lam (Cof aI)(Cof aJ)^T + s3 eps_ijm (F (aI x aJ))_m
//  StVK: (aJ . S aI) I + mu (F aJ)(F aI)^T + mu (aI.aJ) F F^T + lam (F aI)(F aJ)^T
template <class R>
__device__ __forceinline__ void pair_block(int kind, const QpPair<R>& q, const R* vI, const R* vJ, R* acc) {
  R dot = vI[0] * vJ[0] + vI[1] * vJ[1] + vI[2] * vJ[2];
  if (kind == HOEFEM_MAT_SNH) {
    R cr[3] = {vI[1] * vJ[2] - vI[2] * vJ[1], vI[2] * vJ[0] - vI[0] * vJ[2], vI[0] * vJ[1] - vI[1] * vJ[0]};
    R w[3];
    mat3vec(q.T, cr, w);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) acc[3 * i + j] += q.s2 * vI[3 + i] * vJ[3 + j] + q.s4 * vI[6 + i] * vJ[6 + j];
    R d1 = q.s1 * dot;
    acc[0] += d1; acc[4] += d1; acc[8] += d1;
    // eps_ijm w_m: (0,1)=w2 (0,2)=-w1 (1,0)=-w2 (1,2)=w0 (2,0)=w1 (2,1)=-w0
    R s3 = q.s3;
    acc[1] += s3 * w[2]; acc[2] -= s3 * w[1];
    acc[3] -= s3 * w[2]; acc[5] += s3 * w[0];
    acc[6] += s3 * w[1]; acc[7] -= s3 * w[0];
  } else {
    R d0 = vJ[0] * vI[6] + vJ[1] * vI[7] + vJ[2] * vI[8];  // aJ . S aI
    R mu = q.s1, lam = q.s4;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        acc[3 * i + j] += mu * vJ[3 + i] * vI[3 + j] + mu * dot * q.T[3 * i + j] + lam * vI[3 + i] * vJ[3 + j];
    acc[0] += d0; acc[4] += d0; acc[8] += d0;
  }
}

__device__ __forceinline__ void quad_rule(const BlockDev& b, int e, int& q0, int& nq) {
  if (b.uniform) { q0 = 0; nq = b.nq; }
  else { q0 = b.qoff[e]; nq = b.qoff[e + 1] - q0; }
}

}  // namespace
}  // namespace hoefem
