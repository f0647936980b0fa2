// Parallel cyclic Jacobi eigen-decomposition of a small symmetric matrix held
// in shared memory by one CTA (Schwarz fallback blocks, element PSD
// projection).
#pragma once

#include <cuda_runtime.h>

#include "kernels_common.cuh"

namespace hoefem {

// Jacobi rotation parameters zeroing A[p][q] (same formulas as the oracle).
__device__ __forceinline__ void jacobi_cs(double app, double aqq, double apq, double& c, double& s) {
  if (apq == 0.0) { c = 1.0; s = 0.0; return; }
  double theta = (aqq - app) / (2.0 * apq);
  double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
  c = 1.0 / sqrt(t * t + 1.0);
  s = t * c;
}

// A: m x m (m even; rows / columns >= dim are padding), V: m x m, set to the
// identity by the caller; cs / sn: m / 2 scratch each; s_red: 2 shared
// doubles.  Round-robin ordering: m/2 disjoint rotations per round, applied
// to the rows and then the columns of A (and the columns of V); sweeps until
// the off-diagonal mass is below 1e-32 of the total (at most 40).  On return
// the eigenvalues are A's diagonal and the eigenvectors V's columns.  Every
// thread of the CTA must call it.
__device__ __forceinline__ void jacobi_eigen_block(double* A, double* V, double* cs, double* sn, int m, int dim,
                                                   double* s_red) {
  const int half = m / 2;
  for (int sweep = 0; sweep < 40; ++sweep) {
    // convergence test on the off-diagonal mass
    double off = 0.0, tot = 0.0;
    for (int k = threadIdx.x; k < m * m; k += blockDim.x) {
      double x = A[k] * A[k];
      tot += x;
      if (k / m != k % m) off += x;
    }
    double vv[2] = {off, tot};
    block_sum<2>(vv);
    if (threadIdx.x == 0) { s_red[0] = vv[0]; s_red[1] = vv[1]; }
    __syncthreads();
    if (s_red[0] == 0.0 || s_red[0] <= 1e-32 * s_red[1]) break;
    for (int round = 0; round < m - 1; ++round) {
      for (int k = threadIdx.x; k < half; k += blockDim.x) {
        int p, q;
        if (k == 0) { p = round; q = m - 1; }
        else { p = (round + k) % (m - 1); q = (round - k + (m - 1)) % (m - 1); }
        if (p > q) { int t = p; p = q; q = t; }
        double c = 1.0, s = 0.0;
        if (q < dim) jacobi_cs(A[p * m + p], A[q * m + q], A[p * m + q], c, s);
        cs[k] = c;
        sn[k] = s;
      }
      __syncthreads();
      // rows p, q of A
      for (int it = threadIdx.x; it < half * m; it += blockDim.x) {
        int k = it / m, j = it % m;
        double s = sn[k];
        if (s == 0.0) continue;
        int p, q;
        if (k == 0) { p = round; q = m - 1; }
        else { p = (round + k) % (m - 1); q = (round - k + (m - 1)) % (m - 1); }
        if (p > q) { int t = p; p = q; q = t; }
        double c = cs[k];
        double a = A[p * m + j], b = A[q * m + j];
        A[p * m + j] = c * a - s * b;
        A[q * m + j] = s * a + c * b;
      }
      __syncthreads();
      // columns p, q of A and V
      for (int it = threadIdx.x; it < half * m; it += blockDim.x) {
        int k = it % half, i = it / half;
        double s = sn[k];
        if (s == 0.0) continue;
        int p, q;
        if (k == 0) { p = round; q = m - 1; }
        else { p = (round + k) % (m - 1); q = (round - k + (m - 1)) % (m - 1); }
        if (p > q) { int t = p; p = q; q = t; }
        double c = cs[k];
        double a = A[i * m + p], b = A[i * m + q];
        A[i * m + p] = c * a - s * b;
        A[i * m + q] = s * a + c * b;
        double va = V[i * m + p], vb = V[i * m + q];
        V[i * m + p] = c * va - s * vb;
        V[i * m + q] = s * va + c * vb;
      }
      __syncthreads();
    }
  }
}

}  // namespace hoefem
