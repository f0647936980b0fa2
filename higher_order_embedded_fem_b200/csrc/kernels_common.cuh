// Device helpers shared by the sparse, CG and Schwarz kernels.
#pragma once

#include <cuda_runtime.h>

#include "internal.h"

namespace hoefem {

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Three row sums of node a computed by a group of L lanes (L = 32, 16 or 8;
// sub-lane sl in [0, L)); a < 0 gives zeros.  All 32 lanes of the warp must
// call it (the group reduction uses xor shuffles inside aligned L-lane groups).
// Matrix values are FP64 or FP32 (V); products and sums are FP64.
template <int L, class V>
__device__ __forceinline__ void node_row_dot(const NodeRows& A, const V* __restrict__ vals,
                                             const double* __restrict__ x, int a, int sl, double& s0, double& s1,
                                             double& s2) {
  s0 = s1 = s2 = 0.0;
  if (a >= 0) {
    const long long b = A.base[a];
    if (A.diag_only && A.diag_only[a]) {
      if (sl == 0) {
        s0 = (double)vals[b] * x[3 * a];
        s1 = (double)vals[b + 1] * x[3 * a + 1];
        s2 = (double)vals[b + 2] * x[3 * a + 2];
      }
    } else {
      const int o = A.adj_off[a], d = A.adj_off[a + 1] - o;
      const long long rl = 3LL * d;
      for (int s = sl; s < d; s += L) {
        const int nb = A.adj[o + s];
        const double x0 = x[3 * nb], x1 = x[3 * nb + 1], x2 = x[3 * nb + 2];
        const V* r0 = vals + b + 3 * s;
        s0 += (double)r0[0] * x0 + (double)r0[1] * x1 + (double)r0[2] * x2;
        const V* r1 = r0 + rl;
        s1 += (double)r1[0] * x0 + (double)r1[1] * x1 + (double)r1[2] * x2;
        const V* r2 = r1 + rl;
        s2 += (double)r2[0] * x0 + (double)r2[1] * x1 + (double)r2[2] * x2;
      }
    }
  }
#pragma unroll
  for (int off = L / 2; off > 0; off >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, off);
    s1 += __shfl_xor_sync(0xffffffffu, s1, off);
    s2 += __shfl_xor_sync(0xffffffffu, s2, off);
  }
}

// Iterates the nodes of a node-row matrix with L lanes per node:
// body(a, sl) is called by every lane, with a = -1 for lanes whose group has
// no node in this round (they must still take part in the reductions).
template <int L, class F>
__device__ __forceinline__ void for_each_node(int nv, F&& body) {
  constexpr int G = 32 / L;
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const int grp = lane / L, sl = lane % L;
  for (int a0 = (blockIdx.x * wpb + (threadIdx.x >> 5)) * G; a0 < nv; a0 += gridDim.x * wpb * G) {
    const int a = a0 + grp;
    body(a < nv ? a : -1, sl);
  }
}

// Dispatch a kernel template instance on the lanes-per-node setting.
#define HOEFEM_LANES_DISPATCH(lanes, KERNEL_CALL) \
  do {                                            \
    if ((lanes) == 8) {                           \
      constexpr int LN = 8;                       \
      KERNEL_CALL;                                \
    } else if ((lanes) == 16) {                   \
      constexpr int LN = 16;                      \
      KERNEL_CALL;                                \
    } else {                                      \
      constexpr int LN = 32;                      \
      KERNEL_CALL;                                \
    }                                             \
  } while (0)

// Block sum of K values (blockDim.x multiple of 32, <= 1024); result in
// thread 0.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K]) {
  __shared__ double sh[K][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum_d(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) sh[k][w] = v[k];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double t = lane < nw ? sh[k][lane] : 0.0;
      v[k] = warp_sum_d(t);
    }
  }
  __syncthreads();
}

// Grid-wide deterministic reduction of K values: every block writes its
// partials, the last block to finish sums them in block order.  Returns true
// in the last block (all threads); `tot` is valid in its thread 0.
template <int K>
__device__ __forceinline__ bool grid_reduce_last_k(double (&v)[K], double* partials, unsigned* counter,
                                                   double (&tot)[K]) {
  __shared__ bool s_last;
  block_sum<K>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) partials[(size_t)k * gridDim.x + blockIdx.x] = v[k];
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  // fixed order: thread t sums blocks t, t+blockDim, ... then a tree
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] += __ldcg(partials + (size_t)k * gridDim.x + i);
  block_sum<K>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) tot[k] = acc[k];
    *counter = 0u;
  }
  return true;
}

__device__ __forceinline__ bool grid_reduce_last(double v, double* partials, unsigned* counter, double& tot) {
  double a[1] = {v}, t[1];
  bool last = grid_reduce_last_k<1>(a, partials, counter, t);
  tot = t[0];
  return last;
}

}  // namespace hoefem
