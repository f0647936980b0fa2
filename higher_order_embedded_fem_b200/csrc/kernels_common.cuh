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

// SpMV variant code L: lanes per node = L % 100 (8, 16 or 32); L >= 100
// selects the column-streaming traversal.
template <int L>
struct LaneCfg {
  static constexpr int lanes = L % 100;
  static constexpr bool stream = L >= 100;
};

// Three row sums of node a computed by a group of LaneCfg<L>::lanes lanes
// (sub-lane sl in [0, lanes)); a < 0 gives zeros.  All 32 lanes of the warp
// must call it (the group reduction uses xor shuffles inside aligned groups).
// Matrix values are FP64 or FP32 (V); products and sums are FP64.
// Neighbour-major traversal (L < 100): a lane takes whole neighbours (its
// 3 x 3 block in the node's three rows).  Column-streaming traversal
// (L >= 100): a lane takes scalar columns c = sl, sl + lanes, ... of the
// node's rows, so consecutive lanes read consecutive values of each row
// (fully coalesced) and share one x gather across the three rows.
template <int L, class V>
__device__ __forceinline__ void node_row_dot(const NodeRows& A, const V* __restrict__ vals,
                                             const double* __restrict__ x, int a, int sl, double& s0, double& s1,
                                             double& s2) {
  constexpr int LNS = LaneCfg<L>::lanes;
  s0 = s1 = s2 = 0.0;
  if (a >= 0) {
    const long long b = A.base[a];
    if (A.diag_only && A.diag_only[a]) {
      if (sl == 0) {
        s0 = (double)vals[b] * x[3 * a];
        s1 = (double)vals[b + 1] * x[3 * a + 1];
        s2 = (double)vals[b + 2] * x[3 * a + 2];
      }
    } else if constexpr (LaneCfg<L>::stream) {
      const int o = A.adj_off[a], d = A.adj_off[a + 1] - o;
      const int rl = 3 * d;
      const V* r0 = vals + b;
#pragma unroll 4
      for (int c = sl; c < rl; c += LNS) {
        const int s = c / 3, j = c - 3 * s;
        const double xv = x[3 * A.adj[o + s] + j];
        s0 += (double)r0[c] * xv;
        s1 += (double)r0[rl + c] * xv;
        s2 += (double)r0[2 * rl + c] * xv;
      }
    } else {
      const int o = A.adj_off[a], d = A.adj_off[a + 1] - o;
      const long long rl = 3LL * d;
#pragma unroll 2
      for (int s = sl; s < d; s += LNS) {
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
  for (int off = LNS / 2; off > 0; off >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, off);
    s1 += __shfl_xor_sync(0xffffffffu, s1, off);
    s2 += __shfl_xor_sync(0xffffffffu, s2, off);
  }
}

// Iterates the nodes of a node-row matrix with LaneCfg<L>::lanes lanes per
// node: body(a, sl) is called by every lane, with a = -1 for lanes whose group
// has no node (they must still take part in the reductions).  With
// A.sched, warps take chunks of NF consecutive nodes from a global work
// counter until the nodes run out (dynamic load balance: node degrees vary
// and a fixed grid-stride split leaves a tail); node_sched_finish resets the
// counters in the last block.  Without A.sched: a grid-stride loop.
template <int L, class F>
__device__ __forceinline__ void for_each_node(const NodeRows& A, F&& body) {
  constexpr int LNS = LaneCfg<L>::lanes;
  constexpr int G = 32 / LNS;
  constexpr int NF = G >= 4 ? 16 : 8;
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  const int grp = lane / LNS, sl = lane % LNS;
  const int nv = A.count();
  const int* __restrict__ list = A.nodes;
  if (A.sched == nullptr) {
    for (int a0 = (blockIdx.x * wpb + (threadIdx.x >> 5)) * G; a0 < nv; a0 += gridDim.x * wpb * G) {
      const int i = a0 + grp;
      body(i < nv ? (list ? list[i] : i) : -1, sl);
    }
    return;
  }
  // (claiming the next chunk before processing the current one measured
  // slower: the chunk is claimed when the warp is free)
  for (;;) {
    unsigned start = 0;
    if (lane == 0) start = atomicAdd(A.sched, (unsigned)NF);
    start = __shfl_sync(0xffffffffu, start, 0);
    if (start >= (unsigned)nv) break;
    const int end = min((int)start + NF, nv);
#pragma unroll 1
    for (int a0 = (int)start; a0 < (int)start + NF; a0 += G) {
      const int i = a0 + grp;
      body(i < end ? (list ? list[i] : i) : -1, sl);
    }
  }
}

// The diagonal-only nodes of A (A.dnodes): body(dof, A_dd * x_dof) for each
// of their DOFs, grid-stride over all threads.
template <class V, class F>
__device__ __forceinline__ void for_each_diag_dof(const NodeRows& A, const V* __restrict__ vals,
                                                  const double* __restrict__ x, F&& body) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * A.ndnodes; t += gridDim.x * blockDim.x) {
    const int a = A.dnodes[t / 3], i = t - 3 * (t / 3);
    const int dof = 3 * a + i;
    body(dof, (double)vals[A.base[a] + i] * x[dof]);
  }
}

// End of a dynamically scheduled node loop: every thread of the block must
// call it; the last block to arrive resets the counters for the next launch.
__device__ __forceinline__ void node_sched_finish(const NodeRows& A) {
  if (A.sched == nullptr) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(A.sched + 1, 1u);
    if (t == gridDim.x - 1) {
      A.sched[0] = 0u;
      A.sched[1] = 0u;
      __threadfence();
    }
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
    } else if ((lanes) == 108) {                  \
      constexpr int LN = 108;                     \
      KERNEL_CALL;                                \
    } else if ((lanes) == 116) {                  \
      constexpr int LN = 116;                     \
      KERNEL_CALL;                                \
    } else if ((lanes) == 132) {                  \
      constexpr int LN = 132;                     \
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

// Nodes per dynamically fetched chunk for lane configuration L.
template <int L>
struct NodeChunk {
  static constexpr int G = 32 / LaneCfg<L>::lanes;
  static constexpr int NF = G >= 4 ? 16 : 8;
  // the CG's partial-sum buffer holds one entry per chunk of at least 8 nodes
  static_assert(NF >= 8, "node chunks smaller than the partial-sum buffer allows");
};
__host__ __device__ inline int node_chunk_count(int count, int nf) { return (count + nf - 1) / nf; }

// Dynamically scheduled node loop with a deterministic reduction of K values:
// body(a, sl, acc) adds its contribution into acc (any lane); each fetched
// chunk of NF consecutive nodes is summed by its warp in a fixed order and
// stored at part[k * C + chunk] (C chunks), whichever warp took it.
// node_reduce_finish sums the chunks in index order.  Requires A.sched.
template <int L, int K, class F>
__device__ __forceinline__ void for_each_node_reduce(const NodeRows& A, double* __restrict__ part, F&& body) {
  constexpr int LNS = LaneCfg<L>::lanes;
  constexpr int G = NodeChunk<L>::G, NF = NodeChunk<L>::NF;
  const int lane = threadIdx.x & 31;
  const int grp = lane / LNS, sl = lane % LNS;
  const int count = A.count();
  const int C = node_chunk_count(count, NF);
  const int* __restrict__ list = A.nodes;
  for (;;) {
    unsigned start = 0;
    if (lane == 0) start = atomicAdd(A.sched, (unsigned)NF);
    start = __shfl_sync(0xffffffffu, start, 0);
    if (start >= (unsigned)count) break;
    const int end = min((int)start + NF, count);
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
#pragma unroll 1
    for (int a0 = (int)start; a0 < (int)start + NF; a0 += G) {
      const int i = a0 + grp;
      body(i < end ? (list ? list[i] : i) : -1, sl, acc);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double v = warp_sum_d(acc[k]);
      if (lane == 0) part[(size_t)k * C + start / NF] = v;
    }
  }
}

// Finishes a kernel that used for_each_node_reduce<L, K>: `extra` holds each
// thread's share of a statically scheduled part of the same sums (may be 0);
// it is block-summed into part[K * C + k * gridDim.x + block].  The last block
// to arrive resets the scheduling counters and returns true with tot = the
// chunk sums (index order) plus the block sums (block order) in thread 0.
// Every thread of every block must call it.
template <int L, int K>
__device__ __forceinline__ bool node_reduce_finish(const NodeRows& A, double* __restrict__ part,
                                                   double (&extra)[K], double (&tot)[K]) {
  __shared__ bool s_last;
  const int C = node_chunk_count(A.count(), NodeChunk<L>::NF);
  block_sum<K>(extra);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) part[(size_t)K * C + (size_t)k * gridDim.x + blockIdx.x] = extra[k];
    __threadfence();
    const unsigned t = atomicAdd(A.sched + 1, 1u);
    s_last = (t == gridDim.x - 1);
    if (s_last) {
      A.sched[0] = 0u;
      A.sched[1] = 0u;
    }
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  for (int c = threadIdx.x; c < C; c += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] += __ldcg(part + (size_t)k * C + c);
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] += __ldcg(part + (size_t)K * C + (size_t)k * gridDim.x + b);
  block_sum<K>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) tot[k] = acc[k];
  }
  return true;
}

}  // namespace hoefem
