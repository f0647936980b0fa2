// Sparse and vector kernels on the node-row CSR layout (FP64).
//
// Reference: spmv_csr (fenris/src/sparse.rs:1164-1199) and MKL
// mkl_sparse_d_mv (simulation_toolbox/src/fem/newton_cg.rs:595-619),
// compute_jacobian_combination_into (system_assembly.rs:196-235) with
// add_assign_linear_combination_par (sparse.rs:909-952) and
// apply_homogeneous_dirichlet_bc_csr (fenris/src/assembly.rs:799-869).
//
// SpMV: one warp per node computes its three rows.  The neighbour list is
// read once for the three rows (their column structure is identical), each
// lane takes a neighbour slot, gathers x[3b..3b+2] once and multiplies it
// with the 3x3 block of the three rows.  Values are streamed exactly once
// (8 B/nnz), the adjacency costs 4 B per 9 nnz and x is gathered from L2.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "kernels_common.cuh"

namespace hoefem {

namespace {

template <int L>
__global__ void __launch_bounds__(256) k_spmv(NodeRows A, const double* __restrict__ vals,
                                              const double* __restrict__ x, double* __restrict__ y, double alpha,
                                              double beta) {
  for_each_node<L>(A, [&](int a, int sl) {
    double s0, s1, s2;
    node_row_dot<L>(A, vals, x, a, sl, s0, s1, s2);
    if (a >= 0 && sl == 0) {
      double y0 = (beta == 0.0) ? 0.0 : beta * y[3 * a];
      double y1 = (beta == 0.0) ? 0.0 : beta * y[3 * a + 1];
      double y2 = (beta == 0.0) ? 0.0 : beta * y[3 * a + 2];
      y[3 * a] = y0 + alpha * s0;
      y[3 * a + 1] = y1 + alpha * s1;
      y[3 * a + 2] = y2 + alpha * s2;
    }
  });
  node_sched_finish(A);
  for_each_diag_dof(A, vals, x, [&](int dof, double v) {
    y[dof] = ((beta == 0.0) ? 0.0 : beta * y[dof]) + alpha * v;
  });
}

// out = ck*K + cd*D + cm*M (in the reference's order: fill 0, += ck K,
// += cd D, += cm M), then Dirichlet rows / columns; diagonal of Dirichlet rows
// = |first non-zero diagonal| (found by the first pass, see
// k_first_nonzero_diag).
__global__ void __launch_bounds__(256) k_combine(NodeRows A, double ck, const double* __restrict__ K, double cd,
                                                 const double* __restrict__ D, double cm,
                                                 const double* __restrict__ M, double* __restrict__ out) {
  const long long nnz = A.base[A.nv];
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (K) v += ck * K[k];
    if (D) v += cd * D[k];
    if (M) v += cm * M[k];
    out[k] = v;
  }
}

// Smallest row index with a non-zero diagonal entry (atomicMin).
__global__ void k_first_nonzero_diag(NodeRows A, const double* __restrict__ vals, unsigned long long* first) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < A.nv; a += gridDim.x * blockDim.x) {
    int s = A.diag_slot[a];
    if (s < 0) continue;
    int d = A.adj_off[a + 1] - A.adj_off[a];
    for (int i = 0; i < 3; ++i) {
      double v = vals[A.base[a] + (long long)i * 3 * d + 3 * s + i];
      if (v != 0.0) {
        atomicMin(first, (unsigned long long)(3 * a + i));
        break;
      }
    }
  }
}

__global__ void k_dirichlet(NodeRows A, const unsigned char* __restrict__ bc, double* __restrict__ vals,
                            const unsigned long long* first) {
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  double scale = 1.0;
  unsigned long long f = *first;
  if (f != ~0ull) {
    int a0 = (int)(f / 3), i0 = (int)(f % 3);
    int d0 = A.adj_off[a0 + 1] - A.adj_off[a0];
    scale = fabs(vals[A.base[a0] + (long long)i0 * 3 * d0 + 3 * A.diag_slot[a0] + i0]);
  }
  __syncthreads();  // every thread has read the scale before any write
  // grid-wide: the scale entry may be rewritten by this kernel (it is a
  // diagonal entry and keeps its value unless its row is a Dirichlet row, in
  // which case it becomes `scale` itself), so the value read is stable.
  for (int a = blockIdx.x * wpb + (threadIdx.x >> 5); a < A.nv; a += gridDim.x * wpb) {
    const int o = A.adj_off[a], d = A.adj_off[a + 1] - o;
    const long long b = A.base[a];
    for (int i = 0; i < 3; ++i) {
      const int r = 3 * a + i;
      const bool rbc = bc[r];
      for (int s = lane; s < d; s += 32) {
        const int nb = A.adj[o + s];
        for (int j = 0; j < 3; ++j) {
          const int c = 3 * nb + j;
          long long k = b + (long long)i * 3 * d + 3 * s + j;
          if (rbc) vals[k] = (c == r) ? scale : 0.0;
          else if (bc[c]) vals[k] = 0.0;
        }
      }
    }
  }
}

__global__ void k_fill_u64(unsigned long long* p, unsigned long long v) { *p = v; }

}  // namespace

// Multiprocessor count of the current device (queried once per device).
int device_sms() {
  static std::atomic<int> cache[64];
  int dev = 0;
  HOEFEM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) dev = 0;
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    HOEFEM_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    if (v <= 0) v = 1;
    cache[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

size_t reduce_partials_count() { return (size_t)device_sms() * 64; }

// Grid of the node-row kernels: with dynamic node scheduling, one CTA per
// resident slot (8 CTAs of 256 threads per SM) or fewer for small matrices;
// the two-value deterministic reductions fit their partials buffer
// (reduce_partials_count() doubles).
int spmv_grid(int nv, int lanes) {
  int nodes_per_block = 8 * (32 / (lanes % 100));
  int g = (nv + nodes_per_block - 1) / nodes_per_block;
  const int cap = device_sms() * 8;
  return g < cap ? (g > 0 ? g : 1) : cap;
}

void spmv_node_rows(const NodeRows& A, const double* vals, const double* x, double* y, double alpha, double beta,
                    cudaStream_t s) {
  HOEFEM_LANES_DISPATCH(A.lanes,
                        (note_launch(), k_spmv<LN><<<spmv_grid(A.nv, LN), 256, 0, s>>>(A, vals, x, y, alpha, beta)));
  HOEFEM_CUDA(cudaGetLastError());
}

// Autotuner for the node-row SpMV: times the 8 / 16 / 32 lanes-per-node
// variants on this matrix structure (5 launches each after 2 warm-up
// launches, CUDA events on stream s) and returns the fastest.
int autotune_spmv_lanes(NodeRows A, const double* vals, cudaStream_t s, float* best_ms) {
  const int n = 3 * A.nv;
  double *x = nullptr, *y = nullptr;
  HOEFEM_CUDA(cudaMallocAsync(&x, sizeof(double) * (n ? n : 1), s));
  HOEFEM_CUDA(cudaMallocAsync(&y, sizeof(double) * (n ? n : 1), s));
  HOEFEM_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * (n ? n : 1), s));
  // Inside CG the operator streams from HBM (matrix, preconditioner and
  // vectors exceed L2), so each timed launch follows an L2 flush (a write of
  // a buffer larger than L2); the median of 3 launches decides.
  const size_t flush_bytes = (size_t)192 << 20;
  void* flush = nullptr;
  HOEFEM_CUDA(cudaMallocAsync(&flush, flush_bytes, s));
  cudaEvent_t e0, e1;
  HOEFEM_CUDA(cudaEventCreate(&e0));
  HOEFEM_CUDA(cudaEventCreate(&e1));
  int best = 32;
  float best_t = 1e30f;
  const int cand[6] = {8, 16, 32, 108, 116, 132};
  for (int c : cand) {
    A.lanes = c;
    spmv_node_rows(A, vals, x, y, 1.0, 0.0, s);
    float t[3];
    for (int k = 0; k < 3; ++k) {
      HOEFEM_CUDA(cudaMemsetAsync(flush, k + 1, flush_bytes, s));
      HOEFEM_CUDA(cudaEventRecord(e0, s));
      spmv_node_rows(A, vals, x, y, 1.0, 0.0, s);
      HOEFEM_CUDA(cudaEventRecord(e1, s));
      HOEFEM_CUDA(cudaEventSynchronize(e1));
      HOEFEM_CUDA(cudaEventElapsedTime(&t[k], e0, e1));
    }
    std::sort(t, t + 3);
    if (t[1] < best_t) { best_t = t[1]; best = c; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(flush, s);
  cudaFreeAsync(x, s);
  cudaFreeAsync(y, s);
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  if (best_ms) *best_ms = best_t;
  return best;
}

void jacobian_combination(const Model& m, double ck, const double* K, double cm, const double* M,
                          const unsigned char* bc_dof, double* out, double* d_scratch, cudaStream_t s, double cd,
                          const double* D) {
  NodeRows A = m.rows();
  (note_launch(), k_combine<<<device_sms() * 8, 256, 0, s>>>(A, ck, K, cd, D, cm, M, out));
  if (bc_dof) {
    unsigned long long* first = reinterpret_cast<unsigned long long*>(d_scratch);
    (note_launch(), k_fill_u64<<<1, 1, 0, s>>>(first, ~0ull));
    (note_launch(), k_first_nonzero_diag<<<(A.nv + 255) / 256, 256, 0, s>>>(A, out, first));
    // The scale entry is read before any thread writes: k_dirichlet reads it
    // at entry, and a Dirichlet diagonal entry is overwritten with `scale`
    // itself, so the race is benign (all writers store the same value).
    (note_launch(), k_dirichlet<<<spmv_grid(A.nv, 32), 256, 0, s>>>(A, bc_dof, out, first));
  }
  HOEFEM_CUDA(cudaGetLastError());
}

// ---- deterministic reductions -------------------------------------------------
namespace {
__global__ void __launch_bounds__(256) k_dot(const double* __restrict__ a, const double* __restrict__ b, long long n,
                                             double* out, double* partials, unsigned* counter) {
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v += a[i] * b[i];
  double tot;
  if (grid_reduce_last(v, partials, counter, tot) && threadIdx.x == 0) *out = tot;
}
}  // namespace

int reduce_blocks_for(i64 n) {
  i64 g = (n + 1023) / 1024;
  if (g < 1) g = 1;
  const i64 cap = (i64)device_sms() * 4;
  if (g > cap) g = cap;
  return (int)g;
}

void dot_device(const double* a, const double* b, i64 n, double* out, double* partials, unsigned* counter,
                cudaStream_t s) {
  (note_launch(), k_dot<<<reduce_blocks_for(n), 256, 0, s>>>(a, b, n, out, partials, counter));
  HOEFEM_CUDA(cudaGetLastError());
}

}  // namespace hoefem
