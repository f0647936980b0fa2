// Preconditioned conjugate gradient on the device.
//
// Reference: ConjugateGradient::solve_with_guess_ (fenris/src/cg.rs:376-482)
// with RelativeResidualCriterion (cg.rs:77-124).  The loop control lives on
// the device: each kernel of an iteration starts by reading a `done` word in
// the solver state, and the last block of every reduction applies the
// reference's tests (pAp <= 0 -> IndefiniteOperator, zTr <= 0 ->
// IndefinitePreconditioner, ||r|| <= tol ||b|| -> converged, iterations >=
// max -> MaxIterationsReached) and sets it.  The host replays a CUDA graph of
// `chunk` iterations and reads the state once per chunk, so a solve costs one
// host round trip per chunk instead of per iteration, and the result (x,
// iteration count, status) is the one the sequential loop would produce.
// All reductions are deterministic: the node-row kernels fetch chunks of
// nodes dynamically but sum each chunk in a fixed order and the chunks in
// index order; the vector kernels use a fixed grid and sum block partials in
// block order.  A Schwarz preconditioner is applied either as dense products
// with its symmetrized inverted subdomain blocks plus a per-node gather
// (default) or as an SpMV over its assembled values.  The SpMV variants of
// the operator (and of an assembled Schwarz apply) are chosen online per
// value precision by timing the first chunks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "internal.h"
#include "kernels_common.cuh"
#include "learned.h"
#include "solver.h"

namespace hoefem {

int spmv_grid(int nv, int lanes);

namespace {

constexpr int TPB = 256;

// r = b - A x ; partial b.b, r.r
template <int L, class VA>
__global__ void __launch_bounds__(TPB) k_cg_init(NodeRows A, const VA* __restrict__ vals,
                                                 const double* __restrict__ x, const double* __restrict__ b,
                                                 double* __restrict__ r, double* part, CgState* st) {
  for_each_node_reduce<L, 2>(A, part, [&](int a, int sl, double (&acc)[2]) {
    double s[3];
    node_row_dot<L>(A, vals, x, a, sl, s[0], s[1], s[2]);
    if (a >= 0 && sl == 0) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double bi = b[3 * a + i];
        double ri = bi - s[i];
        r[3 * a + i] = ri;
        acc[0] += bi * bi;
        acc[1] += ri * ri;
      }
    }
  });
  double extra[2] = {0.0, 0.0}, tot[2];
  if (node_reduce_finish<L, 2>(A, part, extra, tot) && threadIdx.x == 0) {
    st->bnorm = sqrt(tot[0]);
    st->rr = tot[1];
  }
}

// z = M r  (mode: 0 identity, 1 diagonal) ; partial z.r ; when `init` the
// last block stores zTr, otherwise it forms beta = zTr_next / zTr.
__global__ void __launch_bounds__(TPB) k_cg_prec_vec(int n, int mode, const double* __restrict__ d,
                                                     const double* __restrict__ r, double* __restrict__ z,
                                                     double* partials, unsigned* counter, CgState* st, int init) {
  if (!init && st->done) return;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double ri = r[i];
    double zi = mode == 1 ? d[i] * ri : ri;
    z[i] = zi;
    acc[0] += zi * ri;
  }
  double tot[1];
  if (grid_reduce_last_k<1>(acc, partials, counter, tot) && threadIdx.x == 0) {
    if (init) st->zTr = tot[0];
    else {
      st->beta = tot[0] / st->zTr;
      st->zTr = tot[0];
    }
  }
}

// z = P r with P a node-row matrix (Schwarz) ; partial z.r.
template <int L, class VP>
__global__ void __launch_bounds__(TPB) k_cg_prec_spmv(NodeRows P, const VP* __restrict__ pv,
                                                      const double* __restrict__ r, double* __restrict__ z,
                                                      double* part, CgState* st, int init) {
  if (!init && st->done) return;
  for_each_node_reduce<L, 1>(P, part, [&](int a, int sl, double (&acc)[1]) {
    double s[3];
    node_row_dot<L>(P, pv, r, a, sl, s[0], s[1], s[2]);
    if (a >= 0 && sl == 0) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        z[3 * a + i] = s[i];
        acc[0] += s[i] * r[3 * a + i];
      }
    }
  });
  // untreated (diagonal-only) nodes, elementwise
  double extra[1] = {0.0}, tot[1];
  for_each_diag_dof(P, pv, r, [&](int dof, double v) {
    z[dof] = v;
    extra[0] += v * r[dof];
  });
  if (node_reduce_finish<L, 1>(P, part, extra, tot) && threadIdx.x == 0) {
    if (init) st->zTr = tot[0];
    else {
      st->beta = tot[0] / st->zTr;
      st->zTr = tot[0];
    }
  }
}

// Schwarz apply as dense block products: y_s = B_s r_s for every subdomain s
// (B_s the symmetric part of the inverted block, row-major dim x dim).  B_s is
// symmetric, so thread j accumulates column j over the rows: every row is
// read by consecutive threads (coalesced) and no reduction is needed.
constexpr int SCHWARZ_BLOCK_TPB = 96;  // >= 3 x 27 rows of a Hex27 subdomain

template <class VB>
__global__ void __launch_bounds__(SCHWARZ_BLOCK_TPB) k_cg_schwarz_blocks(const int* __restrict__ sub_off,
                                                                         const int* __restrict__ sub_nodes,
                                                                         const long long* __restrict__ stage_off,
                                                                         const VB* __restrict__ B,
                                                                         const int* __restrict__ slot,
                                                                         const double* __restrict__ r,
                                                                         const double* __restrict__ Ap,
                                                                         double* __restrict__ y, const CgState* st,
                                                                         int init, int update) {
  if (!init && st->done) return;
  __shared__ double rs[SCHWARZ_BLOCK_TPB];
  const int s = blockIdx.x;
  const int o = sub_off[s];
  const int dim = 3 * (sub_off[s + 1] - o);
  const int j = threadIdx.x;
  if (j < dim) {
    // with `update`: the residual after this iteration's step, r - alpha Ap
    // (the same expression the gather stores)
    const int d = 3 * sub_nodes[o + j / 3] + j % 3;
    rs[j] = update ? r[d] - st->alpha * Ap[d] : r[d];
  }
  __syncthreads();
  if (j >= dim) return;
  const VB* Bs = B + stage_off[s];
  double acc = 0.0;
#pragma unroll 9
  for (int i = 0; i < dim; ++i) acc += (double)Bs[(size_t)i * dim + j] * rs[i];
  y[3 * slot[o + j / 3] + j % 3] = acc;
}

// z = P r from the block products (each node: its consecutive slots, its
// subdomains in ascending order; untreated nodes: their diagonal value times
// r) ; z.r ; when `init` the last block stores zTr, otherwise it forms beta.
// With `update` it also takes the CG step of this iteration first (x += alpha
// p, r -= alpha Ap, r.r, iteration count and convergence, as k_cg_update):
// the block products already used the updated residual.
template <class VP>
__global__ void __launch_bounds__(TPB) k_cg_schwarz_gather(int n, const int* __restrict__ pair_off,
                                                           const double* __restrict__ y,
                                                           const unsigned char* __restrict__ diag_only,
                                                           const long long* __restrict__ pbase,
                                                           const VP* __restrict__ pv, double* __restrict__ r,
                                                           double* __restrict__ z, double* __restrict__ x,
                                                           const double* __restrict__ p,
                                                           const double* __restrict__ Ap, double* partials,
                                                           unsigned* counter, CgState* st, int init, int update) {
  if (!init && st->done) return;
  const double alpha = update ? st->alpha : 0.0;
  double acc[2] = {0.0, 0.0};  // r.r (update only), z.r
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double ri = r[t];
    if (update) {
      x[t] = x[t] + alpha * p[t];
      ri = r[t] - alpha * Ap[t];
      r[t] = ri;
      acc[0] += ri * ri;
    }
    const int a = t / 3, i = t - 3 * a;
    double v = 0.0;
    if (diag_only[a]) {
      v = (double)pv[pbase[a] + i] * ri;
    } else {
      for (int q = pair_off[a]; q < pair_off[a + 1]; ++q) v += y[3 * q + i];
    }
    z[t] = v;
    acc[1] += v * ri;
  }
  double tot[2];
  if (grid_reduce_last_k<2>(acc, partials, counter, tot) && threadIdx.x == 0) {
    if (init) {
      st->zTr = tot[1];
    } else if (update) {
      st->rr = tot[0];
      st->iters += 1;
      if (sqrt(tot[0]) <= st->tol * st->bnorm) { st->done = 1; st->status = HOEFEM_OK; }
      else if (st->max_iter >= 0 && st->iters >= st->max_iter) {
        st->done = 1;
        st->status = HOEFEM_CG_MAX_ITERATIONS;
      } else {
        st->beta = tot[1] / st->zTr;
        st->zTr = tot[1];
      }
    } else {
      st->beta = tot[1] / st->zTr;
      st->zTr = tot[1];
    }
  }
}

__global__ void k_cg_copy(int n, const double* __restrict__ a, double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// Initial convergence test (loop head of cg.rs:419-441 before any update).
__global__ void k_cg_init_check(CgState* st) {
  st->iters = 0;
  st->beta = 0.0;  // first direction p = z (the streamed CG forms z + beta p)
  st->done = 0;
  st->status = HOEFEM_OK;
  if (st->bnorm == 0.0) {
    st->done = 2;  // x must be zeroed by the host
    return;
  }
  if (sqrt(st->rr) <= st->tol * st->bnorm) { st->done = 1; return; }
  if (st->max_iter >= 0 && st->iters >= st->max_iter) { st->done = 1; st->status = HOEFEM_CG_MAX_ITERATIONS; }
}

// Three row sums of node a in FP32: FP32 values times the FP32 copy of the
// operand (one 16-byte entry per node), FP32 sums, the same traversals as
// node_row_dot; the products carry the values' own rounding (as the streamed
// engine's FP32 tiles).
template <int L>
__device__ __forceinline__ void node_row_dot_f32(const NodeRows& A, const float* __restrict__ vals,
                                                 const float4* __restrict__ x4, int a, int sl, float& s0, float& s1,
                                                 float& s2) {
  constexpr int LNS = LaneCfg<L>::lanes;
  s0 = s1 = s2 = 0.f;
  if (a >= 0) {
    const long long b = A.base[a];
    if (A.diag_only && A.diag_only[a]) {
      if (sl == 0) {
        const float4 xv = x4[a];
        s0 = vals[b] * xv.x;
        s1 = vals[b + 1] * xv.y;
        s2 = vals[b + 2] * xv.z;
      }
    } else if constexpr (LaneCfg<L>::stream) {
      const int o = A.adj_off[a], d = A.adj_off[a + 1] - o;
      const int rl = 3 * d;
      const float* r0 = vals + b;
      const float* xf = reinterpret_cast<const float*>(x4);
#pragma unroll 4
      for (int c = sl; c < rl; c += LNS) {
        const int s = c / 3, j = c - 3 * s;
        const float xv = xf[4 * A.adj[o + s] + j];
        s0 += r0[c] * xv;
        s1 += r0[rl + c] * xv;
        s2 += r0[2 * rl + c] * xv;
      }
    } else {
      const int o = A.adj_off[a], d = A.adj_off[a + 1] - o;
      const long long rl = 3LL * d;
#pragma unroll 2
      for (int s = sl; s < d; s += LNS) {
        const float4 xv = x4[A.adj[o + s]];
        const float* r0 = vals + b + 3 * s;
        s0 += r0[0] * xv.x + r0[1] * xv.y + r0[2] * xv.z;
        const float* r1 = r0 + rl;
        s1 += r1[0] * xv.x + r1[1] * xv.y + r1[2] * xv.z;
        const float* r2 = r1 + rl;
        s2 += r2[0] * xv.x + r2[1] * xv.y + r2[2] * xv.z;
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

// Ap = A p with FP32 values and the FP32 copy of p ; pAp with the FP64 p ;
// checks ; alpha
template <int L>
__global__ void __launch_bounds__(TPB) k_cg_Ap32(NodeRows A, const float* __restrict__ vals,
                                                 const float4* __restrict__ p4, const double* __restrict__ p,
                                                 double* __restrict__ Ap, double* part, CgState* st) {
  if (st->done) return;
  for_each_node_reduce<L, 1>(A, part, [&](int a, int sl, double (&acc)[1]) {
    float f[3];
    node_row_dot_f32<L>(A, vals, p4, a, sl, f[0], f[1], f[2]);
    if (a >= 0 && sl == 0) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double si = (double)f[i];
        Ap[3 * a + i] = si;
        acc[0] += p[3 * a + i] * si;
      }
    }
  });
  double extra[1] = {0.0}, tot[1];
  if (node_reduce_finish<L, 1>(A, part, extra, tot) && threadIdx.x == 0) {
    double pAp = tot[0];
    st->pAp = pAp;
    if (pAp <= 0.0) { st->done = 1; st->status = HOEFEM_CG_INDEFINITE_OPERATOR; }
    else if (st->zTr <= 0.0) { st->done = 1; st->status = HOEFEM_CG_INDEFINITE_PRECONDITIONER; }
    else st->alpha = st->zTr / pAp;
  }
}

// p = z + beta p (beta = 0: p = z) and its FP32 copy, one node per thread
__global__ void __launch_bounds__(TPB) k_cg_p4(int nv, const double* __restrict__ z, double* __restrict__ p,
                                               float4* __restrict__ p4, const CgState* st, int copy) {
  if (!copy && st->done) return;
  const double beta = copy ? 0.0 : st->beta;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nv; a += gridDim.x * blockDim.x) {
    double q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      q[k] = copy ? z[3 * a + k] : z[3 * a + k] + beta * p[3 * a + k];
      p[3 * a + k] = q[k];
    }
    p4[a] = make_float4((float)q[0], (float)q[1], (float)q[2], 0.f);
  }
}

// Ap = A p ; pAp ; checks ; alpha
template <int L, class VA>
__global__ void __launch_bounds__(TPB) k_cg_Ap(NodeRows A, const VA* __restrict__ vals,
                                               const double* __restrict__ p, double* __restrict__ Ap, double* part,
                                               CgState* st) {
  if (st->done) return;
  for_each_node_reduce<L, 1>(A, part, [&](int a, int sl, double (&acc)[1]) {
    double s[3];
    node_row_dot<L>(A, vals, p, a, sl, s[0], s[1], s[2]);
    if (a >= 0 && sl == 0) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        Ap[3 * a + i] = s[i];
        acc[0] += p[3 * a + i] * s[i];
      }
    }
  });
  double extra[1] = {0.0}, tot[1];
  if (node_reduce_finish<L, 1>(A, part, extra, tot) && threadIdx.x == 0) {
    double pAp = tot[0];
    st->pAp = pAp;
    if (pAp <= 0.0) { st->done = 1; st->status = HOEFEM_CG_INDEFINITE_OPERATOR; }
    else if (st->zTr <= 0.0) { st->done = 1; st->status = HOEFEM_CG_INDEFINITE_PRECONDITIONER; }
    else st->alpha = st->zTr / pAp;
  }
}

// x += alpha p ; r -= alpha Ap ; (fused z = M r for identity / diagonal) ;
// r.r ; iteration count and convergence.
__global__ void __launch_bounds__(TPB) k_cg_update(int n, int fuse_mode, const double* __restrict__ d,
                                                   double* __restrict__ x, double* __restrict__ r,
                                                   const double* __restrict__ p, const double* __restrict__ Ap,
                                                   double* __restrict__ z, double* partials, unsigned* counter,
                                                   CgState* st) {
  if (st->done) return;
  const double alpha = st->alpha;
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = x[i] + alpha * p[i];
    double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    acc[0] += ri * ri;
    if (fuse_mode > 0) {
      double zi = fuse_mode == 2 ? d[i] * ri : ri;
      z[i] = zi;
      acc[1] += zi * ri;
    }
  }
  double tot[2];
  if (grid_reduce_last_k<2>(acc, partials, counter, tot) && threadIdx.x == 0) {
    st->rr = tot[0];
    st->iters += 1;
    if (sqrt(tot[0]) <= st->tol * st->bnorm) { st->done = 1; st->status = HOEFEM_OK; }
    else if (st->max_iter >= 0 && st->iters >= st->max_iter) {
      st->done = 1;
      st->status = HOEFEM_CG_MAX_ITERATIONS;
    } else if (fuse_mode > 0) {
      st->beta = tot[1] / st->zTr;
      st->zTr = tot[1];
    }
  }
}

// p = z + beta p
__global__ void __launch_bounds__(TPB) k_cg_p(int n, const double* __restrict__ z, double* __restrict__ p,
                                              const CgState* st) {
  if (st->done) return;
  const double beta = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = z[i] + beta * p[i];
}

// Residual replacement (reliable update) of the mixed-precision CG: before the
// true residual overwrites r, keep the recurrence's z.r in pAp.
__global__ void k_cg_save_ztr(CgState* st) { st->pAp = st->zTr; }

// After r = b - A64 x and z = P r: convergence test on the true residual.
// `resume`: the recurrence had stopped as converged; if the true residual has
// not, iterate on with the direction p = z + (z.r / z.r_old) p.
__global__ void k_cg_reliable(CgState* st, int resume) {
  if (sqrt(st->rr) <= st->tol * st->bnorm) {
    st->done = 1;
    st->status = HOEFEM_OK;
    return;
  }
  if (!resume) return;
  if (st->max_iter >= 0 && st->iters >= st->max_iter) {
    st->done = 1;
    st->status = HOEFEM_CG_MAX_ITERATIONS;
    return;
  }
  st->done = 0;
  st->status = HOEFEM_OK;
  st->beta = st->zTr / st->pAp;
}

// ---- flexible CG with the learned coarse correction ------------------------

// r_old = r; zr_old = z.r of this iteration (before the update).
__global__ void k_fcg_save(int n, const double* __restrict__ r, double* __restrict__ r_old, CgState* st) {
  if (st->done) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) st->zr_old = st->zTr;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r_old[i] = r[i];
}

// z.r, z.r_old, c.r, c.r_old; the last block keeps the correction c if
// c.r > 0, scaled by w = min(1, z.r / c.r) so that the coarse term never
// outweighs the Schwarz term along r (the network predicts the coarse part
// of the error, which the Schwarz term partly contains already); then
// z' = z + w c, z'.r is the new zTr and (init = 0)
// beta = (z'.r - z'.r_old) / zr_old.
__global__ void __launch_bounds__(256) k_fcg_dots(int n, const double* __restrict__ z, const double* __restrict__ c,
                                                  const double* __restrict__ r, const double* __restrict__ r_old,
                                                  double* partials, unsigned* counter, CgState* st, int init) {
  if (!init && st->done) return;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = r[i], zi = z[i], ci = c[i];
    acc[0] += zi * ri;
    acc[2] += ci * ri;
    if (!init) {
      const double ro = r_old[i];
      acc[1] += zi * ro;
      acc[3] += ci * ro;
    }
  }
  double tot[4];
  if (grid_reduce_last_k<4>(acc, partials, counter, tot) && threadIdx.x == 0) {
    const bool keep = tot[2] > 0.0;
    const double wgt = keep ? fmin(1.0, fmax(tot[0], 0.0) / tot[2]) : 0.0;
    st->learned_flag = keep ? 1 : 0;
    st->learned_weight = wgt;
    if (keep) st->learned_kept += 1;
    else st->learned_dropped += 1;
    const double zr = tot[0] + wgt * tot[2];
    if (!init) {
      const double zro = tot[1] + wgt * tot[3];
      st->beta = (zr - zro) / st->zr_old;
    }
    st->zTr = zr;
  }
}

// p = z + w c + beta p (init: p = z + w c).
__global__ void __launch_bounds__(256) k_fcg_p(int n, const double* __restrict__ z, const double* __restrict__ c,
                                               double* __restrict__ p, const CgState* st, int init) {
  if (!init && st->done) return;
  const double f = st->learned_flag ? st->learned_weight : 0.0, beta = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double zi = z[i] + f * c[i];
    p[i] = init ? zi : zi + beta * p[i];
  }
}

int vec_grid(i64 n) { return reduce_blocks_for(n); }

__global__ void k_axpy(int n, double a, const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += a * x[i];
}

__global__ void k_to_f32(long long n, const double* __restrict__ a, float* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

}  // namespace

void CgWork::init(Model* model) {
  m = model;
  n = model->ndof;
  x.alloc(n); b.alloc(n); r.alloc(n); z.alloc(n); p.alloc(n); Ap.alloc(n);
  // node-chunk partials (<= nv / 8 chunks) + block partials, K <= 2 values
  partials.alloc(std::max<size_t>(reduce_partials_count(), 2 * ((size_t)model->nv / 8 + 2) + 2 * 4096));
  st.alloc(1);
  counter.alloc(1);
  HOEFEM_CUDA(cudaMemsetAsync(counter.p, 0, sizeof(unsigned), model->stream));
  if (!h_st) HOEFEM_CUDA(cudaMallocHost(&h_st, sizeof(CgState)));
}

CgWork::~CgWork() {
  for (auto& g : graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (h_st) cudaFreeHost(h_st);
  for (auto* e : {&tev[0], &tev[1], &sev[0], &sev[1]})
    if (*e) cudaEventDestroy(*e);
  if (fcg_exec) cudaGraphExecDestroy(fcg_exec);
  for (auto& t : tuning) {
    if (t.e0) cudaEventDestroy(t.e0);
    if (t.e1) cudaEventDestroy(t.e1);
  }
}

void to_f32(const double* a, float* b, long long n, cudaStream_t s) {
  (note_launch(), k_to_f32<<<device_sms() * 8, 256, 0, s>>>(n, a, b));
  HOEFEM_CUDA(cudaGetLastError());
}

namespace {

// Operator values: FP64 or FP32 (exactly one set).
struct Operator {
  const double* v64;
  const float* v32;
};

const void* prec_key(const Precond* P, bool p32) {
  if (!P) return nullptr;
  if (P->kind == PREC_SCHWARZ) return p32 ? (const void*)P->vals32.p : (const void*)P->vals.p;
  return (const void*)P->diag.p;
}

int lanes_for(const Model& m, bool f32) { return f32 && m.spmv_lanes32 ? m.spmv_lanes32 : m.spmv_lanes; }
int lanes_for(const Precond& p, bool f32) { return f32 && p.spmv_lanes32 ? p.spmv_lanes32 : p.spmv_lanes; }

void enqueue_Ap(CgWork& w, Operator A, cudaStream_t s) {
  NodeRows R = w.m->rows();
  R.lanes = lanes_for(*w.m, A.v32 != nullptr);
  HOEFEM_REQUIRE(R.sched, HOEFEM_ERR_INVALID_ARGUMENT, "node-row matrix without scheduling counters");
  HOEFEM_LANES_DISPATCH(R.lanes, {
    const int sg = spmv_grid(R.count(), LN);
    if (A.v32)
      (note_launch(), k_cg_Ap32<LN><<<sg, TPB, 0, s>>>(R, A.v32, w.p32.p, w.p.p, w.Ap.p, w.partials.p, w.st.p));
    else
      (note_launch(), k_cg_Ap<LN, double><<<sg, TPB, 0, s>>>(R, A.v64, w.p.p, w.Ap.p, w.partials.p, w.st.p));
  });
}

// p = z + beta p (copy: p = z), with the FP32 copy when the operator is FP32
void enqueue_p(CgWork& w, bool f32, bool copy, cudaStream_t s) {
  const int n = (int)w.n;
  if (f32)
    (note_launch(), k_cg_p4<<<vec_grid(n / 3), TPB, 0, s>>>(n / 3, w.z.p, w.p.p, w.p32.p, w.st.p, copy ? 1 : 0));
  else if (copy)
    (note_launch(), k_cg_copy<<<vec_grid(n), TPB, 0, s>>>(n, w.z.p, w.p.p));
  else
    (note_launch(), k_cg_p<<<vec_grid(n), TPB, 0, s>>>(n, w.z.p, w.p.p, w.st.p));
}

// update (block apply only): fuse this iteration's x / r step into the apply
void enqueue_prec_spmv(CgWork& w, const Precond* P, bool p32, int init, cudaStream_t s, int update = 0) {
  if (P->block_apply) {
    const int n = (int)w.n;
    HOEFEM_REQUIRE(!p32 || P->nsub == 0 || P->bsym32.p, HOEFEM_ERR_INVALID_ARGUMENT,
                   "FP32 Schwarz blocks missing (update the preconditioner for FP32)");
    if (P->nsub > 0) {
      if (p32)
        (note_launch(), k_cg_schwarz_blocks<float><<<(int)P->nsub, SCHWARZ_BLOCK_TPB, 0, s>>>(
                            P->d_sub_off.p, P->d_sub_nodes.p, P->d_stage_off.p, P->bsym32.p, P->d_npair.p, w.r.p, w.Ap.p, P->ysub.p,
                            w.st.p, init, update));
      else
        (note_launch(), k_cg_schwarz_blocks<double><<<(int)P->nsub, SCHWARZ_BLOCK_TPB, 0, s>>>(
                            P->d_sub_off.p, P->d_sub_nodes.p, P->d_stage_off.p, P->bsym.p, P->d_npair.p, w.r.p, w.Ap.p, P->ysub.p,
                            w.st.p, init, update));
    }
    if (p32)
      (note_launch(), k_cg_schwarz_gather<float><<<vec_grid(n), TPB, 0, s>>>(
                          n, P->d_npair_off.p, P->ysub.p, P->d_diag_only.p, P->d_base.p, P->vals32.p,
                          w.r.p, w.z.p, w.x.p, w.p.p, w.Ap.p, w.partials.p, w.counter.p, w.st.p, init, update));
    else
      (note_launch(), k_cg_schwarz_gather<double><<<vec_grid(n), TPB, 0, s>>>(
                          n, P->d_npair_off.p, P->ysub.p, P->d_diag_only.p, P->d_base.p, P->vals.p,
                          w.r.p, w.z.p, w.x.p, w.p.p, w.Ap.p, w.partials.p, w.counter.p, w.st.p, init, update));
    return;
  }
  NodeRows PR = P->rows();
  PR.lanes = lanes_for(*P, p32);
  HOEFEM_LANES_DISPATCH(PR.lanes, {
    const int g = spmv_grid(PR.nv, LN);
    if (p32)
      (note_launch(), k_cg_prec_spmv<LN, float><<<g, TPB, 0, s>>>(PR, P->vals32.p, w.r.p, w.z.p, w.partials.p,
                                                                  w.st.p, init));
    else
      (note_launch(), k_cg_prec_spmv<LN, double><<<g, TPB, 0, s>>>(PR, P->vals.p, w.r.p, w.z.p, w.partials.p,
                                                                   w.st.p, init));
  });
}

void enqueue_iteration(CgWork& w, Operator A, const Precond* P, bool p32, cudaStream_t s) {
  const int n = (int)w.n;
  const int vg = vec_grid(n);
  enqueue_Ap(w, A, s);
  const int kind = P ? P->kind : PREC_NONE;
  if (kind == PREC_SCHWARZ && P->block_apply) {
    enqueue_prec_spmv(w, P, p32, 0, s, 1);  // the step fused into the apply
  } else if (kind == PREC_SCHWARZ) {
    (note_launch(), k_cg_update<<<vg, TPB, 0, s>>>(n, 0, nullptr, w.x.p, w.r.p, w.p.p, w.Ap.p, w.z.p, w.partials.p,
                                                   w.counter.p, w.st.p));
    enqueue_prec_spmv(w, P, p32, 0, s);
  } else {
    int mode = kind == PREC_DIAGONAL ? 2 : 1;
    (note_launch(), k_cg_update<<<vg, TPB, 0, s>>>(n, mode, kind == PREC_DIAGONAL ? P->diag.p : nullptr, w.x.p, w.r.p,
                                                   w.p.p, w.Ap.p, w.z.p, w.partials.p, w.counter.p, w.st.p));
  }
  enqueue_p(w, A.v32 != nullptr, false, s);
}

CgWork::Graph& graph_for(CgWork& w, Operator A, const Precond* P, bool p32) {
  // the key also holds the SpMV variants the graph was captured with
  const intptr_t variants = (intptr_t)lanes_for(*w.m, A.v32 != nullptr) * 1024 +
                            (P && P->kind == PREC_SCHWARZ ? (P->block_apply ? 1000 : lanes_for(*P, p32)) : 0);
  const void* key[4] = {A.v32 ? (const void*)A.v32 : (const void*)A.v64, (const void*)P, prec_key(P, p32),
                        (const void*)(intptr_t)(((P ? P->kind : 0) * 2 + (p32 ? 1 : 0)) + 8 * variants)};
  for (auto& g : w.graphs)
    if (g.exec && std::equal(key, key + 4, g.key)) return g;
  if (w.graphs.size() >= 4) {
    cudaGraphExecDestroy(w.graphs.front().exec);
    w.graphs.erase(w.graphs.begin());
  }
  CgWork::Graph G;
  std::copy(key, key + 4, G.key);
  cudaStream_t cs;
  HOEFEM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t g;
  HOEFEM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  g_capture_count = 0;
  for (int k = 0; k < w.chunk; ++k) enqueue_iteration(w, A, P, p32, cs);
  G.kernels = g_capture_count;
  g_capture_count = -1;
  HOEFEM_CUDA(cudaStreamEndCapture(cs, &g));
  HOEFEM_CUDA(cudaGraphInstantiate(&G.exec, g, 0));
  cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  w.graphs.push_back(G);
  return w.graphs.back();
}

// PCG on A with preconditioner P: x = w.x (initial guess), b = w.b.
// With A64 (reliable updates): A holds FP32 values of the same matrix; the
// initial residual and every residual replacement use the FP64 values A64.
// A replacement runs at a chunk boundary when the recurrence residual has
// dropped by `delta` since the last one, and whenever the recurrence reports
// convergence (which then has to hold for the true residual).
int run_pcg(CgWork& w, Operator A, const Precond* P, bool p32, double tol, i64 max_iter, i64* iters,
            cudaStream_t s, const double* A64 = nullptr, double delta = 0.0, i64* replacements = nullptr) {
  NodeRows R = w.m->rows();
  const int n = (int)w.n;
  const int kind = P ? P->kind : PREC_NONE;
  HOEFEM_REQUIRE(!P || P->ready, HOEFEM_ERR_INVALID_ARGUMENT, "preconditioner has not been updated");
  if (P && !P->block_apply) precond_assemble(*P, s);  // the SpMV apply reads every entry
  // automatic engine choice: each engine's first solve builds its one-time
  // structures (graphs, stream layouts) and is not timed; its second solve of
  // at least 20 iterations is timed whole (set-up, packing, replacements and
  // launches included), per iteration
  const int pk = !P ? 0 : (P->kind == PREC_DIAGONAL ? 1 : 2);
  CgWork::EngineTune& et = w.etune[(A.v32 != nullptr ? 3 : 0) + pk];
  // below ~220 nodes per SM the streamed kernel's two grid barriers per
  // iteration cost more than the graphs' launches, and sampling it (a stream
  // layout built on the host) costs more than a short-lived solver can win:
  // the chunked engine without sampling
  if (w.stream_mode == 0 && et.choice < 0 && w.m->nv < (i64)CgWork::STREAM_MIN_NODES) et.choice = 0;
  if (!w.tev[0]) {
    HOEFEM_CUDA(cudaEventCreate(&w.tev[0]));
    HOEFEM_CUDA(cudaEventCreate(&w.tev[1]));
  }
  if (w.stream_mode == 0 && et.choice < 0) HOEFEM_CUDA(cudaEventRecord(w.tev[0], s));
  CgState init{};
  init.tol = tol;
  init.max_iter = max_iter;
  HOEFEM_CUDA(cudaMemcpyAsync(w.st.p, &init, sizeof(CgState), cudaMemcpyHostToDevice, s));
  const int vg = vec_grid(n);
  HOEFEM_REQUIRE(R.sched, HOEFEM_ERR_INVALID_ARGUMENT, "node-row matrix without scheduling counters");
  auto true_residual = [&](const double* vals64) {
    R.lanes = lanes_for(*w.m, false);
    HOEFEM_LANES_DISPATCH(R.lanes, {
      const int sg = spmv_grid(R.nv, LN);
      (note_launch(), k_cg_init<LN, double><<<sg, TPB, 0, s>>>(R, vals64, w.x.p, w.b.p, w.r.p, w.partials.p,
                                                               w.st.p));
    });
  };
  auto prec_init = [&]() {
    if (kind == PREC_SCHWARZ) {
      enqueue_prec_spmv(w, P, p32, 1, s);
    } else {
      (note_launch(), k_cg_prec_vec<<<vg, TPB, 0, s>>>(n, kind == PREC_DIAGONAL ? 1 : 0,
                                                       kind == PREC_DIAGONAL ? P->diag.p : nullptr, w.r.p, w.z.p,
                                                       w.partials.p, w.counter.p, w.st.p, 1));
    }
  };
  if (A64) {
    true_residual(A64);
  } else {
    R.lanes = lanes_for(*w.m, A.v32 != nullptr);
    HOEFEM_LANES_DISPATCH(R.lanes, {
      const int sg = spmv_grid(R.nv, LN);
      if (A.v32)
        (note_launch(), k_cg_init<LN, float><<<sg, TPB, 0, s>>>(R, A.v32, w.x.p, w.b.p, w.r.p, w.partials.p,
                                                                w.st.p));
      else
        (note_launch(), k_cg_init<LN, double><<<sg, TPB, 0, s>>>(R, A.v64, w.x.p, w.b.p, w.r.p, w.partials.p,
                                                                 w.st.p));
    });
  }
  prec_init();
  if (A.v32 && !w.p32.p) w.p32.alloc(n / 3);
  enqueue_p(w, A.v32 != nullptr, true, s);
  (note_launch(), k_cg_init_check<<<1, 1, 0, s>>>(w.st.p));
  HOEFEM_CUDA(cudaGetLastError());
  HOEFEM_CUDA(cudaMemcpyAsync(w.h_st, w.st.p, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  if (w.h_st->done == 2) {
    HOEFEM_CUDA(cudaMemsetAsync(w.x.p, 0, sizeof(double) * n, s));
    *iters = 0;
    return HOEFEM_OK;
  }
  if (w.h_st->done) {
    *iters = w.h_st->iters;
    return w.h_st->status;
  }
  const bool f32 = A.v32 != nullptr;
  const double* vals64 = A64 ? A64 : A.v64;
  // persistent streamed CG: the operator (FP64 values, FP32 in the mixed
  // form) and the Schwarz blocks packed into their stream layouts, then one
  // launch per residual replacement
  w.last_tune = (f32 ? 3 : 0) + pk;
  bool want_stream = w.stream_mode == 2;
  if (w.stream_mode == 0) want_stream = et.choice >= 0 ? et.choice == 1 : et.phase >= 2;
  const bool streamed =
      want_stream && vals64 && cg_stream_usable(w, P) && cg_stream_prepare(w, vals64, f32, P, p32, s);
  HOEFEM_REQUIRE(streamed || w.stream_mode != 2, HOEFEM_ERR_INVALID_ARGUMENT,
                 "the streamed CG cannot run this solve (preconditioner, device or layout)");
  if (w.stream_mode == 0 && want_stream && !streamed) et.choice = 0;  // cannot stream: chunked from now on
  // phases: 0 chunked set-up solve, 1 chunked timed, 2 streamed set-up, 3 streamed timed
  auto sample = [&](int engine) {
    if (w.stream_mode != 0 || et.choice >= 0 || (et.phase >= 2) != (engine == 1)) return;
    if ((et.phase & 1) == 0) {
      ++et.phase;
      return;
    }
    HOEFEM_CUDA(cudaEventRecord(w.tev[1], s));
    HOEFEM_CUDA(cudaEventSynchronize(w.tev[1]));
    const i64 n_it = w.h_st->iters;
    if (n_it < 20) return;
    float ms = 0.f;
    HOEFEM_CUDA(cudaEventElapsedTime(&ms, w.tev[0], w.tev[1]));
    et.us_per_it[engine] = 1e3 * ms / (double)n_it;
    if (++et.phase == 4) et.choice = et.us_per_it[1] < et.us_per_it[0] ? 1 : 0;
  };
  if (streamed) {
    cg_stream_arm(w, A64 ? delta : 0.0, s);
    w.stream_ms = 0.f;
    const i64 cap_s = max_iter >= 0 ? max_iter : 10 * (i64)n;
    i64 nrep_s = 0;
    for (;;) {
      const i64 it0 = w.h_st->iters;
      cg_stream_iterate(w, f32, P, p32, A64 != nullptr, s);
      w.stream_iterations += w.h_st->iters - it0;
      // a launch that ran no iteration found the solve finished by the
      // replacement before it
      const bool ran = w.h_st->iters > it0;
      if (A64 && ran) {
        const bool conv = w.h_st->done && w.h_st->status == HOEFEM_OK;
        const bool trig = !w.h_st->done && w.h_st->replace;
        if (conv || trig) {
          (note_launch(), k_cg_save_ztr<<<1, 1, 0, s>>>(w.st.p));
          true_residual(A64);
          prec_init();
          // resume after a converged recurrence: beta = z.r / z.r_old; the
          // kernel forms the direction z + beta p itself.  No host round trip
          // here: if the true residual meets the tolerance, the next launch
          // returns at once and the loop ends on its state.
          (note_launch(), k_cg_reliable<<<1, 1, 0, s>>>(w.st.p, conv ? 1 : 0));
          cg_stream_arm(w, delta, s);
          ++nrep_s;
          if (conv) {
            // the recurrence claimed convergence: the true residual usually
            // confirms it, so read the outcome instead of launching a kernel
            // that would return at once
            HOEFEM_CUDA(cudaMemcpyAsync(w.h_st, w.st.p, sizeof(CgState), cudaMemcpyDeviceToHost, s));
            HOEFEM_CUDA(cudaStreamSynchronize(s));
            if (w.h_st->done) break;
          }
          continue;
        }
      }
      if (w.h_st->done) break;
      if (w.h_st->iters >= cap_s) {
        if (replacements) *replacements = nrep_s;
        *iters = w.h_st->iters;
        return HOEFEM_CG_MAX_ITERATIONS;
      }
    }
    sample(1);
    if (replacements) *replacements = nrep_s;
    *iters = w.h_st->iters;
    return w.h_st->status;
  }
  // online SpMV variant choice: candidate pairs (operator lanes, Schwarz lanes)
  // (with the block apply the Schwarz SpMV variant plays no part)
  const bool schwarz = P && P->kind == PREC_SCHWARZ && !P->block_apply;
  static const int cand_lanes[4] = {8, 16, 32, 132};
  const int ncand = schwarz ? 16 : 4;
  CgWork::Tuning& tu = w.tuning[f32 ? 1 : 0];
  if (!w.online_tuning || w.m->spmv_pinned || (schwarz && P->spmv_pinned)) tu.done = true;
  if (!tu.done && !tu.e0) {
    HOEFEM_CUDA(cudaEventCreate(&tu.e0));
    HOEFEM_CUDA(cudaEventCreate(&tu.e1));
  }
  auto set_candidate = [&](int c) {
    const int lj = cand_lanes[c % 4], lp = cand_lanes[c / 4];
    if (f32) w.m->spmv_lanes32 = lj;
    else w.m->spmv_lanes = lj;
    if (schwarz) {
      Precond* Pm = const_cast<Precond*>(P);
      if (p32) Pm->spmv_lanes32 = lp;
      else Pm->spmv_lanes = lp;
    }
  };
  // without an iteration limit CG is still bounded: 10 n iterations
  const i64 cap = max_iter >= 0 ? max_iter : 10 * (i64)n;
  const i64 max_chunks = (cap + w.chunk - 1) / w.chunk + 2;
  double rr_ref = w.h_st->rr;
  // the engine sample of this solve counts only if the SpMV variants were already tuned
  const bool sample_chunked = tu.done;
  i64 nrep = 0;
  for (i64 c = 0; c < max_chunks; ++c) {
    const i64 it0 = w.h_st->iters;
    const bool timing = !tu.done;
    if (timing) set_candidate(tu.next);
    CgWork::Graph& G = graph_for(w, A, P, p32);
    if (timing) HOEFEM_CUDA(cudaEventRecord(tu.e0, s));
    HOEFEM_CUDA(cudaGraphLaunch(G.exec, s));
    g_launch_count.fetch_add(G.kernels, std::memory_order_relaxed);
    if (timing) HOEFEM_CUDA(cudaEventRecord(tu.e1, s));
    HOEFEM_CUDA(cudaMemcpyAsync(w.h_st, w.st.p, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    HOEFEM_CUDA(cudaStreamSynchronize(s));
    if (timing) {
      // a chunk that ran all its iterations is a valid sample of candidate tu.next
      if (w.h_st->iters - it0 == w.chunk) {
        float ms = 0.f;
        HOEFEM_CUDA(cudaEventElapsedTime(&ms, tu.e0, tu.e1));
        if (ms < tu.best_ms) {
          tu.best_ms = ms;
          tu.best = tu.next;
        }
        if (++tu.next == ncand) tu.done = true;
      }
      set_candidate(tu.done ? tu.best : tu.next);
    }
    if (A64) {
      const bool conv = w.h_st->done && w.h_st->status == HOEFEM_OK;
      const bool trig = !w.h_st->done && w.h_st->rr <= delta * delta * rr_ref;
      if (conv || trig) {
        (note_launch(), k_cg_save_ztr<<<1, 1, 0, s>>>(w.st.p));
        true_residual(A64);
        prec_init();
        (note_launch(), k_cg_reliable<<<1, 1, 0, s>>>(w.st.p, conv ? 1 : 0));
        if (conv) enqueue_p(w, A.v32 != nullptr, false, s);
        HOEFEM_CUDA(cudaGetLastError());
        HOEFEM_CUDA(cudaMemcpyAsync(w.h_st, w.st.p, sizeof(CgState), cudaMemcpyDeviceToHost, s));
        HOEFEM_CUDA(cudaStreamSynchronize(s));
        rr_ref = w.h_st->rr;
        ++nrep;
      }
    }
    if (w.on_chunk && !w.h_st->done) w.on_chunk(s);
    if (w.h_st->done) break;
  }
  if (sample_chunked) sample(0);
  if (replacements) *replacements = nrep;
  *iters = w.h_st->iters;
  if (!w.h_st->done) return HOEFEM_CG_MAX_ITERATIONS;
  return w.h_st->status;
}

}  // namespace

int cg_solve(CgWork& w, const double* vals, const Precond* P, double tol, i64 max_iter, i64* iters, cudaStream_t s) {
  return run_pcg(w, Operator{vals, nullptr}, P, false, tol, max_iter, iters, s);
}

// Mixed precision: PCG whose operator (and Schwarz preconditioner) values are
// FP32 while vectors, dot products and residual updates stay FP64, with
// residual replacement against the FP64 operator (reliable updates,
// Sleijpen & van der Vorst 1996): the Krylov recurrence is never restarted,
// and the stopping test ||b - A64 x|| <= tol ||b|| holds for the true FP64
// residual.
int cg_solve_reliable(CgWork& w, const double* A64, const float* A32, const Precond* P, double tol, i64 max_iter,
                      double delta, i64* iters, i64* replacements, cudaStream_t s) {
  const bool p32 = P && P->kind == PREC_SCHWARZ && P->vals32.p;
  return run_pcg(w, Operator{nullptr, A32}, P, p32, tol, max_iter, iters, s, A64, delta, replacements);
}

// Flexible PCG with the learned two-level preconditioner (Notay's flexible CG
// recurrence, since the network makes the preconditioner depend on r): per
// iteration Ap and alpha as PCG, x / r updated, z = P r (the Schwarz or
// diagonal apply of the plain solver), c = the network's coarse correction of
// r, kept only if c.r > 0 (otherwise the iteration is the plain PCG step with
// the flexible beta), p = z + c + beta p.  No host round trip inside an
// iteration: the chunks of iterations are replayed as CUDA graphs, as in the
// plain solver.
int cg_solve_learned(CgWork& w, const double* vals, const Precond* P, Learned* L, double tol, i64 max_iter,
                     i64* iters, i64* kept, i64* dropped, cudaStream_t s) {
  HOEFEM_REQUIRE(L && L->trained, HOEFEM_ERR_INVALID_ARGUMENT, "learned correction not trained");
  HOEFEM_REQUIRE(!P || P->ready, HOEFEM_ERR_INVALID_ARGUMENT, "preconditioner has not been updated");
  if (P && !P->block_apply) precond_assemble(*P, s);  // the SpMV apply reads every entry
  NodeRows R = w.m->rows();
  const int n = (int)w.n;
  const int vg = vec_grid(n);
  const int kind = P ? P->kind : PREC_NONE;
  if (w.r_old.n < (size_t)n) w.r_old.alloc(n);
  double* c = L->e.p;
  CgState init{};
  init.tol = tol;
  init.max_iter = max_iter;
  HOEFEM_CUDA(cudaMemcpyAsync(w.st.p, &init, sizeof(CgState), cudaMemcpyHostToDevice, s));
  R.lanes = lanes_for(*w.m, false);
  HOEFEM_LANES_DISPATCH(R.lanes, {
    const int sg = spmv_grid(R.nv, LN);
    (note_launch(), k_cg_init<LN, double><<<sg, TPB, 0, s>>>(R, vals, w.x.p, w.b.p, w.r.p, w.partials.p, w.st.p));
  });
  auto plain_prec = [&](cudaStream_t cs) {
    if (kind == PREC_SCHWARZ) enqueue_prec_spmv(w, P, false, 1, cs);
    else
      (note_launch(), k_cg_prec_vec<<<vg, TPB, 0, cs>>>(n, kind == PREC_DIAGONAL ? 1 : 0,
                                                        kind == PREC_DIAGONAL ? P->diag.p : nullptr, w.r.p, w.z.p,
                                                        w.partials.p, w.counter.p, w.st.p, 1));
  };
  plain_prec(s);
  L->predict_device(w.r.p, &w.st.p->rr, c, s);
  (note_launch(), k_fcg_dots<<<vg, TPB, 0, s>>>(n, w.z.p, c, w.r.p, nullptr, w.partials.p, w.counter.p, w.st.p, 1));
  (note_launch(), k_fcg_p<<<vg, TPB, 0, s>>>(n, w.z.p, c, w.p.p, w.st.p, 1));
  (note_launch(), k_cg_init_check<<<1, 1, 0, s>>>(w.st.p));
  HOEFEM_CUDA(cudaGetLastError());
  HOEFEM_CUDA(cudaMemcpyAsync(w.h_st, w.st.p, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  auto finish = [&](int status) {
    *iters = w.h_st->iters;
    *kept = w.h_st->learned_kept;
    *dropped = w.h_st->learned_dropped;
    return status;
  };
  if (w.h_st->done == 2) {
    HOEFEM_CUDA(cudaMemsetAsync(w.x.p, 0, sizeof(double) * n, s));
    return finish(HOEFEM_OK);
  }
  if (w.h_st->done) return finish(w.h_st->status);
  // one graph of w.chunk iterations
  if (!w.fcg_exec || w.fcg_key[0] != (const void*)vals || w.fcg_key[1] != (const void*)P ||
      w.fcg_key[2] != (const void*)L) {
    if (w.fcg_exec) cudaGraphExecDestroy(w.fcg_exec);
    w.fcg_exec = nullptr;
    cudaStream_t cs;
    HOEFEM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    HOEFEM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    g_capture_count = 0;
    for (int k = 0; k < w.chunk; ++k) {
      enqueue_Ap(w, Operator{vals, nullptr}, cs);
      (note_launch(), k_fcg_save<<<vg, TPB, 0, cs>>>(n, w.r.p, w.r_old.p, w.st.p));
      (note_launch(), k_cg_update<<<vg, TPB, 0, cs>>>(n, 0, nullptr, w.x.p, w.r.p, w.p.p, w.Ap.p, w.z.p,
                                                      w.partials.p, w.counter.p, w.st.p));
      plain_prec(cs);
      L->predict_device(w.r.p, &w.st.p->rr, c, cs);
      (note_launch(), k_fcg_dots<<<vg, TPB, 0, cs>>>(n, w.z.p, c, w.r.p, w.r_old.p, w.partials.p, w.counter.p,
                                                     w.st.p, 0));
      (note_launch(), k_fcg_p<<<vg, TPB, 0, cs>>>(n, w.z.p, c, w.p.p, w.st.p, 0));
    }
    w.fcg_kernels = g_capture_count;
    g_capture_count = -1;
    HOEFEM_CUDA(cudaStreamEndCapture(cs, &g));
    HOEFEM_CUDA(cudaGraphInstantiate(&w.fcg_exec, g, 0));
    cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    w.fcg_key[0] = vals;
    w.fcg_key[1] = P;
    w.fcg_key[2] = L;
  }
  const i64 cap = max_iter >= 0 ? max_iter : 10 * (i64)n;
  const i64 max_chunks = (cap + w.chunk - 1) / w.chunk + 2;
  for (i64 ch = 0; ch < max_chunks; ++ch) {
    HOEFEM_CUDA(cudaGraphLaunch(w.fcg_exec, s));
    g_launch_count.fetch_add(w.fcg_kernels, std::memory_order_relaxed);
    HOEFEM_CUDA(cudaMemcpyAsync(w.h_st, w.st.p, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    HOEFEM_CUDA(cudaStreamSynchronize(s));
    if (w.h_st->done) break;
  }
  if (!w.h_st->done) return finish(HOEFEM_CG_MAX_ITERATIONS);
  return finish(w.h_st->status);
}

}  // namespace hoefem
