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
// All reductions are deterministic (fixed grid, block partials summed in
// block order by the last block).
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "kernels_common.cuh"
#include "solver.h"

namespace hoefem {

int spmv_grid(int nv);

namespace {

constexpr int TPB = 256;

// r = b - A x ; partial b.b, r.r
__global__ void __launch_bounds__(TPB) k_cg_init(NodeRows A, const double* __restrict__ vals,
                                                 const double* __restrict__ x, const double* __restrict__ b,
                                                 double* __restrict__ r, double* partials, unsigned* counter,
                                                 CgState* st) {
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  double acc[2] = {0.0, 0.0};
  for (int a = blockIdx.x * wpb + (threadIdx.x >> 5); a < A.nv; a += gridDim.x * wpb) {
    double s[3];
    node_row_dot(A, vals, x, a, lane, s[0], s[1], s[2]);
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double bi = b[3 * a + i];
        double ri = bi - s[i];
        r[3 * a + i] = ri;
        acc[0] += bi * bi;
        acc[1] += ri * ri;
      }
    }
  }
  double tot[2];
  if (grid_reduce_last_k<2>(acc, partials, counter, tot) && threadIdx.x == 0) {
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
__global__ void __launch_bounds__(TPB) k_cg_prec_spmv(NodeRows P, const double* __restrict__ pv,
                                                      const double* __restrict__ r, double* __restrict__ z,
                                                      double* partials, unsigned* counter, CgState* st, int init) {
  if (!init && st->done) return;
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  double acc[1] = {0.0};
  for (int a = blockIdx.x * wpb + (threadIdx.x >> 5); a < P.nv; a += gridDim.x * wpb) {
    double s[3];
    node_row_dot(P, pv, r, a, lane, s[0], s[1], s[2]);
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        z[3 * a + i] = s[i];
        acc[0] += s[i] * r[3 * a + i];
      }
    }
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

__global__ void k_cg_copy(int n, const double* __restrict__ a, double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// Initial convergence test (loop head of cg.rs:419-441 before any update).
__global__ void k_cg_init_check(CgState* st) {
  st->iters = 0;
  st->done = 0;
  st->status = HOEFEM_OK;
  if (st->bnorm == 0.0) {
    st->done = 2;  // x must be zeroed by the host
    return;
  }
  if (sqrt(st->rr) <= st->tol * st->bnorm) { st->done = 1; return; }
  if (st->max_iter >= 0 && st->iters >= st->max_iter) { st->done = 1; st->status = HOEFEM_CG_MAX_ITERATIONS; }
}

// Ap = A p ; pAp ; checks ; alpha
__global__ void __launch_bounds__(TPB) k_cg_Ap(NodeRows A, const double* __restrict__ vals,
                                               const double* __restrict__ p, double* __restrict__ Ap,
                                               double* partials, unsigned* counter, CgState* st) {
  if (st->done) return;
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  double acc[1] = {0.0};
  for (int a = blockIdx.x * wpb + (threadIdx.x >> 5); a < A.nv; a += gridDim.x * wpb) {
    double s[3];
    node_row_dot(A, vals, p, a, lane, s[0], s[1], s[2]);
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        Ap[3 * a + i] = s[i];
        acc[0] += p[3 * a + i] * s[i];
      }
    }
  }
  double tot[1];
  if (grid_reduce_last_k<1>(acc, partials, counter, tot) && threadIdx.x == 0) {
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

int vec_grid(i64 n) { return reduce_blocks_for(n); }

}  // namespace

void CgWork::init(Model* model) {
  m = model;
  n = model->ndof;
  x.alloc(n); b.alloc(n); r.alloc(n); z.alloc(n); p.alloc(n); Ap.alloc(n);
  partials.alloc(4 * 148 * 16);
  st.alloc(1);
  counter.alloc(1);
  HOEFEM_CUDA(cudaMemsetAsync(counter.p, 0, sizeof(unsigned), model->stream));
  if (!h_st) HOEFEM_CUDA(cudaMallocHost(&h_st, sizeof(CgState)));
}

CgWork::~CgWork() {
  if (graph) cudaGraphExecDestroy(graph);
  if (h_st) cudaFreeHost(h_st);
}

static void enqueue_iteration(CgWork& w, const double* vals, const Precond* P, cudaStream_t s) {
  NodeRows A = w.m->rows();
  const int n = (int)w.n;
  const int sg = spmv_grid(A.nv), vg = vec_grid(n);
  (note_launch(), k_cg_Ap<<<sg, TPB, 0, s>>>(A, vals, w.p.p, w.Ap.p, w.partials.p, w.counter.p, w.st.p));
  const int kind = P ? P->kind : PREC_NONE;
  if (kind == PREC_SCHWARZ) {
    (note_launch(), k_cg_update<<<vg, TPB, 0, s>>>(n, 0, nullptr, w.x.p, w.r.p, w.p.p, w.Ap.p, w.z.p, w.partials.p, w.counter.p,
                                   w.st.p));
    NodeRows PR = P->rows();
    (note_launch(), k_cg_prec_spmv<<<spmv_grid(PR.nv), TPB, 0, s>>>(PR, P->vals.p, w.r.p, w.z.p, w.partials.p, w.counter.p, w.st.p, 0));
  } else {
    int mode = kind == PREC_DIAGONAL ? 2 : 1;
    (note_launch(), k_cg_update<<<vg, TPB, 0, s>>>(n, mode, kind == PREC_DIAGONAL ? P->diag.p : nullptr, w.x.p, w.r.p, w.p.p, w.Ap.p,
                                   w.z.p, w.partials.p, w.counter.p, w.st.p));
  }
  (note_launch(), k_cg_p<<<vg, TPB, 0, s>>>(n, w.z.p, w.p.p, w.st.p));
}

int cg_solve(CgWork& w, const double* vals, const Precond* P, double tol, i64 max_iter, i64* iters, cudaStream_t s) {
  NodeRows A = w.m->rows();
  const int n = (int)w.n;
  const int kind = P ? P->kind : PREC_NONE;
  HOEFEM_REQUIRE(!P || P->ready, HOEFEM_ERR_INVALID_ARGUMENT, "preconditioner has not been updated");
  // state
  CgState init{};
  init.tol = tol;
  init.max_iter = max_iter;
  HOEFEM_CUDA(cudaMemcpyAsync(w.st.p, &init, sizeof(CgState), cudaMemcpyHostToDevice, s));
  const int sg = spmv_grid(A.nv), vg = vec_grid(n);
  (note_launch(), k_cg_init<<<sg, TPB, 0, s>>>(A, vals, w.x.p, w.b.p, w.r.p, w.partials.p, w.counter.p, w.st.p));
  if (kind == PREC_SCHWARZ) {
    NodeRows PR = P->rows();
    (note_launch(), k_cg_prec_spmv<<<spmv_grid(PR.nv), TPB, 0, s>>>(PR, P->vals.p, w.r.p, w.z.p, w.partials.p, w.counter.p, w.st.p, 1));
  } else {
    (note_launch(), k_cg_prec_vec<<<vg, TPB, 0, s>>>(n, kind == PREC_DIAGONAL ? 1 : 0, kind == PREC_DIAGONAL ? P->diag.p : nullptr,
                                     w.r.p, w.z.p, w.partials.p, w.counter.p, w.st.p, 1));
  }
  (note_launch(), k_cg_copy<<<vg, TPB, 0, s>>>(n, w.z.p, w.p.p));
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
  // (re)build the chunk graph when the operator / preconditioner changed
  const void* key0 = vals;
  const void* key1 = P ? (const void*)P : nullptr;
  const void* key2 = P ? (kind == PREC_SCHWARZ ? (const void*)P->vals.p : (const void*)P->diag.p) : nullptr;
  if (!w.graph || w.graph_key[0] != key0 || w.graph_key[1] != key1 || w.graph_key[2] != key2 || w.graph_kind != kind) {
    if (w.graph) { cudaGraphExecDestroy(w.graph); w.graph = nullptr; }
    cudaStream_t cs;
    HOEFEM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    HOEFEM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    g_capture_count = 0;
    for (int k = 0; k < w.chunk; ++k) enqueue_iteration(w, vals, P, cs);
    w.graph_kernels = g_capture_count;
    g_capture_count = -1;
    HOEFEM_CUDA(cudaStreamEndCapture(cs, &g));
    HOEFEM_CUDA(cudaGraphInstantiate(&w.graph, g, 0));
    cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    w.graph_key[0] = key0;
    w.graph_key[1] = key1;
    w.graph_key[2] = key2;
    w.graph_kind = kind;
  }
  const i64 max_chunks = max_iter >= 0 ? (max_iter + w.chunk - 1) / w.chunk + 2 : (i64)1 << 40;
  for (i64 c = 0; c < max_chunks; ++c) {
    HOEFEM_CUDA(cudaGraphLaunch(w.graph, s));
    g_launch_count.fetch_add(w.graph_kernels, std::memory_order_relaxed);
    HOEFEM_CUDA(cudaMemcpyAsync(w.h_st, w.st.p, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    HOEFEM_CUDA(cudaStreamSynchronize(s));
    if (w.h_st->done) break;
  }
  *iters = w.h_st->iters;
  if (!w.h_st->done) return HOEFEM_CG_MAX_ITERATIONS;
  return w.h_st->status;
}

}  // namespace hoefem
