// Batched Newton-CG steps of many independent scenes.
//
// Not in the reference (its integrator advances one model at a time,
// simulation_toolbox/src/fem/newton_cg.rs:43-106); each scene follows the
// same path as a single NewtonCgIntegrator3d step with the diagonal
// preconditioner (the reference's choice without a Schwarz component,
// newton_cg.rs:137-143).
//
// The scenes are concatenated into one model (node ranges are contiguous per
// scene; Tet10 and Hex27 elements form one block each, with per-element Lame
// parameters).  Greedy first-fit coloring of the concatenated element list
// gives every scene exactly its own coloring (scenes share no node), so one
// launch per color serves all scenes and every scene's assembly is the one it
// would get alone.  Everything per scene (Dirichlet diagonal scale,
// representative force, Newton tolerance, residual norms, line-search
// parameter, CG scalars and stopping tests) lives in per-scene arrays; the
// reductions are segmented (one block per scene over its contiguous node
// range, fixed order) so each scene's result is deterministic and independent
// of the others.  Converged scenes are masked out of further updates.  The CG
// iterations of all scenes advance together, either in CUDA-graph chunks of
// per-phase kernels or inside one persistent cooperative launch per solve;
// an autotuner times both (the persistent one at each grid size) on the first
// solve.  The engines share every arithmetic step, so they give the same bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>

#include "internal.h"
#include "kernels_common.cuh"
#include "solver.h"
#include "stream_pipe.cuh"

namespace hoefem {

int spmv_grid(int nv, int lanes);
void greedy_coloring(const i64* conn, i64 ne, int nn, i64 nv, std::vector<i64>& color_off,
                     std::vector<int>& color_elems);

namespace {

constexpr int TPB = 256;

struct SegCg {
  double bnorm, zTr, pAp, rr, alpha, beta;
  long long iters;
  int done;  // 0 running, 1 finished, 2 zero rhs
  int status;
};

// ---- node chunks --------------------------------------------------------------
// Every scene's node range is split into chunks of at most CHN nodes; chunk c
// covers nodes [clo[c], clo[c + 1]) of scene cscene[c] and scene s owns chunks
// [cs_off[s], cs_off[s + 1]).  The CG kernels run one CTA per chunk: a CTA
// whose scene has finished returns at once, so an iteration costs what the
// active scenes need (no node scan, no shared work counter), and each CTA
// writes its chunk's partial sums cpart[k * nch + c].  The per-scene sums add
// a scene's chunk partials in chunk order: deterministic, and independent of
// the other scenes.
constexpr int CHN = 256;

struct Chunks {
  const int* lo;     // nch + 1
  const int* scene;  // nch
  const int* cs_off;  // nscene + 1
  int n;
};

// The chunk's nodes with LaneCfg<L>::lanes lanes per node: body(a, sl), a = -1
// for lanes without a node (all lanes of a warp take part).
template <int L, class F>
__device__ __forceinline__ void for_chunk_nodes(int lo, int hi, F&& body) {
  constexpr int LNS = LaneCfg<L>::lanes;
  constexpr int G = 32 / LNS;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int grp = lane / LNS, sl = lane % LNS;
  for (int a0 = lo + w * G; a0 < hi; a0 += nw * G) {
    const int a = a0 + grp;
    body(a < hi ? a : -1, sl);
  }
}

template <int K>
__device__ __forceinline__ void chunk_store(double (&acc)[K], double* __restrict__ cpart, int nch, int c) {
  block_sum<K>(acc);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) cpart[(size_t)k * nch + c] = acc[k];
}

// per-scene sums of the chunk partials (block per scene, fixed order)
template <int K>
__device__ __forceinline__ void scene_sum(const Chunks ch, const double* __restrict__ cpart, int s,
                                          double (&out)[K]) {
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  for (int c = ch.cs_off[s] + threadIdx.x; c < ch.cs_off[s + 1]; c += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] += cpart[(size_t)k * ch.n + c];
  block_sum<K>(acc);
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = acc[k];
}

// The same sums by one warp (lane-strided over the scene's chunks, then the
// xor tree): the CG scalars of both engines come from here.
template <int K>
__device__ __forceinline__ void scene_sum_warp(const Chunks ch, const double* __restrict__ cpart, int s,
                                               double (&out)[K]) {
  const int lane = threadIdx.x & 31;
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  for (int c = ch.cs_off[s] + lane; c < ch.cs_off[s + 1]; c += 32)
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] += cpart[(size_t)k * ch.n + c];
#pragma unroll
  for (int k = 0; k < K; ++k) out[k] = warp_sum_d(acc[k]);
}

// The scalar step of a running scene (cg.rs:376-482 per scene) from its sums v.
// mode 0: init (b.b, r.r) ; 1: zTr init ; 2: pAp -> alpha ; 3: (r.r, z.r) ->
// convergence, beta.
__device__ __forceinline__ void scene_update(int mode, SegCg& c, const double (&v)[2], double tol,
                                             long long max_iter) {
  if (mode == 0) {
    c.bnorm = sqrt(v[0]);
    c.rr = v[1];
  } else if (mode == 1) {
    c.zTr = v[0];
    c.iters = 0;
    c.status = HOEFEM_OK;
    if (c.bnorm == 0.0) { c.done = 2; return; }
    if (sqrt(c.rr) <= tol * c.bnorm) { c.done = 1; return; }
    if (max_iter >= 0 && c.iters >= max_iter) { c.done = 1; c.status = HOEFEM_CG_MAX_ITERATIONS; }
  } else if (mode == 2) {
    c.pAp = v[0];
    if (v[0] <= 0.0) { c.done = 1; c.status = HOEFEM_CG_INDEFINITE_OPERATOR; }
    else if (c.zTr <= 0.0) { c.done = 1; c.status = HOEFEM_CG_INDEFINITE_PRECONDITIONER; }
    else c.alpha = c.zTr / v[0];
  } else {
    c.rr = v[0];
    c.iters += 1;
    if (sqrt(v[0]) <= tol * c.bnorm) { c.done = 1; c.status = HOEFEM_OK; }
    else if (max_iter >= 0 && c.iters >= max_iter) { c.done = 1; c.status = HOEFEM_CG_MAX_ITERATIONS; }
    else {
      c.beta = v[1] / c.zTr;
      c.zTr = v[1];
    }
  }
}

// Scenes already finished (or masked out) keep their state; mode 1 resets
// their iteration count and status.
__device__ __forceinline__ void scene_finalize_warp(int mode, const Chunks ch, const double* __restrict__ cpart,
                                                    SegCg& c, int s, double tol, long long max_iter) {
  const int lane = threadIdx.x & 31;
  if (c.done) {
    if (mode == 1 && lane == 0) {
      c.iters = 0;
      c.status = HOEFEM_OK;
    }
    return;
  }
  double v[2];
  scene_sum_warp<2>(ch, cpart, s, v);
  if (lane == 0) scene_update(mode, c, v, tol, max_iter);
}

// one warp per scene
__global__ void k_seg_finalize(int mode, const Chunks ch, const double* __restrict__ cpart, SegCg* st, double tol,
                               long long max_iter) {
  const int s = blockIdx.x;
  scene_finalize_warp(mode, ch, cpart, st[s], s, tol, max_iter);
}

// The operand x of the node-row products: a vector, or the next search
// direction z + beta p formed on the fly (p = z in the first iteration).
struct XVec {
  const double* __restrict__ v;
  __device__ __forceinline__ double operator()(long long k) const { return v[k]; }
};
struct XDir {
  const double* __restrict__ z;
  const double* __restrict__ p;
  double beta;
  int first;
  __device__ __forceinline__ double operator()(long long k) const { return first ? z[k] : fma(beta, p[k], z[k]); }
};

// node_row_dot (the same traversals and sums) with the operand read through
// an accessor.
template <int L, class X>
__device__ __forceinline__ void node_row_dot_x(const NodeRows& A, const double* __restrict__ vals, const X& x, int a,
                                               int sl, double& s0, double& s1, double& s2) {
  constexpr int LNS = LaneCfg<L>::lanes;
  s0 = s1 = s2 = 0.0;
  if (a >= 0) {
    const long long b = A.base[a];
    if (A.diag_only && A.diag_only[a]) {
      if (sl == 0) {
        s0 = vals[b] * x(3LL * a);
        s1 = vals[b + 1] * x(3LL * a + 1);
        s2 = vals[b + 2] * x(3LL * a + 2);
      }
    } else if constexpr (LaneCfg<L>::stream) {
      const int o = A.adj_off[a], d = A.adj_off[a + 1] - o;
      const int rl = 3 * d;
      const double* r0 = vals + b;
#pragma unroll 4
      for (int c = sl; c < rl; c += LNS) {
        const int s = c / 3, j = c - 3 * s;
        const double xv = x(3LL * A.adj[o + s] + j);
        s0 += r0[c] * xv;
        s1 += r0[rl + c] * xv;
        s2 += r0[2 * rl + c] * xv;
      }
    } else {
      const int o = A.adj_off[a], d = A.adj_off[a + 1] - o;
      const long long rl = 3LL * d;
#pragma unroll 2
      for (int s = sl; s < d; s += LNS) {
        const long long nb = A.adj[o + s];
        const double x0 = x(3 * nb), x1 = x(3 * nb + 1), x2 = x(3 * nb + 2);
        const double* r0 = vals + b + 3 * s;
        s0 += r0[0] * x0 + r0[1] * x1 + r0[2] * x2;
        const double* r1 = r0 + rl;
        s1 += r1[0] * x0 + r1[1] * x1 + r1[2] * x2;
        const double* r2 = r1 + rl;
        s2 += r2[0] * x0 + r2[1] * x1 + r2[2] * x2;
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

// ---- per-chunk CG steps (chunk c of a running scene, the whole CTA) --------------

// r = b - A x ; chunk partials b.b, r.r
template <int L>
__device__ __forceinline__ void chunk_init(const NodeRows& A, const double* __restrict__ vals,
                                           const double* __restrict__ x, const double* __restrict__ b,
                                           double* __restrict__ r, const Chunks ch, double* __restrict__ cpart, int c) {
  double acc[2] = {0.0, 0.0};
  const XVec xv{x};
  for_chunk_nodes<L>(ch.lo[c], ch.lo[c + 1], [&](int a, int sl) {
    double s[3];
    node_row_dot_x<L>(A, vals, xv, a, sl, s[0], s[1], s[2]);
    if (a >= 0 && sl == 0) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double bi = b[3 * a + i], ri = bi - s[i];
        r[3 * a + i] = ri;
        acc[0] = fma(bi, bi, acc[0]);
        acc[1] = fma(ri, ri, acc[1]);
      }
    }
  });
  chunk_store<2>(acc, cpart, ch.n, c);
}

// z = d r (and p = z when p is given) ; chunk partials z.r
__device__ __forceinline__ void chunk_prec0(const Chunks ch, const double* __restrict__ d,
                                            const double* __restrict__ r, double* __restrict__ z,
                                            double* __restrict__ p, double* __restrict__ cpart, int c) {
  double acc[2] = {0.0, 0.0};
  for (int k = 3 * ch.lo[c] + threadIdx.x; k < 3 * ch.lo[c + 1]; k += blockDim.x) {
    double zi = d[k] * r[k];
    z[k] = zi;
    if (p) p[k] = zi;
    acc[0] = fma(zi, r[k], acc[0]);
  }
  chunk_store<2>(acc, cpart, ch.n, c);
}

// Ap = A p with p read through `pa` (and written to pout when given) ;
// chunk partials p.Ap
template <int L, class X>
__device__ __forceinline__ void chunk_Ap(const NodeRows& A, const double* __restrict__ vals, const X& pa,
                                         double* __restrict__ pout, double* __restrict__ Ap, const Chunks ch,
                                         double* __restrict__ cpart, int c) {
  double acc[2] = {0.0, 0.0};
  for_chunk_nodes<L>(ch.lo[c], ch.lo[c + 1], [&](int a, int sl) {
    double s[3];
    node_row_dot_x<L>(A, vals, pa, a, sl, s[0], s[1], s[2]);
    if (a >= 0 && sl == 0) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double pi = pa(3LL * a + i);
        if (pout) pout[3 * a + i] = pi;
        Ap[3 * a + i] = s[i];
        acc[0] = fma(pi, s[i], acc[0]);
      }
    }
  });
  chunk_store<2>(acc, cpart, ch.n, c);
}

// x += alpha p ; r -= alpha Ap ; z = d r ; chunk partials r.r, z.r
__device__ __forceinline__ void chunk_update(const Chunks ch, double al, const double* __restrict__ d,
                                             double* __restrict__ x, double* __restrict__ r,
                                             const double* __restrict__ p, const double* __restrict__ Ap,
                                             double* __restrict__ z, double* __restrict__ cpart, int c) {
  double acc[2] = {0.0, 0.0};
  for (int k = 3 * ch.lo[c] + threadIdx.x; k < 3 * ch.lo[c + 1]; k += blockDim.x) {
    x[k] = fma(al, p[k], x[k]);
    const double ri = fma(-al, Ap[k], r[k]);
    r[k] = ri;
    const double zi = d[k] * ri;
    z[k] = zi;
    acc[0] = fma(ri, ri, acc[0]);
    acc[1] = fma(zi, ri, acc[1]);
  }
  chunk_store<2>(acc, cpart, ch.n, c);
}

// ---- graph engine: one kernel per phase, one CTA per chunk ------------------------

template <int L>
__global__ void __launch_bounds__(TPB) k_seg_init(NodeRows A, const double* __restrict__ vals,
                                                  const double* __restrict__ x, const double* __restrict__ b,
                                                  double* __restrict__ r, const Chunks ch, const SegCg* __restrict__ st,
                                                  double* __restrict__ cpart) {
  const int c = blockIdx.x;
  if (st[ch.scene[c]].done) return;
  chunk_init<L>(A, vals, x, b, r, ch, cpart, c);
}

__global__ void __launch_bounds__(TPB) k_seg_prec0(const Chunks ch, const SegCg* __restrict__ st,
                                                   const double* __restrict__ d, const double* __restrict__ r,
                                                   double* __restrict__ z, double* __restrict__ p,
                                                   double* __restrict__ cpart) {
  const int c = blockIdx.x;
  if (st[ch.scene[c]].done) return;
  chunk_prec0(ch, d, r, z, p, cpart, c);
}

template <int L>
__global__ void __launch_bounds__(TPB) k_seg_Ap(NodeRows A, const double* __restrict__ vals,
                                                const double* __restrict__ p, double* __restrict__ Ap, const Chunks ch,
                                                const SegCg* __restrict__ st, double* __restrict__ cpart) {
  const int c = blockIdx.x;
  if (st[ch.scene[c]].done) return;
  chunk_Ap<L>(A, vals, XVec{p}, nullptr, Ap, ch, cpart, c);
}

__global__ void __launch_bounds__(TPB) k_seg_update(const Chunks ch, const SegCg* __restrict__ st,
                                                    const double* __restrict__ d, double* __restrict__ x,
                                                    double* __restrict__ r, const double* __restrict__ p,
                                                    const double* __restrict__ Ap, double* __restrict__ z,
                                                    double* __restrict__ cpart) {
  const int c = blockIdx.x;
  const SegCg& sc = st[ch.scene[c]];
  if (sc.done) return;
  chunk_update(ch, sc.alpha, d, x, r, p, Ap, z, cpart, c);
}

// p = z + beta p
__global__ void __launch_bounds__(TPB) k_seg_p(const Chunks ch, const SegCg* __restrict__ st,
                                               const double* __restrict__ z, double* __restrict__ p) {
  const int c = blockIdx.x;
  const SegCg& sc = st[ch.scene[c]];
  if (sc.done) return;
  const double be = sc.beta;
  for (int k = 3 * ch.lo[c] + threadIdx.x; k < 3 * ch.lo[c + 1]; k += blockDim.x) p[k] = fma(be, p[k], z[k]);
}

// ---- persistent engine: one cooperative launch per solve --------------------------
// In every phase the CTAs claim chunks from a shared counter (the work of the
// scenes still running spreads over all CTAs).  Between phases a grid barrier: the last CTA
// to arrive applies the scene updates (one warp per scene, the same sums and
// steps as k_seg_finalize) and counts the scenes still running before it
// releases the others.  The search direction is double-buffered and formed on
// the fly inside A p (z + beta p_old), which drops the third barrier of the
// graph engine's iteration.  Every wait is bounded (2 s): a wait that runs
// out raises `abort`, and every CTA returns.
struct SegGrid {
  unsigned count;  // CTAs arrived at the current barrier
  unsigned gen;    // barrier generation
  int active;      // scenes still running after the last scene update
  int abort;       // a wait ran out
  int next;        // next chunk to claim in the current phase
};

struct PersistArgs {
  NodeRows A;
  const double* vals;
  const double* d;
  const double* b;
  double* x;
  double* r;
  double* z;
  double* p0;
  double* p1;
  double* Ap;
  double* cpart;
  Chunks ch;
  SegCg* st;
  int nscene;
  double tol;
  long long max_iter;
  long long max_loop;  // bound on the kernel's own iterations
  SegGrid* g;
};

// The last CTA's scene updates: each warp takes SPW scenes at a time and issues
// all their loads before the sums (the same lane-strided sums and xor trees as
// scene_finalize_warp, so the same bits), then the count of running scenes.
__device__ void persist_scene_updates(const PersistArgs& P, int mode) {
  constexpr int SPW = 4;
  __shared__ int s_cnt;
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const Chunks ch = P.ch;
  int cnt = 0;
  for (int s0 = w * SPW; s0 < P.nscene; s0 += nw * SPW) {
    int lo[SPW], hi[SPW], run[SPW];
#pragma unroll
    for (int j = 0; j < SPW; ++j) {
      const int s = s0 + j;
      run[j] = s < P.nscene ? (P.st[s].done == 0) : 0;
      lo[j] = s < P.nscene ? ch.cs_off[s] : 0;
      hi[j] = s < P.nscene ? ch.cs_off[s + 1] : 0;
    }
    double acc[SPW][2];
#pragma unroll
    for (int j = 0; j < SPW; ++j) {
      acc[j][0] = acc[j][1] = 0.0;
      if (run[j])
        for (int c = lo[j] + lane; c < hi[j]; c += 32) {
          acc[j][0] += P.cpart[c];
          acc[j][1] += P.cpart[(size_t)ch.n + c];
        }
    }
#pragma unroll
    for (int j = 0; j < SPW; ++j) {
      const double v[2] = {warp_sum_d(acc[j][0]), warp_sum_d(acc[j][1])};
      const int s = s0 + j;
      if (lane == 0 && s < P.nscene) {
        SegCg& c = P.st[s];
        if (run[j]) scene_update(mode, c, v, P.tol, P.max_iter);
        else if (mode == 1) {
          c.iters = 0;
          c.status = HOEFEM_OK;
        }
        if (!c.done) ++cnt;
      }
    }
  }
  if (lane == 0 && cnt) atomicAdd(&s_cnt, cnt);
  __syncthreads();
  if (threadIdx.x == 0) P.g->active = s_cnt;
}

// Grid barrier with the scene updates of `mode`; false if a wait ran out.
// The last CTA also resets the chunk counter of the next phase.
__device__ bool persist_sync(const PersistArgs& P, int mode) {
  __shared__ int s_last, s_ok;
  __shared__ unsigned s_gen;
  __syncthreads();
  if (threadIdx.x == 0) {
    s_gen = *(volatile unsigned*)&P.g->gen;
    __threadfence();
    s_last = atomicAdd(&P.g->count, 1u) == gridDim.x - 1u;
    s_ok = 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    persist_scene_updates(P, mode);
    if (threadIdx.x == 0) {
      P.g->count = 0u;
      P.g->next = 0;
      __threadfence();
      atomicAdd(&P.g->gen, 1u);
    }
  } else if (threadIdx.x == 0) {
    const uint64_t t0 = pipe::clock_ns();
    for (;;) {
      if (*(volatile unsigned*)&P.g->gen != s_gen) break;
      if (*(volatile int*)&P.g->abort) {
        s_ok = 0;
        break;
      }
      if (pipe::clock_ns() - t0 > pipe::HOEFEM_WAIT_NS) {
        atomicExch(&P.g->abort, 1);
        s_ok = 0;
        break;
      }
      __nanosleep(128);
    }
    __threadfence();
  }
  __syncthreads();
  return s_ok != 0;
}

// The chunks of a phase, claimed one at a time from the shared counter
// (dynamic balance: chunk costs differ by element kind and scenes finish at
// different iterations); body(c) for every claimed chunk of a running scene.
template <class F>
__device__ __forceinline__ void persist_chunks(const PersistArgs& P, F&& body) {
  __shared__ int s_chunk;
  for (;;) {
    if (threadIdx.x == 0) s_chunk = atomicAdd(&P.g->next, 1);
    __syncthreads();
    const int c = s_chunk;
    __syncthreads();
    if (c >= P.ch.n) break;
    const SegCg& sc = P.st[P.ch.scene[c]];
    if (!sc.done) body(c, sc);
  }
}

template <int L>
__global__ void __launch_bounds__(TPB, 5) k_seg_persistent(const PersistArgs P) {
  const Chunks ch = P.ch;
  persist_chunks(P, [&](int c, const SegCg&) { chunk_init<L>(P.A, P.vals, P.x, P.b, P.r, ch, P.cpart, c); });
  if (!persist_sync(P, 0)) return;
  persist_chunks(P, [&](int c, const SegCg&) { chunk_prec0(ch, P.d, P.r, P.z, nullptr, P.cpart, c); });
  if (!persist_sync(P, 1)) return;
  for (long long it = 0; it < P.max_loop; ++it) {
    if (*(volatile int*)&P.g->active == 0) break;
    const double* pold = (it & 1) ? P.p1 : P.p0;
    double* pnew = (it & 1) ? P.p0 : P.p1;
    persist_chunks(P, [&](int c, const SegCg& sc) {
      const XDir pa{P.z, pold, sc.beta, it == 0 ? 1 : 0};
      chunk_Ap<L>(P.A, P.vals, pa, pnew, P.Ap, ch, P.cpart, c);
    });
    if (!persist_sync(P, 2)) return;
    persist_chunks(P, [&](int c, const SegCg& sc) {
      chunk_update(ch, sc.alpha, P.d, P.x, P.r, pnew, P.Ap, P.z, P.cpart, c);
    });
    if (!persist_sync(P, 3)) return;
  }
}

template <int L>
int persistent_blocks_per_sm() {
  int occ = 0;
  HOEFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_seg_persistent<L>, TPB, 0));
  return occ;
}

template <int L>
void launch_persistent(const PersistArgs& args, int G, cudaStream_t s) {
  PersistArgs a = args;
  void* kargs[] = {&a};
  note_launch();
  HOEFEM_CUDA(cudaLaunchCooperativeKernel((const void*)k_seg_persistent<L>, G, TPB, kargs, 0, s));
}

// per-scene sum of squares of a vector into out[s]: chunk partials, then scenes
__global__ void __launch_bounds__(TPB) k_chunk_norm2(const Chunks ch, const double* __restrict__ v,
                                                     double* __restrict__ cpart) {
  const int c = blockIdx.x;
  double acc[1] = {0.0};
  for (int k = 3 * ch.lo[c] + threadIdx.x; k < 3 * ch.lo[c + 1]; k += blockDim.x) acc[0] += v[k] * v[k];
  chunk_store<1>(acc, cpart, ch.n, c);
}

__global__ void k_seg_norm2(const Chunks ch, const double* __restrict__ cpart, double* __restrict__ out) {
  double v[1];
  scene_sum<1>(ch, cpart, blockIdx.x, v);
  if (threadIdx.x == 0) out[blockIdx.x] = v[0];
}

// Dirichlet with a per-scene diagonal scale (first non-zero diagonal of the scene)
__global__ void k_seg_first_diag(NodeRows A, const double* __restrict__ vals, const int* __restrict__ scene_of,
                                 unsigned long long* first) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < A.nv; a += gridDim.x * blockDim.x) {
    int s = A.diag_slot[a];
    if (s < 0) continue;
    int d = A.adj_off[a + 1] - A.adj_off[a];
    for (int i = 0; i < 3; ++i) {
      double v = vals[A.base[a] + (long long)i * 3 * d + 3 * s + i];
      if (v != 0.0) {
        atomicMin(first + scene_of[a], (unsigned long long)(3 * a + i));
        break;
      }
    }
  }
}

__global__ void k_seg_scale(int nscene, NodeRows A, const double* __restrict__ vals,
                            const unsigned long long* __restrict__ first, double* __restrict__ scale) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nscene) return;
  unsigned long long f = first[s];
  double sc = 1.0;
  if (f != ~0ull) {
    int a0 = (int)(f / 3), i0 = (int)(f % 3);
    int d0 = A.adj_off[a0 + 1] - A.adj_off[a0];
    sc = fabs(vals[A.base[a0] + (long long)i0 * 3 * d0 + 3 * A.diag_slot[a0] + i0]);
  }
  scale[s] = sc;
}

__global__ void k_seg_dirichlet(NodeRows A, const unsigned char* __restrict__ bc, const int* __restrict__ scene_of,
                                const double* __restrict__ scale, double* __restrict__ vals) {
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  for (int a = blockIdx.x * wpb + (threadIdx.x >> 5); a < A.nv; a += gridDim.x * wpb) {
    const int o = A.adj_off[a], d = A.adj_off[a + 1] - o;
    const long long b = A.base[a];
    const double sc = scale[scene_of[a]];
    for (int i = 0; i < 3; ++i) {
      const int r = 3 * a + i;
      const bool rbc = bc[r];
      for (int s = lane; s < d; s += 32) {
        const int nb = A.adj[o + s];
        for (int j = 0; j < 3; ++j) {
          const int c = 3 * nb + j;
          long long k = b + (long long)i * 3 * d + 3 * s + j;
          if (rbc) vals[k] = (c == r) ? sc : 0.0;
          else if (bc[c]) vals[k] = 0.0;
        }
      }
    }
  }
}

__global__ void k_combine2(long long nnz, double ck, const double* __restrict__ K, const double* __restrict__ M,
                           double* __restrict__ out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (K) v += ck * K[k];
    v += 1.0 * M[k];
    out[k] = v;
  }
}

__global__ void k_diag_inv(NodeRows A, const int* __restrict__ scene_of, const double* __restrict__ J,
                           double* __restrict__ d, int* err) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * A.nv) return;
  int a = t / 3, i = t % 3;
  double v = 0.0;
  int s = A.diag_slot[a];
  if (s >= 0) {
    int dd = A.adj_off[a + 1] - A.adj_off[a];
    v = J[A.base[a] + (long long)i * 3 * dd + 3 * s + i];
  }
  if (v != 0.0) d[t] = 1.0 / v;
  else {
    d[t] = 0.0;
    atomicCAS(err + scene_of[a], 0, HOEFEM_ERR_ZERO_DIAGONAL);
  }
}

// vector ops with per-scene coefficients / masks (scene of a dof = scene_of[dof / 3])
__global__ void k_seg_state(int n, const int* __restrict__ scene_of, const double* __restrict__ up,
                            const double* __restrict__ vn, const double* __restrict__ w, double dt,
                            const unsigned char* __restrict__ bc, double* __restrict__ us, double* __restrict__ vs) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double uu = up[i] + w[i] * dt, vv = vn[i] + w[i];
    if (bc[i]) { uu = 0.0; vv = 0.0; }
    us[i] = uu;
    vs[i] = vv;
  }
}

__global__ void k_seg_axpy(int n, const int* __restrict__ scene_of, const double* __restrict__ coef,
                           const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double c = coef[scene_of[i / 3]];
    if (c != 0.0) y[i] = c * x[i] + 1.0 * y[i];
  }
}

__global__ void k_vcopy(int n, const double* __restrict__ a, double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

__global__ void k_F2(int n, const double* __restrict__ f, const unsigned char* __restrict__ bc, double dt,
                     double* __restrict__ F) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double fi = bc[i] ? 0.0 : f[i];
    F[i] = fi * (dt * -1.0);
  }
}

__global__ void k_be_init2(int n, const double* __restrict__ u, const double* __restrict__ v, double dt,
                           double* __restrict__ up, double* __restrict__ vn, double* __restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    vn[i] = v[i];
    up[i] = u[i] + v[i] * dt;
    w[i] = 0.0;
  }
}

__global__ void k_be_final2(int n, const int* __restrict__ scene_of, const unsigned char* __restrict__ ok,
                            const double* __restrict__ w, double dt, const unsigned char* __restrict__ bc,
                            double* __restrict__ u, double* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!ok[scene_of[i / 3]]) continue;
    double vv = v[i] + w[i];
    double uu = u[i] + vv * dt;
    if (bc[i]) { uu = 0.0; vv = 0.0; }
    v[i] = vv;
    u[i] = uu;
  }
}

__global__ void k_bc_uv2(int n, const unsigned char* __restrict__ bc, double* __restrict__ u, double* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (bc[i]) {
      u[i] = 0.0;
      v[i] = 0.0;
    }
}

__global__ void k_masked_copy(int n, const int* __restrict__ scene_of, const unsigned char* __restrict__ mask,
                              const double* __restrict__ a, double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (mask[scene_of[i / 3]]) b[i] = a[i];
}

__global__ void k_fillv(int n, double v, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

__global__ void k_gdens(int n, double g, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = (i % 3 == 2) ? g : 0.0;
}

__global__ void k_seg_mask_done(int nscene, const unsigned char* __restrict__ active, SegCg* st) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nscene) st[s].done = active[s] ? 0 : 1;
}

}  // namespace

struct Batch {
  Model m;
  int nscene = 0;
  std::vector<int> node_off;  // nscene + 1
  std::vector<int> scene_of;  // per node
  std::vector<unsigned char> bc_host;
  int mat_kind = HOEFEM_MAT_SNH;
  double density = 1000.0, gravity = -9.81;
  double cg_tol = 1e-5;
  i64 cg_max = 500, newton_max = 100;
  int chunk = 8;
  // device
  DBuf<int> d_node_off, d_scene_of;
  DBuf<int> d_clo, d_cscene, d_cs_off;  // node chunks (see Chunks)
  int nch = 0;
  DBuf<unsigned char> d_bc, d_ok, d_active;
  DBuf<unsigned char> emask;  // scenes whose elements the force / stiffness kernels evaluate
  DBuf<double> M, K, J, gforce, up, vn, w, F, dx, us, vs, f, u, v, diag, x, b, r, z, p, Ap, cpart, scale, coef, nrm;
  DBuf<unsigned long long> first;
  DBuf<SegCg> st;
  DBuf<int> err;
  std::vector<double> rep;
  std::vector<SegCg> h_st;
  cudaGraphExec_t graph = nullptr;
  long long graph_kernels = 0;
  // CG engine: requested (HOEFEM_CG_ENGINE_*, CTAs per multiprocessor for the
  // persistent engine, 0 = as many as fit) and the autotuner's choice
  int cg_engine = HOEFEM_CG_ENGINE_AUTO, cg_ctas = 0;
  int tuned_engine = -1, tuned_ctas = 0, persist_occ = 0;
  std::vector<float> tune_ms;
  DBuf<double> p2;  // second search-direction buffer of the persistent engine
  DBuf<SegGrid> sgrid;
  // per-scene results of the last step
  std::vector<i64> st_newton, st_cg_solves, st_cg_total, st_cg_max, st_substeps;
  std::vector<int> status, st_cg_last;
  std::vector<double> st_residual;
  double ms_total = 0.0;
  ~Batch() {
    if (graph) cudaGraphExecDestroy(graph);
  }

  int vg() const { return reduce_blocks_for(m.ndof); }
  Chunks chunks() const { return Chunks{d_clo.p, d_cscene.p, d_cs_off.p, nch}; }

  void seg_norm2(const double* vec, std::vector<double>& out) {
    cudaStream_t s = m.stream;
    (note_launch(), k_chunk_norm2<<<nch, TPB, 0, s>>>(chunks(), vec, cpart.p));
    (note_launch(), k_seg_norm2<<<nscene, TPB, 0, s>>>(chunks(), cpart.p, nrm.p));
    out.resize(nscene);
    HOEFEM_CUDA(cudaMemcpyAsync(out.data(), nrm.p, sizeof(double) * nscene, cudaMemcpyDeviceToHost, s));
    HOEFEM_CUDA(cudaStreamSynchronize(s));
  }

  void dirichlet(double* vals) {
    cudaStream_t s = m.stream;
    NodeRows A = m.rows();
    std::vector<unsigned long long> init(nscene, ~0ull);
    HOEFEM_CUDA(cudaMemcpyAsync(first.p, init.data(), sizeof(unsigned long long) * nscene, cudaMemcpyHostToDevice, s));
    (note_launch(), k_seg_first_diag<<<(A.nv + 255) / 256, 256, 0, s>>>(A, vals, d_scene_of.p, first.p));
    (note_launch(), k_seg_scale<<<(nscene + 127) / 128, 128, 0, s>>>(nscene, A, vals, first.p, scale.p));
    (note_launch(), k_seg_dirichlet<<<spmv_grid(A.nv, 32), 256, 0, s>>>(A, d_bc.p, d_scene_of.p, scale.p, vals));
    HOEFEM_CUDA(cudaGetLastError());
  }

  void setup() {
    cudaStream_t s = m.stream;
    const int n = (int)m.ndof;
    d_node_off.upload(node_off, s);
    d_scene_of.upload(scene_of, s);
    {
      std::vector<int> clo, cscene, cs_off(1, 0);
      for (int k = 0; k < nscene; ++k) {
        for (int a = node_off[k]; a < node_off[k + 1]; a += CHN) {
          clo.push_back(a);
          cscene.push_back(k);
        }
        cs_off.push_back((int)clo.size());
      }
      nch = (int)clo.size();
      clo.push_back((int)m.nv);
      HOEFEM_REQUIRE(nch > 0, HOEFEM_ERR_INVALID_ARGUMENT, "batch without nodes");
      d_clo.upload(clo, s);
      d_cscene.upload(cscene, s);
      d_cs_off.upload(cs_off, s);
    }
    d_bc.upload(bc_host, s);
    for (auto* bf : {&M, &K, &J}) bf->alloc(m.nnz);
    for (auto* bf : {&gforce, &up, &vn, &w, &F, &dx, &us, &vs, &f, &u, &v, &diag, &x, &b, &r, &z, &p, &Ap})
      bf->alloc(n);
    cpart.alloc(2 * (size_t)nch);
    for (auto* bf : {&scale, &coef, &nrm}) bf->alloc(nscene);
    first.alloc(nscene);
    st.alloc(nscene);
    d_ok.alloc(nscene);
    d_active.alloc(nscene);
    err.alloc(nscene);
    err.zero(s);
    K.zero(s);
    launch_mass(m, density, K.p, s);
    HOEFEM_CUDA(cudaMemcpyAsync(M.p, K.p, sizeof(double) * m.nnz, cudaMemcpyDeviceToDevice, s));
    dirichlet(M.p);
    check_device_error(m);
    m.spmv_lanes = autotune_spmv_lanes(m.rows(), M.p, s);
    (note_launch(), k_fillv<<<vg(), TPB, 0, s>>>(n, std::sqrt((10.0 * 10.0) / 3.0), us.p));
    spmv_node_rows(m.rows(), M.p, us.p, vs.p, 1.0, 0.0, s);
    seg_norm2(vs.p, rep);
    for (double& x2 : rep) x2 = std::sqrt(x2);
    (note_launch(), k_gdens<<<vg(), TPB, 0, s>>>(n, gravity, us.p));
    spmv_node_rows(m.rows(), M.p, us.p, gforce.p, 1.0, 0.0, s);
    HOEFEM_CUDA(cudaStreamSynchronize(s));
  }

  void set_emask(const std::vector<unsigned char>& mask) {
    HOEFEM_CUDA(cudaMemcpyAsync(emask.p, mask.data(), nscene, cudaMemcpyHostToDevice, m.stream));
  }

  // F(w) for the scenes in `mask` (other scenes' entries are not meaningful);
  // returns per-scene ||F||^2
  void eval_F(double dt, const std::vector<unsigned char>& mask, std::vector<double>& fsq) {
    cudaStream_t s = m.stream;
    const int n = (int)m.ndof;
    set_emask(mask);
    (note_launch(), k_seg_state<<<vg(), TPB, 0, s>>>(n, d_scene_of.p, up.p, vn.p, w.p, dt, d_bc.p, us.p, vs.p));
    (note_launch(), k_vcopy<<<vg(), TPB, 0, s>>>(n, gforce.p, f.p));
    launch_forces(m, MatDev{mat_kind, 0.0, 0.0}, us.p, f.p, s);
    (note_launch(), k_F2<<<vg(), TPB, 0, s>>>(n, f.p, d_bc.p, dt, F.p));
    spmv_node_rows(m.rows(), M.p, w.p, F.p, 1.0, 1.0, s);
    check_device_error(m);
    seg_norm2(F.p, fsq);
  }

  void enqueue_iter(cudaStream_t s) {
    NodeRows A = m.rows();
    const Chunks ch = chunks();
    HOEFEM_LANES_DISPATCH(A.lanes, (note_launch(), k_seg_Ap<LN><<<nch, TPB, 0, s>>>(A, J.p, p.p, Ap.p, ch, st.p,
                                                                                   cpart.p)));
    (note_launch(), k_seg_finalize<<<nscene, 32, 0, s>>>(2, ch, cpart.p, st.p, cg_tol, cg_max));
    (note_launch(), k_seg_update<<<nch, TPB, 0, s>>>(ch, st.p, diag.p, x.p, r.p, p.p, Ap.p, z.p, cpart.p));
    (note_launch(), k_seg_finalize<<<nscene, 32, 0, s>>>(3, ch, cpart.p, st.p, cg_tol, cg_max));
    (note_launch(), k_seg_p<<<nch, TPB, 0, s>>>(ch, st.p, z.p, p.p));
  }

  void ensure_graph() {
    if (graph) return;
    cudaStream_t cs;
    HOEFEM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    HOEFEM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    g_capture_count = 0;
    for (int k = 0; k < chunk; ++k) enqueue_iter(cs);
    graph_kernels = g_capture_count;
    g_capture_count = -1;
    HOEFEM_CUDA(cudaStreamEndCapture(cs, &g));
    HOEFEM_CUDA(cudaGraphInstantiate(&graph, g, 0));
    cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
  }

  // the active scenes start from x = 0, the others are marked finished
  void cg_start(const std::vector<unsigned char>& active) {
    cudaStream_t s = m.stream;
    HOEFEM_CUDA(cudaMemcpyAsync(d_active.p, active.data(), nscene, cudaMemcpyHostToDevice, s));
    (note_launch(), k_seg_mask_done<<<(nscene + 127) / 128, 128, 0, s>>>(nscene, d_active.p, st.p));
    HOEFEM_CUDA(cudaMemsetAsync(x.p, 0, sizeof(double) * m.ndof, s));
  }

  // graph engine: the set-up kernels, then graphs of `chunk` iterations until
  // every scene has finished (the host reads the scene states between graphs)
  void cg_graphs() {
    cudaStream_t s = m.stream;
    NodeRows A = m.rows();
    const Chunks ch = chunks();
    HOEFEM_LANES_DISPATCH(A.lanes, (note_launch(), k_seg_init<LN><<<nch, TPB, 0, s>>>(A, J.p, x.p, b.p, r.p, ch,
                                                                                     st.p, cpart.p)));
    (note_launch(), k_seg_finalize<<<nscene, 32, 0, s>>>(0, ch, cpart.p, st.p, cg_tol, cg_max));
    (note_launch(), k_seg_prec0<<<nch, TPB, 0, s>>>(ch, st.p, diag.p, r.p, z.p, p.p, cpart.p));
    (note_launch(), k_seg_finalize<<<nscene, 32, 0, s>>>(1, ch, cpart.p, st.p, cg_tol, cg_max));
    HOEFEM_CUDA(cudaGetLastError());
    ensure_graph();
    h_st.resize(nscene);
    const i64 max_chunks = (cg_max >= 0 ? cg_max : 10 * m.ndof) / chunk + 2;
    for (i64 c = 0; c <= max_chunks; ++c) {
      HOEFEM_CUDA(cudaMemcpyAsync(h_st.data(), st.p, sizeof(SegCg) * nscene, cudaMemcpyDeviceToHost, s));
      HOEFEM_CUDA(cudaStreamSynchronize(s));
      bool all = true;
      for (auto& c2 : h_st) all = all && c2.done;
      if (all) break;
      HOEFEM_CUDA(cudaGraphLaunch(graph, s));
      g_launch_count.fetch_add(graph_kernels, std::memory_order_relaxed);
    }
    // zero-rhs scenes: x = 0 already (x was zeroed and never updated)
  }

  int persistent_occupancy() {
    if (persist_occ == 0) {
      HOEFEM_LANES_DISPATCH(m.rows().lanes, persist_occ = persistent_blocks_per_sm<LN>());
      HOEFEM_REQUIRE(persist_occ >= 1, HOEFEM_ERR_CUDA, "persistent batched CG kernel does not fit on a multiprocessor");
    }
    return persist_occ;
  }

  // persistent engine: one cooperative launch runs the whole solve of every
  // active scene with `per` CTAs per multiprocessor (0: as many as fit)
  void cg_persistent(int per) {
    cudaStream_t s = m.stream;
    NodeRows A = m.rows();
    const int occ = persistent_occupancy();
    per = per <= 0 ? occ : std::min(per, occ);
    const int G = std::max(1, std::min(nch, per * device_sms()));
    if (!p2.p) p2.alloc(m.ndof);
    if (!sgrid.p) sgrid.alloc(1);
    HOEFEM_CUDA(cudaMemsetAsync(sgrid.p, 0, sizeof(SegGrid), s));
    PersistArgs a;
    a.A = A;
    a.vals = J.p;
    a.d = diag.p;
    a.b = b.p;
    a.x = x.p;
    a.r = r.p;
    a.z = z.p;
    a.p0 = p.p;
    a.p1 = p2.p;
    a.Ap = Ap.p;
    a.cpart = cpart.p;
    a.ch = chunks();
    a.st = st.p;
    a.nscene = nscene;
    a.tol = cg_tol;
    a.max_iter = cg_max;
    a.max_loop = (cg_max >= 0 ? cg_max : 10 * m.ndof) + 2;
    a.g = sgrid.p;
    HOEFEM_LANES_DISPATCH(A.lanes, launch_persistent<LN>(a, G, s));
    h_st.resize(nscene);
    SegGrid hg;
    HOEFEM_CUDA(cudaMemcpyAsync(h_st.data(), st.p, sizeof(SegCg) * nscene, cudaMemcpyDeviceToHost, s));
    HOEFEM_CUDA(cudaMemcpyAsync(&hg, sgrid.p, sizeof(SegGrid), cudaMemcpyDeviceToHost, s));
    HOEFEM_CUDA(cudaStreamSynchronize(s));
    if (hg.abort) throw Error(HOEFEM_ERR_DEVICE_TIMEOUT, "persistent batched CG: device wait ran out");
  }

  void run_cg(const std::vector<unsigned char>& active, int engine, int per) {
    cg_start(active);
    if (engine == HOEFEM_CG_ENGINE_STREAMED) cg_persistent(per);
    else cg_graphs();
  }

  // Autotuner: the first solve runs once per candidate (the graph engine, then
  // the persistent engine at 1, 2, 4, ... CTAs per multiprocessor up to the
  // occupancy limit) and the fastest is kept.  Every candidate is a complete
  // solve of the same system with the same arithmetic, so the last one leaves
  // the result.
  void tune(const std::vector<unsigned char>& active) {
    cudaStream_t s = m.stream;
    ensure_graph();
    std::vector<std::pair<int, int>> cand = {{HOEFEM_CG_ENGINE_CHUNKED, 0}};
    const int occ = persistent_occupancy();
    for (int k = 1; k < occ; k *= 2) cand.push_back({HOEFEM_CG_ENGINE_STREAMED, k});
    cand.push_back({HOEFEM_CG_ENGINE_STREAMED, occ});
    cudaEvent_t e0, e1;
    HOEFEM_CUDA(cudaEventCreate(&e0));
    HOEFEM_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    tune_ms.clear();
    for (auto& c : cand) {
      HOEFEM_CUDA(cudaEventRecord(e0, s));
      run_cg(active, c.first, c.second);
      HOEFEM_CUDA(cudaEventRecord(e1, s));
      HOEFEM_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      HOEFEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      tune_ms.push_back(ms);
      if (ms < best) {
        best = ms;
        tuned_engine = c.first;
        tuned_ctas = c.second;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }

  // batched PCG with the diagonal preconditioner on J for the active scenes
  void cg(const std::vector<unsigned char>& active) {
    if (cg_engine != HOEFEM_CG_ENGINE_AUTO) return run_cg(active, cg_engine, cg_ctas);
    if (tuned_engine < 0) return tune(active);
    run_cg(active, tuned_engine, tuned_ctas);
  }

  // One backward-Euler step of the scenes in `part` (newton.rs:131-170 per
  // scene): per-scene status into status[], successful scenes' (u, v) advanced.
  void be_step(double dt, const std::vector<unsigned char>& part) {
    cudaStream_t s = m.stream;
    const int n = (int)m.ndof;
    (note_launch(), k_be_init2<<<vg(), TPB, 0, s>>>(n, u.p, v.p, dt, up.p, vn.p, w.p));
    std::vector<double> fsq, tol(nscene);
    for (int k = 0; k < nscene; ++k) tol[k] = dt * (1e-5 * rep[k]);
    eval_F(dt, part, fsq);
    std::vector<unsigned char> active(nscene);
    std::vector<i64> iter(nscene, 0);
    for (int k = 0; k < nscene; ++k)
      if (part[k]) status[k] = HOEFEM_OK;
    for (;;) {
      bool any = false;
      for (int k = 0; k < nscene; ++k) {
        active[k] = part[k] && status[k] == HOEFEM_OK && std::sqrt(fsq[k]) > tol[k];
        if (active[k] && iter[k] == newton_max) {
          status[k] = HOEFEM_NEWTON_MAX_ITERATIONS;
          active[k] = 0;
        }
        any = any || active[k];
      }
      if (!any) break;
      // J = dt^2 K + M with the per-scene Dirichlet scale, diagonal preconditioner
      (note_launch(), k_seg_state<<<vg(), TPB, 0, s>>>(n, d_scene_of.p, up.p, vn.p, w.p, dt, d_bc.p, us.p, vs.p));
      K.zero(s);
      set_emask(active);
      launch_stiffness(m, MatDev{mat_kind, 0.0, 0.0}, us.p, K.p, s);
      (note_launch(), k_combine2<<<device_sms() * 8, TPB, 0, s>>>(m.nnz, -(-dt * dt), K.p, M.p, J.p));
      dirichlet(J.p);
      (note_launch(), k_diag_inv<<<(n + 255) / 256, 256, 0, s>>>(m.rows(), d_scene_of.p, J.p, diag.p, err.p));
      check_device_error(m);
      std::vector<int> e(nscene);
      HOEFEM_CUDA(cudaMemcpyAsync(e.data(), err.p, sizeof(int) * nscene, cudaMemcpyDeviceToHost, s));
      HOEFEM_CUDA(cudaStreamSynchronize(s));
      bool zero_diag = false;
      for (int k = 0; k < nscene; ++k)
        if (e[k] && active[k]) {
          status[k] = e[k];
          active[k] = 0;
          zero_diag = true;
        }
      if (zero_diag || std::count(e.begin(), e.end(), 0) != nscene) err.zero(s);
      (note_launch(), k_vcopy<<<vg(), TPB, 0, s>>>(n, F.p, b.p));
      cg(active);
      for (int k = 0; k < nscene; ++k) {
        if (!active[k]) continue;
        st_cg_solves[k] += 1;
        st_cg_total[k] += h_st[k].iters;
        st_cg_max[k] = std::max<i64>(st_cg_max[k], h_st[k].iters);
        int cs = h_st[k].status;
        st_cg_last[k] = cs;
        // MaxIterationsReached and IndefiniteOperator are tolerated (newton_cg.rs:776-797)
        if (!(cs == HOEFEM_OK || cs == HOEFEM_CG_MAX_ITERATIONS || cs == HOEFEM_CG_INDEFINITE_OPERATOR)) {
          status[k] = cs;
          active[k] = 0;
        }
      }
      // dx = -x
      (note_launch(), k_fillv<<<vg(), TPB, 0, s>>>(n, 0.0, dx.p));
      std::vector<double> minus_one(nscene, -1.0);
      HOEFEM_CUDA(cudaMemcpyAsync(coef.p, minus_one.data(), sizeof(double) * nscene, cudaMemcpyHostToDevice, s));
      (note_launch(), k_seg_axpy<<<vg(), TPB, 0, s>>>(n, d_scene_of.p, coef.p, x.p, dx.p));
      // per-scene backtracking line search (newton.rs:171-248)
      std::vector<double> g0(nscene), alpha(nscene, 1.0), alpha_prev(nscene, 0.0), tail(nscene, 0.25);
      std::vector<int> kk(nscene, 1);
      std::vector<unsigned char> ls(active);
      for (int k = 0; k < nscene; ++k) g0[k] = 0.5 * fsq[k];
      const double initial[4] = {0.0, 1.0, 0.75, 0.5};
      for (;;) {
        std::vector<double> da(nscene, 0.0);
        bool anyls = false;
        for (int k = 0; k < nscene; ++k)
          if (ls[k]) {
            da[k] = alpha[k] - alpha_prev[k];
            anyls = true;
          }
        if (!anyls) break;
        HOEFEM_CUDA(cudaMemcpyAsync(coef.p, da.data(), sizeof(double) * nscene, cudaMemcpyHostToDevice, s));
        (note_launch(), k_seg_axpy<<<vg(), TPB, 0, s>>>(n, d_scene_of.p, coef.p, dx.p, w.p));
        std::vector<double> nf;
        eval_F(dt, ls, nf);
        for (int k = 0; k < nscene; ++k) {
          if (!ls[k]) continue;
          fsq[k] = nf[k];
          const double g = 0.5 * nf[k];
          if (g <= (1.0 - 1e-4 * alpha[k]) * g0[k]) {
            ls[k] = 0;
          } else if (alpha[k] < 1e-6) {
            ls[k] = 0;
            status[k] = HOEFEM_LINE_SEARCH_FAILED;
          } else {
            alpha_prev[k] = alpha[k];
            ++kk[k];
            if (kk[k] < 4) alpha[k] = initial[kk[k]];
            else {
              alpha[k] = tail[k];
              tail[k] *= 0.25;
            }
          }
        }
      }
      for (int k = 0; k < nscene; ++k)
        if (active[k] && status[k] == HOEFEM_OK) iter[k] += 1;
    }
    std::vector<unsigned char> ok(nscene);
    for (int k = 0; k < nscene; ++k) {
      ok[k] = part[k] && status[k] == HOEFEM_OK;
      if (ok[k]) {
        st_newton[k] = iter[k];
        st_residual[k] = std::sqrt(fsq[k]);
      }
    }
    HOEFEM_CUDA(cudaMemcpyAsync(d_ok.p, ok.data(), nscene, cudaMemcpyHostToDevice, s));
    (note_launch(), k_be_final2<<<vg(), TPB, 0, s>>>(n, d_scene_of.p, d_ok.p, w.p, dt, d_bc.p, u.p, v.p));
    HOEFEM_CUDA(cudaGetLastError());
  }

  // integrate_model_with_substeps for every scene: a scene whose step fails is
  // retried alone from its initial state with 5x as many substeps, until
  // 1000 substeps (newton_cg.rs:245-291).  ud, vd: device, concatenated.
  int step(double* ud, double* vd, double dt) {
    cudaStream_t s = m.stream;
    const int n = (int)m.ndof;
    cudaEvent_t e0, e1;
    HOEFEM_CUDA(cudaEventCreate(&e0));
    HOEFEM_CUDA(cudaEventCreate(&e1));
    HOEFEM_CUDA(cudaEventRecord(e0, s));
    status.assign(nscene, HOEFEM_OK);
    st_newton.assign(nscene, 0);
    st_cg_solves.assign(nscene, 0);
    st_cg_total.assign(nscene, 0);
    st_cg_max.assign(nscene, 0);
    st_cg_last.assign(nscene, HOEFEM_OK);
    st_substeps.assign(nscene, 1);
    st_residual.assign(nscene, 0.0);
    (note_launch(), k_bc_uv2<<<vg(), TPB, 0, s>>>(n, d_bc.p, ud, vd));
    std::vector<unsigned char> pending(nscene, 1), final_status(nscene, 0);
    std::vector<int> result(nscene, HOEFEM_OK);
    i64 num = 1;
    for (;;) {
      (note_launch(), k_vcopy<<<vg(), TPB, 0, s>>>(n, ud, u.p));
      (note_launch(), k_vcopy<<<vg(), TPB, 0, s>>>(n, vd, v.p));
      std::vector<unsigned char> part(pending);
      const double sdt = dt / (double)num;
      for (i64 k = 0; k < num; ++k) {
        try {
          be_step(sdt, part);
        } catch (Error& err2) {
          if (err2.code == HOEFEM_ERR_CUDA || err2.code == HOEFEM_ERR_OUT_OF_MEMORY ||
              err2.code == HOEFEM_ERR_DEVICE_TIMEOUT)
            throw;
          for (int q = 0; q < nscene; ++q)
            if (part[q]) status[q] = err2.code;
        }
        for (int q = 0; q < nscene; ++q)
          if (part[q] && status[q] != HOEFEM_OK) {
            part[q] = 0;
            result[q] = status[q];
          }
      }
      // scenes that finished all substeps: copy out
      std::vector<unsigned char> done(nscene, 0);
      bool retry = false;
      for (int q = 0; q < nscene; ++q) {
        if (!pending[q]) continue;
        if (part[q]) {
          done[q] = 1;
          result[q] = HOEFEM_OK;
          st_substeps[q] = num;
          pending[q] = 0;
        } else if (num * 5 >= 1000) {
          result[q] = HOEFEM_SUBSTEPPING_FAILED;
          st_substeps[q] = num * 5;
          pending[q] = 0;
        } else {
          retry = true;
        }
      }
      HOEFEM_CUDA(cudaMemcpyAsync(d_ok.p, done.data(), nscene, cudaMemcpyHostToDevice, s));
      (note_launch(), k_masked_copy<<<vg(), TPB, 0, s>>>(n, d_scene_of.p, d_ok.p, u.p, ud));
      (note_launch(), k_masked_copy<<<vg(), TPB, 0, s>>>(n, d_scene_of.p, d_ok.p, v.p, vd));
      if (!retry) break;
      num *= 5;
    }
    status = result;
    HOEFEM_CUDA(cudaEventRecord(e1, s));
    HOEFEM_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    HOEFEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    ms_total = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int worst = HOEFEM_OK;
    for (int k = 0; k < nscene; ++k)
      if (status[k] != HOEFEM_OK) worst = status[k];
    return worst;
  }
};

// ---- construction from per-scene models ------------------------------------------
// Every scene's blocks of one element kind become one merged block (node
// indices shifted by the scene's node offset, per-element Lame parameters);
// the merged quadrature stays uniform when all contributing blocks share one
// rule, otherwise it is stored per element.
Batch* batch_build(const std::vector<const Model*>& scenes, const std::vector<MatDev>& mats, double density,
                   const i64* bc_off, const i64* bc_nodes, bool gravity_enabled, double gravity) {
  const int ns = (int)scenes.size();
  HOEFEM_REQUIRE(ns > 0, HOEFEM_ERR_INVALID_ARGUMENT, "empty batch");
  for (int k = 1; k < ns; ++k)
    HOEFEM_REQUIRE(mats[k].kind == mats[0].kind, HOEFEM_ERR_INVALID_ARGUMENT,
                   "all scenes of a batch use one material model");
  std::unique_ptr<Batch> B(new Batch());
  Model& m = B->m;
  B->nscene = ns;
  B->mat_kind = mats[0].kind;
  B->density = density;
  B->gravity = gravity_enabled ? gravity : 0.0;
  B->node_off.assign(ns + 1, 0);
  for (int k = 0; k < ns; ++k) {
    HOEFEM_REQUIRE(scenes[k]->nv > 0 && !scenes[k]->blocks.empty(), HOEFEM_ERR_INVALID_ARGUMENT,
                   "scene without vertices or elements");
    HOEFEM_REQUIRE(B->node_off[k] + scenes[k]->nv < (1LL << 31) / 3, HOEFEM_ERR_INVALID_ARGUMENT,
                   "batch too large");
    B->node_off[k + 1] = B->node_off[k] + (int)scenes[k]->nv;
  }
  m.nv = B->node_off.back();
  m.X.reserve(3 * m.nv);
  B->scene_of.resize(m.nv);
  B->bc_host.assign(3 * m.nv, 0);
  // which kinds appear, and whether each merged block can keep one rule
  const int kinds[2] = {HOEFEM_ELEM_TET10, HOEFEM_ELEM_HEX27};
  for (int ki = 0; ki < 2; ++ki) {
    const Block* first = nullptr;
    bool uniform = true;
    i64 ne = 0;
    for (const Model* sm : scenes)
      for (const Block* b : sm->blocks) {
        if (b->kind != kinds[ki]) continue;
        ne += b->ne;
        if (!b->uniform) uniform = false;
        else if (!first) first = b;
        else if (b->qw != first->qw || b->qp != first->qp) uniform = false;
      }
    if (ne == 0) continue;
    Block* mb = new Block();
    m.blocks.push_back(mb);
    mb->kind = kinds[ki];
    mb->nn = kinds[ki] == HOEFEM_ELEM_TET10 ? 10 : 27;
    mb->uniform = uniform;
    mb->conn.reserve(ne * mb->nn);
    mb->emat.reserve(2 * ne);
    if (uniform) {
      mb->qw = first->qw;
      mb->qp = first->qp;
    } else {
      mb->qoff.reserve(ne + 1);
      mb->qoff.push_back(0);
    }
    for (int k = 0; k < ns; ++k)
      for (const Block* b : scenes[k]->blocks) {
        if (b->kind != kinds[ki]) continue;
        const i64 shift = B->node_off[k];
        for (i64 c : b->conn) mb->conn.push_back(c + shift);
        for (i64 e = 0; e < b->ne; ++e) {
          mb->emat.push_back(mats[k].mu);
          mb->emat.push_back(mats[k].lambda);
          mb->escene.push_back(k);
          if (!uniform) {
            const i64 q0 = b->uniform ? 0 : b->qoff[e];
            const i64 q1 = b->uniform ? (i64)b->qw.size() : b->qoff[e + 1];
            mb->qw.insert(mb->qw.end(), b->qw.begin() + q0, b->qw.begin() + q1);
            mb->qp.insert(mb->qp.end(), b->qp.begin() + 3 * q0, b->qp.begin() + 3 * q1);
            mb->qoff.push_back(mb->qoff.back() + (q1 - q0));
          }
        }
        mb->ne += b->ne;
      }
  }
  for (int k = 0; k < ns; ++k) {
    const Model* sm = scenes[k];
    m.X.insert(m.X.end(), sm->X.begin(), sm->X.end());
    for (int a = B->node_off[k]; a < B->node_off[k + 1]; ++a) B->scene_of[a] = k;
    if (bc_off)
      for (i64 q = bc_off[k]; q < bc_off[k + 1]; ++q) {
        const i64 a = bc_nodes[q];
        HOEFEM_REQUIRE(a >= 0 && a < sm->nv, HOEFEM_ERR_INVALID_ARGUMENT, "Dirichlet node out of range");
        for (int i = 0; i < 3; ++i) B->bc_host[3 * (B->node_off[k] + a) + i] = 1;
      }
  }
  finalize_model(m);
  ensure_device(m);
  B->setup();
  B->emask.alloc(ns);
  for (Block* b : m.blocks) b->scene_active = B->emask.p;
  return B.release();
}

void batch_delete(Batch* b) { delete b; }
Model& batch_model(Batch* b) { return b->m; }
int batch_step(Batch* b, double* u, double* v, double dt) { return b->step(u, v, dt); }
void batch_set_cg_engine(Batch* b, int engine, int ctas_per_sm) {
  HOEFEM_REQUIRE(engine >= HOEFEM_CG_ENGINE_AUTO && engine <= HOEFEM_CG_ENGINE_STREAMED && ctas_per_sm >= 0,
                 HOEFEM_ERR_INVALID_ARGUMENT, "bad CG engine");
  b->cg_engine = engine;
  b->cg_ctas = ctas_per_sm;
  b->tuned_engine = -1;
  b->tuned_ctas = 0;
  b->tune_ms.clear();
}
void batch_cg_choice(Batch* b, int* engine, int* ctas_per_sm, std::vector<float>* tune_ms) {
  if (b->cg_engine != HOEFEM_CG_ENGINE_AUTO) {
    *engine = b->cg_engine;
    *ctas_per_sm = b->cg_ctas;
  } else {
    *engine = b->tuned_engine < 0 ? HOEFEM_CG_ENGINE_AUTO : b->tuned_engine;
    *ctas_per_sm = b->tuned_ctas;
  }
  if (tune_ms) *tune_ms = b->tune_ms;
}
void batch_set_tolerances(Batch* b, double tol, i64 cg_max, i64 newton_max) {
  b->cg_tol = tol;
  b->cg_max = cg_max;
  b->newton_max = newton_max;
}
const std::vector<int>& batch_node_offsets(Batch* b) { return b->node_off; }
void batch_scene_stats(Batch* b, int k, hoefem_step_stats* out, int* status) {
  hoefem_step_stats st{};
  if (k < (int)b->status.size()) {
    st.newton_iterations = b->st_newton[k];
    st.num_cg_solves = b->st_cg_solves[k];
    st.total_cg_iterations = b->st_cg_total[k];
    st.max_cg_iterations = b->st_cg_max[k];
    st.substeps = b->st_substeps[k];
    st.last_cg_status = b->st_cg_last[k];
    st.residual_norm = b->st_residual[k];
    *status = b->status[k];
  } else {
    *status = HOEFEM_OK;
  }
  st.representative_force = b->rep[k];
  st.ms_total = b->ms_total;
  *out = st;
}

}  // namespace hoefem
