// Persistent streamed conjugate gradient.
//
// Reference: ConjugateGradient::solve_with_guess_ (fenris/src/cg.rs:376-482)
// with RelativeResidualCriterion (cg.rs:77-124), the Schwarz apply of
// SchwarzPreconditioner (simulation_toolbox/src/fem/newton_cg.rs:297-350) and
// the diagonal preconditioner (newton_cg.rs:534-593): the same recurrence,
// tests and outcomes as the chunked kernels of cg.cu, in one cooperative
// launch per solve (per residual replacement in the mixed-precision form).
//
// A CG iteration reads the operator values and the Schwarz blocks once each;
// everything else (vectors, 1 MB each on the benchmark) stays in L2.  The
// kernel keeps that stream flowing: one CTA per SM, a producer warp whose
// lane 0 issues bulk asynchronous copies (cp.async.bulk, no multicast) of
// work items of up to 14 KB into a ring of shared-memory stages, cycling
// through the CTA's fixed item list (its operator tiles, then its Schwarz
// row records) across iterations and refilling each stage as soon as its
// warp releases it (in any order across stages, so that one busy warp does
// not hold up the others' copies), and 12 consumer warps that compute from
// the stages.  Stage k % NS belongs to consumer warp k % NW (NS a multiple of
// NW), so each stage is used and released in order by one warp.
//
// Work is partitioned by node: a CTA owns a contiguous node range, split into
// segments whose halo (every neighbour node of the segment's nodes) fits in
// shared memory.  The tiles' neighbour lists and the Schwarz records' column
// lists are 16-bit indices into that halo, and the vectors an item needs are
// gathered into it once per phase by all consumer threads, so the per-node
// loops read shared memory only.  The Schwarz blocks are distributed by rows:
// the 3 rows of a subdomain block that belong to a node are stored with the
// node's owner, so z = P r of an own node is a sum of local row products and
// an iteration needs two grid barriers:
//   P1  per segment: direction p = z + beta p_old (double-buffered) on the
//       halo, stored for the own nodes; Ap = A p for the own nodes; p.Ap
//   --- grid barrier (alpha) ---
//   P2  per segment: residual r' = r_old - alpha Ap on the halo (r is
//       double-buffered: other CTAs still gather r_old while the owners
//       write r_new); the own nodes' Schwarz rows y = B_s r'_s per
//       incidence; then the own DOFs: x += alpha p, r_new = r', z = the sum
//       of the node's rows in subdomain order (untreated nodes: 1 / a_ii;
//       diagonal / identity preconditioners: z from r' directly); r.r, z.r
//   --- grid barrier (beta, convergence) ---
// Vectors this kernel writes are read through L2 only (ld.global.cg): another
// SM's L1 may still hold lines from an earlier phase, and the grid barrier's
// fences do not invalidate them.
// Each reduction is deterministic: a CTA sums its warps in warp order, and
// after the barrier every CTA sums the CTA partials in CTA order, so all CTAs
// take the same decisions (alpha, beta, convergence) without another barrier.
// Every wait is bounded (stream_pipe.cuh); a wait that runs out raises a
// grid-wide abort, the CTAs leave at their next barrier, copies in flight
// land before a CTA exits, and the host gets HOEFEM_ERR_DEVICE_TIMEOUT.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <vector>

#include "internal.h"
#include "kernels_common.cuh"
#include "solver.h"
#include "stream_partition.h"
#include "stream_pipe.cuh"

namespace hoefem {

namespace {

constexpr int NW = 12;                  // consumer warps
constexpr int NS = 12;                  // ring stages
constexpr int STAGE = 14336;            // bytes per stage (and per work item)
constexpr int THREADS = 32 * (NW + 1);  // + the producer warp (the last one)
constexpr int CONSUMERS = 32 * NW;
// item headers: int records, int first record, 2 x pad; then per record an
// int4: operator tiles (record offset, degree, 3 x own halo index, node),
// Schwarz items (record offset, block dimension, slot, 0)
constexpr int ITEM_HDR = 16;
constexpr int MAX_DIM = 81;      // Schwarz block dimension bound (3 x 27 nodes)
constexpr int HALO_MAX = 1152;   // halo nodes of one segment
constexpr int ZMAX = 1536;       // Schwarz row results (3 per incidence) of one segment
constexpr size_t SMEM_RING = (size_t)NS * STAGE;
// ring, FP64 halo (3 per node), Schwarz row results, FP32 halo (4 per node)
constexpr size_t SMEM_BYTES = SMEM_RING + (size_t)3 * HALO_MAX * 8 + (size_t)ZMAX * 8 + (size_t)HALO_MAX * 16;
static_assert(SMEM_BYTES + 2048 <= 227 * 1024, "shared memory (dynamic + static)");
static_assert(NS % NW == 0, "each ring stage must belong to one consumer warp");
static_assert(STAGE % 16 == 0 && SMEM_RING % 16 == 0, "bulk copies need 16-byte sizes and offsets");
static_assert(3 * HALO_MAX < 65536, "halo-local indices are 16-bit");

__host__ __device__ constexpr long long align16(long long x) { return (x + 15) & ~15LL; }

struct Args {
  const unsigned char* op;
  const CgsItem* op_items;
  const int* op_item_off;
  const int* node_range;
  const CgsSeg* segs;
  const int* seg_off;
  const int* halo;
  const unsigned char* sw;
  const CgsItem* sw_items;
  const int* sw_item_off;
  const double* sw_scale;  // FP16 blocks: per-subdomain scale
  const int* slot_sub;     // per slot: subdomain (FP16 scale lookup)
  const int* pair_off;     // nv + 1: a node's slots (Schwarz incidences, subdomains ascending)
  const unsigned char* diag_only;
  const long long* pbase;
  const double* pvals;  // assembled Schwarz values (untreated nodes' 1 / a_ii)
  const double* dinv;   // diagonal preconditioner
  double* x;
  double* r0;
  double* r1;
  double* z;
  double* Ap;
  double* pb0;
  double* pb1;
  CgState* st;
  double* part;  // 3 x grid
  unsigned* bar;
  int* err;  // [0] abort flag, [1] error code
  int reliable;
  unsigned long long* prof;  // optional: 16 cycle counters per CTA (phase profile)
};

// The direction and the residual step, written once so that every use of a
// value (halo gathers, own-node stores, the update) rounds identically.
__device__ __forceinline__ double cg_dir(double z, double beta, double pold) { return __fma_rn(beta, pold, z); }
__device__ __forceinline__ double cg_res(double r, double alpha, double ap) { return __fma_rn(-alpha, ap, r); }

template <class V>
__device__ __forceinline__ double ldv(const V* p) {
  return (double)*p;
}
template <>
__device__ __forceinline__ double ldv<__half>(const __half* p) {
  return (double)__half2float(*p);
}

// Warp-uniform bounded wait for a full stage.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, unsigned parity) {
  const uint64_t t0 = pipe::clock_ns();
  for (;;) {
    const bool mine = pipe::mbar_test(bar, parity);
    if (__all_sync(0xffffffffu, mine)) return true;
    const int late = (pipe::clock_ns() - t0) > pipe::HOEFEM_WAIT_NS;
    if (__shfl_sync(0xffffffffu, late, 0)) return false;
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// First item index j >= j0 of an iteration (item base kb) owned by warp w.
__device__ __forceinline__ int first_item(long long kb, int j0, int w) {
  const int m = (int)((kb + j0) % NW);
  return j0 + ((w - m) % NW + NW) % NW;
}

// Sum of part[0 .. G) in CTA order, the same in every CTA (warp 0).
__device__ __forceinline__ double sum_partials(const double* part, int G, int lane) {
  double v = 0.0;
  for (int i = lane; i < G; i += 32) v += __ldcg(part + i);
  return warp_sum(v);
}

// Halo node of a halo-local DOF index 3 hl (hl < HALO_MAX): hl = x / 3 by a
// multiply and shift, exact for x < 98,304.
__device__ __forceinline__ int halo_node(int x) { return (x * 43691) >> 17; }
static_assert(3 * HALO_MAX < 98304, "halo_node range");

// Gather batches: each thread first issues the loads of GB entries, then
// computes and stores, so that GB L2 round trips overlap instead of chaining.
constexpr int GB = 8;

// For t < n3 (halo entry t / 3, component t % 3, DOF g = 3 halo[t / 3] + t % 3):
// mode 0: s[t] = va + c vb at g (the direction z + beta p_old), also stored to
// pnew for g in [d0, d1); mode 1: s[t] = va - c vb at g (r_old - alpha Ap).
// With s32 non-null the value is also stored rounded to FP32 at s32[4 (t / 3) + t % 3]
// (the FP32 halo of the FP32-value products).
template <int MODE>
__device__ __forceinline__ void gather_halo(const int* __restrict__ halo, int n3, int d0, int d1,
                                            const double* __restrict__ va, const double* __restrict__ vb, double c,
                                            double* __restrict__ s, double* __restrict__ pnew,
                                            float* __restrict__ s32 = nullptr) {
  for (int t0 = (int)threadIdx.x; t0 < n3; t0 += GB * CONSUMERS) {
    int g[GB];
#pragma unroll
    for (int u = 0; u < GB; ++u) {
      const int t = t0 + u * CONSUMERS;
      g[u] = -1;
      if (t < n3) {
        const int hl = t / 3;
        g[u] = 3 * __ldg(halo + hl) + (t - 3 * hl);
      }
    }
    double a[GB], b[GB];
#pragma unroll
    for (int u = 0; u < GB; ++u) {
      a[u] = g[u] >= 0 ? __ldcg(va + g[u]) : 0.0;
      b[u] = g[u] >= 0 ? __ldcg(vb + g[u]) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < GB; ++u) {
      if (g[u] < 0) continue;
      const int t = t0 + u * CONSUMERS;
      double dv;
      if (MODE == 0) {
        dv = cg_dir(a[u], c, b[u]);
        if (g[u] >= d0 && g[u] < d1) pnew[g[u]] = dv;
      } else {
        dv = cg_res(a[u], c, b[u]);
      }
      s[t] = dv;
      if (s32) {
        const int hl = t / 3;
        s32[4 * hl + (t - 3 * hl)] = (float)dv;
      }
    }
  }
}

template <class VA, class VB, int PK>
__global__ void __launch_bounds__(THREADS, 1) k_cg_stream(Args A) {
  extern __shared__ __align__(128) unsigned char ring[];
  double* s_halo = reinterpret_cast<double*>(ring + SMEM_RING);  // 3 x HALO_MAX
  double* s_zp = s_halo + 3 * HALO_MAX;                           // ZMAX
  float4* s_h32 = reinterpret_cast<float4*>(s_zp + ZMAX);          // HALO_MAX
  constexpr bool OP32 = sizeof(VA) == 4, SW32 = sizeof(VB) < 8;
  __shared__ __align__(8) uint64_t full[NS];
  __shared__ __align__(8) uint64_t empty[NS];
  __shared__ volatile int s_stop;
  __shared__ int s_fail, s_gok;
  __shared__ double s_red[NW][2];
  __shared__ double s_bc[3];
  __shared__ unsigned long long s_prof[16];
  // a solve that an earlier kernel finished (the true residual after a
  // replacement met the tolerance) runs no iteration: uniform over the grid
  if (*(const volatile int*)&A.st->done) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x, G = gridDim.x;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      pipe::mbar_init(&full[i], 1);
      pipe::mbar_init(&empty[i], 1);
    }
    s_stop = 0;
    s_fail = 0;
    for (int i = 0; i < 16; ++i) s_prof[i] = 0ull;
    pipe::mbar_fence_init();
  }
  __syncthreads();
  // phase profile: thread 0 times its own path through the phases, the
  // producer its idle polling
  const bool prof = A.prof != nullptr;
  const bool timer = prof && threadIdx.x == 0;
  auto tick = [&]() -> unsigned long long { return timer ? (unsigned long long)clock64() : 0ull; };
  auto tock = [&](int slot, unsigned long long t0) {
    if (timer) s_prof[slot] += (unsigned long long)clock64() - t0;
  };
  const int op0 = A.op_item_off[c], nop = A.op_item_off[c + 1] - op0;
  const int sw0 = PK == 2 ? A.sw_item_off[c] : 0;
  const int nsw = PK == 2 ? A.sw_item_off[c + 1] - sw0 : 0;
  const int per = nop + nsw;

  if (warp == NW) {
    // ---- producer: each stage s carries items s, s + NS, s + 2 NS, ... (the
    // CTA's items cycled over the iterations); a stage is refilled as soon as
    // its warp has released it, whatever the other stages are doing ----
    if (lane != 0) return;
    const unsigned long long tp0 = prof ? (unsigned long long)clock64() : 0ull;
    unsigned long long twait = 0ull, tw = tp0;
    const uint64_t pol_keep = pipe::policy_evict_last(), pol_stream = pipe::policy_evict_first();
    long long next[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) next[i] = i;
    bool late = false;
    uint64_t t_idle = 0;
    while (per > 0 && !s_stop) {
      bool progress = false;
#pragma unroll
      for (int st = 0; st < NS; ++st) {
        const long long k = next[st];
        const long long use = k / NS;
        if (use > 0 && !pipe::mbar_test(&empty[st], (unsigned)((use - 1) & 1))) continue;
        const int j = (int)(k % per);
        const CgsItem it = j < nop ? A.op_items[op0 + j] : A.sw_items[sw0 + (j - nop)];
        const unsigned char* src = (j < nop ? A.op : A.sw) + it.off;
        pipe::mbar_arrive_expect_tx(&full[st], (unsigned)it.bytes);
        pipe::bulk_g2s_hint(ring + (size_t)st * STAGE, src, (unsigned)it.bytes, &full[st],
                            it.keep ? pol_keep : pol_stream);
        next[st] = k + NS;
        progress = true;
      }
      if (progress) {
        t_idle = 0;
        if (prof) tw = (unsigned long long)clock64();
      } else {
        const uint64_t now = pipe::clock_ns();
        if (t_idle == 0) {
          t_idle = now;
        } else if (now - t_idle > pipe::HOEFEM_WAIT_NS) {
          late = true;
          break;
        }
        if (prof) {
          const unsigned long long c1 = (unsigned long long)clock64();
          twait += c1 - tw;
          tw = c1;
        }
      }
    }
    if (late && !s_stop) {
      atomicExch(&A.err[0], 1);
      atomicCAS(&A.err[1], 0, (int)HOEFEM_ERR_DEVICE_TIMEOUT);
    }
    // the copies still in flight (each stage's last issued item) land before
    // the CTA exits
#pragma unroll
    for (int st = 0; st < NS; ++st) {
      const long long k = next[st] - NS;
      if (k >= 0) pipe::mbar_wait(&full[st], (unsigned)((k / NS) & 1));
    }
    if (prof) {
      atomicAdd(A.prof + 16 * c + 10, twait);
      atomicAdd(A.prof + 16 * c + 11, (unsigned long long)clock64() - tp0);
    }
    return;
  }

  // ---- consumers ----
  const int w = warp;
  const int sg0 = A.seg_off[c], sg1 = A.seg_off[c + 1];
  CgState* st = A.st;
  double zTr = st->zTr, beta = st->beta, alpha = st->alpha, pAp = st->pAp, rr = st->rr;
  const double bnorm = st->bnorm, tol = st->tol, rr_ref = st->rr_ref, delta2 = st->delta2;
  long long iters = st->iters;
  const long long max_iter = st->max_iter;
  int status = HOEFEM_OK, done = 0, replace = 0, pcur = 0, rcur = 0;
  long long it = 0;
  const int grp = lane >> 3, gl = lane & 7;  // operator tiles: node group and its lane
  auto fail = [&]() {
    s_fail = 1;
    atomicExch(&A.err[0], 1);
    atomicCAS(&A.err[1], 0, (int)HOEFEM_ERR_DEVICE_TIMEOUT);
  };
  // CTA barrier of the consumers, then the grid barrier; uniform outcome
  auto grid_sync = [&]() -> bool {
    pipe::named_sync(1, CONSUMERS);
    if (threadIdx.x == 0) s_gok = pipe::grid_barrier_leader(A.bar, &A.err[0]) && !s_fail;
    pipe::named_sync(1, CONSUMERS);
    return s_gok != 0;
  };
  bool ok = true;
  for (;;) {
    const long long kb = it * per;
    const double* pold = (it & 1) ? A.pb1 : A.pb0;
    double* pnew = (it & 1) ? A.pb0 : A.pb1;
    const double* rold = (it & 1) ? A.r1 : A.r0;
    double* rnew = (it & 1) ? A.r0 : A.r1;
    // ---- P1: p = z + beta p_old on each segment's halo, Ap = A p, p.Ap ----
    double acc = 0.0;
    for (int sg = sg0; sg < sg1; ++sg) {
      const CgsSeg S = A.segs[sg];
      unsigned long long t0 = tick();
      pipe::named_sync(1, CONSUMERS);  // the previous segment is done with the halo
      gather_halo<0>(A.halo + S.halo_off, 3 * S.halo_n, 3 * S.n0, 3 * S.n1, A.z, pold, beta, s_halo, pnew,
                     OP32 ? reinterpret_cast<float*>(s_h32) : nullptr);
      pipe::named_sync(1, CONSUMERS);
      tock(0, t0);
      t0 = tick();
      for (int j = first_item(kb, S.j0, w); j < S.j1; j += NW) {
        const long long k = kb + j;
        const int s = (int)(k % NS);
        const unsigned long long tw = tick();
        if (!warp_wait(&full[s], (unsigned)((k / NS) & 1))) {
          if (lane == 0) fail();
          break;
        }
        tock(2, tw);
        const unsigned char* t = ring + (size_t)s * STAGE;
        const int nn = *(const int*)t;
        // four node rows per pass, 8 lanes each (records sorted by degree, so
        // the four have similar lengths); 3-level reductions per group
        for (int q0 = 0; q0 < nn; q0 += 4) {
          const int q = q0 + grp;
          const bool has = q < nn;
          const int4 h = has ? *(const int4*)(t + ITEM_HDR + 16 * q) : make_int4(0, 0, 0, 0);
          const int d = h.y;
          const unsigned short* loc = (const unsigned short*)(t + h.x);
          const VA* v = (const VA*)(t + h.x + align16(2LL * d));
          double s0 = 0.0, s1 = 0.0, s2 = 0.0;
          if constexpr (OP32) {
            // FP32 values times the FP32 halo (one 16-byte load per block),
            // FP32 sums: the products carry the values' own rounding
            float f0 = 0.f, f1 = 0.f, f2 = 0.f;
            const float* vf = reinterpret_cast<const float*>(v);
            for (int e = gl; e < d; e += 8) {
              const float4 pv = s_h32[halo_node(loc[e])];
              f0 += vf[e] * pv.x + vf[d + e] * pv.y + vf[2 * d + e] * pv.z;
              f1 += vf[3 * d + e] * pv.x + vf[4 * d + e] * pv.y + vf[5 * d + e] * pv.z;
              f2 += vf[6 * d + e] * pv.x + vf[7 * d + e] * pv.y + vf[8 * d + e] * pv.z;
            }
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) {
              f0 += __shfl_xor_sync(0xffffffffu, f0, o);
              f1 += __shfl_xor_sync(0xffffffffu, f1, o);
              f2 += __shfl_xor_sync(0xffffffffu, f2, o);
            }
            s0 = f0;
            s1 = f1;
            s2 = f2;
          } else {
            for (int e = gl; e < d; e += 8) {
              const double* pd = s_halo + loc[e];
              const double q0v = pd[0], q1v = pd[1], q2v = pd[2];
              s0 += ldv(v + e) * q0v + ldv(v + d + e) * q1v + ldv(v + 2 * d + e) * q2v;
              s1 += ldv(v + 3 * d + e) * q0v + ldv(v + 4 * d + e) * q1v + ldv(v + 5 * d + e) * q2v;
              s2 += ldv(v + 6 * d + e) * q0v + ldv(v + 7 * d + e) * q1v + ldv(v + 8 * d + e) * q2v;
            }
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) {
              s0 += __shfl_xor_sync(0xffffffffu, s0, o);
              s1 += __shfl_xor_sync(0xffffffffu, s1, o);
              s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            }
          }
          if (has && gl == 0) {
            const int a3 = 3 * h.w;
            const double* pa = s_halo + h.z;
            A.Ap[a3] = s0;
            A.Ap[a3 + 1] = s1;
            A.Ap[a3 + 2] = s2;
            acc += pa[0] * s0;
            acc += pa[1] * s1;
            acc += pa[2] * s2;
          }
        }
        __syncwarp();
        if (lane == 0) pipe::mbar_arrive(&empty[s]);
      }
      tock(1, t0);
    }
    unsigned long long tb = tick();
    acc = warp_sum(acc);
    if (lane == 0) s_red[w][0] = acc;
    pipe::named_sync(1, CONSUMERS);
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < NW; ++i) t += s_red[i][0];
      A.part[c] = t;
    }
    if (!grid_sync()) {
      ok = false;
      break;
    }
    if (w == 0) {
      const double t = sum_partials(A.part, G, lane);
      if (lane == 0) s_bc[0] = t;
    }
    pipe::named_sync(1, CONSUMERS);
    tock(3, tb);
    pAp = s_bc[0];
    if (pAp <= 0.0 || zTr <= 0.0) {
      done = 1;
      status = pAp <= 0.0 ? HOEFEM_CG_INDEFINITE_OPERATOR : HOEFEM_CG_INDEFINITE_PRECONDITIONER;
      pcur = (int)((it + 1) & 1);
      rcur = (int)(it & 1);
      break;
    }
    alpha = zTr / pAp;
    // ---- P2: r' on the halo, Schwarz rows, own DOFs ----
    double racc = 0.0, zacc = 0.0;
    for (int sg = sg0; sg < sg1; ++sg) {
      const CgsSeg S = A.segs[sg];
      unsigned long long t0 = tick();
      if (PK == 2) {
        pipe::named_sync(1, CONSUMERS);  // the previous segment is done with the halo and s_zp
        gather_halo<1>(A.halo + S.halo_off, 3 * S.halo_n, 0, 0, rold, A.Ap, alpha, s_halo, nullptr,
                       SW32 ? reinterpret_cast<float*>(s_h32) : nullptr);
        pipe::named_sync(1, CONSUMERS);
        tock(4, t0);
        t0 = tick();
        for (int j = first_item(kb, nop + S.sj0, w); j < nop + S.sj1; j += NW) {
          const long long k = kb + j;
          const int s = (int)(k % NS);
          const unsigned long long tw = tick();
          if (!warp_wait(&full[s], (unsigned)((k / NS) & 1))) {
            if (lane == 0) fail();
            break;
          }
          tock(6, tw);
          const unsigned char* t = ring + (size_t)s * STAGE;
          const int nr = *(const int*)t;
          // one block row per lane: row i of record q is sum_m B[i][3m + c] r'(node m, c)
          for (int rho = lane; rho < 3 * nr; rho += 32) {
            const int q = rho / 3, i = rho - 3 * q;
            const int4 h = *(const int4*)(t + ITEM_HDR + 16 * q);
            const int dim = h.y, ns = dim / 3;
            const unsigned short* cols = (const unsigned short*)(t + h.x);
            const VB* v = (const VB*)(t + h.x + align16(2LL * ns)) + (size_t)i * dim;
            double b0 = 0.0, b1 = 0.0, b2 = 0.0;
            if constexpr (SW32) {
              float c0 = 0.f, c1 = 0.f, c2 = 0.f;
              for (int m = 0; m < ns; ++m) {
                const float4 hr = s_h32[halo_node(cols[m])];
                c0 += (float)v[3 * m] * hr.x;
                c1 += (float)v[3 * m + 1] * hr.y;
                c2 += (float)v[3 * m + 2] * hr.z;
              }
              b0 = c0;
              b1 = c1;
              b2 = c2;
            } else {
              for (int m = 0; m < ns; ++m) {
                const double* hr = s_halo + cols[m];
                b0 += ldv(v + 3 * m) * hr[0];
                b1 += ldv(v + 3 * m + 1) * hr[1];
                b2 += ldv(v + 3 * m + 2) * hr[2];
              }
            }
            const double sc = sizeof(VB) == 2 ? A.sw_scale[__ldg(A.slot_sub + h.z)] : 1.0;
            s_zp[3 * (h.z - S.q0) + i] = ((b0 + b1) + b2) * sc;
          }
          __syncwarp();
          if (lane == 0) pipe::mbar_arrive(&empty[s]);
        }
        pipe::named_sync(1, CONSUMERS);  // every row result of the segment is in s_zp
        tock(5, t0);
      }
      // own DOFs of the segment
      t0 = tick();
      for (int t = 3 * S.n0 + (int)threadIdx.x; t < 3 * S.n1; t += CONSUMERS) {
        const int a = t / 3, i = t - 3 * a;
        const double pc = __ldcg(pnew + t);
        const double xv = __ldcg(A.x + t);
        double rn;
        if (PK == 2) rn = s_halo[3 * (S.own_lo + a - S.n0) + i];
        else rn = cg_res(__ldcg(rold + t), alpha, __ldcg(A.Ap + t));
        double zv;
        if (PK == 2) {
          if (__ldg(A.diag_only + a)) {
            zv = __ldg(A.pvals + __ldg(A.pbase + a) + i) * rn;
          } else {
            // the node's subdomains in ascending order (zero if it has none)
            zv = 0.0;
            const int q1 = __ldg(A.pair_off + a + 1);
            for (int q = __ldg(A.pair_off + a); q < q1; ++q) zv += s_zp[3 * (q - S.q0) + i];
          }
        } else if (PK == 1) {
          zv = __ldg(A.dinv + t) * rn;
        } else {
          zv = rn;
        }
        A.x[t] = __fma_rn(alpha, pc, xv);
        rnew[t] = rn;
        A.z[t] = zv;
        racc += rn * rn;
        zacc += zv * rn;
      }
      tock(8, t0);
    }
    unsigned long long tu = tick();
    racc = warp_sum(racc);
    zacc = warp_sum(zacc);
    if (lane == 0) {
      s_red[w][0] = racc;
      s_red[w][1] = zacc;
    }
    pipe::named_sync(1, CONSUMERS);
    if (threadIdx.x == 0) {
      double t0 = 0.0, t1 = 0.0;
      for (int i = 0; i < NW; ++i) {
        t0 += s_red[i][0];
        t1 += s_red[i][1];
      }
      A.part[G + c] = t0;
      A.part[2 * G + c] = t1;
    }
    if (!grid_sync()) {
      ok = false;
      break;
    }
    if (w == 0) {
      const double t0 = sum_partials(A.part + G, G, lane);
      const double t1 = sum_partials(A.part + 2 * G, G, lane);
      if (lane == 0) {
        s_bc[1] = t0;
        s_bc[2] = t1;
      }
    }
    pipe::named_sync(1, CONSUMERS);
    tock(9, tu);
    rr = s_bc[1];
    const double zr = s_bc[2];
    iters += 1;
    ++it;
    pcur = (int)(it & 1);
    rcur = (int)(it & 1);
    if (sqrt(rr) <= tol * bnorm) {
      done = 1;
      status = HOEFEM_OK;
      break;
    }
    if (max_iter >= 0 && iters >= max_iter) {
      done = 1;
      status = HOEFEM_CG_MAX_ITERATIONS;
      break;
    }
    beta = zr / zTr;
    zTr = zr;
    if (A.reliable && rr <= delta2 * rr_ref) {
      replace = 1;
      break;
    }
  }
  if (c == 0 && threadIdx.x == 0) {
    if (ok) {
      st->zTr = zTr;
      st->beta = beta;
      st->alpha = alpha;
      st->pAp = pAp;
      st->rr = rr;
      st->iters = iters;
      st->done = done;
      st->status = status;
      st->replace = replace;
      st->pcur = pcur;
      st->rcur = rcur;
    } else {
      st->done = 1;
      st->status = HOEFEM_ERR_DEVICE_TIMEOUT;
      st->replace = 0;
      st->pcur = 0;
      st->rcur = 0;
    }
  }
  pipe::named_sync(1, CONSUMERS);
  if (threadIdx.x == 0) {
    s_stop = 1;
    if (prof) {
      for (int i = 0; i < 10; ++i) atomicAdd(A.prof + 16 * c + i, s_prof[i]);
      atomicAdd(A.prof + 16 * c + 12, (unsigned long long)it);
    }
  }
}

// ---- stream layouts -----------------------------------------------------------

// Item headers and 16-bit halo-local index lists (once per layout).  The
// records are numbered in stream order; record r of item (first = item.a)
// is first + r: its index list (rec_count[.] entries from idx[rec_src[.]])
// goes to rec_idx_off[.] and its header is (offset in the item, fy, fz, fw).
__global__ void k_item_layout(int nitems, const CgsItem* __restrict__ items, const long long* __restrict__ rec_idx_off,
                              const int* __restrict__ rec_src, const int* __restrict__ rec_count,
                              const unsigned short* __restrict__ idx, const int* __restrict__ fy,
                              const int* __restrict__ fz, const int* __restrict__ fw, unsigned char* __restrict__ data) {
  const int item = blockIdx.x;
  if (item >= nitems) return;
  const CgsItem it = items[item];
  unsigned char* t = data + it.off;
  const int nr = it.b, first = it.a;
  if (threadIdx.x == 0) {
    ((int*)t)[0] = nr;
    ((int*)t)[1] = first;
    ((int*)t)[2] = 0;
    ((int*)t)[3] = 0;
  }
  for (int q = threadIdx.x; q < nr; q += blockDim.x)
    ((int4*)(t + ITEM_HDR))[q] =
        make_int4((int)(rec_idx_off[first + q] - it.off), fy[first + q], fz[first + q], fw[first + q]);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  for (int q = warp; q < nr; q += nwarp) {
    const int o = rec_src[first + q], n = rec_count[first + q];
    unsigned short* dst = (unsigned short*)(data + rec_idx_off[first + q]);
    for (int e = lane; e < n; e += 32) dst[e] = idx[o + e];
  }
}

// Operator values into the node records' planes: entry (3a + i, 3b + j) of
// the scalar CSR (offset base[a] + i 3d + 3 slot(b) + j) goes to plane 3i + j,
// position slot(b).  One warp per node.
template <class V>
__global__ void __launch_bounds__(256) k_op_pack(int nv, const long long* __restrict__ base,
                                                 const int* __restrict__ adj_off, const long long* __restrict__ val_off,
                                                 const double* __restrict__ vals, unsigned char* __restrict__ data) {
  const int lane = threadIdx.x & 31;
  for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < nv; a += (gridDim.x * blockDim.x) >> 5) {
    const int d = adj_off[a + 1] - adj_off[a];
    const double* src = vals + base[a];
    V* dst = (V*)(data + val_off[a]);
    const int rl = 3 * d;
    for (int cidx = lane; cidx < 9 * d; cidx += 32) {
      const int i = cidx / rl, rem = cidx - i * rl;
      const int sl = rem / 3, j = rem - 3 * sl;
      dst[(3 * i + j) * d + sl] = (V)src[cidx];
    }
  }
}

// Largest magnitude of each subdomain block (FP16 scale).
__global__ void __launch_bounds__(256) k_sw_scale(const int* __restrict__ sub_off,
                                                  const long long* __restrict__ stage_off,
                                                  const double* __restrict__ B, double* __restrict__ scale) {
  const int s = blockIdx.x;
  const int dim = 3 * (sub_off[s + 1] - sub_off[s]);
  const double* src = B + stage_off[s];
  __shared__ double s_max[8];
  double m = 0.0;
  for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) m = fmax(m, fabs(src[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) mx = fmax(mx, s_max[i]);
    scale[s] = mx > 0.0 ? mx : 1.0;
  }
}

// Schwarz rows into the slot records: slot q (subdomain s, local node I) gets
// rows 3I .. 3I + 2 of the symmetrized inverted block (row-major dim x dim at
// stage_off[s]), FP16 divided by the block's scale.  One warp per slot.
template <class V>
__global__ void __launch_bounds__(256) k_sw_pack(int nslot, const int* __restrict__ slot_sub,
                                                 const int* __restrict__ slot_local, const int* __restrict__ sub_off,
                                                 const long long* __restrict__ stage_off, const double* __restrict__ B,
                                                 const double* __restrict__ scale,
                                                 const long long* __restrict__ rec_val_off,
                                                 unsigned char* __restrict__ data) {
  const int lane = threadIdx.x & 31;
  for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nslot; q += (gridDim.x * blockDim.x) >> 5) {
    const int s = slot_sub[q], I = slot_local[q];
    const int dim = 3 * (sub_off[s + 1] - sub_off[s]);
    const double* src = B + stage_off[s] + (long long)3 * I * dim;
    V* dst = (V*)(data + rec_val_off[q]);
    const double inv = sizeof(V) == 2 ? 1.0 / scale[s] : 1.0;
    for (int k = lane; k < 3 * dim; k += 32) {
      if constexpr (sizeof(V) == 2) dst[k] = __float2half_rn((float)(src[k] * inv));
      else dst[k] = (V)src[k];
    }
  }
}

__global__ void k_cg_stream_arm(CgState* st, double delta2) {
  st->rr_ref = st->rr;
  st->delta2 = delta2;
  st->replace = 0;
  st->pcur = 0;
  st->rcur = 0;
}

// Item weights for the range splits of stream_partition.h: the item's bytes,
// plus extra[i] when given.
std::vector<long long> item_weights(const std::vector<CgsItem>& items, const std::vector<long long>* extra) {
  std::vector<long long> w(items.size());
  for (size_t i = 0; i < items.size(); ++i) w[i] = (long long)items[i].bytes + (extra ? (*extra)[i] : 0LL);
  return w;
}

// Packs consecutive records (byte sizes rec[r], each 16-aligned) into items of
// at most STAGE bytes with a header; item.a = first record, item.b = records;
// the records' absolute offsets go to rec_off.  False if one record alone
// does not fit.
bool pack_items(const std::vector<long long>& rec, long long& pos, std::vector<CgsItem>& items,
                std::vector<long long>& rec_off) {
  const size_t n = rec.size();
  size_t a = 0;
  while (a < n) {
    size_t b = a;
    long long recs = 0;
    while (b < n) {
      const long long hdr = align16(ITEM_HDR + 16 * (long long)(b - a + 1));
      if (hdr + recs + rec[b] > STAGE) break;
      recs += rec[b];
      ++b;
    }
    if (b == a) return false;
    const long long hdr = align16(ITEM_HDR + 16 * (long long)(b - a));
    long long o = pos + hdr;
    for (size_t q = a; q < b; ++q) {
      rec_off[q] = o;
      o += rec[q];
    }
    CgsItem it{};
    it.off = pos;
    it.bytes = (int)(hdr + recs);
    it.a = (int)a;
    it.b = (int)(b - a);
    items.push_back(it);
    pos = o;
    a = b;
  }
  return true;
}

// Incidence (slot) structure of a Schwarz preconditioner in node-major slot
// order: the slots of node a are [pair_off[a], pair_off[a+1]), its subdomains
// ascending; slot_sub / slot_local give (subdomain, local node index).
void schwarz_slots(const Precond& P, i64 nv, std::vector<int>& pair_off, std::vector<int>& slot_sub,
                   std::vector<int>& slot_local) {
  pair_off.assign(nv + 1, 0);
  for (i64 k = 0; k < P.sub_off[P.nsub]; ++k) pair_off[P.sub_nodes[k] + 1] += 1;
  for (i64 a = 0; a < nv; ++a) pair_off[a + 1] += pair_off[a];
  std::vector<int> fill(pair_off.begin(), pair_off.end() - 1);
  slot_sub.assign(P.sub_off[P.nsub], 0);
  slot_local.assign(P.sub_off[P.nsub], 0);
  for (i64 s = 0; s < P.nsub; ++s)
    for (i64 k = P.sub_off[s]; k < P.sub_off[s + 1]; ++k) {
      const int q = fill[P.sub_nodes[k]]++;
      slot_sub[q] = (int)s;
      slot_local[q] = (int)(k - P.sub_off[s]);
    }
}

// Operator layout for value size vsize (and, with a Schwarz preconditioner,
// segments that also bound its incidences); false if a node row does not fit
// a stage or a halo.  Tiles are runs of consecutive nodes; the CTAs get
// contiguous tile ranges of about equal bytes; a CTA's tiles are cut into
// segments whose halo fits HALO_MAX nodes and whose Schwarz incidences fit
// ZMAX / 3.
bool build_op_layout(CgStreamOp& L, Model& m, int vsize, int G, const Precond* P, cudaStream_t s) {
  const i64 nv = m.nv;
  for (i64 q = 0; q < nv; ++q)
    HOEFEM_REQUIRE(m.diag_slot[q] >= 0, HOEFEM_ERR_PATTERN, "streamed CG: a node row without its diagonal block");
  std::vector<int> pair_off, slot_sub, slot_local;
  const bool sw = P && P->kind == PREC_SCHWARZ && P->nsub > 0;
  if (sw) schwarz_slots(*P, nv, pair_off, slot_sub, slot_local);
  auto incid = [&](i64 a) { return sw ? pair_off[a + 1] - pair_off[a] : 0; };
  auto rec_bytes = [&](i64 a) {
    const long long d = m.adj_off[a + 1] - m.adj_off[a];
    return align16(2 * d) + align16(9 * d * vsize);
  };
  // tiles: runs of nodes within a stage and a halo
  std::vector<CgsItem> items;
  std::vector<long long> val_off(nv), idx_off(nv);
  std::vector<int> stamp(nv, -1), rec_node;
  long long pos = 0;
  i64 a = 0;
  int tile_id = 0;
  while (a < nv) {
    const long long start = pos;
    long long recs = 0;
    int uniq = 0, inc = 0;
    i64 b = a;
    std::vector<long long> rec_rel;
    while (b < nv) {
      const long long rec = rec_bytes(b);
      const long long hdr = align16(ITEM_HDR + 16 * (b - a + 1));
      if (hdr + recs + rec > STAGE) break;
      int add = 0;
      for (int e = m.adj_off[b]; e < m.adj_off[b + 1]; ++e) add += stamp[m.adj[e]] != tile_id;
      if (uniq + add > HALO_MAX || 3 * (inc + incid(b)) > ZMAX) break;
      for (int e = m.adj_off[b]; e < m.adj_off[b + 1]; ++e) stamp[m.adj[e]] = tile_id;
      uniq += add;
      inc += incid(b);
      rec_rel.push_back(recs);
      recs += rec;
      ++b;
    }
    if (b == a) return false;  // one node row exceeds a stage or a halo
    const long long hdr = align16(ITEM_HDR + 16 * (b - a));
    // records in order of decreasing degree (groups of four similar rows)
    std::vector<i64> order;
    for (i64 q = a; q < b; ++q) order.push_back(q);
    std::stable_sort(order.begin(), order.end(), [&](i64 x, i64 y) {
      return m.adj_off[x + 1] - m.adj_off[x] > m.adj_off[y + 1] - m.adj_off[y];
    });
    long long o = start + hdr;
    for (i64 q : order) {
      const long long d = m.adj_off[q + 1] - m.adj_off[q];
      idx_off[q] = o;
      val_off[q] = idx_off[q] + align16(2 * d);
      o += rec_bytes(q);
      rec_node.push_back((int)q);
    }
    CgsItem it{};
    it.off = start;
    it.bytes = (int)(hdr + recs);
    it.a = (int)(rec_node.size() - order.size());  // first record (stream order)
    it.b = (int)(b - a);
    it.c = (int)a;  // first node
    items.push_back(it);
    pos = start + hdr + recs;
    a = b;
    ++tile_id;
  }
  std::vector<int> off, nrange(G + 1);
  // CTA ranges balanced for the two phases (split_two_phase): Schwarz
  // bytes counted at the operator's value size cost 1.30 times the operator
  // tile bytes per byte with FP32 values and 0.84 times with FP64 values
  // (phase times per CTA on the benchmark cylinder)
  std::vector<long long> swb;
  if (sw) {
    swb.assign(items.size(), 0);
    for (size_t j = 0; j < items.size(); ++j)
      for (i64 q = items[j].c; q < items[j].c + items[j].b; ++q)
        for (int k = pair_off[q]; k < pair_off[q + 1]; ++k)
          swb[j] += 9LL * (P->sub_off[slot_sub[k] + 1] - P->sub_off[slot_sub[k]]) * vsize;
  }
  // one segment per CTA range where possible: halo and Schwarz incidences of
  // the range within the segment bounds (stamps of the range being built)
  struct SegFit {
    const Model& m;
    const std::vector<CgsItem>& items;
    std::vector<int> stamp;
    std::function<int(i64)> incid;
    int id = 0, uniq = 0, inc = 0;
    void start(int i) {
      ++id;
      uniq = inc = 0;
      add(i);
    }
    bool add(int i) {
      int tinc = 0;
      for (i64 q = items[i].c; q < items[i].c + items[i].b; ++q) {
        tinc += incid(q);
        for (int e = m.adj_off[q]; e < m.adj_off[q + 1]; ++e)
          if (stamp[m.adj[e]] != id) {
            stamp[m.adj[e]] = id;
            ++uniq;
          }
      }
      inc += tinc;
      return uniq <= HALO_MAX && 3 * inc <= ZMAX;
    }
  } fit{m, items, std::vector<int>(nv, 0), incid};
  if (sw) {
    const double kappa = vsize == 8 ? 0.84 : 1.30;
    std::vector<double> wa(items.size()), wb(items.size());
    for (size_t i = 0; i < items.size(); ++i) {
      wa[i] = (double)items[i].bytes;
      wb[i] = kappa * (double)swb[i];
    }
    if (!split_two_phase(wa, wb, G, off, fit)) split_weighted(item_weights(items, &swb), G, off);
  } else {
    split_weighted(item_weights(items, nullptr), G, off);
  }
  for (int g = 0; g <= G; ++g) nrange[g] = off[g] < (int)items.size() ? items[off[g]].c : (int)nv;
  // segments: halo-local neighbour indices (sorted halo, times 3), own halo index
  std::vector<CgsSeg> segs;
  std::vector<int> seg_off(G + 1, 0), halo;
  std::vector<unsigned short> loc_adj(m.adj.size());
  std::vector<int> self_loc(nv, 0), deg(nv);
  std::vector<int> local(nv, -1);
  std::fill(stamp.begin(), stamp.end(), -1);
  int seg_id = 0;
  for (int g = 0; g < G; ++g) {
    seg_off[g] = (int)segs.size();
    int j = off[g];
    while (j < off[g + 1]) {
      std::vector<int> hs;
      int j1 = j, inc = 0;
      while (j1 < off[g + 1]) {
        const CgsItem& it = items[j1];
        int add = 0, tinc = 0;
        for (i64 q = it.c; q < it.c + it.b; ++q) {
          tinc += incid(q);
          for (int e = m.adj_off[q]; e < m.adj_off[q + 1]; ++e)
            if (stamp[m.adj[e]] != seg_id) {
              stamp[m.adj[e]] = seg_id;
              ++add;
              hs.push_back(m.adj[e]);
            }
        }
        if ((int)hs.size() > HALO_MAX || 3 * (inc + tinc) > ZMAX) {
          if (j1 == j) return false;
          for (int r = 0; r < add; ++r) {
            stamp[hs.back()] = -1;
            hs.pop_back();
          }
          break;
        }
        inc += tinc;
        ++j1;
      }
      std::sort(hs.begin(), hs.end());
      for (size_t h = 0; h < hs.size(); ++h) local[hs[h]] = (int)h;
      CgsSeg S{};
      S.j0 = j - off[g];
      S.j1 = j1 - off[g];
      S.halo_off = (int)halo.size();
      S.halo_n = (int)hs.size();
      S.n0 = items[j].c;
      S.n1 = items[j1 - 1].c + items[j1 - 1].b;
      S.own_lo = local[S.n0];
      S.q0 = sw ? pair_off[S.n0] : 0;
      S.q1 = sw ? pair_off[S.n1] : 0;
      halo.insert(halo.end(), hs.begin(), hs.end());
      for (int t = j; t < j1; ++t)
        for (i64 q = items[t].c; q < items[t].c + items[t].b; ++q) {
          for (int e = m.adj_off[q]; e < m.adj_off[q + 1]; ++e)
            loc_adj[e] = (unsigned short)(3 * local[m.adj[e]]);
          self_loc[q] = 3 * local[q];  // every node is its own neighbour (diagonal block)
          deg[q] = m.adj_off[q + 1] - m.adj_off[q];
        }
      segs.push_back(S);
      ++seg_id;
      j = j1;
    }
  }
  seg_off[G] = (int)segs.size();
  L.data.alloc(pos);
  L.items.upload(items, s);
  L.item_off.upload(off, s);
  L.h_items = items;
  L.h_item_off = off;
  L.h_segs = segs;
  L.h_seg_off = seg_off;
  L.h_halo = halo;
  L.keep_applied = -1;
  L.node_range.upload(nrange, s);
  L.val_off.upload(val_off, s);
  L.segs.upload(segs, s);
  L.seg_off.upload(seg_off, s);
  L.halo.upload(halo, s);
  // per record (stream order): its node's list and header fields
  std::vector<long long> r_idx_off(nv);
  std::vector<int> r_src(nv), r_cnt(nv), r_y(nv), r_z(nv);
  for (i64 r = 0; r < nv; ++r) {
    const int q = rec_node[r];
    r_idx_off[r] = idx_off[q];
    r_src[r] = m.adj_off[q];
    r_cnt[r] = deg[q];
    r_y[r] = deg[q];
    r_z[r] = self_loc[q];
  }
  DBuf<unsigned short> d_loc;
  DBuf<int> d_src, d_cnt, d_y, d_z, d_w;
  DBuf<long long> d_idx_off;
  d_loc.upload(loc_adj, s);
  d_src.upload(r_src, s);
  d_cnt.upload(r_cnt, s);
  d_y.upload(r_y, s);
  d_z.upload(r_z, s);
  d_w.upload(rec_node, s);
  d_idx_off.upload(r_idx_off, s);
  L.bytes = pos;
  L.grid = G;
  (note_launch(), k_item_layout<<<(int)items.size(), 256, 0, s>>>((int)items.size(), L.items.p, d_idx_off.p, d_src.p,
                                                                    d_cnt.p, d_loc.p, d_y.p, d_z.p, d_w.p, L.data.p));
  HOEFEM_CUDA(cudaGetLastError());
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  L.vsize = vsize;
  L.seg_for = sw ? (const void*)P : nullptr;
  return true;
}

// Schwarz row records in the segments of the operator layout L: for each
// segment the slots of its nodes (node-major), each record the 16-bit
// halo-local indices (times 3) of the subdomain's nodes and its 3 block rows.
bool build_sw_layout(CgStreamSchwarz& S, const Precond& P, CgStreamOp& L, int vsize, i64 nv, cudaStream_t s) {
  std::vector<int> pair_off, slot_sub, slot_local;
  schwarz_slots(P, nv, pair_off, slot_sub, slot_local);
  const i64 nslot = (i64)slot_sub.size();
  std::vector<long long> rec(nslot), rec_off(nslot), val_off(nslot);
  std::vector<int> cols_off(nslot + 1, 0), dims(nslot), slot_id(nslot);
  for (i64 q = 0; q < nslot; ++q) {
    const int ns = (int)(P.sub_off[slot_sub[q] + 1] - P.sub_off[slot_sub[q]]);
    dims[q] = 3 * ns;
    slot_id[q] = (int)q;
    rec[q] = align16(2LL * ns) + align16(3LL * (3 * ns) * vsize);
    cols_off[q + 1] = cols_off[q] + ns;
  }
  std::vector<unsigned short> cols(cols_off[nslot]);
  std::vector<int> local(nv, -1);
  const int G = L.grid;
  std::vector<CgsItem> items;
  std::vector<int> item_off(G + 1, 0);
  std::vector<CgsSeg> segs = L.h_segs;
  long long pos = 0;
  for (int g = 0; g < G; ++g) {
    item_off[g] = (int)items.size();
    for (int sg = L.h_seg_off[g]; sg < L.h_seg_off[g + 1]; ++sg) {
      CgsSeg& Sg = segs[sg];
      for (int h = 0; h < Sg.halo_n; ++h) local[L.h_halo[Sg.halo_off + h]] = h;
      const int q0 = pair_off[Sg.n0], q1 = pair_off[Sg.n1];
      bool inside = true;
      for (int q = q0; q < q1 && inside; ++q) {
        const i64 sd = slot_sub[q];
        for (i64 k = P.sub_off[sd]; k < P.sub_off[sd + 1]; ++k) {
          const int l = local[P.sub_nodes[k]];
          if (l < 0) {
            inside = false;  // a subdomain node outside the segment's halo
            break;
          }
          cols[cols_off[q] + (k - P.sub_off[sd])] = (unsigned short)(3 * l);
        }
      }
      for (int h = 0; h < Sg.halo_n; ++h) local[L.h_halo[Sg.halo_off + h]] = -1;
      if (!inside) return false;
      Sg.sj0 = (int)items.size() - item_off[g];
      if (q1 > q0) {
        std::vector<long long> r(rec.begin() + q0, rec.begin() + q1), ro(q1 - q0);
        const size_t first = items.size();
        if (!pack_items(r, pos, items, ro)) return false;
        for (size_t i = first; i < items.size(); ++i) items[i].a += q0;  // first slot of the item
        for (int q = q0; q < q1; ++q) {
          rec_off[q] = ro[q - q0];
          val_off[q] = rec_off[q] + align16(2LL * (dims[q] / 3));
        }
      }
      Sg.sj1 = (int)items.size() - item_off[g];
    }
  }
  item_off[G] = (int)items.size();
  S.data.alloc(pos);
  S.items.upload(items, s);
  S.item_off.upload(item_off, s);
  S.h_items = items;
  S.h_item_off = item_off;
  S.keep_applied = -1;
  S.rec_val_off.upload(val_off, s);
  S.slot_sub.upload(slot_sub, s);
  S.slot_local.upload(slot_local, s);
  S.scale.alloc(std::max<i64>(P.nsub, 1));
  // the segments now carry their Schwarz item ranges
  L.h_segs = segs;
  L.segs.upload(segs, s);
  std::vector<int> ncols(nslot), zeros(nslot, 0);
  for (i64 q = 0; q < nslot; ++q) ncols[q] = cols_off[q + 1] - cols_off[q];
  DBuf<unsigned short> d_cols;
  DBuf<int> d_cols_off, d_ncols, d_dims, d_slot, d_zero;
  DBuf<long long> d_rec_off;
  d_cols.upload(cols, s);
  d_cols_off.upload(cols_off, s);
  d_ncols.upload(ncols, s);
  d_dims.upload(dims, s);
  d_slot.upload(slot_id, s);
  d_zero.upload(zeros, s);
  d_rec_off.upload(rec_off, s);
  if (!items.empty())
    (note_launch(), k_item_layout<<<(int)items.size(), 256, 0, s>>>((int)items.size(), S.items.p, d_rec_off.p,
                                                                      d_cols_off.p, d_ncols.p, d_cols.p, d_dims.p,
                                                                      d_slot.p, d_zero.p, S.data.p));
  HOEFEM_CUDA(cudaGetLastError());
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  S.bytes = pos;
  S.grid = G;
  S.vsize = vsize;
  S.built_for = &P;
  S.op_for = &L;
  return true;
}

// L2 keep flags for a budget of `budget` bytes over all CTAs: each CTA keeps
// up to budget / G bytes, its Schwarz records first, then its operator tiles
// from the start of its list.
void apply_keep(CgStreamOp& L, CgStreamSchwarz* S, long long budget, cudaStream_t s) {
  const int G = L.grid;
  const long long per = budget / G;
  for (auto& it : L.h_items) it.keep = 0;
  if (S)
    for (auto& it : S->h_items) it.keep = 0;
  for (int c = 0; c < G; ++c) {
    long long rem = per;
    if (S)
      for (int j = S->h_item_off[c]; j < S->h_item_off[c + 1]; ++j)
        if (S->h_items[j].bytes <= rem) {
          S->h_items[j].keep = 1;
          rem -= S->h_items[j].bytes;
        }
    for (int j = L.h_item_off[c]; j < L.h_item_off[c + 1]; ++j)
      if (L.h_items[j].bytes <= rem) {
        L.h_items[j].keep = 1;
        rem -= L.h_items[j].bytes;
      }
  }
  L.items.upload(L.h_items, s);
  L.keep_applied = budget;
  if (S) {
    S->items.upload(S->h_items, s);
    S->keep_applied = budget;
  }
}

template <class VA, class VB, int PK>
void launch_engine(const Args& args, int G, cudaStream_t s) {
  auto fn = k_cg_stream<VA, VB, PK>;
  static bool configured[64] = {};
  int dev = 0;
  HOEFEM_CUDA(cudaGetDevice(&dev));
  const size_t smem = SMEM_BYTES;
  if (dev >= 0 && dev < 64 && !configured[dev]) {
    HOEFEM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    HOEFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, THREADS, smem));
    HOEFEM_REQUIRE(occ >= 1, HOEFEM_ERR_CUDA, "streamed CG kernel does not fit on a multiprocessor");
    configured[dev] = true;
  }
  Args a = args;
  void* kargs[] = {&a};
  note_launch();
  HOEFEM_CUDA(cudaLaunchCooperativeKernel((const void*)fn, G, THREADS, kargs, smem, s));
}

}  // namespace

bool cg_stream_usable(CgWork& w, const Precond* P) {
  if (w.stream_mode == 1 || w.on_chunk) return false;
  int dev = 0, coop = 0;
  HOEFEM_CUDA(cudaGetDevice(&dev));
  HOEFEM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop || w.m->nv == 0) return false;
  if (P && P->kind == PREC_SCHWARZ && (P->nsub == 0 || 3 * P->max_nodes > MAX_DIM)) return false;
  return true;
}

bool cg_stream_prepare(CgWork& w, const double* A64, bool f32, const Precond* P, bool p32, cudaStream_t s) {
  Model& m = *w.m;
  const int G = device_sms();
  CgStreamOp& L = f32 ? w.sop32 : w.sop64;
  const int vsize = f32 ? 4 : 8;
  const bool sw = P && P->kind == PREC_SCHWARZ && P->nsub > 0;
  const void* seg_for = sw ? (const void*)P : nullptr;
  if (L.vsize != vsize || L.grid != G || L.seg_for != seg_for) {
    if (L.vsize == -vsize && L.seg_for == seg_for) return false;  // layout known not to fit
    if (!build_op_layout(L, m, vsize, G, P, s)) {
      L.vsize = -vsize;
      L.seg_for = seg_for;
      return false;
    }
    w.ssw.vsize = 0;  // the Schwarz records follow the operator segments
  }
  if (sw) {
    const int sv = p32 ? (w.schwarz_half ? 2 : 4) : 8;
    CgStreamSchwarz& S = w.ssw;
    if (S.vsize != sv || S.grid != G || S.built_for != (const void*)P || S.op_for != (const void*)&L) {
      if (!build_sw_layout(S, *P, L, sv, m.nv, s)) {
        S.vsize = 0;
        return false;
      }
    }
    const int nslot = (int)P->sub_off[P->nsub];
    const int ng = std::min(std::max(1, (nslot + 7) / 8), device_sms() * 8);
    if (sv == 2)
      (note_launch(), k_sw_scale<<<(int)P->nsub, 256, 0, s>>>(P->d_sub_off.p, P->d_stage_off.p, P->bsym.p,
                                                               S.scale.p));
    if (sv == 8)
      (note_launch(), k_sw_pack<double><<<ng, 256, 0, s>>>(nslot, S.slot_sub.p, S.slot_local.p, P->d_sub_off.p,
                                                            P->d_stage_off.p, P->bsym.p, S.scale.p,
                                                            S.rec_val_off.p, S.data.p));
    else if (sv == 4)
      (note_launch(), k_sw_pack<float><<<ng, 256, 0, s>>>(nslot, S.slot_sub.p, S.slot_local.p, P->d_sub_off.p,
                                                           P->d_stage_off.p, P->bsym.p, S.scale.p,
                                                           S.rec_val_off.p, S.data.p));
    else
      (note_launch(), k_sw_pack<__half><<<ng, 256, 0, s>>>(nslot, S.slot_sub.p, S.slot_local.p, P->d_sub_off.p,
                                                            P->d_stage_off.p, P->bsym.p, S.scale.p,
                                                            S.rec_val_off.p, S.data.p));
    HOEFEM_CUDA(cudaGetLastError());
  }
  const int ng = std::max(1, (int)((m.nv + 7) / 8));
  if (f32)
    (note_launch(), k_op_pack<float><<<std::min(ng, device_sms() * 8), 256, 0, s>>>(
                        (int)m.nv, m.d_base.p, m.d_adj_off.p, L.val_off.p, A64, L.data.p));
  else
    (note_launch(), k_op_pack<double><<<std::min(ng, device_sms() * 8), 256, 0, s>>>(
                        (int)m.nv, m.d_base.p, m.d_adj_off.p, L.val_off.p, A64, L.data.p));
  HOEFEM_CUDA(cudaGetLastError());
  {
    const long long budget = w.l2_keep < 0 ? 0 : w.l2_keep;
    CgStreamSchwarz* S = sw ? &w.ssw : nullptr;
    if (L.keep_applied != budget || (S && S->keep_applied != budget)) apply_keep(L, S, budget, s);
  }
  if (w.p2.n < (size_t)w.n) w.p2.alloc(w.n);
  if (w.r2.n < (size_t)w.n) w.r2.alloc(w.n);
  if (w.spart.n < (size_t)(3 * G)) w.spart.alloc(3 * G);
  if (!w.sbar.p) w.sbar.alloc(1);
  if (!w.serr.p) w.serr.alloc(2);
  if (!w.sev[0]) {
    HOEFEM_CUDA(cudaEventCreate(&w.sev[0]));
    HOEFEM_CUDA(cudaEventCreate(&w.sev[1]));
  }
  return true;
}

void cg_stream_phase_us(CgWork& w, double* out, double* out_max, double* busy) {
  for (int i = 0; i < 12; ++i) out[i] = out_max[i] = 0.0;
  busy[0] = busy[1] = 0.0;
  if (!w.phase_profile || !w.sprof.p) return;
  std::vector<unsigned long long> h(w.sprof.n);
  HOEFEM_CUDA(cudaMemcpy(h.data(), w.sprof.p, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  const int G = (int)(w.sprof.n / 16);
  unsigned long long its = 0;
  for (int c = 0; c < G; ++c) its = std::max(its, h[16 * c + 12]);
  if (w.sclock_khz <= 0.0) {
    int dev = 0, khz = 0;
    HOEFEM_CUDA(cudaGetDevice(&dev));
    HOEFEM_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev));
    w.sclock_khz = khz > 0 ? khz : 1.0;
  }
  if (its > 0) {
    const double us = 1.0 / (double)its / (w.sclock_khz * 1e-3);
    for (int i = 0; i < 12; ++i) {
      double sum = 0.0, mx = 0.0;
      for (int c = 0; c < G; ++c) {
        sum += (double)h[16 * c + i];
        mx = std::max(mx, (double)h[16 * c + i]);
      }
      out[i] = sum / G * us;
      out_max[i] = mx * us;
    }
    // work outside the grid barriers: halo gathers, operator tiles, Schwarz
    // chunks, own-DOF update
    double bsum = 0.0, bmax = 0.0;
    for (int c = 0; c < G; ++c) {
      const double b = (double)(h[16 * c + 0] + h[16 * c + 1] + h[16 * c + 4] + h[16 * c + 5] + h[16 * c + 8]);
      bsum += b;
      bmax = std::max(bmax, b);
    }
    busy[0] = bsum / G * us;
    busy[1] = bmax * us;
  }
  HOEFEM_CUDA(cudaMemset(w.sprof.p, 0, w.sprof.n * sizeof(unsigned long long)));
}

void cg_stream_arm(CgWork& w, double delta, cudaStream_t s) {
  (note_launch(), k_cg_stream_arm<<<1, 1, 0, s>>>(w.st.p, delta * delta));
  HOEFEM_CUDA(cudaGetLastError());
}

void cg_stream_iterate(CgWork& w, bool f32, const Precond* P, bool p32, bool reliable, cudaStream_t s) {
  (void)p32;
  Model& m = *w.m;
  CgStreamOp& L = f32 ? w.sop32 : w.sop64;
  const int G = L.grid;
  const int pk = !P ? 0 : (P->kind == PREC_DIAGONAL ? 1 : 2);
  Args a{};
  a.op = L.data.p;
  a.op_items = L.items.p;
  a.op_item_off = L.item_off.p;
  a.node_range = L.node_range.p;
  a.segs = L.segs.p;
  a.seg_off = L.seg_off.p;
  a.halo = L.halo.p;
  if (pk == 2) {
    a.sw = w.ssw.data.p;
    a.sw_items = w.ssw.items.p;
    a.sw_item_off = w.ssw.item_off.p;
    a.sw_scale = w.ssw.scale.p;
    a.slot_sub = w.ssw.slot_sub.p;
    a.pair_off = P->d_npair_off.p;
    a.diag_only = P->d_diag_only.p;
    a.pbase = P->d_base.p;
    a.pvals = P->vals.p;
  }
  if (pk == 1) a.dinv = P->diag.p;
  a.x = w.x.p;
  a.r0 = w.r.p;
  a.r1 = w.r2.p;
  a.z = w.z.p;
  a.Ap = w.Ap.p;
  a.pb0 = w.p.p;
  a.pb1 = w.p2.p;
  a.st = w.st.p;
  a.part = w.spart.p;
  a.bar = w.sbar.p;
  a.err = w.serr.p;
  a.reliable = reliable ? 1 : 0;
  if (w.phase_profile) {
    if (w.sprof.n < (size_t)(16 * G)) {
      w.sprof.alloc(16 * G);
      w.sprof.zero(s);
    }
    a.prof = w.sprof.p;
  }
  HOEFEM_CUDA(cudaMemsetAsync(w.sbar.p, 0, sizeof(unsigned), s));
  HOEFEM_CUDA(cudaMemsetAsync(w.serr.p, 0, 2 * sizeof(int), s));
  HOEFEM_CUDA(cudaEventRecord(w.sev[0], s));
  const int sv = w.ssw.vsize;
  if (pk == 2) {
    if (!f32) launch_engine<double, double, 2>(a, G, s);
    else if (sv == 2) launch_engine<float, __half, 2>(a, G, s);
    else if (sv == 4) launch_engine<float, float, 2>(a, G, s);
    else launch_engine<float, double, 2>(a, G, s);
  } else if (pk == 1) {
    if (f32) launch_engine<float, float, 1>(a, G, s);
    else launch_engine<double, double, 1>(a, G, s);
  } else {
    if (f32) launch_engine<float, float, 0>(a, G, s);
    else launch_engine<double, double, 0>(a, G, s);
  }
  HOEFEM_CUDA(cudaGetLastError());
  HOEFEM_CUDA(cudaEventRecord(w.sev[1], s));
  int herr[2] = {0, 0};
  HOEFEM_CUDA(cudaMemcpyAsync(w.h_st, w.st.p, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaMemcpyAsync(herr, w.serr.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  HOEFEM_CUDA(cudaEventElapsedTime(&ms, w.sev[0], w.sev[1]));
  w.stream_ms += ms;
  w.stream_ms_total += ms;
  w.stream_launches += 1;
  w.last_f32 = f32;
  if (herr[0] || herr[1]) throw Error(herr[1] ? herr[1] : HOEFEM_ERR_DEVICE_TIMEOUT, "streamed CG: device wait ran out");
  // the current direction and residual back into w.p / w.r
  if (w.h_st->pcur == 1)
    HOEFEM_CUDA(cudaMemcpyAsync(w.p.p, w.p2.p, sizeof(double) * m.ndof, cudaMemcpyDeviceToDevice, s));
  if (w.h_st->rcur == 1)
    HOEFEM_CUDA(cudaMemcpyAsync(w.r.p, w.r2.p, sizeof(double) * m.ndof, cudaMemcpyDeviceToDevice, s));
}

}  // namespace hoefem
