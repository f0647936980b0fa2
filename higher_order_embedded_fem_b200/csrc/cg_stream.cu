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
// 16 KB work items into a ring of shared-memory stages, cycling through the
// CTA's fixed item list (its operator tiles, then its Schwarz chunks) across
// iterations and gated only by free stages, and 12 consumer warps that
// compute from the stages.  Stage k % NS belongs to consumer warp k % NW
// (NS a multiple of NW), so each stage is used and released in order by one
// warp.  Phases of an iteration, separated by grid barriers:
//   P1  Ap = A p with the direction formed on the fly, p = z + beta p_old
//       (double-buffered), stored for the CTA's own nodes; p.Ap partials
//   P2  Schwarz block products y_s = B_s (r - alpha Ap)_s into node-major slots
//   P3  own DOFs: x += alpha p, r -= alpha Ap, z = sum of the node's slots (or
//       diag / identity), r.r and z.r partials
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
#include <cmath>
#include <vector>

#include "internal.h"
#include "kernels_common.cuh"
#include "solver.h"
#include "stream_pipe.cuh"

namespace hoefem {

namespace {

constexpr int NW = 12;                 // consumer warps
constexpr int NS = 12;                 // ring stages
constexpr int STAGE = 16384;           // bytes per stage (and per work item)
constexpr int THREADS = 32 * (NW + 1);  // + the producer warp (the last one)
constexpr int CONSUMERS = 32 * NW;
constexpr int TILE_HDR = 16;  // int nodes, int first node, 2 x pad; then (record offset, degree) per node
constexpr int MAX_DIM = 84;   // Schwarz block dimension bound (3 x 27 nodes, padded)
static_assert(NS % NW == 0, "each ring stage must belong to one consumer warp");

__host__ __device__ constexpr long long align16(long long x) { return (x + 15) & ~15LL; }

struct Args {
  const unsigned char* op;
  const CgsItem* op_items;
  const int* op_item_off;
  const int* node_range;
  const unsigned char* sw;
  const CgsItem* sw_items;
  const int* sw_item_off;
  const int* sub_off;
  const int* sub_nodes;
  const int* slot;      // slot of every (subdomain, node) incidence
  const int* pair_off;  // nv + 1: a node's slots
  const unsigned char* diag_only;
  const long long* pbase;
  const double* pvals;     // assembled Schwarz values (untreated nodes' 1 / a_ii)
  const double* sw_scale;  // FP16 blocks: per-subdomain scale
  const double* dinv;      // diagonal preconditioner
  double* ysub;
  double* x;
  double* r;
  double* z;
  double* Ap;
  double* pb0;
  double* pb1;
  CgState* st;
  double* part;  // 3 x grid
  unsigned* bar;
  int* err;  // [0] abort flag, [1] error code
  int reliable;
};

// The direction and the residual step, written once so that every use of a
// value (neighbour gathers, own-node stores, block products, the update)
// rounds identically.
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

template <class VA, class VB, int PK>
__global__ void __launch_bounds__(THREADS, 1) k_cg_stream(Args A) {
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ __align__(8) uint64_t full[NS];
  __shared__ __align__(8) uint64_t empty[NS];
  __shared__ volatile int s_stop;
  __shared__ int s_fail, s_gok;
  __shared__ double s_red[NW][2];
  __shared__ double s_rs[NW][MAX_DIM];
  __shared__ double s_bc[3];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x, G = gridDim.x;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NS; ++i) {
      pipe::mbar_init(&full[i], 1);
      pipe::mbar_init(&empty[i], 1);
    }
    s_stop = 0;
    s_fail = 0;
    pipe::mbar_fence_init();
  }
  __syncthreads();
  const int op0 = A.op_item_off[c], nop = A.op_item_off[c + 1] - op0;
  const int sw0 = PK == 2 ? A.sw_item_off[c] : 0;
  const int nsw = PK == 2 ? A.sw_item_off[c + 1] - sw0 : 0;
  const int per = nop + nsw;

  if (warp == NW) {
    // ---- producer: cycle through the CTA's items, gated by free stages ----
    if (lane != 0) return;
    long long k = 0;
    bool late = false;
    while (per > 0 && !s_stop) {
      const int j = (int)(k % per);
      const CgsItem it = j < nop ? A.op_items[op0 + j] : A.sw_items[sw0 + (j - nop)];
      const unsigned char* src = (j < nop ? A.op : A.sw) + it.off;
      const int s = (int)(k % NS);
      const long long use = k / NS;
      if (use > 0 && !pipe::mbar_wait(&empty[s], (unsigned)((use - 1) & 1), &s_stop)) {
        late = !s_stop;
        break;
      }
      pipe::mbar_arrive_expect_tx(&full[s], (unsigned)it.bytes);
      pipe::bulk_g2s(ring + (size_t)s * STAGE, src, (unsigned)it.bytes, &full[s]);
      ++k;
    }
    if (late) {
      atomicExch(&A.err[0], 1);
      atomicCAS(&A.err[1], 0, (int)HOEFEM_ERR_DEVICE_TIMEOUT);
    }
    // the copies still in flight (the last NS issued) land before the CTA exits
    for (long long q = k > NS ? k - NS : 0; q < k; ++q) pipe::mbar_wait(&full[q % NS], (unsigned)((q / NS) & 1));
    return;
  }

  // ---- consumers ----
  const int w = warp;
  const int n0 = A.node_range[c], n1 = A.node_range[c + 1];
  CgState* st = A.st;
  double zTr = st->zTr, beta = st->beta, alpha = st->alpha, pAp = st->pAp, rr = st->rr;
  const double bnorm = st->bnorm, tol = st->tol, rr_ref = st->rr_ref, delta2 = st->delta2;
  long long iters = st->iters;
  const long long max_iter = st->max_iter;
  int status = HOEFEM_OK, done = 0, replace = 0, pcur = 0;
  long long it = 0;
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
    // ---- P1: Ap = A p, p = z + beta p_old, p.Ap ----
    double acc = 0.0;
    for (int j = first_item(kb, 0, w); j < nop; j += NW) {
      const long long k = kb + j;
      const int s = (int)(k % NS);
      if (!warp_wait(&full[s], (unsigned)((k / NS) & 1))) {
        if (lane == 0) fail();
        break;
      }
      const unsigned char* t = ring + (size_t)s * STAGE;
      const int nn = *(const int*)t;
      const int a0 = *(const int*)(t + 4);
      for (int q = 0; q < nn; ++q) {
        const int2 h = *(const int2*)(t + TILE_HDR + 8 * q);
        const int d = h.y;
        const int* adj = (const int*)(t + h.x);
        const VA* v = (const VA*)(t + h.x + align16(4LL * d));
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll 2
        for (int e = lane; e < d; e += 32) {
          const int b3 = 3 * adj[e];
          const double q0 = cg_dir(__ldcg(A.z + b3), beta, __ldcg(pold + b3));
          const double q1 = cg_dir(__ldcg(A.z + b3 + 1), beta, __ldcg(pold + b3 + 1));
          const double q2 = cg_dir(__ldcg(A.z + b3 + 2), beta, __ldcg(pold + b3 + 2));
          s0 += ldv(v + e) * q0 + ldv(v + d + e) * q1 + ldv(v + 2 * d + e) * q2;
          s1 += ldv(v + 3 * d + e) * q0 + ldv(v + 4 * d + e) * q1 + ldv(v + 5 * d + e) * q2;
          s2 += ldv(v + 6 * d + e) * q0 + ldv(v + 7 * d + e) * q1 + ldv(v + 8 * d + e) * q2;
        }
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        if (lane == 0) {
          const int a3 = 3 * (a0 + q);
          const double sv[3] = {s0, s1, s2};
#pragma unroll
          for (int i = 0; i < 3; ++i) {
            const double pa = cg_dir(__ldcg(A.z + a3 + i), beta, __ldcg(pold + a3 + i));
            pnew[a3 + i] = pa;
            A.Ap[a3 + i] = sv[i];
            acc += pa * sv[i];
          }
        }
      }
      __syncwarp();
      if (lane == 0) pipe::mbar_arrive(&empty[s]);
    }
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
    pAp = s_bc[0];
    if (pAp <= 0.0) {
      done = 1;
      status = HOEFEM_CG_INDEFINITE_OPERATOR;
      pcur = (int)((it + 1) & 1);
      break;
    }
    if (zTr <= 0.0) {
      done = 1;
      status = HOEFEM_CG_INDEFINITE_PRECONDITIONER;
      pcur = (int)((it + 1) & 1);
      break;
    }
    alpha = zTr / pAp;
    // ---- P2: Schwarz block products on the updated residual ----
    if (PK == 2) {
      for (int j = first_item(kb, nop, w); j < per; j += NW) {
        const long long k = kb + j;
        const int s = (int)(k % NS);
        if (!warp_wait(&full[s], (unsigned)((k / NS) & 1))) {
          if (lane == 0) fail();
          break;
        }
        const CgsItem itm = A.sw_items[sw0 + (j - nop)];
        const int sd = itm.a, row0 = itm.b, nrows = itm.c;
        const int o = A.sub_off[sd];
        const int dim = 3 * (A.sub_off[sd + 1] - o);
        double* rs = s_rs[w];
        for (int jj = lane; jj < dim; jj += 32) {
          const int dd = 3 * A.sub_nodes[o + jj / 3] + jj % 3;
          rs[jj] = cg_res(__ldcg(A.r + dd), alpha, __ldcg(A.Ap + dd));
        }
        __syncwarp();
        const VB* blk = (const VB*)(ring + (size_t)s * STAGE);
        const double sc = sizeof(VB) == 2 ? A.sw_scale[sd] : 1.0;
        for (int i = lane; i < nrows; i += 32) {
          const VB* row = blk + (size_t)i * dim;
          double b0 = 0.0, b1 = 0.0, b2 = 0.0;
          for (int jj = 0; jj < dim; jj += 3) {
            b0 += ldv(row + jj) * rs[jj];
            b1 += ldv(row + jj + 1) * rs[jj + 1];
            b2 += ldv(row + jj + 2) * rs[jj + 2];
          }
          const int gi = row0 + i;
          A.ysub[3 * A.slot[o + gi / 3] + gi % 3] = ((b0 + b1) + b2) * sc;
        }
        __syncwarp();
        if (lane == 0) pipe::mbar_arrive(&empty[s]);
      }
      if (!grid_sync()) {
        ok = false;
        break;
      }
    }
    // ---- P3: own DOFs: x, r, z, r.r, z.r ----
    double racc = 0.0, zacc = 0.0;
    for (int t = 3 * n0 + (int)threadIdx.x; t < 3 * n1; t += CONSUMERS) {
      const double pc = __ldcg(pnew + t);
      A.x[t] = __fma_rn(alpha, pc, __ldcg(A.x + t));
      const double rn = cg_res(__ldcg(A.r + t), alpha, __ldcg(A.Ap + t));
      A.r[t] = rn;
      double zv;
      if (PK == 2) {
        const int a = t / 3, i = t - 3 * a;
        if (A.diag_only[a]) {
          zv = A.pvals[A.pbase[a] + i] * rn;
        } else {
          zv = 0.0;
          for (int q = A.pair_off[a]; q < A.pair_off[a + 1]; ++q) zv += __ldcg(A.ysub + 3 * q + i);
        }
      } else if (PK == 1) {
        zv = A.dinv[t] * rn;
      } else {
        zv = rn;
      }
      A.z[t] = zv;
      racc += rn * rn;
      zacc += zv * rn;
    }
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
    rr = s_bc[1];
    const double zr = s_bc[2];
    iters += 1;
    ++it;
    pcur = (int)(it & 1);
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
    } else {
      st->done = 1;
      st->status = HOEFEM_ERR_DEVICE_TIMEOUT;
      st->replace = 0;
      st->pcur = 0;
    }
  }
  pipe::named_sync(1, CONSUMERS);
  if (threadIdx.x == 0) s_stop = 1;
}

// ---- stream layouts -----------------------------------------------------------

// Tile headers and neighbour lists (once per layout).
__global__ void k_op_layout(int ntiles, const CgsItem* __restrict__ items, const int* __restrict__ adj_off,
                            const int* __restrict__ adj, const long long* __restrict__ val_off,
                            unsigned char* __restrict__ data) {
  const int tile = blockIdx.x;
  if (tile >= ntiles) return;
  const CgsItem it = items[tile];
  unsigned char* t = data + it.off;
  const int nn = it.b;
  if (threadIdx.x == 0) {
    ((int*)t)[0] = nn;
    ((int*)t)[1] = it.a;
    ((int*)t)[2] = 0;
    ((int*)t)[3] = 0;
  }
  for (int q = threadIdx.x; q < nn; q += blockDim.x) {
    const int a = it.a + q;
    const int d = adj_off[a + 1] - adj_off[a];
    const long long rec = val_off[a] - align16(4LL * d) - it.off;
    ((int2*)(t + TILE_HDR))[q] = make_int2((int)rec, d);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  for (int q = warp; q < nn; q += nwarp) {
    const int a = it.a + q;
    const int o = adj_off[a], d = adj_off[a + 1] - o;
    int* dst = (int*)(data + val_off[a] - align16(4LL * d));
    for (int e = lane; e < d; e += 32) dst[e] = adj[o + e];
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

// Schwarz blocks (symmetrized inverses, row-major dim x dim at stage_off[s])
// into row chunks; FP16 blocks are divided by their largest magnitude first.
template <class V>
__global__ void __launch_bounds__(256) k_sw_pack(const int* __restrict__ sub_off, const long long* __restrict__ stage_off,
                                                 const double* __restrict__ B, const long long* __restrict__ chunk_base,
                                                 const int* __restrict__ rpc, double* __restrict__ scale,
                                                 unsigned char* __restrict__ data) {
  const int s = blockIdx.x;
  const int dim = 3 * (sub_off[s + 1] - sub_off[s]);
  const double* src = B + stage_off[s];
  const int rows = rpc[s];
  const long long cbytes = align16((long long)rows * dim * (long long)sizeof(V));
  double inv = 1.0;
  if (sizeof(V) == 2) {
    __shared__ double s_max[8];
    double m = 0.0;
    for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) m = fmax(m, fabs(src[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
    __syncthreads();
    double mx = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) mx = fmax(mx, s_max[i]);
    if (mx > 0.0) inv = 1.0 / mx;
    if (threadIdx.x == 0) scale[s] = mx > 0.0 ? mx : 1.0;
  }
  for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) {
    const int row = k / dim, col = k - row * dim;
    const int ch = row / rows, rin = row - ch * rows;
    V* dst = (V*)(data + chunk_base[s] + ch * cbytes);
    if constexpr (sizeof(V) == 2) dst[rin * dim + col] = __float2half_rn((float)(src[k] * inv));
    else dst[rin * dim + col] = (V)src[k];
  }
}

__global__ void k_cg_stream_arm(CgState* st, double delta2) {
  st->rr_ref = st->rr;
  st->delta2 = delta2;
  st->replace = 0;
  st->pcur = 0;
}

// Splits `n` items with byte sizes `bytes` into G contiguous groups of about
// equal bytes: off[0..G].
void split_items(const std::vector<CgsItem>& items, int G, std::vector<int>& off) {
  long long total = 0;
  for (auto& it : items) total += it.bytes;
  off.assign(G + 1, 0);
  long long cum = 0;
  int g = 1;
  for (size_t i = 0; i < items.size(); ++i) {
    cum += items[i].bytes;
    while (g < G && cum * (long long)G >= total * (long long)g) off[g++] = (int)(i + 1);
  }
  while (g <= G) off[g++] = (int)items.size();
}

// Operator layout for value size vsize; false if a node row does not fit a
// stage (the streamed CG is then not used).
bool build_op_layout(CgStreamOp& L, Model& m, int vsize, int G, cudaStream_t s) {
  const i64 nv = m.nv;
  std::vector<CgsItem> items;
  std::vector<long long> val_off(nv);
  long long pos = 0;
  i64 a = 0;
  while (a < nv) {
    const long long start = pos;
    long long recs = 0;
    i64 b = a;
    std::vector<long long> rec_rel;
    while (b < nv) {
      const long long d = m.adj_off[b + 1] - m.adj_off[b];
      const long long rec = align16(4 * d) + align16(9 * d * vsize);
      const long long hdr = align16(TILE_HDR + 8 * (b - a + 1));
      if (hdr + recs + rec > STAGE) break;
      rec_rel.push_back(recs);
      recs += rec;
      ++b;
    }
    if (b == a) return false;  // one node row exceeds a stage
    const long long hdr = align16(TILE_HDR + 8 * (b - a));
    for (i64 q = a; q < b; ++q) {
      const long long d = m.adj_off[q + 1] - m.adj_off[q];
      val_off[q] = start + hdr + rec_rel[q - a] + align16(4 * d);
    }
    CgsItem it{};
    it.off = start;
    it.bytes = (int)(hdr + recs);
    it.a = (int)a;
    it.b = (int)(b - a);
    items.push_back(it);
    pos = start + hdr + recs;
    a = b;
  }
  std::vector<int> off, nrange(G + 1);
  split_items(items, G, off);
  for (int g = 0; g <= G; ++g) nrange[g] = off[g] < (int)items.size() ? items[off[g]].a : (int)nv;
  L.data.alloc(pos);
  L.items.upload(items, s);
  L.item_off.upload(off, s);
  L.node_range.upload(nrange, s);
  L.val_off.upload(val_off, s);
  L.bytes = pos;
  L.grid = G;
  (note_launch(), k_op_layout<<<(int)items.size(), 256, 0, s>>>((int)items.size(), L.items.p, m.d_adj_off.p,
                                                                  m.d_adj.p, L.val_off.p, L.data.p));
  HOEFEM_CUDA(cudaGetLastError());
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  L.vsize = vsize;
  return true;
}

void build_sw_layout(CgStreamSchwarz& L, const Precond& P, int vsize, int G, cudaStream_t s) {
  std::vector<CgsItem> items;
  std::vector<long long> base(P.nsub);
  std::vector<int> rpc(P.nsub);
  long long pos = 0;
  for (i64 sd = 0; sd < P.nsub; ++sd) {
    const int dim = (int)(3 * (P.sub_off[sd + 1] - P.sub_off[sd]));
    const int maxrows = std::max(1, STAGE / (dim * vsize));
    const int nch = (dim + maxrows - 1) / maxrows;
    const int rows = (dim + nch - 1) / nch;
    const long long cbytes = align16((long long)rows * dim * vsize);
    base[sd] = pos;
    rpc[sd] = rows;
    for (int ch = 0; ch < nch; ++ch) {
      const int r0 = ch * rows, r1 = std::min(dim, r0 + rows);
      CgsItem it{};
      it.off = pos + ch * cbytes;
      it.bytes = (int)align16((long long)(r1 - r0) * dim * vsize);
      it.a = (int)sd;
      it.b = r0;
      it.c = r1 - r0;
      items.push_back(it);
    }
    pos += nch * cbytes;
  }
  std::vector<int> off;
  split_items(items, G, off);
  L.data.alloc(pos);
  L.items.upload(items, s);
  L.item_off.upload(off, s);
  L.chunk_base.upload(base, s);
  L.rows_per_chunk.upload(rpc, s);
  L.scale.alloc(std::max<i64>(P.nsub, 1));
  L.bytes = pos;
  L.grid = G;
  L.vsize = vsize;
  L.built_for = &P;
  HOEFEM_CUDA(cudaStreamSynchronize(s));
}

template <class VA, class VB, int PK>
void launch_engine(const Args& args, int G, cudaStream_t s) {
  auto fn = k_cg_stream<VA, VB, PK>;
  static bool configured[64] = {};
  int dev = 0;
  HOEFEM_CUDA(cudaGetDevice(&dev));
  const size_t smem = (size_t)NS * STAGE;
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
  if (w.stream_mode != 2 || w.on_chunk) return false;
  int dev = 0, coop = 0;
  HOEFEM_CUDA(cudaGetDevice(&dev));
  HOEFEM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop || w.m->nv == 0) return false;
  if (P && P->kind == PREC_SCHWARZ && (!P->block_apply || P->nsub == 0 || 3 * P->max_nodes > MAX_DIM)) return false;
  return true;
}

void cg_stream_prepare(CgWork& w, const double* A64, bool f32, const Precond* P, bool p32, cudaStream_t s) {
  Model& m = *w.m;
  const int G = device_sms();
  CgStreamOp& L = f32 ? w.sop32 : w.sop64;
  const int vsize = f32 ? 4 : 8;
  if (L.vsize != vsize || L.grid != G) {
    if (!build_op_layout(L, m, vsize, G, s))
      throw Error(HOEFEM_ERR_INVALID_ARGUMENT, "a node row exceeds the streamed CG's stage size");
  }
  const int ng = std::max(1, (int)((m.nv + 7) / 8));
  if (f32)
    (note_launch(), k_op_pack<float><<<std::min(ng, device_sms() * 8), 256, 0, s>>>(
                        (int)m.nv, m.d_base.p, m.d_adj_off.p, L.val_off.p, A64, L.data.p));
  else
    (note_launch(), k_op_pack<double><<<std::min(ng, device_sms() * 8), 256, 0, s>>>(
                        (int)m.nv, m.d_base.p, m.d_adj_off.p, L.val_off.p, A64, L.data.p));
  HOEFEM_CUDA(cudaGetLastError());
  if (P && P->kind == PREC_SCHWARZ && P->nsub > 0) {
    const int sv = p32 ? (w.schwarz_half ? 2 : 4) : 8;
    CgStreamSchwarz& S = w.ssw;
    if (S.vsize != sv || S.grid != G || S.built_for != (const void*)P) build_sw_layout(S, *P, sv, G, s);
    const int ns = (int)P->nsub;
    if (sv == 8)
      (note_launch(), k_sw_pack<double><<<ns, 256, 0, s>>>(P->d_sub_off.p, P->d_stage_off.p, P->bsym.p,
                                                            S.chunk_base.p, S.rows_per_chunk.p, S.scale.p, S.data.p));
    else if (sv == 4)
      (note_launch(), k_sw_pack<float><<<ns, 256, 0, s>>>(P->d_sub_off.p, P->d_stage_off.p, P->bsym.p,
                                                           S.chunk_base.p, S.rows_per_chunk.p, S.scale.p, S.data.p));
    else
      (note_launch(), k_sw_pack<__half><<<ns, 256, 0, s>>>(P->d_sub_off.p, P->d_stage_off.p, P->bsym.p,
                                                            S.chunk_base.p, S.rows_per_chunk.p, S.scale.p, S.data.p));
    HOEFEM_CUDA(cudaGetLastError());
  }
  if (w.p2.n < (size_t)w.n) w.p2.alloc(w.n);
  if (w.spart.n < (size_t)(3 * G)) w.spart.alloc(3 * G);
  if (!w.sbar.p) w.sbar.alloc(1);
  if (!w.serr.p) w.serr.alloc(2);
  if (!w.sev[0]) {
    HOEFEM_CUDA(cudaEventCreate(&w.sev[0]));
    HOEFEM_CUDA(cudaEventCreate(&w.sev[1]));
  }
}

void cg_stream_arm(CgWork& w, double delta, cudaStream_t s) {
  (note_launch(), k_cg_stream_arm<<<1, 1, 0, s>>>(w.st.p, delta * delta));
  HOEFEM_CUDA(cudaGetLastError());
}

void cg_stream_iterate(CgWork& w, bool f32, const Precond* P, bool p32, bool reliable, cudaStream_t s) {
  Model& m = *w.m;
  CgStreamOp& L = f32 ? w.sop32 : w.sop64;
  const int G = L.grid;
  const int pk = !P ? 0 : (P->kind == PREC_DIAGONAL ? 1 : 2);
  Args a{};
  a.op = L.data.p;
  a.op_items = L.items.p;
  a.op_item_off = L.item_off.p;
  a.node_range = L.node_range.p;
  if (P && P->kind == PREC_SCHWARZ) {
    a.sub_off = P->d_sub_off.p;
    a.sub_nodes = P->d_sub_nodes.p;
    a.slot = P->d_npair.p;
    a.pair_off = P->d_npair_off.p;
    a.diag_only = P->d_diag_only.p;
    a.pbase = P->d_base.p;
    a.pvals = P->vals.p;
    a.ysub = P->ysub.p;
    if (P->nsub > 0) {
      a.sw = w.ssw.data.p;
      a.sw_items = w.ssw.items.p;
      a.sw_item_off = w.ssw.item_off.p;
      a.sw_scale = w.ssw.scale.p;
    }
  }
  if (P && P->kind == PREC_DIAGONAL) a.dinv = P->diag.p;
  a.x = w.x.p;
  a.r = w.r.p;
  a.z = w.z.p;
  a.Ap = w.Ap.p;
  a.pb0 = w.p.p;
  a.pb1 = w.p2.p;
  a.st = w.st.p;
  a.part = w.spart.p;
  a.bar = w.sbar.p;
  a.err = w.serr.p;
  a.reliable = reliable ? 1 : 0;
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
  if (w.h_st->pcur == 1)
    HOEFEM_CUDA(cudaMemcpyAsync(w.p.p, w.p2.p, sizeof(double) * m.ndof, cudaMemcpyDeviceToDevice, s));
}

}  // namespace hoefem
