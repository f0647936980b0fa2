// Tet10 element stiffness on the tensor cores (tcgen05, TF32 x 3), then a
// gather of the element blocks into the CSR values.
//
// Reference: the element stiffness contraction of fenris/src/assembly.rs
// (ElementStiffnessAssembler, :726-797) with the material tangent contraction
// of fenris/src/solid/materials.rs:689-743, scattered as in
// assembly.rs:252-314 (add_element_row_to_csr_row).  Same matrix as the
// CUDA-core kernel of elements.cu (FP32 element arithmetic), computed as one
// large GEMM instead of per-pair register accumulations.
//
// The contraction.  With reference gradients g_I^q = dN_I/dxi at point q and
// the per-point vectors a^(m) = sqrt(w_q |det J|) (row m of J^-1), the node
// pair block is bilinear in the reference gradients:
//   K_IJ[i][j] = sum_q sum_{m,n} g_I^q[m] g_J^q[n] C_e[(i,j); (q,m,n)],
//   C_e[(i,j); (q,m,n)] = pair_block(point q; a^(m), a^(n))[i][j]
// (pair_block is bilinear in its two node vectors).  Psi[(I,J); (q,m,n)] =
// g_I^q[m] g_J^q[n] is the same for every element of a block with one
// quadrature rule, so all element matrices are the product
//   D[(e,i,j); (I,J)] = C[(e,i,j); (q,m,n)] . Psi[(I,J); (q,m,n)]^T,
// M = 9 rows per element (14 elements per 128-row tile), N = 55 node pairs
// I >= J (padded to 64), K = 9 per quadrature point (7 points per K chunk of
// 64 columns, the 64th zero; 14 points = 2 chunks).
//
// Precision: FP32 inputs split as x = hi + lo with hi = tf32(x), lo =
// tf32(x - hi); D = C_hi Psi_hi + C_lo Psi_hi + C_hi Psi_lo accumulated in
// FP32 in tensor memory (the dropped lo.lo term is below FP32 rounding).
//
// The kernel (one CTA per SM, persistent over the element tiles):
//   16 producer warps: per K chunk, the per-point state (F, material, the
//     vectors a, F a, M1 a of m = 0..2) of the chunk's 98 (element, point)
//     items, then the 9 pair blocks of each item, split, into the chunk's A
//     operand (hi, lo) in the UMMA K-major no-swizzle layout; two chunk
//     buffers so that the next chunk is built while the tensor core runs;
//   1 MMA warp: allocates 128 TMEM columns (two 64-column accumulators) and
//     issues, per chunk, 8 K-steps x 3 tcgen05.mma (M 128, N 64, K 8); a
//     tcgen05.commit releases the chunk buffer, another one after a tile's
//     last chunk hands the accumulator to the epilogue;
//   4 epilogue warps: tcgen05.ld of the accumulator rows (one row per
//     thread), stored as element blocks ke[(e * 55 + p) * 9 + 3 i + j].
// The B operand (Psi hi / lo, per block) is built on the host in the same
// layout and copied to shared memory once per CTA.
// All waits are bounded (stream_pipe.cuh): a wait that runs out raises an
// abort flag that every role polls, the MMA warp waits for its last commit,
// and the CTA frees its tensor memory before it returns.
//
// The gather: per CSR node-row block (3 x 3 entries of node pair (a, b)), the
// contributions of the elements that contain both nodes in element order
// (built once on the host), summed in FP64 and added into the values.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "element_math.cuh"
#include "internal.h"
#include "stream_pipe.cuh"

namespace hoefem {

namespace {

constexpr int TC_EPT = 14;          // elements per tile (9 rows each)
constexpr int TC_PPC = 7;           // quadrature points per K chunk
constexpr int TC_MAXCH = 2;         // chunks (quadrature points <= 14)
constexpr int TC_NP = 55;           // Tet10 node pairs I >= J
constexpr int TC_M = 128, TC_N = 64, TC_KC = 64;
constexpr int TC_ITEMS = TC_EPT * TC_PPC;  // (element, point) items per chunk
constexpr int TC_QMAX = TC_PPC * TC_MAXCH;  // quadrature points per element
constexpr int TC_TITEMS = TC_EPT * TC_QMAX; // (element, point) items per tile
constexpr int TC_ITEM_F = 41;       // floats per item: v[3][9], T[9], s1..s4 (odd stride: no bank conflicts)
constexpr int TC_EL_F = 44;         // floats per element: u[30], Ji[9], detJ, mu, lam (corners staged at 30..41 first)
constexpr int EPI_WARPS = 4, MMA_WARP = 4, PROD_WARPS = 16;
constexpr int PROD0 = 32 * (EPI_WARPS + 1);
constexpr int PRODUCERS = 32 * PROD_WARPS;
constexpr int TC_THREADS = PROD0 + PRODUCERS;  // 672
constexpr int A_SPLIT = TC_M * TC_KC * 4;      // 32 KB: one split of one chunk buffer
constexpr int B_SPLIT = TC_N * TC_KC * 4;      // 16 KB: one split of one chunk of Psi
constexpr int OFF_B = 0;                                   // B: [hi, lo][chunk] 64 KB
constexpr int OFF_A = OFF_B + 2 * TC_MAXCH * B_SPLIT;      // A: [buffer][hi, lo] 128 KB
constexpr int OFF_ITEM = OFF_A + 2 * 2 * A_SPLIT;
constexpr int OFF_EL = OFF_ITEM + TC_TITEMS * TC_ITEM_F * 4;
constexpr size_t TC_SMEM = (size_t)OFF_EL + TC_EPT * TC_EL_F * 4;
constexpr int TMEM_COLS = 2 * TC_N;
static_assert(TC_SMEM + 256 <= 227 * 1024, "shared memory (dynamic + static)");
static_assert(TC_TITEMS <= PRODUCERS, "one producer thread per item of a tile");

// Byte offset of (row, k) in a K-major no-swizzle UMMA operand tile with 64
// K columns: 8 x 16-byte core matrices, K-adjacent core matrices 128 B apart
// (leading byte offset), 8-row groups 2048 B apart (stride byte offset).
__host__ __device__ __forceinline__ int canon_off(int row, int k) {
  return (row >> 3) * 2048 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4;
}
constexpr unsigned CANON_LBO = 128, CANON_SBO = 2048;

// Shared-memory matrix descriptor (no swizzle, version 1).
__device__ __forceinline__ uint64_t smem_desc(unsigned addr) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(CANON_LBO >> 4) << 16) |
         ((uint64_t)(CANON_SBO >> 4) << 32) | (1ull << 46);
}
// Instruction descriptor: D FP32, A and B TF32, both K-major, N = 64, M = 128.
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t accum) {
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   pipe::smem_addr(bar))
               : "memory");
}
// 16 columns of this thread's TMEM lane; the wait is in the same asm statement,
// so no use of the registers can be scheduled before it.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct TcArgs {
  BlockDev b;
  const double* X;
  const double* u;
  const float* psi;  // [hi, lo][chunk][B_SPLIT / 4]
  const float* grad; // reference gradients [point][node][3]
  float* ke;         // [ne][55][9]
  MatDev mat;
  int* err;
  int nch;           // K chunks (1 or 2)
  int ntiles;
};

__global__ void __launch_bounds__(TC_THREADS, 1) k_stiffness_tc(TcArgs A) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) uint64_t afull[2], afree[2], accfull[2], accfree[2];
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const BlockDev& b = A.b;
  const int nch = A.nch;

  // ---- setup: barriers, zeroed A buffers (their pad columns stay zero), Psi ----
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2; ++i) {
      pipe::mbar_init(&afull[i], 1);
      pipe::mbar_init(&afree[i], 1);
      pipe::mbar_init(&accfull[i], 1);
      pipe::mbar_init(&accfree[i], EPI_WARPS);
    }
    s_abort = 0;
    pipe::mbar_fence_init();
  }
  {
    float4* a4 = reinterpret_cast<float4*>(sm + OFF_A);
    for (int i = threadIdx.x; i < 4 * A_SPLIT / 16; i += TC_THREADS) a4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    float4* b4 = reinterpret_cast<float4*>(sm + OFF_B);
    const float4* p4 = reinterpret_cast<const float4*>(A.psi);
    for (int s = 0; s < 2; ++s)
      for (int i = threadIdx.x; i < nch * B_SPLIT / 16; i += TC_THREADS)
        b4[s * TC_MAXCH * B_SPLIT / 16 + i] = __ldg(p4 + s * nch * B_SPLIT / 16 + i);
  }
  if (warp == MMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(pipe::smem_addr(&s_tmem)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const int my_tiles = A.ntiles > (int)blockIdx.x ? (A.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nchunks = my_tiles * nch;

  // the first error code wins; the abort flag follows it, so that a role that
  // leaves a wait because of the flag records nothing of its own
  auto raise = [&](int code) {
    atomicCAS(A.err, 0, code);
    __threadfence_block();
    s_abort = 1;
  };

  if (warp >= PROD0 / 32) {
    // ================= producers =================
    const int pt = threadIdx.x - PROD0;
    float* s_item = reinterpret_cast<float*>(sm + OFF_ITEM);
    float* s_el = reinterpret_cast<float*>(sm + OFF_EL);
    // the next tile's node displacements and corners are loaded into
    // registers one tile ahead (producer thread pt < 140 holds node pt % 10 of
    // element pt / 10), so their global latency overlaps the current tile
    static_assert(TC_EPT * 10 <= PRODUCERS, "one producer thread per element node");
    double pu[3] = {0, 0, 0}, px[3] = {0, 0, 0};
    auto prefetch = [&](int tile) {
      const int e0 = tile * TC_EPT;
      if (tile < A.ntiles && pt < min(TC_EPT, b.ne - e0) * 10) {
        const int el = pt / 10, I = pt % 10;
        const int gn = b.conn[I * b.ne + e0 + el];
#pragma unroll
        for (int k = 0; k < 3; ++k) pu[k] = A.u[3 * gn + k];
        if (I < 4) {
#pragma unroll
          for (int k = 0; k < 3; ++k) px[k] = A.X[3 * gn + k];
        }
      }
    };
    prefetch((int)blockIdx.x);
    for (int g = 0; g < nchunks && !s_abort; ++g) {
      const int tl = g / nch, c = g % nch;
      const int tile = (int)blockIdx.x + tl * (int)gridDim.x;
      const int e0 = tile * TC_EPT;
      const int nel = min(TC_EPT, b.ne - e0);
      if (c == 0) {
        // element data of the tile: node displacements and corners, then
        // J^-1, det J and the Lame parameters (over the corners)
        if (pt < nel * 10) {
          const int el = pt / 10, I = pt % 10;
#pragma unroll
          for (int k = 0; k < 3; ++k) s_el[el * TC_EL_F + 3 * I + k] = (float)pu[k];
          if (I < 4) {
#pragma unroll
            for (int k = 0; k < 3; ++k) s_el[el * TC_EL_F + 30 + 3 * I + k] = (float)px[k];
          }
        }
        prefetch(tile + (int)gridDim.x);
        pipe::named_sync(1, PRODUCERS);
        if (pt < nel) {
          float* E = s_el + pt * TC_EL_F;
          float X[12], J[9], Ji[9];
#pragma unroll
          for (int k = 0; k < 12; ++k) X[k] = E[30 + k];
          tet4_jacobian(X, J);
          const float dJ = inv3(J, Ji);
#pragma unroll
          for (int k = 0; k < 9; ++k) E[30 + k] = Ji[k];
          E[39] = dJ;
          const int e = e0 + pt;
          E[40] = (float)(b.emat ? b.emat[2 * e] : A.mat.mu);
          E[41] = (float)(b.emat ? b.emat[2 * e + 1] : A.mat.lambda);
        }
        pipe::named_sync(1, PRODUCERS);
        // stage 1: the state of every (element, point) item of the tile, item
        // el * 14 + q: F = I + H J^-1 with H = sum_I u_I (dN_I/dxi)^T, the
        // material, the vectors a^(m), F a^(m), M1 a^(m) and the pair scalars
        const int el = pt / TC_QMAX, q = pt % TC_QMAX;
        if (pt < TC_TITEMS && el < nel && q < b.nq) {
          const float* E = s_el + el * TC_EL_F;
          const float w = (float)b.qw[q];
          const float* Ji = E + 30;
          const float dJ = E[39];
          const float* gq = A.grad + q * 30;
          float H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
          for (int I = 0; I < 10; ++I) {
            const float g0 = __ldg(gq + 3 * I), g1 = __ldg(gq + 3 * I + 1), g2 = __ldg(gq + 3 * I + 2);
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
              const float uc = E[3 * I + cc];
              H[3 * cc] += uc * g0;
              H[3 * cc + 1] += uc * g1;
              H[3 * cc + 2] += uc * g2;
            }
          }
          float F[9];
#pragma unroll
          for (int cc = 0; cc < 3; ++cc)
#pragma unroll
            for (int k = 0; k < 3; ++k)
              F[3 * cc + k] = H[3 * cc] * Ji[k] + H[3 * cc + 1] * Ji[3 + k] + H[3 * cc + 2] * Ji[6 + k] +
                              (cc == k ? 1.f : 0.f);
          QpState<float> st;
          float* it = s_item + pt * TC_ITEM_F;
          if (dJ == 0.f || !material_state(A.mat.kind, F, E[40], E[41], st, false)) {
            raise(HOEFEM_ERR_SINGULAR);
          } else {
            const float sc = sqrtf(w * fabsf(dJ));
#pragma unroll
            for (int m = 0; m < 3; ++m) {
              const float a[3] = {Ji[3 * m] * sc, Ji[3 * m + 1] * sc, Ji[3 * m + 2] * sc};
              float* v = it + 9 * m;
              v[0] = a[0];
              v[1] = a[1];
              v[2] = a[2];
              mat3vec(st.F, a, v + 3);
              mat3vec(st.M1, a, v + 6);
            }
            QpPair<float> qp;
            qp_pair_from(A.mat.kind, st, qp);
#pragma unroll
            for (int k = 0; k < 9; ++k) it[27 + k] = qp.T[k];
            it[36] = qp.s1;
            it[37] = qp.s2;
            it[38] = qp.s3;
            it[39] = qp.s4;
          }
        }
      }
      pipe::named_sync(1, PRODUCERS);
      // the chunk buffer is free once the MMAs of its previous use completed
      const int bi = g & 1;
      if (g >= 2 && !pipe::mbar_wait(&afree[bi], (unsigned)(((g >> 1) - 1) & 1), &s_abort)) {
        if (!s_abort) raise(HOEFEM_ERR_DEVICE_TIMEOUT);
        break;
      }
      // stage 2: the 9 pair blocks (m, n) of every item, split into hi / lo
      float* a_hi = reinterpret_cast<float*>(sm + OFF_A + bi * 2 * A_SPLIT);
      float* a_lo = reinterpret_cast<float*>(sm + OFF_A + bi * 2 * A_SPLIT + A_SPLIT);
      // task = (ql * 9 + mn) * 14 + el: the lanes of a warp take different
      // elements of one (point, m, n), so their stores land in different banks
      for (int task = pt; task < TC_ITEMS * 9; task += PRODUCERS) {
        const int el = task % TC_EPT, r2 = task / TC_EPT;
        const int mn = r2 % 9, ql = r2 / 9, q = c * TC_PPC + ql;
        const int item = el * TC_QMAX + q;
        if (el >= nel || q >= b.nq) continue;
        const float* it = s_item + item * TC_ITEM_F;
        QpPair<float> qp;
#pragma unroll
        for (int k = 0; k < 9; ++k) qp.T[k] = it[27 + k];
        qp.s1 = it[36];
        qp.s2 = it[37];
        qp.s3 = it[38];
        qp.s4 = it[39];
        const int m = mn / 3, n = mn % 3;
        float acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        pair_block(A.mat.kind, qp, it + 9 * m, it + 9 * n, acc);
        const int k = 9 * ql + mn;
#pragma unroll
        for (int ab = 0; ab < 9; ++ab) {
          const float hi = tf32_round(acc[ab]);
          const float lo = tf32_round(acc[ab] - hi);
          const int o = canon_off(9 * el + ab, k) >> 2;
          a_hi[o] = hi;
          a_lo[o] = lo;
        }
      }
      fence_async_smem();
      pipe::named_sync(1, PRODUCERS);
      if (pt == 0) pipe::mbar_arrive(&afull[bi]);
    }
  } else if (warp == MMA_WARP) {
    // ================= MMA issuer =================
    int last = -1;
    if (lane == 0) {
      const unsigned a_base = pipe::smem_addr(sm + OFF_A), b_base = pipe::smem_addr(sm + OFF_B);
      for (int g = 0; g < nchunks && !s_abort; ++g) {
        const int tl = g / nch, c = g % nch, bi = g & 1, ab = tl & 1;
        if (c == 0 && tl >= 2 && !pipe::mbar_wait(&accfree[ab], (unsigned)(((tl >> 1) - 1) & 1), &s_abort)) {
          if (!s_abort) raise(HOEFEM_ERR_DEVICE_TIMEOUT);
          break;
        }
        if (!pipe::mbar_wait(&afull[bi], (unsigned)((g >> 1) & 1), &s_abort)) {
          if (!s_abort) raise(HOEFEM_ERR_DEVICE_TIMEOUT);
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(ab * TC_N);
        const unsigned ah = a_base + bi * 2 * A_SPLIT, al = ah + A_SPLIT;
        const unsigned bh = b_base + c * B_SPLIT, bl = b_base + TC_MAXCH * B_SPLIT + c * B_SPLIT;
#pragma unroll
        for (int s = 0; s < TC_KC / 8; ++s) {
          const unsigned ko = s * 256;  // 8 TF32 = two 16-byte core matrices along K
          tc_mma(d, smem_desc(ah + ko), smem_desc(bh + ko), (c > 0 || s > 0) ? 1u : 0u);
          tc_mma(d, smem_desc(al + ko), smem_desc(bh + ko), 1u);
          tc_mma(d, smem_desc(ah + ko), smem_desc(bl + ko), 1u);
        }
        tc_commit(&afree[bi]);
        if (c == nch - 1) tc_commit(&accfull[ab]);
        last = g;
      }
      // the last commit (and with it every MMA of this CTA) completes before
      // the tensor memory is released
      if (last >= 0) pipe::mbar_wait(&afree[last & 1], (unsigned)((last >> 1) & 1));
    }
    __syncwarp();
  } else {
    // ================= epilogue =================
    const int row = 32 * warp + lane;
    const int el = row / 9, ab9 = row % 9;
    for (int tl = 0; tl < my_tiles && !s_abort; ++tl) {
      const int ab = tl & 1;
      const int tile = (int)blockIdx.x + tl * (int)gridDim.x;
      const int e0 = tile * TC_EPT;
      const int nel = min(TC_EPT, b.ne - e0);
      bool ok = true;
      if (lane == 0) ok = pipe::mbar_wait(&accfull[ab], (unsigned)((tl >> 1) & 1), &s_abort);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0 && !s_abort) raise(HOEFEM_ERR_DEVICE_TIMEOUT);
        break;
      }
      tc_fence_after();
      float v[TC_N];
      const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(ab * TC_N);
#pragma unroll
      for (int j = 0; j < TC_N / 16; ++j) tmem_ld16(ta + 16 * j, v + 16 * j);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) pipe::mbar_arrive(&accfree[ab]);
      if (el < nel) {
        float* o = A.ke + ((size_t)(e0 + el) * TC_NP) * 9 + ab9;
#pragma unroll
        for (int p = 0; p < TC_NP; ++p) o[9 * p] = v[p];
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == MMA_WARP) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

constexpr int GU = 2;  // contributions loaded together in the gather

// Warp per node row: every 3 x 3 block of the row summed over its element
// contributions (element order), added into the CSR values (assign: stored).
template <class KT>
__global__ void __launch_bounds__(256) k_stiffness_gather(int nv, const int* __restrict__ adj_off,
                                                          const long long* __restrict__ base,
                                                          const int* __restrict__ off, const int* __restrict__ ent,
                                                          const KT* __restrict__ ke, double* __restrict__ vals,
                                                          int assign) {
  const int a = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (a >= nv) return;
  const int s0 = adj_off[a], deg = adj_off[a + 1] - s0;
  const int rl = 3 * deg;
  double* row = vals + base[a];
  for (int s = lane; s < deg; s += 32) {
    const int k0 = off[s0 + s], k1 = off[s0 + s + 1];
    if (k0 == k1 && !assign) continue;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    // two contributions at a time: their codes, then all their loads, then
    // the sums in contribution order
    for (int k = k0; k < k1; k += GU) {
      int code[GU];
#pragma unroll
      for (int u = 0; u < GU; ++u) code[u] = k + u < k1 ? __ldg(ent + k + u) : -1;
      KT v[GU][9];
#pragma unroll
      for (int u = 0; u < GU; ++u) {
        const KT* kb = ke + (size_t)(code[u] >> 1) * 9;
#pragma unroll
        for (int i = 0; i < 9; ++i) v[u][i] = code[u] >= 0 ? __ldg(kb + i) : KT(0);
      }
#pragma unroll
      for (int u = 0; u < GU; ++u) {
        if (code[u] < 0) break;
        if (code[u] & 1) {
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) acc[3 * i + j] += (double)v[u][3 * j + i];
        } else {
#pragma unroll
          for (int i = 0; i < 9; ++i) acc[i] += (double)v[u][i];
        }
      }
    }
    double* o = row + 3 * s;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        if (assign) o[i * rl + j] = acc[3 * i + j];
        else o[i * rl + j] += acc[3 * i + j];
      }
  }
}

// ---- host: reference gradients, Psi image, gather map ------------------------
void tet10_grad_host(int I, const double* xi, double* g) {
  static const int edge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {2, 3}, {1, 3}};
  const double p[4] = {-0.5 * xi[0] - 0.5 * xi[1] - 0.5 * xi[2] - 0.5, 0.5 * xi[0] + 0.5, 0.5 * xi[1] + 0.5,
                       0.5 * xi[2] + 0.5};
  auto g4 = [](int n, double* o) {
    o[0] = n == 0 ? -0.5 : (n == 1 ? 0.5 : 0.0);
    o[1] = n == 0 ? -0.5 : (n == 2 ? 0.5 : 0.0);
    o[2] = n == 0 ? -0.5 : (n == 3 ? 0.5 : 0.0);
  };
  if (I < 4) {
    double gi[3];
    g4(I, gi);
    const double f = 4.0 * p[I] - 1.0;
    for (int k = 0; k < 3; ++k) g[k] = gi[k] * f;
  } else {
    const int a = edge[I - 4][0], c = edge[I - 4][1];
    double ga[3], gc[3];
    g4(a, ga);
    g4(c, gc);
    for (int k = 0; k < 3; ++k) g[k] = ga[k] * 4.0 * p[c] + gc[k] * 4.0 * p[a];
  }
}

float tf32_host(float x) {
  // round to nearest, ties away from zero, on the 10-bit TF32 mantissa
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x1000u) & 0xFFFFE000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

// Node pair (I >= J) of an element with nn nodes, ordered J-major (J = 0:
// I = 0..nn-1, J = 1: I = 1..nn-1, ...), as the element kernels number them.
int pair_index(int nn, int I, int J) { return J * nn - J * (J - 1) / 2 + (I - J); }

// Gather map of a block: per pattern slot, the (element, pair, transposed)
// contributions in element order, as ((e NP + p) << 1) | transposed.
void prepare_gather_map(const Model& m, const Block& blk, cudaStream_t s) {
  if (blk.gmap_ready) return;
  const int nn = blk.nn, np = nn * (nn + 1) / 2;
  const size_t nslot = m.adj.size();
  HOEFEM_REQUIRE(blk.ne * (i64)np * 2 < (i64)2147483647, HOEFEM_ERR_INVALID_ARGUMENT,
                 "too many elements for the stiffness gather map");
  std::vector<int> off(nslot + 1, 0);
  std::vector<int> slot((size_t)blk.ne * nn * nn);
  for (i64 e = 0; e < blk.ne; ++e) {
    const i64* c = blk.conn.data() + e * nn;
    for (int I = 0; I < nn; ++I) {
      const int* b0 = m.adj.data() + m.adj_off[c[I]];
      const int* b1 = m.adj.data() + m.adj_off[c[I] + 1];
      for (int J = 0; J < nn; ++J) {
        const int* it = std::lower_bound(b0, b1, (int)c[J]);
        HOEFEM_REQUIRE(it != b1 && *it == (int)c[J], HOEFEM_ERR_PATTERN, "element node missing from pattern");
        const int sl = (int)(it - m.adj.data());
        slot[((size_t)e * nn + I) * nn + J] = sl;
        off[sl + 1]++;
      }
    }
  }
  for (size_t i = 0; i < nslot; ++i) off[i + 1] += off[i];
  std::vector<int> ent(off[nslot]);
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (i64 e = 0; e < blk.ne; ++e)
    for (int I = 0; I < nn; ++I)
      for (int J = 0; J < nn; ++J) {
        const int sl = slot[((size_t)e * nn + I) * nn + J];
        const int t = I < J ? 1 : 0;
        const int p = t ? pair_index(nn, J, I) : pair_index(nn, I, J);
        ent[fill[sl]++] = (int)(((e * np + p) << 1) | t);
      }
  blk.d_tc_off.upload(off, s);
  blk.d_tc_ent.upload(ent, s);
  blk.gmap_ready = true;
}

// Per node, its (element, local node) incidences in element order, as
// e nn + I: the gather of staged element forces.
void prepare_node_map(const Model& m, const Block& blk, cudaStream_t s) {
  if (blk.nmap_ready) return;
  const int nn = blk.nn;
  HOEFEM_REQUIRE(blk.ne * (i64)nn < (i64)2147483647, HOEFEM_ERR_INVALID_ARGUMENT, "too many elements for the force map");
  std::vector<int> off(m.nv + 1, 0);
  for (i64 k = 0; k < blk.ne * nn; ++k) off[blk.conn[k] + 1]++;
  for (i64 a = 0; a < m.nv; ++a) off[a + 1] += off[a];
  std::vector<int> ent(off[m.nv]);
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (i64 k = 0; k < blk.ne * nn; ++k) ent[fill[blk.conn[k]]++] = (int)k;  // k = e nn + I
  blk.d_noff.upload(off, s);
  blk.d_nent.upload(ent, s);
  blk.nmap_ready = true;
}

__global__ void __launch_bounds__(256) k_forces_gather(int n3, const int* __restrict__ off, const int* __restrict__ ent,
                                                       const double* __restrict__ fst, double* __restrict__ f) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n3) return;
  const int a = t / 3, i = t - 3 * a;
  const int k0 = off[a], k1 = off[a + 1];
  if (k0 == k1) return;
  double acc = 0.0;
  for (int k = k0; k < k1; ++k) acc += fst[(size_t)__ldg(ent + k) * 3 + i];
  f[t] += acc;
}

template <class KT>
void launch_gather(const Model& m, const Block& blk, const KT* ke, double* vals, bool assign, cudaStream_t s) {
  const int nv = (int)m.nv;
  (note_launch(), k_stiffness_gather<KT><<<(nv + 7) / 8, 256, 0, s>>>(nv, m.d_adj_off.p, m.d_base.p, blk.d_tc_off.p,
                                                                         blk.d_tc_ent.p, ke, vals, assign ? 1 : 0));
  HOEFEM_CUDA(cudaGetLastError());
}

void prepare_tc(const Model& m, const Block& blk, cudaStream_t s) {
  const int nq = (int)blk.qw.size();
  const int nch = (nq + TC_PPC - 1) / TC_PPC;
  // Psi image: [hi, lo][chunk][canonical 64 x 64]
  std::vector<float> img((size_t)2 * nch * B_SPLIT / 4, 0.0f);
  for (int c = 0; c < nch; ++c)
    for (int ql = 0; ql < TC_PPC; ++ql) {
      const int q = c * TC_PPC + ql;
      if (q >= nq) break;
      double gr[10][3];
      for (int I = 0; I < 10; ++I) tet10_grad_host(I, &blk.qp[3 * q], gr[I]);
      for (int J = 0; J < 10; ++J)
        for (int I = J; I < 10; ++I) {
          const int p = pair_index(10, I, J);
          for (int mm = 0; mm < 3; ++mm)
            for (int nn = 0; nn < 3; ++nn) {
              const float x = (float)(gr[I][mm] * gr[J][nn]);
              const float hi = tf32_host(x), lo = tf32_host(x - hi);
              const size_t o = (size_t)c * B_SPLIT / 4 + (canon_off(p, 9 * ql + 3 * mm + nn) >> 2);
              img[o] = hi;
              img[(size_t)nch * B_SPLIT / 4 + o] = lo;
            }
        }
    }
  blk.d_tc_psi.upload(img, s);
  // reference gradients per point and node (FP32), read by the point states
  std::vector<float> grad((size_t)nq * 30);
  for (int q = 0; q < nq; ++q)
    for (int I = 0; I < 10; ++I) {
      double g[3];
      tet10_grad_host(I, &blk.qp[3 * q], g);
      for (int k = 0; k < 3; ++k) grad[(size_t)q * 30 + 3 * I + k] = (float)g[k];
    }
  blk.d_tc_grad.upload(grad, s);
  prepare_gather_map(m, blk, s);
  blk.d_tc_ke.alloc((size_t)blk.ne * TC_NP * 9);
  blk.tc_nch = nch;
  blk.tc_ready = true;
}

}  // namespace

bool stiffness_tc_eligible(const Model& m, const Block& blk) {
  if (m.stiffness_path != STIFFNESS_AUTO) return false;
  return blk.kind == HOEFEM_ELEM_TET10 && blk.uniform && !blk.qw.empty() && (int)blk.qw.size() <= TC_PPC * TC_MAXCH &&
         blk.escene.empty() && blk.scene_active == nullptr && blk.ne > 0;
}

void launch_stiffness_tc(const Model& m, const Block& blk, const MatDev& mat, const double* u, double* vals,
                         cudaStream_t s, bool assign) {
  if (!blk.tc_ready) prepare_tc(m, blk, s);
  static bool attr[64] = {};
  int dev = 0;
  HOEFEM_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && !attr[dev]) {
    HOEFEM_CUDA(cudaFuncSetAttribute(k_stiffness_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
    attr[dev] = true;
  }
  TcArgs a;
  a.b = blk.dev();
  a.X = m.d_X.p;
  a.u = u;
  a.psi = blk.d_tc_psi.p;
  a.grad = blk.d_tc_grad.p;
  a.ke = blk.d_tc_ke.p;
  a.mat = mat;
  a.err = m.d_err.p;
  a.nch = blk.tc_nch;
  a.ntiles = (int)((blk.ne + TC_EPT - 1) / TC_EPT);
  const int grid = std::min(device_sms(), a.ntiles);
  (note_launch(), k_stiffness_tc<<<grid, TC_THREADS, TC_SMEM, s>>>(a));
  HOEFEM_CUDA(cudaGetLastError());
  launch_gather<float>(m, blk, blk.d_tc_ke.p, vals, assign, s);
}

bool stiffness_pairs_eligible(const Model& m, const Block& blk) {
  if (m.stiffness_path == STIFFNESS_CUDA_CORES) return false;
  return blk.escene.empty() && blk.scene_active == nullptr && blk.ne > 0;
}

void* stiffness_pair_buffer(const Model& m, const Block& blk, bool f32, cudaStream_t s) {
  prepare_gather_map(m, blk, s);
  const size_t n = (size_t)blk.ne * (blk.nn * (blk.nn + 1) / 2) * 9;
  if (f32) {
    if (blk.d_tc_ke.n < n) blk.d_tc_ke.alloc(n);
    return blk.d_tc_ke.p;
  }
  if (blk.d_pb64.n < n) blk.d_pb64.alloc(n);
  return blk.d_pb64.p;
}

double* forces_stage_buffer(const Model& m, const Block& blk, cudaStream_t s) {
  prepare_node_map(m, blk, s);
  const size_t n = (size_t)blk.ne * blk.nn * 3;
  if (blk.d_fst.n < n) blk.d_fst.alloc(n);
  return blk.d_fst.p;
}

void forces_gather(const Model& m, const Block& blk, double* f, cudaStream_t s) {
  const int n3 = (int)(3 * m.nv);
  (note_launch(), k_forces_gather<<<(n3 + 255) / 256, 256, 0, s>>>(n3, blk.d_noff.p, blk.d_nent.p, blk.d_fst.p, f));
  HOEFEM_CUDA(cudaGetLastError());
}

void stiffness_gather_pairs(const Model& m, const Block& blk, bool f32, double* vals, bool assign, cudaStream_t s) {
  if (f32) launch_gather<float>(m, blk, blk.d_tc_ke.p, vals, assign, s);
  else launch_gather<double>(m, blk, blk.d_pb64.p, vals, assign, s);
}

}  // namespace hoefem
