// Preconditioners: diagonal (Jacobi) and element-wise additive Schwarz.
//
// Reference: DiagonalPreconditioner (simulation_toolbox/src/fem/
// newton_cg.rs:534-593); SchwarzPreconditioner / build_preconditioner_pattern /
// build_schwarz_preconditioner_into / SchwarzElementAssembler /
// invert_element_block (simulation_toolbox/src/fem/schwarz_precond.rs:
// 134-216,250-342, newton_cg.rs:297-370).
//
// Schwarz update on the device, in three steps:
//  1. k_schwarz_gj: one CTA per subdomain gathers its 3n x 3n principal block
//     of the system matrix (element-to-nnz map, no searches) into registers
//     (16 x 16 threads, each a T x T tile) and inverts it by Gauss-Jordan
//     elimination without pivoting.  For a symmetric block every pivot is
//     positive exactly when the block is positive definite; with
//     ||A||_F ||A^-1||_F <= 1e12 (so lambda_min >= 1e-12 lambda_max) the
//     reference's spectrum rule is the plain inverse, which is written to a
//     staging buffer.  Blocks that fail either test are listed for
//     k_schwarz_factor: a parallel cyclic Jacobi eigensolver in shared memory
//     (round-robin ordering: m/2 disjoint rotations per round, rows then
//     columns) that applies the spectrum rule (1/|lambda|, floor
//     1e-12 max|lambda|) and writes the recomposed block V f(L) V^T.
//  2. k_schwarz_scatter: per subdomain color (greedy coloring of the subdomain
//     node lists, as the reference), the staged blocks are added into the
//     preconditioner's own CSR values, so every entry receives its
//     contributions in color order without atomics.
//  3. k_schwarz_untreated: scalar Jacobi 1/a_ii on the untreated nodes.
// The eigen-decomposition replaces LAPACK dsyev (nalgebra-lapack over MKL);
// eigenpairs are not unique, the recomposed block is.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "internal.h"
#include "kernels_common.cuh"
#include "jacobi.cuh"
#include "solver.h"

namespace hoefem {

void greedy_coloring(const i64* conn, i64 ne, int nn, i64 nv, std::vector<i64>& color_off,
                     std::vector<int>& color_elems);
void node_adjacency(i64 nv, const std::vector<const std::vector<i64>*>& conns, const std::vector<int>& nns,
                    std::vector<int>& adj_off, std::vector<int>& adj);

NodeRows Precond::rows() const {
  NodeRows r;
  r.nv = (int)m->nv;
  r.base = d_base.p;
  r.adj_off = d_adj_off.p;
  r.adj = d_adj.p;
  r.diag_slot = d_diag_slot.p;
  r.diag_only = d_diag_only.p;
  r.lanes = spmv_lanes;
  r.sched = d_sched.p;
  r.nodes = d_tnodes.p;
  r.nnodes = (int)tnodes_count;
  r.dnodes = d_untreated.p;
  r.ndnodes = (int)untreated.size();
  return r;
}

namespace {

constexpr int FACTOR_TPB = 256;


// Gauss-Jordan inversion of one SPD principal block per CTA, matrix in
// registers: thread (ty, tx) owns rows ty + 16 ii and columns tx + 16 jj
// (ii, jj < T), padding (index >= dim) is the identity.  Step k broadcasts
// pivot row and column through shared memory (double-buffered: one barrier
// per step).  Blocks with a non-positive pivot or a failed condition
// certificate go to the fallback list.
template <int T>
__global__ void __launch_bounds__(256, 2) k_schwarz_gj(
    int nsub, const int* __restrict__ sub_off, const int* __restrict__ sub_nodes,
    const long long* __restrict__ gmap_off, const int* __restrict__ gmap, const int* __restrict__ adj_off, const long long* __restrict__ jbase,
    const double* __restrict__ J, const long long* __restrict__ stage_off, double* __restrict__ stage,
    int* __restrict__ fallback) {
  constexpr int M = 16 * T;
  __shared__ double s_row[2][M], s_col[2][M], s_piv[2];
  __shared__ int s_g[27], s_rl[27];
  __shared__ long long s_jb[27];
  __shared__ double s_red;
  const int sidx = blockIdx.x;
  const int n = sub_off[sidx + 1] - sub_off[sidx];
  const int dim = 3 * n;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int* nodes = sub_nodes + sub_off[sidx];
  if (threadIdx.x < n) {
    int g = nodes[threadIdx.x];
    s_g[threadIdx.x] = g;
    s_rl[threadIdx.x] = 3 * (adj_off[g + 1] - adj_off[g]);
    s_jb[threadIdx.x] = jbase[g];
  }
  __syncthreads();
  const int* gm = gmap + gmap_off[sidx];
  double a[T][T];
  double fa = 0.0;
#pragma unroll
  for (int ii = 0; ii < T; ++ii) {
    const int r = ty + 16 * ii;
#pragma unroll
    for (int jj = 0; jj < T; ++jj) {
      const int c = tx + 16 * jj;
      double v = (r == c) ? 1.0 : 0.0;
      if (r < dim && c < dim) {
        const int I = r / 3, i = r - 3 * I, Jn = c / 3, j = c - 3 * Jn;
        v = J[s_jb[I] + gm[I * n + Jn] + i * s_rl[I] + j];
        fa += v * v;
      }
      a[ii][jj] = v;
    }
  }
  double v1[1] = {fa};
  block_sum<1>(v1);
  if (threadIdx.x == 0) s_red = sqrt(v1[0]);
  bool ok = true;
  // Step k: the owners of pivot row and column publish them (the pivot
  // itself separately; in its place 1 in the row and -1 in the column) and
  // zero their copies, so that one FMA a_ij - c_i r_j / piv per entry gives the
  // Gauss-Jordan step everywhere: row k -> r_j / piv, column k -> -c_i / piv,
  // pivot -> 1 / piv, the rest the rank-1 update.
  for (int k = 0; k < dim; ++k) {
    const int buf = k & 1;
    const int kq = k >> 4, kr = k & 15;
    if (ty == kr) {
#pragma unroll
      for (int ii = 0; ii < T; ++ii)
        if (ii == kq) {
#pragma unroll
          for (int jj = 0; jj < T; ++jj) {
            const bool pk = (tx == kr) && (jj == kq);
            s_row[buf][tx + 16 * jj] = pk ? 1.0 : a[ii][jj];
            if (pk) s_piv[buf] = a[ii][jj];
            a[ii][jj] = 0.0;
          }
        }
    }
    if (tx == kr) {
#pragma unroll
      for (int jj = 0; jj < T; ++jj)
        if (jj == kq) {
#pragma unroll
          for (int ii = 0; ii < T; ++ii) {
            s_col[buf][ty + 16 * ii] = ((ty == kr) && (ii == kq)) ? -1.0 : a[ii][jj];
            a[ii][jj] = 0.0;
          }
        }
    }
    __syncthreads();
    const double piv = s_piv[buf];
    if (!(piv > 0.0) || !isfinite(piv)) {
      ok = false;
      break;
    }
    const double inv = 1.0 / piv;
    double rj[T], ci[T];
#pragma unroll
    for (int jj = 0; jj < T; ++jj) rj[jj] = s_row[buf][tx + 16 * jj] * inv;
#pragma unroll
    for (int ii = 0; ii < T; ++ii) ci[ii] = s_col[buf][ty + 16 * ii];
#pragma unroll
    for (int ii = 0; ii < T; ++ii)
#pragma unroll
      for (int jj = 0; jj < T; ++jj) a[ii][jj] = __fma_rn(-ci[ii], rj[jj], a[ii][jj]);
  }
  double fi = 0.0;
  if (ok) {
#pragma unroll
    for (int ii = 0; ii < T; ++ii)
#pragma unroll
      for (int jj = 0; jj < T; ++jj) {
        const int r = ty + 16 * ii, c = tx + 16 * jj;
        if (r < dim && c < dim) fi += a[ii][jj] * a[ii][jj];
      }
  }
  double v2[1] = {fi};
  block_sum<1>(v2);  // uniform: `ok` is the same in every thread
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    const double cond = s_red * sqrt(v2[0]);
    s_ok = ok && (cond <= 1e12) && isfinite(cond);
    if (!s_ok) {
      const int slot = atomicAdd(fallback, 1);
      fallback[1 + slot] = sidx;
    }
  }
  __syncthreads();
  if (!s_ok) return;
  double* out = stage + stage_off[sidx];
#pragma unroll
  for (int ii = 0; ii < T; ++ii)
#pragma unroll
    for (int jj = 0; jj < T; ++jj) {
      const int r = ty + 16 * ii, c = tx + 16 * jj;
      if (r < dim && c < dim) out[r * dim + c] = a[ii][jj];
    }
}

// Eigen path for the blocks listed by k_schwarz_gj (count in fallback[0]).
__global__ void __launch_bounds__(FACTOR_TPB) k_schwarz_factor(
    const int* __restrict__ fallback, const int* __restrict__ sub_off, const int* __restrict__ sub_nodes,
    const long long* __restrict__ gmap_off, const int* __restrict__ gmap, const int* __restrict__ adj_off, const long long* __restrict__ jbase,
    const double* __restrict__ J, const long long* __restrict__ stage_off, double* __restrict__ stage, int* err) {
  if ((int)blockIdx.x >= fallback[0]) return;
  extern __shared__ double smem[];
  const int sidx = fallback[1 + blockIdx.x];
  const int n = sub_off[sidx + 1] - sub_off[sidx];
  const int dim = 3 * n;
  const int m = (dim + 1) & ~1;  // even, padded with a dummy index
  double* A = smem;              // m x m
  double* V = A + m * m;         // m x m
  double* cs = V + m * m;        // m/2 cosines
  double* sn = cs + m / 2;       // m/2 sines
  __shared__ int s_g[27];
  __shared__ int s_rl[27];
  __shared__ long long s_jb[27];
  __shared__ double s_red[2];
  const int* nodes = sub_nodes + sub_off[sidx];
  for (int I = threadIdx.x; I < n; I += blockDim.x) {
    int g = nodes[I];
    s_g[I] = g;
    s_rl[I] = 3 * (adj_off[g + 1] - adj_off[g]);
    s_jb[I] = jbase[g];
  }
  __syncthreads();
  // gather the principal block
  const int* gm = gmap + gmap_off[sidx];
  for (int k = threadIdx.x; k < m * m; k += blockDim.x) {
    int r = k / m, c = k % m;
    double v = 0.0;
    if (r < dim && c < dim) {
      int I = r / 3, i = r % 3, Jn = c / 3, j = c % 3;
      v = J[s_jb[I] + gm[I * n + Jn] + i * s_rl[I] + j];
    }
    A[k] = v;
    V[k] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  double* out = stage + stage_off[sidx];

  // ---- general path: cyclic Jacobi eigen-decomposition -------------------------
  jacobi_eigen_block(A, V, cs, sn, m, dim, s_red);
  // spectrum rule of invert_element_block: f = 1/|l| if |l| >= 1e-12 max|l| else 1/(1e-12 max|l|)
  double amax = 0.0;
  for (int k = threadIdx.x; k < dim; k += blockDim.x) amax = fmax(amax, fabs(A[k * m + k]));
  double am[1] = {amax};
  // block max of |lambda| (warp shuffles, then the warp maxima)
  for (int o = 16; o > 0; o >>= 1) am[0] = fmax(am[0], __shfl_xor_sync(0xffffffffu, am[0], o));
  __shared__ double s_max[FACTOR_TPB / 32];
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = am[0];
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, s_max[w]);
    s_red[0] = mx;
  }
  __syncthreads();
  const double lower = 1e-12 * s_red[0];
  for (int k = threadIdx.x; k < dim; k += blockDim.x) {
    double l = A[k * m + k];
    A[k * m + k] = (fabs(l) >= lower) ? 1.0 / fabs(l) : 1.0 / lower;
  }
  __syncthreads();
  if (!(s_red[0] > 0.0) || !isfinite(s_red[0])) {
    if (threadIdx.x == 0) atomicCAS(err, 0, HOEFEM_ERR_NONFINITE);
  }
  // recompose P = V f V^T into the staging buffer (row-major dim x dim)
  for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) {
    int i = k / dim, j = k % dim;
    double s = 0.0;
    for (int t = 0; t < dim; ++t) s += V[i * m + t] * A[t * m + t] * V[j * m + t];
    out[k] = s;
  }
}

__global__ void __launch_bounds__(256) k_schwarz_scatter(const int* __restrict__ subs, int count,
                                                         const int* __restrict__ sub_off,
                                                         const int* __restrict__ sub_nodes,
                                                         const long long* __restrict__ gmap_off,
                                                         const int* __restrict__ smap, const int* __restrict__ padj_off,
                                                         const long long* __restrict__ stage_off,
                                                         const double* __restrict__ stage, double* __restrict__ pv) {
  const int sidx = subs[blockIdx.x];
  const int n = sub_off[sidx + 1] - sub_off[sidx];
  const int dim = 3 * n;
  const int* nodes = sub_nodes + sub_off[sidx];
  const int* sm = smap + gmap_off[sidx];
  const double* blk = stage + stage_off[sidx];
  // symmetric part of the staged block (the Gauss-Jordan inverse is symmetric
  // only up to rounding; the eigen path's recomposition is symmetric exactly)
  for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) {
    int r = k / dim, c = k % dim;
    int I = r / 3, i = r % 3, Jn = c / 3, j = c % 3;
    int g = nodes[I];
    int rl = 3 * (padj_off[g + 1] - padj_off[g]);
    pv[sm[I * n + Jn] + i * rl + j] += 0.5 * (blk[k] + blk[c * dim + r]);
  }
}

// Symmetric part of every staged block (what the scatter adds), kept for the
// block apply.
__global__ void __launch_bounds__(256) k_schwarz_symmetrize(const int* __restrict__ sub_off,
                                                            const long long* __restrict__ stage_off,
                                                            const double* __restrict__ stage,
                                                            double* __restrict__ sym) {
  const int s = blockIdx.x;
  const int dim = 3 * (sub_off[s + 1] - sub_off[s]);
  const double* blk = stage + stage_off[s];
  double* out = sym + stage_off[s];
  for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) {
    const int r = k / dim, c = k % dim;
    out[k] = 0.5 * (blk[k] + blk[c * dim + r]);
  }
}

__global__ void k_schwarz_untreated(int nun, const int* __restrict__ untreated, const long long* __restrict__ pbase,
                                    NodeRows A, const double* __restrict__ J, double* __restrict__ pv, int* err) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * nun) return;
  int a = untreated[t / 3], i = t % 3;
  double v = 0.0;
  int s = A.diag_slot[a];
  if (s >= 0) {
    int d = A.adj_off[a + 1] - A.adj_off[a];
    v = J[A.base[a] + (long long)i * 3 * d + 3 * s + i];
  }
  if (v != 0.0) pv[pbase[a] + i] = 1.0 / v;
  else atomicCAS(err, 0, HOEFEM_ERR_ZERO_DIAGONAL);
}

// Zero the entries of every node row that is not diagonal-only (the
// subdomain entries, before the scatter adds the blocks into them).
__global__ void k_zero_block_rows(int nv, const long long* __restrict__ pbase,
                                  const unsigned char* __restrict__ diag_only, double* __restrict__ pv) {
  for (int a = blockIdx.x; a < nv; a += gridDim.x) {
    if (diag_only[a]) continue;
    const long long b0 = pbase[a], b1 = pbase[a + 1];
    for (long long k = b0 + threadIdx.x; k < b1; k += blockDim.x) pv[k] = 0.0;
  }
}

__global__ void k_diag_inverse(NodeRows A, const double* __restrict__ J, double* __restrict__ d, int* err) {
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
    atomicCAS(err, 0, HOEFEM_ERR_ZERO_DIAGONAL);
  }
}

__global__ void k_mul(int n, const double* __restrict__ d, const double* __restrict__ r, double* __restrict__ z) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = d[i] * r[i];
}

template <int L>
__global__ void k_spmv_plain(NodeRows A, const double* __restrict__ vals, const double* __restrict__ x,
                             double* __restrict__ y) {
  for_each_node<L>(A, [&](int a, int sl) {
    double s0, s1, s2;
    node_row_dot<L>(A, vals, x, a, sl, s0, s1, s2);
    if (a >= 0 && sl == 0) { y[3 * a] = s0; y[3 * a + 1] = s1; y[3 * a + 2] = s2; }
  });
  node_sched_finish(A);
  for_each_diag_dof(A, vals, x, [&](int dof, double v) { y[dof] = v; });
}

}  // namespace

int spmv_grid(int nv, int lanes);

void precond_create_schwarz(Precond& p, const i64* sub_off, const i64* sub_nodes, i64 nsub, const i64* untreated,
                            i64 nun) {
  Model& m = *p.m;
  p.kind = PREC_SCHWARZ;
  p.nsub = nsub;
  p.sub_off.assign(sub_off, sub_off + nsub + 1);
  p.sub_nodes.assign(sub_nodes, sub_nodes + sub_off[nsub]);
  p.untreated.assign(untreated, untreated + nun);
  p.max_nodes = 0;
  for (i64 s = 0; s < nsub; ++s) {
    int n = (int)(sub_off[s + 1] - sub_off[s]);
    HOEFEM_REQUIRE(n >= 1 && n <= 27, HOEFEM_ERR_INVALID_ARGUMENT, "Schwarz subdomains must have 1..27 nodes");
    p.max_nodes = std::max(p.max_nodes, n);
    for (i64 k = sub_off[s]; k < sub_off[s + 1]; ++k)
      HOEFEM_REQUIRE(sub_nodes[k] >= 0 && sub_nodes[k] < m.nv, HOEFEM_ERR_INVALID_ARGUMENT, "node out of range");
  }
  // pattern of build_preconditioner_pattern: subdomain blocks + untreated diagonal
  // Ragged subdomains: gather per-size groups for node_adjacency.
  std::vector<std::vector<i64>> bysize(28);
  for (i64 s = 0; s < nsub; ++s) {
    int n = (int)(sub_off[s + 1] - sub_off[s]);
    bysize[n].insert(bysize[n].end(), sub_nodes + sub_off[s], sub_nodes + sub_off[s + 1]);
  }
  std::vector<const std::vector<i64>*> conns;
  std::vector<int> nns;
  for (int n = 1; n <= 27; ++n)
    if (!bysize[n].empty()) { conns.push_back(&bysize[n]); nns.push_back(n); }
  node_adjacency(m.nv, conns, nns, p.adj_off, p.adj);
  p.diag_only.assign(m.nv, 0);
  for (i64 a : p.untreated) {
    HOEFEM_REQUIRE(a >= 0 && a < m.nv, HOEFEM_ERR_INVALID_ARGUMENT, "untreated node out of range");
    HOEFEM_REQUIRE(p.adj_off[a + 1] == p.adj_off[a], HOEFEM_ERR_INVALID_ARGUMENT,
                   "untreated node belongs to a subdomain");
    p.diag_only[a] = 1;
  }
  p.base.assign(m.nv + 1, 0);
  p.diag_slot.assign(m.nv, -1);
  for (i64 a = 0; a < m.nv; ++a) {
    i64 d = p.adj_off[a + 1] - p.adj_off[a];
    p.base[a + 1] = p.base[a] + (p.diag_only[a] ? 3 : 9 * d);
    const int* b0 = p.adj.data() + p.adj_off[a];
    const int* e0 = p.adj.data() + p.adj_off[a + 1];
    const int* it = std::lower_bound(b0, e0, (int)a);
    if (it != e0 && *it == a) p.diag_slot[a] = (int)(it - b0);
  }
  p.nnz = p.base[m.nv];
  HOEFEM_REQUIRE(p.nnz < (i64)2147483647, HOEFEM_ERR_INVALID_ARGUMENT, "Schwarz pattern exceeds 2^31 non-zeros");
  // gather map (system pattern) and scatter map (preconditioner pattern)
  std::vector<long long> gmap_off(nsub + 1, 0), stage_off(nsub + 1, 0);
  for (i64 s = 0; s < nsub; ++s) {
    i64 n = sub_off[s + 1] - sub_off[s];
    gmap_off[s + 1] = gmap_off[s] + n * n;
    stage_off[s + 1] = stage_off[s] + 9 * n * n;
  }
  std::vector<int> gmap(gmap_off[nsub]), smap(gmap_off[nsub]);
  for (i64 s = 0; s < nsub; ++s) {
    i64 n = sub_off[s + 1] - sub_off[s];
    const i64* nd = sub_nodes + sub_off[s];
    for (i64 I = 0; I < n; ++I)
      for (i64 J = 0; J < n; ++J) {
        i64 a = nd[I], b = nd[J];
        const int* m0 = m.adj.data() + m.adj_off[a];
        const int* m1 = m.adj.data() + m.adj_off[a + 1];
        const int* it = std::lower_bound(m0, m1, (int)b);
        HOEFEM_REQUIRE(it != m1 && *it == b, HOEFEM_ERR_PATTERN, "subdomain block not in the system pattern");
        gmap[gmap_off[s] + I * n + J] = (int)(3 * (it - m0));
        const int* p0 = p.adj.data() + p.adj_off[a];
        const int* p1 = p.adj.data() + p.adj_off[a + 1];
        const int* jt = std::lower_bound(p0, p1, (int)b);
        smap[gmap_off[s] + I * n + J] = (int)(p.base[a] + 3 * (jt - p0));
      }
  }
  // colors of the subdomains (sequential_greedy_coloring of the node lists)
  {
    // ragged greedy coloring: pad to a dense layout with repeated first node
    int mx = p.max_nodes;
    std::vector<i64> dense(nsub * (size_t)mx);
    for (i64 s = 0; s < nsub; ++s)
      for (int k = 0; k < mx; ++k) {
        i64 n = sub_off[s + 1] - sub_off[s];
        dense[s * mx + k] = sub_nodes[sub_off[s] + std::min<i64>(k, n - 1)];
      }
    greedy_coloring(dense.data(), nsub, mx, m.nv, p.color_off, p.color_subs);
  }
  cudaStream_t st = m.stream;
  std::vector<int> so(p.sub_off.begin(), p.sub_off.end()), sn(p.sub_nodes.begin(), p.sub_nodes.end());
  std::vector<int> un(p.untreated.begin(), p.untreated.end());
  p.d_sub_off.upload(so, st);
  p.d_sub_nodes.upload(sn, st);
  p.d_untreated.upload(un, st);
  // rows with subdomain entries (or none at all) are visited by the row
  // kernels; the untreated nodes are applied elementwise
  std::vector<int> tn;
  for (i64 a = 0; a < m.nv; ++a)
    if (!p.diag_only[a]) tn.push_back((int)a);
  p.tnodes_count = (i64)tn.size();
  if (!tn.empty()) p.d_tnodes.upload(tn, st);
  p.d_gmap_off.upload(gmap_off, st);
  p.d_gmap.upload(gmap, st);
  p.d_smap.upload(smap, st);
  p.d_color_subs.upload(p.color_subs, st);
  p.d_adj_off.upload(p.adj_off, st);
  p.d_adj.upload(p.adj, st);
  p.d_diag_slot.upload(p.diag_slot, st);
  p.d_base.upload(p.base, st);
  p.d_diag_only.upload(p.diag_only, st);
  p.d_stage_off.upload(stage_off, st);
  {
    // block apply: every (subdomain, node) incidence gets a slot; a node's
    // slots are consecutive, its subdomains in ascending order
    std::vector<int> poff(m.nv + 1, 0), slot(sub_off[nsub]);
    for (i64 s = 0; s < nsub; ++s)
      for (i64 k = sub_off[s]; k < sub_off[s + 1]; ++k) poff[sub_nodes[k] + 1] += 1;
    for (i64 a = 0; a < m.nv; ++a) poff[a + 1] += poff[a];
    std::vector<int> fill(poff.begin(), poff.end() - 1);
    for (i64 s = 0; s < nsub; ++s)
      for (i64 k = sub_off[s]; k < sub_off[s + 1]; ++k) slot[k] = fill[sub_nodes[k]]++;
    p.d_npair_off.upload(poff, st);
    p.d_npair.upload(slot, st);
    p.ysub.alloc(3 * sub_off[nsub]);
    p.bsym.alloc(stage_off[nsub]);
    p.block_apply = 3 * p.max_nodes <= 96;  // one thread per block row
  }
  p.vals.alloc(p.nnz);
  p.vals.zero(st);
  p.staging.alloc(stage_off[nsub]);
  p.d_err.alloc(1);
  p.d_fallback.alloc(1 + nsub);
  p.d_sched.alloc(2);
  p.d_sched.zero(st);
  p.d_err.zero(st);
  HOEFEM_CUDA(cudaStreamSynchronize(st));
  int m_max = (3 * p.max_nodes + 1) & ~1;
  size_t smem = (size_t)(2 * m_max * m_max + m_max) * sizeof(double);
  HOEFEM_CUDA(cudaFuncSetAttribute(k_schwarz_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  p.spmv_lanes = autotune_spmv_lanes(p.rows(), p.vals.p, st);
}

static void check_err(DBuf<int>& e, cudaStream_t s) {
  int v = 0;
  HOEFEM_CUDA(cudaMemcpyAsync(&v, e.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  if (v) {
    HOEFEM_CUDA(cudaMemsetAsync(e.p, 0, sizeof(int), s));
    throw Error(v, v == HOEFEM_ERR_ZERO_DIAGONAL ? "Can not construct preconditioner: diagonal entry is zero"
                                                 : "non-finite Schwarz block");
  }
}

// Adds the symmetric part of every staged block into the assembled values
// (one launch per Schwarz color: no two blocks of a color share a node).
static void scatter_blocks(Precond& p, cudaStream_t s) {
  const int nc = (int)p.color_off.size() - 1;
  for (int c = 0; c < nc; ++c) {
    int b = (int)p.color_off[c], cnt = (int)(p.color_off[c + 1] - b);
    if (cnt)
      (note_launch(), k_schwarz_scatter<<<cnt, 256, 0, s>>>(p.d_color_subs.p + b, cnt, p.d_sub_off.p, p.d_sub_nodes.p,
                                                             p.d_gmap_off.p, p.d_smap.p, p.d_adj_off.p, p.d_stage_off.p,
                                                             p.staging.p, p.vals.p));
  }
}

void precond_update(Precond& p, const double* J, cudaStream_t s) {
  Model& m = *p.m;
  NodeRows A = m.rows();
  if (p.kind == PREC_DIAGONAL) {
    if (p.diag.n < (size_t)m.ndof) p.diag.alloc(m.ndof);
    if (!p.d_err.p) { p.d_err.alloc(1); p.d_err.zero(s); }
    (note_launch(), k_diag_inverse<<<(int)((m.ndof + 255) / 256), 256, 0, s>>>(A, J, p.diag.p, p.d_err.p));
    HOEFEM_CUDA(cudaGetLastError());
    check_err(p.d_err, s);
    p.ready = true;
    return;
  }
  // with the block apply the subdomain entries are scattered on demand
  const bool lazy = p.block_apply && p.nsub > 0;
  if (!lazy) p.vals.zero(s);
  if (p.nsub > 0) {
    HOEFEM_CUDA(cudaMemsetAsync(p.d_fallback.p, 0, sizeof(int), s));
    const int dmax = 3 * p.max_nodes;
#define HOEFEM_GJ(TT)                                                                                               \
  (note_launch(), k_schwarz_gj<TT><<<(int)p.nsub, 256, 0, s>>>((int)p.nsub, p.d_sub_off.p, p.d_sub_nodes.p,         \
                                                               p.d_gmap_off.p, p.d_gmap.p, m.d_adj_off.p, m.d_base.p, J,\
                                                               p.d_stage_off.p, p.staging.p, p.d_fallback.p))
    if (dmax <= 32) HOEFEM_GJ(2);
    else if (dmax <= 48) HOEFEM_GJ(3);
    else if (dmax <= 64) HOEFEM_GJ(4);
    else HOEFEM_GJ(6);
#undef HOEFEM_GJ
    int m_max = (dmax + 1) & ~1;
    size_t smem = (size_t)(2 * m_max * m_max + m_max) * sizeof(double);
    (note_launch(), k_schwarz_factor<<<(int)p.nsub, FACTOR_TPB, smem, s>>>(p.d_fallback.p, p.d_sub_off.p,
                                                                           p.d_sub_nodes.p, p.d_gmap_off.p, p.d_gmap.p,
                                                                           m.d_adj_off.p, m.d_base.p, J, p.d_stage_off.p,
                                                                           p.staging.p, p.d_err.p));
    HOEFEM_CUDA(cudaGetLastError());
    (note_launch(), k_schwarz_symmetrize<<<(int)p.nsub, 256, 0, s>>>(p.d_sub_off.p, p.d_stage_off.p, p.staging.p,
                                                                      p.bsym.p));
    if (!lazy) scatter_blocks(p, s);
  }
  if (!p.untreated.empty())
    (note_launch(), k_schwarz_untreated<<<(int)((3 * p.untreated.size() + 255) / 256), 256, 0, s>>>(
        (int)p.untreated.size(), p.d_untreated.p, p.d_base.p, A, J, p.vals.p, p.d_err.p));
  HOEFEM_CUDA(cudaGetLastError());
  check_err(p.d_err, s);
  if (p.want_fp32) precond_to_fp32(p, s);
  p.vals_complete = !lazy;
  p.ready = true;
}

void precond_assemble(const Precond& p, cudaStream_t s) {
  if (p.kind != PREC_SCHWARZ || !p.ready || p.vals_complete) return;
  Precond& q = const_cast<Precond&>(p);
  const int nv = (int)q.m->nv;
  (note_launch(), k_zero_block_rows<<<std::min(nv, device_sms() * 16), 128, 0, s>>>(nv, q.d_base.p, q.d_diag_only.p,
                                                                                  q.vals.p));
  scatter_blocks(q, s);
  if (q.vals32.p) to_f32(q.vals.p, q.vals32.p, q.nnz, s);
  HOEFEM_CUDA(cudaGetLastError());
  q.vals_complete = true;
}

// FP32 copies of the Schwarz values: the assembled CSR and the symmetrized
// blocks of the block apply (both, so that either apply can run in FP32).
void precond_to_fp32(Precond& p, cudaStream_t s) {
  if (p.vals32.n < (size_t)p.nnz) p.vals32.alloc(p.nnz);
  to_f32(p.vals.p, p.vals32.p, p.nnz, s);
  if (p.nsub > 0) {
    if (p.bsym32.n < p.bsym.n) p.bsym32.alloc(p.bsym.n);
    to_f32(p.bsym.p, p.bsym32.p, (long long)p.bsym.n, s);
  }
}

void precond_apply(const Precond& p, const double* r, double* z, cudaStream_t s) {
  HOEFEM_REQUIRE(p.ready, HOEFEM_ERR_INVALID_ARGUMENT, "preconditioner has not been updated");
  if (p.kind == PREC_DIAGONAL) {
    int n = (int)p.m->ndof;
    (note_launch(), k_mul<<<reduce_blocks_for(n), 256, 0, s>>>(n, p.diag.p, r, z));
  } else {
    precond_assemble(p, s);
    NodeRows PR = p.rows();
    HOEFEM_LANES_DISPATCH(PR.lanes,
                          (note_launch(), k_spmv_plain<LN><<<spmv_grid(PR.nv, LN), 256, 0, s>>>(PR, p.vals.p, r, z)));
  }
  HOEFEM_CUDA(cudaGetLastError());
}

}  // namespace hoefem
