// Learned coarse correction for the Schwarz-preconditioned CG solves.
//
// Not in the reference (an addition on top of its Newton-CG path).  A small
// MLP predicts the coarse part of the converged correction e = A^-1 r of a
// residual r:
//  * coarse space: the nodes are split into S coarse subdomains by recursive
//    coordinate bisection; each carries NM = 32 local polynomial vector modes
//    (3 components x {1, x, y, z, xy, yz, zx, x^2, y^2, z^2} + 2 cubic bending
//    modes), zero on Dirichlet dofs, orthonormalised per subdomain;
//  * features of subdomain s (F = 64): the NM local projections Phi_s^T r_s,
//    the NG = 29 projections of r on global polynomial modes, and the
//    subdomain centroid; projections are divided by ||r||;
//  * MLP F -> 256 -> 256 -> NM (ReLU), trained on (features(r), Phi_s^T e /
//    ||r||) pairs from plain Schwarz-CG solves: the right-hand side b with
//    the converged solution x* (the pair a warm start is asked for), and
//    optionally the iterates (r_k, e_k = x* - x_k); features and targets are
//    standardised per column with the training set's statistics; FP32 master
//    weights, hand-written forward / backward / Adam kernels;
//  * inference: BF16 weights and activations on the tensor cores (mma.sync
//    m16n8k16, FP32 accumulation), x0 = ||r|| sum_s Phi_s c_s.
// The integrator uses x0 as the initial guess of a Jacobian solve only if it
// lowers the residual (||b - A x0|| < ||b||); otherwise the plain solve runs
// from zero.  The plain Schwarz-CG always finishes the solve to its own
// tolerance on ||b||.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

#include "internal.h"
#include "kernels_common.cuh"
#include "learned.h"

namespace hoefem {

namespace {

// ---- host setup helpers ---------------------------------------------------------
// Recursive coordinate bisection of `ids` into `parts` parts (parts power of 2).
void rcb(const std::vector<double>& X, std::vector<int>& ids, int lo, int hi, int parts, int first_part,
         std::vector<int>& part_of) {
  if (parts == 1) {
    for (int k = lo; k < hi; ++k) part_of[ids[k]] = first_part;
    return;
  }
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int k = lo; k < hi; ++k)
    for (int d = 0; d < 3; ++d) {
      mn[d] = std::min(mn[d], X[3 * ids[k] + d]);
      mx[d] = std::max(mx[d], X[3 * ids[k] + d]);
    }
  int ax = 0;
  for (int d = 1; d < 3; ++d)
    if (mx[d] - mn[d] > mx[ax] - mn[ax]) ax = d;
  int mid = lo + (hi - lo) / 2;
  std::nth_element(ids.begin() + lo, ids.begin() + mid, ids.begin() + hi, [&](int a, int b) {
    double xa = X[3 * a + ax], xb = X[3 * b + ax];
    return xa < xb || (xa == xb && a < b);
  });
  rcb(X, ids, lo, mid, parts / 2, first_part, part_of);
  rcb(X, ids, mid, hi, parts / 2, first_part + parts / 2, part_of);
}

// Modified Gram-Schmidt of k vectors of length n (row-major k x n); vectors
// that become numerically zero are left zero.
void mgs(std::vector<double>& V, int k, size_t n) {
  for (int i = 0; i < k; ++i) {
    double* vi = &V[i * n];
    for (int j = 0; j < i; ++j) {
      const double* vj = &V[j * n];
      double d = 0;
      for (size_t t = 0; t < n; ++t) d += vi[t] * vj[t];
      for (size_t t = 0; t < n; ++t) vi[t] -= d * vj[t];
    }
    double nr = 0;
    for (size_t t = 0; t < n; ++t) nr += vi[t] * vi[t];
    nr = std::sqrt(nr);
    if (nr > 1e-10) for (size_t t = 0; t < n; ++t) vi[t] /= nr;
    else for (size_t t = 0; t < n; ++t) vi[t] = 0;
  }
}

// polynomial vector mode k (0..31) at local coordinates (x, y, z); returns the
// component c it lives on and its value.
double mode_value(int k, double x, double y, double z, int& comp) {
  if (k < 30) {
    comp = k / 10;
    switch (k % 10) {
      case 0: return 1.0;
      case 1: return x;
      case 2: return y;
      case 3: return z;
      case 4: return x * y;
      case 5: return y * z;
      case 6: return z * x;
      case 7: return x * x;
      case 8: return y * y;
      default: return z * z;
    }
  }
  comp = k - 30;  // x and y components: cubic bending along z
  return z * z * z;
}

// ---- device kernels --------------------------------------------------------------
constexpr int TPB = 256;

// G[g] = psi_g . r in two deterministic passes: block (c, g) sums DOF chunk c
// of mode g into part[g * C + c], then one thread per mode adds its C chunk
// sums in chunk order (one block per mode alone was latency-bound: 29 blocks
// for 29 x ndof products).
constexpr int GP_CHUNKS = 32;
static_assert(Learned::NG <= 32, "one warp sums the global modes");
__global__ void k_global_proj(int n, const float* __restrict__ psi, const double* __restrict__ r,
                              double* __restrict__ part) {
  const int c = blockIdx.x, g = blockIdx.y;
  const int chunk = (n + GP_CHUNKS - 1) / GP_CHUNKS;
  const int i0 = c * chunk, i1 = min(n, i0 + chunk);
  const float* p = psi + (size_t)g * n;
  double acc = 0.0;
  for (int i = i0 + (int)threadIdx.x; i < i1; i += blockDim.x) acc += (double)p[i] * r[i];
  double v[1] = {acc};
  block_sum<1>(v);
  if (threadIdx.x == 0) part[g * GP_CHUNKS + c] = v[0];
}
__global__ void k_global_proj_sum(int ng, const double* __restrict__ part, float* __restrict__ G) {
  const int g = threadIdx.x;
  if (g >= ng) return;
  double s = 0.0;
  for (int c = 0; c < GP_CHUNKS; ++c) s += part[g * GP_CHUNKS + c];
  G[g] = (float)s;
}

// X[s] = [Phi_s^T r_s / rn, G / rn, centroid_s]
__global__ void k_features(int S, const int* __restrict__ sub_off, const int* __restrict__ sub_dofs,
                           const float* __restrict__ phi, const double* __restrict__ r, const float* __restrict__ G,
                           const float* __restrict__ centroid, const double* __restrict__ rn_ptr, float* __restrict__ X) {
  const int s = blockIdx.x;
  const int b = sub_off[s], n = sub_off[s + 1] - b;
  const float* ph = phi + (size_t)Learned::NM * b;
  const double rn = *rn_ptr;
  const double inv = rn > 0 ? 1.0 / rn : 0.0;
  // warp w computes modes w, w + 8, ...
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = w; k < Learned::NM; k += blockDim.x >> 5) {
    double acc = 0.0;
    for (int i = lane; i < n; i += 32) acc += (double)ph[(size_t)k * n + i] * r[sub_dofs[b + i]];
    acc = warp_sum_d(acc);
    if (lane == 0) X[(size_t)s * Learned::F + k] = (float)(acc * inv);
  }
  for (int g = threadIdx.x; g < Learned::NG; g += blockDim.x)
    X[(size_t)s * Learned::F + Learned::NM + g] = (float)(G[g] * inv);
  if (threadIdx.x < 3) X[(size_t)s * Learned::F + Learned::NM + Learned::NG + threadIdx.x] = centroid[3 * s + threadIdx.x];
}

// T[s] = Phi_s^T e_s / rn
__global__ void k_targets(int S, const int* __restrict__ sub_off, const int* __restrict__ sub_dofs,
                          const float* __restrict__ phi, const double* __restrict__ e, const double* __restrict__ rn_ptr,
                          float* __restrict__ T) {
  const int s = blockIdx.x;
  const int b = sub_off[s], n = sub_off[s + 1] - b;
  const float* ph = phi + (size_t)Learned::NM * b;
  const double rn = *rn_ptr;
  const double inv = rn > 0 ? 1.0 / rn : 0.0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int k = w; k < Learned::NM; k += blockDim.x >> 5) {
    double acc = 0.0;
    for (int i = lane; i < n; i += 32) acc += (double)ph[(size_t)k * n + i] * e[sub_dofs[b + i]];
    acc = warp_sum_d(acc);
    if (lane == 0) T[(size_t)s * Learned::NM + k] = (float)(acc * inv);
  }
}

// x0[dofs of s] = rn * sum_k Phi_s[k] c_s[k]
__global__ void k_apply(int S, const int* __restrict__ sub_off, const int* __restrict__ sub_dofs,
                        const float* __restrict__ phi, const float* __restrict__ C, const double* __restrict__ rn_ptr,
                        double* __restrict__ x0) {
  const int s = blockIdx.x;
  const int b = sub_off[s], n = sub_off[s + 1] - b;
  const float* ph = phi + (size_t)Learned::NM * b;
  __shared__ float c[Learned::NM];
  if (threadIdx.x < Learned::NM) c[threadIdx.x] = C[(size_t)s * Learned::NM + threadIdx.x];
  __syncthreads();
  const double rn = *rn_ptr;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double acc = 0.0;
#pragma unroll 8
    for (int k = 0; k < Learned::NM; ++k) acc += (double)ph[(size_t)k * n + i] * c[k];
    x0[sub_dofs[b + i]] = rn * acc;
  }
}

__global__ void k_sqrt_to(const double* __restrict__ rr, double* __restrict__ out) { *out = sqrt(fmax(*rr, 0.0)); }

__global__ void k_sub(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ c) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c[i] = a[i] - b[i];
}

__global__ void k_norm(int n, const double* __restrict__ a, double* out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += a[i] * a[i];
  double v[1] = {acc};
  block_sum<1>(v);
  if (threadIdx.x == 0) *out = sqrt(v[0]);
}

// ---- FP32 GEMM (training): C = op(A) op(B) (+bias) (ReLU), C row-major M x N.
// A: M x K (TA = 0: A[m*lda+k]; TA = 1: A[k*lda+m]); B: K x N (TB = 0:
// B[k*ldb+n]; TB = 1: B[n*ldb+k]).  64 x 64 tiles, 256 threads, 4 x 4 per thread.
template <int TA, int TB>
__global__ void __launch_bounds__(256) k_gemm_f32(int M, int N, int K, const float* __restrict__ A, int lda,
                                                  const float* __restrict__ B, int ldb, float* __restrict__ C, int ldc,
                                                  const float* __restrict__ bias, int relu) {
  __shared__ float As[16][65];
  __shared__ float Bs[16][65];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int i = threadIdx.x; i < 64 * 16; i += 256) {
      int mm = i / 16, kk = i % 16, gm = m0 + mm, gk = k0 + kk;
      As[kk][mm] = (gm < M && gk < K) ? (TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk]) : 0.f;
    }
    for (int i = threadIdx.x; i < 16 * 64; i += 256) {
      int kk = i / 64, nn = i % 64, gk = k0 + kk, gn = n0 + nn;
      Bs[kk][nn] = (gk < K && gn < N) ? (TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) { a[i] = As[kk][ty * 4 + i]; b[i] = Bs[kk][tx * 4 + i]; }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gm = m0 + ty * 4 + i, gn = n0 + tx * 4 + j;
      if (gm < M && gn < N) {
        float v = acc[i][j] + (bias ? bias[gn] : 0.f);
        if (relu) v = fmaxf(v, 0.f);
        C[(size_t)gm * ldc + gn] = v;
      }
    }
}

// dY3 = 2 (Y3 - T) / (rows * cols); loss partial sums
__global__ void k_mse_grad(int n, float scale, const float* __restrict__ Y, const float* __restrict__ T,
                           float* __restrict__ dY, double* loss) {
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float d = Y[i] - T[i];
    dY[i] = 2.f * d * scale;
    acc += (double)d * d;
  }
  double v[1] = {acc};
  block_sum<1>(v);
  if (threadIdx.x == 0) atomicAdd(loss, v[0] * scale);
}

// dY *= (Y > 0)
__global__ void k_relu_mask(int n, const float* __restrict__ Y, float* __restrict__ dY) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (!(Y[i] > 0.f)) dY[i] = 0.f;
}

// db[j] = sum_i dY[i, j]
__global__ void k_colsum(int rows, int cols, const float* __restrict__ dY, float* __restrict__ db) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  float acc = 0.f;
  for (int i = 0; i < rows; ++i) acc += dY[(size_t)i * cols + j];
  db[j] = acc;
}

__global__ void k_adam(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi;
    float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void k_f32_to_bf16_t(int K, int N, const float* __restrict__ W, uint16_t* __restrict__ Wt) {
  // W: K x N row-major -> Wt: N x K row-major (i.e. W column-major), BF16 round to nearest even
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= K * N) return;
  int k = i / N, n = i % N;
  uint32_t u = __float_as_uint(W[i]);
  u += 0x7FFFu + ((u >> 16) & 1u);
  Wt[(size_t)n * K + k] = (uint16_t)(u >> 16);
}

__global__ void k_f32_to_bf16(int n, const float* __restrict__ a, uint16_t* __restrict__ b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t u = __float_as_uint(a[i]);
  u += 0x7FFFu + ((u >> 16) & 1u);
  b[i] = (uint16_t)(u >> 16);
}

// BF16 tensor-core GEMM (inference): C = A Wt^T + bias (ReLU), A: M x K BF16
// row-major, Wt: N x K BF16 row-major, FP32 accumulation (mma.sync m16n8k16).
// Each warp computes one 16 x 8 tile.  M % 16 == 0, N % 8 == 0, K % 16 == 0.
// Output written as FP32 (Cf) and / or BF16 (Cb).
__global__ void k_gemm_bf16_tc(int M, int N, int K, const uint16_t* __restrict__ A, const uint16_t* __restrict__ Wt,
                               const float* __restrict__ bias, int relu, float* __restrict__ Cf,
                               uint16_t* __restrict__ Cb) {
  const int lane = threadIdx.x & 31;
  const int tile = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int tiles_n = N / 8;
  if (tile >= (M / 16) * tiles_n) return;
  const int m0 = (tile / tiles_n) * 16, n0 = (tile % tiles_n) * 8;
  const int g = lane >> 2, t = lane & 3;
  float c[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += 16) {
    const uint32_t* a_lo = reinterpret_cast<const uint32_t*>(A + (size_t)(m0 + g) * K + k0);
    const uint32_t* a_hi = reinterpret_cast<const uint32_t*>(A + (size_t)(m0 + g + 8) * K + k0);
    uint32_t a0 = a_lo[t], a1 = a_hi[t], a2 = a_lo[t + 4], a3 = a_hi[t + 4];
    const uint32_t* bcol = reinterpret_cast<const uint32_t*>(Wt + (size_t)(n0 + g) * K + k0);
    uint32_t b0 = bcol[t], b1 = bcol[t + 4];
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
  }
  const int rows[2] = {m0 + g, m0 + g + 8};
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      int col = n0 + 2 * t + j;
      float v = c[2 * h + j] + (bias ? bias[col] : 0.f);
      if (relu) v = fmaxf(v, 0.f);
      if (Cf) Cf[(size_t)rows[h] * N + col] = v;
      if (Cb) {
        uint32_t u = __float_as_uint(v);
        u += 0x7FFFu + ((u >> 16) & 1u);
        Cb[(size_t)rows[h] * N + col] = (uint16_t)(u >> 16);
      }
    }
}

__global__ void k_gather_rows(int rows, int width, const long long* __restrict__ idx, const float* __restrict__ src,
                              float* __restrict__ dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * width) return;
  int r = i / width, c = i % width;
  dst[i] = src[idx[r] * width + c];
}

// dst = (src[idx] - mean) / std, row by row
__global__ void k_gather_rows_std(int rows, int width, const long long* __restrict__ idx,
                                  const float* __restrict__ src, const float* __restrict__ mean,
                                  const float* __restrict__ sd, float* __restrict__ dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * width) return;
  int r = i / width, c = i % width;
  dst[i] = (src[idx[r] * width + c] - mean[c]) / sd[c];
}

__global__ void k_standardise(int rows, int width, const float* __restrict__ mean, const float* __restrict__ sd,
                              float* __restrict__ x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * width) return;
  int c = i % width;
  x[i] = (x[i] - mean[c]) / sd[c];
}

__global__ void k_unstandardise(int rows, int width, const float* __restrict__ mean, const float* __restrict__ sd,
                                float* __restrict__ y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * width) return;
  int c = i % width;
  y[i] = mean[c] + sd[c] * y[i];
}

void gemm(int M, int N, int K, const float* A, int lda, int ta, const float* B, int ldb, int tb, float* C, int ldc,
          const float* bias, int relu, cudaStream_t s) {
  dim3 grid((N + 63) / 64, (M + 63) / 64);
  if (!ta && !tb) (note_launch(), k_gemm_f32<0, 0><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, relu));
  else if (ta && !tb) (note_launch(), k_gemm_f32<1, 0><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, relu));
  else if (!ta && tb) (note_launch(), k_gemm_f32<0, 1><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, relu));
  else (note_launch(), k_gemm_f32<1, 1><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, relu));
  HOEFEM_CUDA(cudaGetLastError());
}

}  // namespace

Learned::~Learned() {
  if (h_scal) cudaFreeHost(h_scal);
}

void Learned::setup(Model* model, const unsigned char* bc_mask, int num_sub, uint64_t seed) {
  m = model;
  S = num_sub;
  HOEFEM_REQUIRE(S >= 2 && (S & (S - 1)) == 0 && S <= 4096, HOEFEM_ERR_INVALID_ARGUMENT,
                 "number of coarse subdomains must be a power of two in [2, 4096]");
  HOEFEM_REQUIRE(m->nv >= S, HOEFEM_ERR_INVALID_ARGUMENT, "fewer nodes than coarse subdomains");
  const i64 nv = m->nv, ndof = m->ndof;
  bc.assign(bc_mask, bc_mask + ndof);
  cudaStream_t s = m->stream;
  // partition
  std::vector<int> ids(nv), part(nv);
  std::iota(ids.begin(), ids.end(), 0);
  rcb(m->X, ids, 0, (int)nv, S, 0, part);
  std::vector<int> cnt(S + 1, 0);
  for (i64 a = 0; a < nv; ++a) cnt[part[a] + 1] += 3;
  for (int k = 0; k < S; ++k) cnt[k + 1] += cnt[k];
  sub_off = cnt;
  sub_dofs.assign(ndof, 0);
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  for (i64 a = 0; a < nv; ++a)
    for (int c = 0; c < 3; ++c) sub_dofs[fill[part[a]]++] = (int)(3 * a + c);
  // bounding box for normalised coordinates
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (i64 a = 0; a < nv; ++a)
    for (int d = 0; d < 3; ++d) {
      mn[d] = std::min(mn[d], m->X[3 * a + d]);
      mx[d] = std::max(mx[d], m->X[3 * a + d]);
    }
  double ext = std::max({mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2], 1e-300});
  // local modes per subdomain
  std::vector<float> phi((size_t)NM * ndof);
  centroid.assign(3 * S, 0.f);
  for (int sidx = 0; sidx < S; ++sidx) {
    const int b = sub_off[sidx], n = sub_off[sidx + 1] - b;
    double c0[3] = {0, 0, 0}, lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; i += 3) {
      int a = sub_dofs[b + i] / 3;
      for (int d = 0; d < 3; ++d) {
        double x = m->X[3 * a + d];
        c0[d] += x;
        lo[d] = std::min(lo[d], x);
        hi[d] = std::max(hi[d], x);
      }
    }
    const int nn = std::max(n / 3, 1);
    for (int d = 0; d < 3; ++d) {
      c0[d] /= nn;
      centroid[3 * sidx + d] = (float)((c0[d] - mn[d]) / ext * 2.0 - 1.0);
    }
    double h = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-12}) * 0.5;
    std::vector<double> V((size_t)NM * n, 0.0);
    for (int k = 0; k < NM; ++k)
      for (int i = 0; i < n; ++i) {
        int dof = sub_dofs[b + i], a = dof / 3, c = dof % 3;
        int comp;
        double v = mode_value(k, (m->X[3 * a] - c0[0]) / h, (m->X[3 * a + 1] - c0[1]) / h, (m->X[3 * a + 2] - c0[2]) / h,
                              comp);
        V[(size_t)k * n + i] = (comp == c && !bc[dof]) ? v : 0.0;
      }
    mgs(V, NM, n);
    for (size_t t = 0; t < V.size(); ++t) phi[(size_t)NM * b + t] = (float)V[t];
  }
  // global modes
  std::vector<double> G((size_t)NG * ndof, 0.0);
  for (int k = 0; k < NG; ++k)
    for (i64 a = 0; a < nv; ++a) {
      double x = (m->X[3 * a] - mn[0]) / ext * 2 - 1, y = (m->X[3 * a + 1] - mn[1]) / ext * 2 - 1,
             z = (m->X[3 * a + 2] - mn[2]) / ext * 2 - 1;
      int comp;
      double v = mode_value(k, x, y, z, comp);
      i64 dof = 3 * a + comp;
      G[(size_t)k * ndof + dof] = bc[dof] ? 0.0 : v;
    }
  mgs(G, NG, ndof);
  std::vector<float> Gf(G.begin(), G.end());
  d_sub_off.upload(sub_off, s);
  d_sub_dofs.upload(sub_dofs, s);
  d_phi.upload(phi, s);
  d_psi.upload(Gf, s);
  d_centroid.upload(centroid, s);
  d_gproj.alloc(NG);
  d_gpart.alloc((size_t)NG * GP_CHUNKS);
  // MLP parameters (He initialisation, seeded)
  n_params = (size_t)F * H + H + (size_t)H * H + H + (size_t)H * NM + NM;
  std::vector<float> p0(n_params, 0.f);
  std::mt19937_64 rng(seed);
  auto init = [&](size_t off, int fan_in, size_t count) {
    std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / fan_in));
    for (size_t i = 0; i < count; ++i) p0[off + i] = (float)nd(rng);
  };
  init(0, F, (size_t)F * H);
  init((size_t)F * H + H, H, (size_t)H * H);
  init((size_t)F * H + H + (size_t)H * H + H, H, (size_t)H * NM);
  // the output layer starts small so that an untrained model predicts ~0
  for (size_t i = 0; i < (size_t)H * NM; ++i) p0[(size_t)F * H + H + (size_t)H * H + H + i] *= 0.01f;
  params.upload(p0, s);
  for (auto* b : {&grads, &adam_m, &adam_v}) {
    b->alloc(n_params);
    b->zero(s);
  }
  params_bf16.alloc((size_t)F * H + (size_t)H * H + (size_t)H * NM);
  {
    std::vector<float> zf(F, 0.f), of(F, 1.f), zt(NM, 0.f), ot(NM, 1.f);
    x_mean.upload(zf, s);
    x_std.upload(of, s);
    t_mean.upload(zt, s);
    t_std.upload(ot, s);
  }
  max_batch = std::max(S, 1024);
  for (auto* b : {&X, &dY1}) b->alloc((size_t)max_batch * std::max(F, H));
  for (auto* b : {&Y1, &Y2, &dY2}) b->alloc((size_t)max_batch * H);
  for (auto* b : {&Y3, &T, &dY3}) b->alloc((size_t)max_batch * NM);
  e.alloc(ndof);
  rtmp.alloc(ndof);
  partials.alloc(reduce_partials_count());
  scal.alloc(8);
  counter.alloc(1);
  counter.zero(s);
  HOEFEM_CUDA(cudaMallocHost(&h_scal, 8 * sizeof(double)));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
}

double Learned::features(const double* r, float* Xout, cudaStream_t s) {
  const int ndof = (int)m->ndof;
  (note_launch(), k_norm<<<1, 1024, 0, s>>>(ndof, r, scal.p));
  (note_launch(), k_global_proj<<<dim3(GP_CHUNKS, NG), 256, 0, s>>>(ndof, d_psi.p, r, d_gpart.p));
  (note_launch(), k_global_proj_sum<<<1, 32, 0, s>>>(NG, d_gpart.p, d_gproj.p));
  (note_launch(), k_features<<<S, 256, 0, s>>>(S, d_sub_off.p, d_sub_dofs.p, d_phi.p, r, d_gproj.p, d_centroid.p,
                                               scal.p, Xout));
  HOEFEM_CUDA(cudaGetLastError());
  HOEFEM_CUDA(cudaMemcpyAsync(h_scal, scal.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  return h_scal[0];
}

void Learned::targets(const double* ev, double rnorm, float* Tout, cudaStream_t s) {
  h_scal[1] = rnorm;
  HOEFEM_CUDA(cudaMemcpyAsync(scal.p + 1, h_scal + 1, sizeof(double), cudaMemcpyHostToDevice, s));
  (note_launch(), k_targets<<<S, 256, 0, s>>>(S, d_sub_off.p, d_sub_dofs.p, d_phi.p, ev, scal.p + 1, Tout));
  HOEFEM_CUDA(cudaGetLastError());
}

void Learned::apply(const float* C, double rnorm, double* x0, cudaStream_t s) {
  h_scal[2] = rnorm;
  HOEFEM_CUDA(cudaMemcpyAsync(scal.p + 2, h_scal + 2, sizeof(double), cudaMemcpyHostToDevice, s));
  (note_launch(), k_apply<<<S, 256, 0, s>>>(S, d_sub_off.p, d_sub_dofs.p, d_phi.p, C, scal.p + 2, x0));
  HOEFEM_CUDA(cudaGetLastError());
}

void Learned::add_pair(const double* r, const double* ev, cudaStream_t s) {
  if (n_data + S > cap_data) {
    long long cap = std::max<long long>(2 * cap_data, 32768);
    DBuf<float> nx, nt;
    nx.alloc((size_t)cap * F);
    nt.alloc((size_t)cap * NM);
    if (n_data) {
      HOEFEM_CUDA(cudaMemcpyAsync(nx.p, data_X.p, sizeof(float) * n_data * F, cudaMemcpyDeviceToDevice, s));
      HOEFEM_CUDA(cudaMemcpyAsync(nt.p, data_T.p, sizeof(float) * n_data * NM, cudaMemcpyDeviceToDevice, s));
    }
    HOEFEM_CUDA(cudaStreamSynchronize(s));
    std::swap(nx.p, data_X.p);
    std::swap(nx.n, data_X.n);
    std::swap(nt.p, data_T.p);
    std::swap(nt.n, data_T.n);
    cap_data = cap;
  }
  double rn = features(r, data_X.p + (size_t)n_data * F, s);
  if (!(rn > 0.0)) return;
  targets(ev, rn, data_T.p + (size_t)n_data * NM, s);
  n_data += S;
}

void Learned::forward(const float* Xin, int rows, bool bf16, cudaStream_t s) {
  const float* W1 = params.p;
  const float* b1 = W1 + (size_t)F * H;
  const float* W2 = b1 + H;
  const float* b2 = W2 + (size_t)H * H;
  const float* W3 = b2 + H;
  const float* b3 = W3 + (size_t)H * NM;
  if (!bf16) {
    gemm(rows, H, F, Xin, F, 0, W1, H, 0, Y1.p, H, b1, 1, s);
    gemm(rows, H, H, Y1.p, H, 0, W2, H, 0, Y2.p, H, b2, 1, s);
    gemm(rows, NM, H, Y2.p, H, 0, W3, NM, 0, Y3.p, NM, b3, 0, s);
    return;
  }
  HOEFEM_REQUIRE(rows % 16 == 0, HOEFEM_ERR_INVALID_ARGUMENT, "BF16 inference needs a multiple of 16 rows");
  uint16_t* xb = reinterpret_cast<uint16_t*>(dY1.p);               // rows x F BF16
  uint16_t* y1b = reinterpret_cast<uint16_t*>(dY2.p);              // rows x H BF16
  uint16_t* y2b = reinterpret_cast<uint16_t*>(dY2.p) + (size_t)max_batch * H;  // second half of dY2 (as BF16)
  const uint16_t* W1t = params_bf16.p;
  const uint16_t* W2t = W1t + (size_t)F * H;
  const uint16_t* W3t = W2t + (size_t)H * H;
  (note_launch(), k_f32_to_bf16<<<(rows * F + 255) / 256, 256, 0, s>>>(rows * F, Xin, xb));
  auto tc = [&](int M, int N, int K, const uint16_t* A, const uint16_t* W, const float* bias, int relu, float* Cf,
                uint16_t* Cb) {
    int tiles = (M / 16) * (N / 8);
    (note_launch(), k_gemm_bf16_tc<<<(tiles + 7) / 8, 256, 0, s>>>(M, N, K, A, W, bias, relu, Cf, Cb));
  };
  tc(rows, H, F, xb, W1t, b1, 1, nullptr, y1b);
  tc(rows, H, H, y1b, W2t, b2, 1, nullptr, y2b);
  tc(rows, NM, H, y2b, W3t, b3, 0, Y3.p, nullptr);
  HOEFEM_CUDA(cudaGetLastError());
}

void Learned::refresh_bf16(cudaStream_t s) {
  const float* W1 = params.p;
  const float* W2 = W1 + (size_t)F * H + H;
  const float* W3 = W2 + (size_t)H * H + H;
  uint16_t* o = params_bf16.p;
  (note_launch(), k_f32_to_bf16_t<<<(F * H + 255) / 256, 256, 0, s>>>(F, H, W1, o));
  (note_launch(), k_f32_to_bf16_t<<<(H * H + 255) / 256, 256, 0, s>>>(H, H, W2, o + (size_t)F * H));
  (note_launch(), k_f32_to_bf16_t<<<(H * NM + 255) / 256, 256, 0, s>>>(H, NM, W3, o + (size_t)F * H + (size_t)H * H));
  HOEFEM_CUDA(cudaGetLastError());
}

float Learned::train_step(const float* Xb, const float* Tb, int rows, float lr, cudaStream_t s) {
  float* W1 = params.p;
  float* W2 = W1 + (size_t)F * H + H;
  float* W3 = W2 + (size_t)H * H + H;
  float* gW1 = grads.p;
  float* gb1 = gW1 + (size_t)F * H;
  float* gW2 = gb1 + H;
  float* gb2 = gW2 + (size_t)H * H;
  float* gW3 = gb2 + H;
  float* gb3 = gW3 + (size_t)H * NM;
  forward(Xb, rows, false, s);
  HOEFEM_CUDA(cudaMemsetAsync(scal.p + 3, 0, sizeof(double), s));
  const int no = rows * NM;
  (note_launch(), k_mse_grad<<<std::min((no + 255) / 256, 1024), 256, 0, s>>>(no, 1.f / no, Y3.p, Tb, dY3.p,
                                                                                scal.p + 3));
  // layer 3
  gemm(H, NM, rows, Y2.p, H, 1, dY3.p, NM, 0, gW3, NM, nullptr, 0, s);
  (note_launch(), k_colsum<<<(NM + 127) / 128, 128, 0, s>>>(rows, NM, dY3.p, gb3));
  gemm(rows, H, NM, dY3.p, NM, 0, W3, NM, 1, dY2.p, H, nullptr, 0, s);
  (note_launch(), k_relu_mask<<<(rows * H + 255) / 256, 256, 0, s>>>(rows * H, Y2.p, dY2.p));
  // layer 2
  gemm(H, H, rows, Y1.p, H, 1, dY2.p, H, 0, gW2, H, nullptr, 0, s);
  (note_launch(), k_colsum<<<(H + 127) / 128, 128, 0, s>>>(rows, H, dY2.p, gb2));
  gemm(rows, H, H, dY2.p, H, 0, W2, H, 1, dY1.p, H, nullptr, 0, s);
  (note_launch(), k_relu_mask<<<(rows * H + 255) / 256, 256, 0, s>>>(rows * H, Y1.p, dY1.p));
  // layer 1
  gemm(F, H, rows, Xb, F, 1, dY1.p, H, 0, gW1, H, nullptr, 0, s);
  (note_launch(), k_colsum<<<(H + 127) / 128, 128, 0, s>>>(rows, H, dY1.p, gb1));
  if (lr > 0.f) {
    ++adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f - std::pow(b1, (float)adam_t), c2 = 1.f - std::pow(b2, (float)adam_t);
    (note_launch(), k_adam<<<(int)std::min<size_t>((n_params + 255) / 256, 4096), 256, 0, s>>>(
        (int)n_params, params.p, grads.p, adam_m.p, adam_v.p, lr, b1, b2, 1e-8f, c1, c2));
  }
  HOEFEM_CUDA(cudaGetLastError());
  HOEFEM_CUDA(cudaMemcpyAsync(h_scal + 3, scal.p + 3, sizeof(double), cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  (void)W1;
  return (float)h_scal[3];
}

void Learned::train(long long steps, int batch, float lr, uint64_t seed, float* loss_hist, cudaStream_t s) {
  HOEFEM_REQUIRE(n_data > 0, HOEFEM_ERR_INVALID_ARGUMENT, "no training pairs collected");
  HOEFEM_REQUIRE(batch > 0 && batch <= max_batch, HOEFEM_ERR_INVALID_ARGUMENT, "bad batch size");
  // column statistics of the training set (FP64 sums on the host)
  {
    std::vector<float> hx((size_t)n_data * F), ht((size_t)n_data * NM);
    HOEFEM_CUDA(cudaMemcpyAsync(hx.data(), data_X.p, sizeof(float) * hx.size(), cudaMemcpyDeviceToHost, s));
    HOEFEM_CUDA(cudaMemcpyAsync(ht.data(), data_T.p, sizeof(float) * ht.size(), cudaMemcpyDeviceToHost, s));
    HOEFEM_CUDA(cudaStreamSynchronize(s));
    auto stats = [&](const std::vector<float>& d, int w, DBuf<float>& mean, DBuf<float>& sd) {
      std::vector<double> s1(w, 0.0), s2(w, 0.0);
      for (long long r = 0; r < n_data; ++r)
        for (int c = 0; c < w; ++c) {
          double v = d[(size_t)r * w + c];
          s1[c] += v;
          s2[c] += v * v;
        }
      std::vector<float> mu(w), sg(w);
      double smax = 0.0;
      std::vector<double> sdv(w);
      for (int c = 0; c < w; ++c) {
        double mc = s1[c] / n_data;
        sdv[c] = std::sqrt(std::max(s2[c] / n_data - mc * mc, 0.0));
        smax = std::max(smax, sdv[c]);
        mu[c] = (float)mc;
      }
      for (int c = 0; c < w; ++c) sg[c] = (float)std::max({sdv[c], 1e-6 * smax, 1e-30});
      mean.upload(mu, s);
      sd.upload(sg, s);
    };
    stats(hx, F, x_mean, x_std);
    stats(ht, NM, t_mean, t_std);
  }
  std::mt19937_64 rng(seed);
  std::uniform_int_distribution<long long> pick(0, n_data - 1);
  std::vector<long long> idx(batch);
  DBuf<long long> d_idx;
  d_idx.alloc(batch);
  for (long long k = 0; k < steps; ++k) {
    for (auto& v : idx) v = pick(rng);
    HOEFEM_CUDA(cudaMemcpyAsync(d_idx.p, idx.data(), sizeof(long long) * batch, cudaMemcpyHostToDevice, s));
    (note_launch(), k_gather_rows_std<<<(batch * F + 255) / 256, 256, 0, s>>>(batch, F, d_idx.p, data_X.p, x_mean.p,
                                                                              x_std.p, X.p));
    (note_launch(), k_gather_rows_std<<<(batch * NM + 255) / 256, 256, 0, s>>>(batch, NM, d_idx.p, data_T.p,
                                                                               t_mean.p, t_std.p, T.p));
    float l = train_step(X.p, T.p, batch, lr, s);
    if (loss_hist) loss_hist[k] = l;
  }
  refresh_bf16(s);
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  trained = true;
}

void Learned::predict(const double* r, double* x0, cudaStream_t s) {
  double rn = features(r, X.p, s);
  if (!(rn > 0.0)) {
    HOEFEM_CUDA(cudaMemsetAsync(x0, 0, sizeof(double) * m->ndof, s));
    return;
  }
  (note_launch(), k_standardise<<<(S * F + 255) / 256, 256, 0, s>>>(S, F, x_mean.p, x_std.p, X.p));
  forward(X.p, S, use_bf16 != 0, s);
  (note_launch(), k_unstandardise<<<(S * NM + 255) / 256, 256, 0, s>>>(S, NM, t_mean.p, t_std.p, Y3.p));
  HOEFEM_CUDA(cudaMemsetAsync(x0, 0, sizeof(double) * m->ndof, s));
  apply(Y3.p, rn, x0, s);
}

void Learned::predict_device(const double* r, const double* rr, double* x0, cudaStream_t s) {
  const int ndof = (int)m->ndof;
  (note_launch(), k_sqrt_to<<<1, 1, 0, s>>>(rr, scal.p));
  (note_launch(), k_global_proj<<<dim3(GP_CHUNKS, NG), 256, 0, s>>>(ndof, d_psi.p, r, d_gpart.p));
  (note_launch(), k_global_proj_sum<<<1, 32, 0, s>>>(NG, d_gpart.p, d_gproj.p));
  (note_launch(), k_features<<<S, 256, 0, s>>>(S, d_sub_off.p, d_sub_dofs.p, d_phi.p, r, d_gproj.p, d_centroid.p,
                                               scal.p, X.p));
  (note_launch(), k_standardise<<<(S * F + 255) / 256, 256, 0, s>>>(S, F, x_mean.p, x_std.p, X.p));
  forward(X.p, S, use_bf16 != 0, s);
  (note_launch(), k_unstandardise<<<(S * NM + 255) / 256, 256, 0, s>>>(S, NM, t_mean.p, t_std.p, Y3.p));
  HOEFEM_CUDA(cudaMemsetAsync(x0, 0, sizeof(double) * ndof, s));
  (note_launch(), k_apply<<<S, 256, 0, s>>>(S, d_sub_off.p, d_sub_dofs.p, d_phi.p, Y3.p, scal.p, x0));
  HOEFEM_CUDA(cudaGetLastError());
}

}  // namespace hoefem
