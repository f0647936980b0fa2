// Stiffness with element-wise projection onto positive semidefiniteness, the
// matrix of stiffness-proportional damping.
//
// Reference: DefaultSemidefiniteProjection (fenris/src/assembly.rs:549-564)
// inside compute_stiffness_matrix_into(projected = true) /
// compute_damping_matrix_into (simulation_toolbox/src/fem/system_assembly.rs:
// 107-193): every element matrix is eigen-decomposed, its negative
// eigenvalues are set to zero, and the recomposed matrix is assembled.
//
// Three passes per block:
//  1. k_stiffness in staging mode: the dense FP64 element matrices of all
//     elements (one launch, no coloring needed);
//  2. k_psd_project: one CTA per element, parallel cyclic Jacobi in shared
//     memory, V max(L, 0) V^T written back in place;
//  3. k_stage_scatter: per element color, the staged matrices are added into
//     the CSR values through the element-to-nnz map (no atomics; every entry
//     receives its contributions in color order, as the reference).
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "jacobi.cuh"
#include "kernels_common.cuh"

namespace hoefem {

void launch_stiffness_staged(const Model& m, const Block& blk, const MatDev& mat, const double* u, double* stage,
                             cudaStream_t s);

namespace {

constexpr int PSD_TPB = 256;

__global__ void __launch_bounds__(PSD_TPB) k_psd_project(int dim, double* __restrict__ stage) {
  extern __shared__ double smem[];
  const int m = (dim + 1) & ~1;
  double* A = smem;
  double* V = A + m * m;
  double* cs = V + m * m;
  double* sn = cs + m / 2;
  __shared__ double s_red[2];
  double* ke = stage + (size_t)blockIdx.x * dim * dim;
  for (int k = threadIdx.x; k < m * m; k += blockDim.x) {
    const int r = k / m, c = k % m;
    A[k] = (r < dim && c < dim) ? ke[r * dim + c] : 0.0;
    V[k] = (r == c) ? 1.0 : 0.0;
  }
  __syncthreads();
  jacobi_eigen_block(A, V, cs, sn, m, dim, s_red);
  // eigenvalues max(lambda, 0) on the diagonal of A
  for (int k = threadIdx.x; k < dim; k += blockDim.x) A[k * m + k] = fmax(A[k * m + k], 0.0);
  __syncthreads();
  for (int k = threadIdx.x; k < dim * dim; k += blockDim.x) {
    const int i = k / dim, j = k % dim;
    double s = 0.0;
    for (int t = 0; t < dim; ++t) s += V[i * m + t] * A[t * m + t] * V[j * m + t];
    ke[k] = s;
  }
}

// Adds the staged element matrices of one color into the CSR values.
template <int NN>
__global__ void __launch_bounds__(256) k_stage_scatter(const BlockDev b, const int* __restrict__ elems, int count,
                                                       const int* __restrict__ adj_off,
                                                       const long long* __restrict__ base,
                                                       const double* __restrict__ stage, double* __restrict__ vals) {
  constexpr int D = 3 * NN;
  const int idx = blockIdx.x;
  if (idx >= count) return;
  const int e = elems[idx];
  const double* ke = stage + (size_t)e * D * D;
  const int* em = b.emap + (size_t)e * NN * NN;
  for (int k = threadIdx.x; k < D * D; k += blockDim.x) {
    const int r = k / D, c = k % D;
    const int I = r / 3, i = r - 3 * I, Jn = c / 3, j = c - 3 * Jn;
    const int gI = b.conn[I * b.ne + e];
    const int rl = 3 * (adj_off[gI + 1] - adj_off[gI]);
    vals[base[gI] + em[I * NN + Jn] + (long long)i * rl + j] += ke[k];
  }
}

}  // namespace

// Stiffness at u with every element matrix projected onto PSD, added into vals.
void launch_stiffness_projected(Model& m, const MatDev& mat, const double* u, double* vals, cudaStream_t s) {
  size_t need = 0;
  for (const Block* bp : m.blocks) need = std::max(need, (size_t)bp->ne * 9 * bp->nn * bp->nn);
  if (m.d_stage.n < need) m.d_stage.alloc(need);
  for (const Block* bp : m.blocks) {
    if (bp->ne == 0) continue;
    const int dim = 3 * bp->nn;
    const int mm = (dim + 1) & ~1;
    const size_t smem = sizeof(double) * (2 * (size_t)mm * mm + mm);
    launch_stiffness_staged(m, *bp, mat, u, m.d_stage.p, s);
    HOEFEM_CUDA(cudaFuncSetAttribute(k_psd_project, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    (note_launch(), k_psd_project<<<(int)bp->ne, PSD_TPB, smem, s>>>(dim, m.d_stage.p));
    BlockDev bd = bp->dev();
    const int nc = (int)bp->color_off.size() - 1;
    for (int c = 0; c < nc; ++c) {
      const int b0 = (int)bp->color_off[c], cnt = (int)(bp->color_off[c + 1] - b0);
      if (cnt <= 0) continue;
      if (bp->kind == HOEFEM_ELEM_TET10)
        (note_launch(), k_stage_scatter<10><<<cnt, 256, 0, s>>>(bd, bp->d_color_elems.p + b0, cnt, m.d_adj_off.p,
                                                                m.d_base.p, m.d_stage.p, vals));
      else
        (note_launch(), k_stage_scatter<27><<<cnt, 256, 0, s>>>(bd, bp->d_color_elems.p + b0, cnt, m.d_adj_off.p,
                                                                m.d_base.p, m.d_stage.p, vals));
    }
  }
  HOEFEM_CUDA(cudaGetLastError());
}

}  // namespace hoefem
