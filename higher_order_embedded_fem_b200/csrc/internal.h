// Internal declarations shared by the libhoefem sources (host + device).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <stdexcept>
#include <string>
#include <vector>

#include "hoefem.h"

namespace hoefem {

using i64 = int64_t;

// Launch accounting: every kernel launch site calls note_launch(); launches
// recorded while a CUDA graph is being captured are counted into the graph
// (capture_count) and added per replay instead.
extern std::atomic<long long> g_launch_count;
extern thread_local long long g_capture_count;  // -1 when not capturing
inline void note_launch() {
  if (g_capture_count >= 0) ++g_capture_count;
  else g_launch_count.fetch_add(1, std::memory_order_relaxed);
}

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define HOEFEM_CUDA(x)                                                                                   \
  do {                                                                                                   \
    cudaError_t e_ = (x);                                                                                \
    if (e_ != cudaSuccess)                                                                               \
      throw ::hoefem::Error(e_ == cudaErrorMemoryAllocation ? HOEFEM_ERR_OUT_OF_MEMORY : HOEFEM_ERR_CUDA, \
                            std::string(#x) + ": " + cudaGetErrorString(e_));                            \
  } while (0)

#define HOEFEM_REQUIRE(cond, code, msg) \
  do {                                  \
    if (!(cond)) throw ::hoefem::Error((code), (msg)); \
  } while (0)

// Device buffer owned by a handle (plain cudaMalloc, freed on destruction).
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    HOEFEM_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) HOEFEM_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), h.size(), s); }
  void zero(cudaStream_t s) {
    if (n) HOEFEM_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
};

// Node-row description of a CSR matrix whose three rows per node share the
// same column structure, with three consecutive columns per neighbour node:
// entry (3a+i, 3b+j) is at base[a] + i * 3 * deg(a) + 3 * slot(b in adj(a)) + j.
// Rows of `diag_only` nodes hold a single diagonal entry each (base[a] + i).
struct NodeRows {
  int nv = 0;
  const long long* base = nullptr;  // row_offsets[3a]
  const int* adj_off = nullptr;     // nv + 1
  const int* adj = nullptr;         // sorted neighbour nodes
  const int* diag_slot = nullptr;   // slot of a in adj(a) (-1 for diag_only nodes)
  const unsigned char* diag_only = nullptr;  // may be null
  int lanes = 32;  // SpMV variant: lanes per node (8, 16, 32), +100 for column streaming; autotuned
  unsigned* sched = nullptr;  // 2 words: node work counter, finished-block counter (dynamic scheduling)
  // optional: the row-node kernels visit only `nodes` (nnodes entries), and
  // the diagonal-only nodes `dnodes` (ndnodes) are applied elementwise
  const int* nodes = nullptr;
  int nnodes = 0;
  const int* dnodes = nullptr;
  int ndnodes = 0;
  __host__ __device__ int count() const { return nodes ? nnodes : nv; }
};

// Per-block device data.
struct BlockDev {
  int kind = 0;     // HOEFEM_ELEM_*
  int nn = 0;       // nodes per element
  int ne = 0;
  const int* conn = nullptr;   // SoA: conn[I * ne + e]
  int uniform = 1;
  int nq = 0;                  // points of the uniform rule
  const int* qoff = nullptr;   // ne + 1 (non-uniform)
  const double* qw = nullptr;
  const double* qp = nullptr;  // xyz interleaved
  const int* emap = nullptr;   // [e * nn * nn + I * nn + J] = nnz index of (3 gI, 3 gJ) - base[gI]
  const double* emat = nullptr;  // optional per-element Lame parameters (mu, lambda) pairs
  // optional (batched scenes): element -> scene and a per-scene flag; elements
  // of scenes whose flag is 0 are skipped by the force / stiffness kernels
  const int* escene = nullptr;
  const unsigned char* scene_active = nullptr;
};

struct Block {
  int kind = 0, nn = 0;
  i64 ne = 0;
  std::vector<i64> conn;  // row-major ne x nn (host)
  bool uniform = true;
  std::vector<i64> qoff;
  std::vector<double> qw, qp;
  std::vector<i64> color_off;   // ncolors + 1
  std::vector<int> color_elems;  // elements ordered by color
  DBuf<int> d_conn, d_qoff, d_emap, d_color_elems;
  DBuf<double> d_qw, d_qp;
  std::vector<double> emat;  // optional per-element (mu, lambda)
  DBuf<double> d_emat;
  std::vector<int> escene;   // optional element -> scene (batched scenes)
  DBuf<int> d_escene;
  const unsigned char* scene_active = nullptr;  // non-owning device mask, per scene
  // tensor-core stiffness (stiffness_tc.cu), built on first use: the reference
  // gradient operator (TF32 hi / lo image), the per-slot gather map and the
  // element blocks
  mutable DBuf<float> d_tc_psi, d_tc_grad, d_tc_ke;
  mutable DBuf<int> d_tc_off, d_tc_ent;
  mutable DBuf<double> d_pb64;  // FP64 node-pair blocks of the staged CUDA-core path
  mutable DBuf<double> d_fst;   // staged element node forces
  mutable DBuf<int> d_noff, d_nent;  // per node: its (element, local node) incidences
  mutable int tc_nch = 0;
  mutable bool tc_ready = false, gmap_ready = false, nmap_ready = false;
  BlockDev dev() const;
};

// Element stiffness / force implementation: automatic (tensor cores for the
// blocks they cover: Tet10 with one quadrature rule of at most 14 points,
// FP32 element arithmetic; staged whole-block CUDA-core kernels for the
// rest), staged CUDA-core kernels only, or the colored scatter kernels.
enum StiffnessPath { STIFFNESS_AUTO = 0, STIFFNESS_CUDA_CORES = 1, STIFFNESS_STAGED = 2 };

struct Model {
  int device = 0;
  cudaStream_t stream = nullptr;
  i64 nv = 0;
  std::vector<double> X;
  std::vector<Block*> blocks;
  bool finalized = false;
  bool on_device = false;
  i64 ndof = 0, nnz = 0, num_elements = 0;
  // node structure of the shared pattern (host)
  std::vector<int> adj_off, adj, diag_slot;
  std::vector<long long> base;
  // device
  DBuf<double> d_X;
  DBuf<int> d_adj_off, d_adj, d_diag_slot, d_err;
  DBuf<unsigned> d_sched;  // SpMV dynamic-scheduling counters (zero between launches)
  DBuf<double> d_stage;    // dense element matrices (projected stiffness), allocated on first use
  DBuf<long long> d_base;
  int spmv_lanes = 32;    // SpMV variant for FP64 values (autotuned)
  int spmv_lanes32 = 0;   // SpMV variant for FP32 values (0: as spmv_lanes)
  bool spmv_pinned = false;  // set explicitly by the caller: no autotuning
  int stiffness_path = STIFFNESS_AUTO;
  NodeRows rows() const;
  ~Model();
};

struct MatDev {
  int kind;
  double mu, lambda;
};

// ---- element kernels (elements.cu) -----------------------------------------
void launch_forces(const Model& m, const MatDev& mat, const double* u, double* f, cudaStream_t s);
enum Precision { PRECISION_FP64 = 0, PRECISION_FP32 = 1 };
// Element stiffness with the element arithmetic in FP64 or FP32; the CSR
// values are accumulated in FP64 either way.  Adds into vals, or with assign
// stores K(u) (a single tensor-core block writes every entry; otherwise vals
// is cleared first).
void launch_stiffness(const Model& m, const MatDev& mat, const double* u, double* vals, cudaStream_t s,
                      int precision = PRECISION_FP64, bool assign = false);
void launch_mass(const Model& m, double density, double* vals, cudaStream_t s);
// Tensor-core Tet10 stiffness (stiffness_tc.cu): eligibility of a block for
// FP32 element arithmetic, and the launch (element blocks on the tensor
// cores, then the gather into vals, adding).
bool stiffness_tc_eligible(const Model& m, const Block& blk);
void launch_stiffness_tc(const Model& m, const Block& blk, const MatDev& mat, const double* u, double* vals,
                         cudaStream_t s, bool assign = false);
// CUDA-core element stiffness of a whole block in one launch into staged
// node-pair blocks, then the same gather (not for batched scenes): the
// block's pair buffer (FP32 or FP64 blocks), and the gather into vals.
bool stiffness_pairs_eligible(const Model& m, const Block& blk);
void* stiffness_pair_buffer(const Model& m, const Block& blk, bool f32, cudaStream_t s);
void stiffness_gather_pairs(const Model& m, const Block& blk, bool f32, double* vals, bool assign, cudaStream_t s);
// Staged element forces of a whole block (same eligibility): the buffer
// (element-major node forces) and the per-node gather adding into f.
double* forces_stage_buffer(const Model& m, const Block& blk, cudaStream_t s);
void forces_gather(const Model& m, const Block& blk, double* f, cudaStream_t s);
// Stiffness with every element matrix projected onto PSD (negative eigenvalues
// set to zero) before the colored scatter; adds into vals.
void launch_stiffness_projected(Model& m, const MatDev& mat, const double* u, double* vals, cudaStream_t s);

// ---- sparse / vector kernels (linalg.cu) -----------------------------------
// y = beta*y + alpha*A x on a node-row matrix.
void spmv_node_rows(const NodeRows& A, const double* vals, const double* x, double* y, double alpha, double beta,
                    cudaStream_t s);
// Times the lanes-per-node variants of the node-row SpMV on this structure
// and returns the fastest (8, 16 or 32); best_ms (optional) gets its time.
int autotune_spmv_lanes(NodeRows A, const double* vals, cudaStream_t s, float* best_ms = nullptr);
// Fills out = c_k * K + c_d * D + c_m * M (any may be null; summed in that
// order) and applies homogeneous Dirichlet rows / columns for the dof mask
// (may be null).
void jacobian_combination(const Model& m, double ck, const double* K, double cm, const double* M,
                          const unsigned char* bc_dof, double* out, double* d_scratch, cudaStream_t s,
                          double cd = 0.0, const double* D = nullptr);
// Deterministic reductions: result written to *out (device).
void dot_device(const double* a, const double* b, i64 n, double* out, double* partials, unsigned* counter,
                cudaStream_t s);
int reduce_blocks_for(i64 n);
// Multiprocessor count of the current device, and the size of a partials
// buffer that holds every deterministic grid reduction's block partials.
int device_sms();
size_t reduce_partials_count();

void finalize_model(Model& m);
void ensure_device(Model& m);
void export_pattern(const std::vector<int>& adj_off, const std::vector<int>& adj, const std::vector<long long>& base,
                    const std::vector<unsigned char>* diag_only, i64 nv, int64_t* ro, int64_t* ci);

// ---- errors ----------------------------------------------------------------
void check_device_error(const Model& m);  // reads and clears d_err

}  // namespace hoefem
