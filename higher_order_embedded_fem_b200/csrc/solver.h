// Preconditioner and CG declarations (internal).
#pragma once

#include <functional>

#include "internal.h"

namespace hoefem {

enum PrecondKind { PREC_NONE = 0, PREC_DIAGONAL = 1, PREC_SCHWARZ = 2 };

struct Precond {
  int kind = PREC_DIAGONAL;
  Model* m = nullptr;
  bool ready = false;
  DBuf<double> diag;  // inverse diagonal (DIAGONAL) or scratch
  // ---- Schwarz ----
  i64 nsub = 0;
  int max_nodes = 0;
  std::vector<i64> sub_off, sub_nodes, untreated;
  std::vector<i64> color_off;
  std::vector<int> color_subs;
  std::vector<int> adj_off, adj, diag_slot;
  std::vector<long long> base;
  std::vector<unsigned char> diag_only;
  DBuf<int> d_adj_off, d_adj, d_diag_slot, d_sub_off, d_sub_nodes, d_gmap, d_smap, d_color_subs, d_untreated;
  DBuf<long long> d_base, d_gmap_off;
  DBuf<unsigned char> d_diag_only;
  DBuf<double> vals, staging;
  DBuf<float> vals32;  // FP32 copy of the Schwarz values (mixed-precision apply)
  bool want_fp32 = false;
  DBuf<long long> d_stage_off;
  DBuf<int> d_err;
  DBuf<int> d_fallback;
  DBuf<unsigned> d_sched;  // SpMV dynamic-scheduling counters of the Schwarz pattern  // [0]: count, [1..]: subdomains for the eigen path
  i64 nnz = 0;
  int spmv_lanes = 32;   // SpMV variant of the Schwarz apply, FP64 values
  int spmv_lanes32 = 0;  // FP32 values (0: as spmv_lanes)
  bool spmv_pinned = false;  // set explicitly by the caller: no autotuning
  DBuf<int> d_tnodes;      // nodes with subdomain rows (the rest are untreated, diagonal only)
  i64 tnodes_count = 0;
  // Block apply (CG): the symmetrized inverted subdomain blocks (staging
  // layout) applied as dense products into ysub (3 entries per subdomain
  // node), then summed per node over its subdomains in subdomain order.
  bool block_apply = true;
  DBuf<double> bsym;
  DBuf<float> bsym32;
  DBuf<double> ysub;
  DBuf<int> d_npair_off;  // nv + 1: a node's slots in ysub (3 entries each)
  DBuf<int> d_npair;      // slot of every (subdomain, node) incidence (sub_nodes order)
  NodeRows rows() const;
};

void precond_create_schwarz(Precond& p, const i64* sub_off, const i64* sub_nodes, i64 nsub, const i64* untreated,
                            i64 nun);
void precond_update(Precond& p, const double* system_vals, cudaStream_t s);
void precond_apply(const Precond& p, const double* r, double* z, cudaStream_t s);
void precond_to_fp32(Precond& p, cudaStream_t s);

struct CgState {
  double bnorm, tol, zTr, pAp, rr, alpha, beta;
  long long iters, max_iter;
  int done, status;
};

struct CgWork {
  Model* m = nullptr;
  i64 n = 0;
  DBuf<double> x, b, r, z, p, Ap, partials;
  DBuf<CgState> st;
  DBuf<unsigned> counter;
  CgState* h_st = nullptr;  // pinned
  struct Graph {
    const void* key[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;
  };
  std::vector<Graph> graphs;  // chunk graphs per (operator, preconditioner, precision, SpMV variants)
  // Online choice of the SpMV variants (operator x Schwarz apply) per value
  // precision: the first chunks of the first solves run one candidate pair
  // each and are timed; the fastest pair is kept.
  struct Tuning {
    int next = 0;  // candidate index to measure next
    bool done = false;
    float best_ms = 1e30f;
    int best = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
  };
  Tuning tuning[2];  // [0] FP64 values, [1] FP32 values
  bool online_tuning = true;
  int chunk = 8;
  // called on the host after every chunk of iterations (solver state synced)
  std::function<void(cudaStream_t)> on_chunk;
  void init(Model* model);
  ~CgWork();
};

// Solves A x = b with x = work.x (initial guess) and b = work.b on the model
// pattern values `vals`.  Returns HOEFEM_OK or a HOEFEM_CG_* status.
int cg_solve(CgWork& w, const double* vals, const Precond* P, double tol, i64 max_iter, i64* iters, cudaStream_t s);
// FP64 iterative refinement around an FP32-operator / FP32-preconditioner PCG.
int cg_solve_reliable(CgWork& w, const double* A64, const float* A32, const Precond* P, double tol, i64 max_iter,
                      double delta, i64* iters, i64* replacements, cudaStream_t s);
void to_f32(const double* a, float* b, long long n, cudaStream_t s);

}  // namespace hoefem
