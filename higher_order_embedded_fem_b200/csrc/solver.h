// Preconditioner and CG declarations (internal).
#pragma once

#include <functional>
#include <vector>

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
  // With the block apply the CG reads the symmetrized blocks and, from the
  // assembled values, only the untreated (diagonal-only) entries, which every
  // update writes; the subdomain entries are scattered into the values when
  // something reads them (precond_assemble).
  mutable bool vals_complete = false;
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
// Completes the assembled values (subdomain entries) if an update left them
// out; before any read of P's CSR values.
void precond_assemble(const Precond& p, cudaStream_t s);
void precond_apply(const Precond& p, const double* r, double* z, cudaStream_t s);
void precond_to_fp32(Precond& p, cudaStream_t s);

struct CgState {
  double bnorm, tol, zTr, pAp, rr, alpha, beta;
  long long iters, max_iter;
  int done, status;
  // streamed CG: residual-replacement trigger (rr <= delta2 * rr_ref), the
  // flag it raises, and which direction buffer holds the current direction
  double rr_ref, delta2;
  int replace, pcur, rcur, pad;
  // flexible CG with the learned coarse correction: z_k.r_k of the previous
  // iteration, whether this iteration's correction was kept, and the counts
  double zr_old, learned_weight;
  long long learned_kept, learned_dropped;
  int learned_flag, pad2;
};

// One unit of a streamed kernel's work: `bytes` (multiple of 16, at most one
// ring stage) at byte offset `off` of a stream buffer, plus kind-specific
// fields (operator tile: a = first node, b = nodes; Schwarz chunk:
// a = subdomain, b = first row, c = rows) and keep = 1 for items whose copy
// asks L2 to keep the lines (evict last) rather than stream them.
struct CgsItem {
  long long off;
  int bytes, a, b, c;
  int keep, pad;
};

// A run of a CTA's own nodes [n0, n1) that share one staged halo (`halo_n`
// nodes listed from `halo_off` of the halo array, sorted; the own nodes are
// halo entries own_lo ..): its operator tiles are the CTA's items [j0, j1),
// its Schwarz row items the CTA's Schwarz items [sj0, sj1), covering the
// subdomain incidences (node-major slots) [q0, q1) of its nodes.
struct CgsSeg {
  int j0, j1;
  int halo_off, halo_n;
  int n0, n1;
  int sj0, sj1;
  int q0, q1;
  int own_lo, pad;
};

// Stream layouts of the persistent CG (cg_stream.cu): the operator as tiles
// of whole node rows (header, 16-bit halo-local neighbour indices, 9 value
// planes per node) and the Schwarz blocks as row chunks, each split into
// contiguous per-CTA item ranges balanced by bytes and into halo segments.
struct CgStreamOp {
  int vsize = 0;  // value bytes (8 FP64, 4 FP32); 0 = not built
  int grid = 0;
  DBuf<unsigned char> data;
  DBuf<CgsItem> items;
  DBuf<int> item_off;    // grid + 1
  DBuf<int> node_range;  // grid + 1
  DBuf<long long> val_off;  // per node: byte offset of its value planes
  DBuf<CgsSeg> segs;
  DBuf<int> seg_off;  // grid + 1
  DBuf<int> halo;     // halo node lists of the segments
  long long bytes = 0;      // streamed bytes per apply
  std::vector<CgsItem> h_items;  // host copies (L2 keep flags)
  std::vector<int> h_item_off;
  std::vector<CgsSeg> h_segs;  // host copies (the Schwarz layout follows the segments)
  std::vector<int> h_seg_off, h_halo;
  long long keep_applied = -1;
  const void* seg_for = nullptr;  // the preconditioner whose incidences bound the segments
};
// Schwarz blocks distributed by rows: every subdomain incidence (subdomain
// s, its local node I; node-major slot order) is a record of the block's rows
// 3I .. 3I + 2 plus the halo-local indices of the subdomain's nodes, stored
// with the operator segment that owns the node.
struct CgStreamSchwarz {
  int vsize = 0;  // 8, 4 or 2 (FP16 with a per-subdomain scale)
  int grid = 0;
  const void* built_for = nullptr;
  const void* op_for = nullptr;  // the operator layout whose segments it follows
  DBuf<unsigned char> data;
  DBuf<CgsItem> items;
  DBuf<int> item_off;
  DBuf<long long> rec_val_off;  // per slot: byte offset of its 3 rows
  DBuf<int> slot_sub;           // per slot: subdomain
  DBuf<int> slot_local;         // per slot: local node index in the subdomain
  DBuf<double> scale;           // per subdomain (FP16 only)
  long long bytes = 0;
  std::vector<CgsItem> h_items;
  std::vector<int> h_item_off;
  long long keep_applied = -1;
};

struct CgWork {
  Model* m = nullptr;
  i64 n = 0;
  DBuf<double> x, b, r, z, p, Ap, partials;
  // FP32 copy of the search direction (one 16-byte entry per node) for the
  // FP32 operator products of the mixed form's chunked engine
  DBuf<float4> p32;
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
  // Persistent streamed CG (cg_stream.cu): mode 0 automatic (used whenever
  // the device, the preconditioner and the layouts allow), 1 off (graphs of
  // kernel chunks), 2 required (error if it cannot run); schwarz_half stores
  // the mixed-precision Schwarz blocks in FP16 with a per-subdomain scale.
  int stream_mode = 0;
  bool schwarz_half = false;
  // automatic engine choice per (operator precision, preconditioner kind):
  // the first solves with at least 20 iterations are timed on the chunked
  // engine (once its SpMV variants are tuned), then on the streamed one; the
  // faster per-iteration time decides for the later solves
  // automatic engine choice: models with fewer nodes use the chunked engine
  static constexpr int STREAM_MIN_NODES = 32768;
  struct EngineTune {
    int phase = 0;  // 0 / 1: chunked set-up / timed solve, 2 / 3: streamed set-up / timed, 4: decided
    double us_per_it[2] = {0.0, 0.0};
    int choice = -1;  // 0 chunked, 1 streamed
  };
  EngineTune etune[6];
  int last_tune = 0;  // entry of the last solve
  cudaEvent_t tev[2] = {nullptr, nullptr};
  // flexible CG with the learned correction: r_k, its graph and what it was captured for
  DBuf<double> r_old;
  cudaGraphExec_t fcg_exec = nullptr;
  const void* fcg_key[3] = {nullptr, nullptr, nullptr};
  long long fcg_kernels = 0;
  CgStreamOp sop64, sop32;
  CgStreamSchwarz ssw;
  DBuf<double> p2, r2, spart;
  DBuf<unsigned> sbar;
  DBuf<int> serr;
  long long stream_launches = 0, stream_iterations = 0;
  float stream_ms = 0.f;         // device time of the persistent launches (last solve)
  double stream_ms_total = 0.0;  // summed over solves until reset by the caller
  bool last_f32 = false;         // precision of the last streamed solve
  bool phase_profile = false;    // per-phase cycle counters in the streamed CG
  // L2 residency budget of the streamed CG (bytes over all CTAs; -1: default,
  // a share of the device's L2): that many bytes of each iteration's stream,
  // the Schwarz chunks first, are copied with an evict-last policy so that
  // they are still in L2 in the next iteration, the rest evict-first
  long long l2_keep = -1;
  long long l2_keep_applied = -2;
  DBuf<unsigned long long> sprof;  // grid x 16 counters (cycles), summed over launches
  double sclock_khz = 0.0;
  cudaEvent_t sev[2] = {nullptr, nullptr};
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

struct Learned;
// Flexible PCG (FP64) with the two-level preconditioner z = P r + c(r), c the
// learned coarse correction of the current residual, kept in an iteration
// only if c.r > 0; beta = z_{k+1}.(r_{k+1} - r_k) / z_k.r_k.  kept / dropped
// count the iterations with and without the correction.
int cg_solve_learned(CgWork& w, const double* vals, const Precond* P, Learned* L, double tol, i64 max_iter,
                     i64* iters, i64* kept, i64* dropped, cudaStream_t s);

// Streamed CG (cg_stream.cu).  cg_stream_usable: whether the persistent
// kernel can run this solve; cg_stream_prepare packs the operator (FP64
// values, converted to the stream precision) and the Schwarz blocks into
// their stream layouts; cg_stream_iterate runs iterations from the current
// state (x, r, z, zTr in w; direction = z + beta * w.p) until convergence,
// an error outcome, the iteration limit or a residual-replacement trigger,
// and leaves the current direction in w.p.
bool cg_stream_usable(CgWork& w, const Precond* P);
// (false: the layouts do not fit the kernel's stages or halos)
bool cg_stream_prepare(CgWork& w, const double* A64, bool f32, const Precond* P, bool p32, cudaStream_t s);
void cg_stream_iterate(CgWork& w, bool f32, const Precond* P, bool p32, bool reliable, cudaStream_t s);
// Per-phase microseconds per iteration of the streamed CG since the last
// reset (zeros without HOEFEM_CG_PHASE_PROFILE); resets the counters.
void cg_stream_phase_us(CgWork& w, double* out12, double* max12, double* busy2);
// Sets the residual-replacement reference rr_ref = rr (current state) and
// delta^2, clears the replacement flag.
void cg_stream_arm(CgWork& w, double delta, cudaStream_t s);

}  // namespace hoefem
