// Newton-CG backward Euler integrator.
//
// Reference: NewtonCgIntegrator3d / integrate_model_with_substeps /
// integrate_model / NewtonCgDynamicSystem (simulation_toolbox/src/fem/
// newton_cg.rs:43-295,413-802), backward_euler_step +
// BackwardEulerImplicitFunction (hamilton2/src/integrators/euler.rs:76-199),
// newton_line_search + BacktrackingLineSearch (hamilton2/src/newton.rs:
// 76-248), system_assembly.rs:30-235, fe_model.rs:423-431,489-515.
//
// The control flow (Newton iterations, line-search trials, substep retries)
// stays on the host, as in the reference; every vector / matrix operation is
// a device kernel on the model's stream.  Host round trips per Newton
// iteration: one norm per residual evaluation and one state read per CG chunk.
#include <cuda_runtime.h>

#include <cmath>
#include <memory>

#include "internal.h"
#include "kernels_common.cuh"
#include "solver.h"
#include "learned.h"

namespace hoefem {

namespace {

constexpr int TPB = 256;

__global__ void k_be_init(int n, const double* __restrict__ u, const double* __restrict__ v, double dt,
                          double* __restrict__ up, double* __restrict__ vn, double* __restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    vn[i] = v[i];
    up[i] = u[i] + v[i] * dt;
    w[i] = 0.0;
  }
}

// u = u_p + dt w, v = v_n + w, Dirichlet values (homogeneous) applied.
__global__ void k_be_state(int n, const double* __restrict__ up, const double* __restrict__ vn,
                           const double* __restrict__ w, double dt, const unsigned char* __restrict__ bc,
                           double* __restrict__ us, double* __restrict__ vs) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double uu = up[i] + w[i] * dt, vv = vn[i] + w[i];
    if (bc && bc[i]) { uu = 0.0; vv = 0.0; }
    us[i] = uu;
    vs[i] = vv;
  }
}

__global__ void k_copy(int n, const double* __restrict__ a, double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// F = -dt * f with Dirichlet rows of f zeroed first (eval_f + eval_into)
__global__ void k_F(int n, const double* __restrict__ f, const unsigned char* __restrict__ bc, double dt,
                    double* __restrict__ F) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double fi = (bc && bc[i]) ? 0.0 : f[i];
    F[i] = fi * (dt * -1.0);
  }
}

__global__ void k_zero_bc(int n, const unsigned char* __restrict__ bc, double* __restrict__ f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (bc[i]) f[i] = 0.0;
}

__global__ void k_axpy_w(int n, double da, const double* __restrict__ dx, double* __restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] = da * dx[i] + 1.0 * w[i];
}

// y = a y + b  (in place on y)
__global__ void k_axpby(int n, double a, double* __restrict__ y, const double* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a * y[i] + b[i];
}

__global__ void k_scale(int n, double a, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] *= a;
}

// Learned warm start on the device (w: [0] F.F, [1] d.J d, [2] d.F, [3] r0.r0,
// [4] accepted, [5] rejected, [6] sum of sqrt(r0.r0 / F.F), [7] alpha).
__global__ void k_warm_alpha(double* w) {
  const double dJd = w[1], db = w[2];
  w[7] = (dJd > 0.0 && db > 0.0) ? db / dJd : 0.0;
}
// r0 = F - alpha J d (r0 holds J d on entry)
__global__ void k_warm_residual(int n, const double* __restrict__ w, double* __restrict__ r0,
                                const double* __restrict__ F) {
  const double a = w[7];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) r0[i] = -a * r0[i] + F[i];
}
// x = alpha d if alpha > 0 and ||r0|| < ||F|| (x is zero on entry); counters
__global__ void k_warm_accept(int n, double* __restrict__ w, const double* __restrict__ d, double* __restrict__ x) {
  const double a = w[7], rr = w[3], bb = w[0];
  const bool keep = a > 0.0 && rr < bb;
  if (keep)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = a * d[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (keep) {
      w[4] += 1.0;
      w[6] += sqrt(rr / bb);
    } else {
      w[5] += 1.0;
    }
  }
}

__global__ void k_neg(int n, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] *= -1.0;
}

__global__ void k_be_final(int n, const double* __restrict__ w, double dt, const unsigned char* __restrict__ bc,
                           double* __restrict__ u, double* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double vv = v[i] + w[i];
    double uu = u[i] + vv * dt;
    if (bc && bc[i]) { uu = 0.0; vv = 0.0; }
    v[i] = vv;
    u[i] = uu;
  }
}

__global__ void k_bc_uv(int n, const unsigned char* __restrict__ bc, double* __restrict__ u, double* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (bc[i]) { u[i] = 0.0; v[i] = 0.0; }
}

__global__ void k_fill(int n, double v, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

__global__ void k_gravity_density(int n, double g, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = (i % 3 == 2) ? g : 0.0;
}

}  // namespace

struct Integrator {
  Model* m = nullptr;
  MatDev mat{};
  double density = 1000.0;
  std::vector<i64> bc_nodes;
  bool gravity_enabled = true;
  double gravity = -9.81;
  Precond* P = nullptr;
  std::unique_ptr<Precond> own;
  double cg_tol = 1e-5;
  i64 cg_max = 500, newton_max = 100;
  int precision = PRECISION_FP64;  // PRECISION_FP32: mixed (FP32 element stiffness, FP32 operator / Schwarz apply
                                   // inside FP64 iterative refinement)
  double delta = 0.1;  // reliable-update threshold of the mixed CG
  DBuf<float> J32;
  Learned* learned = nullptr;
  int learned_mode = 0;  // 0 off, 1 warm start, 2 collect (b, x*), 3 collect (b, x*) and CG iterates,
                         // 4 two-level preconditioner (flexible CG, FP64)
  DBuf<double> x0, r0, lw;
  cudaEvent_t lev[2] = {nullptr, nullptr};
  bool lev_pending = false;
  // the warm start's kernels as one CUDA graph (captured per learned model)
  cudaGraphExec_t ws_exec = nullptr;
  const void* ws_key = nullptr;
  long long ws_kernels = 0;
  std::vector<DBuf<double>*> snaps;  // collected (x_k, r_k) pairs of the current solve
  double rep_force = 0.0;
  // damping D = gamma M + alpha K_proj(u) from the (sub)step's initial state
  // (compute_damping_matrix_into, system_assembly.rs:145-193)
  bool has_mass_damping = false, has_stiffness_damping = false, has_damping = false;
  double mass_damping = 0.0, stiffness_damping = 0.0;
  DBuf<double> D;
  DBuf<unsigned char> bc;
  DBuf<double> M, K, J, gforce, up, vn, w, F, dx, us, vs, f, u, v, partials, scalars;
  DBuf<unsigned> counter;
  double* h_scalar = nullptr;
  CgWork cg;
  hoefem_step_stats stats{};
  i64 stats_replacements = 0;
  cudaEvent_t ev[2] = {nullptr, nullptr};

  ~Integrator() {
    if (h_scalar) cudaFreeHost(h_scalar);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (auto& e : lev)
      if (e) cudaEventDestroy(e);
    if (ws_exec) cudaGraphExecDestroy(ws_exec);
  }

  int grid() const { return reduce_blocks_for(m->ndof); }

  double norm_sq(const double* a) { return dot(a, a); }

  double dot(const double* a, const double* b) {
    dot_device(a, b, m->ndof, scalars.p, partials.p, counter.p, m->stream);
    HOEFEM_CUDA(cudaMemcpyAsync(h_scalar, scalars.p, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    HOEFEM_CUDA(cudaStreamSynchronize(m->stream));
    return *h_scalar;
  }

  void setup() {
    cudaStream_t s = m->stream;
    const int n = (int)m->ndof;
    bc.alloc(n);
    std::vector<unsigned char> hb(n, 0);
    for (i64 a : bc_nodes) {
      HOEFEM_REQUIRE(a >= 0 && a < m->nv, HOEFEM_ERR_INVALID_ARGUMENT, "boundary node out of range");
      for (int i = 0; i < 3; ++i) hb[3 * a + i] = 1;
    }
    HOEFEM_CUDA(cudaMemcpyAsync(bc.p, hb.data(), n, cudaMemcpyHostToDevice, s));
    for (auto* b : {&M, &K, &J}) b->alloc(m->nnz);
    for (auto* b : {&gforce, &up, &vn, &w, &F, &dx, &us, &vs, &f, &u, &v}) b->alloc(n);
    partials.alloc(reduce_partials_count());
    scalars.alloc(8);
    counter.alloc(1);
    counter.zero(s);
    HOEFEM_CUDA(cudaMallocHost(&h_scalar, 8 * sizeof(double)));
    for (auto& e : ev) HOEFEM_CUDA(cudaEventCreate(&e));
    cg.init(m);
    // mass matrix with Dirichlet (fe_model.rs:489-515)
    K.zero(s);
    launch_mass(*m, density, K.p, s);
    jacobian_combination(*m, 0.0, nullptr, 1.0, K.p, bc_nodes.empty() ? nullptr : bc.p, M.p, scalars.p, s);
    check_device_error(*m);
    if (!m->spmv_pinned) m->spmv_lanes = autotune_spmv_lanes(m->rows(), M.p, s);
    // representative force ||M a||, a_i = sqrt(a^2 / 3), a = 10 (fe_model.rs:423-431)
    (note_launch(), k_fill<<<grid(), TPB, 0, s>>>(n, std::sqrt((10.0 * 10.0) / 3.0), us.p));
    spmv_node_rows(m->rows(), M.p, us.p, vs.p, 1.0, 0.0, s);
    rep_force = std::sqrt(norm_sq(vs.p));
    // gravity force M g (system_assembly.rs:30-75, newton_cg.rs:248-255)
    if (gravity_enabled) (note_launch(), k_gravity_density<<<grid(), TPB, 0, s>>>(n, gravity, us.p));
    else (note_launch(), k_fill<<<grid(), TPB, 0, s>>>(n, 0.0, us.p));
    spmv_node_rows(m->rows(), M.p, us.p, gforce.p, 1.0, 0.0, s);
    HOEFEM_CUDA(cudaStreamSynchronize(s));
    if (!P) {
      own.reset(new Precond());
      own->kind = PREC_DIAGONAL;
      own->m = m;
      P = own.get();
    }
  }

  float elapsed() {
    float ms = 0.f;
    HOEFEM_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    return ms;
  }

  // f = M g + f_int(u) with Dirichlet rows zeroed (eval_f, newton_cg.rs:441-478)
  void eval_f(const double* ud, const double* vd, double* out) {
    cudaStream_t s = m->stream;
    const int n = (int)m->ndof;
    (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, ud, us.p));
    (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, vd, vs.p));
    if (!bc_nodes.empty()) (note_launch(), k_bc_uv<<<grid(), TPB, 0, s>>>(n, bc.p, us.p, vs.p));
    (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, gforce.p, out));
    launch_forces(*m, mat, us.p, out, s);
    if (has_damping) spmv_node_rows(m->rows(), D.p, vs.p, out, -1.0, 1.0, s);  // f += -D v
    if (!bc_nodes.empty()) (note_launch(), k_zero_bc<<<grid(), TPB, 0, s>>>(n, bc.p, out));
    check_device_error(*m);
  }

  // F(w) = M w - dt f(t + dt, u_p + dt w, v_n + w); returns ||F||^2
  double eval_F(double dt) {
    cudaStream_t s = m->stream;
    const int n = (int)m->ndof;
    const unsigned char* bcp = bc_nodes.empty() ? nullptr : bc.p;
    HOEFEM_CUDA(cudaEventRecord(ev[0], s));
    (note_launch(), k_be_state<<<grid(), TPB, 0, s>>>(n, up.p, vn.p, w.p, dt, bcp, us.p, vs.p));
    (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, gforce.p, f.p));
    launch_forces(*m, mat, us.p, f.p, s);
    if (has_damping) spmv_node_rows(m->rows(), D.p, vs.p, f.p, -1.0, 1.0, s);  // f += -D v
    HOEFEM_CUDA(cudaEventRecord(ev[1], s));
    (note_launch(), k_F<<<grid(), TPB, 0, s>>>(n, f.p, bcp, dt, F.p));
    spmv_node_rows(m->rows(), M.p, w.p, F.p, 1.0, 1.0, s);
    double r = norm_sq(F.p);
    stats.ms_assemble_forces += elapsed();
    check_device_error(*m);
    return r;
  }

  int solve_jacobian(double dt) {
    cudaStream_t s = m->stream;
    const int n = (int)m->ndof;
    const unsigned char* bcp = bc_nodes.empty() ? nullptr : bc.p;
    HOEFEM_CUDA(cudaEventRecord(ev[0], s));
    (note_launch(), k_be_state<<<grid(), TPB, 0, s>>>(n, up.p, vn.p, w.p, dt, bcp, us.p, vs.p));
    launch_stiffness(*m, mat, us.p, K.p, s, precision, /*assign=*/true);
    // J = gamma M - beta D - alpha K with alpha = -dt^2, beta = -dt, gamma = 1
    jacobian_combination(*m, -(-dt * dt), K.p, 1.0, M.p, bcp, J.p, scalars.p + 4, s, -(-dt),
                         has_damping ? D.p : nullptr);
    HOEFEM_CUDA(cudaEventRecord(ev[1], s));
    check_device_error(*m);
    stats.ms_assemble_stiffness += elapsed();
    HOEFEM_CUDA(cudaEventRecord(ev[0], s));
    P->want_fp32 = (precision == PRECISION_FP32);
    precond_update(*P, J.p, s);
    HOEFEM_CUDA(cudaEventRecord(ev[1], s));
    HOEFEM_CUDA(cudaEventSynchronize(ev[1]));
    stats.ms_precond_update += elapsed();
    HOEFEM_CUDA(cudaMemsetAsync(cg.x.p, 0, sizeof(double) * n, s));
    (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, F.p, cg.b.p));
    if (learned && learned_mode == 1 && learned->trained) warm_start(s);
    const bool collecting = learned && learned_mode >= 2 && precision == PRECISION_FP64;
    if (collecting && learned_mode == 3) start_collect();
    i64 it = 0;
    HOEFEM_CUDA(cudaEventRecord(ev[0], s));
    int st;
    if (learned && learned_mode == 4 && learned->trained && precision == PRECISION_FP64) {
      i64 kept = 0, dropped = 0;
      st = cg_solve_learned(cg, J.p, P, learned, cg_tol, cg_max, &it, &kept, &dropped, s);
      stats.learned_accepted += kept;
      stats.learned_rejected += dropped;
    } else if (precision == PRECISION_FP32) {
      if (J32.n < (size_t)m->nnz) J32.alloc(m->nnz);
      to_f32(J.p, J32.p, m->nnz, s);
      i64 reps = 0;
      st = cg_solve_reliable(cg, J.p, J32.p, P, cg_tol, cg_max, delta, &it, &reps, s);
      stats_replacements += reps;
    } else {
      st = cg_solve(cg, J.p, P, cg_tol, cg_max, &it, s);
    }
    HOEFEM_CUDA(cudaEventRecord(ev[1], s));
    HOEFEM_CUDA(cudaEventSynchronize(ev[1]));
    stats.ms_cg += elapsed();
    account_warm_start();
    stats.num_cg_solves += 1;
    stats.total_cg_iterations += it;
    if (it > stats.max_cg_iterations) stats.max_cg_iterations = it;
    stats.last_cg_status = st;
    if (collecting) finish_collect(st, s);
    (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, cg.x.p, dx.p));
    // MaxIterationsReached and IndefiniteOperator are tolerated (newton_cg.rs:776-797)
    if (st == HOEFEM_OK || st == HOEFEM_CG_MAX_ITERATIONS || st == HOEFEM_CG_INDEFINITE_OPERATOR) return HOEFEM_OK;
    return st;
  }

  // Learned warm start with the residual guard: the MLP's correction d,
  // scaled by the energy-optimal alpha = d.F / d.J d (the minimiser of the
  // J-norm error along d), kept only if ||F - alpha J d|| < ||F||.
  void warm_start(cudaStream_t s) {
    // all on the device, no host synchronisation: the prediction from the
    // residual and its norm, the energy-optimal scale, the guard, and x set
    // only when the guard passes; the counters are read after the step.  The
    // ~20 small kernels run as one CUDA graph (fixed buffers per integrator).
    const int n = (int)m->ndof;
    if (x0.n < (size_t)n) { x0.alloc(n); r0.alloc(n); }
    if (!lw.p) {
      lw.alloc(8);
      for (auto& e : lev) HOEFEM_CUDA(cudaEventCreate(&e));
    }
    if (!ws_exec || ws_key != (const void*)learned) {
      if (ws_exec) cudaGraphExecDestroy(ws_exec);
      ws_exec = nullptr;
      cudaStream_t cs;
      HOEFEM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      cudaGraph_t g;
      HOEFEM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      g_capture_count = 0;
      enqueue_warm_start(cs);
      ws_kernels = g_capture_count;
      g_capture_count = -1;
      HOEFEM_CUDA(cudaStreamEndCapture(cs, &g));
      HOEFEM_CUDA(cudaGraphInstantiate(&ws_exec, g, 0));
      HOEFEM_CUDA(cudaGraphDestroy(g));
      HOEFEM_CUDA(cudaStreamDestroy(cs));
      ws_key = (const void*)learned;
    }
    HOEFEM_CUDA(cudaEventRecord(lev[0], s));
    HOEFEM_CUDA(cudaGraphLaunch(ws_exec, s));
    g_launch_count.fetch_add(ws_kernels, std::memory_order_relaxed);
    HOEFEM_CUDA(cudaEventRecord(lev[1], s));
    lev_pending = true;
  }

  void enqueue_warm_start(cudaStream_t s) {
    const int n = (int)m->ndof;
    dot_device(F.p, F.p, n, lw.p + 0, partials.p, counter.p, s);
    learned->predict_device(F.p, lw.p + 0, x0.p, s);
    spmv_node_rows(m->rows(), J.p, x0.p, r0.p, 1.0, 0.0, s);
    dot_device(x0.p, r0.p, n, lw.p + 1, partials.p, counter.p, s);
    dot_device(x0.p, F.p, n, lw.p + 2, partials.p, counter.p, s);
    (note_launch(), k_warm_alpha<<<1, 1, 0, s>>>(lw.p));
    (note_launch(), k_warm_residual<<<grid(), TPB, 0, s>>>(n, lw.p, r0.p, F.p));
    dot_device(r0.p, r0.p, n, lw.p + 3, partials.p, counter.p, s);
    (note_launch(), k_warm_accept<<<grid(), TPB, 0, s>>>(n, lw.p, x0.p, cg.x.p));
  }

  // Time of the last warm start (its events have completed once the solve has
  // been waited for).
  void account_warm_start() {
    if (!lev_pending) return;
    float ms = 0.f;
    HOEFEM_CUDA(cudaEventElapsedTime(&ms, lev[0], lev[1]));
    stats.ms_learned += ms;
    lev_pending = false;
  }

  // Training-pair collection: snapshot (x_k, r_k) after every CG chunk.
  void start_collect() {
    for (auto* b : snaps) delete b;
    snaps.clear();
    cg.on_chunk = [this](cudaStream_t st) {
      if (snaps.size() >= 64) return;
      const int n = (int)m->ndof;
      auto* xs = new DBuf<double>();
      auto* rs = new DBuf<double>();
      xs->alloc(n);
      rs->alloc(n);
      HOEFEM_CUDA(cudaMemcpyAsync(xs->p, cg.x.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      HOEFEM_CUDA(cudaMemcpyAsync(rs->p, cg.r.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      snaps.push_back(xs);
      snaps.push_back(rs);
    };
  }

  void finish_collect(int status, cudaStream_t s) {
    cg.on_chunk = nullptr;
    const int n = (int)m->ndof;
    if (status == HOEFEM_OK) {
      // the right-hand side itself: r = b, e = x*
      learned->add_pair(cg.b.p, cg.x.p, s);
      if (x0.n < (size_t)n) { x0.alloc(n); r0.alloc(n); }
      for (size_t k = 0; k + 1 < snaps.size(); k += 2) {
        // e_k = x* - x_k
        (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, cg.x.p, x0.p));
        (note_launch(), k_axpy_w<<<grid(), TPB, 0, s>>>(n, -1.0, snaps[k]->p, x0.p));
        learned->add_pair(snaps[k + 1]->p, x0.p, s);
      }
    }
    HOEFEM_CUDA(cudaStreamSynchronize(s));
    for (auto* b : snaps) delete b;
    snaps.clear();
  }

  // Damping matrix of the (sub)step starting at state u (no boundary
  // conditions on D; the stiffness part is assembled with element-wise PSD
  // projection, then D = 0 + alpha K_proj + gamma M).
  void compute_damping() {
    has_damping = has_mass_damping || has_stiffness_damping;
    if (!has_damping) return;
    cudaStream_t s = m->stream;
    if (D.n < (size_t)m->nnz) D.alloc(m->nnz);
    if (has_stiffness_damping) {
      K.zero(s);
      launch_stiffness_projected(*m, mat, u.p, K.p, s);
      check_device_error(*m);
    }
    jacobian_combination(*m, stiffness_damping, has_stiffness_damping ? K.p : nullptr, mass_damping,
                         has_mass_damping ? M.p : nullptr, nullptr, D.p, scalars.p + 4, s);
  }

  int be_step(double dt) {
    cudaStream_t s = m->stream;
    const int n = (int)m->ndof;
    compute_damping();
    (note_launch(), k_be_init<<<grid(), TPB, 0, s>>>(n, u.p, v.p, dt, up.p, vn.p, w.p));
    const double tol = dt * (1e-5 * rep_force);
    double fsq = eval_F(dt);
    i64 iter = 0;
    while (std::sqrt(fsq) > tol) {
      if (iter == newton_max) return HOEFEM_NEWTON_MAX_ITERATIONS;
      int st = solve_jacobian(dt);
      if (st != HOEFEM_OK) return st;
      (note_launch(), k_neg<<<grid(), TPB, 0, s>>>(n, dx.p));
      const double c = 1e-4, alpha_min = 1e-6;
      const double g0 = 0.5 * fsq;
      const double initial[4] = {0.0, 1.0, 0.75, 0.5};
      double alpha_prev = 0.0, alpha = 1.0, tail = 0.25;
      int k = 1;
      for (;;) {
        (note_launch(), k_axpy_w<<<grid(), TPB, 0, s>>>(n, alpha - alpha_prev, dx.p, w.p));
        fsq = eval_F(dt);
        double g = 0.5 * fsq;
        if (g <= (1.0 - c * alpha) * g0) break;
        if (alpha < alpha_min) return HOEFEM_LINE_SEARCH_FAILED;
        alpha_prev = alpha;
        stats.line_search_backtracks += 1;
        ++k;
        if (k < 4) alpha = initial[k];
        else { alpha = tail; tail *= 0.25; }
      }
      ++iter;
    }
    stats.newton_iterations = iter;
    stats.residual_norm = std::sqrt(fsq);
    (note_launch(), k_be_final<<<grid(), TPB, 0, s>>>(n, w.p, dt, bc_nodes.empty() ? nullptr : bc.p, u.p, v.p));
    HOEFEM_CUDA(cudaGetLastError());
    return HOEFEM_OK;
  }

  // integrate_model_with_substeps: u, v device pointers (length ndof)
  int step(double* ud, double* vd, double t, double dt) {
    (void)t;
    cudaStream_t s = m->stream;
    const int n = (int)m->ndof;
    stats = hoefem_step_stats{};
    if (lw.p) lw.zero(s);
    cg.stream_launches = 0;
    cg.stream_iterations = 0;
    cg.stream_ms_total = 0.0;
    stats.representative_force = rep_force;
    cudaEvent_t t0, t1;
    HOEFEM_CUDA(cudaEventCreate(&t0));
    HOEFEM_CUDA(cudaEventCreate(&t1));
    HOEFEM_CUDA(cudaEventRecord(t0, s));
    if (!bc_nodes.empty()) (note_launch(), k_bc_uv<<<grid(), TPB, 0, s>>>(n, bc.p, ud, vd));
    i64 num = 1;
    int result = HOEFEM_OK;
    for (;;) {
      (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, ud, u.p));
      (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, vd, v.p));
      double sdt = dt / (double)num;
      bool failed = false;
      for (i64 k = 0; k < num; ++k) {
        int r;
        try {
          r = be_step(sdt);
        } catch (Error& e) {
          if (e.code == HOEFEM_ERR_CUDA || e.code == HOEFEM_ERR_OUT_OF_MEMORY) throw;
          r = e.code;
        }
        if (r != HOEFEM_OK) { failed = true; result = r; break; }
      }
      if (!failed) { result = HOEFEM_OK; break; }
      num *= 5;
      if (num >= 1000) { result = HOEFEM_SUBSTEPPING_FAILED; break; }
    }
    stats.substeps = num;
    if (result == HOEFEM_OK) {
      (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, u.p, ud));
      (note_launch(), k_copy<<<grid(), TPB, 0, s>>>(n, v.p, vd));
    }
    HOEFEM_CUDA(cudaEventRecord(t1, s));
    HOEFEM_CUDA(cudaEventSynchronize(t1));
    float ms = 0.f;
    HOEFEM_CUDA(cudaEventElapsedTime(&ms, t0, t1));
    stats.ms_total = ms;
    if (lw.p && learned_mode == 1) {
      double h[8];
      HOEFEM_CUDA(cudaMemcpy(h, lw.p, sizeof(h), cudaMemcpyDeviceToHost));
      stats.learned_accepted += (i64)h[4];
      stats.learned_rejected += (i64)h[5];
      if (h[4] > 0.0) stats.learned_residual_ratio = h[6] / h[4];
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return result;
  }
};

Integrator* integrator_new(Model* m, const hoefem_material* mat, double density, const i64* bc_nodes, i64 nbc,
                           int gravity_enabled, double gravity, Precond* P) {
  std::unique_ptr<Integrator> it(new Integrator());
  it->m = m;
  it->mat = MatDev{mat->kind, mat->mu, mat->lambda};
  it->density = density;
  it->bc_nodes.assign(bc_nodes, bc_nodes + nbc);
  it->gravity_enabled = gravity_enabled != 0;
  it->gravity = gravity;
  it->P = P;
  it->setup();
  return it.release();
}
void integrator_delete(Integrator* it) { delete it; }
void integrator_set_learned(Integrator* it, Learned* l, int mode) {
  it->learned = l;
  it->learned_mode = l ? mode : 0;
}
void integrator_set_precision(Integrator* it, int precision, double delta) {
  it->precision = precision;
  it->delta = delta;
}
void integrator_set_damping(Integrator* it, bool has_mass, double mass_coeff, bool has_stiffness,
                            double stiffness_coeff) {
  it->has_mass_damping = has_mass;
  it->mass_damping = mass_coeff;
  it->has_stiffness_damping = has_stiffness;
  it->stiffness_damping = stiffness_coeff;
}

void integrator_set_tolerances(Integrator* it, double tol, i64 cg_max, i64 newton_max) {
  it->cg_tol = tol;
  it->cg_max = cg_max;
  it->newton_max = newton_max;
}
int integrator_step(Integrator* it, double* ud, double* vd, double t, double dt) { return it->step(ud, vd, t, dt); }
hoefem_step_stats integrator_stats(Integrator* it) { return it->stats; }
CgWork* integrator_cg(Integrator* it) { return &it->cg; }
const Precond* integrator_precond(Integrator* it) { return it->P; }
const double* integrator_mass(Integrator* it) { return it->M.p; }
void integrator_eval_f(Integrator* it, const double* ud, const double* vd, double* f) { it->eval_f(ud, vd, f); }

}  // namespace hoefem
