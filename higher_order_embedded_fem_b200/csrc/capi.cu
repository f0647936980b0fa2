// extern "C" entry points of libhoefem (declared in include/hoefem.h).
// Each entry point validates its arguments, stages host arrays through
// stream-ordered device allocations when `mem` is HOEFEM_MEM_HOST, runs the
// device path and converts exceptions into hoefem_status codes.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "internal.h"
#include "scene.h"
#include "solver.h"
#include "learned.h"

namespace hoefem {
struct Integrator;
Integrator* integrator_new(Model* m, const hoefem_material* mat, double density, const i64* bc_nodes, i64 nbc,
                           int gravity_enabled, double gravity, Precond* P);
void integrator_delete(Integrator* it);
void integrator_set_tolerances(Integrator* it, double tol, i64 cg_max, i64 newton_max);
void integrator_set_damping(Integrator* it, bool has_mass, double mass_coeff, bool has_stiffness,
                            double stiffness_coeff);
void integrator_set_precision(Integrator* it, int precision, double delta);
CgWork* integrator_cg(Integrator* it);
const Precond* integrator_precond(Integrator* it);
void integrator_set_learned(Integrator* it, Learned* l, int mode);
int integrator_step(Integrator* it, double* ud, double* vd, double t, double dt);
hoefem_step_stats integrator_stats(Integrator* it);
const double* integrator_mass(Integrator* it);
void integrator_eval_f(Integrator* it, const double* ud, const double* vd, double* f);
void jacobian_combination_noalloc(Model& m, double ck, const double* K, double cm, const double* M,
                                  const long long* bc_nodes, long long num_bc, double* out);
struct Batch;
Batch* batch_build(const std::vector<const Model*>& scenes, const std::vector<MatDev>& mats, double density,
                   const i64* bc_off, const i64* bc_nodes, bool gravity_enabled, double gravity);
void batch_delete(Batch* b);
Model& batch_model(Batch* b);
int batch_step(Batch* b, double* u, double* v, double dt);
void batch_set_tolerances(Batch* b, double tol, i64 cg_max, i64 newton_max);
void batch_set_cg_engine(Batch* b, int engine, int ctas_per_sm);
void batch_cg_choice(Batch* b, int* engine, int* ctas_per_sm, std::vector<float>* tune_ms);
const std::vector<int>& batch_node_offsets(Batch* b);
void batch_scene_stats(Batch* b, int k, hoefem_step_stats* out, int* status);
void greedy_coloring(const i64* conn, i64 ne, int nn, i64 nv, std::vector<i64>& color_off,
                     std::vector<int>& color_elems);
}  // namespace hoefem

namespace hoefem {
std::atomic<long long> g_launch_count{0};
thread_local long long g_capture_count = -1;
}  // namespace hoefem

using namespace hoefem;

struct hoefem_model_s {
  Model m;
  std::unique_ptr<CgWork> cg;
  cudaStream_t own_stream = nullptr;
  ~hoefem_model_s() {
    if (own_stream) m.stream = own_stream;  // the Model destroys its own stream only
  }
};
struct hoefem_precond_s {
  Precond p;
};
struct hoefem_integrator_s {
  Integrator* it = nullptr;
  hoefem_model_s* model = nullptr;
  ~hoefem_integrator_s() { integrator_delete(it); }
};
struct hoefem_learned_s {
  Learned l;
  hoefem_model_s* model = nullptr;
};
struct hoefem_scene_s {
  Scene* s = nullptr;
  ~hoefem_scene_s() { delete s; }
};
struct hoefem_batch_s {
  Batch* b = nullptr;
  cudaStream_t own_stream = nullptr;
  ~hoefem_batch_s() {
    if (b && own_stream) batch_model(b).stream = own_stream;
    batch_delete(b);
  }
};

namespace {

thread_local std::string g_error;

int fail(int code, const char* msg) {
  g_error = msg;
  return code;
}

#define API_BEGIN try {
#define API_END                                                \
  }                                                            \
  catch (const Error& e) {                                     \
    return fail(e.code, e.what());                             \
  }                                                            \
  catch (const std::bad_alloc&) {                              \
    return fail(HOEFEM_ERR_OUT_OF_MEMORY, "host out of memory"); \
  }                                                            \
  catch (const std::exception& e) {                            \
    return fail(HOEFEM_ERR_INVALID_ARGUMENT, e.what());        \
  }                                                            \
  return HOEFEM_OK;

// A device view of a caller array: the pointer itself for device memory, a
// stream-ordered temporary (copied in / out) for host memory.
struct View {
  double* d = nullptr;
  double* host = nullptr;
  size_t n = 0;
  bool owned = false;
  cudaStream_t s = nullptr;
  View(const double* p, size_t count, int mem, cudaStream_t st, bool copy_in) : n(count), s(st) {
    HOEFEM_REQUIRE(p != nullptr || count == 0, HOEFEM_ERR_INVALID_ARGUMENT, "null array");
    HOEFEM_REQUIRE(mem == HOEFEM_MEM_HOST || mem == HOEFEM_MEM_DEVICE, HOEFEM_ERR_INVALID_ARGUMENT, "bad mem flag");
    if (mem == HOEFEM_MEM_DEVICE) {
      d = const_cast<double*>(p);
    } else {
      owned = true;
      host = const_cast<double*>(p);
      HOEFEM_CUDA(cudaMallocAsync(&d, (count ? count : 1) * sizeof(double), s));
      if (copy_in && count) HOEFEM_CUDA(cudaMemcpyAsync(d, p, count * sizeof(double), cudaMemcpyHostToDevice, s));
    }
  }
  void copy_out() {
    if (owned && n) HOEFEM_CUDA(cudaMemcpyAsync(host, d, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  ~View() {
    if (owned && d) cudaFreeAsync(d, s);
  }
};

Model& model_of(hoefem_model m) {
  HOEFEM_REQUIRE(m != nullptr, HOEFEM_ERR_INVALID_ARGUMENT, "null model");
  return m->m;
}

Model& device_model(hoefem_model m) {
  Model& mm = model_of(m);
  ensure_device(mm);
  return mm;
}

MatDev mat_of(const hoefem_material* mat) {
  HOEFEM_REQUIRE(mat != nullptr, HOEFEM_ERR_INVALID_ARGUMENT, "null material");
  HOEFEM_REQUIRE(mat->kind == HOEFEM_MAT_STVK || mat->kind == HOEFEM_MAT_SNH, HOEFEM_ERR_INVALID_ARGUMENT,
                 "unknown material kind");
  return MatDev{mat->kind, mat->mu, mat->lambda};
}

void sync(Model& m) { HOEFEM_CUDA(cudaStreamSynchronize(m.stream)); }

}  // namespace

namespace hoefem {
struct Embedding;
Embedding* embedding_create(const double* bgX, i64 nbv, const i64* bg_conn, i64 nbc, int npc, const double* eX,
                            i64 nev, const i64* tets, i64 nt, double lower, double upper);
void embedding_destroy(Embedding* e);
void embedding_cells(const Embedding& e, i64* ne, i64* ni, i64* nf, int* cls, double* cut);
i64 embedding_quadrature(Embedding& e, const double* tw, const double* tp, i64 nq, double stab_factor,
                         const double* sw, const double* sp, i64 ns);
void embedding_copy_quadrature(const Embedding& e, i64* off, double* w, double* p);
void quadrature_simplify(i64 nrules, const i64* off, const double* w, const double* p, int strength, i64* out_off,
                         double* out_w, double* out_p);
}  // namespace hoefem

extern "C" {

const char* hoefem_last_error(void) { return g_error.c_str(); }
int hoefem_abi_version(void) { return HOEFEM_ABI_VERSION; }

int hoefem_launch_count(int64_t* count) {
  if (!count) return fail(HOEFEM_ERR_INVALID_ARGUMENT, "null output");
  *count = g_launch_count.load();
  return HOEFEM_OK;
}

int hoefem_set_device(int device) {
  API_BEGIN
  HOEFEM_CUDA(cudaSetDevice(device));
  API_END
}

int hoefem_lame_from_young_poisson(double young, double poisson, double* mu, double* lambda) {
  if (!mu || !lambda) return fail(HOEFEM_ERR_INVALID_ARGUMENT, "null output");
  double m = 0.5 * young / (1.0 + poisson);
  *mu = m;
  *lambda = 0.5 * m * poisson / (1.0 - 2.0 * poisson);
  return HOEFEM_OK;
}

// ---- model -----------------------------------------------------------------
int hoefem_model_create(const double* vertices, int64_t num_vertices, hoefem_model* out) {
  API_BEGIN
  HOEFEM_REQUIRE(out && (vertices || num_vertices == 0) && num_vertices >= 0, HOEFEM_ERR_INVALID_ARGUMENT,
                 "bad arguments");
  auto* h = new hoefem_model_s();
  h->m.nv = num_vertices;
  h->m.X.assign(vertices, vertices + 3 * num_vertices);
  *out = h;
  API_END
}

int hoefem_model_add_block(hoefem_model m, int element_kind, const int64_t* connectivity, int64_t num_elements,
                           const int64_t* quad_offsets, const double* quad_weights, const double* quad_points,
                           int64_t num_quad_points) {
  API_BEGIN
  Model& mm = model_of(m);
  HOEFEM_REQUIRE(!mm.finalized, HOEFEM_ERR_INVALID_ARGUMENT, "model already finalized");
  HOEFEM_REQUIRE(element_kind == HOEFEM_ELEM_TET10 || element_kind == HOEFEM_ELEM_HEX27, HOEFEM_ERR_INVALID_ARGUMENT,
                 "unsupported element kind");
  HOEFEM_REQUIRE(num_elements >= 0 && (connectivity || num_elements == 0), HOEFEM_ERR_INVALID_ARGUMENT,
                 "bad connectivity");
  HOEFEM_REQUIRE(num_quad_points >= 0 && quad_weights && quad_points, HOEFEM_ERR_INVALID_ARGUMENT,
                 "missing quadrature");
  std::unique_ptr<Block> b(new Block());
  b->kind = element_kind;
  b->nn = element_kind == HOEFEM_ELEM_TET10 ? 10 : 27;
  b->ne = num_elements;
  b->conn.assign(connectivity, connectivity + num_elements * b->nn);
  b->uniform = quad_offsets == nullptr;
  if (!b->uniform) {
    b->qoff.assign(quad_offsets, quad_offsets + num_elements + 1);
    HOEFEM_REQUIRE(b->qoff[0] == 0 && b->qoff[num_elements] == num_quad_points, HOEFEM_ERR_INVALID_ARGUMENT,
                   "quadrature offsets do not match the number of points");
    for (int64_t e = 0; e < num_elements; ++e)
      HOEFEM_REQUIRE(b->qoff[e + 1] >= b->qoff[e], HOEFEM_ERR_INVALID_ARGUMENT, "decreasing quadrature offsets");
  }
  b->qw.assign(quad_weights, quad_weights + num_quad_points);
  b->qp.assign(quad_points, quad_points + 3 * num_quad_points);
  mm.blocks.push_back(b.release());
  API_END
}

int hoefem_model_finalize(hoefem_model m) {
  API_BEGIN
  finalize_model(model_of(m));
  API_END
}

int hoefem_model_destroy(hoefem_model m) {
  API_BEGIN
  delete m;
  API_END
}

int hoefem_model_set_stream(hoefem_model m, void* stream) {
  API_BEGIN
  Model& mm = device_model(m);
  if (!m->own_stream) m->own_stream = mm.stream;
  HOEFEM_CUDA(cudaStreamSynchronize(mm.stream));
  mm.stream = stream ? (cudaStream_t)stream : m->own_stream;
  API_END
}

int hoefem_model_autotune(hoefem_model m, int32_t* lanes) {
  API_BEGIN
  Model& mm = device_model(m);
  DBuf<double> v;
  v.alloc(mm.nnz);
  v.zero(mm.stream);
  mm.spmv_lanes = autotune_spmv_lanes(mm.rows(), v.p, mm.stream);
  if (lanes) *lanes = mm.spmv_lanes;
  API_END
}

int hoefem_model_set_spmv_variant(hoefem_model m, int32_t variant) {
  API_BEGIN
  Model& mm = device_model(m);
  HOEFEM_REQUIRE(variant == 8 || variant == 16 || variant == 32 || variant == 108 || variant == 116 || variant == 132,
                 HOEFEM_ERR_INVALID_ARGUMENT, "unknown SpMV variant");
  mm.spmv_lanes = variant;
  mm.spmv_lanes32 = variant;
  mm.spmv_pinned = true;
  API_END
}

int hoefem_model_set_stiffness_path(hoefem_model m, int path) {
  API_BEGIN
  Model& mm = device_model(m);
  HOEFEM_REQUIRE(path == HOEFEM_STIFFNESS_AUTO || path == HOEFEM_STIFFNESS_CUDA_CORES || path == HOEFEM_STIFFNESS_STAGED,
                 HOEFEM_ERR_INVALID_ARGUMENT, "unknown stiffness path");
  mm.stiffness_path = path == HOEFEM_STIFFNESS_AUTO ? STIFFNESS_AUTO
                      : path == HOEFEM_STIFFNESS_STAGED ? STIFFNESS_STAGED : STIFFNESS_CUDA_CORES;
  API_END
}

int hoefem_model_get_spmv_variants(hoefem_model m, int32_t* fp64_values, int32_t* fp32_values) {
  API_BEGIN
  Model& mm = model_of(m);
  if (fp64_values) *fp64_values = mm.spmv_lanes;
  if (fp32_values) *fp32_values = mm.spmv_lanes32 ? mm.spmv_lanes32 : mm.spmv_lanes;
  API_END
}

int hoefem_model_sizes(hoefem_model m, int64_t* ndof, int64_t* nnz, int64_t* num_elements, int64_t* num_blocks) {
  API_BEGIN
  Model& mm = model_of(m);
  HOEFEM_REQUIRE(mm.finalized, HOEFEM_ERR_NOT_FINALIZED, "model is not finalized");
  if (ndof) *ndof = mm.ndof;
  if (nnz) *nnz = mm.nnz;
  if (num_elements) *num_elements = mm.num_elements;
  if (num_blocks) *num_blocks = (int64_t)mm.blocks.size();
  API_END
}

int hoefem_model_pattern(hoefem_model m, int64_t* row_offsets, int64_t* column_indices) {
  API_BEGIN
  Model& mm = model_of(m);
  HOEFEM_REQUIRE(mm.finalized, HOEFEM_ERR_NOT_FINALIZED, "model is not finalized");
  HOEFEM_REQUIRE(row_offsets && column_indices, HOEFEM_ERR_INVALID_ARGUMENT, "null output");
  export_pattern(mm.adj_off, mm.adj, mm.base, nullptr, mm.nv, row_offsets, column_indices);
  API_END
}

int hoefem_model_num_colors(hoefem_model m, int block, int64_t* num_colors) {
  API_BEGIN
  Model& mm = model_of(m);
  HOEFEM_REQUIRE(mm.finalized, HOEFEM_ERR_NOT_FINALIZED, "model is not finalized");
  HOEFEM_REQUIRE(block >= 0 && block < (int)mm.blocks.size() && num_colors, HOEFEM_ERR_INVALID_ARGUMENT, "bad block");
  *num_colors = (int64_t)mm.blocks[block]->color_off.size() - 1;
  API_END
}

int hoefem_model_colors(hoefem_model m, int block, int64_t* color_offsets, int64_t* element_labels) {
  API_BEGIN
  Model& mm = model_of(m);
  HOEFEM_REQUIRE(mm.finalized, HOEFEM_ERR_NOT_FINALIZED, "model is not finalized");
  HOEFEM_REQUIRE(block >= 0 && block < (int)mm.blocks.size() && color_offsets && element_labels,
                 HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  const Block& b = *mm.blocks[block];
  for (size_t c = 0; c < b.color_off.size(); ++c) color_offsets[c] = b.color_off[c];
  for (size_t k = 0; k < b.color_elems.size(); ++k) element_labels[k] = b.color_elems[k];
  API_END
}

int hoefem_assemble_elastic_pseudo_forces_into(hoefem_model m, const hoefem_material* mat, const double* u, double* f,
                                               int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  MatDev md = mat_of(mat);
  View U(u, mm.ndof, mem, mm.stream, true), F(f, mm.ndof, mem, mm.stream, true);
  launch_forces(mm, md, U.d, F.d, mm.stream);
  F.copy_out();
  sync(mm);
  check_device_error(mm);
  API_END
}

int hoefem_assemble_stiffness_into(hoefem_model m, const hoefem_material* mat, const double* u, double* values,
                                   int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  MatDev md = mat_of(mat);
  View U(u, mm.ndof, mem, mm.stream, true), V(values, mm.nnz, mem, mm.stream, true);
  launch_stiffness(mm, md, U.d, V.d, mm.stream);
  V.copy_out();
  sync(mm);
  check_device_error(mm);
  API_END
}

int hoefem_assemble_stiffness_into_precision(hoefem_model m, const hoefem_material* mat, const double* u,
                                             double* values, int precision, int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  MatDev md = mat_of(mat);
  HOEFEM_REQUIRE(precision == HOEFEM_PRECISION_FP64 || precision == HOEFEM_PRECISION_MIXED,
                 HOEFEM_ERR_INVALID_ARGUMENT, "bad precision");
  View U(u, mm.ndof, mem, mm.stream, true), V(values, mm.nnz, mem, mm.stream, true);
  launch_stiffness(mm, md, U.d, V.d, mm.stream, precision == HOEFEM_PRECISION_MIXED ? PRECISION_FP32 : PRECISION_FP64);
  V.copy_out();
  sync(mm);
  check_device_error(mm);
  API_END
}

int hoefem_assemble_projected_stiffness_into(hoefem_model m, const hoefem_material* mat, const double* u,
                                             double* values, int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  MatDev md = mat_of(mat);
  View U(u, mm.ndof, mem, mm.stream, true), V(values, mm.nnz, mem, mm.stream, true);
  launch_stiffness_projected(mm, md, U.d, V.d, mm.stream);
  V.copy_out();
  sync(mm);
  check_device_error(mm);
  API_END
}

int hoefem_assemble_mass_into(hoefem_model m, double density, double* values, int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  View V(values, mm.nnz, mem, mm.stream, true);
  launch_mass(mm, density, V.d, mm.stream);
  V.copy_out();
  sync(mm);
  check_device_error(mm);
  API_END
}

static void bc_mask(Model& mm, const int64_t* nodes, int64_t n, DBuf<unsigned char>& mask) {
  std::vector<unsigned char> h(mm.ndof, 0);
  for (int64_t k = 0; k < n; ++k) {
    HOEFEM_REQUIRE(nodes[k] >= 0 && nodes[k] < mm.nv, HOEFEM_ERR_INVALID_ARGUMENT, "boundary node out of range");
    for (int i = 0; i < 3; ++i) h[3 * nodes[k] + i] = 1;
  }
  mask.upload(h, mm.stream);
}

int hoefem_apply_dirichlet_bc_csr(hoefem_model m, const int64_t* nodes, int64_t num_nodes, double* values, int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  HOEFEM_REQUIRE(nodes || num_nodes == 0, HOEFEM_ERR_INVALID_ARGUMENT, "null nodes");
  DBuf<unsigned char> mask;
  bc_mask(mm, nodes, num_nodes, mask);
  DBuf<double> scratch;
  scratch.alloc(1);
  View V(values, mm.nnz, mem, mm.stream, true);
  DBuf<double> tmp;
  tmp.alloc(mm.nnz);
  HOEFEM_CUDA(cudaMemcpyAsync(tmp.p, V.d, mm.nnz * sizeof(double), cudaMemcpyDeviceToDevice, mm.stream));
  jacobian_combination(mm, 0.0, nullptr, 1.0, tmp.p, mask.p, V.d, scratch.p, mm.stream);
  V.copy_out();
  sync(mm);
  API_END
}

int hoefem_jacobian_combination(hoefem_model m, double c_stiffness, const double* stiffness_values, double c_mass,
                                const double* mass_values, const int64_t* bc_nodes, int64_t num_bc, double* out,
                                int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  DBuf<unsigned char> mask;
  if (num_bc > 0) bc_mask(mm, bc_nodes, num_bc, mask);
  DBuf<double> scratch;
  scratch.alloc(1);
  View K(stiffness_values, stiffness_values ? mm.nnz : 0, mem, mm.stream, true);
  View M(mass_values, mass_values ? mm.nnz : 0, mem, mm.stream, true);
  View O(out, mm.nnz, mem, mm.stream, false);
  jacobian_combination(mm, c_stiffness, stiffness_values ? K.d : nullptr, c_mass, mass_values ? M.d : nullptr,
                       num_bc > 0 ? mask.p : nullptr, O.d, scratch.p, mm.stream);
  O.copy_out();
  sync(mm);
  API_END
}

int hoefem_jacobian_combination_damped(hoefem_model m, double c_stiffness, const double* stiffness_values,
                                       double c_damping, const double* damping_values, double c_mass,
                                       const double* mass_values, const int64_t* bc_nodes, int64_t num_bc,
                                       double* out, int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  DBuf<unsigned char> mask;
  if (num_bc > 0) bc_mask(mm, bc_nodes, num_bc, mask);
  DBuf<double> scratch;
  scratch.alloc(1);
  View K(stiffness_values, stiffness_values ? mm.nnz : 0, mem, mm.stream, true);
  View D(damping_values, damping_values ? mm.nnz : 0, mem, mm.stream, true);
  View M(mass_values, mass_values ? mm.nnz : 0, mem, mm.stream, true);
  View O(out, mm.nnz, mem, mm.stream, false);
  jacobian_combination(mm, c_stiffness, stiffness_values ? K.d : nullptr, c_mass, mass_values ? M.d : nullptr,
                       num_bc > 0 ? mask.p : nullptr, O.d, scratch.p, mm.stream, c_damping,
                       damping_values ? D.d : nullptr);
  O.copy_out();
  sync(mm);
  API_END
}

int hoefem_jacobian_combination_noalloc(hoefem_model m, double c_stiffness, const double* stiffness_values,
                                        double c_mass, const double* mass_values, const int64_t* bc_nodes,
                                        int64_t num_bc, double* out) {
  API_BEGIN
  Model& mm = model_of(m);
  jacobian_combination_noalloc(mm, c_stiffness, stiffness_values, c_mass, mass_values,
                               reinterpret_cast<const long long*>(bc_nodes), num_bc, out);
  API_END
}

int hoefem_spmv(hoefem_model m, double beta, double* y, double alpha, const double* values, const double* x, int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  View V(values, mm.nnz, mem, mm.stream, true), X(x, mm.ndof, mem, mm.stream, true),
      Y(y, mm.ndof, mem, mm.stream, beta != 0.0);
  spmv_node_rows(mm.rows(), V.d, X.d, Y.d, alpha, beta, mm.stream);
  Y.copy_out();
  sync(mm);
  API_END
}

// ---- preconditioners -------------------------------------------------------
int hoefem_precond_create_diagonal(hoefem_model m, hoefem_precond* out) {
  API_BEGIN
  Model& mm = device_model(m);
  HOEFEM_REQUIRE(out, HOEFEM_ERR_INVALID_ARGUMENT, "null output");
  auto* h = new hoefem_precond_s();
  h->p.kind = PREC_DIAGONAL;
  h->p.m = &mm;
  *out = h;
  API_END
}

int hoefem_precond_create_schwarz(hoefem_model m, const int64_t* subdomain_offsets, const int64_t* subdomain_nodes,
                                  int64_t num_subdomains, const int64_t* untreated_nodes, int64_t num_untreated,
                                  hoefem_precond* out) {
  API_BEGIN
  Model& mm = device_model(m);
  HOEFEM_REQUIRE(out && subdomain_offsets && num_subdomains >= 0 && num_untreated >= 0, HOEFEM_ERR_INVALID_ARGUMENT,
                 "bad arguments");
  std::unique_ptr<hoefem_precond_s> h(new hoefem_precond_s());
  h->p.m = &mm;
  static const int64_t none = 0;
  precond_create_schwarz(h->p, subdomain_offsets, subdomain_nodes ? subdomain_nodes : &none, num_subdomains,
                         untreated_nodes ? untreated_nodes : &none, num_untreated);
  *out = h.release();
  API_END
}

int hoefem_precond_update(hoefem_precond p, const double* system_values, int mem) {
  API_BEGIN
  HOEFEM_REQUIRE(p, HOEFEM_ERR_INVALID_ARGUMENT, "null preconditioner");
  Model& mm = *p->p.m;
  View V(system_values, mm.nnz, mem, mm.stream, true);
  precond_update(p->p, V.d, mm.stream);
  sync(mm);
  API_END
}

int hoefem_precond_apply(hoefem_precond p, const double* r, double* z, int mem) {
  API_BEGIN
  HOEFEM_REQUIRE(p, HOEFEM_ERR_INVALID_ARGUMENT, "null preconditioner");
  Model& mm = *p->p.m;
  View R(r, mm.ndof, mem, mm.stream, true), Z(z, mm.ndof, mem, mm.stream, false);
  precond_apply(p->p, R.d, Z.d, mm.stream);
  Z.copy_out();
  sync(mm);
  API_END
}

int hoefem_precond_set_spmv_variant(hoefem_precond p, int32_t variant) {
  API_BEGIN
  HOEFEM_REQUIRE(p && p->p.kind == PREC_SCHWARZ, HOEFEM_ERR_INVALID_ARGUMENT, "not a Schwarz preconditioner");
  HOEFEM_REQUIRE(variant == 8 || variant == 16 || variant == 32 || variant == 108 || variant == 116 || variant == 132,
                 HOEFEM_ERR_INVALID_ARGUMENT, "unknown SpMV variant");
  p->p.spmv_lanes = variant;
  p->p.spmv_lanes32 = variant;
  p->p.spmv_pinned = true;
  API_END
}

int hoefem_precond_set_block_apply(hoefem_precond p, int32_t on) {
  API_BEGIN
  HOEFEM_REQUIRE(p && p->p.kind == PREC_SCHWARZ, HOEFEM_ERR_INVALID_ARGUMENT, "not a Schwarz preconditioner");
  HOEFEM_REQUIRE(!on || 3 * p->p.max_nodes <= 96, HOEFEM_ERR_INVALID_ARGUMENT,
                 "block apply supports subdomains of at most 32 nodes");
  p->p.block_apply = on != 0;
  if (!on) precond_assemble(p->p, p->p.m->stream);  // the SpMV apply reads every entry
  API_END
}

int hoefem_precond_get_spmv_variants(hoefem_precond p, int32_t* fp64_values, int32_t* fp32_values) {
  API_BEGIN
  HOEFEM_REQUIRE(p, HOEFEM_ERR_INVALID_ARGUMENT, "null preconditioner");
  if (fp64_values) *fp64_values = p->p.spmv_lanes;
  if (fp32_values) *fp32_values = p->p.spmv_lanes32 ? p->p.spmv_lanes32 : p->p.spmv_lanes;
  API_END
}

int hoefem_precond_nnz(hoefem_precond p, int64_t* nnz) {
  API_BEGIN
  HOEFEM_REQUIRE(p && nnz, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  *nnz = p->p.kind == PREC_SCHWARZ ? p->p.nnz : p->p.m->ndof;
  API_END
}

int hoefem_precond_pattern(hoefem_precond p, int64_t* row_offsets, int64_t* column_indices) {
  API_BEGIN
  HOEFEM_REQUIRE(p && row_offsets && column_indices, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  const Precond& pp = p->p;
  if (pp.kind == PREC_SCHWARZ) {
    export_pattern(pp.adj_off, pp.adj, pp.base, &pp.diag_only, pp.m->nv, row_offsets, column_indices);
  } else {
    for (int64_t i = 0; i <= pp.m->ndof; ++i) row_offsets[i] = i;
    for (int64_t i = 0; i < pp.m->ndof; ++i) column_indices[i] = i;
  }
  API_END
}

int hoefem_precond_values(hoefem_precond p, double* values) {
  API_BEGIN
  HOEFEM_REQUIRE(p && values, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  const Precond& pp = p->p;
  HOEFEM_REQUIRE(pp.ready, HOEFEM_ERR_INVALID_ARGUMENT, "preconditioner has not been updated");
  precond_assemble(pp, pp.m->stream);
  const double* src = pp.kind == PREC_SCHWARZ ? pp.vals.p : pp.diag.p;
  size_t n = pp.kind == PREC_SCHWARZ ? (size_t)pp.nnz : (size_t)pp.m->ndof;
  HOEFEM_CUDA(cudaMemcpyAsync(values, src, n * sizeof(double), cudaMemcpyDeviceToHost, pp.m->stream));
  HOEFEM_CUDA(cudaStreamSynchronize(pp.m->stream));
  API_END
}

int hoefem_precond_destroy(hoefem_precond p) {
  API_BEGIN
  delete p;
  API_END
}

// ---- CG ------------------------------------------------------------------------
int hoefem_cg_solve(hoefem_model m, const double* system_values, hoefem_precond p, const double* b, double* x,
                    double tol, int64_t max_iter, int64_t* iterations, int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  HOEFEM_REQUIRE(iterations, HOEFEM_ERR_INVALID_ARGUMENT, "null iterations");
  HOEFEM_REQUIRE(!p || p->p.m == &mm, HOEFEM_ERR_INVALID_ARGUMENT, "preconditioner of another model");
  if (!m->cg) {
    m->cg.reset(new CgWork());
    m->cg->init(&mm);
  }
  CgWork& w = *m->cg;
  w.stream_launches = 0;
  w.stream_iterations = 0;
  w.stream_ms_total = 0.0;
  View A(system_values, mm.nnz, mem, mm.stream, true);
  View B(b, mm.ndof, mem, mm.stream, true), X(x, mm.ndof, mem, mm.stream, true);
  HOEFEM_CUDA(cudaMemcpyAsync(w.b.p, B.d, mm.ndof * sizeof(double), cudaMemcpyDeviceToDevice, mm.stream));
  HOEFEM_CUDA(cudaMemcpyAsync(w.x.p, X.d, mm.ndof * sizeof(double), cudaMemcpyDeviceToDevice, mm.stream));
  i64 it = 0;
  int st = cg_solve(w, A.d, p ? &p->p : nullptr, tol, max_iter, &it, mm.stream);
  HOEFEM_CUDA(cudaMemcpyAsync(X.d, w.x.p, mm.ndof * sizeof(double), cudaMemcpyDeviceToDevice, mm.stream));
  X.copy_out();
  sync(mm);
  *iterations = it;
  if (st != HOEFEM_OK) return fail(st, "CG did not converge");
  API_END
}

int hoefem_cg_solve_mixed(hoefem_model m, const double* system_values, hoefem_precond p, const double* b, double* x,
                          double tol, int64_t max_iter, double delta, int64_t* iterations, int mem) {
  API_BEGIN
  Model& mm = device_model(m);
  HOEFEM_REQUIRE(iterations && delta > 0.0 && delta < 1.0, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  HOEFEM_REQUIRE(!p || p->p.m == &mm, HOEFEM_ERR_INVALID_ARGUMENT, "preconditioner of another model");
  if (!m->cg) {
    m->cg.reset(new CgWork());
    m->cg->init(&mm);
  }
  CgWork& w = *m->cg;
  w.stream_launches = 0;
  w.stream_iterations = 0;
  w.stream_ms_total = 0.0;
  View A(system_values, mm.nnz, mem, mm.stream, true);
  View B(b, mm.ndof, mem, mm.stream, true), X(x, mm.ndof, mem, mm.stream, true);
  DBuf<float> A32;
  A32.alloc(mm.nnz);
  to_f32(A.d, A32.p, mm.nnz, mm.stream);
  if (p && p->p.kind == PREC_SCHWARZ && p->p.ready && (!p->p.vals32.p || !p->p.want_fp32)) {
    p->p.want_fp32 = true;
    precond_to_fp32(p->p, mm.stream);
  }
  HOEFEM_CUDA(cudaMemcpyAsync(w.b.p, B.d, mm.ndof * sizeof(double), cudaMemcpyDeviceToDevice, mm.stream));
  HOEFEM_CUDA(cudaMemcpyAsync(w.x.p, X.d, mm.ndof * sizeof(double), cudaMemcpyDeviceToDevice, mm.stream));
  i64 it = 0, replacements = 0;
  int st = cg_solve_reliable(w, A.d, A32.p, p ? &p->p : nullptr, tol, max_iter, delta, &it, &replacements, mm.stream);
  HOEFEM_CUDA(cudaMemcpyAsync(X.d, w.x.p, mm.ndof * sizeof(double), cudaMemcpyDeviceToDevice, mm.stream));
  X.copy_out();
  sync(mm);
  *iterations = it;
  if (st != HOEFEM_OK) return fail(st, "CG did not converge");
  API_END
}

// ---- integrator ----------------------------------------------------------------
int hoefem_integrator_create(hoefem_model m, const hoefem_material* mat, double density, const int64_t* bc_nodes,
                             int64_t num_bc, int gravity_enabled, double gravity, hoefem_precond precond,
                             hoefem_integrator* out) {
  API_BEGIN
  Model& mm = device_model(m);
  mat_of(mat);
  HOEFEM_REQUIRE(out && (bc_nodes || num_bc == 0), HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  HOEFEM_REQUIRE(!precond || precond->p.m == &mm, HOEFEM_ERR_INVALID_ARGUMENT, "preconditioner of another model");
  std::unique_ptr<hoefem_integrator_s> h(new hoefem_integrator_s());
  h->model = m;
  h->it = integrator_new(&mm, mat, density, bc_nodes, num_bc, gravity_enabled, gravity,
                         precond ? &precond->p : nullptr);
  *out = h.release();
  API_END
}

int hoefem_integrator_set_tolerances(hoefem_integrator it, double cg_tol, int64_t cg_max_iter,
                                     int64_t newton_max_iter) {
  API_BEGIN
  HOEFEM_REQUIRE(it && cg_tol > 0.0, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  integrator_set_tolerances(it->it, cg_tol, cg_max_iter, newton_max_iter);
  API_END
}

int hoefem_integrator_set_precision(hoefem_integrator it, int precision, double delta) {
  API_BEGIN
  HOEFEM_REQUIRE(it && (precision == HOEFEM_PRECISION_FP64 || precision == HOEFEM_PRECISION_MIXED) &&
                     delta > 0.0 && delta < 1.0,
                 HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  integrator_set_precision(it->it, precision == HOEFEM_PRECISION_MIXED ? PRECISION_FP32 : PRECISION_FP64, delta);
  API_END
}

static void set_engine(CgWork& w, int engine, int options) {
  HOEFEM_REQUIRE(engine >= HOEFEM_CG_ENGINE_AUTO && engine <= HOEFEM_CG_ENGINE_STREAMED, HOEFEM_ERR_INVALID_ARGUMENT,
                 "unknown CG engine");
  HOEFEM_REQUIRE((options & ~(HOEFEM_CG_SCHWARZ_FP16 | HOEFEM_CG_PHASE_PROFILE)) == 0, HOEFEM_ERR_INVALID_ARGUMENT,
                 "unknown CG engine option");
  w.stream_mode = engine;
  w.schwarz_half = (options & HOEFEM_CG_SCHWARZ_FP16) != 0;
  w.phase_profile = (options & HOEFEM_CG_PHASE_PROFILE) != 0;
}

static void engine_stats(CgWork& w, const Precond* P, hoefem_cg_engine_stats* out) {
  HOEFEM_REQUIRE(out, HOEFEM_ERR_INVALID_ARGUMENT, "null stats");
  out->launches = w.stream_launches;
  out->iterations = w.stream_iterations;
  out->device_ms = w.stream_ms_total;
  out->operator_bytes = w.sop32.vsize && w.last_f32 ? w.sop32.bytes : w.sop64.bytes;
  out->schwarz_bytes = (P && P->kind == PREC_SCHWARZ) ? w.ssw.bytes : 0;
  cg_stream_phase_us(w, out->phase_us, out->phase_us_max, out->busy_us);
  const CgWork::EngineTune& et = w.etune[w.last_tune];
  out->auto_us_per_iteration[0] = et.us_per_it[0];
  out->auto_us_per_iteration[1] = et.us_per_it[1];
  out->auto_choice = et.choice;
}

int hoefem_integrator_set_cg_engine(hoefem_integrator it, int engine, int options) {
  API_BEGIN
  HOEFEM_REQUIRE(it, HOEFEM_ERR_INVALID_ARGUMENT, "null integrator");
  set_engine(*integrator_cg(it->it), engine, options);
  API_END
}

int hoefem_model_set_cg_engine(hoefem_model m, int engine, int options) {
  API_BEGIN
  Model& mm = device_model(m);
  if (!m->cg) {
    m->cg.reset(new CgWork());
    m->cg->init(&mm);
  }
  set_engine(*m->cg, engine, options);
  API_END
}

int hoefem_integrator_set_cg_l2_keep(hoefem_integrator it, int64_t bytes) {
  API_BEGIN
  HOEFEM_REQUIRE(it, HOEFEM_ERR_INVALID_ARGUMENT, "null integrator");
  integrator_cg(it->it)->l2_keep = bytes < 0 ? -1 : bytes;
  API_END
}

int hoefem_model_set_cg_l2_keep(hoefem_model m, int64_t bytes) {
  API_BEGIN
  Model& mm = device_model(m);
  if (!m->cg) {
    m->cg.reset(new CgWork());
    m->cg->init(&mm);
  }
  m->cg->l2_keep = bytes < 0 ? -1 : bytes;
  API_END
}

int hoefem_integrator_cg_engine_stats(hoefem_integrator it, hoefem_cg_engine_stats* out) {
  API_BEGIN
  HOEFEM_REQUIRE(it, HOEFEM_ERR_INVALID_ARGUMENT, "null integrator");
  engine_stats(*integrator_cg(it->it), integrator_precond(it->it), out);
  API_END
}

int hoefem_model_cg_engine_stats(hoefem_model m, hoefem_cg_engine_stats* out) {
  API_BEGIN
  HOEFEM_REQUIRE(m && m->cg, HOEFEM_ERR_INVALID_ARGUMENT, "no CG has run on this model");
  engine_stats(*m->cg, nullptr, out);
  API_END
}

int hoefem_integrator_step(hoefem_integrator it, double* u, double* v, double t, double dt, int mem) {
  API_BEGIN
  HOEFEM_REQUIRE(it && dt > 0.0, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  Model& mm = it->model->m;
  View U(u, mm.ndof, mem, mm.stream, true), V(v, mm.ndof, mem, mm.stream, true);
  int st = integrator_step(it->it, U.d, V.d, t, dt);
  U.copy_out();
  V.copy_out();
  sync(mm);
  if (st != HOEFEM_OK) return fail(st, "time step failed");
  API_END
}

int hoefem_integrator_set_damping(hoefem_integrator it, int has_mass, double mass_coeff, int has_stiffness,
                                  double stiffness_coeff) {
  API_BEGIN
  HOEFEM_REQUIRE(it, HOEFEM_ERR_INVALID_ARGUMENT, "null integrator");
  integrator_set_damping(it->it, has_mass != 0, mass_coeff, has_stiffness != 0, stiffness_coeff);
  API_END
}

int hoefem_integrator_stats(hoefem_integrator it, hoefem_step_stats* out) {
  API_BEGIN
  HOEFEM_REQUIRE(it && out, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  *out = integrator_stats(it->it);
  API_END
}

int hoefem_integrator_mass(hoefem_integrator it, double* values) {
  API_BEGIN
  HOEFEM_REQUIRE(it && values, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  Model& mm = it->model->m;
  HOEFEM_CUDA(cudaMemcpyAsync(values, integrator_mass(it->it), mm.nnz * sizeof(double), cudaMemcpyDeviceToHost,
                              mm.stream));
  sync(mm);
  API_END
}

int hoefem_integrator_eval_f(hoefem_integrator it, const double* u, const double* v, double* f, int mem) {
  API_BEGIN
  HOEFEM_REQUIRE(it, HOEFEM_ERR_INVALID_ARGUMENT, "null integrator");
  Model& mm = it->model->m;
  View U(u, mm.ndof, mem, mm.stream, true), V(v, mm.ndof, mem, mm.stream, true), F(f, mm.ndof, mem, mm.stream, false);
  integrator_eval_f(it->it, U.d, V.d, F.d);
  F.copy_out();
  sync(mm);
  API_END
}

int hoefem_integrator_destroy(hoefem_integrator it) {
  API_BEGIN
  delete it;
  API_END
}

// ---- learned coarse correction -----------------------------------------------------
int hoefem_learned_create(hoefem_model m, const int64_t* bc_nodes, int64_t num_bc, int num_subdomains,
                          uint64_t seed, hoefem_learned* out) {
  API_BEGIN
  Model& mm = device_model(m);
  HOEFEM_REQUIRE(out && (bc_nodes || num_bc == 0), HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  std::vector<unsigned char> mask(mm.ndof, 0);
  for (int64_t k = 0; k < num_bc; ++k) {
    HOEFEM_REQUIRE(bc_nodes[k] >= 0 && bc_nodes[k] < mm.nv, HOEFEM_ERR_INVALID_ARGUMENT, "node out of range");
    for (int i = 0; i < 3; ++i) mask[3 * bc_nodes[k] + i] = 1;
  }
  std::unique_ptr<hoefem_learned_s> h(new hoefem_learned_s());
  h->model = m;
  h->l.setup(&mm, mask.data(), num_subdomains, seed);
  *out = h.release();
  API_END
}

int hoefem_learned_destroy(hoefem_learned l) {
  API_BEGIN
  delete l;
  API_END
}

int hoefem_learned_num_pairs(hoefem_learned l, int64_t* n) {
  API_BEGIN
  HOEFEM_REQUIRE(l && n, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  *n = l->l.n_data;
  API_END
}

int hoefem_learned_num_params(hoefem_learned l, int64_t* n) {
  API_BEGIN
  HOEFEM_REQUIRE(l && n, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  *n = (int64_t)l->l.n_params;
  API_END
}

int hoefem_learned_add_pair(hoefem_learned l, const double* r, const double* e, int mem) {
  API_BEGIN
  HOEFEM_REQUIRE(l, HOEFEM_ERR_INVALID_ARGUMENT, "null handle");
  Model& mm = l->model->m;
  View R(r, mm.ndof, mem, mm.stream, true), E(e, mm.ndof, mem, mm.stream, true);
  l->l.add_pair(R.d, E.d, mm.stream);
  sync(mm);
  API_END
}

int hoefem_learned_train(hoefem_learned l, int64_t steps, int32_t batch, float lr, uint64_t seed, float* loss_history) {
  API_BEGIN
  HOEFEM_REQUIRE(l && steps >= 0 && lr >= 0.f, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  l->l.train(steps, batch, lr, seed, loss_history, l->model->m.stream);
  API_END
}

int hoefem_learned_forward_backward(hoefem_learned l, const float* X, const float* T, int32_t rows, float* loss,
                                    float* grads, float* out) {
  API_BEGIN
  HOEFEM_REQUIRE(l && X && T && rows > 0 && rows <= l->l.max_batch, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  Learned& L = l->l;
  cudaStream_t s = l->model->m.stream;
  DBuf<float> dX, dT;
  dX.upload(X, (size_t)rows * Learned::F, s);
  dT.upload(T, (size_t)rows * Learned::NM, s);
  float lv = L.train_step(dX.p, dT.p, rows, 0.f, s);
  if (loss) *loss = lv;
  if (grads) HOEFEM_CUDA(cudaMemcpyAsync(grads, L.grads.p, sizeof(float) * L.n_params, cudaMemcpyDeviceToHost, s));
  if (out) HOEFEM_CUDA(cudaMemcpyAsync(out, L.Y3.p, sizeof(float) * rows * Learned::NM, cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  API_END
}

int hoefem_learned_infer(hoefem_learned l, const float* X, int32_t rows, int32_t bf16, float* out) {
  API_BEGIN
  HOEFEM_REQUIRE(l && X && out && rows > 0 && rows <= l->l.max_batch, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  Learned& L = l->l;
  cudaStream_t s = l->model->m.stream;
  DBuf<float> dX;
  dX.upload(X, (size_t)rows * Learned::F, s);
  if (bf16) L.refresh_bf16(s);
  L.forward(dX.p, rows, bf16 != 0, s);
  HOEFEM_CUDA(cudaMemcpyAsync(out, L.Y3.p, sizeof(float) * rows * Learned::NM, cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  API_END
}

int hoefem_learned_get_weights(hoefem_learned l, float* w) {
  API_BEGIN
  HOEFEM_REQUIRE(l && w, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  cudaStream_t s = l->model->m.stream;
  HOEFEM_CUDA(cudaMemcpyAsync(w, l->l.params.p, sizeof(float) * l->l.n_params, cudaMemcpyDeviceToHost, s));
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  API_END
}

int hoefem_learned_set_weights(hoefem_learned l, const float* w) {
  API_BEGIN
  HOEFEM_REQUIRE(l && w, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  cudaStream_t s = l->model->m.stream;
  HOEFEM_CUDA(cudaMemcpyAsync(l->l.params.p, w, sizeof(float) * l->l.n_params, cudaMemcpyHostToDevice, s));
  l->l.refresh_bf16(s);
  HOEFEM_CUDA(cudaStreamSynchronize(s));
  l->l.trained = true;
  API_END
}

int hoefem_learned_predict(hoefem_learned l, const double* r, double* x0, int mem) {
  API_BEGIN
  HOEFEM_REQUIRE(l, HOEFEM_ERR_INVALID_ARGUMENT, "null handle");
  Model& mm = l->model->m;
  View R(r, mm.ndof, mem, mm.stream, true), X0(x0, mm.ndof, mem, mm.stream, false);
  if (l->l.use_bf16) l->l.refresh_bf16(mm.stream);
  l->l.predict(R.d, X0.d, mm.stream);
  X0.copy_out();
  sync(mm);
  API_END
}

int hoefem_integrator_set_learned(hoefem_integrator it, hoefem_learned l, int mode) {
  API_BEGIN
  HOEFEM_REQUIRE(it && mode >= 0 && mode <= 4, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  HOEFEM_REQUIRE(!l || l->model == it->model, HOEFEM_ERR_INVALID_ARGUMENT, "learned correction of another model");
  integrator_set_learned(it->it, l ? &l->l : nullptr, mode);
  API_END
}

// ---- batched scenes --------------------------------------------------------
int hoefem_batch_create(const hoefem_model* models, int32_t num_scenes, const hoefem_material* materials,
                        double density, const int64_t* bc_offsets, const int64_t* bc_nodes, int gravity_enabled,
                        double gravity, hoefem_batch* out) {
  API_BEGIN
  HOEFEM_REQUIRE(out && models && materials && num_scenes > 0, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  HOEFEM_REQUIRE(!bc_offsets || bc_nodes || bc_offsets[num_scenes] == 0, HOEFEM_ERR_INVALID_ARGUMENT,
                 "missing Dirichlet nodes");
  std::vector<const Model*> ms(num_scenes);
  std::vector<MatDev> mats(num_scenes);
  for (int k = 0; k < num_scenes; ++k) {
    ms[k] = &model_of(models[k]);
    mats[k] = mat_of(materials + k);
    if (bc_offsets)
      HOEFEM_REQUIRE(bc_offsets[k + 1] >= bc_offsets[k], HOEFEM_ERR_INVALID_ARGUMENT, "decreasing Dirichlet offsets");
  }
  std::unique_ptr<hoefem_batch_s> h(new hoefem_batch_s());
  h->b = batch_build(ms, mats, density, bc_offsets, bc_nodes, gravity_enabled != 0, gravity);
  *out = h.release();
  API_END
}

int hoefem_batch_destroy(hoefem_batch b) {
  API_BEGIN
  delete b;
  API_END
}

int hoefem_batch_set_stream(hoefem_batch b, void* stream) {
  API_BEGIN
  HOEFEM_REQUIRE(b, HOEFEM_ERR_INVALID_ARGUMENT, "null batch");
  Model& mm = batch_model(b->b);
  if (!b->own_stream) b->own_stream = mm.stream;
  HOEFEM_CUDA(cudaStreamSynchronize(mm.stream));
  mm.stream = stream ? (cudaStream_t)stream : b->own_stream;
  API_END
}

int hoefem_batch_set_tolerances(hoefem_batch b, double cg_tol, int64_t cg_max_iter, int64_t newton_max_iter) {
  API_BEGIN
  HOEFEM_REQUIRE(b && cg_tol >= 0.0 && newton_max_iter >= 0, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  batch_set_tolerances(b->b, cg_tol, cg_max_iter, newton_max_iter);
  API_END
}

int hoefem_batch_set_cg_engine(hoefem_batch b, int32_t engine, int32_t ctas_per_sm) {
  API_BEGIN
  HOEFEM_REQUIRE(b, HOEFEM_ERR_INVALID_ARGUMENT, "null batch");
  batch_set_cg_engine(b->b, engine, ctas_per_sm);
  API_END
}

int hoefem_batch_cg_choice(hoefem_batch b, int32_t* engine, int32_t* ctas_per_sm, float* tune_ms,
                           int32_t* num_candidates) {
  API_BEGIN
  HOEFEM_REQUIRE(b && engine && ctas_per_sm, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  int e = 0, c = 0;
  std::vector<float> t;
  batch_cg_choice(b->b, &e, &c, &t);
  *engine = e;
  *ctas_per_sm = c;
  if (num_candidates) {
    const int cap = *num_candidates;
    *num_candidates = (int32_t)t.size();
    if (tune_ms)
      for (int k = 0; k < cap && k < (int)t.size(); ++k) tune_ms[k] = t[k];
  }
  API_END
}

int hoefem_batch_sizes(hoefem_batch b, int64_t* num_scenes, int64_t* ndof, int64_t* nnz, int64_t* dof_offsets) {
  API_BEGIN
  HOEFEM_REQUIRE(b, HOEFEM_ERR_INVALID_ARGUMENT, "null batch");
  Model& mm = batch_model(b->b);
  const std::vector<int>& no = batch_node_offsets(b->b);
  if (num_scenes) *num_scenes = (int64_t)no.size() - 1;
  if (ndof) *ndof = mm.ndof;
  if (nnz) *nnz = mm.nnz;
  if (dof_offsets)
    for (size_t k = 0; k < no.size(); ++k) dof_offsets[k] = 3 * (int64_t)no[k];
  API_END
}

int hoefem_batch_step(hoefem_batch b, double* u, double* v, double t, double dt, int mem) {
  API_BEGIN
  (void)t;
  HOEFEM_REQUIRE(b && dt > 0.0, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  Model& mm = batch_model(b->b);
  View U(u, mm.ndof, mem, mm.stream, true), V(v, mm.ndof, mem, mm.stream, true);
  int st = batch_step(b->b, U.d, V.d, dt);
  U.copy_out();
  V.copy_out();
  sync(mm);
  if (st != HOEFEM_OK) return fail(st, "time step failed for at least one scene");
  API_END
}

int hoefem_batch_scene_stats(hoefem_batch b, int32_t scene, hoefem_step_stats* out, int32_t* status) {
  API_BEGIN
  HOEFEM_REQUIRE(b && out && status, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  HOEFEM_REQUIRE(scene >= 0 && scene < (int)batch_node_offsets(b->b).size() - 1, HOEFEM_ERR_INVALID_ARGUMENT,
                 "scene out of range");
  int st = 0;
  batch_scene_stats(b->b, scene, out, &st);
  *status = st;
  API_END
}

// ---- scenes ---------------------------------------------------------------------
int hoefem_scene_create_tet10_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cells_per_unit,
                                  hoefem_scene* out) {
  API_BEGIN
  HOEFEM_REQUIRE(out && unit > 0 && ux > 0 && uy > 0 && uz > 0 && cells_per_unit > 0, HOEFEM_ERR_INVALID_ARGUMENT,
                 "bad arguments");
  auto* h = new hoefem_scene_s();
  h->s = scene_tet10_box(unit, ux, uy, uz, cells_per_unit);
  *out = h;
  API_END
}

int hoefem_scene_create_hex27_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cells_per_unit,
                                  hoefem_scene* out) {
  API_BEGIN
  HOEFEM_REQUIRE(out && unit > 0 && ux > 0 && uy > 0 && uz > 0 && cells_per_unit > 0, HOEFEM_ERR_INVALID_ARGUMENT,
                 "bad arguments");
  auto* h = new hoefem_scene_s();
  h->s = scene_hex27_box(unit, ux, uy, uz, cells_per_unit);
  *out = h;
  API_END
}

int hoefem_scene_create_embedded_cylinder(int64_t n, double r_inner, double r_outer, int q_min, int q_max,
                                          uint64_t seed, hoefem_scene* out) {
  API_BEGIN
  HOEFEM_REQUIRE(out && n > 0 && r_outer > r_inner && r_inner >= 0 && q_min >= 1 && q_max >= q_min,
                 HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  auto* h = new hoefem_scene_s();
  h->s = scene_embedded_cylinder(n, r_inner, r_outer, q_min, q_max, seed);
  *out = h;
  API_END
}

int hoefem_scene_info_get(hoefem_scene s, hoefem_scene_info* info) {
  API_BEGIN
  HOEFEM_REQUIRE(s && info, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  std::memset(info, 0, sizeof(*info));
  info->num_vertices = (int64_t)s->s->X.size() / 3;
  info->num_blocks = (int64_t)s->s->blocks.size();
  for (size_t b = 0; b < s->s->blocks.size() && b < 2; ++b) {
    const SceneBlock& sb = s->s->blocks[b];
    info->block_kind[b] = sb.kind;
    info->block_elements[b] = (int64_t)sb.conn.size() / sb.nn;
    info->block_quad_points[b] = (int64_t)sb.qw.size();
    info->block_uniform[b] = sb.uniform ? 1 : 0;
  }
  info->cell_size = s->s->cell_size;
  API_END
}

int hoefem_scene_vertices(hoefem_scene s, double* vertices) {
  API_BEGIN
  HOEFEM_REQUIRE(s && vertices, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  std::memcpy(vertices, s->s->X.data(), s->s->X.size() * sizeof(double));
  API_END
}

int hoefem_scene_block(hoefem_scene s, int block, int64_t* connectivity, int64_t* quad_offsets, double* quad_weights,
                       double* quad_points) {
  API_BEGIN
  HOEFEM_REQUIRE(s && block >= 0 && block < (int)s->s->blocks.size(), HOEFEM_ERR_INVALID_ARGUMENT, "bad block");
  const SceneBlock& b = s->s->blocks[block];
  if (connectivity) std::memcpy(connectivity, b.conn.data(), b.conn.size() * sizeof(int64_t));
  if (quad_offsets && !b.uniform) std::memcpy(quad_offsets, b.qoff.data(), b.qoff.size() * sizeof(int64_t));
  if (quad_weights) std::memcpy(quad_weights, b.qw.data(), b.qw.size() * sizeof(double));
  if (quad_points) std::memcpy(quad_points, b.qp.data(), b.qp.size() * sizeof(double));
  API_END
}

int hoefem_scene_volume_fractions(hoefem_scene s, double* fractions) {
  API_BEGIN
  HOEFEM_REQUIRE(s && fractions, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  scene_volume_fractions(*s->s, fractions);
  API_END
}

int hoefem_scene_nodes_below(hoefem_scene s, int axis, double value, int64_t* nodes, int64_t* count) {
  API_BEGIN
  HOEFEM_REQUIRE(s && count && axis >= 0 && axis < 3, HOEFEM_ERR_INVALID_ARGUMENT, "bad arguments");
  int64_t k = 0;
  const int64_t nv = (int64_t)s->s->X.size() / 3;
  for (int64_t a = 0; a < nv; ++a)
    if (s->s->X[3 * a + axis] <= value) {
      if (nodes) nodes[k] = a;
      ++k;
    }
  *count = k;
  API_END
}

int hoefem_scene_destroy(hoefem_scene s) {
  API_BEGIN
  delete s;
  API_END
}

int hoefem_random_normal(uint64_t seed, int64_t n, double sigma, double* out) {
  API_BEGIN
  HOEFEM_REQUIRE(out || n == 0, HOEFEM_ERR_INVALID_ARGUMENT, "null output");
  random_normal(seed, n, sigma, out);
  API_END
}

int hoefem_tet_quadrature(int strength, double* weights, double* points, int64_t* num_points) {
  API_BEGIN
  std::vector<double> w, p;
  HOEFEM_REQUIRE(tet_quadrature(strength, w, p), HOEFEM_ERR_INVALID_ARGUMENT, "tet rule strength must be 1, 2, 3 or 5");
  if (num_points) *num_points = (int64_t)w.size();
  if (weights) std::copy(w.begin(), w.end(), weights);
  if (points) std::copy(p.begin(), p.end(), points);
  API_END
}

int hoefem_embed_mesh_3d(const double* bg_vertices, int64_t num_bg_vertices, const int64_t* bg_connectivity,
                         int64_t num_bg_cells, int bg_nodes_per_cell, const double* emb_vertices,
                         int64_t num_emb_vertices, const int64_t* emb_tets, int64_t num_emb_tets,
                         double lower_volume_threshold, double upper_volume_threshold, hoefem_embedding* out) {
  API_BEGIN
  HOEFEM_REQUIRE(out && bg_vertices && bg_connectivity && (emb_vertices || num_emb_vertices == 0) &&
                     (emb_tets || num_emb_tets == 0),
                 HOEFEM_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  *out = (hoefem_embedding)embedding_create(bg_vertices, num_bg_vertices, (const i64*)bg_connectivity, num_bg_cells,
                                            bg_nodes_per_cell, emb_vertices, num_emb_vertices, (const i64*)emb_tets,
                                            num_emb_tets, lower_volume_threshold, upper_volume_threshold);
  API_END
}

int hoefem_embedding_cells(hoefem_embedding e, int64_t* num_exterior, int64_t* num_interior, int64_t* num_interface,
                           int32_t* cell_class, double* cut_volume) {
  API_BEGIN
  HOEFEM_REQUIRE(e, HOEFEM_ERR_INVALID_ARGUMENT, "null embedding");
  embedding_cells(*(const Embedding*)e, (i64*)num_exterior, (i64*)num_interior, (i64*)num_interface, cell_class,
                  cut_volume);
  API_END
}

int hoefem_embedding_quadrature(hoefem_embedding e, const double* tet_weights, const double* tet_points,
                                int64_t tet_num_points, double stab_factor, const double* stab_weights,
                                const double* stab_points, int64_t stab_num_points, int64_t* total_points) {
  API_BEGIN
  HOEFEM_REQUIRE(e && total_points, HOEFEM_ERR_INVALID_ARGUMENT, "null argument");
  *total_points = embedding_quadrature(*(Embedding*)e, tet_weights, tet_points, tet_num_points, stab_factor,
                                       stab_weights, stab_points, stab_num_points);
  API_END
}

int hoefem_embedding_copy_quadrature(hoefem_embedding e, int64_t* offsets, double* weights, double* points) {
  API_BEGIN
  HOEFEM_REQUIRE(e && offsets && weights && points, HOEFEM_ERR_INVALID_ARGUMENT, "null argument");
  embedding_copy_quadrature(*(const Embedding*)e, (i64*)offsets, weights, points);
  API_END
}

int hoefem_embedding_destroy(hoefem_embedding e) {
  API_BEGIN
  embedding_destroy((Embedding*)e);
  API_END
}

int hoefem_quadrature_simplify(int64_t num_rules, const int64_t* offsets, const double* weights,
                               const double* points, int strength, int64_t* out_offsets, double* out_weights,
                               double* out_points) {
  API_BEGIN
  HOEFEM_REQUIRE(offsets && out_offsets && (num_rules == 0 || (weights && points && out_weights && out_points)),
                 HOEFEM_ERR_INVALID_ARGUMENT, "null argument");
  quadrature_simplify(num_rules, (const i64*)offsets, weights, points, strength, (i64*)out_offsets, out_weights,
                      out_points);
  API_END
}

}  // extern "C"
