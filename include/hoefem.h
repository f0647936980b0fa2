/*
 * hoefem.h — C ABI of the B200 (sm_100a) implementation of the per-step hot
 * path of the higher-order embedded FEM method (reference project:
 * InteractiveComputerGraphics/higher_order_embedded_fem, Rust).
 *
 * The reference exposes this path as Rust traits called by its integrator.
 * Every entry point below replaces one of those trait methods; the comment of
 * each cites the reference item (path inside the reference project : line).
 * All arithmetic is IEEE FP64 unless an entry point says otherwise.
 *
 * Conventions
 *  - Returns: every function returns a hoefem_status (0 = success).  The
 *    reference panics or returns Box<dyn Error>; this ABI never aborts.
 *  - Memory: vectors / value arrays passed to compute entry points live in the
 *    space named by the `mem` argument (HOEFEM_MEM_HOST: host memory, copied
 *    in/out inside the call; HOEFEM_MEM_DEVICE: device pointers on the current
 *    CUDA device, used in place).  Setup arrays (meshes, quadrature, patterns)
 *    are always host memory.
 *  - Indices are int64 (the reference uses usize); DOF numbering is node-major
 *    (dof = 3 * node + component), as in the reference.
 *  - Accumulation: "_into" entry points ADD into their output, like the
 *    reference's `*_into` / `*_into_par` methods.
 *  - Threading: a handle is used by one host thread at a time; calls on one
 *    handle are ordered on that handle's CUDA stream and synchronous on return.
 */
#ifndef HOEFEM_H
#define HOEFEM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HOEFEM_ABI_VERSION 1

typedef enum {
  HOEFEM_OK = 0,
  HOEFEM_ERR_INVALID_ARGUMENT = 1,
  HOEFEM_ERR_CUDA = 2,
  HOEFEM_ERR_OUT_OF_MEMORY = 3,
  /* singular reference Jacobian or deformation gradient: the reference panics
     ("Jacobian must be invertible", "TODO: Handle singular F?") */
  HOEFEM_ERR_SINGULAR = 4,
  HOEFEM_ERR_NONFINITE = 5,
  /* an element entry is missing from the CSR pattern or an element repeats a
     node (reference: "Could not find column index associated with node") */
  HOEFEM_ERR_PATTERN = 6,
  /* zero diagonal while building a preconditioner (newton_cg.rs:560-576,
     schwarz_precond.rs:203-210) */
  HOEFEM_ERR_ZERO_DIAGONAL = 7,
  HOEFEM_ERR_NOT_FINALIZED = 8,
  /* a bounded device-side wait of a persistent kernel ran out (no
     counterpart in the reference; the kernel wound down instead of spinning) */
  HOEFEM_ERR_DEVICE_TIMEOUT = 9,
  /* CG outcomes, fenris/src/cg.rs:277-286 SolveErrorKind */
  HOEFEM_CG_INDEFINITE_OPERATOR = 10,
  HOEFEM_CG_INDEFINITE_PRECONDITIONER = 11,
  HOEFEM_CG_MAX_ITERATIONS = 12,
  /* Newton / integrator outcomes, hamilton2/src/newton.rs:26-33 and
     simulation_toolbox/src/fem/newton_cg.rs:146-228 */
  HOEFEM_NEWTON_MAX_ITERATIONS = 20,
  HOEFEM_LINE_SEARCH_FAILED = 21,
  HOEFEM_SUBSTEPPING_FAILED = 22,
  HOEFEM_ERR_NO_DEVICE = 31
} hoefem_status;

typedef enum { HOEFEM_MEM_HOST = 0, HOEFEM_MEM_DEVICE = 1 } hoefem_mem;

/* Element kinds (fenris/src/element.rs: Tet10 :1790-1972, Hex27 :1244-1444). */
typedef enum { HOEFEM_ELEM_TET10 = 1, HOEFEM_ELEM_HEX27 = 3 } hoefem_element_kind;

/* Material models (fenris/src/solid/materials.rs: StVK :177-219, Stable
   Neo-Hookean :221-377).  Lame parameters are the un-reparametrised ones; the
   SNH re-parametrisation (materials.rs:242-253) happens inside the kernels. */
typedef enum { HOEFEM_MAT_STVK = 0, HOEFEM_MAT_SNH = 1 } hoefem_material_kind;

/* An ElasticMaterialModel<f64, U3> (fenris/src/solid/mod.rs:21-87) as a POD
   descriptor passed to the kernels instead of a trait object. */
typedef struct {
  int32_t kind;  /* hoefem_material_kind */
  double mu;
  double lambda;
} hoefem_material;

const char* hoefem_last_error(void);
int hoefem_abi_version(void);
/* Number of kernels this library has launched in this process (graph
   replays counted per kernel).  Instrumentation; no reference counterpart. */
int hoefem_launch_count(int64_t* count);
/* Selects the CUDA device used by handles created afterwards on this thread. */
int hoefem_set_device(int device);

/* LameParameters::from(YoungPoisson), fenris/src/solid/materials.rs:27-38.
   Reproduces the reference's lambda = 0.5*mu*nu/(1-2nu) (documented erratum,
   a factor 4 below the textbook value) so results match the reference. */
int hoefem_lame_from_young_poisson(double young, double poisson, double* mu, double* lambda);

/* ------------------------------------------------------------------------ */
/* Model: NodalModel3d (fenris/src/model.rs:32-117) / EmbeddedModel3d
   (fenris/src/embedding/mod.rs:39-59,243-283).  A model is a vertex array
   plus one or more element blocks assembled in order; each block has its own
   greedy coloring (paradis/src/coloring.rs:48-72).  A NodalModel is one block;
   an EmbeddedModel is an interior block (uniform rule) followed by an
   interface block (one rule per element). */
typedef struct hoefem_model_s* hoefem_model;

int hoefem_model_create(const double* vertices /* num_vertices x 3 */, int64_t num_vertices, hoefem_model* out);
/* connectivity: num_elements x nodes_per_element (row-major).  quadrature:
   when quad_offsets == NULL every element uses the same rule of
   num_quad_points points; otherwise element e uses points
   [quad_offsets[e], quad_offsets[e+1]) (num_elements+1 offsets).
   Weights are in reference measure (sum w |det J| = element volume). */
int hoefem_model_add_block(hoefem_model m, int element_kind, const int64_t* connectivity, int64_t num_elements,
                           const int64_t* quad_offsets, const double* quad_weights,
                           const double* quad_points /* x3 */, int64_t num_quad_points);
/* Builds the shared CSR pattern (CsrParAssembler::assemble_pattern,
   fenris/src/assembly.rs:177-249), the colorings, the element-to-nnz maps and
   uploads everything to the device. */
int hoefem_model_finalize(hoefem_model m);
int hoefem_model_destroy(hoefem_model m);
/* Runs the model's work (and that of its preconditioners / integrator) on a
   caller stream (a cudaStream_t, e.g. torch.cuda.current_stream().cuda_stream);
   NULL restores the model's own stream.  Calls stay synchronous on return.
   No counterpart in the reference (its path is synchronous host code). */
int hoefem_model_set_stream(hoefem_model m, void* stream);
/* Autotunes the lanes-per-node of the node-row SpMV kernels for this
   model's pattern (8, 16 or 32; the integrator does this at creation) and
   returns the choice.  No counterpart in the reference. */
int hoefem_model_autotune(hoefem_model m, int32_t* lanes);
/* Selects the SpMV variant explicitly: lanes per node 8, 16 or 32
   (neighbour-major), or 108, 116, 132 (the same lane counts, column-streaming
   traversal), for FP64 and FP32 values, and turns the automatic choice off.
   Otherwise hoefem_model_autotune / integrator set-up time the variants on
   the SpMV alone, and the first CG solves time candidate pairs (operator,
   Schwarz apply) chunk by chunk per value precision and keep the fastest. */
int hoefem_model_set_spmv_variant(hoefem_model m, int32_t variant);
/* The SpMV variants in use for FP64 and FP32 operator values. */
int hoefem_model_get_spmv_variants(hoefem_model m, int32_t* fp64_values, int32_t* fp32_values);
/* Element stiffness (and force) implementation.  HOEFEM_STIFFNESS_AUTO
   (default): with FP32 element arithmetic (HOEFEM_PRECISION_MIXED), Tet10
   blocks with one quadrature rule of at most 14 points run on the tensor
   cores (tcgen05 TF32 with a hi / lo split of both operands, three products;
   the element blocks of all elements as one GEMM against the block's
   reference-gradient operator); every other block runs the CUDA-core kernel
   over the whole block in one launch into staged node-pair blocks; both then
   gather the blocks into the CSR values (forces likewise, per node).
   HOEFEM_STIFFNESS_STAGED: the staged CUDA-core kernels for every block (no
   tensor cores).  HOEFEM_STIFFNESS_CUDA_CORES: one launch per element color
   with the scatter into the values (the path batched scenes always take).
   All three add the same values up to the order of the FP64 additions.  No
   counterpart in the reference. */
typedef enum {
  HOEFEM_STIFFNESS_AUTO = 0,
  HOEFEM_STIFFNESS_CUDA_CORES = 1,
  HOEFEM_STIFFNESS_STAGED = 2
} hoefem_stiffness_path;
int hoefem_model_set_stiffness_path(hoefem_model m, int path);
int hoefem_model_sizes(hoefem_model m, int64_t* ndof, int64_t* nnz, int64_t* num_elements, int64_t* num_blocks);
/* row_offsets: ndof+1, column_indices: nnz (SparsityPattern, sparse.rs:297-410) */
int hoefem_model_pattern(hoefem_model m, int64_t* row_offsets, int64_t* column_indices);
int hoefem_model_num_colors(hoefem_model m, int block, int64_t* num_colors);
/* DisjointSubsets labels per color (paradis/src/lib.rs:78-190): color_offsets
   has num_colors+1 entries, element_labels are block-local element indices. */
int hoefem_model_colors(hoefem_model m, int block, int64_t* color_offsets, int64_t* element_labels);

/* ElasticityModelParallel::assemble_elastic_pseudo_forces_into_par
   (fenris/src/solid/mod.rs:129-134; impls solid/impl_model.rs:111-127,
   embedding/mod.rs:516-554): f += f_int(u), f_e = -sum_q P J^-T grad N w|det J|. */
int hoefem_assemble_elastic_pseudo_forces_into(hoefem_model m, const hoefem_material* mat, const double* u, double* f,
                                               int mem);
/* ElasticityModelParallel::assemble_stiffness_into_par
   (fenris/src/solid/mod.rs:144-151, assembly.rs:252-314): values += K(u) on the
   model pattern; colored scatter without atomics, one launch per color. */
int hoefem_assemble_stiffness_into(hoefem_model m, const hoefem_material* mat, const double* u, double* values,
                                   int mem);
/* hoefem_assemble_stiffness_into with the element arithmetic in the given
   precision (HOEFEM_PRECISION_MIXED: FP32 kinematics, material tangent and
   pair contractions; the CSR values are accumulated in FP64).  No counterpart
   in the reference (its stiffness is FP64). */
int hoefem_assemble_stiffness_into_precision(hoefem_model m, const hoefem_material* mat, const double* u,
                                             double* values, int precision, int mem);
/* ElasticityModel::assemble_mass(density).to_csr (solid/mod.rs:106,
   assembly.rs:624-671): values += M on the model pattern. */
/* assemble_transformed_stiffness_into_par with DefaultSemidefiniteProjection
   (fenris/src/assembly.rs:549-564; compute_stiffness_matrix_into with
   projected = true, simulation_toolbox/src/fem/system_assembly.rs:107-142):
   every element matrix is eigen-decomposed and its negative eigenvalues set
   to zero before the colored scatter.  Adds into values. */
int hoefem_assemble_projected_stiffness_into(hoefem_model m, const hoefem_material* mat, const double* u,
                                             double* values, int mem);
int hoefem_assemble_mass_into(hoefem_model m, double density, double* values, int mem);
/* apply_homogeneous_dirichlet_bc_csr (fenris/src/assembly.rs:799-869) on
   values of the model pattern; nodes are host indices. */
int hoefem_apply_dirichlet_bc_csr(hoefem_model m, const int64_t* nodes, int64_t num_nodes, double* values, int mem);
/* compute_jacobian_combination_into (simulation_toolbox/src/fem/
   system_assembly.rs:196-235) without damping: out = (0 + c_k K) + c_m M,
   then Dirichlet rows/columns. */
int hoefem_jacobian_combination(hoefem_model m, double c_stiffness, const double* stiffness_values, double c_mass,
                                const double* mass_values, const int64_t* bc_nodes, int64_t num_bc, double* out,
                                int mem);
/* hoefem_jacobian_combination without any device allocation.  No counterpart
   in the reference: for callers that cannot allocate device memory while
   they step (a host that reserves its device memory budget up front, or a
   real-time loop that must not wait on the allocator).  stiffness_values /
   mass_values (either may be NULL) and out are device pointers on the
   model's device (nnz each); bc_nodes is a host array.  The call runs on the
   model's device and restores the caller's current device on return.  Scratch (the
   Dirichlet DOF mask, the node list and the diagonal-scale word) is a fixed
   array inside the library, one per device, sized for at most 4,194,304 DOFs
   and 262,144 Dirichlet nodes; larger inputs return
   HOEFEM_ERR_INVALID_ARGUMENT.  The mask is cleared on every call.  The
   model must already be resident on the device (any compute entry point
   puts it there).  The first call on each device looks up the scratch
   address (cudaGetSymbolAddress) and should come before any stream capture.
   All calls on one device share the one scratch: calls that overlap in time
   (other threads or streams) race and must be serialised by the caller.
   Synchronous on return, like every entry point. */
int hoefem_jacobian_combination_noalloc(hoefem_model m, double c_stiffness, const double* stiffness_values,
                                        double c_mass, const double* mass_values, const int64_t* bc_nodes,
                                        int64_t num_bc, double* out);
/* compute_jacobian_combination_into with a damping matrix
   (system_assembly.rs:196-235): out = c_stiffness K + c_damping D + c_mass M
   (summed in that order; any array may be NULL), then Dirichlet as above. */
int hoefem_jacobian_combination_damped(hoefem_model m, double c_stiffness, const double* stiffness_values,
                                       double c_damping, const double* damping_values, double c_mass,
                                       const double* mass_values, const int64_t* bc_nodes, int64_t num_bc,
                                       double* out, int mem);
/* spmv_csr (fenris/src/sparse.rs:1164-1199) / LinearOperator::apply for the
   model pattern (cg.rs:15-17): y = beta*y + alpha*A x. */
int hoefem_spmv(hoefem_model m, double beta, double* y, double alpha, const double* values, const double* x, int mem);

/* ------------------------------------------------------------------------ */
/* SystemPreconditioner (simulation_toolbox/src/fem/newton_cg.rs:397-411). */
typedef struct hoefem_precond_s* hoefem_precond;

/* DiagonalPreconditioner (newton_cg.rs:534-593). */
int hoefem_precond_create_diagonal(hoefem_model m, hoefem_precond* out);
/* SchwarzPreconditioner (newton_cg.rs:297-370; schwarz_precond.rs:26-216):
   one subdomain per node list (the reference uses the interface elements whose
   embedded volume fraction is below a threshold), scalar Jacobi for untreated
   nodes.  Builds build_preconditioner_pattern (schwarz_precond.rs:134-169). */
int hoefem_precond_create_schwarz(hoefem_model m, const int64_t* subdomain_offsets, const int64_t* subdomain_nodes,
                                  int64_t num_subdomains, const int64_t* untreated_nodes, int64_t num_untreated,
                                  hoefem_precond* out);
/* SystemPreconditioner::update (newton_cg.rs:352-365 / 556-571): system values
   on the model pattern. */
int hoefem_precond_update(hoefem_precond p, const double* system_values, int mem);
/* LinearOperator::apply of the preconditioner: z = P r. */
int hoefem_precond_apply(hoefem_precond p, const double* r, double* z, int mem);
/* Schwarz pattern / values for inspection (nnz first, then the arrays). */
int hoefem_precond_nnz(hoefem_precond p, int64_t* nnz);
/* How the CG applies a Schwarz preconditioner (no reference counterpart; the
   reference applies the assembled CSR matrix with MKL): on (default) = the
   symmetrized inverted subdomain blocks as dense products, summed per node in
   subdomain order; off = SpMV over the assembled values.  Both are P r; they
   differ only in rounding.  hoefem_precond_apply always uses the CSR. */
int hoefem_precond_set_block_apply(hoefem_precond p, int32_t on);
/* SpMV variant of the Schwarz apply (as hoefem_model_set_spmv_variant);
   chosen by the autotuner at creation and by the CG's online choice
   otherwise. */
int hoefem_precond_set_spmv_variant(hoefem_precond p, int32_t variant);
int hoefem_precond_get_spmv_variants(hoefem_precond p, int32_t* fp64_values, int32_t* fp32_values);
int hoefem_precond_pattern(hoefem_precond p, int64_t* row_offsets, int64_t* column_indices);
int hoefem_precond_values(hoefem_precond p, double* values /* host */);
int hoefem_precond_destroy(hoefem_precond p);

/* ------------------------------------------------------------------------ */
/* ConjugateGradient::solve_with_guess (fenris/src/cg.rs:368-482) with a
   RelativeResidualCriterion (cg.rs:77-124): stops when ||r|| <= tol ||b||.
   x holds the initial guess on entry.  p == NULL means no preconditioner.
   Returns HOEFEM_OK or one of the HOEFEM_CG_* outcomes; *iterations is always
   written (CgOutput::num_iterations). */
int hoefem_cg_solve(hoefem_model m, const double* system_values, hoefem_precond p, const double* b, double* x,
                    double tol, int64_t max_iter, int64_t* iterations, int mem);

/* Mixed-precision variant of hoefem_cg_solve: PCG with FP32 operator values
   (converted from system_values) and, for a Schwarz preconditioner, FP32
   preconditioner values; vectors, dot products and residual updates FP64.
   The recurrence residual is replaced by the true FP64 residual b - A x
   (reliable update) whenever it has dropped by the factor `delta` (0 < delta
   < 1) since the last replacement, and before the solve stops, so
   ||b - A x|| <= tol ||b|| holds in FP64.  Each replacement costs an FP64
   operator product and a preconditioner apply (and, on the streamed engine, a
   new launch): on the benchmark cylinder delta = 1e-3 needs 3 launches per
   solve instead of 7 at 0.1, with the same iteration count.  No counterpart
   in the reference. */
int hoefem_cg_solve_mixed(hoefem_model m, const double* system_values, hoefem_precond p, const double* b, double* x,
                          double tol, int64_t max_iter, double delta, int64_t* iterations, int mem);

/* ------------------------------------------------------------------------ */
/* NewtonCgIntegrator3d (simulation_toolbox/src/fem/newton_cg.rs:43-295):
   backward Euler (hamilton2/src/integrators/euler.rs:155-199) solved by
   Newton with backtracking line search (hamilton2/src/newton.rs:76-248), the
   Jacobian M + dt^2 K solved by preconditioned CG; failures retried with
   5x substeps up to 1000.  Homogeneous Dirichlet nodes (u = v = 0), scalar
   gravity on the last component (system_assembly.rs:30-75), no damping. */
typedef struct hoefem_integrator_s* hoefem_integrator;

typedef struct {
  int64_t newton_iterations;     /* of the last backward Euler solve */
  int64_t num_cg_solves;         /* over all substeps */
  int64_t total_cg_iterations;
  int64_t max_cg_iterations;
  int64_t substeps;
  int32_t last_cg_status;
  double residual_norm;          /* ||F(w)|| at exit */
  double representative_force;   /* fe_model.rs:423-431 */
  double ms_assemble_forces;     /* device time per phase, last step */
  double ms_assemble_stiffness;
  double ms_precond_update;
  double ms_cg;
  double ms_total;
  /* learned coarse correction: warm starts accepted / rejected by the
     residual guard, and the mean ||b - A x0|| / ||b|| of the accepted ones */
  int64_t learned_accepted;
  int64_t learned_rejected;
  double learned_residual_ratio;
  double ms_learned;
  /* backtracking line search (newton.rs:171-248): reductions of alpha below 1
     over all Newton iterations and substep attempts of the step */
  int64_t line_search_backtracks;
} hoefem_step_stats;

/* precond: a preconditioner of this model (ownership stays with the caller),
   or NULL for the diagonal preconditioner.  The mass matrix (with Dirichlet),
   representative force and gravity force are built here (fe_model.rs:489-515). */
int hoefem_integrator_create(hoefem_model m, const hoefem_material* mat, double density, const int64_t* bc_nodes,
                             int64_t num_bc, int gravity_enabled, double gravity, hoefem_precond precond,
                             hoefem_integrator* out);
/* Defaults follow the reference: cg_tol 1e-5, cg_max_iter 500,
   newton_max_iter 100 (newton_cg.rs:282-286,761-773). */
int hoefem_integrator_set_tolerances(hoefem_integrator it, double cg_tol, int64_t cg_max_iter,
                                     int64_t newton_max_iter);
/* Rayleigh damping of the material (MaterialComponent mass / stiffness
   damping coefficients, newton_cg.rs:90-100): at the start of every
   (sub)step D = mass_coeff M + stiffness_coeff K_proj(u) with the element-wise
   PSD-projected stiffness (compute_damping_matrix_into,
   system_assembly.rs:145-193); f gains -D v and the Jacobian dt D.  has_* = 0
   is the reference's None.  Default: no damping. */
int hoefem_integrator_set_damping(hoefem_integrator it, int has_mass, double mass_coeff, int has_stiffness,
                                  double stiffness_coeff);
/* Arithmetic of the step.  HOEFEM_PRECISION_FP64: the reference's FP64
   everywhere.  HOEFEM_PRECISION_MIXED: element stiffness arithmetic in FP32
   (CSR accumulation FP64), Schwarz blocks built in FP64 and applied in FP32,
   and the Jacobian solve as hoefem_cg_solve_mixed (FP32 operator /
   preconditioner values, FP64 vectors, reliable updates with threshold
   `delta`, stop at ||b - A x|| <= cg_tol ||b|| in FP64).  Forces, the Newton
   residual and the line search stay FP64.  No counterpart in the reference
   (an addition on top of its FP64 path). */
typedef enum { HOEFEM_PRECISION_FP64 = 0, HOEFEM_PRECISION_MIXED = 1 } hoefem_precision;
int hoefem_integrator_set_precision(hoefem_integrator it, int precision, double delta);
/* CG engine of the integrator's Jacobian solves and of hoefem_cg_solve /
   hoefem_cg_solve_mixed on a model (no counterpart in the reference, whose CG
   is one host loop).  Two engines run the same recurrence: CUDA graphs of
   kernel chunks, and the persistent streamed CG (one cooperative launch per
   solve, the operator and the Schwarz blocks streamed through shared memory;
   for no preconditioner, diagonal, or Schwarz with subdomains of at most 27
   nodes).  HOEFEM_CG_ENGINE_AUTO (default): models with fewer than 32,768
   nodes use the graphs; for larger ones, per operator precision and
   preconditioner kind, each engine's first solve sets it up (graphs, stream
   layouts) and its next solve of at least 20 iterations is timed whole
   (the solve's set-up, value packing, residual replacements and launches
   included); the engine with the lower time per iteration is kept; HOEFEM_CG_ENGINE_CHUNKED:
   always the graphs; HOEFEM_CG_ENGINE_STREAMED: the streamed CG or
   HOEFEM_ERR_INVALID_ARGUMENT.  options (bit mask):
   HOEFEM_CG_SCHWARZ_FP16: in the mixed-precision form the streamed CG keeps
   the Schwarz blocks in FP16 scaled by each block's largest magnitude;
   HOEFEM_CG_PHASE_PROFILE: the streamed CG records per-phase cycle counts
   (hoefem_cg_engine_stats.phase_us).  In the mixed-precision form the
   streamed CG multiplies the FP32 (or FP16) operator and Schwarz values with
   an FP32 copy of the direction / residual and sums a row's products in FP32;
   the vectors, the dot products and the CG recurrence stay FP64. */
typedef enum {
  HOEFEM_CG_ENGINE_AUTO = 0,
  HOEFEM_CG_ENGINE_CHUNKED = 1,
  HOEFEM_CG_ENGINE_STREAMED = 2
} hoefem_cg_engine;
enum { HOEFEM_CG_SCHWARZ_FP16 = 1, HOEFEM_CG_PHASE_PROFILE = 2 };
int hoefem_integrator_set_cg_engine(hoefem_integrator it, int engine, int options);
int hoefem_model_set_cg_engine(hoefem_model m, int engine, int options);
/* Streamed-CG counters of the last step (integrator) or solve (model):
   persistent launches, iterations they ran, their summed device time (ms) and
   the bytes one iteration streams (operator tiles + Schwarz chunks); with
   HOEFEM_CG_PHASE_PROFILE, microseconds per iteration (mean over CTAs) of:
   [0] operator halo gather, [1] operator tiles, [2] of which waiting for
   tile data, [3] CTA + grid barrier after the operator, [4] Schwarz residual
   gather, [5] Schwarz chunks, [6] of which waiting for chunk data, [7] grid
   barrier after the Schwarz products, [8] own-DOF update, [9] grid barrier
   and reductions after it, [10] producer waiting for free stages, [11]
   producer lifetime.  Automatic engine choice for the last solve's operator
   precision and preconditioner kind: the sampled whole-solve microseconds per
   iteration of the chunked and the streamed engine (0 until sampled) and the choice
   (-1 undecided, 0 chunked, 1 streamed).  With the phase profile also the
   largest value of each phase over the CTAs, and the mean and largest time per
   iteration a CTA spends outside the grid barriers ([0] + [1] + [4] + [5] +
   [8]): their ratio is the load imbalance the barriers wait for. */
typedef struct {
  int64_t launches, iterations;
  double device_ms;
  int64_t operator_bytes, schwarz_bytes;
  double phase_us[12];
  double auto_us_per_iteration[2];
  int32_t auto_choice;
  double phase_us_max[12];
  double busy_us[2];
} hoefem_cg_engine_stats;
int hoefem_integrator_cg_engine_stats(hoefem_integrator it, hoefem_cg_engine_stats* out);
int hoefem_model_cg_engine_stats(hoefem_model m, hoefem_cg_engine_stats* out);
/* L2 residency budget of the streamed CG (no counterpart in the reference):
   bytes of each iteration's stream (over all CTAs; the Schwarz chunks first,
   then operator tiles) copied with an evict-last L2 policy so that they are
   still cached in the next iteration, the rest with evict-first.  bytes < 0:
   the default, 0 (on the benchmark cylinder every kept budget measured
   slower than streaming everything). */
int hoefem_integrator_set_cg_l2_keep(hoefem_integrator it, int64_t bytes);
int hoefem_model_set_cg_l2_keep(hoefem_model m, int64_t bytes);
/* One time step: u, v (ndof) updated in place. */
int hoefem_integrator_step(hoefem_integrator it, double* u, double* v, double t, double dt, int mem);
int hoefem_integrator_stats(hoefem_integrator it, hoefem_step_stats* out);
/* Mass matrix values (model pattern, Dirichlet applied) for inspection. */
int hoefem_integrator_mass(hoefem_integrator it, double* values /* host */);
/* NewtonCgDynamicSystem::eval_f (newton_cg.rs:441-478): f = M g + f_int(u)
   with Dirichlet rows zeroed. */
int hoefem_integrator_eval_f(hoefem_integrator it, const double* u, const double* v, double* f, int mem);
int hoefem_integrator_destroy(hoefem_integrator it);

/* ------------------------------------------------------------------------ */
/* Learned coarse correction (no counterpart in the reference: an addition on
   top of its plain Schwarz-CG).  The nodes are split into num_subdomains
   coarse subdomains (recursive coordinate bisection, power of two), each with
   32 orthonormal local polynomial modes; an MLP 64 -> 256 -> 256 -> 32 maps
   per-subdomain residual features to the coarse coefficients of the converged
   correction.  Trained with the library's own forward / backward / Adam
   kernels on (residual, converged correction) pairs that plain Schwarz-CG
   solves generate; inference in BF16 on the tensor cores.  In an integrator
   it is a warm start that is kept only if it lowers the residual. */
typedef struct hoefem_learned_s* hoefem_learned;

int hoefem_learned_create(hoefem_model m, const int64_t* bc_nodes, int64_t num_bc, int num_subdomains,
                          uint64_t seed, hoefem_learned* out);
int hoefem_learned_destroy(hoefem_learned l);
int hoefem_learned_num_pairs(hoefem_learned l, int64_t* num_pairs);
int hoefem_learned_num_params(hoefem_learned l, int64_t* num_params);
/* Adds the pairs (features(r), coarse coefficients of e) for one residual r
   and its correction e (device or host vectors, ndof each). */
int hoefem_learned_add_pair(hoefem_learned l, const double* r, const double* e, int mem);
/* steps of Adam on random mini-batches of `batch` pairs (FP32 master weights);
   loss_history (host, may be NULL) receives the mean squared error per step. */
int hoefem_learned_train(hoefem_learned l, int64_t steps, int32_t batch, float lr, uint64_t seed,
                         float* loss_history);
/* Host buffers: X rows x 64 features, T rows x 32 targets; outputs the MSE
   loss, the gradient of every parameter (num_params, same layout as the
   weights) and the network output (rows x 32), with no update. */
int hoefem_learned_forward_backward(hoefem_learned l, const float* X, const float* T, int32_t rows, float* loss,
                                    float* grads, float* out);
/* Inference on host features X (rows x 64, rows % 16 == 0 for bf16). */
int hoefem_learned_infer(hoefem_learned l, const float* X, int32_t rows, int32_t bf16, float* out);
int hoefem_learned_get_weights(hoefem_learned l, float* w);
int hoefem_learned_set_weights(hoefem_learned l, const float* w);
/* x0 = predicted correction of residual r. */
int hoefem_learned_predict(hoefem_learned l, const double* r, double* x0, int mem);
/* mode 0: off, 1: warm start with the guard, 2: collect training pairs from
   the integrator's plain FP64 CG solves (right-hand side b with the converged
   solution), 3: as 2 plus every CG chunk's iterate (r_k, x* - x_k), 4:
   two-level preconditioner beside the Schwarz (or diagonal) one in the FP64
   Jacobian solves: flexible PCG with z = P r + c(r), the network's coarse
   correction c(r) of every iteration's residual kept only when c.r > 0
   (hoefem_step_stats.learned_accepted / learned_rejected count the
   iterations with and without it). */
int hoefem_integrator_set_learned(hoefem_integrator it, hoefem_learned l, int mode);

/* ------------------------------------------------------------------------ */
/* Batched steps of many independent scenes (no counterpart in the reference,
   whose integrator advances one model at a time: an addition for throughput
   on small scenes).  Each scene takes the path of hoefem_integrator_step with
   the diagonal preconditioner (newton_cg.rs:131-295): its own Dirichlet
   scale, representative force, Newton tolerance, CG scalars, line search and
   substepping.  All scenes share every kernel launch: the scenes' elements
   are merged per element kind (per-element Lame parameters), colored once
   (each scene keeps its own greedy coloring) and the CG iterations of all
   scenes run together with per-scene stopping tests, in CUDA-graph chunks or
   in one persistent launch per solve (hoefem_batch_set_cg_engine).
   models: num_scenes models (not necessarily finalized; their vertices,
   blocks and quadrature are copied); materials: one per scene, all of one
   kind; bc_offsets (num_scenes+1) / bc_nodes: Dirichlet nodes per scene, local
   node numbers (both NULL for none).  The batch's DOF vector is the scenes'
   DOF vectors concatenated in order (hoefem_batch_sizes gives the offsets). */
typedef struct hoefem_batch_s* hoefem_batch;

int hoefem_batch_create(const hoefem_model* models, int32_t num_scenes, const hoefem_material* materials,
                        double density, const int64_t* bc_offsets, const int64_t* bc_nodes, int gravity_enabled,
                        double gravity, hoefem_batch* out);
int hoefem_batch_destroy(hoefem_batch b);
int hoefem_batch_set_stream(hoefem_batch b, void* stream);
/* Defaults as hoefem_integrator_set_tolerances: 1e-5, 500, 100. */
int hoefem_batch_set_tolerances(hoefem_batch b, double cg_tol, int64_t cg_max_iter, int64_t newton_max_iter);
/* CG engine of the batch (no counterpart in the reference).
   HOEFEM_CG_ENGINE_CHUNKED: CUDA graphs of 8 iterations of per-phase kernels
   (one CTA per 256-node chunk), the host reads the scene states between
   graphs.  HOEFEM_CG_ENGINE_STREAMED: one persistent cooperative launch per
   solve runs every iteration of every scene (grid barriers with bounded waits;
   a wait that runs out gives HOEFEM_ERR_DEVICE_TIMEOUT) with ctas_per_sm CTAs
   per multiprocessor (0: as many as fit).  HOEFEM_CG_ENGINE_AUTO (default):
   the autotuner runs the first solve once per candidate (the graphs, then the
   persistent launch at 1, 2, 4, ... CTAs per multiprocessor) and keeps the
   fastest.  All engines give bitwise the same results. */
int hoefem_batch_set_cg_engine(hoefem_batch b, int32_t engine, int32_t ctas_per_sm);
/* The engine in use (HOEFEM_CG_ENGINE_AUTO while the autotuner has not run
   yet) and its CTAs per multiprocessor; tune_ms (capacity *num_candidates,
   may be NULL) receives the autotuner's time per candidate in the order above,
   *num_candidates their number (0 before tuning). */
int hoefem_batch_cg_choice(hoefem_batch b, int32_t* engine, int32_t* ctas_per_sm, float* tune_ms,
                           int32_t* num_candidates);
/* dof_offsets: num_scenes+1 (may be NULL). */
int hoefem_batch_sizes(hoefem_batch b, int64_t* num_scenes, int64_t* ndof, int64_t* nnz, int64_t* dof_offsets);
/* One time step of every scene; u, v (total ndof) updated in place for every
   scene that succeeded.  Returns the status of a failed scene if any failed
   (the others are still advanced); per-scene status via scene_stats. */
int hoefem_batch_step(hoefem_batch b, double* u, double* v, double t, double dt, int mem);
int hoefem_batch_scene_stats(hoefem_batch b, int32_t scene, hoefem_step_stats* out, int32_t* status);

/* ------------------------------------------------------------------------ */
/* Synthetic scenes (input construction; not part of the reference hot path).
   Restates the reference's procedural meshes and refinements:
   create_rectangular_uniform_hex_mesh (fenris/src/geometry/procedural.rs:
   191-250), Max triangulation (geometry/polymesh.rs:402-500) + Tet4
   conversion (mesh_convert.rs:639-727) + Tet10 / Hex27 refinement
   (mesh_convert.rs:41-75,163-244,296-406), keep_cells (mesh.rs:321-366). */
typedef struct hoefem_scene_s* hoefem_scene;

/* Box [0, unit*ux] x [0, unit*uy] x [0, unit*uz], cells_per_unit cells per unit,
   each hex split into 6 Tet10; one uniform block with tet_quadrature_strength_5. */
int hoefem_scene_create_tet10_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cells_per_unit,
                                  hoefem_scene* out);
/* The same box as Hex27 elements (no clipping); one uniform block with
   hex_quadrature_strength_5. */
int hoefem_scene_create_hex27_box(double unit, int64_t ux, int64_t uy, int64_t uz, int64_t cells_per_unit,
                                  hoefem_scene* out);
/* Unit-box Hex27 grid (n^3 cells) clipped to the hollow cylinder with axis z
   through (0.5, 0.5), radii [r_inner, r_outer], full height.  Cells with volume
   fraction < 1e-4 are removed, >= 0.999 are interior (hex_quadrature_strength_5),
   the rest are interface cells with Q ~ U{q_min..q_max} seeded uniform points
   and Dirichlet(1) weights summing to 8*phi (reference measure). */
int hoefem_scene_create_embedded_cylinder(int64_t n, double r_inner, double r_outer, int q_min, int q_max,
                                          uint64_t seed, hoefem_scene* out);

typedef struct {
  int64_t num_vertices;
  int64_t num_blocks;
  int32_t block_kind[2];
  int64_t block_elements[2];
  int64_t block_quad_points[2]; /* total points stored for the block */
  int32_t block_uniform[2];     /* 1: one rule for all elements */
  double cell_size;
} hoefem_scene_info;

int hoefem_scene_info_get(hoefem_scene s, hoefem_scene_info* info);
int hoefem_scene_vertices(hoefem_scene s, double* vertices);
/* quad_offsets is written only for non-uniform blocks (num_elements+1). */
int hoefem_scene_block(hoefem_scene s, int block, int64_t* connectivity, int64_t* quad_offsets, double* quad_weights,
                       double* quad_points);
/* Volume fraction of each interface element from its quadrature
   (schwarz_precond.rs:65-127): sum_q w |det J| / cell volume. */
int hoefem_scene_volume_fractions(hoefem_scene s, double* fractions /* interface elements */);
/* Nodes with coordinate `axis` <= value (sorted ascending); count first with nodes == NULL. */
int hoefem_scene_nodes_below(hoefem_scene s, int axis, double value, int64_t* nodes, int64_t* count);
int hoefem_scene_destroy(hoefem_scene s);

/* Seeded N(0, sigma^2) samples (splitmix64 + Box-Muller), identical on all hosts. */
int hoefem_random_normal(uint64_t seed, int64_t n, double sigma, double* out);

/* tet_quadrature_strength_{1,2,3,5} (fenris/src/quadrature.rs:570-781) on the
   [-1,1]^3 corner simplex: query the count with weights == NULL. */
int hoefem_tet_quadrature(int strength, double* weights, double* points, int64_t* num_points);

/* ---- embedded quadrature construction (host arrays; computed on the device) ----
   embed_mesh_3d_with_opts (fenris/src/embedding/embedding3d.rs:57-196): every
   background cell (Hex8 or Hex27 connectivity, the first 8 nodes its corners,
   planar faces) is intersected with the embedded Tet4 mesh and classified by
   the intersection volume V against its own volume Vc: exterior if
   V < lower Vc, interface if V < upper Vc, interior otherwise (EmbedOptions
   defaults 1e-4 / 0.999).  Errors: HOEFEM_ERR_INVALID_ARGUMENT (indices out of
   range, degenerate input), HOEFEM_ERR_NO_DEVICE. */
typedef struct hoefem_embedding_s* hoefem_embedding;
int hoefem_embed_mesh_3d(const double* bg_vertices, int64_t num_bg_vertices, const int64_t* bg_connectivity,
                         int64_t num_bg_cells, int bg_nodes_per_cell, const double* emb_vertices,
                         int64_t num_emb_vertices, const int64_t* emb_tets, int64_t num_emb_tets,
                         double lower_volume_threshold, double upper_volume_threshold, hoefem_embedding* out);
/* Cell counts; cell_class (0 exterior, 1 interior, 2 interface) and the
   intersection volume per background cell (either may be NULL). */
int hoefem_embedding_cells(hoefem_embedding e, int64_t* num_exterior, int64_t* num_interior, int64_t* num_interface,
                           int32_t* cell_class, double* cut_volume);
/* compute_interface_quadrature_rules / compute_element_embedded_quadrature
   (embedding3d.rs:233-289,355-397): the tet rule on every tetrahedron of each
   interface cell's cut polyhedron, mapped to the background element's
   reference coordinates (w |det J_tet| / |det J_bg|), plus optional
   stabilization (stab_factor x the stabilization rule, StabilizationOptions).
   Interface cells in cell order; returns the total point count. */
int hoefem_embedding_quadrature(hoefem_embedding e, const double* tet_weights, const double* tet_points,
                                int64_t tet_num_points, double stab_factor, const double* stab_weights,
                                const double* stab_points, int64_t stab_num_points, int64_t* total_points);
/* The rules of the last hoefem_embedding_quadrature: offsets (num_interface + 1),
   weights (total), points (total x 3). */
int hoefem_embedding_copy_quadrature(hoefem_embedding e, int64_t* offsets, double* weights, double* points);
int hoefem_embedding_destroy(hoefem_embedding e);
/* simplify_quadrature / optimize_quadrature
   (fenris/src/embedding/quadrature_reduction.rs:107-260): every rule with more
   points than the number r of Chebyshev moments up to `strength` (0..5) is
   reduced to at most r of its points with non-negative weights and the same
   moments.  Outputs use the offsets layout and fit in input-sized buffers. */
int hoefem_quadrature_simplify(int64_t num_rules, const int64_t* offsets, const double* weights,
                               const double* points, int strength, int64_t* out_offsets, double* out_weights,
                               double* out_points);

#ifdef __cplusplus
}
#endif
#endif /* HOEFEM_H */
