/*
 * apf_b200.h — C ABI of libapf_b200, the B200 (sm_100a) implementation of the
 * data-parallel core of one adaptive cycle of the space-time parabolic FEM of
 * Rsmeets99/DoubleAdapParabolicFEM.
 *
 * Plain C: pointers, sizes and int32 status codes (APF_OK == 0; negative on error,
 * message via apf_ctx_last_error).  No call aborts and no device code traps.
 * One context per host thread; a context is not thread-safe.
 *
 * Each entry point names the reference interface it replaces (paths relative to
 * the reference project root).
 */
#ifndef APF_B200_H
#define APF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------- */
#define APF_OK 0
#define APF_ERR_INVALID (-1)       /* bad argument / inconsistent sizes */
#define APF_ERR_CUDA (-2)          /* CUDA runtime error */
#define APF_ERR_CAPACITY (-3)      /* a per-row candidate buffer overflowed */
#define APF_ERR_NUMERIC (-4)       /* non-positive diagonal, breakdown, non-finite value */
#define APF_ERR_NOT_CONVERGED (-5) /* iterative solve missed its tolerance */
#define APF_ERR_NO_DEVICE (-6)     /* no CUDA device */
#define APF_ERR_INTERNAL (-7)

/* ---- initial data u0 of the examples (algorithm/examples/space_time_2d/initial_data_2d_examples.hpp,
 *      algorithm/examples/space_time_1d/initial_data_1d_examples.hpp) */
#define APF_U0_SIN_SIN 0 /* smooth_initial: sin(pi x) sin(pi y) in 2+1D, sin(pi x) in 1+1D */
#define APF_U0_ONE 1     /* non_matching_initial: 1 */
#define APF_U0_ZERO 2

/* ---- blocks of an assembled system ---------------------------------------- */
#define APF_BLOCK_A_Y 0  /* A_y   (n_lambda x n_lambda) */
#define APF_BLOCK_B 1    /* B     (n_u x n_lambda), lower-left orientation */
#define APF_BLOCK_BT 2   /* B^T   (n_lambda x n_u) == CSC arrays of B */
#define APF_BLOCK_C 3    /* C_signed (n_u x n_u) */
#define APF_BLOCK_K 4    /* K = [A_y B^T; B C_signed] ((n_lambda+n_u)^2) */
#define APF_BLOCK_HHAT 5 /* parabolic graph-norm Schur approximation (n_u x n_u) */
#define APF_BLOCK_BDT 6  /* time-derivative part of B (n_u x n_lambda) */
#define APF_BLOCK_AX 7   /* X-space spatial stiffness (n_u x n_u) */
#define APF_N_BLOCKS 8

#define APF_VEC_F 0 /* lambda right-hand side (n_lambda) */
#define APF_VEC_G 1 /* u right-hand side (n_u) */

typedef struct apf_ctx apf_ctx;
typedef struct apf_system apf_system;

/* Space-time mesh, DOF maps and coefficients: the host-side inputs of
 * finite_element::system::assemble_main_system_blocks
 * (src/finite_element/system/assemble_saddle_problem.hpp:131-364) for 2+1D tensor
 * P_p x P_p Lagrange prisms, p in {1,2}.
 *
 * Cells are affine prisms; geometry row = x0 y0 x1 y1 x2 y2 t0 t1 (the reference
 * cell's vertex order, src/finite_element/geometry/cell_geometry.hpp:188-242).
 * Restrictions are the flattened CellRestriction of
 * src/finite_element/assembly/constrained_dofs.hpp:37-226: local row (cell c,
 * local i) owns entries [offsets[c*ndof+i], offsets[c*ndof+i+1]) of (dofs,
 * weights); ndof = (p+1)(p+2)/2 * (p+1); local index = i_space*(p+1) + i_time
 * (src/finite_element/basis/functions/triangular_prism_lagrange.hpp:27-30).
 * The diffusion tensor and the load are constant per Y cell.
 *
 * dim_space = 1 selects the 1+1D path (P1 only, tensor P1 x P1 Lagrange quadrilaterals,
 * the reference's generic assembly branch with the local forms of
 * src/finite_element/assembly/detail/local_bilinear_forms.hpp:24-81,
 * local_mixed_bilinear_forms.hpp:15-153 and local_trace_bilinear_forms.hpp:20-49, Gauss
 * orders QSpace = QTime = 3): geometry row = x0 x1 t0 t1 (spatial vertices 0 and 1,
 * temporal vertices 0 and 1), ndof = 4 with local index = i_space*2 + i_time
 * (src/finite_element/tables/quadrilateral_basis_tables.hpp:33-35), m_cells one scalar per
 * Y cell.  dim_space = 0 or 2 is the 2+1D path. */
typedef struct apf_problem_desc
{
    int p;
    int n_y_cells;
    int n_x_cells;
    int n_lambda; /* true DOFs of the test space Y (broken in time) */
    int n_u;      /* true DOFs of the trial space X (continuous in time) */
    const double* y_geometry;   /* [n_y_cells*8] */
    const double* x_geometry;   /* [n_x_cells*8] */
    const int32_t* y_to_x;      /* [n_y_cells] active X ancestor of each Y cell */
    const int32_t* y_restr_offsets; /* [n_y_cells*ndof+1] */
    const int32_t* y_restr_dofs;    /* [y_restr_nnz] */
    const double* y_restr_weights;  /* [y_restr_nnz] */
    int32_t y_restr_nnz;
    const int32_t* x_restr_offsets; /* [n_x_cells*ndof+1] */
    const int32_t* x_restr_dofs;
    const double* x_restr_weights;
    int32_t x_restr_nnz;
    const double* m_cells;   /* [n_y_cells*3] (m00, m01, m11) or NULL = identity */
    const double* ell_cells; /* [n_y_cells] constant load per Y cell or NULL = zero */
    int u0_kind;             /* APF_U0_* */
    double zero_tol;         /* per-local-entry filter, reference default 1e-15 */
    double g_scale;          /* reference default -1 */
    int dim_space;           /* 1 = 1+1D, 2 (or 0) = 2+1D */
} apf_problem_desc;

/* ---- context ----------------------------------------------------------------- */
/* stream: a cudaStream_t (NULL = the context creates its own non-blocking stream). */
int apf_ctx_create(int device, void* stream, apf_ctx** out);
void apf_ctx_destroy(apf_ctx* ctx);
const char* apf_ctx_last_error(const apf_ctx* ctx);
int apf_ctx_synchronize(apf_ctx* ctx);
/* Number of kernels the library has launched in this process. */
int64_t apf_ctx_kernel_launches(const apf_ctx* ctx);
/* Per-kernel CUDA-event timing on the context's stream plus host wall time of the
 * library's stages (the GPU counterpart of the reference's TimingRecorder,
 * src/finite_element/detail/timing.hpp): enable 1 = kernels and stages, 2 = stages only
 * (no per-launch events), 0 = off.  Every call resets the totals. */
int apf_ctx_set_timing(apf_ctx* ctx, int enable);
/* JSON object {"kernel": [launches, total_ms], ...}; valid until the next call. */
const char* apf_ctx_timing_report(apf_ctx* ctx);
/* The library allocates from the device's default stream-ordered pool and keeps freed
 * memory there.  apf_ctx_reserve_pool grows the pool to at least `bytes` at once (one
 * allocation, freed again on the context's stream) so that later allocations are carved
 * from it rather than mapped one by one; apf_ctx_pool_stats reports the pool's reserved
 * and used bytes (current and high-water marks; any pointer may be NULL). */
int apf_ctx_reserve_pool(apf_ctx* ctx, int64_t bytes);
int apf_ctx_pool_stats(apf_ctx* ctx, int64_t* reserved, int64_t* reserved_high, int64_t* used, int64_t* used_high);

/* ---- assembly ------------------------------------------------------------------ */
/* Replaces finite_element::system::assemble_main_system_blocks<QS,QT,Backend>
 * (src/finite_element/system/assemble_saddle_problem.hpp:131) and
 * la::saddle::make_saddle_point_blocks + compose_saddle_point_matrix
 * (src/linear_algebra/system/saddle_point_system.hpp:105-141,
 *  src/linear_algebra/assembly/compose_block_system.hpp:116).
 * Builds A_y, B, B^T, C_signed, K, f and g on the device.  Pattern = union over
 * cells of the restricted local entries with |a_ij| > zero_tol, duplicates summed
 * (explicit zeros kept), exactly as scatter.hpp:66-115 + setFromTriplets.
 * inputs_on_device: 1 if every pointer in desc is a device pointer, 0 if host. */
int apf_assemble_main_system(apf_ctx* ctx, const apf_problem_desc* desc, int inputs_on_device,
                             apf_system** out);

/* Replaces finite_element::assembly::assemble_parabolic_graph_norm_approximation
 * (src/finite_element/assembly/main_system/parabolic_graph_norm.hpp:22-65) with
 * la::preconditioners::parabolic_graph_norm_approximation
 * (src/linear_algebra/preconditioners/schur_approximations.hpp:237-287):
 * Hhat = -C_signed + B_dt diag(A_y)^-1 B_dt^T + A_x.  Also keeps B_dt and A_x. */
int apf_assemble_graph_norm(apf_ctx* ctx, apf_system* sys, double diagonal_tolerance);

/* Two-pass full saddle assembly of the direct-solver path.  Replaces
 * finite_element::assembly::assemble_main_full_saddle_two_pass_2d
 * (src/finite_element/assembly/main_system/two_pass_full_saddle_2d.hpp:468), called from
 * solve_main_system.hpp:1855-1942, with its pattern cache TwoPassFullSaddleAssemblyCache2D
 * (same file :325-373).  2+1D only, as the reference (static_assert at :520).
 * Pattern pass (:740-790): the structural union over Y cells of the restricted (Y x Y),
 * (X ancestor x Y) and transposed couplings and over bottom X cells of (X x X).  Numeric
 * pass (scatter_matrix_by_slots, :431-459): the local entries with |a_ij| > zero_tol added
 * into that pattern in cell order.  Then prune(1.0, zero_tol) (:1720): every entry with
 * |value| <= zero_tol is dropped.  The result is block APF_BLOCK_K of *out (the only block
 * it holds) and the right-hand side [f; g] (APF_VEC_F, APF_VEC_G).
 * cache (NULL = none): the pattern of the last call is reused while the mesh and its DOF
 * maps are unchanged (sizes and a fingerprint of the restriction rows, the Y -> X map and
 * the bottom cells; the reference keys on the spaces' version counters), so a later call
 * with new coefficients (m_cells, ell_cells, u0_kind, geometry of the same topology) runs
 * the numeric pass only.  A cache belongs to one context and is destroyed before it. */
typedef struct apf_two_pass_cache apf_two_pass_cache;
int apf_two_pass_cache_create(apf_ctx* ctx, apf_two_pass_cache** out);
void apf_two_pass_cache_destroy(apf_two_pass_cache* cache);
/* pattern passes run, pattern reuses (the reference's pattern_reuse_count), entries of the
 * kept pattern (any pointer may be NULL) */
int apf_two_pass_cache_stats(const apf_two_pass_cache* cache, int64_t* pattern_builds, int64_t* pattern_reuses,
                             int64_t* pattern_entries);
int apf_assemble_full_saddle_two_pass(apf_ctx* ctx, const apf_problem_desc* desc, int inputs_on_device,
                                      apf_two_pass_cache* cache, apf_system** out);

/* Block sizes; nnz counts stored entries (explicit zeros included). */
int apf_system_block_info(const apf_system* sys, int block, int32_t* rows, int32_t* cols, int64_t* nnz);
/* Copy a block in CSR form.  to_device: 1 = destination pointers are device memory. */
int apf_system_block_copy(apf_ctx* ctx, const apf_system* sys, int block, int32_t* row_ptr,
                          int32_t* col_idx, double* values, int to_device);
/* Device pointers of a block's CSR arrays (owned by sys; valid until sys is destroyed). */
int apf_system_block_device_ptrs(const apf_system* sys, int block, const int32_t** row_ptr,
                                 const int32_t** col_idx, const double** values);
int apf_system_vector_copy(apf_ctx* ctx, const apf_system* sys, int which, double* out, int to_device);
void apf_system_destroy(apf_system* sys);

/* ---- block-preconditioned MINRES ------------------------------------------------ */
#define APF_PRECOND_AMG_BLOCK 0 /* blkdiag(A_y, Hhat), one SA-AMG V-cycle per block */
#define APF_PRECOND_LEARNED 1   /* learned preconditioner (falls back to APF_PRECOND_AMG_BLOCK) */

/* Mirrors the fields of la::concepts::SolverOptions the MINRES path reads
 * (src/linear_algebra/concepts/solver.hpp:212-255). */
typedef struct apf_solver_options
{
    double tolerance;                 /* true relative residual target (reference yml: 1e-8) */
    int max_iterations;               /* reference default 20000 in the runner */
    int use_true_residual_batching;   /* reference default 1 */
    int true_residual_check_interval; /* reference default 100 */
    int preconditioner;               /* APF_PRECOND_* */
    int amg_smooth_steps;             /* damped-Jacobi sweeps per side of the V-cycle (>= 1) */
    double amg_strength;              /* strength-of-connection threshold (e.g. 0.08) */
    int amg_coarse_size;              /* dense coarsest solve at or below this size */
    int amg_aggressive_levels;        /* finest levels aggregated from a distance-2 independent set
                                         (larger aggregates, cheaper V-cycles); default 1, 0 = distance 1 */
    int amg_vcycles;                  /* V-cycles per block application: 1 (default) = z = V r; 2 = the
                                         two-step iteration z = s V r, z += s V (r - A z) with
                                         s = 1 / (1.1 lambda_max(V A)) estimated by power iteration
                                         before every solve: a fixed SPD operator (eigenvalues of its
                                         product with A: 2 mu - mu^2, mu in (0, 1)) with about half the
                                         condition number, for high-contrast coefficients */
} apf_solver_options;

/* Mirrors SolverDiagnostics.iterative_stats (src/linear_algebra/concepts/solver.hpp:186-197). */
typedef struct apf_solver_diagnostics
{
    int iterations;
    int residual_check_batches;
    int converged;                /* accepted by the FP64 true residual */
    int backend_converged;
    double backend_reported_error;
    double final_true_residual;   /* ||K x - b||_2 / ||b||_2 */
    double setup_seconds;         /* preconditioner setup */
    double solve_seconds;
    int amg_levels_lambda, amg_levels_u;
    int64_t amg_nnz_lambda, amg_nnz_u;
    int preconditioner_used;      /* APF_PRECOND_*: LEARNED, or AMG_BLOCK after a fallback */
    int learned_fallback;         /* 1: the learned run missed the tolerance, plain run from its iterate */
} apf_solver_diagnostics;

void apf_solver_options_default(apf_solver_options* opt);

/* Preconditioner setup for the assembled system (requires apf_assemble_graph_norm).
 * Replaces ParabolicGraphNormBlockPreconditioner::compute_from_graph_norm
 * (src/linear_algebra/eigen_backend/preconditioners/parabolic_graph_norm_minres.hpp:55-111). */
int apf_setup_preconditioner(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt);

/* Solve K [lambda; u] = [f; g] by block-preconditioned MINRES with true-residual batches.
 * Replaces SaddlePreconditionedSolveDispatcher<Backend>::solve ->
 * solve_minres_with_parabolic_graph_norm
 * (src/linear_algebra/eigen_backend/preconditioners/solve_saddle_system.hpp:32-121,
 *  parabolic_graph_norm_minres.hpp:232-369).  Sets up the preconditioner if needed.
 * initial_guess: NULL (zero start) or n_lambda+n_u values; solution: n_lambda+n_u values
 * (may be NULL: the solution stays on the device).  Returns APF_ERR_NOT_CONVERGED with
 * diag filled when the true residual misses the tolerance (the reference throws
 * PreconditionedSolveFailure, parabolic_graph_norm_minres.hpp:357-366). */
int apf_solve_minres(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt, const double* initial_guess,
                     double* solution, int pointers_on_device, apf_solver_diagnostics* diag);
/* The same with another right-hand side rhs (n_lambda + n_u values) in place of the
 * assembled [f; g]: the correction equation K d = b - K x0 of an initial guess x0 that the
 * reference's dispatcher solves when MainSystemInitialGuess::solve_correction_equation is
 * set (src/linear_algebra/eigen_backend/preconditioners/solve_saddle_system.hpp:75-86). */
int apf_solve_minres_with_rhs(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt, const double* rhs,
                              const double* initial_guess, double* solution, int pointers_on_device,
                              apf_solver_diagnostics* diag);
/* The correction equation on the device: r = [f; g] - K x0, MINRES on K d = r from zero (its
 * tolerance relative to ||r||), solution = x0 + d, which the system then holds.  The
 * reference's dispatcher forms r = rhs - K x0 on the host and returns x0 + d
 * (src/linear_algebra/eigen_backend/preconditioners/solve_saddle_system.hpp:75-86,
 * src/finite_element/system/solve_main_system.hpp:1547-1560 for the direct path).
 * x0: n_lambda + n_u values; solution may be NULL (kept on the device only). */
int apf_solve_minres_correction(apf_ctx* ctx, apf_system* sys, const apf_solver_options* opt, const double* x0,
                                double* solution, int pointers_on_device, apf_solver_diagnostics* diag);
/* ||[f; g] - K x|| and ||[f; g]|| on the device, x NULL = the solution the system holds: the
 * post-solve residual the reference records in Summary diagnostics mode
 * (src/finite_element/system/solve_main_system.hpp:540-572, 651-700) and, with x = x0, its
 * initial-guess residual (solve_main_system.hpp:587-604). */
int apf_system_residual_norms(apf_ctx* ctx, apf_system* sys, const double* x, int pointers_on_device,
                              double* residual_norm, double* rhs_norm);
/* Replace the solution the system holds (n_lambda + n_u values; read by apf_estimate,
 * apf_x_indicators and apf_g_estimator): e.g. x0 + d after the correction equation's solve
 * for d, as the reference's dispatcher returns it. */
int apf_system_set_solution(apf_ctx* ctx, apf_system* sys, const double* x, int pointers_on_device);
/* z = P^{-1} r with the set-up preconditioner: block 0 = A_y part (n_lambda values),
 * 1 = Hhat part (n_u values), 2 = the full block operator (n_lambda + n_u).  For tests
 * and diagnostics (symmetry, PCG quality) of the preconditioner. */
int apf_preconditioner_apply(apf_ctx* ctx, apf_system* sys, int block, const double* r, double* z,
                             int pointers_on_device);
/* ---- equilibrated-flux estimator ------------------------------------------------ */
/* Totals of the last estimate (the reference's CellwiseEquilibratedFluxError /
 * CellwiseTimeSlabEstimatorError totals, time_slab_cellwise_errors.hpp:325-450). */
typedef struct apf_estimator_result
{
    double flux_squared;           /* sum_K ||M^-1/2 (sigma + M grad theta~)||^2_K */
    double divergence_squared;     /* sum_K ||l - d_t u - div sigma||^2_K */
    double reconstruction_squared; /* sum_K ||lambda_delta - lambda~||^2_{Y,K} */
    double eta_squared;            /* flux + reconstruction */
    int n_slabs;
    int n_patches;
    int max_patch_cells;
    int reconstruction_iterations;
    double reconstruction_residual; /* relative residual of the slab reconstruction solve */
} apf_estimator_result;

/* The estimator of one inner iteration for p = 1 or 2, on the solution of the last
 * apf_solve_minres call:
 *   lambda~ : slab Riesz reconstruction, A_y lambda~ = f - B^T u (Y is broken in time, so
 *             this is every slab's reconstruction system at once), replacing
 *             TimeSlabReconstruction::solve_all_slabs (src/finite_element/time_slabs/
 *             time_slab_reconstruction.hpp:584);
 *   sigma_a : one mixed RT_p x P_p local problem per (time slab, spatial vertex) patch,
 *             replacing TimeSlabEquilibratedFluxReconstruction2plus1d::solve_all_patches
 *             (time_slab_equilibrated_flux_reconstruction.hpp:2515) with the bordered
 *             dense system of dense_local_error_blocks_2d.hpp:812-905;
 *   indicators per Y cell: compute_equilibrated_flux_error_squared_by_source_cell_2plus1d
 *             (time_slab_equilibrated_flux_indicators.hpp:203), the reconstruction term of
 *             compute_Y_error_squared_by_source_cell (time_slab_error_norms.hpp:946) and
 *             their sum (time_slab_estimator_combination.hpp).
 * y_vertex_ids: [n_y_cells*3] spatial vertex ids of every Y cell (the reference mesh's
 * cell.spatial_vertex_ids); host or device per pointers_on_device.  Y cells must
 * coincide with their X ancestors.
 * 1+1D systems (dim_space = 1, p = 1) use the edge-patch estimator instead:
 * TimeSlabEquilibratedFluxReconstruction1plus1d (time_slab_equilibrated_flux_reconstruction.hpp:
 * 773-1880; patches from time_slab_edge_patch_builder.hpp:353-537, flux space
 * patch_flux_space_1d.hpp, scalar space patch_scalar_space.hpp, local forms
 * local_error_bilinear_forms.hpp and local_error_linear_forms.hpp) and
 * compute_equilibrated_flux_error_squared_by_source_cell_1plus1d
 * (time_slab_equilibrated_flux_indicators.hpp:23-190); y_vertex_ids is not used (NULL).  Output arrays ([n_y_cells] each, host or device per
 * pointers_on_device) may be NULL. */
/* ---- batches of independent problems ----------------------------------------------- */
/* Several independent problems assembled as one system (their cells, DOFs and vertex ids
 * concatenated with offsets, so every stage runs over all of them in one launch): part p
 * owns lambda rows [lambda_offsets[p], lambda_offsets[p+1]) and u rows
 * [u_offsets[p], u_offsets[p+1]) (host arrays of n_parts + 1, starting at 0, ending at
 * n_lambda / n_u).  No reference counterpart (a batching form; the reference solves one
 * problem per call).  Later apf_solve_minres calls accept the solve only when every part's
 * ||b_p - K_p x_p|| / ||b_p|| <= tolerance, the reference's acceptance test
 * (iterative_residual_acceptance.hpp:32-54) per problem; apf_system_part_residuals copies
 * those residuals of the last solve (n_parts doubles, host).  n_parts = 0 clears it. */
int apf_system_set_partition(apf_ctx* ctx, apf_system* sys, int n_parts, const int32_t* lambda_offsets,
                             const int32_t* u_offsets);
int apf_system_part_residuals(apf_ctx* ctx, const apf_system* sys, double* out);

/* Precision of the 2+1D P1 patch solves of later apf_estimate calls on this context (no
 * reference counterpart: the reference factors every patch in FP64):
 *   APF_PATCH_FP64         FP64 assembly and partial-pivot LU (default);
 *   APF_PATCH_FP32_REFINED the patch matrix assembled and factored in FP32, then one FP64
 *                          iterative-refinement step (FP64 residual formed from the local
 *                          entries, correction solved with the FP32 factors).
 * p = 2 and 1+1D patches always use FP64 (APF_ERR_INVALID from apf_estimate otherwise). */
#define APF_PATCH_FP64 0
#define APF_PATCH_FP32_REFINED 1
int apf_ctx_set_patch_precision(apf_ctx* ctx, int precision);

/* Launch-shape autotuner of the patch solves (no reference counterpart): patches are
 * sorted into size buckets (at most 32, 48, 64, 96, 144 unknowns) and every bucket is
 * solved by teams of W warps per patch.  With autotuning on (the default) the first
 * apf_estimate that meets a (degree, precision, bucket) times W = 1, 2 and 4 on that
 * bucket's own patches and keeps the fastest for the context; the values do not depend on
 * W.  enable = 0 uses the kept choices (or the size rule W = 1 / 2 / 4 for buckets up to
 * 48 / 64 / larger where none was made), enable < 0 forgets them and turns tuning on.
 * The report is a JSON
 * object {"p1_fp64_n64": {"warps_per_patch": 2, "patches": ..., "ms_w1_w2_w4": [...]}, ...},
 * valid until the next call. */
int apf_ctx_set_autotune(apf_ctx* ctx, int enable);
const char* apf_ctx_autotune_report(apf_ctx* ctx);

int apf_estimate(apf_ctx* ctx, apf_system* sys, const int32_t* y_vertex_ids, int pointers_on_device,
                 double* flux_squared, double* divergence_squared, double* reconstruction_squared,
                 double* eta_squared, apf_estimator_result* result);
/* Keep (keep = 1) the equilibrated flux of the following 2+1D apf_estimate calls on the device
 * for apf_flux_sample, or drop it (0).  The reference's TimeSlabEquilibratedFluxReconstruction
 * keeps its patch fluxes for sigma_and_div_sigma_on_slab_cell
 * (src/finite_element/time_slabs/time_slab_equilibrated_flux_reconstruction.hpp:1317-1341),
 * which its snapshot writer samples
 * (src/finite_element/io/write_time_slab_flux_reconstruction_samples_binary.hpp:17-174). */
int apf_system_keep_flux(apf_ctx* ctx, apf_system* sys, int keep);
/* The cells the kept flux lives on (the Y cells, or the slab cells they are cut into when Y
 * cells span several time slabs): their count, and per cell its time slab (slabs in time
 * order) and source Y cell (index in the system's Y cell order).  slab / source_y_cell may be
 * NULL (count only). */
int apf_flux_cells(apf_ctx* ctx, const apf_system* sys, int32_t* n_cells, int32_t* slab, int32_t* source_y_cell);
/* sigma_x, sigma_y, div sigma (values: n_points x 3) of the kept flux at physical points
 * (points: n_points x 3 as x, y, t), point i on kept cell cell[i]: the sum of the cell's
 * vertex-patch fluxes, as sigma_and_div_sigma_on_slab_cell evaluates it. */
int apf_flux_sample(apf_ctx* ctx, apf_system* sys, int32_t n_points, const int32_t* cell, const double* points,
                    double* values, int pointers_on_device);

/* ---- X-marking indicators -------------------------------------------------------- */
/* Totals of XMarkingIndicatorComponents (algorithm/adaptive_result.hpp:294-320). */
typedef struct apf_x_indicator_totals
{
    double lambda_y_squared;      /* sum_K int_K grad_x lambda . M grad_x lambda */
    double initial_trace_squared; /* sum_K ||u0 - u(., 0)||^2 over the t = 0 faces */
    double eta_squared;           /* their sum */
} apf_x_indicator_totals;

/* The adaptive driver's X-marking indicators on the solution of the last apf_solve_minres
 * call, replacing compute_x_marking_indicator_components
 * (algorithm/detail/indicator_utilities.hpp:443-473):
 *   lambda_by_y[K] = int_K grad_x lambda_delta . M grad_x lambda_delta  (per Y cell, :115-171),
 *   lambda_by_x    = lambda_by_y summed onto each Y cell's X ancestor (:405-433),
 *   trace_by_x[K]  = ||u0 - u_delta(., 0)||^2 on the t = 0 face of X cell K, 0 elsewhere
 *                    (:336-400, the bottom Duffy rule of the main assembly),
 *   eta_by_x       = lambda_by_x + trace_by_x.
 * Arrays (any may be NULL): n_y_cells / n_x_cells values, host or device. */
int apf_x_indicators(apf_ctx* ctx, apf_system* sys, int pointers_on_device, double* lambda_by_y, double* lambda_by_x,
                     double* trace_by_x, double* eta_by_x, apf_x_indicator_totals* totals);
/* rho^2 (lambda^2 + (1 + 1/(rho + 1/2)^2) trace^2), replacing
 * compute_y_estimator_threshold_squared (indicator_utilities.hpp:475-491); rho <= 0 gives
 * APF_ERR_INVALID (the reference throws). */
int apf_y_estimator_threshold_squared(double rho, double lambda_y_squared, double initial_trace_squared,
                                      double* threshold_squared);

/* ---- G^delta estimator ------------------------------------------------------------ */
typedef struct apf_g_estimator_result
{
    double lambda_difference_squared; /* ||lambda_G - lambda_delta||^2 in the A_G energy */
    double solve_relative_residual;   /* ||rhs_G - A_G lambda_G|| / ||rhs_G|| of the CG solve */
    int solve_iterations;
    int n_g;                          /* true DOFs of G */
} apf_g_estimator_result;

/* The adaptive driver's G^delta estimator on the solution of the last apf_solve_minres
 * call, replacing AdaptiveDriver::compute_g_estimator_for_accepted_inner_iteration_
 * (algorithm/adaptive_driver.hpp:2690-2900): the space G of degree p+1 on the system's Y
 * cells (broken in time, FESpace<GT, FiniteElementTraits<GT, p+1, p+1>, SpaceOnlyPolicy>),
 * given by its flattened CellRestriction (host arrays: offsets [n_y_cells * ndof_G + 1] with
 * ndof_G = (p+2)(p+3)/2 (p+2), the Y cells in the system's order; n_g true DOFs);
 * A_G lambda_G = f_G - B(X, G)^T u_delta solved by AMG-preconditioned CG to the relative
 * residual `tolerance` (the reference solves directly), and ||lambda_G - lambda_delta||^2_{A_G}
 * with lambda_delta prolonged nodally into G (g_lambda_difference_squared).  2+1D systems of
 * degree 1 (G of degree 2).  APF_ERR_NOT_CONVERGED when CG misses the tolerance. */
int apf_g_estimator(apf_ctx* ctx, apf_system* sys, int32_t n_g, const int32_t* g_restr_offsets,
                    const int32_t* g_restr_dofs, const double* g_restr_weights, int32_t g_restr_nnz, double tolerance,
                    apf_g_estimator_result* result);

/* ---- estimator artifacts ---------------------------------------------------------- */
/* The reference's binary files of an estimate, written from per-cell arrays (host, or
 * device with pointers_on_device = 1 and a context; ctx may be NULL for host arrays).
 * cell_ids are the mesh ids of the source (Y) cells, one per value.  Entry order: by
 * decreasing value (eta for the components file), ties by increasing cell id, as
 * CellwiseSquaredError::sorted_descending (src/finite_element/time_slabs/
 * time_slab_cellwise_errors.hpp:54-68); sort_descending = 0 keeps the given order (the
 * reference then writes its hash map's order).  Replaces
 * write_cellwise_error_binary (src/finite_element/io/write_cellwise_error_binary.hpp:24-79):
 *   int32 [version 1, n], int32 cell_ids[n], float64 values[n];
 * and write_cellwise_error_components_binary
 * (src/finite_element/io/write_cellwise_error_components_binary.hpp:12-88):
 *   int32 [version 1, n, 4], int32 cell_ids[n], float64 flux[n], recon[n], divergence[n],
 *   eta[n]  (the equilibrated-flux, reconstruction, divergence-residual and total
 *   indicators squared, as apf_estimate returns them). */
int apf_write_cellwise_error_binary(apf_ctx* ctx, const char* path, int32_t n_cells, const int32_t* cell_ids,
                                    const double* values, int pointers_on_device, int sort_descending);
int apf_write_cellwise_error_components_binary(apf_ctx* ctx, const char* path, int32_t n_cells,
                                               const int32_t* cell_ids, const double* flux, const double* recon,
                                               const double* divergence, const double* eta, int pointers_on_device,
                                               int sort_descending);
/* The driver's x_indicator_components.bin from the X-marking indicators (apf_x_indicators'
 * per-X-cell arrays; x_cell_ids = mesh ids of the active X cells).  Replaces
 * adaptive_algorithm::output::detail::write_x_indicator_components_binary
 * (algorithm/output/iteration_snapshot_writer.hpp:173-233):
 *   int32 [version 1, n, 3], int32 cell_ids[n], float64 lambda_y[n], initial_trace[n],
 *   eta[n], entries by decreasing eta, ties by increasing cell id. */
int apf_write_x_indicator_components_binary(apf_ctx* ctx, const char* path, int32_t n_x_cells,
                                            const int32_t* x_cell_ids, const double* lambda_by_x,
                                            const double* trace_by_x, const double* eta_by_x, int pointers_on_device);

/* ---- allocation-free residual check ---------------------------------------------- */
/* No counterpart in the reference: an addition for callers that cannot allocate device
 * memory where they need the check -- e.g. a solver loop whose device memory is all owned
 * by its own pool, or a job running the GPU so full that a late cudaMalloc could fail.
 * Computes ||b - K x||_2 and ||b - K x||_2 / ||b||_2 (||b|| = 0: the absolute value) for a
 * CSR matrix K (rows x rows, int32 indices, f64 values) and vectors x, b, all device
 * pointers, on the context's stream.  Allocates no device memory: its scratch is one
 * fixed 64 KiB device array shared by all calls on a device, so at most 16,777,216 rows
 * (larger K: APF_ERR_CAPACITY).  The first call on a device looks the array's address up
 * and loads the entry point's kernels onto the device (under lazy module loading their code
 * would otherwise be loaded, taking device memory, at first launch): only that first call
 * may allocate, so make it at set-up, before any stream capture.  Calls whose GPU work
 * overlaps race on the shared array.  Results are written to the host doubles given (either
 * may be NULL). */
int apf_true_residual_noalloc(apf_ctx* ctx, int32_t rows, const int32_t* row_ptr, const int32_t* col_idx,
                              const double* values, const double* x, const double* b, double* absolute_residual,
                              double* relative_residual);

/* Device pointer of the last solution (n_lambda + n_u values, owned by sys). */
int apf_system_solution_device_ptr(const apf_system* sys, const double** solution);

/* ---- learned preconditioner (no counterpart in the reference) -------------------- */
/* The reference's MINRES preconditioner is blkdiag(A_y, Hhat)^-1 by sparse Cholesky
 * (parabolic_graph_norm_minres.hpp:46-181); here each block is one SA-AMG V-cycle.  The
 * learned variant keeps that structure and replaces the damped-Jacobi weights omega/a_ii of
 * every non-coarsest level by w_i^(o) = omega/a_ii exp(0.5 tanh(y_i^(o))), y_i = MLP(f_i),
 * f_i = 8 scale-free features of matrix row i, o = 0 for the first pre-smoothing sweep and
 * 1 for the later ones (post-smoothing runs them in reverse order), and scales each
 * level's coarse correction by alpha_l = 2 sigmoid(theta_l).  The MLP (8 -> 32 -> 32 -> 2,
 * tanh) runs in BF16 with FP32 accumulation on the tensor cores at preconditioner set-up;
 * the V-cycles stay symmetric and a Gershgorin bound keeps every sweep convergent, so the
 * preconditioner is SPD.  Parameters: APF_LEARNED_NUM_PARAMS floats (layout in
 * apf_learned.cuh); all zero gives the plain weights and alpha = 1. */
#define APF_LEARNED_NUM_PARAMS 1442
typedef struct apf_learned_model apf_learned_model;
int apf_learned_model_create(apf_learned_model** out);
int apf_learned_model_destroy(apf_learned_model* model);
int apf_learned_model_set_params(apf_learned_model* model, const float* params, int n);
int apf_learned_model_get_params(const apf_learned_model* model, float* params, int n);
/* Model used by set-ups with preconditioner = APF_PRECOND_LEARNED (NULL clears; the context
 * keeps a copy of the parameters). */
int apf_ctx_set_learned_model(apf_ctx* ctx, const apf_learned_model* model);
/* Training objective on an assembled system whose preconditioner is set up: the
 * energy-norm contraction of `steps` stationary V-cycle iterations of both blocks,
 *   L = sum_block mean_sample (1/steps) log(||E^steps e||_T^2 / ||e||_T^2),  E = I - V T,
 * T = A_y and Hhat, e = E^burn_in e0 (no gradient through the burn-in), e0 = start vectors
 * ([samples][n_lambda + n_u], NULL: seeded normal vectors), and dL/dparams
 * (APF_LEARNED_NUM_PARAMS floats, host, may be NULL) by reverse mode through the V-cycles
 * and the MLP (FP32 forward / backward kernels). */
int apf_learned_loss_and_grad(apf_ctx* ctx, apf_system* sys, const apf_learned_model* model, int samples, int steps,
                              int burn_in, uint64_t seed, const double* start_vectors, int pointers_on_device,
                              double* loss, float* grad);
/* y = MLP(features) for n rows of 8 features, 2 outputs per row (y[2 i + o]): precision
 * 0 = FP32 CUDA cores (training pass), 1 = BF16 tensor cores with FP32 accumulation
 * (inference). */
int apf_learned_forward(apf_ctx* ctx, const apf_learned_model* model, int n, const float* features, float* y,
                        int precision, int pointers_on_device);

/* ---- AMG hierarchy inspection (tests and the oracle's V-cycle restatement) ---------- */
/* block 0 = A_y, 1 = Hhat (its hierarchy is built on the filtered Hhat_F). */
int apf_amg_info(apf_ctx* ctx, apf_system* sys, int block, int* levels, int* dense_coarse, int* coarse_sweeps,
                 int* smooth_steps);
/* rows, nnz of A_l and (l < levels-1) P_l, the Jacobi omega_l and the coarse scale alpha_l */
int apf_amg_level_info(apf_ctx* ctx, apf_system* sys, int block, int level, int* rows, int64_t* nnz_a,
                       int64_t* nnz_p, double* omega, double* alpha);
/* CSR arrays (host) of A_l (which = 0) or P_l (which = 1) */
int apf_amg_level_copy(apf_ctx* ctx, apf_system* sys, int block, int level, int which, int32_t* row_ptr,
                       int32_t* col_idx, double* values);
/* smoother weights of level l (host, rows values) for sweep class o (0: first sweep,
 * 1: later sweeps): omega_l / a_ii, or the learned weights */
int apf_amg_level_weights(apf_ctx* ctx, apf_system* sys, int block, int level, int o, double* weights);
/* row features of level l (host, rows x 8 floats) as the learned model sees them */
int apf_amg_level_features(apf_ctx* ctx, apf_system* sys, int block, int level, float* features);

#ifdef __cplusplus
}
#endif
#endif
