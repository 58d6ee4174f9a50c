/*
 * sparsesolv_b200.h -- C ABI of the B200 (sm_100a) solve path.
 *
 * Every entry point takes plain pointers and sizes. Host pointers carry host
 * data; the `_dev` variants take device pointers that the caller keeps
 * resident in HBM -- every array argument of a `_dev` call, freedofs masks
 * included, is device memory (a host pointer is refused with
 * SSV_ERR_INVALID_ARG). All calls are synchronous on return (the work runs on the
 * handle's own CUDA stream). A handle is not safe for concurrent use from two
 * threads (the reference's objects keep mutable work buffers the same way,
 * include/sparsesolv/preconditioners/ic_preconditioner.hpp:555-563).
 *
 * Status: every function returns SSV_OK (0) or an SSV_ERR_* code; the message
 * of the last failure on the calling thread is ssv_last_error(). The Python
 * layer maps SSV_ERR_RUNTIME -> RuntimeError (reference std::runtime_error),
 * SSV_ERR_INVALID_ARG -> ValueError (std::invalid_argument), SSV_ERR_TYPE ->
 * TypeError (py::type_error), SSV_ERR_ALLOC -> MemoryError (std::bad_alloc).
 *
 * Scalars: SSV_F64 = double, SSV_C128 = complex<double> stored as interleaved
 * (re, im) doubles, exactly the layout of std::complex<double>.
 */
#ifndef SPARSESOLV_B200_H
#define SPARSESOLV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SSV_VERSION_MAJOR 0
#define SSV_VERSION_MINOR 1
#define SSV_VERSION_PATCH 0

enum ssv_status {
    SSV_OK = 0,
    SSV_ERR_INVALID_ARG = 1, /* std::invalid_argument in the reference     */
    SSV_ERR_RUNTIME = 2,     /* std::runtime_error in the reference        */
    SSV_ERR_CUDA = 3,        /* a CUDA runtime call failed                 */
    SSV_ERR_NO_DEVICE = 4,   /* no CUDA device: this library has no CPU path */
    SSV_ERR_TYPE = 5,        /* wrong scalar type for this object          */
    SSV_ERR_TIMEOUT = 6,     /* a bounded device wait gave up              */
    SSV_ERR_ALLOC = 7        /* device allocation failed                   */
};

enum ssv_dtype { SSV_F64 = 0, SSV_C128 = 1 };

/* NormType, include/sparsesolv/core/types.hpp:43-47 */
enum ssv_norm_type { SSV_NORM_RHS = 0, SSV_NORM_INITIAL_RESIDUAL = 1, SSV_NORM_CUSTOM = 2 };

/* Krylov methods of SparseSolvSolver, include/sparsesolv/ngsolve/sparsesolv_solvers.hpp:112-128 */
enum ssv_method { SSV_METHOD_ICCG = 0, SSV_METHOD_SGSMRTR = 1, SSV_METHOD_CG = 2, SSV_METHOD_COCR = 3 };

/* Precision of a preconditioner application (new: no reference counterpart).
 * FP64 is the drop-in; FP32 stores L / auxiliary matrices in float and applies
 * in float while the outer Krylov recurrence stays in double. */
enum ssv_precision { SSV_PREC_FP64 = 0, SSV_PREC_FP32 = 1, SSV_PREC_FP32_NODAL = 2 };

/*
 * Field-for-field mirror of sparsesolv::SolverConfig
 * (include/sparsesolv/core/solver_config.hpp:33-159). Booleans are int 0/1.
 * ssv_config_default() fills the reference defaults.
 */
typedef struct ssv_config {
    double tolerance;                 /* 1e-10 */
    int32_t max_iterations;           /* 1000  */
    double abs_tolerance;             /* 1e-12 */
    int32_t norm_type;                /* SSV_NORM_RHS */
    double custom_norm;               /* 1.0   */
    double shift_parameter;           /* 1.05  */
    int32_t diagonal_scaling;         /* 0     */
    int32_t auto_shift;               /* 0     */
    double shift_increment;           /* 0.05  */
    double max_shift_value;           /* 5.0   */
    double min_diagonal_threshold;    /* 1e-6  */
    double zero_diagonal_replacement; /* 1e-10 */
    int32_t max_shift_trials;         /* 100   */
    int32_t divergence_check;         /* 0 = None, 1 = StagnationCount */
    double divergence_threshold;      /* 1000  */
    int32_t divergence_count;         /* 100   */
    int32_t save_best_result;         /* 1     */
    int32_t save_residual_history;    /* 0     */
    int32_t conjugate;                /* 0     */
    int32_t use_abmc;                 /* 0     */
    int32_t abmc_block_size;          /* 4     */
    int32_t abmc_num_colors;          /* 4     */
    int32_t abmc_reorder_spmv;        /* 0     */
    int32_t abmc_use_rcm;             /* 0     */
    int32_t precision;                /* SSV_PREC_FP64 (new knob) */
} ssv_config;

/* sparsesolv::SolverResult, include/sparsesolv/core/types.hpp:29-37.
 * The residual history goes to a caller buffer (ssv_solver_solve). */
typedef struct ssv_result {
    int32_t converged;
    int32_t iterations;
    double final_residual;
    int32_t history_len;      /* entries written (<= history_cap)           */
    int32_t history_total;    /* entries the reference would have produced  */
    double actual_shift;      /* IC shift after auto-shift (ICCG only)      */
    double setup_seconds;     /* host wall time of preconditioner setup     */
    double solve_seconds;     /* host wall time of the Krylov iteration     */
    int64_t kernel_launches;  /* device kernels this call launched          */
} ssv_result;

/* Per-phase timing of one Krylov iteration (measurement hook, no reference
 * counterpart): each phase is re-launched `reps` times on the library's
 * stream between CUDA events, after a solve on the same handle. */
#define SSV_MAX_PHASES 8
typedef struct ssv_phase_profile {
    int32_t num_phases;
    char names[SSV_MAX_PHASES][24];
    double ms[SSV_MAX_PHASES];        /* mean device time per phase execution */
    double bytes[SSV_MAX_PHASES];     /* algorithmic bytes per phase execution */
    int32_t kernels[SSV_MAX_PHASES];  /* kernel launches per phase execution */
} ssv_phase_profile;

typedef struct ssv_matrix ssv_matrix;   /* device-resident CSR              */
typedef struct ssv_solver ssv_solver;   /* SparseSolvSolver state           */
typedef struct ssv_precond ssv_precond; /* IC / AMS / complex-AMS           */
typedef struct ssv_batch ssv_batch;     /* batched COCR over a frequency family */
typedef struct ssv_mlp ssv_mlp;         /* learned initial-guess predictor      */

/* One timed SpMM launch shape of the batch autotuner. */
typedef struct ssv_batch_tune_entry {
    int32_t freq_tile;    /* frequencies whose columns one pass over K and M forms */
    int32_t lanes;        /* threads per matrix row (32 / lanes rows per warp)     */
    int32_t grid_x;       /* blocks per frequency tile                             */
    double microseconds;  /* mean time of one SpMM launch                          */
} ssv_batch_tune_entry;

/* ---- library ----------------------------------------------------------- */
void ssv_version(int* major, int* minor, int* patch);
const char* ssv_last_error(void);
/* Watchdog of the device-looped solves (new: no reference counterpart). Every
 * iterative solve loops its iteration graph on the device and stops after
 * maxiter + 4 loop bodies at most (a state that never reports done: the
 * solve fails with SSV_ERR_TIMEOUT and the context stays usable).
 * max_loops > 0 sets that cap for every later solve of the process; 0
 * restores the default. */
void ssv_set_loop_guard(int32_t max_loops);
/* Device-allocation budget (new: no reference counterpart; a test hook for
 * the allocation-failure paths). bytes >= 0: every later device allocation of
 * the library is charged against the remaining budget, and one that does not
 * fit fails with SSV_ERR_ALLOC before any CUDA allocation is tried, the call
 * returning that code with its objects left as they were before it; bytes < 0
 * removes the limit (the default). Process-wide. */
void ssv_set_alloc_budget(int64_t bytes);
/* Number of CUDA devices and the name of device 0 (no allocation). */
int ssv_device_info(int* count, char* name, int name_cap);
/* Reference defaults of SolverConfig (solver_config.hpp:39-157). */
void ssv_config_default(ssv_config* cfg);

/* ---- CSR matrix (replaces SparseMatrixView / SparseMatrixCSR,
 *      include/sparsesolv/core/sparse_matrix_view.hpp:68-81,
 *      include/sparsesolv/core/sparse_matrix_csr.hpp:19-30) ---------------- */
/* Copies the CSR (int32 row_ptr[rows+1], col_idx[nnz], values[nnz] of dtype)
 * into HBM. Column indices must be sorted within each row. */
int ssv_matrix_create(int32_t rows, int32_t cols, const int32_t* row_ptr,
                      const int32_t* col_idx, const void* values, int32_t dtype,
                      ssv_matrix** out);
/* Re-uploads the values (same pattern): the reference's "matrix modified in
 * place, then Update()" semantics (compact_ams.hpp:82-86). */
int ssv_matrix_update_values(ssv_matrix* A, const void* values);
int ssv_matrix_destroy(ssv_matrix* A);
int ssv_matrix_info(const ssv_matrix* A, int32_t* rows, int32_t* cols,
                    int64_t* nnz, int32_t* dtype);
/* y = A x (SparseMatrixView::multiply, sparse_matrix_view.hpp:139-147). */
int ssv_matrix_spmv(ssv_matrix* A, const void* x, void* y);
/* Copies A's CSR arrays to host buffers (row_ptr rows + 1, col_idx and values
 * nnz entries; values as doubles, two per entry for complex). New, no
 * reference counterpart: reads back matrices assembled on the device. */
int ssv_matrix_export(const ssv_matrix* A, int32_t* row_ptr, int32_t* col_idx, void* values);

/* On-device assembly (new, no reference counterpart: NGSolve assembles the
 * reference's matrices) of a tetrahedral mesh's lowest-order Nedelec system:
 * K = sum_t nu_t Ke_t (curl-curl), M = sum_t kappa_t Me_t (mass; nu or kappa
 * NULL = 1), on the pattern of the edges sharing an element (columns sorted,
 * every entry summed in element order), and the discrete gradient G (ne x nv,
 * -1 at an edge's first vertex, +1 at its second). Host inputs: coords (nv x 3),
 * tets (nt x 4 vertex ids), tet_edges (nt x 6 edge ids of the local edges
 * (0,1),(0,2),(0,3),(1,2),(1,3),(2,3)), signs (nt x 6, +1 where the local edge
 * runs as the global one, else -1), edge_verts (ne x 2). Outputs: three new
 * F64 matrix handles. */
int ssv_hcurl_assemble(int32_t nv, const double* coords, int32_t nt, const int32_t* tets,
                       const int32_t* tet_edges, const int8_t* signs, int32_t ne,
                       const int32_t* edge_verts, const double* nu, const double* kappa,
                       ssv_matrix** K, ssv_matrix** M, ssv_matrix** G);
int ssv_matrix_spmv_dev(ssv_matrix* A, const void* d_x, void* d_y);

/* ---- SparseSolvSolver (ngsolve/sparsesolv_solvers.hpp:33-239) ---------- */
/* freedofs: one byte per row (nonzero = free) or NULL for all free. */
int ssv_solver_create(ssv_matrix* A, const uint8_t* freedofs, ssv_solver** out);
int ssv_solver_destroy(ssv_solver* s);
/* SparseSolvSolver::Solve (sparsesolv_solvers.hpp:73-160): x is the initial
 * guess on entry (free DOFs only) and the solution on return (free DOFs
 * written, constrained DOFs untouched). method: "ICCG"/"iccg", "SGSMRTR"/
 * "sgsmrtr", "CG"/"cg", "COCR"/"cocr"; any other string fails with
 * SSV_ERR_RUNTIME and the reference's message. history may be NULL. */
int ssv_solver_solve(ssv_solver* s, const char* method, const ssv_config* cfg,
                     const void* b, void* x, ssv_result* res,
                     double* history, int32_t history_cap);
/* Same, with b and x in device memory (inputs resident in HBM). */
int ssv_solver_solve_dev(ssv_solver* s, const char* method, const ssv_config* cfg,
                         const void* d_b, void* d_x, ssv_result* res,
                         double* history, int32_t history_cap);

/* Times each phase of one iteration of `method` on the buffers of the last
 * ssv_solver_solve[_dev] call of this handle (same method and options). */
int ssv_solver_profile(ssv_solver* s, const char* method, const ssv_config* cfg, int32_t reps,
                       ssv_phase_profile* out);

/* ---- preconditioners ---------------------------------------------------- */
/* ICPreconditioner factory (sparsesolv_python_export.hpp:176-207) without the
 * implicit Update(): call ssv_precond_update() to factorise. */
int ssv_ic_create(ssv_matrix* A, const uint8_t* freedofs, double shift,
                  ssv_precond** out);
/* SGSPreconditioner factory (sparsesolv_python_export.hpp:209-230) over
 * SparseSolvSGSPreconditioner (ngsolve/sparsesolv_precond.hpp:230-250) and
 * sparsesolv::SGSPreconditioner (preconditioners/sgs_preconditioner.hpp):
 * M^{-1} = (D + U)^{-1} D (D + L)^{-1} on the FreeDofs view of A, output zero
 * on constrained DOFs. ssv_precond_update computes it (the factory calls it
 * once), ssv_precond_apply[_dev] applies it, ssv_precond_destroy frees it. */
int ssv_sgs_create(ssv_matrix* A, const uint8_t* freedofs, ssv_precond** out);
/* CompactAMGPreconditioner factory (sparsesolv_python_export.hpp:359-404) over
 * CompactAMG (preconditioners/compact_amg.hpp:49-183): PMIS coarsening, direct
 * interpolation, Galerkin coarse matrices, l1-Jacobi smoothing, a direct
 * coarsest solve below 10*min_coarse rows; set up on the FreeDofs view of the
 * real matrix A (SSV_ERR_TYPE for complex); Mult = one V-cycle from x = 0 with
 * constrained outputs zeroed (ssv_precond_apply[_dev]); ssv_precond_update
 * rebuilds it from A's current values. */
int ssv_amg_create(ssv_matrix* A, const uint8_t* freedofs, double theta, int32_t max_levels,
                   int32_t min_coarse, int32_t num_smooth, ssv_precond** out);
/* AMG hierarchy of a CompactAMG handle: sizes[2l] = rows, sizes[2l+1] = nnz. */
int ssv_amg_levels(const ssv_precond* p, int32_t* sizes, int32_t cap, int32_t* num_levels);
/* Options of SparseSolvICPreconditioner (sparsesolv_precond.hpp:200-223):
 * use_abmc, abmc_block_size, abmc_num_colors, diagonal_scaling, shift and the
 * auto-shift fields are read from cfg; they take effect at the next update. */
int ssv_ic_set_config(ssv_precond* p, const ssv_config* cfg);
/* Update(): BuildSparseMatrixView + ICPreconditioner::setup
 * (sparsesolv_precond.hpp:188-191, ic_preconditioner.hpp:69-201). */
int ssv_precond_update(ssv_precond* p);
/* Mult (sparsesolv_precond.hpp:123-136): y = M^{-1} x, constrained DOFs 0. */
int ssv_precond_apply(ssv_precond* p, const void* x, void* y);
int ssv_precond_apply_dev(ssv_precond* p, const void* d_x, void* d_y);
/* Block form of Mult for the CompactAMS / ComplexCompactAMS handles (new, no
 * reference counterpart; the batched COCR driver's per-frequency apply):
 * nrhs right-hand sides (1 or 4) in one cycle, row-interleaved: x[i*nrhs + c]
 * is row i of column c (complex: Re/Im pairs). Each column gets the result of
 * ssv_precond_apply up to reduction order. Host buffers; SSV_ERR_TYPE for
 * other preconditioners, SSV_ERR_INVALID_ARG for another nrhs. */
int ssv_precond_apply_block(ssv_precond* p, int32_t nrhs, const void* x, void* y);
/* Actual IC shift after auto-shift (ICPreconditioner::actual_shift). */
int ssv_ic_actual_shift(const ssv_precond* p, double* shift);
int ssv_precond_destroy(ssv_precond* p);

/* ---- COCRSolver with external preconditioner
 *      (COCRSolverNGS::Mult, ngsolve/sparsesolv_solvers.hpp:273-369) ------- */
/* x is zeroed on entry (the reference has no initial-guess path). pre may be
 * NULL (identity). iterations receives COCRSolverNGS::GetIterations(). */
int ssv_cocr_solve(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs,
                   int32_t maxiter, double tol, int32_t printrates,
                   const void* b, void* x, int32_t* iterations);
int ssv_cocr_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs,
                       int32_t maxiter, double tol, int32_t printrates,
                       const void* d_b, void* d_x, int32_t* iterations);

/* ---- refined COCR: the mixed-precision form's Krylov driver (new: no
 *      reference counterpart; each cycle is the COCRSolverNGS recurrence) ----
 * FP64 defect correction around COCR: cycles of the recurrence of
 * ssv_cocr_solve, each started from the FP64 true residual r = P(b - A x) of
 * the current x (rt = M^{-1} r, p = rt, q = P A p) and ended once its
 * recurrence residual has dropped by restart_drop (0 < restart_drop < 1)
 * from the residual it started from (or on tol, a breakdown, maxiter). The
 * solve ends when the true relative residual ||P(b - A x)|| / ||P b|| <= tol.
 * This is what keeps an FP32-form preconditioner usable under COCR: the
 * plain recurrence (rt -= alpha M^{-1} q) assumes an exactly linear M^{-1}
 * and stalls near M^{-1}'s rounding level. The breakdown thresholds (1e-30 on
 * |mu|, |rho|) scale with (||r_start|| / ||P b||)^2. x is zeroed on entry.
 * info: iterations = recurrence steps over all cycles, cycles, converged
 * (true residual <= tol), true_residual (relative, FP64). */
typedef struct ssv_refine_info {
    int32_t iterations;
    int32_t cycles;
    int32_t converged;
    int32_t pad_;
    double true_residual;
} ssv_refine_info;
int ssv_cocr_refined_solve(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter,
                           double tol, double restart_drop, int32_t printrates, const void* b, void* x,
                           ssv_refine_info* info);
int ssv_cocr_refined_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter,
                               double tol, double restart_drop, int32_t printrates, const void* d_b,
                               void* d_x, ssv_refine_info* info);
/* Measurement hook (no reference counterpart): kernels launched by the last
 * ssv_cocr_solve[_dev] / ssv_cocr_refined_solve[_dev] of the calling thread
 * (graph kernel nodes times executed loop bodies, plus the set-up launches). */
int ssv_cocr_last_launches(int64_t* launches);

/* ---- Compact AMS (include/sparsesolv/preconditioners/compact_ams.hpp,
 *      complex_compact_ams.hpp; factories sparsesolv_python_export.hpp:410-530) */
/* CompactAMS(mat, grad, freedofs, coord_x/y/z, cycle_type, num_smooth,
 * theta, print_level, correction_weight) ctor + Setup (compact_ams.hpp:53-77,
 * 243-271), or with complex_form != 0 ComplexCompactAMS (complex_compact_ams.hpp:
 * 31-89): A is the real HCurl (auxiliary) matrix, G the discrete gradient
 * (rows = HCurl DOFs, cols = H1 DOFs), coordinates of the H1 vertices. The
 * complex form applies to complex vectors of length ndof_complex (0 = rows of
 * A). Applied with ssv_precond_apply[_dev]; used by ssv_pcg_solve and
 * ssv_cocr_solve. */
int ssv_ams_create(ssv_matrix* A, ssv_matrix* G, const uint8_t* freedofs,
                   const double* coord_x, const double* coord_y, const double* coord_z,
                   int32_t cycle_type, int32_t num_smooth, double theta,
                   double correction_weight, int32_t complex_form, int32_t ndof_complex,
                   ssv_precond** out);
/* Update() / Update(new_mat) (compact_ams.hpp:82-97): rebuild the matrix part
 * (BC matrix, Galerkin products, AMG hierarchies) keeping the geometry.
 * new_A may be NULL (re-read A's current values). Dimension mismatch ->
 * SSV_ERR_INVALID_ARG (the reference's std::invalid_argument). */
int ssv_ams_update(ssv_precond* p, ssv_matrix* new_A);
/* Hierarchy of subspace s (0 = gradient, 1..3 = Nedelec x, y, z): per level
 * rows and nnz into sizes[2l], sizes[2l+1]. */
int ssv_ams_levels(const ssv_precond* p, int32_t subspace, int32_t* sizes, int32_t cap,
                   int32_t* num_levels);
/* New (no reference counterpart): the FP32-preconditioner form. With
 * SSV_PREC_FP32_NODAL (AMS only) the gradient hierarchy stays FP64 and the
 * three nodal hierarchies take the FP32 form (the split that keeps COCR
 * convergent on mass-dominated eddy-current systems, whose gradient-space
 * matrices span many decades). With
 * SSV_PREC_FP32 every matrix of the AMS hierarchy, the l1 norms and the work
 * vectors of the cycle are FP32; the coarsest solve and the cycle's FP64
 * input/output stay FP64. Switching re-uploads the hierarchy (no new set-up);
 * Update() keeps the current form. */
int ssv_ams_set_precision(ssv_precond* p, int32_t precision);
int ssv_ams_get_precision(const ssv_precond* p, int32_t* precision);
/* Measurement hook (no reference counterpart): per-phase device time of one
 * AMS cycle on nrhs (1 or 4) right-hand sides -- the whole cycle, one fine
 * residual pass, one fine smoothing pass, the gradient V-cycle, the three
 * nodal V-cycles, the G and Pi transfers -- each re-launched reps times
 * between CUDA events, with the algorithmic bytes of one execution. flags:
 * SSV_PROFILE_COLD times every launch alone after evicting the L2 (a 256 MiB
 * write; the buffer is kept until exit), the HBM-bound case; 0 times the
 * launches back to back (operands that fit in L2 stay there). */
#define SSV_PROFILE_COLD 1
int ssv_ams_profile(ssv_precond* p, int32_t nrhs, int32_t reps, int32_t flags, ssv_phase_profile* out);
/* Measurement hook (no reference counterpart): per-level device time (ms,
 * warm, mean of reps back-to-back launches) of one subspace's V-cycle on one
 * right-hand side: the down product R_l into ms_r[l] and the up product U_l
 * into ms_u[l] for every level run one by one (cap entries at most), their
 * launch shapes (lanes * 10 + rows per group) in shape_r / shape_u, and the
 * last step (the dense tail, or the coarsest solve's two launches) in
 * *last_ms. *levels receives the number of levels run one by one, the last
 * included. */
int ssv_ams_profile_levels(ssv_precond* p, int32_t subspace, int32_t reps, double* ms_r, double* ms_u,
                           int32_t* shape_r, int32_t* shape_u, int32_t cap, double* last_ms, int32_t* levels);
/* Measurement hook (no reference counterpart): wall seconds of the last
 * set-up of p (create, Update() or a precision switch) into times[0..3]:
 * total, host hierarchy (BC matrix, Galerkin products, coarsening,
 * interpolation, coarse operators, coarsest factors), fused level products,
 * launch-shape tuner; the rest of the total is device uploads. */
int ssv_ams_setup_times(const ssv_precond* p, double* times);
/* Parity hook (no reference counterpart): level `level` of subspace s
 * (0 gradient, 1..3 Nedelec x, y, z) of the hierarchy as set up, FP64 and
 * unscaled: what = 0 the level matrix A_l (CompactAMG Level::A), 1 the
 * interpolation P_l. *nnz receives its nonzeros; row_ptr (rows + 1),
 * col_idx and values are filled when cap >= *nnz. *on_device (may be NULL)
 * = 1 when the hierarchy was set up on the device. */
int ssv_ams_level_matrix(const ssv_precond* p, int32_t subspace, int32_t level, int32_t what, int32_t* row_ptr,
                         int32_t* col_idx, double* values, int32_t cap, int32_t* nnz, int32_t* on_device);
/* Parity hook (no reference counterpart): one subspace correction of the
 * cycle on its own, in the current form. From the residual r (rows x nv host
 * doubles, nv = 2 for ComplexCompactAMS: Re/Im pairs): b_s = the restricted
 * residual (G^T r, or Pi_s^T r), x_s = the subspace V-cycle's result (both
 * h1_rows x nv, in the hierarchy's coordinates: diagonally scaled where the
 * hierarchy is FP32), corr = w P_s x_s (rows x nv). subspace: 0 gradient,
 * 1..3 Nedelec x, y, z. */
int ssv_ams_subspace_apply(ssv_precond* p, int32_t subspace, const double* r, double* b_s, double* x_s,
                           double* corr);

/* ---- CG with an external preconditioner (new: the reference's AMS scripts
 *      drive it with NGSolve's krylovspace.CGSolver) ---------------------------
 * The sparsesolv::CGSolver recurrence (solvers/cg_solver.hpp:64-146,
 * iterative_solver.hpp:135-279) on the FreeDofs view of A, z = M^{-1} r by
 * pre (NULL = identity); x is the initial guess on entry (free entries) and
 * the solution on return. */
int ssv_pcg_solve(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, const ssv_config* cfg,
                  const void* b, void* x, ssv_result* res, double* history, int32_t history_cap);
int ssv_pcg_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, const ssv_config* cfg,
                      const void* d_b, void* d_x, ssv_result* res, double* history,
                      int32_t history_cap);

/* GMRESSolver (GMRESSolverNGS, ngsolve/sparsesolv_solvers.hpp:409-584;
 * factory sparsesolv_python_export.hpp:643-697): right-preconditioned GMRES
 * with modified Gram-Schmidt and Givens rotations, x0 = 0, restart after
 * `restart` steps (0 = maxiter), stop when |g_{j+1}| / ||P b|| < tol;
 * iterations = total Arnoldi steps. pre may be NULL (identity). */
int ssv_gmres_solve(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter, double tol,
                    int32_t restart, const void* b, void* x, int32_t* iterations);
int ssv_gmres_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter, double tol,
                        int32_t restart, const void* d_b, void* d_x, int32_t* iterations);

/* ---- host-side set-up logic exposed for parity checks (no device work) --- */
/* ABMCSchedule::build (include/sparsesolv/core/abmc_ordering.hpp:83-121).
 * color_offsets needs room for n+1 entries, block_offsets n+1, ordering and
 * reverse n each. */
int ssv_abmc_build(int32_t n, const int32_t* row_ptr, const int32_t* col_idx,
                   int32_t block_size, int32_t target_colors,
                   int32_t* num_colors, int32_t* num_blocks,
                   int32_t* color_offsets, int32_t* block_offsets,
                   int32_t* ordering, int32_t* reverse_ordering);
/* LevelSchedule::build_from_lower / build_from_upper
 * (include/sparsesolv/core/level_schedule.hpp:58-135): level_of[i] = level of
 * row i; returns the level count in num_levels. upper != 0 builds from an
 * upper-triangular pattern. */
int ssv_level_schedule(int32_t n, const int32_t* row_ptr, const int32_t* col_idx,
                       int32_t upper, int32_t* level_of, int32_t* num_levels);
/* compute_rcm_ordering (include/sparsesolv/core/rcm_ordering.hpp:38-140), the
 * pre-ordering of the abmc_use_rcm path: ordering[old] = new,
 * reverse_ordering[new] = old (n entries each). */
int ssv_rcm_order(int32_t n, const int32_t* row_ptr, const int32_t* col_idx, int32_t* ordering,
                  int32_t* reverse_ordering);

/* ---- batched COCR over a frequency family (new: no reference counterpart) -
 * A_f = K + j*omega_f*M for num_freq frequencies (K, M real, square, one size;
 * their patterns are merged), nrhs right-hand sides per frequency (1 or 4),
 * one ComplexCompactAMS preconditioner per frequency (pre[f], NULL =
 * identity; FP64 or FP32 form). Every one of the num_freq*nrhs columns runs
 * the COCRSolverNGS recurrence (ngsolve/sparsesolv_solvers.hpp:273-369) on the
 * FreeDofs view: x0 = 0, stop when ||r||/||b|| <= tol, iterations = j+1 on
 * convergence, maxiter otherwise; a finished column is frozen while the rest
 * continue. One SpMM pass reads K and M once per tile of frequencies; the tile,
 * lanes per row and grid are picked at create time by timing the candidates
 * on this matrix (ssv_batch_tuning lists them). The iteration is one CUDA
 * graph. The preconditioners and matrices must outlive the batch; Update() of
 * a preconditioner is picked up by the next solve. */
int ssv_batch_create(ssv_matrix* K, ssv_matrix* M, int32_t num_freq, const double* omegas,
                     ssv_precond* const* pre, int32_t nrhs, const uint8_t* freedofs,
                     ssv_batch** out);
int ssv_batch_destroy(ssv_batch* b);
/* rhs, sol: num_freq*nrhs complex vectors of n entries, [f][r][row]
 * (host pointers; _dev: device pointers). iterations, converged (int32) and
 * residuals (final ||r||/||b||, double) get num_freq*nrhs entries; each may be
 * NULL. */
int ssv_batch_cocr_solve(ssv_batch* b, int32_t maxiter, double tol, const void* rhs, void* sol,
                         int32_t* iterations, int32_t* converged, double* residuals);
int ssv_batch_cocr_solve_dev(ssv_batch* b, int32_t maxiter, double tol, const void* d_rhs, void* d_sol,
                             int32_t* iterations, int32_t* converged, double* residuals);
/* Residual replacement: every `every`-th step sets the preconditioned
 * residual to M^{-1} r instead of its recurrence (0 = never, < 0 = automatic:
 * every 10th step when a preconditioner is in the FP32 form, whose rounding
 * makes it not exactly linear, so the recurrence drifts; never otherwise). */
int ssv_batch_set_replacement(ssv_batch* b, int32_t every);
/* Refined form (new: no reference counterpart; the per-column form of
 * ssv_cocr_refined_solve): restart_drop in (0, 1) makes every column run
 * cycles of the recurrence, each started from its FP64 true residual and
 * ended once its residual has dropped by restart_drop; a column is done when
 * its true relative residual is <= tol (converged) or it is out of
 * iterations. residuals then hold the true relative residuals, iterations the
 * recurrence steps over all cycles. 0 (the default) = the plain recurrence.
 * Residual replacement is off in the refined form. */
int ssv_batch_set_refinement(ssv_batch* b, double restart_drop);
/* Cycles (graph loops) of the last solve (1 for the plain form). */
int ssv_batch_last_cycles(const ssv_batch* b, int32_t* cycles);
/* Autotuner record: up to cap entries, *count = entries measured, *chosen =
 * index of the shape in use. */
int ssv_batch_tuning(const ssv_batch* b, ssv_batch_tune_entry* entries, int32_t cap, int32_t* count,
                     int32_t* chosen);
/* Device time of the last solve (CUDA events on the library's stream): the
 * whole solve and its iteration loop, executed loop bodies, kernel launches. */
int ssv_batch_last_timing(const ssv_batch* b, double* device_ms, double* loop_ms, int32_t* loops,
                          int64_t* kernel_launches);

/* ---- learned initial guess (new: no reference counterpart) ----------------
 * A per-sample MLP out = w2 . relu(W1 x + b1) + b2 with in_dim inputs
 * (<= 32) and `hidden` units (<= 128), FP32, trained and evaluated on the GPU
 * by the library's own kernels. Parameters as one float array: W1 (hidden x
 * in_dim, row-major), b1 (hidden), w2 (hidden), b2 (1). Training minimises the
 * mean squared error with Adam (beta 0.9 / 0.999, eps 1e-8) over minibatches
 * of a fresh permutation per epoch; gradients are summed in a fixed order. */
int ssv_mlp_create(int32_t in_dim, int32_t hidden, uint64_t seed, ssv_mlp** out);
int ssv_mlp_destroy(ssv_mlp* m);
int ssv_mlp_num_params(const ssv_mlp* m, int32_t* count);
int ssv_mlp_get_params(const ssv_mlp* m, float* params);
/* Also resets the Adam state. */
int ssv_mlp_set_params(ssv_mlp* m, const float* params);
/* Gradient of the mean squared error over n samples (X row-major n x in_dim,
 * host pointers) and the loss -- the hook the CPU gradient check uses. */
int ssv_mlp_gradients(ssv_mlp* m, const float* X, const float* y, int64_t n, float* grad, float* loss);
/* Minibatch Adam on device-resident data; *loss = loss of the last batch. */
int ssv_mlp_train_dev(ssv_mlp* m, const float* d_X, const float* d_y, int64_t n, int32_t epochs,
                      int32_t batch, float lr, uint64_t seed, float* loss);
int ssv_mlp_predict_dev(ssv_mlp* m, const float* d_X, int64_t n, float* d_out);

/* ---- allocation-free SpMV + dot (no counterpart in the reference) -------- */
/* y = A x and *d_dot = x^T y for a real CSR matrix (int32 row_ptr/col_idx,
 * double values), every pointer in device memory, for callers that must not
 * allocate device memory (a framework that owns the device's memory pool, a
 * fixed memory budget, a real-time loop where an allocation could stall or
 * fail). It calls no cudaMalloc/cudaFree or allocating library routine: its
 * scratch (one partial sum per 32 rows plus a counter) is a fixed ~512 KB
 * array inside the library, held by every GPU that loads it until exit.
 * Limit: rows <= 2,097,152 (larger sizes fail with SSV_ERR_INVALID_ARG).
 * The first call on a device looks up the array's device address (make it
 * before any stream capture) and keeps it for the process: calls must not
 * span a cudaDeviceReset. Calls that overlap on the GPU share the array and
 * race. Every pointer must be device memory (host pointers are refused with
 * SSV_ERR_INVALID_ARG). Runs on the legacy default stream and is synchronous
 * on return; callers that produced the inputs on a non-blocking stream must
 * synchronise that stream first. */
int ssv_spmv_dot_noalloc(int32_t rows, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                         const double* d_values, const double* d_x, double* d_y, double* d_dot);

#ifdef __cplusplus
}
#endif

#endif /* SPARSESOLV_B200_H */
