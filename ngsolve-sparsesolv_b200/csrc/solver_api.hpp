// solver_api.hpp -- non-template entry points between the C ABI layer and
// the device orchestration.
#pragma once

#include "objects.cuh"

namespace ssv {

int parse_method(const char* m);
void solver_solve_dev(ssv_solver* sv, const char* method, const ssv_config& cfg, const void* d_b,
                      void* d_x, ssv_result* res, double* hist, int hist_cap);
void solver_profile(ssv_solver* sv, const char* method, const ssv_config& cfg, int reps,
                    ssv_phase_profile* out);
void precond_update(ssv_precond* p);
void precond_apply_dev(ssv_precond* p, const void* d_x, void* d_y);
double precond_actual_shift(const ssv_precond* p);
void matrix_spmv_dev(ssv_matrix* A, const void* d_x, void* d_y);
void cocr_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* d_fd, int maxiter, double tol,
                    int printrates, const void* d_b, void* d_x, int* iterations);
void cocr_refined_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* d_fd, int maxiter, double tol,
                            double restart_drop, int printrates, const void* d_b, void* d_x,
                            ssv_refine_info* info);
int64_t cocr_last_launches();
void gmres_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* d_fd, int maxiter, double tol, int restart,
                     const void* d_b, void* d_x, int* iterations);
void mrtr_forget(const ssv_solver* s);
void cocr_forget(const ssv_matrix* A);

template <typename S>
void ic_apply_dev(ssv_precond* p, const S* x, S* y, const KState* st, cudaStream_t s);
// SGSPreconditioner (sgs.cu): Update() and Mult
void sgs_update(ssv_precond* p);
template <typename S>
void sgs_apply_dev(ssv_precond* p, const S* x, S* y, const KState* st, cudaStream_t s);

// y = M^{-1} x for any preconditioner handle, stream-ordered, no host sync
// (so it can sit inside a captured iteration graph).
template <typename S>
void precond_apply_any(ssv_precond* p, const S* x, S* y, const KState* st, cudaStream_t s);
template <>
void precond_apply_any<double>(ssv_precond* p, const double* x, double* y, const KState* st, cudaStream_t s);
template <>
void precond_apply_any<zdouble>(ssv_precond* p, const zdouble* x, zdouble* y, const KState* st, cudaStream_t s);
// Changes whenever the preconditioner's device structures are rebuilt.
unsigned precond_generation(const ssv_precond* p);

// on-device assembly of a tetrahedral mesh's Nedelec K, M and gradient G (assembly.cu)
void hcurl_assemble(int nv, const double* xyz, int nt, const int* tets, const int* tet_edges, const int8_t* signs,
                    int ne, const int* edge_verts, const double* nu, const double* kappa, ssv_matrix** K,
                    ssv_matrix** M, ssv_matrix** G);

// Compact AMS (ams.cu)
AmsState* ams_create(const ssv_matrix* A, const ssv_matrix* G, const uint8_t* fd, const double* cx,
                     const double* cy, const double* cz, int cycle_type, int num_smooth, double theta, double w,
                     int complex_form, int ndof_complex);
void ams_update(AmsState* a, const ssv_matrix* A);
// CompactAMGPreconditioner (ams.cu): host set-up, FP64 V-cycle on the device
AmgOnly* amg_create(const ssv_matrix* A, const uint8_t* fd, double theta, int max_levels, int min_coarse,
                    int num_smooth);
void amg_update(AmgOnly* g, const ssv_matrix* A);
int amg_levels(const AmgOnly* g, int* sizes, int cap);
int ams_levels(const AmsState* a, int sub, int* sizes, int cap);
int ams_level_matrix(const AmsState* a, int sub, int l, int what, int* rp, int* ci, double* v, int cap);
bool ams_on_device(const AmsState* a);
void ams_set_precision(AmsState* a, int precision);
// wall seconds of the last set-up: total, host hierarchy, fused products, shape tuner
void ams_setup_times(const AmsState* a, double* t);
int ams_precision(const AmsState* a);
// Block application to nrhs right-hand sides ([row][rhs] interleaved; complex
// form: Re/Im pairs), after ams_reserve_block(a, nrhs).
void ams_reserve_block(AmsState* a, int nrhs);
void ams_profile(AmsState* a, int nrhs, int reps, int flags, ssv_phase_profile* out);
int ams_profile_levels(AmsState* a, int sub, int reps, double* ms_r, double* ms_u, int* shape_r, int* shape_u,
                       int cap, double* last_ms);
void ams_apply_block(AmsState* a, const double* in, double* out, int nrhs, const KState* st, cudaStream_t s);
// one subspace correction on its own (host arrays; parity hook)
void ams_subspace_apply(AmsState* a, int sub, const double* r, double* bs, double* xs, double* corr);

// Batched COCR over a frequency family (batch.cu)
ssv_batch* batch_create(ssv_matrix* K, ssv_matrix* M, int F, const double* omegas, ssv_precond* const* pre, int R,
                        const uint8_t* fd);
void batch_destroy(ssv_batch* B);
void batch_cocr_solve_dev(ssv_batch* B, int maxiter, double tol, const void* d_b, void* d_x, int* iters, int* conv,
                          double* res);
void batch_cocr_solve_host(ssv_batch* B, int maxiter, double tol, const void* b, void* x, int* iters, int* conv,
                           double* res);
int batch_tuning(const ssv_batch* B, ssv_batch_tune_entry* e, int cap, int* chosen);
void batch_last_timing(const ssv_batch* B, double* ms, double* loop_ms, int* loops, int64_t* launches,
                       int* cycles);
void batch_set_replacement(ssv_batch* B, int every);
void batch_set_refinement(ssv_batch* B, double restart_drop);

// Learned initial-guess MLP (mlp.cu)
ssv_mlp* mlp_create(int D, int H, uint64_t seed);
void mlp_destroy(ssv_mlp* m);
int mlp_nparams(const ssv_mlp* m);
void mlp_get_params(const ssv_mlp* m, float* p);
void mlp_set_params(ssv_mlp* m, const float* p);
void mlp_gradients_host(ssv_mlp* m, const float* X, const float* Y, int64_t n, float* grad, float* loss);
void mlp_train_dev(ssv_mlp* m, const float* X, const float* Y, int64_t n, int epochs, int batch, float lr,
                   uint64_t seed, float* last_loss);
void mlp_predict_dev(ssv_mlp* m, const float* X, int64_t n, float* out);

// CG with an external preconditioner and an initial guess (cocr_ngs.cu)
void pcg_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* d_fd, const ssv_config& cfg, const void* d_b,
                   void* d_x, ssv_result* res, double* hist, int hist_cap);

}  // namespace ssv
