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
void mrtr_forget(const ssv_solver* s);
void cocr_forget(const ssv_matrix* A);

template <typename S>
void ic_apply_dev(ssv_precond* p, const S* x, S* y, const KState* st, cudaStream_t s);

}  // namespace ssv
