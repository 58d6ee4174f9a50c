// ref_driver.cpp -- TEST INFRASTRUCTURE: drives the reference's own,
// unmodified headers (ksugahar/ngsolve-sparsesolv, include/sparsesolv/, the
// NGSolve-free half) so that the oracle and the GPU path can be pinned against
// the reference itself. oracle/build_oracle.py compiles it, with -I pointing
// at the reference checkout, into oracle/_ref/libssv_ref.so (git-ignored).
//
// The NGSolve adapter (ngsolve/sparsesolv_solvers.hpp) cannot compile without
// NGSolve, so ref_solve restates its few lines of FreeDofs handling
// (BuildSparseMatrixView, ngsolve/sparsesolv_precond.hpp:60-74, and
// SparseSolvSolver::Solve, ngsolve/sparsesolv_solvers.hpp:81-137) around the
// reference's own solve_iccg / solve_sgsmrtr / CGSolver / COCRSolver calls.
#include <sparsesolv/sparsesolv.hpp>

#include <omp.h>

#include <chrono>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "../include/sparsesolv_b200.h"

namespace {

thread_local std::string g_err;

sparsesolv::SolverConfig to_config(const ssv_config& c) {
    sparsesolv::SolverConfig s;
    s.tolerance = c.tolerance;
    s.max_iterations = c.max_iterations;
    s.abs_tolerance = c.abs_tolerance;
    s.norm_type = c.norm_type == SSV_NORM_RHS ? sparsesolv::NormType::RHS
                : c.norm_type == SSV_NORM_INITIAL_RESIDUAL ? sparsesolv::NormType::InitialResidual
                : sparsesolv::NormType::Custom;
    s.custom_norm = c.custom_norm;
    s.shift_parameter = c.shift_parameter;
    s.diagonal_scaling = c.diagonal_scaling != 0;
    s.auto_shift = c.auto_shift != 0;
    s.shift_increment = c.shift_increment;
    s.max_shift_value = c.max_shift_value;
    s.min_diagonal_threshold = c.min_diagonal_threshold;
    s.zero_diagonal_replacement = c.zero_diagonal_replacement;
    s.max_shift_trials = c.max_shift_trials;
    s.divergence_check = c.divergence_check ? sparsesolv::DivergenceCheck::StagnationCount
                                            : sparsesolv::DivergenceCheck::None;
    s.divergence_threshold = c.divergence_threshold;
    s.divergence_count = c.divergence_count;
    s.save_best_result = c.save_best_result != 0;
    s.save_residual_history = c.save_residual_history != 0;
    s.conjugate = c.conjugate != 0;
    s.use_abmc = c.use_abmc != 0;
    s.abmc_block_size = c.abmc_block_size;
    s.abmc_num_colors = c.abmc_num_colors;
    s.abmc_reorder_spmv = c.abmc_reorder_spmv != 0;
    s.abmc_use_rcm = c.abmc_use_rcm != 0;
    return s;
}

template <typename S>
int solve_impl(int n, const int* rp, const int* ci, const S* vals, const unsigned char* fd,
               const std::string& method, const ssv_config& cfg, const S* b, S* x,
               ssv_result* res, double* hist, int hist_cap) {
    using namespace sparsesolv;
    const int nnz = rp[n];
    std::vector<S> mv(vals, vals + nnz);
    std::vector<S> bm(b, b + n), xm(x, x + n);
    if (fd) {
        for (int i = 0; i < n; ++i)
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                const int j = ci[k];
                if (!fd[i]) mv[k] = (j == i) ? S(1) : S(0);
                else if (!fd[j]) mv[k] = S(0);
            }
        for (int i = 0; i < n; ++i) {
            if (!fd[i]) { bm[i] = S(0); xm[i] = S(0); }
        }
    }
    SparseMatrixView<S> view(n, n, rp, ci, mv.data());
    SolverConfig sc = to_config(cfg);
    SolverResult r;
    auto t0 = std::chrono::steady_clock::now();
    if (method == "ICCG" || method == "iccg") {
        r = solve_iccg(view, bm.data(), xm.data(), n, sc);
    } else if (method == "SGSMRTR" || method == "sgsmrtr") {
        r = solve_sgsmrtr(view, bm.data(), xm.data(), n, sc);
    } else if (method == "CG" || method == "cg") {
        CGSolver<S> solver; solver.set_config(sc);
        r = solver.solve(view, bm.data(), xm.data(), n, nullptr);
    } else if (method == "COCR" || method == "cocr") {
        COCRSolver<S> solver; solver.set_config(sc);
        r = solver.solve(view, bm.data(), xm.data(), n, nullptr);
    } else {
        g_err = "SparseSolvSolver: Unknown method '" + method + "'. Available: ICCG, SGSMRTR, CG, COCR";
        return SSV_ERR_RUNTIME;
    }
    auto t1 = std::chrono::steady_clock::now();
    for (int i = 0; i < n; ++i)
        if (!fd || fd[i]) x[i] = xm[i];
    std::memset(res, 0, sizeof(*res));
    res->converged = r.converged ? 1 : 0;
    res->iterations = r.iterations;
    res->final_residual = r.final_residual;
    res->history_total = static_cast<int>(r.residual_history.size());
    res->history_len = res->history_total < hist_cap ? res->history_total : hist_cap;
    for (int i = 0; i < res->history_len; ++i) hist[i] = r.residual_history[i];
    res->solve_seconds = std::chrono::duration<double>(t1 - t0).count();
    return 0;
}

template <typename S>
int ic_mult_impl(int n, const int* rp, const int* ci, const S* vals, const unsigned char* fd,
                 const ssv_config& cfg, const S* x, S* y, double* actual_shift) {
    using namespace sparsesolv;
    const int nnz = rp[n];
    std::vector<S> mv(vals, vals + nnz);
    if (fd) {
        for (int i = 0; i < n; ++i)
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                const int j = ci[k];
                if (!fd[i]) mv[k] = (j == i) ? S(1) : S(0);
                else if (!fd[j]) mv[k] = S(0);
            }
    }
    SparseMatrixView<S> view(n, n, rp, ci, mv.data());
    ICPreconditioner<S> pre(cfg.shift_parameter);
    pre.set_config(to_config(cfg));
    pre.setup(view);
    pre.apply(x, y, n);
    if (fd)
        for (int i = 0; i < n; ++i)
            if (!fd[i]) y[i] = S(0);
    if (actual_shift) *actual_shift = pre.actual_shift();
    return 0;
}

template <typename S>
int sgs_mult_impl(int n, const int* rp, const int* ci, const S* vals, const unsigned char* fd, const S* x, S* y) {
    using namespace sparsesolv;
    const int nnz = rp[n];
    std::vector<S> mv(vals, vals + nnz);
    if (fd) {
        for (int i = 0; i < n; ++i)
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                const int j = ci[k];
                if (!fd[i]) mv[k] = (j == i) ? S(1) : S(0);
                else if (!fd[j]) mv[k] = S(0);
            }
    }
    SparseMatrixView<S> view(n, n, rp, ci, mv.data());
    SGSPreconditioner<S> pre;
    pre.setup(view);
    pre.apply(x, y, n);
    if (fd)
        for (int i = 0; i < n; ++i)
            if (!fd[i]) y[i] = S(0);
    return 0;
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

void ref_set_threads(int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
}

int ref_get_threads(void) { return omp_get_max_threads(); }

int ref_solve(int n, const int* rp, const int* ci, const void* vals, int dtype,
              const unsigned char* freedofs, const char* method, const ssv_config* cfg,
              const void* b, void* x, ssv_result* res, double* hist, int hist_cap) {
    try {
        if (dtype == SSV_F64)
            return solve_impl<double>(n, rp, ci, static_cast<const double*>(vals), freedofs,
                                      method ? method : "", *cfg, static_cast<const double*>(b),
                                      static_cast<double*>(x), res, hist, hist_cap);
        using Z = std::complex<double>;
        return solve_impl<Z>(n, rp, ci, static_cast<const Z*>(vals), freedofs, method ? method : "",
                             *cfg, static_cast<const Z*>(b), static_cast<Z*>(x), res, hist, hist_cap);
    } catch (const std::exception& e) {
        g_err = e.what();
        return SSV_ERR_RUNTIME;
    }
}

int ref_ic_mult(int n, const int* rp, const int* ci, const void* vals, int dtype,
                const unsigned char* freedofs, const ssv_config* cfg, const void* x, void* y,
                double* actual_shift) {
    try {
        if (dtype == SSV_F64)
            return ic_mult_impl<double>(n, rp, ci, static_cast<const double*>(vals), freedofs, *cfg,
                                        static_cast<const double*>(x), static_cast<double*>(y),
                                        actual_shift);
        using Z = std::complex<double>;
        return ic_mult_impl<Z>(n, rp, ci, static_cast<const Z*>(vals), freedofs, *cfg,
                               static_cast<const Z*>(x), static_cast<Z*>(y), actual_shift);
    } catch (const std::exception& e) {
        g_err = e.what();
        return SSV_ERR_RUNTIME;
    }
}

int ref_abmc_build(int n, const int* rp, const int* ci, int block_size, int target_colors,
                   int* num_colors, int* num_blocks, int* color_offsets, int* block_offsets,
                   int* ordering, int* reverse) {
    sparsesolv::ABMCSchedule s;
    s.build(rp, ci, n, block_size, target_colors);
    *num_colors = s.num_colors();
    *num_blocks = s.num_blocks();
    if (n <= 0) return 0;
    std::memcpy(color_offsets, s.color_offsets.data(), sizeof(int) * s.color_offsets.size());
    std::memcpy(block_offsets, s.block_offsets.data(), sizeof(int) * s.block_offsets.size());
    std::memcpy(ordering, s.ordering.data(), sizeof(int) * n);
    std::memcpy(reverse, s.reverse_ordering.data(), sizeof(int) * n);
    // color_blocks is the identity map in the reference's numbering; checked here
    for (size_t k = 0; k < s.color_blocks.size(); ++k)
        if (s.color_blocks[k] != static_cast<int>(k)) return SSV_ERR_RUNTIME;
    return 0;
}

int ref_level_schedule(int n, const int* rp, const int* ci, int upper, int* level_of,
                       int* num_levels) {
    sparsesolv::LevelSchedule ls;
    if (upper) ls.build_from_upper(rp, ci, n);
    else ls.build_from_lower(rp, ci, n);
    *num_levels = ls.num_levels();
    for (int l = 0; l < ls.num_levels(); ++l)
        for (int r : ls.levels[l]) level_of[r] = l;
    return 0;
}

int ref_sgs_mult(int n, const int* rp, const int* ci, const void* vals, int dtype, const unsigned char* freedofs,
                 const void* x, void* y) {
    try {
        if (dtype == SSV_F64)
            return sgs_mult_impl<double>(n, rp, ci, static_cast<const double*>(vals), freedofs,
                                         static_cast<const double*>(x), static_cast<double*>(y));
        using Z = std::complex<double>;
        return sgs_mult_impl<Z>(n, rp, ci, static_cast<const Z*>(vals), freedofs, static_cast<const Z*>(x),
                                static_cast<Z*>(y));
    } catch (const std::exception& e) {
        g_err = e.what();
        return SSV_ERR_RUNTIME;
    }
}

int ref_rcm(int n, const int* rp, const int* ci, int* ordering, int* reverse) {
    std::vector<int> o, r;
    sparsesolv::compute_rcm_ordering(rp, ci, n, o, r);
    if (n <= 0) return 0;
    std::memcpy(ordering, o.data(), sizeof(int) * n);
    std::memcpy(reverse, r.data(), sizeof(int) * n);
    return 0;
}

}  // extern "C"
