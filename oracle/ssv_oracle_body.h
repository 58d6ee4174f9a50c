/*
 * ssv_oracle_body.h -- TEST INFRASTRUCTURE (the oracle), not product code.
 *
 * Scalar-generic body of the CPU restatement, included by ssv_oracle.c once
 * with T = double and once with T = double _Complex. Macros provided by the
 * includer: T, SFX(name), IS_COMPLEX, CONJ(a), NORM2(a) (= |a|^2, std::norm),
 * SABS(a) (= std::abs), FROM_REAL(d).
 *
 * Every routine is serial and follows the reference's operation order per row,
 * so its results equal the reference's single-thread results bit for bit
 * (threaded reference runs differ only in the summation order of reductions).
 */

/* ------------------------------------------------------------------------ */
/* CSR helpers                                                               */
/* ------------------------------------------------------------------------ */

/* SparseMatrixView::multiply, core/sparse_matrix_view.hpp:139-147 */
static void SFX(spmv)(int n, const int* rp, const int* ci, const T* v, const T* x, T* y) {
    for (int i = 0; i < n; ++i) {
        T s = FROM_REAL(0.0);
        for (int k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
        y[i] = s;
    }
}

/* SparseMatrixView::operator() (binary search), sparse_matrix_view.hpp:124-132 */
static T SFX(entry)(const int* rp, const int* ci, const T* v, int i, int j) {
    int lo = rp[i], hi = rp[i + 1];
    while (lo < hi) {
        int mid = lo + (hi - lo) / 2;
        if (ci[mid] < j) lo = mid + 1; else hi = mid;
    }
    if (lo < rp[i + 1] && ci[lo] == j) return v[lo];
    return FROM_REAL(0.0);
}

typedef struct {
    int rows, cols;
    int* rp; int* ci; T* v;
} SFX(csr);

static void SFX(csr_free)(SFX(csr)* m) {
    free(m->rp); free(m->ci); free(m->v);
    m->rp = NULL; m->ci = NULL; m->v = NULL; m->rows = m->cols = 0;
}

/* SparseMatrixCSR::transpose, core/sparse_matrix_csr.hpp:47-72 */
static void SFX(csr_transpose)(const SFX(csr)* a, SFX(csr)* t) {
    int nnz = a->rp[a->rows];
    t->rows = a->cols; t->cols = a->rows;
    t->rp = (int*)calloc((size_t)a->cols + 1, sizeof(int));
    t->ci = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    t->v = (T*)malloc(sizeof(T) * (size_t)(nnz > 0 ? nnz : 1));
    for (int k = 0; k < nnz; ++k) t->rp[a->ci[k] + 1]++;
    for (int i = 0; i < a->cols; ++i) t->rp[i + 1] += t->rp[i];
    int* cnt = (int*)calloc((size_t)a->cols + 1, sizeof(int));
    for (int i = 0; i < a->rows; ++i)
        for (int k = a->rp[i]; k < a->rp[i + 1]; ++k) {
            int j = a->ci[k];
            int pos = t->rp[j] + cnt[j]++;
            t->ci[pos] = i; t->v[pos] = a->v[k];
        }
    free(cnt);
}

/* ICPreconditioner::reorder_matrix_with_perm, ic_preconditioner.hpp:925-989:
 * entry (i,j) -> (perm[i], perm[j]), rows sorted by column. */
static void SFX(reorder)(int n, const int* rp, const int* ci, const T* v, const int* perm,
                         SFX(csr)* out) {
    out->rows = out->cols = n;
    out->rp = (int*)calloc((size_t)n + 1, sizeof(int));
    for (int i = 0; i < n; ++i) out->rp[perm[i] + 1] += rp[i + 1] - rp[i];
    for (int i = 0; i < n; ++i) out->rp[i + 1] += out->rp[i];
    int nnz = out->rp[n];
    out->ci = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    out->v = (T*)malloc(sizeof(T) * (size_t)(nnz > 0 ? nnz : 1));
    int* pos = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) pos[i] = out->rp[i];
    for (int i = 0; i < n; ++i) {
        int ni = perm[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            int p = pos[ni]++;
            out->ci[p] = perm[ci[k]]; out->v[p] = v[k];
        }
    }
    free(pos);
    /* insertion sort per row (rows are short; column indices are distinct) */
    for (int i = 0; i < n; ++i) {
        for (int k = out->rp[i] + 1; k < out->rp[i + 1]; ++k) {
            int c = out->ci[k]; T x = out->v[k]; int m = k - 1;
            while (m >= out->rp[i] && out->ci[m] > c) {
                out->ci[m + 1] = out->ci[m]; out->v[m + 1] = out->v[m]; --m;
            }
            out->ci[m + 1] = c; out->v[m + 1] = x;
        }
    }
}

/* ICPreconditioner::extract_lower_triangular, ic_preconditioner.hpp:1075-1115 */
static void SFX(extract_lower)(int n, const int* rp, const int* ci, const T* v, SFX(csr)* L) {
    L->rows = L->cols = n;
    L->rp = (int*)calloc((size_t)n + 1, sizeof(int));
    for (int i = 0; i < n; ++i) {
        int c = 0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) if (ci[k] <= i) ++c;
        L->rp[i + 1] = L->rp[i] + c;
    }
    int nnz = L->rp[n];
    L->ci = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    L->v = (T*)malloc(sizeof(T) * (size_t)(nnz > 0 ? nnz : 1));
    for (int i = 0; i < n; ++i) {
        int pos = L->rp[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] <= i) { L->ci[pos] = ci[k]; L->v[pos] = v[k]; ++pos; }
    }
}

/* ------------------------------------------------------------------------ */
/* IC preconditioner                                                         */
/* ------------------------------------------------------------------------ */

typedef struct {
    ssv_config cfg;
    double shift_parameter, actual_shift;
    int n;
    int use_abmc;          /* ABMC schedule built */
    SFX(csr) L, Lt;
    T* inv_diag;
    T* original_values;
    double* scaling;       /* NULL when diagonal scaling is off */
    orc_abmc abmc;
    SFX(csr) reordered;    /* kept only for abmc_reorder_spmv */
    int* composite_perm;
    double* composite_scaling; /* stays NULL on a fresh setup (see ic_setup) */
    T *temp, *temp2, *xperm, *yperm;
} SFX(ic);

static void SFX(ic_free)(SFX(ic)* p) {
    SFX(csr_free)(&p->L); SFX(csr_free)(&p->Lt); SFX(csr_free)(&p->reordered);
    free(p->inv_diag); free(p->original_values); free(p->scaling);
    orc_abmc_free(&p->abmc);
    free(p->composite_perm); free(p->composite_scaling);
    free(p->temp); free(p->temp2); free(p->xperm); free(p->yperm);
    memset(p, 0, sizeof(*p));
}

/* compute_scaling_factors, ic_preconditioner.hpp:1120-1134 */
static void SFX(ic_scaling)(SFX(ic)* p) {
    int n = p->n;
    p->scaling = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        int d = p->L.rp[i + 1] - 1;
        if (d >= p->L.rp[i] && p->L.ci[d] == i) {
            double a = SABS(p->L.v[d]);
            p->scaling[i] = (a > 0.0) ? 1.0 / sqrt(a) : 1.0;
        } else {
            p->scaling[i] = 1.0;
        }
    }
}

/* apply_scaling_to_L, ic_preconditioner.hpp:1139-1149 */
static void SFX(ic_apply_scaling_to_L)(SFX(ic)* p) {
    for (int i = 0; i < p->n; ++i)
        for (int k = p->L.rp[i]; k < p->L.rp[i + 1]; ++k) {
            int j = p->L.ci[k];
            p->L.v[k] = p->original_values[k] * FROM_REAL(p->scaling[i]) * FROM_REAL(p->scaling[j]);
        }
}

/* Shifted IC(0) with auto-shift restart. compute_ic_factorization
 * (ic_preconditioner.hpp:1161-1273) and the colour-parallel
 * compute_ic_factorization_abmc (:1287-1417) give the same factor: rows of one
 * colour never depend on each other, and a breakdown anywhere in a trial
 * restarts with the same shift increment in both. Rows are processed in index
 * order (which is colour order in the ABMC numbering). Returns 0, or -1 on a
 * missing diagonal (the reference throws runtime_error). */
static int SFX(ic_factorize)(SFX(ic)* p, int* bad_row) {
    const int n = p->n;
    SFX(csr)* L = &p->L;
    p->inv_diag = (T*)realloc(p->inv_diag, sizeof(T) * (size_t)(n > 0 ? n : 1));
    double shift = p->shift_parameter;
    double increment = p->cfg.shift_increment;
    int restart = 1, trials = 0;
    const int nnz = L->rp[n];
    while (restart) {
        restart = 0;
        if (trials > 0) {
            memcpy(L->v, p->original_values, sizeof(T) * (size_t)nnz);
            if (p->cfg.diagonal_scaling) SFX(ic_apply_scaling_to_L)(p);
        } else if (p->cfg.diagonal_scaling) {
            SFX(ic_apply_scaling_to_L)(p);
        }
        int need_restart = 0;
        for (int i = 0; i < n; ++i) {
            const int rs = L->rp[i], re = L->rp[i + 1];
            for (int kk = rs; kk < re - 1; ++kk) {
                const int j = L->ci[kk];
                if (j >= i) break;
                T s = L->v[kk];
                const int js = L->rp[j], je = L->rp[j + 1];
                for (int ii = rs; ii < kk; ++ii) {
                    const int k = L->ci[ii];
                    if (k >= j) break;
                    for (int jj = js; jj < je; ++jj) {
                        if (L->ci[jj] == k) { s -= L->v[ii] * L->v[jj] * p->inv_diag[k]; break; }
                        else if (L->ci[jj] > k) break;
                    }
                }
                L->v[kk] = s;
            }
            const int dp = re - 1;
            if (dp < rs || L->ci[dp] != i) { *bad_row = i; return -1; }
            T orig = L->v[dp];
            T s = orig * FROM_REAL(shift);
            for (int kk = rs; kk < dp; ++kk) {
                const int k = L->ci[kk];
                if (k >= i) break;
                s -= L->v[kk] * L->v[kk] * p->inv_diag[k];
            }
            L->v[dp] = s;
            double abs_s = SABS(s);
            if (p->cfg.auto_shift) {
                double abs_o = SABS(orig);
                if (abs_s < p->cfg.min_diagonal_threshold && abs_o > 0.0) need_restart = 1;
            }
            if (abs_s > p->cfg.zero_diagonal_replacement) {
                p->inv_diag[i] = FROM_REAL(1.0) / s;
            } else {
                T safe = FROM_REAL(p->cfg.zero_diagonal_replacement);
                L->v[dp] = safe;
                p->inv_diag[i] = FROM_REAL(1.0) / safe;
            }
        }
        if (p->cfg.auto_shift && need_restart) {
            if (shift < p->cfg.max_shift_value && trials < p->cfg.max_shift_trials) {
                shift += increment; increment *= 2; trials++; restart = 1;
            }
        }
    }
    p->actual_shift = shift;
    return 0;
}

/* ICPreconditioner::setup, ic_preconditioner.hpp:69-201 (fresh object: the
 * pattern cache of :74-81 never hits in SparseSolvSolver, which builds a new
 * preconditioner per Solve, sparsesolv.hpp:52-54). */
static int SFX(ic_setup)(SFX(ic)* p, const ssv_config* cfg, int n, const int* rp, const int* ci,
                         const T* v, int* bad_row) {
    memset(p, 0, sizeof(*p));
    p->cfg = *cfg;
    p->shift_parameter = cfg->shift_parameter;
    p->n = n;
    size_t nb = sizeof(T) * (size_t)(n > 0 ? n : 1);
    if (cfg->use_abmc) {
        if (cfg->abmc_use_rcm) return -2; /* RCM pre-ordering: not restated */
        orc_abmc_build_into(&p->abmc, n, rp, ci, cfg->abmc_block_size, cfg->abmc_num_colors);
        p->use_abmc = p->abmc.num_colors > 0;
        SFX(reorder)(n, rp, ci, v, p->abmc.ordering, &p->reordered);
        p->temp = (T*)calloc(1, nb);
        if (cfg->diagonal_scaling) p->temp2 = (T*)calloc(1, nb);
        p->xperm = (T*)calloc(1, nb);
        p->yperm = (T*)calloc(1, nb);
        /* build_composite_permutations (:584-608) runs at :125, before the
         * scaling factors exist (:162): on a fresh setup composite_scaling_
         * stays empty, so apply_abmc* (:665,:809) never scales. */
        p->composite_perm = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
        for (int i = 0; i < n; ++i) p->composite_perm[i] = p->abmc.ordering[i];
        p->composite_scaling = NULL;
        SFX(extract_lower)(n, p->reordered.rp, p->reordered.ci, p->reordered.v, &p->L);
        if (!cfg->abmc_reorder_spmv) SFX(csr_free)(&p->reordered);
    } else {
        SFX(extract_lower)(n, rp, ci, v, &p->L);
        p->temp = (T*)calloc(1, nb);
        if (cfg->diagonal_scaling) p->temp2 = (T*)calloc(1, nb);
    }
    int nnzL = p->L.rp[n];
    if (cfg->auto_shift || cfg->diagonal_scaling) {
        p->original_values = (T*)malloc(sizeof(T) * (size_t)(nnzL > 0 ? nnzL : 1));
        memcpy(p->original_values, p->L.v, sizeof(T) * (size_t)nnzL);
    }
    if (cfg->diagonal_scaling) SFX(ic_scaling)(p);
    if (SFX(ic_factorize)(p, bad_row) != 0) return -1;
    SFX(csr_transpose)(&p->L, &p->Lt);
    return 0;
}

/* forward_substitution[_abmc] (:1010-1034, :1430-1447): colour/level order
 * equals index order, so a sequential sweep gives identical values. */
static void SFX(ic_forward)(const SFX(ic)* p, const T* x, T* y) {
    for (int i = 0; i < p->n; ++i) {
        T s = x[i];
        const int ls = p->L.rp[i], le = p->L.rp[i + 1] - 1;
        for (int k = ls; k < le; ++k) s -= p->L.v[k] * y[p->L.ci[k]];
        y[i] = s / p->L.v[le];
    }
}

/* backward_substitution[_abmc] (:1042-1066, :1454-1471) */
static void SFX(ic_backward)(const SFX(ic)* p, const T* x, T* y) {
    for (int i = p->n - 1; i >= 0; --i) {
        T s = FROM_REAL(0.0);
        const int ls = p->Lt.rp[i] + 1, le = p->Lt.rp[i + 1];
        for (int k = ls; k < le; ++k) s -= p->Lt.v[k] * y[p->Lt.ci[k]];
        y[i] = s * p->inv_diag[i] + x[i];
    }
}

/* ICPreconditioner::apply (:215-225) -> apply_abmc_serial (:753-778) or
 * apply_level_schedule (:620-646). */
static void SFX(ic_apply)(SFX(ic)* p, const T* x, T* y) {
    const int n = p->n;
    if (p->use_abmc) {
        const int* perm = p->composite_perm;
        if (p->composite_scaling) {
            for (int i = 0; i < n; ++i) p->xperm[perm[i]] = x[i] * FROM_REAL(p->composite_scaling[i]);
        } else {
            for (int i = 0; i < n; ++i) p->xperm[perm[i]] = x[i];
        }
        SFX(ic_forward)(p, p->xperm, p->temp);
        SFX(ic_backward)(p, p->temp, p->yperm);
        if (p->composite_scaling) {
            for (int i = 0; i < n; ++i) y[i] = p->yperm[perm[i]] * FROM_REAL(p->composite_scaling[i]);
        } else {
            for (int i = 0; i < n; ++i) y[i] = p->yperm[perm[i]];
        }
    } else if (p->cfg.diagonal_scaling && p->scaling) {
        for (int i = 0; i < n; ++i) p->temp[i] = x[i] * FROM_REAL(p->scaling[i]);
        SFX(ic_forward)(p, p->temp, p->temp2);
        SFX(ic_backward)(p, p->temp2, p->temp);
        for (int i = 0; i < n; ++i) y[i] = p->temp[i] * FROM_REAL(p->scaling[i]);
    } else {
        SFX(ic_forward)(p, x, p->temp);
        SFX(ic_backward)(p, p->temp, y);
    }
}

/* apply_in_reordered_space (:299-318), used by Path 1 (abmc_reorder_spmv).
 * This is the single-thread semantics; the reference's multi-thread fused
 * variant (:360-464) reads already-scaled y values in its backward sweep when
 * diagonal scaling is on, so its result depends on the thread count. */
static void SFX(ic_apply_reordered)(SFX(ic)* p, const T* x, T* y) {
    const int n = p->n;
    if (p->cfg.diagonal_scaling && p->scaling) {
        for (int i = 0; i < n; ++i) p->xperm[i] = x[i] * FROM_REAL(p->scaling[i]);
        SFX(ic_forward)(p, p->xperm, p->temp);
        SFX(ic_backward)(p, p->temp, p->xperm);
        for (int i = 0; i < n; ++i) y[i] = p->xperm[i] * FROM_REAL(p->scaling[i]);
    } else {
        SFX(ic_forward)(p, x, p->temp);
        SFX(ic_backward)(p, p->temp, y);
    }
}

/* ------------------------------------------------------------------------ */
/* Iterative solver base (solvers/iterative_solver.hpp)                      */
/* ------------------------------------------------------------------------ */

typedef void (*SFX(apply_fn))(void* ctx, const T* x, T* y);

typedef struct {
    ssv_config cfg;
    int n;
    const int* rp; const int* ci; const T* v;
    const T* b; T* x;
    T *r, *z, *p, *Ap;
    T* best_x; double best_residual;
    double norm_b, normalizer;
    double* hist; int hist_cap; int hist_len;
    int bad_count;
    SFX(apply_fn) pre; void* pre_ctx; /* NULL = identity */
} SFX(solver);

static void SFX(hist_push)(SFX(solver)* s, double v) {
    if (s->hist && s->hist_len < s->hist_cap) s->hist[s->hist_len] = v;
    s->hist_len++;
}

static double SFX(norm)(const T* v, int n) {
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += NORM2(v[i]);
    return sqrt(sum);
}

/* dot_product, iterative_solver.hpp:303-322 */
static T SFX(dot)(const SFX(solver)* s, const T* a, const T* b) {
    T sum = FROM_REAL(0.0);
    if (s->cfg.conjugate) { for (int i = 0; i < s->n; ++i) sum += CONJ(a[i]) * b[i]; }
    else { for (int i = 0; i < s->n; ++i) sum += a[i] * b[i]; }
    return sum;
}

static T SFX(udot)(const T* a, const T* b, int n) {
    T sum = FROM_REAL(0.0);
    for (int i = 0; i < n; ++i) sum += a[i] * b[i];
    return sum;
}

static void SFX(solver_alloc)(SFX(solver)* s) {
    size_t nb = sizeof(T) * (size_t)(s->n > 0 ? s->n : 1);
    s->r = (T*)calloc(1, nb); s->z = (T*)calloc(1, nb);
    s->p = (T*)calloc(1, nb); s->Ap = (T*)calloc(1, nb);
    s->best_x = NULL;
}

static void SFX(solver_free)(SFX(solver)* s) {
    free(s->r); free(s->z); free(s->p); free(s->Ap); free(s->best_x);
}

/* prepare_iteration, iterative_solver.hpp:135-180 */
static void SFX(prepare)(SFX(solver)* s) {
    const int n = s->n;
    if (s->cfg.save_best_result) {
        s->best_x = (T*)calloc(1, sizeof(T) * (size_t)(n > 0 ? n : 1));
    }
    s->best_residual = DBL_MAX;
    SFX(spmv)(n, s->rp, s->ci, s->v, s->x, s->r);
    for (int i = 0; i < n; ++i) s->r[i] = s->b[i] - s->r[i];
    s->norm_b = SFX(norm)(s->b, n);
    double init_norm_r = SFX(norm)(s->r, n);
    switch (s->cfg.norm_type) {
        case SSV_NORM_RHS: s->normalizer = s->norm_b; break;
        case SSV_NORM_INITIAL_RESIDUAL: s->normalizer = init_norm_r; break;
        default: s->normalizer = s->cfg.custom_norm; break;
    }
    if (s->normalizer < 1e-15) s->normalizer = 1.0;
    s->hist_len = 0;
    if (s->cfg.save_residual_history) SFX(hist_push)(s, init_norm_r / s->normalizer);
    s->bad_count = 0;
}

/* check_convergence, iterative_solver.hpp:217-249 */
static int SFX(check)(SFX(solver)* s, double norm_r) {
    double rel = norm_r / s->normalizer;
    if (s->cfg.save_residual_history) SFX(hist_push)(s, rel);
    if (s->cfg.save_best_result && rel < s->best_residual) {
        s->best_residual = rel;
        memcpy(s->best_x, s->x, sizeof(T) * (size_t)s->n);
    }
    if (rel < s->cfg.tolerance || norm_r < s->cfg.abs_tolerance) return 1;
    if (s->cfg.divergence_check) {
        if (rel >= s->best_residual * s->cfg.divergence_threshold) {
            s->bad_count++;
        } else {
            s->bad_count = 0;
        }
    }
    return 0;
}

static int SFX(diverging)(const SFX(solver)* s) {
    return s->cfg.divergence_check && s->bad_count >= s->cfg.divergence_count;
}

/* build_result, iterative_solver.hpp:262-279 */
static void SFX(result)(SFX(solver)* s, int converged, int iters, double final_norm, ssv_result* res) {
    res->converged = converged;
    res->iterations = iters;
    res->final_residual = final_norm / s->normalizer;
    if (!converged && s->cfg.save_best_result) {
        memcpy(s->x, s->best_x, sizeof(T) * (size_t)s->n);
        res->final_residual = s->best_residual;
    }
    res->history_total = s->cfg.save_residual_history ? s->hist_len : 0;
    res->history_len = res->history_total < s->hist_cap ? res->history_total : s->hist_cap;
}

/* apply_preconditioner_fused_dot, iterative_solver.hpp:200-209: z = M^{-1} r,
 * returns dot(r, z) (conjugated if cfg.conjugate). */
static T SFX(pre_fused_dot)(SFX(solver)* s) {
    if (s->pre) s->pre(s->pre_ctx, s->r, s->z);
    else memcpy(s->z, s->r, sizeof(T) * (size_t)s->n);
    return SFX(dot)(s, s->r, s->z);
}

/* CGSolver::do_iterate, solvers/cg_solver.hpp:64-146 */
static void SFX(cg_iterate)(SFX(solver)* s, ssv_result* res) {
    const int n = s->n;
    T *r = s->r, *z = s->z, *p = s->p, *Ap = s->Ap, *x = s->x;
    T rz_old = SFX(pre_fused_dot)(s);
    memcpy(p, z, sizeof(T) * (size_t)n);
    for (int iter = 0; iter < s->cfg.max_iterations; ++iter) {
        T pAp = FROM_REAL(0.0);
        for (int i = 0; i < n; ++i) {
            T acc = FROM_REAL(0.0);
            for (int k = s->rp[i]; k < s->rp[i + 1]; ++k) acc += s->v[k] * p[s->ci[k]];
            Ap[i] = acc;
            pAp += (s->cfg.conjugate ? CONJ(p[i]) : p[i]) * acc;
        }
        if (SABS(pAp) < 1e-30) {
            double nr = SFX(norm)(r, n);
            if (SFX(check)(s, nr)) { SFX(result)(s, 1, iter + 1, nr, res); return; }
            SFX(result)(s, 0, iter, nr, res); return;
        }
        T alpha = rz_old / pAp;
        double nr2 = 0.0;
        for (int i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
            nr2 += NORM2(r[i]);
        }
        double nr = sqrt(nr2);
        if (SFX(check)(s, nr)) { SFX(result)(s, 1, iter + 1, nr, res); return; }
        if (SFX(diverging)(s)) { SFX(result)(s, 0, iter + 1, nr, res); return; }
        T rz_new = SFX(pre_fused_dot)(s);
        T beta = rz_new / rz_old;
        rz_old = rz_new;
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    SFX(result)(s, 0, s->cfg.max_iterations, SFX(norm)(r, n), res);
}

/* COCRSolver::do_iterate, solvers/cocr_solver.hpp:69-168 (unconjugated dots,
 * preconditioner through plain apply). */
static void SFX(cocr_iterate)(SFX(solver)* s, ssv_result* res) {
    const int n = s->n;
    T *r = s->r, *rt = s->z, *p = s->p, *q = s->Ap, *x = s->x;
    size_t nb = sizeof(T) * (size_t)(n > 0 ? n : 1);
    T* qt = (T*)calloc(1, nb);
    T* t = (T*)calloc(1, nb);
    if (s->pre) s->pre(s->pre_ctx, r, rt); else memcpy(rt, r, sizeof(T) * (size_t)n);
    memcpy(p, rt, sizeof(T) * (size_t)n);
    SFX(spmv)(n, s->rp, s->ci, s->v, p, q);
    T rho = SFX(udot)(rt, q, n);
    int done = 0;
    for (int iter = 0; iter < s->cfg.max_iterations && !done; ++iter) {
        if (s->pre) s->pre(s->pre_ctx, q, qt); else memcpy(qt, q, sizeof(T) * (size_t)n);
        T mu = SFX(udot)(qt, q, n);
        if (SABS(mu) < 1e-30) {
            double nr = SFX(norm)(r, n);
            if (SFX(check)(s, nr)) SFX(result)(s, 1, iter + 1, nr, res);
            else SFX(result)(s, 0, iter, nr, res);
            done = 1; break;
        }
        T alpha = rho / mu;
        double nr2 = 0.0;
        for (int i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
            rt[i] -= alpha * qt[i];
            nr2 += NORM2(r[i]);
        }
        double nr = sqrt(nr2);
        if (SFX(check)(s, nr)) { SFX(result)(s, 1, iter + 1, nr, res); done = 1; break; }
        if (SFX(diverging)(s)) { SFX(result)(s, 0, iter + 1, nr, res); done = 1; break; }
        T rho_new = FROM_REAL(0.0);
        for (int i = 0; i < n; ++i) {
            T acc = FROM_REAL(0.0);
            for (int k = s->rp[i]; k < s->rp[i + 1]; ++k) acc += s->v[k] * rt[s->ci[k]];
            t[i] = acc;
            rho_new += rt[i] * acc;
        }
        if (SABS(rho) < 1e-30) { SFX(result)(s, 0, iter + 1, nr, res); done = 1; break; }
        T beta = rho_new / rho;
        rho = rho_new;
        for (int i = 0; i < n; ++i) { p[i] = rt[i] + beta * p[i]; q[i] = t[i] + beta * q[i]; }
    }
    if (!done) SFX(result)(s, 0, s->cfg.max_iterations, SFX(norm)(r, n), res);
    free(qt); free(t);
}

/* ------------------------------------------------------------------------ */
/* SGS-MRTR (solvers/sgs_mrtr_solver.hpp)                                    */
/* ------------------------------------------------------------------------ */

/* forward_solve (:322-334) / backward_solve (:341-355); the level order equals
 * index order for the dependencies, so a sequential sweep is identical. */
static void SFX(mrtr_fwd)(const SFX(csr)* L, const T* rhs, T* y) {
    for (int i = 0; i < L->rows; ++i) {
        T s = rhs[i];
        const int re = L->rp[i + 1] - 1;
        for (int k = L->rp[i]; k < re; ++k) s -= L->v[k] * y[L->ci[k]];
        y[i] = s / L->v[re];
    }
}

static void SFX(mrtr_bwd)(const SFX(csr)* Lt, const T* rhs, T* y) {
    for (int i = Lt->rows - 1; i >= 0; --i) {
        T s = rhs[i];
        const int rs = Lt->rp[i], re = Lt->rp[i + 1];
        if (rs >= re) { y[i] = FROM_REAL(0.0); continue; }
        for (int k = rs + 1; k < re; ++k) s -= Lt->v[k] * y[Lt->ci[k]];
        y[i] = s / Lt->v[rs];
    }
}

static void SFX(mrtr_solve)(SFX(solver)* s, ssv_result* res) {
    const int n = s->n;
    size_t nb = sizeof(T) * (size_t)(n > 0 ? n : 1);
    T *x2 = (T*)calloc(1, nb), *D = (T*)calloc(1, nb), *iD = (T*)calloc(1, nb);
    T *b2 = (T*)calloc(1, nb), *rd = (T*)calloc(1, nb), *u = (T*)calloc(1, nb);
    T *y = (T*)calloc(1, nb), *Ard = (T*)calloc(1, nb), *tmp = (T*)calloc(1, nb);
    T* x_orig = s->x;
    /* prepare_iteration :81-150 */
    for (int i = 0; i < n; ++i) {
        T aii = SFX(entry)(s->rp, s->ci, s->v, i, i);
        if (SABS(aii) > 1e-15) {
            D[i] = FROM_REAL(1.0 / sqrt(SABS(aii)));
            iD[i] = FROM_REAL(sqrt(SABS(aii)));
        } else { D[i] = FROM_REAL(1.0); iD[i] = FROM_REAL(1.0); }
    }
    for (int i = 0; i < n; ++i) b2[i] = D[i] * s->b[i];
    for (int i = 0; i < n; ++i) x2[i] = iD[i] * x_orig[i];
    SFX(csr) L, Lt;
    L.rows = L.cols = n;
    L.rp = (int*)calloc((size_t)n + 1, sizeof(int));
    {
        int cnt = 0;
        for (int i = 0; i < n; ++i) {
            for (int k = s->rp[i]; k < s->rp[i + 1]; ++k) if (s->ci[k] <= i) cnt++;
            L.rp[i + 1] = cnt;
        }
        L.ci = (int*)malloc(sizeof(int) * (size_t)(cnt > 0 ? cnt : 1));
        L.v = (T*)malloc(sizeof(T) * (size_t)(cnt > 0 ? cnt : 1));
        int pos = 0;
        for (int i = 0; i < n; ++i)
            for (int k = s->rp[i]; k < s->rp[i + 1]; ++k) {
                int j = s->ci[k];
                if (j <= i) { L.ci[pos] = j; L.v[pos] = D[i] * s->v[k] * D[j]; ++pos; }
            }
    }
    SFX(csr_transpose)(&L, &Lt);
    SFX(spmv)(n, s->rp, s->ci, s->v, x_orig, tmp);
    for (int i = 0; i < n; ++i) s->r[i] = D[i] * (s->b[i] - tmp[i]);
    SFX(spmv)(n, L.rp, L.ci, L.v, b2, tmp);
    double nLb = SFX(norm)(tmp, n);
    s->normalizer = (nLb > 1e-15) ? nLb : 1.0;
    s->x = x2;
    if (s->cfg.save_best_result) s->best_x = (T*)calloc(1, nb);
    s->best_residual = DBL_MAX;
    s->bad_count = 0;
    double norm_r = SFX(norm)(s->r, n);
    s->hist_len = 0;
    if (s->cfg.save_residual_history) SFX(hist_push)(s, norm_r / s->normalizer);
    SFX(mrtr_fwd)(&L, s->r, rd);
    for (int i = 0; i < n; ++i) y[i] = -rd[i];
    for (int i = 0; i < n; ++i) s->p[i] = FROM_REAL(0.0);
    /* do_iterate :152-247 */
    int finished = 0;
    double nb2 = SFX(norm)(b2, n);
    if (nb2 < 1e-30) nb2 = 1.0;
    norm_r = SFX(norm)(s->r, n);
    if (norm_r / nb2 < s->cfg.tolerance * 0.1) {
        SFX(result)(s, 1, 0, norm_r, res);
        finished = 1;
    }
    T zeta = FROM_REAL(1.0), zeta_old = FROM_REAL(1.0), eta = FROM_REAL(0.0), nu = FROM_REAL(1.0);
    int iter = 0;
    for (iter = 0; !finished && iter < s->cfg.max_iterations; ++iter) {
        SFX(mrtr_bwd)(&Lt, rd, u);
        for (int i = 0; i < n; ++i) tmp[i] = rd[i] - u[i];
        SFX(mrtr_fwd)(&L, tmp, Ard);
        for (int i = 0; i < n; ++i) Ard[i] += u[i];
        T Ar_r = SFX(dot)(s, Ard, rd);
        T Ar_Ar = SFX(dot)(s, Ard, Ard);
        if (iter == 0) {
            zeta = Ar_r / Ar_Ar; zeta_old = zeta; eta = FROM_REAL(0.0);
        } else {
            T Ar_y = SFX(dot)(s, Ard, y);
            T denom = nu * Ar_Ar - Ar_y * Ar_y;
            if (SABS(denom) < 1e-60) denom = (REALPART(denom) >= 0) ? FROM_REAL(1e-60) : FROM_REAL(-1e-60);
            T inv = FROM_REAL(1.0) / denom;
            zeta = nu * Ar_r * inv;
            eta = -Ar_y * Ar_r * inv;
        }
        nu = zeta * Ar_r;
        T coeff = eta * zeta_old / zeta;
        for (int i = 0; i < n; ++i) s->p[i] = u[i] + coeff * s->p[i];
        zeta_old = zeta;
        for (int i = 0; i < n; ++i) s->x[i] += zeta * s->p[i];
        for (int i = 0; i < n; ++i) y[i] = eta * y[i] + zeta * Ard[i];
        for (int i = 0; i < n; ++i) rd[i] -= y[i];
        norm_r = SFX(norm)(rd, n);
        if (SFX(check)(s, norm_r)) { SFX(result)(s, 1, iter + 1, norm_r, res); finished = 1; break; }
        if (SFX(diverging)(s)) { SFX(result)(s, 0, iter + 1, norm_r, res); finished = 1; break; }
    }
    if (!finished) {
        norm_r = SFX(norm)(rd, n);
        SFX(result)(s, 0, iter, norm_r, res);
    }
    for (int i = 0; i < n; ++i) x_orig[i] = D[i] * x2[i];
    s->x = x_orig;
    SFX(csr_free)(&L); SFX(csr_free)(&Lt);
    free(x2); free(D); free(iD); free(b2); free(rd); free(u); free(y); free(Ard); free(tmp);
}

/* ------------------------------------------------------------------------ */
/* Entry: SparseSolvSolver::Solve                                            */
/* ------------------------------------------------------------------------ */

static void SFX(ic_apply_cb)(void* ctx, const T* x, T* y) { SFX(ic_apply)((SFX(ic)*)ctx, x, y); }
static void SFX(ic_apply_reordered_cb)(void* ctx, const T* x, T* y) {
    SFX(ic_apply_reordered)((SFX(ic)*)ctx, x, y);
}

/* SparseSolvSolver::Solve, ngsolve/sparsesolv_solvers.hpp:73-160, with
 * BuildSparseMatrixView's FreeDofs rule (ngsolve/sparsesolv_precond.hpp:60-74):
 * constrained rows -> identity rows, constrained columns -> 0. */
static int SFX(solve)(int n, const int* rp, const int* ci, const T* vals, const unsigned char* fd,
                      int method, const ssv_config* cfg_in, const T* b, T* x, ssv_result* res,
                      double* hist, int hist_cap, char* err, int err_cap) {
    int nnz = rp[n];
    T* mv = (T*)malloc(sizeof(T) * (size_t)(nnz > 0 ? nnz : 1));
    memcpy(mv, vals, sizeof(T) * (size_t)nnz);
    size_t nb = sizeof(T) * (size_t)(n > 0 ? n : 1);
    T* bm = (T*)calloc(1, nb);
    T* xm = (T*)calloc(1, nb);
    if (fd) {
        for (int i = 0; i < n; ++i)
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                int j = ci[k];
                if (!fd[i]) mv[k] = (j == i) ? FROM_REAL(1.0) : FROM_REAL(0.0);
                else if (!fd[j]) mv[k] = FROM_REAL(0.0);
            }
        for (int i = 0; i < n; ++i) {
            bm[i] = fd[i] ? b[i] : FROM_REAL(0.0);
            xm[i] = fd[i] ? x[i] : FROM_REAL(0.0);
        }
    } else {
        memcpy(bm, b, sizeof(T) * (size_t)n);
        memcpy(xm, x, sizeof(T) * (size_t)n);
    }
    ssv_config cfg = *cfg_in;
    memset(res, 0, sizeof(*res));
    SFX(solver) s;
    memset(&s, 0, sizeof(s));
    s.cfg = cfg; s.n = n; s.rp = rp; s.ci = ci; s.v = mv; s.b = bm; s.x = xm;
    s.hist = hist; s.hist_cap = hist_cap;
    int rc = 0;
    SFX(solver_alloc)(&s);
    if (method == SSV_METHOD_ICCG) {
        SFX(ic) ic;
        int bad = -1;
        int src = SFX(ic_setup)(&ic, &cfg, n, rp, ci, mv, &bad);
        if (src == -1) {
            snprintf(err, (size_t)err_cap, "IC decomposition failed: missing diagonal element at row %d", bad);
            rc = SSV_ERR_RUNTIME;
        } else if (src == -2) {
            snprintf(err, (size_t)err_cap, "oracle: abmc_use_rcm is not restated");
            rc = SSV_ERR_INVALID_ARG;
        } else {
            res->actual_shift = ic.actual_shift;
            if (cfg.use_abmc && cfg.abmc_reorder_spmv && ic.reordered.rows > 0) {
                /* Path 1, sparsesolv.hpp:60-78 */
                const int* ord = ic.abmc.ordering;
                T* br = (T*)calloc(1, nb); T* xr = (T*)calloc(1, nb);
                for (int i = 0; i < n; ++i) br[ord[i]] = bm[i];
                for (int i = 0; i < n; ++i) xr[ord[i]] = xm[i];
                s.rp = ic.reordered.rp; s.ci = ic.reordered.ci; s.v = ic.reordered.v;
                s.b = br; s.x = xr;
                s.pre = SFX(ic_apply_reordered_cb); s.pre_ctx = &ic;
                SFX(prepare)(&s);
                SFX(cg_iterate)(&s, res);
                for (int i = 0; i < n; ++i) xm[i] = xr[ord[i]];
                free(br); free(xr);
            } else {
                /* Path 3, sparsesolv.hpp:101-104 */
                s.pre = SFX(ic_apply_cb); s.pre_ctx = &ic;
                SFX(prepare)(&s);
                SFX(cg_iterate)(&s, res);
            }
            res->actual_shift = ic.actual_shift;
        }
        SFX(ic_free)(&ic);
    } else if (method == SSV_METHOD_SGSMRTR) {
        SFX(mrtr_solve)(&s, res);
    } else if (method == SSV_METHOD_CG) {
        SFX(prepare)(&s);
        SFX(cg_iterate)(&s, res);
    } else if (method == SSV_METHOD_COCR) {
        SFX(prepare)(&s);
        SFX(cocr_iterate)(&s, res);
    } else {
        rc = SSV_ERR_RUNTIME;
    }
    if (rc == 0) {
        if (fd) { for (int i = 0; i < n; ++i) if (fd[i]) x[i] = xm[i]; }
        else memcpy(x, xm, sizeof(T) * (size_t)n);
    }
    SFX(solver_free)(&s);
    free(mv); free(bm); free(xm);
    return rc;
}

/* ICPreconditioner factory + Update() + Mult (sparsesolv_precond.hpp:123-136,
 * 188-191): y = M^{-1} x with constrained outputs zeroed. */
static int SFX(ic_mult)(int n, const int* rp, const int* ci, const T* vals, const unsigned char* fd,
                        const ssv_config* cfg, const T* x, T* y, double* actual_shift) {
    int nnz = rp[n];
    T* mv = (T*)malloc(sizeof(T) * (size_t)(nnz > 0 ? nnz : 1));
    memcpy(mv, vals, sizeof(T) * (size_t)nnz);
    if (fd) {
        for (int i = 0; i < n; ++i)
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                int j = ci[k];
                if (!fd[i]) mv[k] = (j == i) ? FROM_REAL(1.0) : FROM_REAL(0.0);
                else if (!fd[j]) mv[k] = FROM_REAL(0.0);
            }
    }
    SFX(ic) ic;
    int bad = -1;
    int rc = SFX(ic_setup)(&ic, cfg, n, rp, ci, mv, &bad);
    if (rc == 0) {
        SFX(ic_apply)(&ic, x, y);
        if (fd) for (int i = 0; i < n; ++i) if (!fd[i]) y[i] = FROM_REAL(0.0);
        if (actual_shift) *actual_shift = ic.actual_shift;
    }
    SFX(ic_free)(&ic);
    free(mv);
    return rc;
}

/* SGSPreconditioner factory + Update() + Mult (sparsesolv_precond.hpp:123-136,
 * 230-250; preconditioners/sgs_preconditioner.hpp:67-200): the forward sweep
 * (D + L) t = x, t <- t / inv_diag, the backward sweep (D + U) y = t, on the
 * FreeDofs view, constrained outputs zeroed. Rows of one level set do not
 * depend on each other, so sweeping rows in index order (forward) and in
 * reverse order (backward) gives every row the reference's operands. */
static int SFX(sgs_mult)(int n, const int* rp, const int* ci, const T* vals, const unsigned char* fd,
                         const T* x, T* y) {
    int nnz = rp[n];
    T* mv = (T*)malloc(sizeof(T) * (size_t)(nnz > 0 ? nnz : 1));
    T* inv = (T*)malloc(sizeof(T) * (size_t)(n > 0 ? n : 1));
    T* t = (T*)malloc(sizeof(T) * (size_t)(n > 0 ? n : 1));
    memcpy(mv, vals, sizeof(T) * (size_t)nnz);
    if (fd) {
        for (int i = 0; i < n; ++i)
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                int j = ci[k];
                if (!fd[i]) mv[k] = (j == i) ? FROM_REAL(1.0) : FROM_REAL(0.0);
                else if (!fd[j]) mv[k] = FROM_REAL(0.0);
            }
    }
    for (int i = 0; i < n; ++i) {
        T d = FROM_REAL(0.0);
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) { d = mv[k]; break; }
        inv[i] = SABS(d) > 1e-15 ? FROM_REAL(1.0) / d : FROM_REAL(1.0);
    }
    for (int i = 0; i < n; ++i) {
        T sum = x[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] < i) sum -= mv[k] * t[ci[k]];
        t[i] = sum * inv[i];
    }
    for (int i = 0; i < n; ++i) t[i] = t[i] / inv[i];
    for (int i = n - 1; i >= 0; --i) {
        T sum = t[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] > i) sum -= mv[k] * y[ci[k]];
        y[i] = sum * inv[i];
    }
    if (fd) for (int i = 0; i < n; ++i) if (!fd[i]) y[i] = FROM_REAL(0.0);
    free(mv); free(inv); free(t);
    return 0;
}

/* COCRSolverNGS::Mult, ngsolve/sparsesolv_solvers.hpp:273-369, with the
 * preconditioner given as a callback (identity when NULL). */
static int SFX(cocr_ngs)(int n, const int* rp, const int* ci, const T* vals, const unsigned char* fd,
                         SFX(apply_fn) pre, void* pre_ctx, int maxiter, double tol,
                         const T* rhs, T* sol, int* iterations) {
    size_t nb = sizeof(T) * (size_t)(n > 0 ? n : 1);
    T *r = (T*)calloc(1, nb), *rt = (T*)calloc(1, nb), *p = (T*)calloc(1, nb);
    T *q = (T*)calloc(1, nb), *qt = (T*)calloc(1, nb), *t = (T*)calloc(1, nb);
    for (int i = 0; i < n; ++i) sol[i] = FROM_REAL(0.0);
    memcpy(r, rhs, sizeof(T) * (size_t)n);
    if (fd) for (int i = 0; i < n; ++i) if (!fd[i]) r[i] = FROM_REAL(0.0);
    double rhs_norm = 0.0;
    for (int i = 0; i < n; ++i) rhs_norm += NORM2(r[i]);
    rhs_norm = sqrt(fabs(rhs_norm));
    int j = 0;
    if (rhs_norm < 1e-30) { *iterations = 0; goto done; }
    if (pre) pre(pre_ctx, r, rt); else memcpy(rt, r, sizeof(T) * (size_t)n);
    memcpy(p, rt, sizeof(T) * (size_t)n);
    SFX(spmv)(n, rp, ci, vals, p, q);
    if (fd) for (int i = 0; i < n; ++i) if (!fd[i]) q[i] = FROM_REAL(0.0);
    T rho = SFX(udot)(rt, q, n);
    for (j = 0; j < maxiter; ++j) {
        if (pre) pre(pre_ctx, q, qt); else memcpy(qt, q, sizeof(T) * (size_t)n);
        T mu = SFX(udot)(qt, q, n);
        if (SABS(mu) < 1e-30) break;
        T alpha = rho / mu;
        for (int i = 0; i < n; ++i) {
            sol[i] += alpha * p[i]; r[i] -= alpha * q[i]; rt[i] -= alpha * qt[i];
        }
        double res2 = 0.0;
        for (int i = 0; i < n; ++i) res2 += NORM2(r[i]);
        double resn = sqrt(fabs(res2));
        if (resn / rhs_norm <= tol) { *iterations = j + 1; goto done; }
        SFX(spmv)(n, rp, ci, vals, rt, t);
        if (fd) for (int i = 0; i < n; ++i) if (!fd[i]) t[i] = FROM_REAL(0.0);
        T rho_new = SFX(udot)(rt, t, n);
        if (SABS(rho) < 1e-30) break;
        T beta = rho_new / rho;
        rho = rho_new;
        for (int i = 0; i < n; ++i) { p[i] = rt[i] + beta * p[i]; q[i] = t[i] + beta * q[i]; }
    }
    *iterations = j;
done:
    free(r); free(rt); free(p); free(q); free(qt); free(t);
    return 0;
}
