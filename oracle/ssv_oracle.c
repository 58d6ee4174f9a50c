/*
 * ssv_oracle.c -- TEST INFRASTRUCTURE: the CPU oracle of the B200 solve path.
 *
 * A plain-C restatement of ksugahar/ngsolve-sparsesolv's NGSolve-free solve
 * path (ICCG with ABMC or level-schedule IC(0), CG, COCR, SGS-MRTR, the
 * NGSolve COCRSolver loop), each routine citing the reference file:line it
 * follows (paths relative to the reference's include/sparsesolv/ unless
 * stated). Only tests/, the smoke check and bench.py's CPU-baseline leg load
 * it, to check results (test infrastructure); the product never links or calls it.
 *
 * Pinned against the reference itself: oracle/ref_driver.cpp compiles the
 * reference's own headers into oracle/_ref/libssv_ref.so, and
 * tests/golden/gen_golden.py stores that library's outputs as fixtures.
 */
#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/sparsesolv_b200.h"

/* ------------------------------------------------------------------------ */
/* ABMC ordering, core/abmc_ordering.hpp                                     */
/* ------------------------------------------------------------------------ */

typedef struct {
    int num_colors, num_blocks;
    int* color_offsets;  /* num_colors + 1 */
    int* block_offsets;  /* num_blocks + 1 */
    int* ordering;       /* ordering[old] = new */
    int* reverse;        /* reverse[new] = old  */
} orc_abmc;

static void orc_abmc_free(orc_abmc* a) {
    free(a->color_offsets); free(a->block_offsets); free(a->ordering); free(a->reverse);
    memset(a, 0, sizeof(*a));
}

/* ABMCSchedule::build (:83-121) with make_algebraic_blocks (:147-227),
 * build_block_graph (:235-273), color_graph (:288-353) and
 * build_row_ordering (:365-410). */
static void orc_abmc_build_into(orc_abmc* a, int n, const int* rp, const int* ci,
                                int block_size, int target_colors) {
    memset(a, 0, sizeof(*a));
    if (n <= 0) return;
    if (block_size < 1) block_size = 1;
    if (target_colors < 2) target_colors = 2;
    const int max_blocks = (n + block_size - 1) / block_size;

    /* Stage 1: BFS aggregation. Rows are appended to the block being built
     * (and at the end to the last block), so one flat array holds all blocks. */
    int* assign = (int*)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; ++i) assign[i] = -1; /* -1 free, -2 queued, >=0 block */
    int* brow = (int*)malloc(sizeof(int) * (size_t)n);
    int* bstart = (int*)malloc(sizeof(int) * ((size_t)max_blocks + 2));
    int* queue = (int*)malloc(sizeof(int) * (size_t)n);
    int nblk = 0, nrow = 0, next = 0;
    for (int blk = 0; blk < max_blocks; ++blk) {
        while (next < n && assign[next] >= 0) ++next;
        if (next >= n) break;
        int id = nblk++;
        bstart[id] = nrow;
        int cur = 0;
        assign[next] = id; brow[nrow++] = next; cur++;
        int qh = 0, qt = 0;
        for (int k = rp[next]; k < rp[next + 1]; ++k) {
            int j = ci[k];
            if (assign[j] == -1) { queue[qt++] = j; assign[j] = -2; }
        }
        while (qh < qt && cur < block_size) {
            int row = queue[qh++];
            if (assign[row] >= 0) continue;
            assign[row] = id; brow[nrow++] = row; cur++;
            if (cur >= block_size) break;
            for (int k = rp[row]; k < rp[row + 1]; ++k) {
                int j = ci[k];
                if (assign[j] == -1) { queue[qt++] = j; assign[j] = -2; }
            }
        }
        while (qh < qt) { int row = queue[qh++]; if (assign[row] == -2) assign[row] = -1; }
    }
    for (int i = 0; i < n; ++i) {
        if (assign[i] < 0) {
            if (nblk == 0) { bstart[0] = nrow; nblk = 1; }
            assign[i] = nblk - 1; brow[nrow++] = i;
        }
    }
    bstart[nblk] = nrow;

    /* Stage 2: block adjacency (deduplicated by last_seen). */
    int* last = (int*)malloc(sizeof(int) * (size_t)nblk);
    for (int b = 0; b < nblk; ++b) last[b] = -1;
    int* grp = (int*)calloc((size_t)nblk + 1, sizeof(int));
    size_t gcap = 16 * (size_t)nblk + 16, gn = 0;
    int* gci = (int*)malloc(sizeof(int) * gcap);
    for (int bi = 0; bi < nblk; ++bi) {
        for (int m = bstart[bi]; m < bstart[bi + 1]; ++m) {
            int row = brow[m];
            for (int k = rp[row]; k < rp[row + 1]; ++k) {
                int bj = assign[ci[k]];
                if (bi != bj && last[bj] != bi) {
                    last[bj] = bi;
                    if (gn == gcap) { gcap *= 2; gci = (int*)realloc(gci, sizeof(int) * gcap); }
                    gci[gn++] = bj;
                }
            }
        }
        grp[bi + 1] = (int)gn;
    }

    /* Stage 3: greedy colouring over lower neighbours. */
    int ncol = target_colors;
    for (int i = 0; i < nblk; ++i) {
        int lower = 0;
        for (int k = grp[i]; k < grp[i + 1]; ++k) if (gci[k] < i) ++lower;
        if (lower >= ncol) ncol = lower + 1;
    }
    int* color = (int*)malloc(sizeof(int) * (size_t)nblk);
    int* forbid = (int*)malloc(sizeof(int) * ((size_t)ncol + (size_t)nblk + 1));
    for (int c = 0; c < ncol; ++c) forbid[c] = -1;
    for (int i = 0; i < nblk; ++i) {
        for (int k = grp[i]; k < grp[i + 1]; ++k) {
            int j = gci[k];
            if (j < i && color[j] >= 0) forbid[color[j]] = i;
        }
        int chosen = -1;
        for (int c = 0; c < ncol; ++c) if (forbid[c] != i) { chosen = c; break; }
        if (chosen < 0) { chosen = ncol; forbid[ncol] = -1; ncol++; }
        color[i] = chosen;
    }
    /* colour lists (blocks ascending), empty colours removed */
    int* ccount = (int*)calloc((size_t)ncol, sizeof(int));
    for (int i = 0; i < nblk; ++i) ccount[color[i]]++;
    int* cmap = (int*)malloc(sizeof(int) * (size_t)ncol);
    int nc = 0;
    for (int c = 0; c < ncol; ++c) cmap[c] = ccount[c] > 0 ? nc++ : -1;

    /* Stage 4: row ordering, colour-major, rows sorted inside each block. */
    a->num_colors = nc; a->num_blocks = nblk;
    a->color_offsets = (int*)calloc((size_t)nc + 1, sizeof(int));
    a->block_offsets = (int*)malloc(sizeof(int) * ((size_t)nblk + 1));
    a->ordering = (int*)malloc(sizeof(int) * (size_t)n);
    a->reverse = (int*)malloc(sizeof(int) * (size_t)n);
    for (int c = 0; c < ncol; ++c) if (cmap[c] >= 0) a->color_offsets[cmap[c] + 1] = ccount[c];
    for (int c = 0; c < nc; ++c) a->color_offsets[c + 1] += a->color_offsets[c];
    int row_idx = 0, gid = 0;
    for (int c = 0; c < ncol; ++c) {
        if (cmap[c] < 0) continue;
        for (int b = 0; b < nblk; ++b) {
            if (color[b] != c) continue;
            int s0 = bstart[b], s1 = bstart[b + 1];
            for (int u = s0 + 1; u < s1; ++u) { /* insertion sort of the block's rows */
                int v = brow[u], w = u - 1;
                while (w >= s0 && brow[w] > v) { brow[w + 1] = brow[w]; --w; }
                brow[w + 1] = v;
            }
            a->block_offsets[gid] = row_idx;
            for (int u = s0; u < s1; ++u) {
                a->ordering[brow[u]] = row_idx; a->reverse[row_idx] = brow[u]; ++row_idx;
            }
            ++gid;
        }
    }
    a->block_offsets[nblk] = row_idx;
    free(assign); free(brow); free(bstart); free(queue); free(last); free(grp); free(gci);
    free(color); free(forbid); free(ccount); free(cmap);
}

/* ------------------------------------------------------------------------ */
/* Scalar-generic parts                                                      */
/* ------------------------------------------------------------------------ */

#define T double
#define SFX(name) name##_d
#define CONJ(a) (a)
#define NORM2(a) ((a) * (a))
#define SABS(a) fabs(a)
#define FROM_REAL(d) ((double)(d))
#define REALPART(a) (a)
#include "ssv_oracle_body.h"
#undef T
#undef SFX
#undef CONJ
#undef NORM2
#undef SABS
#undef FROM_REAL
#undef REALPART

typedef double _Complex zc;
#define T zc
#define SFX(name) name##_z
#define CONJ(a) conj(a)
#define NORM2(a) (creal(a) * creal(a) + cimag(a) * cimag(a))
#define SABS(a) cabs(a)
#define FROM_REAL(d) ((zc)(double)(d))
#define REALPART(a) creal(a)
#include "ssv_oracle_body.h"
#undef T
#undef SFX
#undef CONJ
#undef NORM2
#undef SABS
#undef FROM_REAL
#undef REALPART

/* ------------------------------------------------------------------------ */
/* Exported entry points (loaded with ctypes by tests and bench.py)          */
/* ------------------------------------------------------------------------ */

static char g_err[512];

const char* orc_last_error(void) { return g_err; }

static int parse_method(const char* m) {
    if (!m) return -1;
    if (!strcmp(m, "ICCG") || !strcmp(m, "iccg")) return SSV_METHOD_ICCG;
    if (!strcmp(m, "SGSMRTR") || !strcmp(m, "sgsmrtr")) return SSV_METHOD_SGSMRTR;
    if (!strcmp(m, "CG") || !strcmp(m, "cg")) return SSV_METHOD_CG;
    if (!strcmp(m, "COCR") || !strcmp(m, "cocr")) return SSV_METHOD_COCR;
    return -1;
}

void orc_config_default(ssv_config* c) {
    memset(c, 0, sizeof(*c));
    c->tolerance = 1e-10; c->max_iterations = 1000; c->abs_tolerance = 1e-12;
    c->norm_type = SSV_NORM_RHS; c->custom_norm = 1.0; c->shift_parameter = 1.05;
    c->shift_increment = 0.05; c->max_shift_value = 5.0; c->min_diagonal_threshold = 1e-6;
    c->zero_diagonal_replacement = 1e-10; c->max_shift_trials = 100;
    c->divergence_threshold = 1000.0; c->divergence_count = 100; c->save_best_result = 1;
    c->abmc_block_size = 4; c->abmc_num_colors = 4;
}

int orc_abmc_build(int n, const int* rp, const int* ci, int block_size, int target_colors,
                   int* num_colors, int* num_blocks, int* color_offsets, int* block_offsets,
                   int* ordering, int* reverse) {
    orc_abmc a;
    orc_abmc_build_into(&a, n, rp, ci, block_size, target_colors);
    *num_colors = a.num_colors; *num_blocks = a.num_blocks;
    if (n > 0) {
        memcpy(color_offsets, a.color_offsets, sizeof(int) * ((size_t)a.num_colors + 1));
        memcpy(block_offsets, a.block_offsets, sizeof(int) * ((size_t)a.num_blocks + 1));
        memcpy(ordering, a.ordering, sizeof(int) * (size_t)n);
        memcpy(reverse, a.reverse, sizeof(int) * (size_t)n);
    }
    orc_abmc_free(&a);
    return 0;
}

/* LevelSchedule::build_from_lower/upper, core/level_schedule.hpp:58-135 */
int orc_level_schedule(int n, const int* rp, const int* ci, int upper, int* level_of, int* num_levels) {
    int maxl = 0;
    if (n <= 0) { *num_levels = 0; return 0; }
    if (!upper) {
        for (int i = 0; i < n; ++i) {
            int dep = -1;
            for (int k = rp[i]; k < rp[i + 1]; ++k) { int j = ci[k]; if (j < i && level_of[j] > dep) dep = level_of[j]; }
            level_of[i] = dep + 1; if (level_of[i] > maxl) maxl = level_of[i];
        }
    } else {
        for (int i = n - 1; i >= 0; --i) {
            int dep = -1;
            for (int k = rp[i]; k < rp[i + 1]; ++k) { int j = ci[k]; if (j > i && level_of[j] > dep) dep = level_of[j]; }
            level_of[i] = dep + 1; if (level_of[i] > maxl) maxl = level_of[i];
        }
    }
    *num_levels = maxl + 1;
    return 0;
}

int orc_spmv(int n, const int* rp, const int* ci, const void* v, int dtype, const void* x, void* y) {
    if (dtype == SSV_F64) spmv_d(n, rp, ci, (const double*)v, (const double*)x, (double*)y);
    else spmv_z(n, rp, ci, (const zc*)v, (const zc*)x, (zc*)y);
    return 0;
}

/* SparseSolvSolver::Solve (see ssv_oracle_body.h). */
int orc_solve(int n, const int* rp, const int* ci, const void* vals, int dtype,
              const unsigned char* freedofs, const char* method, const ssv_config* cfg,
              const void* b, void* x, ssv_result* res, double* hist, int hist_cap) {
    g_err[0] = 0;
    int m = parse_method(method);
    if (m < 0) {
        snprintf(g_err, sizeof(g_err),
                 "SparseSolvSolver: Unknown method '%s'. Available: ICCG, SGSMRTR, CG, COCR",
                 method ? method : "");
        return SSV_ERR_RUNTIME;
    }
    if (dtype == SSV_F64)
        return solve_d(n, rp, ci, (const double*)vals, freedofs, m, cfg, (const double*)b,
                       (double*)x, res, hist, hist_cap, g_err, (int)sizeof(g_err));
    return solve_z(n, rp, ci, (const zc*)vals, freedofs, m, cfg, (const zc*)b, (zc*)x, res,
                   hist, hist_cap, g_err, (int)sizeof(g_err));
}

int orc_sgs_mult(int n, const int* rp, const int* ci, const void* vals, int dtype, const unsigned char* freedofs,
                 const void* x, void* y) {
    if (dtype == SSV_F64)
        return sgs_mult_d(n, rp, ci, (const double*)vals, freedofs, (const double*)x, (double*)y);
    return sgs_mult_z(n, rp, ci, (const zc*)vals, freedofs, (const zc*)x, (zc*)y);
}

int orc_ic_mult(int n, const int* rp, const int* ci, const void* vals, int dtype,
                const unsigned char* freedofs, const ssv_config* cfg, const void* x, void* y,
                double* actual_shift) {
    if (dtype == SSV_F64)
        return ic_mult_d(n, rp, ci, (const double*)vals, freedofs, cfg, (const double*)x,
                         (double*)y, actual_shift);
    return ic_mult_z(n, rp, ci, (const zc*)vals, freedofs, cfg, (const zc*)x, (zc*)y, actual_shift);
}

/* Preconditioner callback for orc_cocr_solve: y = M^{-1} x on n scalars. */
typedef void (*orc_precond_fn)(void* ctx, const void* x, void* y);

typedef struct { orc_precond_fn fn; void* ctx; } cb_wrap;
static void cb_d(void* c, const double* x, double* y) { cb_wrap* w = (cb_wrap*)c; w->fn(w->ctx, x, y); }
static void cb_z(void* c, const zc* x, zc* y) { cb_wrap* w = (cb_wrap*)c; w->fn(w->ctx, x, y); }

int orc_cocr_solve(int n, const int* rp, const int* ci, const void* vals, int dtype,
                   const unsigned char* freedofs, orc_precond_fn pre, void* pre_ctx,
                   int maxiter, double tol, const void* rhs, void* sol, int* iterations) {
    cb_wrap w = {pre, pre_ctx};
    if (dtype == SSV_F64)
        return cocr_ngs_d(n, rp, ci, (const double*)vals, freedofs, pre ? cb_d : NULL, &w,
                          maxiter, tol, (const double*)rhs, (double*)sol, iterations);
    return cocr_ngs_z(n, rp, ci, (const zc*)vals, freedofs, pre ? cb_z : NULL, &w, maxiter, tol,
                      (const zc*)rhs, (zc*)sol, iterations);
}
