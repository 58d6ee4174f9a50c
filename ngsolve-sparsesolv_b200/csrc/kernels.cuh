// kernels.cuh -- sm_100a kernels of the solve path.
//
// Everything here is HBM/L2-bound sparse work (no tensor cores): CSR SpMV with
// a sub-warp per row, fused vector updates with deterministic two-stage
// reductions (the last block to finish sums the per-block partials in block
// order and runs the Krylov scalar step on the device, so no host round trip
// happens per iteration), and the colour-by-colour IC(0) kernels.
#pragma once

#include "ssv_common.cuh"

namespace ssv {

constexpr int kBlock = 256;  // threads per block of the streaming kernels

// Programmatic dependent launch: the iteration's kernels are launched so that the
// next one in the stream may be scheduled before this one ends. Each waits
// here for its predecessor's completion and memory (griddepcontrol.wait)
// before touching any data, then lets its own successor start launching.
// Launched without the attribute, both instructions have no effect.
__device__ __forceinline__ void pdl_gate() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}


// ---------------------------------------------------------------------------
// Device-resident Krylov state. Scalars are double2 (real methods use .x).
// ---------------------------------------------------------------------------
struct KState {
    // control
    int done;          // 1 once the iteration has finished (any reason)
    int converged;
    int iters;         // SolverResult::iterations
    int status;        // 0 ok, SSV_ERR_TIMEOUT if the loop guard fired
    int it;            // loop index `iter` of the reference's do_iterate
    int loops;         // executed loop bodies (termination guard)
    int breakdown;     // set by a breakdown test, consumed by the next kernel
    int bad_count;     // divergence counter (iterative_solver.hpp:236-246)
    int cur, best;     // x ping-pong buffers: current x and best x (-1 none)
    int hist_len;      // entries of the residual history produced so far
    int pad_;
    // scalars
    double2 rho, rho_new, alpha, beta, denom, scratch;
    double norm_r, normalizer, best_residual, final_norm;
    // configuration
    double tol, abs_tol, div_threshold;
    int maxiter, div_check, div_count, save_best, save_hist, conj, hist_cap, max_loops;
    double* hist;      // device history buffer (hist_cap entries)
    // COCR with an external preconditioner: breakdown threshold on |mu| and
    // |rho| (the reference's 1e-30), and the residual norm at which a cycle
    // of the refined (defect-correction) form ends (0 = never)
    double brk_thr, restart_abs;
    int updates;       // x updates performed in this cycle
    int pad2_;
};

// Reduction epilogues run by the last block of a reduction kernel.
enum RedOp : int {
    RED_STORE = 0,     // out = total
    RED_CG_ALPHA,      // pAp -> alpha = rho / pAp  (cg_solver.hpp:455-465)
    RED_CHECK,         // ||r||^2 -> check_convergence (iterative_solver.hpp:217-249)
    RED_CG_BETA,       // (r,z) -> beta = rz_new / rz_old (cg_solver.hpp:488-490)
    RED_COCR_ALPHA,    // mu -> alpha = rho / mu  (cocr_solver.hpp:105-116)
    RED_COCR_BETA,     // rho_new -> beta, rho breakdown (cocr_solver.hpp:141-155)
};

template <typename S>
__device__ __forceinline__ S s_from2(double2 v) {
    if constexpr (ST<S>::cplx) return S{v.x, v.y};
    else return v.x;
}
template <typename S>
__device__ __forceinline__ double2 s_to2(S v) {
    if constexpr (ST<S>::cplx) return make_double2(v.x, v.y);
    else return make_double2(v, 0.0);
}

__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// Fixed-order block reduction (valid in thread 0).
__device__ __forceinline__ double2 block_sum2(double2 v) {
    __shared__ double2 sh[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum2(v);
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : make_double2(0.0, 0.0);
    if (w == 0) v = warp_sum2(v);
    return v;
}

// check_convergence + the result rules of CG/COCR, on the device.
__device__ inline void dev_check(KState* st, double norm_r, int breakdown, int nxt) {
    st->norm_r = norm_r;
    const double rel = norm_r / st->normalizer;
    if (st->save_hist) {
        if (st->hist_len < st->hist_cap) st->hist[st->hist_len] = rel;
        st->hist_len++;
    }
    if (st->save_best && rel < st->best_residual) {
        st->best_residual = rel;
        st->best = nxt;
    }
    if (!breakdown) st->cur = nxt;
    const bool conv = (rel < st->tol) || (norm_r < st->abs_tol);
    if (breakdown) {  // cg_solver.hpp:456-463 / cocr_solver.hpp:108-114
        st->done = 1;
        st->converged = conv ? 1 : 0;
        st->iters = conv ? st->it + 1 : st->it;
        st->final_norm = norm_r;
        return;
    }
    if (conv) {
        st->done = 1; st->converged = 1; st->iters = st->it + 1; st->final_norm = norm_r;
        return;
    }
    if (st->div_check) {
        if (rel >= st->best_residual * st->div_threshold) st->bad_count++;
        else st->bad_count = 0;
        if (st->bad_count >= st->div_count) {  // is_diverging()
            st->done = 1; st->converged = 0; st->iters = st->it + 1; st->final_norm = norm_r;
        }
    }
}

template <typename S>
__device__ inline void finish_reduction(double2 total, KState* st, int op, double2* out) {
    switch (op) {
        case RED_STORE:
            if (out) *out = total;
            break;
        case RED_CG_ALPHA: {
            S pAp = s_from2<S>(total);
            if (ST<S>::abs(pAp) < 1e-30) st->breakdown = 1;
            else st->alpha = s_to2<S>(ST<S>::div(s_from2<S>(st->rho), pAp));
            break;
        }
        case RED_COCR_ALPHA: {
            S mu = s_from2<S>(total);
            if (ST<S>::abs(mu) < 1e-30) st->breakdown = 1;
            else st->alpha = s_to2<S>(ST<S>::div(s_from2<S>(st->rho), mu));
            break;
        }
        case RED_CHECK:
            break;  // handled by the update kernels (needs the buffer index)
        case RED_CG_BETA: {
            S rz_new = s_from2<S>(total);
            st->beta = s_to2<S>(ST<S>::div(rz_new, s_from2<S>(st->rho)));
            st->rho = total;
            break;
        }
        case RED_COCR_BETA: {
            S rho_new = s_from2<S>(total);
            S rho = s_from2<S>(st->rho);
            if (ST<S>::abs(rho) < 1e-30) {  // cocr_solver.hpp:150-152
                st->done = 1; st->converged = 0; st->iters = st->it + 1; st->final_norm = st->norm_r;
            } else {
                st->beta = s_to2<S>(ST<S>::div(rho_new, rho));
                st->rho = total;
            }
            break;
        }
        default:
            break;
    }
}

// Grid-level deterministic reduction tail: every block stores its partial,
// the last block to arrive sums them in block order. Returns true in the
// thread that holds the final total (thread 0 of the last block).
__device__ inline bool grid_reduce2(double2 part, double2* partials, unsigned int* ticket,
                                    double2& total) {
    __shared__ bool am_last;
    part = block_sum2(part);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = part;
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double2 s = make_double2(0.0, 0.0);
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s = add2(s, __ldcg(&partials[i]));
    s = block_sum2(s);
    if (threadIdx.x == 0) {
        *ticket = 0u;
        total = s;
        return true;
    }
    return false;
}

struct RedBuf {
    double2* partials;
    unsigned int* ticket;
};

// ---------------------------------------------------------------------------
// SpMV family: a sub-warp of LANES threads per row, lanes stride the row; each
// row group takes U rows per pass and issues all their loads before using
// them (more HBM requests in flight; same per-row summation order for any U).
// MODE 0: y = A x.  MODE 1: y = A x and reduce dot(x, y) (conj(x) if conj).
// MODE 2: y = b - A x.  MODE 3: y = A x and reduce x^T y (unconjugated).
// ---------------------------------------------------------------------------
template <typename S, typename SV, int LANES, int MODE, int U = 1>
__global__ void __launch_bounds__(kBlock)
k_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const SV* __restrict__ v,
       const S* __restrict__ x, S* __restrict__ y, const S* __restrict__ b,
       const uint8_t* __restrict__ mask, KState* st, int op, RedBuf red, double2* out) {
    pdl_gate();
    if (st && st->done) return;
    const int sub = threadIdx.x % LANES;
    const int rows_per_block = kBlock / LANES;
    // The loop bound is taken at the warp's first row so that every lane of a
    // warp runs the same trip count: the full-mask shuffles below need all 32
    // lanes (rows past n compute zero and store nothing).
    const int lane_row = (threadIdx.x & 31) / LANES;
    double2 part = make_double2(0.0, 0.0);
    const bool conj = st ? (st->conj != 0) : false;
    for (int row0 = blockIdx.x * rows_per_block * U + threadIdx.x / LANES; row0 - lane_row < n;
         row0 += gridDim.x * rows_per_block * U) {
        int kk[U], ke[U];
        S acc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int row = row0 + u * rows_per_block;
            kk[u] = row < n ? rp[row] + sub : 0;
            ke[u] = row < n ? rp[row + 1] : 0;
            acc[u] = ST<S>::zero();
        }
        while (true) {
            SV a[U];
            int col[U];
            bool any = false;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const bool on = kk[u] < ke[u];
                if (on) {
                    a[u] = v[kk[u]];
                    col[u] = ci[kk[u]];
                } else {
                    col[u] = -1;
                }
                any |= on;
            }
            if (!any) break;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (col[u] >= 0) {
                    acc[u] = ST<S>::fma(hi_of_any(a[u]), x[col[u]], acc[u]);
                    kk[u] += LANES;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int o = LANES / 2; o > 0; o >>= 1) {
                if constexpr (ST<S>::cplx) {
                    acc[u].x += __shfl_down_sync(0xffffffffu, acc[u].x, o, LANES);
                    acc[u].y += __shfl_down_sync(0xffffffffu, acc[u].y, o, LANES);
                } else {
                    acc[u] += __shfl_down_sync(0xffffffffu, acc[u], o, LANES);
                }
            }
            const int row = row0 + u * rows_per_block;
            if (sub == 0 && row < n) {
                S r = acc[u];
                if (mask && !mask[row]) r = ST<S>::zero();  // project() of the NGSolve COCR loop
                if constexpr (MODE == 2) {
                    y[row] = b[row] - r;
                } else {
                    y[row] = r;
                }
                if constexpr (MODE == 1) {
                    S xi = x[row];
                    S d = (conj ? ST<S>::conj(xi) : xi) * r;
                    part = add2(part, s_to2<S>(d));
                } else if constexpr (MODE == 3) {
                    part = add2(part, s_to2<S>(x[row] * r));
                }
            }
        }
    }
    if constexpr (MODE == 1 || MODE == 3) {
        double2 total;
        if (grid_reduce2(part, red.partials, red.ticket, total)) finish_reduction<S>(total, st, op, out);
    }
}

// Generic reductions: dot(a, b) (conj(a) if conj), |a|^2.
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_dot(int n, const S* __restrict__ a, const S* __restrict__ b, int conj, KState* st, int op,
      RedBuf red, double2* out) {
    pdl_gate();
    if (st && st->done && op != RED_STORE) return;
    double2 part = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        S ai = a[i];
        part = add2(part, s_to2<S>((conj ? ST<S>::conj(ai) : ai) * b[i]));
    }
    double2 total;
    if (grid_reduce2(part, red.partials, red.ticket, total)) finish_reduction<S>(total, st, op, out);
}

template <typename S>
__global__ void __launch_bounds__(kBlock)
k_norm2(int n, const S* __restrict__ a, RedBuf red, double2* out) {
    pdl_gate();
    double2 part = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        part.x += ST<S>::norm2(a[i]);
    double2 total;
    if (grid_reduce2(part, red.partials, red.ticket, total)) *out = total;
}

// CG step: x_nxt = x_cur + alpha p ; r -= alpha Ap ; ||r|| -> check.
// With save_best the new x goes to the third buffer (neither current nor
// best), so the best iterate is kept without a copy.
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_cg_update(int n, S* xb0, S* xb1, S* xb2, const S* __restrict__ p, const S* __restrict__ Ap,
            S* __restrict__ r, KState* st, RedBuf red) {
    pdl_gate();
    if (st->done) return;
    const int brk = st->breakdown;
    const int cur = st->cur;
    int nxt = cur;
    if (st->save_best) {
        const int best = st->best;
        for (int c = 0; c < 3; ++c) if (c != cur && c != best) { nxt = c; break; }
    }
    S* xs[3] = {xb0, xb1, xb2};
    const S* xc = xs[cur];
    S* xn = xs[nxt];
    const S alpha = s_from2<S>(st->alpha);
    double2 part = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        S ri = r[i];
        if (!brk) {
            xn[i] = ST<S>::fma(alpha, p[i], xc[i]);
            ri = ri - alpha * Ap[i];
            r[i] = ri;
        }
        part.x += ST<S>::norm2(ri);
    }
    double2 total;
    if (grid_reduce2(part, red.partials, red.ticket, total)) {
        dev_check(st, sqrt(total.x), brk, brk ? cur : nxt);
        st->breakdown = 0;
    }
}

// COCR step (cocr_solver.hpp:118-128): x += alpha p, r -= alpha q,
// rt -= alpha qt, ||r||.
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_cocr_update(int n, S* xb0, S* xb1, S* xb2, const S* __restrict__ p, const S* __restrict__ q,
              const S* __restrict__ qt, S* __restrict__ r, S* __restrict__ rt, KState* st,
              RedBuf red) {
    pdl_gate();
    if (st->done) return;
    const int brk = st->breakdown;
    const int cur = st->cur;
    int nxt = cur;
    if (st->save_best) {
        const int best = st->best;
        for (int c = 0; c < 3; ++c) if (c != cur && c != best) { nxt = c; break; }
    }
    S* xs[3] = {xb0, xb1, xb2};
    const S* xc = xs[cur];
    S* xn = xs[nxt];
    const S alpha = s_from2<S>(st->alpha);
    double2 part = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        S ri = r[i];
        if (!brk) {
            xn[i] = ST<S>::fma(alpha, p[i], xc[i]);
            ri = ri - alpha * q[i];
            r[i] = ri;
            rt[i] = rt[i] - alpha * qt[i];
        }
        part.x += ST<S>::norm2(ri);
    }
    double2 total;
    if (grid_reduce2(part, red.partials, red.ticket, total)) {
        dev_check(st, sqrt(total.x), brk, brk ? cur : nxt);
        st->breakdown = 0;
    }
}

// p = z + beta p (cg_solver.hpp:493-495)
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_pupdate(int n, const S* __restrict__ z, S* __restrict__ p, const KState* st) {
    pdl_gate();
    if (st->done) return;
    const S beta = s_from2<S>(st->beta);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        p[i] = ST<S>::fma(beta, p[i], z[i]);
}

// p = rt + beta p ; q = t + beta q (cocr_solver.hpp:159-162)
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_cocr_pq(int n, const S* __restrict__ rt, const S* __restrict__ t, S* __restrict__ p,
          S* __restrict__ q, const KState* st) {
    pdl_gate();
    if (st->done) return;
    const S beta = s_from2<S>(st->beta);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        p[i] = ST<S>::fma(beta, p[i], rt[i]);
        q[i] = ST<S>::fma(beta, q[i], t[i]);
    }
}

// Loop control, last node of the iteration body: advance `iter`, stop at
// maxiter (cg_solver.hpp:498-500), enforce the loop guard, and steer the
// graph's WHILE node when one is used.
__global__ void k_loop_ctl(KState* st, cudaGraphConditionalHandle h, int use_cond);

// ---------------------------------------------------------------------------
// Vector helpers
// ---------------------------------------------------------------------------
template <typename S>
__global__ void k_copy(int n, const S* __restrict__ a, S* __restrict__ b) {
    pdl_gate();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}

// dst[perm[i]] = src[i] * (mask ? mask[i] : 1)  (gather into a new numbering)
template <typename S>
__global__ void k_scatter_perm(int n, const int* __restrict__ perm, const S* __restrict__ src,
                               S* __restrict__ dst, const uint8_t* __restrict__ mask) {
    pdl_gate();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        S v = src[i];
        if (mask && !mask[i]) v = ST<S>::zero();
        dst[perm[i]] = v;
    }
}

// dst[i] = src[perm[i]], optionally only where mask[i] (else untouched) or
// zeroed where !mask[i] (zero_masked).
template <typename S>
__global__ void k_gather_perm(int n, const int* __restrict__ perm, const S* __restrict__ src,
                              S* __restrict__ dst, const uint8_t* __restrict__ mask, int zero_masked) {
    pdl_gate();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (mask && !mask[i]) {
            if (zero_masked) dst[i] = ST<S>::zero();
            continue;
        }
        dst[i] = perm ? src[perm[i]] : src[i];
    }
}

template <typename S>
__global__ void k_mask_zero(int n, S* __restrict__ a, const uint8_t* __restrict__ mask) {
    pdl_gate();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (!mask[i]) a[i] = ST<S>::zero();
}

template <typename S>
__global__ void k_scale_real(int n, S* __restrict__ a, const double* __restrict__ s) {
    pdl_gate();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a[i] = ST<S>::scale(s[i], a[i]);
}

// BuildSparseMatrixView's FreeDofs rule (ngsolve/sparsesolv_precond.hpp:65-74):
// constrained row -> identity row, constrained column -> 0.
template <typename S>
__global__ void k_bc_values(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            const S* __restrict__ v, const uint8_t* __restrict__ fd, S* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool fi = fd[i] != 0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            S a = v[k];
            if (!fi) a = (j == i) ? ST<S>::one() : ST<S>::zero();
            else if (!fd[j]) a = ST<S>::zero();
            out[k] = a;
        }
    }
}

// out[k] = src[map[k]]
template <typename S>
__global__ void k_gather_values(int64_t m, const int* __restrict__ map, const S* __restrict__ src,
                                S* __restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
         k += (int64_t)gridDim.x * blockDim.x)
        out[k] = src[map[k]];
}

template <typename S, typename SL>
__global__ void k_to_lo(int64_t m, const S* __restrict__ src, SL* __restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
         k += (int64_t)gridDim.x * blockDim.x)
        out[k] = lo_of(src[k]);
}

// ---------------------------------------------------------------------------
// IC(0): factorisation and triangular solves over "units" -- an ABMC block
// (rows sequential inside) or a single row of a level set. A launch covers
// units [u0, u1) of one colour / level; unit u has rows
// rows[uoff[u]] .. rows[uoff[u+1]-1] (rows == nullptr: the identity).
// ---------------------------------------------------------------------------

// L(i,j) updates and the shifted diagonal (ic_preconditioner.hpp:1325-1397).
template <typename S>
__global__ void k_ic_factor(int u0, int u1, const int* __restrict__ uoff, const int* __restrict__ rows,
                            const int* __restrict__ Lrp, const int* __restrict__ Lci, S* __restrict__ Lv,
                            S* __restrict__ inv_diag, double shift, double min_diag, double zero_repl,
                            int auto_shift, int* need_restart) {
    const int u = u0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= u1) return;
    const int qa = uoff ? uoff[u] : u, qb = uoff ? uoff[u + 1] : u + 1;
    for (int q = qa; q < qb; ++q) {
        const int i = rows ? rows[q] : q;
        const int rs = Lrp[i], re = Lrp[i + 1];
        for (int kk = rs; kk < re - 1; ++kk) {
            const int j = Lci[kk];
            if (j >= i) break;
            S s = Lv[kk];
            const int js = Lrp[j], je = Lrp[j + 1];
            int jj = js;
            for (int ii = rs; ii < kk; ++ii) {
                const int k = Lci[ii];
                if (k >= j) break;
                // row j is sorted: resume the scan where the last k stopped
                while (jj < je && Lci[jj] < k) ++jj;
                if (jj < je && Lci[jj] == k) s = s - Lv[ii] * Lv[jj] * inv_diag[k];
            }
            Lv[kk] = s;
        }
        const int dp = re - 1;
        const S orig = Lv[dp];
        S s = orig * ST<S>::from(shift);
        for (int kk = rs; kk < dp; ++kk) {
            const int k = Lci[kk];
            if (k >= i) break;
            s = s - Lv[kk] * Lv[kk] * inv_diag[k];
        }
        Lv[dp] = s;
        const double abs_s = ST<S>::abs(s);
        if (auto_shift && abs_s < min_diag && ST<S>::abs(orig) > 0.0) atomicExch(need_restart, 1);
        if (abs_s > zero_repl) {
            inv_diag[i] = ST<S>::div(ST<S>::one(), s);
        } else {
            const S safe = ST<S>::from(zero_repl);
            Lv[dp] = safe;
            inv_diag[i] = ST<S>::div(ST<S>::one(), safe);
        }
    }
}

// Forward sweep: y_i = (x_i * sc_i - sum_{j<i} L_ij y_j) / L_ii
// (ic_preconditioner.hpp:1021-1031). SL is the storage type of L (FP64 or the
// FP32 form); arithmetic stays in S.
template <typename S, typename SL>
__global__ void __launch_bounds__(128)
k_ic_fwd(int u0, int u1, const int* __restrict__ uoff, const int* __restrict__ rows,
         const int* __restrict__ Lrp, const int* __restrict__ Lci, const SL* __restrict__ Lv,
         const S* __restrict__ x, const double* __restrict__ sc, S* __restrict__ y, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int u = u0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= u1) return;
    const int qa = uoff ? uoff[u] : u, qb = uoff ? uoff[u + 1] : u + 1;
    for (int q = qa; q < qb; ++q) {
        const int i = rows ? rows[q] : q;
        S s = x[i];
        if (sc) s = ST<S>::scale(sc[i], s);
        const int ks = Lrp[i], ke = Lrp[i + 1] - 1;
        for (int k = ks; k < ke; ++k) s = s - hi_of_any(Lv[k]) * y[Lci[k]];
        y[i] = ST<S>::div(s, hi_of_any(Lv[ke]));
    }
}

// Backward sweep: y_i = -(sum_{j>i} L_ji y_j) * D^{-1}_i + x_i
// (ic_preconditioner.hpp:1053-1063), over L^T stored with the diagonal first.
template <typename S, typename SL>
__global__ void __launch_bounds__(128)
k_ic_bwd(int u0, int u1, const int* __restrict__ uoff, const int* __restrict__ rows,
         const int* __restrict__ Urp, const int* __restrict__ Uci, const SL* __restrict__ Uv,
         const SL* __restrict__ inv_diag, const S* __restrict__ x, S* __restrict__ y, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int u = u0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= u1) return;
    const int qa = uoff ? uoff[u] : u, qb = uoff ? uoff[u + 1] : u + 1;
    for (int q = qb - 1; q >= qa; --q) {
        const int i = rows ? rows[q] : q;
        S s = ST<S>::zero();
        const int ks = Urp[i] + 1, ke = Urp[i + 1];
        for (int k = ks; k < ke; ++k) s = s - hi_of_any(Uv[k]) * y[Uci[k]];
        y[i] = s * hi_of_any(inv_diag[i]) + x[i];
    }
}

// ---------------------------------------------------------------------------
// ABMC block sweeps, one sub-warp of LANES (>= rows per block) lanes per
// ABMC block: lane j owns row r0+j. The terms coupling a row to rows of
// earlier colours ("external", a CSR without the block's own columns) are
// gathered by all lanes at once; the couplings inside the block come from a
// packed strictly-lower table (entry (j,t) at j*(j-1)/2+t) and are resolved
// row by row through register shuffles. The loops are warp-uniform.
// ---------------------------------------------------------------------------
template <typename S>
__device__ __forceinline__ S shfl_s(S v, int src, int width) {
    if constexpr (ST<S>::cplx) {
        return S{__shfl_sync(0xffffffffu, v.x, src, width), __shfl_sync(0xffffffffu, v.y, src, width)};
    } else {
        return __shfl_sync(0xffffffffu, v, src, width);
    }
}

// forward: y_i = (x_i*sc_i - sum_ext L_ik y_k - sum_{t<j} L_jt y_t) / L_ii
template <typename S, typename SL, int LANES>
__global__ void __launch_bounds__(128)
k_ic_fwd_blk(int b0, int b1, const int* __restrict__ boff, const int* __restrict__ erp,
             const int* __restrict__ eci, const SL* __restrict__ ev, const SL* __restrict__ iv, int tri,
             const SL* __restrict__ dv, const S* __restrict__ x, const double* __restrict__ sc,
             S* __restrict__ y, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int lane = threadIdx.x % LANES;
    const int gw = (threadIdx.x & 31) / LANES;
    const int stride = gridDim.x * (blockDim.x / LANES);
    for (int b = b0 + blockIdx.x * (blockDim.x / LANES) + threadIdx.x / LANES; b - gw < b1; b += stride) {
        const bool vb = b < b1;
        int r0 = 0, nr = 0;
        if (vb) { r0 = boff[b]; nr = boff[b + 1] - r0; }
        const bool act = vb && lane < nr;
        const int i = r0 + lane;
        S s = ST<S>::zero();
        if (act) {
            s = x[i];
            if (sc) s = ST<S>::scale(sc[i], s);
            const int k1 = erp[i + 1];
            for (int k = erp[i]; k < k1; ++k) s = s - hi_of_any(ev[k]) * y[eci[k]];
        }
        S yi = ST<S>::zero();
        const SL* ib = iv + (size_t)(vb ? b : 0) * tri;
#pragma unroll
        for (int t = 0; t < LANES; ++t) {
            if (act && lane == t) yi = ST<S>::div(s, hi_of_any(dv[i]));
            const S yt = shfl_s(yi, t, LANES);
            if (act && t < lane) s = s - hi_of_any(ib[lane * (lane - 1) / 2 + t]) * yt;
        }
        if (act) y[i] = yi;
    }
}

// backward: y_i = -(sum_ext U_ik y_k + sum_{t>j} L_tj y_t) * D^{-1}_i + x_i
template <typename S, typename SL, int LANES>
__global__ void __launch_bounds__(128)
k_ic_bwd_blk(int b0, int b1, const int* __restrict__ boff, const int* __restrict__ urp,
             const int* __restrict__ uci, const SL* __restrict__ uv, const SL* __restrict__ iv, int tri,
             const SL* __restrict__ inv, const S* __restrict__ x, S* __restrict__ y, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int lane = threadIdx.x % LANES;
    const int gw = (threadIdx.x & 31) / LANES;
    const int stride = gridDim.x * (blockDim.x / LANES);
    for (int b = b0 + blockIdx.x * (blockDim.x / LANES) + threadIdx.x / LANES; b - gw < b1; b += stride) {
        const bool vb = b < b1;
        int r0 = 0, nr = 0;
        if (vb) { r0 = boff[b]; nr = boff[b + 1] - r0; }
        const bool act = vb && lane < nr;
        const int i = r0 + lane;
        S s = ST<S>::zero();
        if (act) {
            const int k1 = urp[i + 1];
            for (int k = urp[i]; k < k1; ++k) s = s - hi_of_any(uv[k]) * y[uci[k]];
        }
        S yi = ST<S>::zero();
        const SL* ib = iv + (size_t)(vb ? b : 0) * tri;
#pragma unroll
        for (int t = LANES - 1; t >= 0; --t) {
            if (act && lane == t) yi = s * hi_of_any(inv[i]) + x[i];
            const S yt = shfl_s(yi, t, LANES);
            if (act && lane < t && t < nr) s = s - hi_of_any(ib[t * (t - 1) / 2 + lane]) * yt;
        }
        if (act) y[i] = yi;
    }
}

// out[k] = src[map[k]], or zero where map[k] < 0
template <typename S, typename SO>
__global__ void k_gather_or_zero(int64_t m, const int* __restrict__ map, const S* __restrict__ src,
                                 SO* __restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int q = map[k];
        if constexpr (std::is_same<S, SO>::value) out[k] = q >= 0 ? src[q] : ST<S>::zero();
        else out[k] = lo_of(q >= 0 ? src[q] : ST<S>::zero());
    }
}

// ---------------------------------------------------------------------------
// Oversized ABMC blocks (the aggregation's leftover rows): one CTA walks the
// block's level sets, rows of a level in parallel, __syncthreads() between
// levels (global writes of the CTA are visible to it after the barrier).
// lev[0..nlev] are offsets into rows[].
// ---------------------------------------------------------------------------
template <typename S, typename SL>
__global__ void __launch_bounds__(256)
k_ic_fwd_cta(int nlev, const int* __restrict__ lev, const int* __restrict__ rows, const int* __restrict__ Lrp,
             const int* __restrict__ Lci, const SL* __restrict__ Lv, const S* __restrict__ x,
             const double* __restrict__ sc, S* y, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    for (int l = 0; l < nlev; ++l) {
        const int q1 = lev[l + 1];
        for (int q = lev[l] + threadIdx.x; q < q1; q += blockDim.x) {
            const int i = rows[q];
            S s = x[i];
            if (sc) s = ST<S>::scale(sc[i], s);
            const int ke = Lrp[i + 1] - 1;
            for (int k = Lrp[i]; k < ke; ++k) s = s - hi_of_any(Lv[k]) * y[Lci[k]];
            y[i] = ST<S>::div(s, hi_of_any(Lv[ke]));
        }
        __syncthreads();
    }
}

template <typename S, typename SL>
__global__ void __launch_bounds__(256)
k_ic_bwd_cta(int nlev, const int* __restrict__ lev, const int* __restrict__ rows, const int* __restrict__ Urp,
             const int* __restrict__ Uci, const SL* __restrict__ Uv, const SL* __restrict__ inv_diag,
             const S* __restrict__ x, S* y, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    for (int l = 0; l < nlev; ++l) {
        const int q1 = lev[l + 1];
        for (int q = lev[l] + threadIdx.x; q < q1; q += blockDim.x) {
            const int i = rows[q];
            S s = ST<S>::zero();
            const int ke = Urp[i + 1];
            for (int k = Urp[i] + 1; k < ke; ++k) s = s - hi_of_any(Uv[k]) * y[Uci[k]];
            y[i] = s * hi_of_any(inv_diag[i]) + x[i];
        }
        __syncthreads();
    }
}

// Oversized ABMC block, staged: the block's rows, their L (forward) or U
// (backward) entries and the values of the couplings to other blocks (final
// before the launch) are copied into shared memory first, so the chain of
// level sets touches only shared memory. Same per-row arithmetic, in the same
// order, as k_ic_fwd_cta / k_ic_bwd_cta. Per-row entry lists: srp (by position
// in rows[]), value index ssrc, column scol, and sloc = the column's position
// within the block (relative to lev[0]) or -1 for a coupling outside it.
template <typename S, typename SL>
struct StagedSmem {
    S* ys;
    S* xs;
    S* eext;
    SL* dg;
    SL* ev;
    int* eloc;
    int* slev;
    int* srow;
};

__host__ __device__ inline size_t staged_align(size_t b) { return (b + 15) & ~size_t(15); }

template <typename S, typename SL>
__host__ __device__ inline size_t staged_bytes(int nr, int ne, int nlev) {
    return 2 * staged_align((size_t)nr * sizeof(S)) + staged_align((size_t)ne * sizeof(S)) +
           staged_align((size_t)nr * sizeof(SL)) + staged_align((size_t)ne * sizeof(SL)) +
           staged_align((size_t)ne * 4) + staged_align((size_t)(nlev + 1) * 4) + staged_align((size_t)(nr + 1) * 4);
}

// Loads of values that other CTAs of the same launch may have written: served
// by L2 (the point of coherence), never by a possibly stale L1 line.
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ zdouble ld_cg(const zdouble* p) {
    const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
    return {v.x, v.y};
}

template <typename S, typename SL, bool FWD>
__device__ __forceinline__ void staged_sweep(unsigned char* smem, int nlev, const int* __restrict__ lev,
                                             const int* __restrict__ rows, const int* __restrict__ srp,
                                             const int* __restrict__ ssrc, const int* __restrict__ scol,
                                             const int* __restrict__ sloc, const int* __restrict__ Lrp,
                                             const SL* __restrict__ vals, const SL* __restrict__ inv_diag,
                                             const S* __restrict__ x, const double* __restrict__ sc, S* y) {
    const int qa = lev[0], qb = lev[nlev];
    const int nr = qb - qa;
    const int ea = srp[qa], ne = srp[qb] - ea;
    unsigned char* p = smem;
    S* ys = reinterpret_cast<S*>(p);   p += staged_align((size_t)nr * sizeof(S));
    S* xs = reinterpret_cast<S*>(p);   p += staged_align((size_t)nr * sizeof(S));
    S* eext = reinterpret_cast<S*>(p); p += staged_align((size_t)ne * sizeof(S));
    SL* dg = reinterpret_cast<SL*>(p); p += staged_align((size_t)nr * sizeof(SL));
    SL* ev = reinterpret_cast<SL*>(p); p += staged_align((size_t)ne * sizeof(SL));
    int* eloc = reinterpret_cast<int*>(p); p += staged_align((size_t)ne * 4);
    int* slev = reinterpret_cast<int*>(p); p += staged_align((size_t)(nlev + 1) * 4);
    int* srow = reinterpret_cast<int*>(p);
    for (int l = threadIdx.x; l <= nlev; l += blockDim.x) slev[l] = lev[l] - qa;
    for (int q = threadIdx.x; q <= nr; q += blockDim.x) srow[q] = srp[qa + q] - ea;
    for (int q = threadIdx.x; q < nr; q += blockDim.x) {
        const int i = rows[qa + q];
        if constexpr (FWD) {
            S v = x[i];
            if (sc) v = ST<S>::scale(sc[i], v);
            xs[q] = v;
            dg[q] = vals[Lrp[i + 1] - 1];
        } else {
            xs[q] = x[i];
            dg[q] = inv_diag[i];
        }
    }
    for (int e = threadIdx.x; e < ne; e += blockDim.x) {
        const int loc = sloc[ea + e];
        eloc[e] = loc;
        ev[e] = vals[ssrc[ea + e]];
        eext[e] = loc < 0 ? ld_cg(y + scol[ea + e]) : ST<S>::zero();
    }
    __syncthreads();
    for (int l = 0; l < nlev; ++l) {
        const int q1 = slev[l + 1];
        for (int q = slev[l] + threadIdx.x; q < q1; q += blockDim.x) {
            S s = FWD ? xs[q] : ST<S>::zero();
            const int e1 = srow[q + 1];
            for (int e = srow[q]; e < e1; ++e) {
                const int loc = eloc[e];
                const S yv = loc < 0 ? eext[e] : ys[loc];
                s = s - hi_of_any(ev[e]) * yv;
            }
            if constexpr (FWD) ys[q] = ST<S>::div(s, hi_of_any(dg[q]));
            else ys[q] = s * hi_of_any(dg[q]) + xs[q];
        }
        __syncthreads();
    }
    for (int q = threadIdx.x; q < nr; q += blockDim.x) y[rows[qa + q]] = ys[q];
}

template <typename S, typename SL, bool FWD>
__global__ void __launch_bounds__(256)
k_ic_sweep_staged(int nlev, const int* __restrict__ lev, const int* __restrict__ rows, const int* __restrict__ srp,
                  const int* __restrict__ ssrc, const int* __restrict__ scol, const int* __restrict__ sloc,
                  const int* __restrict__ Lrp, const SL* __restrict__ vals, const SL* __restrict__ inv_diag,
                  const S* __restrict__ x, const double* __restrict__ sc, S* y, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    extern __shared__ __align__(16) unsigned char smem[];
    staged_sweep<S, SL, FWD>(smem, nlev, lev, rows, srp, ssrc, scol, sloc, Lrp, vals, inv_diag, x, sc, y);
}

}  // namespace ssv
