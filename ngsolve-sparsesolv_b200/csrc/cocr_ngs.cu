// cocr_ngs.cu -- COCRSolver with an external preconditioner
// (COCRSolverNGS::Mult, include/sparsesolv/ngsolve/sparsesolv_solvers.hpp:273-369)
// as one CUDA graph: the preconditioner's kernels are captured into the same
// iteration body, and the scalar steps run in the reductions' last block.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>

#include "objects.cuh"
#include "solver_api.hpp"

namespace ssv {

enum NgsOp : int { NGS_MU = 100, NGS_RHO = 101 };

template <typename S>
__device__ inline void ngs_finish(double2 total, KState* st, int op) {
    if (op == NGS_MU) {  // :323-327 (brk_thr = 1e-30 in the reference's form)
        const S mu = s_from2<S>(total);
        if (ST<S>::abs(mu) < st->brk_thr) { st->done = 1; st->iters = st->it; return; }
        st->alpha = s_to2<S>(ST<S>::div(s_from2<S>(st->rho), mu));
    } else if (op == NGS_RHO) {  // :354-359
        const S rho = s_from2<S>(st->rho);
        if (ST<S>::abs(rho) < st->brk_thr) { st->done = 1; st->iters = st->it; return; }
        st->beta = s_to2<S>(ST<S>::div(s_from2<S>(total), rho));
        st->rho = total;
    }
}

// mu = qt^T q (unconjugated)
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_ngs_dot(int n, const S* __restrict__ a, const S* __restrict__ b, KState* st, int op, RedBuf red) {
    pdl_gate();
    if (st->done) return;
    double2 part = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        part = add2(part, s_to2<S>(a[i] * b[i]));
    double2 total;
    if (grid_reduce2(part, red.partials, red.ticket, total)) ngs_finish<S>(total, st, op);
}

// t = A rt, projected; rho_new = rt^T t
template <typename S, int LANES>
__global__ void __launch_bounds__(kBlock)
k_ngs_spmv_dot(int n, const int* __restrict__ rp, const int* __restrict__ ci, const S* __restrict__ v,
               const S* __restrict__ x, S* __restrict__ y, const uint8_t* __restrict__ mask, KState* st,
               RedBuf red) {
    pdl_gate();
    if (st->done) return;
    const int sub = threadIdx.x % LANES;
    const int rpb = kBlock / LANES;
    const int lane_row = (threadIdx.x & 31) / LANES;  // warp-uniform trip count (full-mask shuffles)
    double2 part = make_double2(0.0, 0.0);
    for (int row = blockIdx.x * rpb + threadIdx.x / LANES; row - lane_row < n; row += gridDim.x * rpb) {
        const bool valid = row < n;
        S acc = ST<S>::zero();
        if (valid)
            for (int k = rp[row] + sub; k < rp[row + 1]; k += LANES) acc = ST<S>::fma(v[k], x[ci[k]], acc);
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1) {
            if constexpr (ST<S>::cplx) {
                acc.x += __shfl_down_sync(0xffffffffu, acc.x, o, LANES);
                acc.y += __shfl_down_sync(0xffffffffu, acc.y, o, LANES);
            } else {
                acc += __shfl_down_sync(0xffffffffu, acc, o, LANES);
            }
        }
        if (sub == 0 && valid) {
            if (mask && !mask[row]) acc = ST<S>::zero();
            y[row] = acc;
            part = add2(part, s_to2<S>(x[row] * acc));
        }
    }
    double2 total;
    if (grid_reduce2(part, red.partials, red.ticket, total)) ngs_finish<S>(total, st, NGS_RHO);
}

// The same through the matrix's sliced-ELL copy (sell.cuh): one warp per
// slice of 32 rows, a lane per row, R steps per round with the next round's
// values and columns loaded before this round's gathers; each row is summed
// in its CSR column order.
template <typename S, int R>
__global__ void __launch_bounds__(kBlock)
k_ngs_sell_dot(int slices, const int* __restrict__ off, const int* __restrict__ rows, const int* __restrict__ ci,
               const S* __restrict__ v, const S* __restrict__ x, S* __restrict__ y, const uint8_t* __restrict__ mask,
               KState* st, RedBuf red) {
    pdl_gate();
    if (st->done) return;
    const int lane = threadIdx.x & 31;
    const int wpb = kBlock / 32;
    double2 part = make_double2(0.0, 0.0);
    for (int sl = blockIdx.x * wpb + threadIdx.x / 32; sl < slices; sl += gridDim.x * wpb) {
        const int e1 = off[sl + 1];
        int e = off[sl] + lane;
        const int row = rows[(size_t)sl * 32 + lane];
        S acc = ST<S>::zero();
        S a[R];
        int col[R];
#pragma unroll
        for (int u = 0; u < R; ++u) {
            const int k = e + 32 * u;
            a[u] = k < e1 ? v[k] : ST<S>::zero();
            col[u] = k < e1 ? ci[k] : -1;
        }
        while (e < e1) {
            const int en = e + 32 * R;
            S an[R];
            int cn[R];
#pragma unroll
            for (int u = 0; u < R; ++u) {
                const int k = en + 32 * u;
                an[u] = k < e1 ? v[k] : ST<S>::zero();
                cn[u] = k < e1 ? ci[k] : -1;
            }
#pragma unroll
            for (int u = 0; u < R; ++u)
                if (col[u] >= 0) acc = ST<S>::fma(a[u], x[col[u]], acc);
#pragma unroll
            for (int u = 0; u < R; ++u) {
                a[u] = an[u];
                col[u] = cn[u];
            }
            e = en;
        }
        if (row >= 0) {
            if (mask && !mask[row]) acc = ST<S>::zero();
            y[row] = acc;
            part = add2(part, s_to2<S>(x[row] * acc));
        }
    }
    double2 total;
    if (grid_reduce2(part, red.partials, red.ticket, total)) ngs_finish<S>(total, st, NGS_RHO);
}

// SSV_KRYLOV_SELL=0: the COCR iteration's SpMV stays on the CSR arrays
static bool krylov_sell_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("SSV_KRYLOV_SELL");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v != 0;
}

// The matrix's sliced-ELL values for the iteration's SpMV, or null (small
// matrices, switched off, or a layout past the int range): the layout is built
// once per matrix, the values gathered again whenever they changed. Called
// outside any capture.
static const double* krylov_sell(ssv_matrix* A, cudaStream_t s) {
    if (!krylov_sell_enabled() || A->rows < 65536) return nullptr;
    if (!A->sell_tried) {  // marked tried only once the layout and its value array exist
        if (!A->sell.build_pattern(A->rows, A->nnz, A->rp.get(), A->ci.get(), s)) {
            A->sell_tried = true;
            return nullptr;
        }
        try {
            A->sell_v.alloc((size_t)std::max<int64_t>(A->sell.entries, 1) * (A->dtype == SSV_F64 ? 1 : 2));
        } catch (...) {
            A->sell.invalidate();
            throw;
        }
        A->sell_vgen = ~A->vgen;  // gather below
        A->sell_tried = true;
    }
    if (A->sell.slices <= 0) return nullptr;
    if (A->sell_vgen != A->vgen) {
        sell_gather(A->sell, A->val.get(), A->dtype == SSV_F64 ? 1 : 2, A->sell_v.get(), s);
        A->sell_vgen = A->vgen;
    }
    return A->sell_v.get();
}

// sol += alpha p ; r -= alpha q ; rt -= alpha qt ; res = sqrt(|r^H r|)
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_ngs_update(int n, S* __restrict__ x, const S* __restrict__ p, const S* __restrict__ q,
             const S* __restrict__ qt, S* __restrict__ r, S* __restrict__ rt, KState* st, RedBuf red) {
    pdl_gate();
    if (st->done) return;
    const S alpha = s_from2<S>(st->alpha);
    double2 part = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = ST<S>::fma(alpha, p[i], x[i]);
        const S ri = r[i] - alpha * q[i];
        r[i] = ri;
        rt[i] = rt[i] - alpha * qt[i];
        part.x += ST<S>::norm2(ri);
    }
    double2 total;
    if (grid_reduce2(part, red.partials, red.ticket, total)) {
        const double res = std::sqrt(std::fabs(total.x));
        st->norm_r = res;
        st->updates++;
        if (st->save_hist) {
            if (st->hist_len < st->hist_cap) st->hist[st->hist_len] = res / st->normalizer;
            st->hist_len++;
        }
        if (res / st->normalizer <= st->tol) {  // :344-347
            st->done = 1;
            st->converged = 1;
            st->iters = st->it + 1;
        } else if (res <= st->restart_abs) {  // refined form: this cycle has done its part
            st->done = 1;
            st->iters = st->it + 1;
        }
    }
}

__global__ void k_ngs_loop_ctl(KState* st, cudaGraphConditionalHandle h, int use_cond) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (!st->done) {
        st->it++;
        if (st->it >= st->maxiter) { st->done = 1; st->iters = st->maxiter; }  // :368
    }
    st->loops++;
    if (!st->done && st->loops >= st->max_loops) { st->done = 1; st->status = SSV_ERR_TIMEOUT; }
    if (use_cond) cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

struct CocrCtx {
    KrylovWork<double> w_d;
    KrylovWork<zdouble> w_z;
    GraphLoop loop, pcg_loop;
    DevBuf<double> vals_bc;
};

static std::map<const ssv_matrix*, std::unique_ptr<CocrCtx>>& cocr_table() {
    static std::map<const ssv_matrix*, std::unique_ptr<CocrCtx>> t;
    return t;
}

void cocr_forget(const ssv_matrix* A) { cocr_table().erase(A); }

template <typename S> KrylovWork<S>& cw_of(CocrCtx& c);
template <> KrylovWork<double>& cw_of<double>(CocrCtx& c) { return c.w_d; }
template <> KrylovWork<zdouble>& cw_of<zdouble>(CocrCtx& c) { return c.w_z; }

template <typename S>
static void apply_pre(ssv_precond* pre, const S* x, S* y, const KState* st, int n, cudaStream_t s) {
    if (pre) precond_apply_any<S>(pre, x, y, st, s);
    else launch_k(k_copy<S>, grid_for(n, kBlock), kBlock, s, n, x, y);
}

static std::string pre_key(const ssv_precond* pre) {
    if (!pre) return "nopre";
    std::string k = std::to_string((size_t)pre) + ":" + std::to_string(pre->kind) + ":" +
                    std::to_string(precond_generation(pre)) + ":" + std::to_string((size_t)pre->xw.get());
    if (pre->kind == 1) {
        k += ":" + std::to_string(pre->A->dtype == SSV_F64 ? pre->ic_d.lo : pre->ic_z.lo) + ":" +
             std::to_string(pre->A->dtype == SSV_F64 ? pre->ic_d.abmc : pre->ic_z.abmc);
    }
    return k;
}

// One COCRSolverNGS solve (refine == nullptr), or the refined form: cycles of
// that recurrence, each started from the FP64 true residual r = P(b - A x) of
// the current x (rt = M^{-1} r, p = rt, q = P A p, rho = rt^T q) and ended when
// its residual has dropped by `drop` from its start (or on tol, a breakdown,
// maxiter); the solve stops once the true residual is <= tol. Continuing the
// same x is defect correction: each cycle solves A d = r for the correction.
// Restarting makes the recurrence consistent again with an M^{-1} that is
// not exactly linear (an FP32-form preconditioner: rt -= alpha M^{-1} q then
// drifts from M^{-1} r, which stalls the plain recurrence near the rounding
// level of M^{-1}). The reference's absolute breakdown tests (|mu|, |rho| <
// 1e-30) are scaled by (||r_start|| / ||b||)^2 in later cycles: mu and rho
// scale with the square of the residual the cycle starts from.
struct RefineOpt {
    double drop;
};

// kernels launched by the last COCR solve of this thread (measurement hook)
thread_local int64_t g_cocr_launches = 0;
int64_t cocr_last_launches() { return g_cocr_launches; }

template <typename S>
static void run_cocr_ngs(ssv_matrix* A, ssv_precond* pre, const uint8_t* fd, int maxiter, double tol,
                         int printrates, const S* d_b, S* d_x, int* iterations, const RefineOpt* refine,
                         ssv_refine_info* info) {
    cudaStream_t s = stream();
    const int n = A->rows;
    auto& ctx_ptr = cocr_table()[A];
    if (!ctx_ptr) ctx_ptr.reset(new CocrCtx());
    CocrCtx& ctx = *ctx_ptr;
    KrylovWork<S>& w = cw_of<S>(ctx);
    const int dev_hist = printrates ? std::max(maxiter, 0) + 2 : 1;
    w.ensure(n, dev_hist);
    const RedBuf red = w.red();
    const int g = grid_for(n, kBlock);
    const S* v = reinterpret_cast<const S*>(A->val.get());
    S *x = d_x, *r = w.r.get(), *rt = w.z.get(), *p = w.p.get(), *q = w.Ap.get(), *qt = w.qt.get(),
      *t = w.t.get();
    if (info) std::memset(info, 0, sizeof(*info));
    g_cocr_launches = 2;
    // sol = 0 ; r = rhs projected ; ||rhs|| (:274-299)
    SSV_CUDA(cudaMemsetAsync(x, 0, sizeof(S) * n, s));
    launch_k(k_gather_perm<S>, g, kBlock, s, n, nullptr, d_b, r, fd, 1);
    launch_k(k_norm2<S>, g, kBlock, s, n, r, red, w.scal.get());
    SSV_LAUNCH_CHECK();
    double2 nb;
    SSV_CUDA(cudaMemcpyAsync(&nb, w.scal.get(), sizeof(nb), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    const double rhs_norm = std::sqrt(std::fabs(nb.x));
    if (rhs_norm < 1e-30) {
        *iterations = 0;
        if (info) info->converged = 1;
        return;
    }
    KState* dst = w.st.get();
    std::string key = "ngs;" + std::to_string(n) + ";" + std::to_string((size_t)pre) + ";" +
                      std::to_string((size_t)fd) + ";" + std::to_string((size_t)x) + ";" +
                      std::to_string((size_t)dst) + ";" + std::to_string(A->lanes) + ";" +
                      std::to_string((size_t)red.partials);
    const double* sv = krylov_sell(A, s);  // before any capture
    key += ";" + pre_key(pre) + ";sell:" + std::to_string((size_t)sv);
    // the iteration graph; captured after the first preconditioner application, which
    // allocates and tunes on first use
    auto build = [&] {
        build_graph_loop(ctx.loop, key, [&](cudaGraphConditionalHandle hc, int use_cond) {
            apply_pre<S>(pre, q, qt, dst, n, s);
            launch_k(k_ngs_dot<S>, g, kBlock, s, n, qt, q, dst, NGS_MU, red);
            launch_k(k_ngs_update<S>, g, kBlock, s, n, x, p, q, qt, r, rt, dst, red);
            if (sv) {
                const int gs = std::max(1, std::min((A->sell.slices + kBlock / 32 - 1) / (kBlock / 32), sm_count() * 8));
                launch_k(k_ngs_sell_dot<S, 4>, gs, kBlock, s, A->sell.slices, A->sell.off.get(), A->sell.rows.get(),
                         A->sell.ci.get(), reinterpret_cast<const S*>(sv), rt, t, fd, dst, red);
            } else {
                const int L = A->lanes & 0xff;
                const int rpb = kBlock / L;
                int gg = std::max(1, std::min((n + rpb - 1) / rpb, sm_count() * 8));
                switch (L) {
                    case 2: launch_k(k_ngs_spmv_dot<S, 2>, gg, kBlock, s, n, A->rp.get(), A->ci.get(), v, rt, t, fd, dst, red); break;
                    case 4: launch_k(k_ngs_spmv_dot<S, 4>, gg, kBlock, s, n, A->rp.get(), A->ci.get(), v, rt, t, fd, dst, red); break;
                    case 8: launch_k(k_ngs_spmv_dot<S, 8>, gg, kBlock, s, n, A->rp.get(), A->ci.get(), v, rt, t, fd, dst, red); break;
                    case 16: launch_k(k_ngs_spmv_dot<S, 16>, gg, kBlock, s, n, A->rp.get(), A->ci.get(), v, rt, t, fd, dst, red); break;
                    default: launch_k(k_ngs_spmv_dot<S, 32>, gg, kBlock, s, n, A->rp.get(), A->ci.get(), v, rt, t, fd, dst, red);
                }
            }
            launch_k(k_cocr_pq<S>, g, kBlock, s, n, rt, t, p, q, dst);
            k_ngs_loop_ctl<<<1, 32, 0, s>>>(dst, hc, use_cond);
            SSV_LAUNCH_CHECK();
        });
    };
    std::vector<double> hs;  // printrates: the residual history over every cycle
    int used = 0, cycles = 0;
    double rs = rhs_norm;  // norm of the residual the cycle starts from
    double true_rel = 1.0;
    bool conv = false;
    KState h;
    while (true) {
        // rt = M^{-1} r ; p = rt ; q = A p projected ; rho = rt^T q
        apply_pre<S>(pre, r, rt, nullptr, n, s);
        launch_k(k_copy<S>, g, kBlock, s, n, rt, p);
        launch_spmv<S, S, 0>(A->lanes, n, A->rp.get(), A->ci.get(), v, p, q, nullptr, fd, nullptr, RED_STORE, red,
                             nullptr, s);
        SSV_LAUNCH_CHECK();
        const int left = maxiter - used;
        std::memset(&h, 0, sizeof(h));
        h.normalizer = rhs_norm;
        h.tol = tol;
        h.maxiter = left;
        h.save_hist = printrates ? 1 : 0;
        h.hist_cap = dev_hist;
        h.hist = w.hist.get();
        h.max_loops = loop_guard(left);
        h.brk_thr = 1e-30 * (rs / rhs_norm) * (rs / rhs_norm);
        h.restart_abs = refine ? refine->drop * rs : 0.0;
        if (left <= 0) { h.done = 1; h.iters = 0; }
        // state first, then rho = rt^T q into it
        SSV_CUDA(cudaMemcpyAsync(dst, &h, sizeof(h), cudaMemcpyHostToDevice, s));
        launch_k(k_dot<S>, g, kBlock, s, n, rt, q, 0, nullptr, RED_STORE, red, &dst->rho);
        SSV_LAUNCH_CHECK();
        if (cycles == 0) build();
        if (left > 0) run_graph_loop(ctx.loop, dst, left);
        SSV_CUDA(cudaMemcpyAsync(&h, dst, sizeof(h), cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
        if (h.status == SSV_ERR_TIMEOUT) fail(SSV_ERR_TIMEOUT, "COCR loop guard fired");
        ++cycles;
        g_cocr_launches += 4 + (pre ? 0 : 1) + (int64_t)ctx.loop.body_nodes * h.loops;
        if (printrates && h.hist_len > 0) {
            const size_t k0 = hs.size();
            hs.resize(k0 + std::min(h.hist_len, dev_hist));
            SSV_CUDA(cudaMemcpy(hs.data() + k0, w.hist.get(), sizeof(double) * (hs.size() - k0),
                                cudaMemcpyDeviceToHost));
        }
        if (!refine) {
            *iterations = h.iters;
            break;
        }
        used += h.updates;
        // FP64 true residual of the current x: r = P(b - A x) (t, free between cycles, holds P b)
        launch_k(k_gather_perm<S>, g, kBlock, s, n, nullptr, d_b, t, fd, 1);
        launch_spmv<S, S, 2>(A->lanes, n, A->rp.get(), A->ci.get(), v, x, r, t, fd, nullptr, RED_STORE, red,
                             nullptr, s);
        launch_k(k_norm2<S>, g, kBlock, s, n, r, red, w.scal.get());
        SSV_LAUNCH_CHECK();
        g_cocr_launches += 3;
        double2 nr;
        SSV_CUDA(cudaMemcpyAsync(&nr, w.scal.get(), sizeof(nr), cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
        rs = std::sqrt(std::fabs(nr.x));
        true_rel = rs / rhs_norm;
        if (printrates) {
            std::printf("COCR cycle %d: %d iterations, true residual = %g\n", cycles, h.updates, true_rel);
            std::fflush(stdout);
        }
        if (true_rel <= tol) { conv = true; break; }
        // out of iterations, or a cycle that could not take a single step
        if (used >= maxiter || h.updates == 0 || rs < 1e-300) break;
    }
    if (refine) {
        *iterations = used;
        if (info) {
            info->iterations = used;
            info->cycles = cycles;
            info->converged = conv ? 1 : 0;
            info->true_residual = true_rel;
        }
    }
    if (printrates) {
        std::printf("COCR iter 0: res = 1\n");
        for (size_t k = 0; k < hs.size(); ++k) std::printf("COCR iter %zu: res = %g\n", k + 1, hs[k]);
        std::fflush(stdout);
    }
}

// CG with an external preconditioner and an initial guess: the
// sparsesolv::CGSolver recurrence (solvers/cg_solver.hpp:64-146 with
// iterative_solver.hpp's bookkeeping) on the FreeDofs view of A (identity
// rows, zero columns; ngsolve/sparsesolv_precond.hpp:60-74), z = M^{-1} r by
// the given preconditioner, x on entry the initial guess (free entries) and on
// return the solution (free entries written). This is the Krylov driver of the
// AMS configurations, where the reference's scripts use NGSolve's CGSolver.
template <typename S>
static void run_pcg(ssv_matrix* A, ssv_precond* pre, const uint8_t* fd, const ssv_config& cfg, const S* d_b,
                    S* d_x, ssv_result* res, double* hist, int hist_cap) {
    cudaStream_t s = stream();
    const int n = A->rows;
    const double t0 = wall_seconds();
    auto& ctx_ptr = cocr_table()[A];
    if (!ctx_ptr) ctx_ptr.reset(new CocrCtx());
    CocrCtx& ctx = *ctx_ptr;
    KrylovWork<S>& w = cw_of<S>(ctx);
    const int dev_hist = cfg.save_residual_history ? std::max(cfg.max_iterations, 0) + 2 : 1;
    w.ensure(n, dev_hist);
    const RedBuf red = w.red();
    const int g = grid_for(n, kBlock);
    int64_t nk = 0;
    const S* v = reinterpret_cast<const S*>(A->val.get());
    if (fd) {
        ctx.vals_bc.alloc(A->val.size());
        k_bc_values<S><<<g, kBlock, 0, s>>>(n, A->rp.get(), A->ci.get(), v, fd, reinterpret_cast<S*>(ctx.vals_bc.get()));
        v = reinterpret_cast<const S*>(ctx.vals_bc.get());
        ++nk;
    }
    launch_k(k_gather_perm<S>, g, kBlock, s, n, nullptr, d_b, w.bw.get(), fd, 1);
    launch_k(k_gather_perm<S>, g, kBlock, s, n, nullptr, d_x, w.xb[0].get(), fd, 1);
    launch_spmv<S, S, 2>(A->lanes, n, A->rp.get(), A->ci.get(), v, w.xb[0].get(), w.r.get(), w.bw.get(), nullptr,
                         nullptr, RED_STORE, red, nullptr, s);
    launch_k(k_norm2<S>, g, kBlock, s, n, w.bw.get(), red, w.scal.get());
    launch_k(k_norm2<S>, g, kBlock, s, n, w.r.get(), red, w.scal.get() + 1);
    SSV_LAUNCH_CHECK();
    nk += 5;
    double2 nrm[2];
    SSV_CUDA(cudaMemcpyAsync(nrm, w.scal.get(), sizeof(nrm), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    const double norm_b = std::sqrt(nrm[0].x), r0 = std::sqrt(nrm[1].x);
    double normalizer = cfg.norm_type == SSV_NORM_RHS ? norm_b
                      : cfg.norm_type == SSV_NORM_INITIAL_RESIDUAL ? r0 : cfg.custom_norm;
    if (normalizer < 1e-15) normalizer = 1.0;
    KState h;
    std::memset(&h, 0, sizeof(h));
    h.cur = 0;
    h.best = -1;
    h.normalizer = normalizer;
    h.best_residual = DBL_MAX;
    h.norm_r = r0;
    h.final_norm = r0;
    h.tol = cfg.tolerance;
    h.abs_tol = cfg.abs_tolerance;
    h.div_threshold = cfg.divergence_threshold;
    h.maxiter = cfg.max_iterations;
    h.div_check = cfg.divergence_check;
    h.div_count = cfg.divergence_count;
    h.save_best = cfg.save_best_result;
    h.save_hist = cfg.save_residual_history;
    h.conj = cfg.conjugate;
    h.hist_cap = dev_hist;
    h.hist = w.hist.get();
    h.max_loops = loop_guard(cfg.max_iterations);
    if (cfg.save_residual_history) {
        const double h0 = r0 / normalizer;
        SSV_CUDA(cudaMemcpyAsync(w.hist.get(), &h0, sizeof(double), cudaMemcpyHostToDevice, s));
        h.hist_len = 1;
    }
    if (cfg.max_iterations <= 0) { h.done = 1; h.iters = std::max(cfg.max_iterations, 0); }
    KState* dst = w.st.get();
    SSV_CUDA(cudaMemcpyAsync(dst, &h, sizeof(h), cudaMemcpyHostToDevice, s));
    S* z = pre ? w.z.get() : w.r.get();
    if (pre) apply_pre<S>(pre, w.r.get(), w.z.get(), nullptr, n, s);
    launch_k(k_dot<S>, g, kBlock, s, n, w.r.get(), z, cfg.conjugate, nullptr, RED_STORE, red, &dst->rho);
    launch_k(k_copy<S>, g, kBlock, s, n, z, w.p.get());
    SSV_LAUNCH_CHECK();
    const std::string key = "pcg;" + std::to_string(n) + ";" + std::to_string((size_t)v) + ";" +
                            std::to_string((size_t)dst) + ";" + std::to_string((size_t)red.partials) + ";" +
                            std::to_string((size_t)w.r.get()) + ";" + pre_key(pre);
    build_graph_loop(ctx.pcg_loop, key, [&](cudaGraphConditionalHandle hc, int use_cond) {
        launch_spmv<S, S, 1>(A->lanes, n, A->rp.get(), A->ci.get(), v, w.p.get(), w.Ap.get(), nullptr, nullptr,
                             dst, RED_CG_ALPHA, red, nullptr, s);
        launch_k(k_cg_update<S>, g, kBlock, s, n, w.xb[0].get(), w.xb[1].get(), w.xb[2].get(), w.p.get(), w.Ap.get(),
                                           w.r.get(), dst, red);
        if (pre) apply_pre<S>(pre, w.r.get(), w.z.get(), dst, n, s);
        launch_k(k_dot<S>, g, kBlock, s, n, w.r.get(), z, cfg.conjugate, dst, RED_CG_BETA, red, nullptr);
        launch_k(k_pupdate<S>, g, kBlock, s, n, z, w.p.get(), dst);
        k_loop_ctl<<<1, 32, 0, s>>>(dst, hc, use_cond);
        SSV_LAUNCH_CHECK();
    });
    SSV_CUDA(cudaStreamSynchronize(s));
    const double t1 = wall_seconds();
    if (cfg.max_iterations > 0) run_graph_loop(ctx.pcg_loop, dst, cfg.max_iterations);
    SSV_CUDA(cudaMemcpyAsync(&h, dst, sizeof(h), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    if (h.status == SSV_ERR_TIMEOUT) fail(SSV_ERR_TIMEOUT, "CG loop guard fired");
    std::memset(res, 0, sizeof(*res));
    res->converged = h.converged;
    res->iterations = h.iters;
    res->final_residual = h.final_norm / h.normalizer;
    int xbuf = h.cur;
    if (!h.converged && cfg.save_best_result) {
        res->final_residual = h.best_residual;
        xbuf = h.best;
    }
    const S* xsrc;
    if (xbuf < 0) { w.t.zero(s); xsrc = w.t.get(); }
    else xsrc = w.xb[xbuf].get();
    launch_k(k_gather_perm<S>, g, kBlock, s, n, nullptr, xsrc, d_x, fd, 0);
    SSV_LAUNCH_CHECK();
    res->kernel_launches = nk + 3 + (int64_t)ctx.pcg_loop.body_nodes * h.loops;
    res->history_total = cfg.save_residual_history ? h.hist_len : 0;
    res->history_len = std::min(std::min(res->history_total, dev_hist), std::max(hist_cap, 0));
    if (hist && res->history_len > 0)
        SSV_CUDA(cudaMemcpyAsync(hist, w.hist.get(), sizeof(double) * res->history_len, cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    res->setup_seconds = t1 - t0;
    res->solve_seconds = wall_seconds() - t1;
}

void pcg_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* d_fd, const ssv_config& cfg, const void* d_b,
                   void* d_x, ssv_result* res, double* hist, int hist_cap) {
    if (A->rows != A->cols) fail(SSV_ERR_INVALID_ARG, "CG: matrix must be square");
    if (pre && !pre->ready) fail(SSV_ERR_RUNTIME, "CG: preconditioner is not set up (call Update())");
    if (pre && pre->vdtype != A->dtype) fail(SSV_ERR_TYPE, "CG: preconditioner scalar type differs from the matrix");
    if (pre && pre->n != A->rows) fail(SSV_ERR_INVALID_ARG, "CG: preconditioner size differs from the matrix");
    if (A->dtype == SSV_F64)
        run_pcg<double>(A, pre, d_fd, cfg, static_cast<const double*>(d_b), static_cast<double*>(d_x), res, hist,
                        hist_cap);
    else
        run_pcg<zdouble>(A, pre, d_fd, cfg, static_cast<const zdouble*>(d_b), static_cast<zdouble*>(d_x), res,
                         hist, hist_cap);
}

static void cocr_any(ssv_matrix* A, ssv_precond* pre, const uint8_t* d_fd, int maxiter, double tol,
                     int printrates, const void* d_b, void* d_x, int* iterations, const RefineOpt* ro,
                     ssv_refine_info* info) {
    if (pre && !pre->ready) fail(SSV_ERR_RUNTIME, "COCRSolver: preconditioner is not set up (call Update())");
    if (pre && pre->vdtype != A->dtype)
        fail(SSV_ERR_TYPE, "COCRSolver: preconditioner scalar type differs from the matrix");
    if (pre && pre->n != A->rows) fail(SSV_ERR_INVALID_ARG, "COCRSolver: preconditioner size differs from the matrix");
    if (A->rows != A->cols) fail(SSV_ERR_INVALID_ARG, "COCRSolver: matrix must be square");
    if (A->dtype == SSV_F64)
        run_cocr_ngs<double>(A, pre, d_fd, maxiter, tol, printrates, static_cast<const double*>(d_b),
                             static_cast<double*>(d_x), iterations, ro, info);
    else
        run_cocr_ngs<zdouble>(A, pre, d_fd, maxiter, tol, printrates, static_cast<const zdouble*>(d_b),
                              static_cast<zdouble*>(d_x), iterations, ro, info);
}

void cocr_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* d_fd, int maxiter, double tol,
                    int printrates, const void* d_b, void* d_x, int* iterations) {
    cocr_any(A, pre, d_fd, maxiter, tol, printrates, d_b, d_x, iterations, nullptr, nullptr);
}

void cocr_refined_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* d_fd, int maxiter, double tol,
                            double restart_drop, int printrates, const void* d_b, void* d_x,
                            ssv_refine_info* info) {
    if (!(restart_drop > 0.0 && restart_drop < 1.0))
        fail(SSV_ERR_INVALID_ARG, "refined COCR: restart_drop must lie in (0, 1)");
    RefineOpt ro{restart_drop};
    int its = 0;
    cocr_any(A, pre, d_fd, maxiter, tol, printrates, d_b, d_x, &its, &ro, info);
}

}  // namespace ssv
