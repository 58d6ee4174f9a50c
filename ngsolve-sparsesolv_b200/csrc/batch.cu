// batch.cu -- batched COCR over a frequency family (new: no reference
// counterpart; the single-system recurrence it runs per column is
// COCRSolverNGS::Mult, ngsolve/sparsesolv_solvers.hpp:273-369).
//
// The family is A_f = K + j omega_f M (K, M real, one sparsity pattern) for F
// frequencies, with R right-hand sides per frequency: C = F * R independent
// COCR recurrences advanced in lock-step. Vectors are stored [f][row][r]
// (complex), so one row of a frequency is R consecutive complex values and
// the per-frequency preconditioner sees the [row][rhs] block layout of the
// AMS block cycle. One SpMM pass reads K and M once for a tile of FB
// frequencies and forms every column's product; the tile (FB), the lanes per
// row and the grid are chosen by an autotuner that times the candidates on
// the actual matrix when the batch is created. The whole iteration (R-column
// AMS cycles of every frequency, the reductions with their per-column scalar
// steps, the vector updates) is one CUDA graph looped by a device-side WHILE
// node, as the single-system solvers are.
//
// Per-column semantics follow the single solve: alpha = rho / mu, beta =
// rho_new / rho with the 1e-30 breakdown tests, convergence when
// ||r|| / ||b|| <= tol (Hermitian norm), iterations = j + 1 on convergence and
// maxiter otherwise. A finished column is frozen (no further updates) while
// the others continue.
//
// Refined form (restart_drop > 0; the single-system ssv_cocr_refined_solve per
// column): every column runs cycles of that recurrence, each started from its
// FP64 true residual and ended once its residual has dropped by restart_drop
// (or on tol, a breakdown, maxiter); a column is finished when its true
// residual is <= tol. The graph loop runs one cycle of every live column; the
// host then computes the true residuals of all columns (one SpMM pass) and
// restarts the columns that need another cycle.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "objects.cuh"
#include "solver_api.hpp"

namespace ssv {

struct BCol {
    double2 alpha, beta, rho;
    double normalizer, res;
    double brk_thr;      // |mu|, |rho| breakdown threshold (1e-30, scaled in refined cycles)
    double restart_abs;  // refined form: ||r|| that ends this column's cycle (0 = never)
    double tres;         // refined form: ||P(b - A x)|| after the last cycle
    int done, converged, iters;
    int work;            // x updates performed (all cycles)
};

struct BState {
    KState ks;  // ks.done: every column finished (set only by the loop control)
    int ncols, ndone;
    double drop;  // refined form's restart_drop (0 = the reference's recurrence only)
    int refined, pad_;
};

enum BtOp : int { BT_TIME = 0, BT_RHO_INIT, BT_RHO, BT_MU, BT_NORM0, BT_UPDATE, BT_TRUE };

__device__ inline void bcol_done(BState* bs, BCol& c, int conv, int iters) {
    c.done = 1;
    c.converged = conv;
    c.iters = iters;
    atomicAdd(&bs->ndone, 1);
}

__device__ inline void bt_finish(BState* bs, BCol* cols, int c, double2 total, int op) {
    if (op == BT_TIME) return;
    BCol& col = cols[c];
    if (op == BT_TRUE) {  // between refined cycles (every column is stopped then)
        col.tres = std::sqrt(std::fabs(total.x));
        return;
    }
    if (col.done) return;
    if (op == BT_RHO_INIT) {
        col.rho = total;
    } else if (op == BT_RHO) {  // :354-359
        const zdouble rho{col.rho.x, col.rho.y};
        if (ST<zdouble>::abs(rho) < col.brk_thr) { bcol_done(bs, col, 0, bs->ks.it); return; }
        const zdouble b = zdiv(zdouble{total.x, total.y}, rho);
        col.beta = make_double2(b.x, b.y);
        col.rho = total;
    } else if (op == BT_MU) {  // :323-327
        const zdouble mu{total.x, total.y};
        if (ST<zdouble>::abs(mu) < col.brk_thr) { bcol_done(bs, col, 0, bs->ks.it); return; }
        const zdouble a = zdiv(zdouble{col.rho.x, col.rho.y}, mu);
        col.alpha = make_double2(a.x, a.y);
    } else if (op == BT_NORM0) {  // :298-301
        col.normalizer = std::sqrt(std::fabs(total.x));
        col.brk_thr = 1e-30;
        col.restart_abs = bs->drop * col.normalizer;
        if (col.normalizer < 1e-30) bcol_done(bs, col, 0, 0);
    } else {  // BT_UPDATE, :338-347
        col.res = std::sqrt(std::fabs(total.x));
        col.work++;
        if (col.res / col.normalizer <= bs->ks.tol) bcol_done(bs, col, 1, bs->ks.it + 1);
        else if (col.res <= col.restart_abs) bcol_done(bs, col, 0, bs->ks.it + 1);
        else if (bs->refined && col.work >= bs->ks.maxiter) bcol_done(bs, col, 0, bs->ks.it + 1);
    }
}

// Sum M complex values over the blocks of this blockIdx.y group. Fixed order
// at every stage (deterministic). True in the last block, totals in tot[].
template <int M>
__device__ bool grid_reduce_cols(double2 (&v)[M], double2* __restrict__ partials, unsigned* ticket,
                                 double2* tot) {
    __shared__ double2 sh[(kBlock / 32) * M];
    __shared__ bool am_last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < M; ++m) v[m] = warp_sum2(v[m]);
    if (lane == 0)
#pragma unroll
        for (int m = 0; m < M; ++m) sh[w * M + m] = v[m];
    __syncthreads();
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        double2 s = make_double2(0.0, 0.0);
        for (int q = 0; q < kBlock / 32; ++q) s = add2(s, sh[q * M + m]);
        partials[(size_t)blockIdx.x * M + m] = s;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) am_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    for (int m = w; m < M; m += kBlock / 32) {  // warp per value, lanes stride the blocks
        double2 s = make_double2(0.0, 0.0);
        for (int b = lane; b < (int)gridDim.x; b += 32) s = add2(s, __ldcg(&partials[(size_t)b * M + m]));
        s = warp_sum2(s);
        if (lane == 0) tot[m] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// y_f = (K + j omega_f M) x_f for the FB frequencies of this blockIdx.y, rows
// of constrained DOFs zeroed, and the per-column x^T y (unconjugated).
template <int R, int FB, int LANES>
__global__ void __launch_bounds__(kBlock)
k_bt_spmm(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ kv,
          const double* __restrict__ mv, const double* __restrict__ omega, const zdouble* __restrict__ x,
          zdouble* __restrict__ y, const uint8_t* __restrict__ mask, BState* bs, BCol* cols,
          double2* partials, unsigned* tickets, int gx_cap, int op) {
    constexpr int Q = FB * R;
    __shared__ int s_skip;
    __shared__ double2 tot[Q];
    if (threadIdx.x == 0) s_skip = bs->ks.done;
    __syncthreads();
    if (s_skip) return;
    const int f0 = blockIdx.y * FB;
    double om[FB];
#pragma unroll
    for (int j = 0; j < FB; ++j) om[j] = omega[f0 + j];
    const int sub = threadIdx.x % LANES;
    const int rpb = kBlock / LANES;
    const int lane_row = (threadIdx.x & 31) / LANES;  // warp-uniform trip count
    double2 part[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) part[q] = make_double2(0.0, 0.0);
    for (int row = blockIdx.x * rpb + threadIdx.x / LANES; row - lane_row < n; row += gridDim.x * rpb) {
        const bool valid = row < n;
        double ar[Q], ai[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) ar[q] = ai[q] = 0.0;
        if (valid) {
            const int k1 = rp[row + 1];
            for (int k = rp[row] + sub; k < k1; k += LANES) {
                const double a = kv[k], m = mv[k];
                const size_t c = (size_t)ci[k];
#pragma unroll
                for (int j = 0; j < FB; ++j) {
                    const double im = om[j] * m;
                    const zdouble* xr = x + ((size_t)(f0 + j) * n + c) * R;
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const zdouble xv = xr[r];
                        ar[j * R + r] += a * xv.x - im * xv.y;
                        ai[j * R + r] += a * xv.y + im * xv.x;
                    }
                }
            }
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                ar[q] += __shfl_down_sync(0xffffffffu, ar[q], o, LANES);
                ai[q] += __shfl_down_sync(0xffffffffu, ai[q], o, LANES);
            }
        if (valid && sub == 0) {
            const bool keep = !mask || mask[row];
#pragma unroll
            for (int j = 0; j < FB; ++j)
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int q = j * R + r;
                    const size_t idx = ((size_t)(f0 + j) * n + row) * R + r;
                    const zdouble t = keep ? zdouble{ar[q], ai[q]} : zdouble{0.0, 0.0};
                    y[idx] = t;
                    if (op != BT_TIME) {
                        const zdouble xi = x[idx];
                        part[q].x += xi.x * t.x - xi.y * t.y;
                        part[q].y += xi.x * t.y + xi.y * t.x;
                    }
                }
        }
    }
    if (grid_reduce_cols<Q>(part, partials + (size_t)blockIdx.y * gx_cap * Q, tickets + blockIdx.y, tot))
        for (int q = threadIdx.x; q < Q; q += blockDim.x) bt_finish(bs, cols, f0 * R + q, tot[q], op);
}

// Per-column a^T b (unconjugated), or ||a||^2 when NORM; frequency = blockIdx.y.
template <int R, bool NORM>
__global__ void __launch_bounds__(kBlock)
k_bt_dot(int n, const zdouble* __restrict__ a, const zdouble* __restrict__ b, BState* bs, BCol* cols,
         double2* partials, unsigned* tickets, int gx_cap, int op) {
    __shared__ int s_skip;
    __shared__ double2 tot[R];
    if (threadIdx.x == 0) s_skip = bs->ks.done;
    __syncthreads();
    if (s_skip) return;
    const int f = blockIdx.y;
    const size_t base = (size_t)f * n * R;
    double2 part[R];
#pragma unroll
    for (int r = 0; r < R; ++r) part[r] = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const size_t idx = base + (size_t)i * R + r;
            const zdouble u = a[idx];
            if constexpr (NORM) {
                part[r].x += u.x * u.x + u.y * u.y;
            } else {
                const zdouble v = b[idx];
                part[r].x += u.x * v.x - u.y * v.y;
                part[r].y += u.x * v.y + u.y * v.x;
            }
        }
    }
    if (grid_reduce_cols<R>(part, partials + (size_t)f * gx_cap * R, tickets + f, tot))
        for (int q = threadIdx.x; q < R; q += blockDim.x) bt_finish(bs, cols, f * R + q, tot[q], op);
}

// r = P(b - t) with t = A x, and ||r||^2 per column (refined form, between
// cycles; every column is stopped, so no skip test)
template <int R>
__global__ void __launch_bounds__(kBlock)
k_bt_resid(int n, const zdouble* __restrict__ b, const zdouble* __restrict__ t, zdouble* __restrict__ r,
           const uint8_t* __restrict__ mask, BState* bs, BCol* cols, double2* partials, unsigned* tickets,
           int gx_cap) {
    __shared__ double2 tot[R];
    const int f = blockIdx.y;
    const size_t base = (size_t)f * n * R;
    double2 part[R];
#pragma unroll
    for (int c = 0; c < R; ++c) part[c] = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool keep = !mask || mask[i];
#pragma unroll
        for (int c = 0; c < R; ++c) {
            const size_t idx = base + (size_t)i * R + c;
            const zdouble v = keep ? b[idx] - t[idx] : zdouble{0.0, 0.0};
            r[idx] = v;
            part[c].x += ST<zdouble>::norm2(v);
        }
    }
    if (grid_reduce_cols<R>(part, partials + (size_t)f * gx_cap * R, tickets + f, tot))
        for (int c = threadIdx.x; c < R; c += blockDim.x) bt_finish(bs, cols, f * R + c, tot[c], BT_TRUE);
}

// sol += alpha p ; r -= alpha q ; rt -= alpha qt (unless the step replaces
// rt by M^{-1} r afterwards) ; ||r||^2 per live column
template <int R, bool UPD_RT>
__global__ void __launch_bounds__(kBlock)
k_bt_update(int n, zdouble* __restrict__ x, const zdouble* __restrict__ p, const zdouble* __restrict__ q,
            const zdouble* __restrict__ qt, zdouble* __restrict__ r, zdouble* __restrict__ rt, BState* bs,
            BCol* cols, double2* partials, unsigned* tickets, int gx_cap) {
    __shared__ int s_skip;
    __shared__ int s_live[R];
    __shared__ zdouble s_alpha[R];
    __shared__ double2 tot[R];
    const int f = blockIdx.y;
    if (threadIdx.x == 0) s_skip = bs->ks.done;
    if (threadIdx.x < R) {
        const BCol& c = cols[f * R + threadIdx.x];
        s_live[threadIdx.x] = !c.done;
        s_alpha[threadIdx.x] = zdouble{c.alpha.x, c.alpha.y};
    }
    __syncthreads();
    if (s_skip) return;
    const size_t base = (size_t)f * n * R;
    double2 part[R];
#pragma unroll
    for (int c = 0; c < R; ++c) part[c] = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < R; ++c) {
            if (!s_live[c]) continue;
            const size_t idx = base + (size_t)i * R + c;
            const zdouble al = s_alpha[c];
            x[idx] = ST<zdouble>::fma(al, p[idx], x[idx]);
            const zdouble ri = r[idx] - al * q[idx];
            r[idx] = ri;
            if constexpr (UPD_RT) rt[idx] = rt[idx] - al * qt[idx];
            part[c].x += ST<zdouble>::norm2(ri);
        }
    }
    if (grid_reduce_cols<R>(part, partials + (size_t)f * gx_cap * R, tickets + f, tot))
        for (int c = threadIdx.x; c < R; c += blockDim.x) bt_finish(bs, cols, f * R + c, tot[c], BT_UPDATE);
}

// p = rt + beta p ; q = t + beta q per live column
template <int R>
__global__ void __launch_bounds__(kBlock)
k_bt_pq(int n, const zdouble* __restrict__ rt, const zdouble* __restrict__ t, zdouble* __restrict__ p,
        zdouble* __restrict__ q, const BState* bs, const BCol* cols) {
    __shared__ int s_skip;
    __shared__ int s_live[R];
    __shared__ zdouble s_beta[R];
    const int f = blockIdx.y;
    if (threadIdx.x == 0) s_skip = bs->ks.done;
    if (threadIdx.x < R) {
        const BCol& c = cols[f * R + threadIdx.x];
        s_live[threadIdx.x] = !c.done;
        s_beta[threadIdx.x] = zdouble{c.beta.x, c.beta.y};
    }
    __syncthreads();
    if (s_skip) return;
    const size_t base = (size_t)f * n * R;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < R; ++c) {
            if (!s_live[c]) continue;
            const size_t idx = base + (size_t)i * R + c;
            const zdouble be = s_beta[c];
            p[idx] = ST<zdouble>::fma(be, p[idx], rt[idx]);
            q[idx] = ST<zdouble>::fma(be, q[idx], t[idx]);
        }
    }
}

__global__ void k_bt_loop_ctl(BState* bs, BCol* cols, cudaGraphConditionalHandle h, int use_cond) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    KState& ks = bs->ks;
    if (!ks.done) {
        ks.it++;
        if (ks.it >= ks.maxiter)  // :368
            for (int c = 0; c < bs->ncols; ++c)
                if (!cols[c].done) {
                    cols[c].done = 1;
                    cols[c].iters = ks.maxiter;
                    bs->ndone++;
                }
        if (bs->ndone >= bs->ncols) ks.done = 1;
    }
    ks.loops++;
    if (!ks.done && ks.loops >= ks.max_loops) { ks.done = 1; ks.status = SSV_ERR_TIMEOUT; }
    if (use_cond) cudaGraphSetConditional(h, ks.done ? 0u : 1u);
}

// user layout [f][r][row] <-> internal [f][row][r]; the gather masks
template <int R>
__global__ void k_bt_gather(int n, int F, const zdouble* __restrict__ user, zdouble* __restrict__ in,
                            const uint8_t* __restrict__ mask) {
    const int64_t total = (int64_t)F * n * R;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t f = q / ((int64_t)n * R);
        const int64_t rem = q - f * n * R;
        const int row = (int)(rem / R), r = (int)(rem % R);
        in[q] = (!mask || mask[row]) ? user[((size_t)f * R + r) * n + row] : zdouble{0.0, 0.0};
    }
}

template <int R>
__global__ void k_bt_scatter(int n, int F, const zdouble* __restrict__ in, zdouble* __restrict__ user) {
    const int64_t total = (int64_t)F * n * R;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t f = q / ((int64_t)n * R);
        const int64_t rem = q - f * n * R;
        const int row = (int)(rem / R), r = (int)(rem % R);
        user[((size_t)f * R + r) * n + row] = in[q];
    }
}

}  // namespace ssv

using ssv::BCol;
using ssv::BState;
using ssv::DevBuf;
using ssv::zdouble;

struct ssv_batch {
    int n = 0, F = 0, R = 0, C = 0;
    int64_t nnz = 0;
    std::vector<double> omegas;
    DevBuf<double> d_omega;
    DevBuf<int> rp, ci;
    DevBuf<double> kv, mv;
    std::vector<ssv_precond*> pre;
    bool has_fd = false;
    DevBuf<uint8_t> fd;
    DevBuf<zdouble> x, r, rt, p, q, qt, t, bw, io_b, io_x;
    DevBuf<BState> bs;
    DevBuf<BCol> cols;
    DevBuf<double2> partials;
    DevBuf<unsigned int> tickets;
    int gx_cap = 0, gx_elem = 0;
    // SpMM launch shape chosen by the autotuner
    int fb = 1, lanes = 8, gx = 1, chosen = -1;
    // residual replacement: every `replace_every`-th step sets rt = M^{-1} r
    // instead of the recurrence (0 = never; -1 = automatic: 10 when a
    // preconditioner is in the FP32 form, whose rounding makes M^{-1} not
    // exactly linear so the recurrence drifts from M^{-1} r)
    int replace_every = -1;
    // refined form (defect correction, true-residual restarts): restart_drop
    // > 0; 0 = the reference's recurrence alone
    double restart_drop = 0.0;
    std::vector<ssv_batch_tune_entry> table;
    ssv::GraphLoop loop;
    // frequencies' preconditioner cycles run as parallel branches; frequencies
    // sharing one preconditioner object share a branch (its work buffers)
    ssv::ForkSet forks;
    std::vector<int> branch_of;
    int branches = 0;
    // last solve
    double last_ms = 0.0, last_loop_ms = 0.0;
    int64_t last_launches = 0;
    int last_loops = 0, last_cycles = 0;
};

namespace ssv {

template <int R, int FB, int L>
static void spmm_launch(const ssv_batch& B, int gx, const zdouble* x, zdouble* y, int op, cudaStream_t s) {
    dim3 grid(gx, B.F / FB);
    k_bt_spmm<R, FB, L><<<grid, kBlock, 0, s>>>(B.n, B.rp.get(), B.ci.get(), B.kv.get(), B.mv.get(), B.d_omega.get(),
                                                x, y, B.has_fd ? B.fd.get() : nullptr, B.bs.get(), B.cols.get(),
                                                B.partials.get(), B.tickets.get(), B.gx_cap, op);
}

template <int R, int FB>
static bool spmm_l(const ssv_batch& B, int lanes, int gx, const zdouble* x, zdouble* y, int op, cudaStream_t s) {
    switch (lanes) {
        case 4: spmm_launch<R, FB, 4>(B, gx, x, y, op, s); return true;
        case 8: spmm_launch<R, FB, 8>(B, gx, x, y, op, s); return true;
        case 16: spmm_launch<R, FB, 16>(B, gx, x, y, op, s); return true;
    }
    return false;
}

// (R, FB) pairs built: FB * R <= 16 keeps the accumulators in registers.
static bool spmm_dispatch(const ssv_batch& B, int fb, int lanes, int gx, const zdouble* x, zdouble* y, int op,
                          cudaStream_t s) {
    if (B.R == 1) {
        switch (fb) {
            case 1: return spmm_l<1, 1>(B, lanes, gx, x, y, op, s);
            case 2: return spmm_l<1, 2>(B, lanes, gx, x, y, op, s);
            case 4: return spmm_l<1, 4>(B, lanes, gx, x, y, op, s);
            case 8: return spmm_l<1, 8>(B, lanes, gx, x, y, op, s);
        }
    } else if (B.R == 4) {
        switch (fb) {
            case 1: return spmm_l<4, 1>(B, lanes, gx, x, y, op, s);
            case 2: return spmm_l<4, 2>(B, lanes, gx, x, y, op, s);
            case 4: return spmm_l<4, 4>(B, lanes, gx, x, y, op, s);
        }
    }
    return false;
}

static void spmm(const ssv_batch& B, const zdouble* x, zdouble* y, int op, cudaStream_t s) {
    if (!spmm_dispatch(B, B.fb, B.lanes, B.gx, x, y, op, s)) fail(SSV_ERR_RUNTIME, "batch SpMM: no kernel for shape");
    SSV_LAUNCH_CHECK();
}

template <int R>
static void elem_kernels_dot(const ssv_batch& B, const zdouble* a, const zdouble* b, int op, bool norm,
                             cudaStream_t s) {
    dim3 grid(B.gx_elem, B.F);
    if (norm)
        k_bt_dot<R, true><<<grid, kBlock, 0, s>>>(B.n, a, b, B.bs.get(), B.cols.get(), B.partials.get(),
                                                  B.tickets.get(), B.gx_cap, op);
    else
        k_bt_dot<R, false><<<grid, kBlock, 0, s>>>(B.n, a, b, B.bs.get(), B.cols.get(), B.partials.get(),
                                                   B.tickets.get(), B.gx_cap, op);
}

static void bt_dot(const ssv_batch& B, const zdouble* a, const zdouble* b, int op, bool norm, cudaStream_t s) {
    if (B.R == 1) elem_kernels_dot<1>(B, a, b, op, norm, s);
    else elem_kernels_dot<4>(B, a, b, op, norm, s);
    SSV_LAUNCH_CHECK();
}

template <bool UPD_RT>
static void bt_update_t(ssv_batch& B, cudaStream_t s) {
    dim3 grid(B.gx_elem, B.F);
    if (B.R == 1)
        k_bt_update<1, UPD_RT><<<grid, kBlock, 0, s>>>(B.n, B.x.get(), B.p.get(), B.q.get(), B.qt.get(),
                                                       B.r.get(), B.rt.get(), B.bs.get(), B.cols.get(),
                                                       B.partials.get(), B.tickets.get(), B.gx_cap);
    else
        k_bt_update<4, UPD_RT><<<grid, kBlock, 0, s>>>(B.n, B.x.get(), B.p.get(), B.q.get(), B.qt.get(),
                                                       B.r.get(), B.rt.get(), B.bs.get(), B.cols.get(),
                                                       B.partials.get(), B.tickets.get(), B.gx_cap);
    SSV_LAUNCH_CHECK();
}

static void bt_update(ssv_batch& B, bool upd_rt, cudaStream_t s) {
    if (upd_rt) bt_update_t<true>(B, s);
    else bt_update_t<false>(B, s);
}

static void bt_pq(ssv_batch& B, cudaStream_t s) {
    dim3 grid(B.gx_elem, B.F);
    if (B.R == 1)
        k_bt_pq<1><<<grid, kBlock, 0, s>>>(B.n, B.rt.get(), B.t.get(), B.p.get(), B.q.get(), B.bs.get(), B.cols.get());
    else
        k_bt_pq<4><<<grid, kBlock, 0, s>>>(B.n, B.rt.get(), B.t.get(), B.p.get(), B.q.get(), B.bs.get(), B.cols.get());
    SSV_LAUNCH_CHECK();
}

// out_f = M_f^{-1} in_f for every frequency (identity without a preconditioner);
// the frequencies are independent and run as parallel branches
static void bt_precond(ssv_batch& B, const zdouble* in, zdouble* out, const KState* st, cudaStream_t s) {
    const size_t blk = (size_t)B.n * B.R;
    B.forks.fork(s, B.branches);
    for (int f = 0; f < B.F; ++f) {
        const zdouble* i = in + f * blk;
        zdouble* o = out + f * blk;
        cudaStream_t fs = B.forks.side[B.branch_of[f]];
        if (B.pre[f])
            ams_apply_block(B.pre[f]->ams.get(), reinterpret_cast<const double*>(i), reinterpret_cast<double*>(o),
                            B.R, st, fs);
        else
            SSV_CUDA(cudaMemcpyAsync(o, i, sizeof(zdouble) * blk, cudaMemcpyDeviceToDevice, fs));
    }
    B.forks.join(s, B.branches);
}

static int grid_x_for(const ssv_batch& B, int rows_per_block, int groups, int per_sm) {
    const int need = (B.n + rows_per_block - 1) / rows_per_block;
    const int want = std::max(1, per_sm * sm_count() / std::max(groups, 1));
    return std::max(1, std::min(std::min(need, want), B.gx_cap));
}

// Times every SpMM shape on the batch's own matrix and keeps the fastest.
static void autotune(ssv_batch& B) {
    cudaStream_t s = stream();
    BState h;
    std::memset(&h, 0, sizeof(h));
    h.ncols = B.C;
    SSV_CUDA(cudaMemcpyAsync(B.bs.get(), &h, sizeof(h), cudaMemcpyHostToDevice, s));
    B.p.zero(s);
    cudaEvent_t e0, e1;
    SSV_CUDA(cudaEventCreate(&e0));
    SSV_CUDA(cudaEventCreate(&e1));
    const int fbs[4] = {1, 2, 4, 8};
    const int lanes_c[3] = {4, 8, 16};
    const int occ[3] = {2, 4, 8};
    float best = 1e30f;
    B.table.clear();
    for (int fb : fbs) {
        if (B.F % fb) continue;
        if (fb * B.R > 16) continue;
        for (int L : lanes_c)
            for (int o : occ) {
                const int gx = grid_x_for(B, kBlock / L, B.F / fb, o);
                bool seen = false;  // small matrices cap several occupancies at one grid
                for (const auto& t : B.table) seen |= t.freq_tile == fb && t.lanes == L && t.grid_x == gx;
                if (seen) continue;
                for (int w = 0; w < 2; ++w) spmm_dispatch(B, fb, L, gx, B.p.get(), B.t.get(), BT_TIME, s);
                SSV_CUDA(cudaEventRecord(e0, s));
                const int reps = 5;
                for (int k = 0; k < reps; ++k) spmm_dispatch(B, fb, L, gx, B.p.get(), B.t.get(), BT_TIME, s);
                SSV_CUDA(cudaEventRecord(e1, s));
                SSV_CUDA(cudaEventSynchronize(e1));
                SSV_LAUNCH_CHECK();
                float ms = 0.f;
                SSV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                ms /= reps;
                ssv_batch_tune_entry te;
                te.freq_tile = fb;
                te.lanes = L;
                te.grid_x = gx;
                te.microseconds = 1e3 * ms;
                B.table.push_back(te);
                if (ms < best) {
                    best = ms;
                    B.chosen = (int)B.table.size() - 1;
                    B.fb = fb;
                    B.lanes = L;
                    B.gx = gx;
                }
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

static std::vector<double> host_values(const ssv_matrix* M) {
    std::vector<double> v(M->nnz);
    SSV_CUDA(cudaMemcpy(v.data(), M->val.get(), sizeof(double) * M->nnz, cudaMemcpyDeviceToHost));
    return v;
}

// Union pattern of K and M (columns sorted per row) with both value arrays.
static void union_pattern(const ssv_matrix* K, const ssv_matrix* M, std::vector<int>& rp, std::vector<int>& ci,
                          std::vector<double>& kv, std::vector<double>& mv) {
    const std::vector<double> hk = host_values(K), hm = host_values(M);
    const int n = K->rows;
    rp.assign(n + 1, 0);
    ci.clear();
    kv.clear();
    mv.clear();
    std::vector<std::pair<int, std::pair<double, double>>> row;
    for (int i = 0; i < n; ++i) {
        row.clear();
        for (int k = K->h_rp[i]; k < K->h_rp[i + 1]; ++k) row.push_back({K->h_ci[k], {hk[k], 0.0}});
        for (int k = M->h_rp[i]; k < M->h_rp[i + 1]; ++k) row.push_back({M->h_ci[k], {0.0, hm[k]}});
        std::stable_sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t k = 0; k < row.size();) {
            const int c = row[k].first;
            double a = 0.0, m = 0.0;
            for (; k < row.size() && row[k].first == c; ++k) {
                a += row[k].second.first;
                m += row[k].second.second;
            }
            ci.push_back(c);
            kv.push_back(a);
            mv.push_back(m);
        }
        rp[i + 1] = (int)ci.size();
    }
}

ssv_batch* batch_create(ssv_matrix* K, ssv_matrix* M, int F, const double* omegas, ssv_precond* const* pre, int R,
                        const uint8_t* fd) {
    if (!K || !M || !omegas || F <= 0) fail(SSV_ERR_INVALID_ARG, "batch: NULL matrix/omegas or no frequency");
    if (K->dtype != SSV_F64 || M->dtype != SSV_F64) fail(SSV_ERR_TYPE, "batch: K and M must be real");
    if (K->rows != K->cols || M->rows != K->rows || M->cols != K->cols)
        fail(SSV_ERR_INVALID_ARG, "batch: K and M must be square and of one size");
    if (R != 1 && R != 4) fail(SSV_ERR_INVALID_ARG, "batch: right-hand sides per frequency must be 1 or 4");
    auto* B = new ssv_batch();
    try {
        cudaStream_t s = stream();
        B->n = K->rows;
        B->F = F;
        B->R = R;
        B->C = F * R;
        B->omegas.assign(omegas, omegas + F);
        B->d_omega.upload(omegas, F, s);
        std::vector<int> rp, ci;
        std::vector<double> kv, mv;
        union_pattern(K, M, rp, ci, kv, mv);
        B->nnz = (int64_t)ci.size();
        B->rp.upload(rp.data(), rp.size(), s);
        B->ci.upload(ci.data(), ci.size(), s);
        B->kv.upload(kv.data(), kv.size(), s);
        B->mv.upload(mv.data(), mv.size(), s);
        if (fd) {
            std::vector<uint8_t> h(fd, fd + B->n);
            for (auto& v : h) v = v ? 1 : 0;
            B->fd.upload(h.data(), h.size(), s);
            B->has_fd = true;
        }
        B->pre.assign(F, nullptr);
        for (int f = 0; f < F; ++f) {
            ssv_precond* p = pre ? pre[f] : nullptr;
            if (p) {
                if (p->kind != 3 || !p->ams)
                    fail(SSV_ERR_TYPE, "batch: preconditioners must be ComplexCompactAMS (or NULL)");
                if (p->n != B->n) fail(SSV_ERR_INVALID_ARG, "batch: preconditioner size differs from the matrix");
                ams_reserve_block(p->ams.get(), R);
            }
            B->pre[f] = p;
        }
        B->branch_of.assign(F, 0);
        for (int f = 0; f < F; ++f) {
            int same = -1;
            for (int g = 0; g < f && same < 0; ++g)
                if (B->pre[f] && B->pre[g] == B->pre[f]) same = B->branch_of[g];
            B->branch_of[f] = same >= 0 ? same : B->branches++;
        }
        B->forks.ensure(B->branches);
        const size_t len = (size_t)F * B->n * R;
        for (DevBuf<zdouble>* v : {&B->x, &B->r, &B->rt, &B->p, &B->q, &B->qt, &B->t, &B->bw}) v->alloc(len);
        B->bs.alloc(1);
        B->cols.alloc(B->C);
        B->gx_cap = sm_count() * 8;
        B->gx_elem = std::max(1, std::min((B->n + kBlock - 1) / kBlock, std::max(1, 4 * sm_count() / F)));
        B->partials.alloc((size_t)F * B->gx_cap * R);
        B->tickets.alloc(F);
        B->tickets.zero(s);
        autotune(*B);
        SSV_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        delete B;
        throw;
    }
    return B;
}

void batch_destroy(ssv_batch* B) { delete B; }

static int replace_period(const ssv_batch& B) {
    if (B.restart_drop > 0.0) return 0;  // the refined cycles restart from the true residual instead
    if (B.replace_every >= 0) return B.replace_every;
    for (const ssv_precond* p : B.pre)
        if (p && ams_precision(p->ams.get()) != SSV_PREC_FP64) return 10;
    return 0;
}

static std::string batch_key(const ssv_batch& B) {
    std::string k = "batch;" + std::to_string((size_t)&B) + ";" + std::to_string(B.fb) + ";" +
                    std::to_string(B.lanes) + ";" + std::to_string(B.gx) + ";" + std::to_string(replace_period(B));
    for (const ssv_precond* p : B.pre)
        k += ";" + (p ? std::to_string((size_t)p) + ":" + std::to_string(precond_generation(p)) : std::string("-"));
    return k;
}

static void bt_resid(ssv_batch& B, cudaStream_t s) {
    dim3 grid(B.gx_elem, B.F);
    const uint8_t* fdp = B.has_fd ? B.fd.get() : nullptr;
    if (B.R == 1)
        k_bt_resid<1><<<grid, kBlock, 0, s>>>(B.n, B.bw.get(), B.t.get(), B.r.get(), fdp, B.bs.get(), B.cols.get(),
                                              B.partials.get(), B.tickets.get(), B.gx_cap);
    else
        k_bt_resid<4><<<grid, kBlock, 0, s>>>(B.n, B.bw.get(), B.t.get(), B.r.get(), fdp, B.bs.get(), B.cols.get(),
                                              B.partials.get(), B.tickets.get(), B.gx_cap);
    SSV_LAUNCH_CHECK();
}

void batch_cocr_solve_dev(ssv_batch* Bp, int maxiter, double tol, const void* d_b, void* d_x, int* iters,
                          int* conv, double* res) {
    ssv_batch& B = *Bp;
    for (const ssv_precond* p : B.pre)
        if (p && !p->ready) fail(SSV_ERR_RUNTIME, "batch: preconditioner is not set up (call Update())");
    cudaStream_t s = stream();
    KState* kst = &B.bs.get()->ks;
    const bool refined = B.restart_drop > 0.0;
    // the iteration graph first (capture only), so the events below time device work alone
    const int period = replace_period(B);
    build_graph_loop(B.loop, batch_key(B), [&](cudaGraphConditionalHandle hc, int use_cond) {
        const int steps = std::max(period, 1);  // the body holds one replacement period
        for (int u = 0; u < steps; ++u) {
            const bool replace = period > 0 && u == steps - 1;
            bt_precond(B, B.q.get(), B.qt.get(), kst, s);
            bt_dot(B, B.qt.get(), B.q.get(), BT_MU, false, s);
            bt_update(B, !replace, s);
            if (replace) bt_precond(B, B.r.get(), B.rt.get(), kst, s);
            spmm(B, B.rt.get(), B.t.get(), BT_RHO, s);
            bt_pq(B, s);
            k_bt_loop_ctl<<<1, 32, 0, s>>>(B.bs.get(), B.cols.get(), hc, use_cond);
            SSV_LAUNCH_CHECK();
        }
    });
    cudaEvent_t e0, e1, e2;
    SSV_CUDA(cudaEventCreate(&e0));
    SSV_CUDA(cudaEventCreate(&e1));
    SSV_CUDA(cudaEventCreate(&e2));
    SSV_CUDA(cudaEventRecord(e0, s));
    BState h;
    std::memset(&h, 0, sizeof(h));
    h.ncols = B.C;
    h.ks.tol = tol;
    h.ks.maxiter = maxiter;
    h.ks.max_loops = loop_guard(maxiter);
    h.drop = refined ? B.restart_drop : 0.0;
    h.refined = refined ? 1 : 0;
    if (maxiter <= 0) {
        h.ks.done = 1;
        h.ndone = B.C;
    }
    SSV_CUDA(cudaMemcpyAsync(B.bs.get(), &h, sizeof(h), cudaMemcpyHostToDevice, s));
    SSV_CUDA(cudaMemsetAsync(B.cols.get(), 0, sizeof(BCol) * B.C, s));
    const size_t len = (size_t)B.F * B.n * B.R;
    const int ge = grid_for((int64_t)len, kBlock);
    int64_t nk = 0;
    // x = 0 ; r = b projected ; ||b|| per column (:274-301)
    B.x.zero(s);
    const zdouble* ub = static_cast<const zdouble*>(d_b);
    const uint8_t* fdp = B.has_fd ? B.fd.get() : nullptr;
    if (B.R == 1) k_bt_gather<1><<<ge, kBlock, 0, s>>>(B.n, B.F, ub, B.r.get(), fdp);
    else k_bt_gather<4><<<ge, kBlock, 0, s>>>(B.n, B.F, ub, B.r.get(), fdp);
    SSV_LAUNCH_CHECK();
    if (refined) SSV_CUDA(cudaMemcpyAsync(B.bw.get(), B.r.get(), sizeof(zdouble) * len, cudaMemcpyDeviceToDevice, s));
    bt_dot(B, B.r.get(), B.r.get(), BT_NORM0, true, s);
    std::vector<BCol> hc(B.C);
    std::vector<char> fin(B.C, 0);
    std::vector<int> work_prev(B.C, 0);
    int cycles = 0, loops = 0;
    while (true) {
        // rt = M^{-1} r ; p = rt ; q = A p ; rho = rt^T q (live columns)
        bt_precond(B, B.r.get(), B.rt.get(), kst, s);
        SSV_CUDA(cudaMemcpyAsync(B.p.get(), B.rt.get(), sizeof(zdouble) * len, cudaMemcpyDeviceToDevice, s));
        spmm(B, B.p.get(), B.q.get(), BT_RHO_INIT, s);
        nk += 4;
        if (cycles == 0) SSV_CUDA(cudaEventRecord(e1, s));
        if (maxiter > 0) run_graph_loop(B.loop, kst, maxiter);
        SSV_CUDA(cudaMemcpyAsync(&h, B.bs.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
        if (h.ks.status == SSV_ERR_TIMEOUT) fail(SSV_ERR_TIMEOUT, "batched COCR loop guard fired");
        ++cycles;
        loops += h.ks.loops;
        if (!refined) {
            SSV_CUDA(cudaMemcpyAsync(hc.data(), B.cols.get(), sizeof(BCol) * B.C, cudaMemcpyDeviceToHost, s));
            break;
        }
        // FP64 true residuals of every column: t = A x, r = P(b - t)
        h.ks.done = 0;  // lets the SpMM run; nothing is live while the host decides
        SSV_CUDA(cudaMemcpyAsync(B.bs.get(), &h, sizeof(h), cudaMemcpyHostToDevice, s));
        spmm(B, B.x.get(), B.t.get(), BT_TIME, s);
        bt_resid(B, s);
        nk += 2;
        SSV_CUDA(cudaMemcpyAsync(hc.data(), B.cols.get(), sizeof(BCol) * B.C, cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
        int restart = 0, ndone = 0;
        for (int c = 0; c < B.C; ++c) {
            BCol& col = hc[c];
            if (!fin[c]) {
                const double tr = col.normalizer > 0 ? col.tres / col.normalizer : 0.0;
                if (col.normalizer < 1e-30 || tr <= tol) {
                    fin[c] = 1;
                    col.converged = 1;
                } else if (col.work >= maxiter || col.work == work_prev[c] || col.tres < 1e-300) {
                    fin[c] = 1;  // out of iterations, or a cycle that could not take a step
                    col.converged = 0;
                } else {  // another cycle from the true residual
                    const double sc = col.tres / col.normalizer;
                    col.done = 0;
                    col.converged = 0;
                    col.restart_abs = B.restart_drop * col.tres;
                    col.brk_thr = 1e-30 * sc * sc;
                    ++restart;
                }
                col.iters = col.work;
                col.res = tr;
                work_prev[c] = col.work;
            }
            ndone += fin[c] ? 1 : 0;
        }
        if (!restart) break;
        h.ks.done = 0;
        h.ks.it = 0;
        h.ks.loops = 0;
        h.ndone = ndone;
        SSV_CUDA(cudaMemcpyAsync(B.cols.get(), hc.data(), sizeof(BCol) * B.C, cudaMemcpyHostToDevice, s));
        SSV_CUDA(cudaMemcpyAsync(B.bs.get(), &h, sizeof(h), cudaMemcpyHostToDevice, s));
    }
    zdouble* ux = static_cast<zdouble*>(d_x);
    if (B.R == 1) k_bt_scatter<1><<<ge, kBlock, 0, s>>>(B.n, B.F, B.x.get(), ux);
    else k_bt_scatter<4><<<ge, kBlock, 0, s>>>(B.n, B.F, B.x.get(), ux);
    SSV_LAUNCH_CHECK();
    SSV_CUDA(cudaEventRecord(e2, s));
    SSV_CUDA(cudaEventSynchronize(e2));
    float ms_all = 0.f, ms_loop = 0.f;
    SSV_CUDA(cudaEventElapsedTime(&ms_all, e0, e2));
    SSV_CUDA(cudaEventElapsedTime(&ms_loop, e1, e2));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    for (int c = 0; c < B.C; ++c) {
        if (iters) iters[c] = hc[c].iters;
        if (conv) conv[c] = hc[c].converged;
        if (res) {
            if (refined) res[c] = hc[c].res;
            else res[c] = hc[c].normalizer > 0 ? hc[c].res / hc[c].normalizer : 0.0;
        }
    }
    B.last_ms = ms_all;
    B.last_loop_ms = ms_loop;
    B.last_loops = loops;
    B.last_cycles = cycles;
    B.last_launches = nk + 2 + (int64_t)B.loop.body_nodes * loops / std::max(period, 1);
}

void batch_cocr_solve_host(ssv_batch* B, int maxiter, double tol, const void* b, void* x, int* iters, int* conv,
                           double* res) {
    const size_t len = (size_t)B->F * B->n * B->R;
    B->io_b.alloc(len);
    B->io_x.alloc(len);
    cudaStream_t s = stream();
    SSV_CUDA(cudaMemcpyAsync(B->io_b.get(), b, sizeof(zdouble) * len, cudaMemcpyHostToDevice, s));
    batch_cocr_solve_dev(B, maxiter, tol, B->io_b.get(), B->io_x.get(), iters, conv, res);
    SSV_CUDA(cudaMemcpyAsync(x, B->io_x.get(), sizeof(zdouble) * len, cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
}

int batch_tuning(const ssv_batch* B, ssv_batch_tune_entry* e, int cap, int* chosen) {
    *chosen = B->chosen;
    for (size_t i = 0; i < B->table.size() && (int)i < cap; ++i) e[i] = B->table[i];
    return (int)B->table.size();
}

void batch_set_replacement(ssv_batch* B, int every) { B->replace_every = every < 0 ? -1 : every; }

void batch_set_refinement(ssv_batch* B, double restart_drop) {
    if (!(restart_drop >= 0.0 && restart_drop < 1.0))
        fail(SSV_ERR_INVALID_ARG, "batch: restart_drop must lie in [0, 1)");
    B->restart_drop = restart_drop;
}

void batch_last_timing(const ssv_batch* B, double* ms, double* loop_ms, int* loops, int64_t* launches,
                       int* cycles) {
    if (cycles) *cycles = B->last_cycles;
    if (ms) *ms = B->last_ms;
    if (loop_ms) *loop_ms = B->last_loop_ms;
    if (loops) *loops = B->last_loops;
    if (launches) *launches = B->last_launches;
}

}  // namespace ssv
