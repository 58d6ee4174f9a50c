// mrtr.cu -- SGS-MRTR (solvers/sgs_mrtr_solver.hpp) on the device.
//
// Split-formula MRTR on D A D (D = |diag A|^{-1/2}) with level-scheduled
// forward / backward sweeps over L = lower(D A D). Per iteration:
// backward sweep, forward sweep on (rd - u), one fused pass that forms
// Ard = L^{-1}(rd-u) + u and the three inner products, and one fused update
// pass with the residual norm; the scalar recurrences (zeta, eta, nu) run on
// the device in the reductions' last block.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "objects.cuh"

namespace ssv {

// D_i = 1/sqrt(|a_ii|), inv_D_i = sqrt(|a_ii|) (sgs_mrtr_solver.hpp:88-97)
template <typename S>
__global__ void k_mrtr_diag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            const S* __restrict__ v, double* __restrict__ D, double* __restrict__ iD) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int lo = rp[i], hi = rp[i + 1];
        while (lo < hi) {  // SparseMatrixView::operator() binary search
            const int mid = lo + (hi - lo) / 2;
            if (ci[mid] < i) lo = mid + 1; else hi = mid;
        }
        const S aii = (lo < rp[i + 1] && ci[lo] == i) ? v[lo] : ST<S>::zero();
        const double a = ST<S>::abs(aii);
        if (a > 1e-15) { D[i] = 1.0 / sqrt(a); iD[i] = sqrt(a); }
        else { D[i] = 1.0; iD[i] = 1.0; }
    }
}

// L_k = D_i * a_k * D_j over the lower pattern (build_L_and_Lt :298-308)
template <typename S>
__global__ void k_mrtr_lvals(int n, const int* __restrict__ Lrp, const int* __restrict__ Lci,
                             const int* __restrict__ Lsrc, const S* __restrict__ v, const double* __restrict__ D,
                             S* __restrict__ Lv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = Lrp[i]; k < Lrp[i + 1]; ++k)
            Lv[k] = ST<S>::scale(D[Lci[k]], ST<S>::scale(D[i], v[Lsrc[k]]));
}

// b2 = D b, x2 = inv_D x, r = D (b - A x); constrained entries of b, x zeroed.
template <typename S>
__global__ void k_mrtr_prep(int n, const double* __restrict__ D, const double* __restrict__ iD,
                            const S* __restrict__ b, const S* __restrict__ x, const S* __restrict__ Ax,
                            const uint8_t* __restrict__ fd, S* __restrict__ b2, S* __restrict__ x2,
                            S* __restrict__ r) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool f = !fd || fd[i];
        const S bi = f ? b[i] : ST<S>::zero();
        b2[i] = ST<S>::scale(D[i], bi);
        x2[i] = ST<S>::scale(iD[i], f ? x[i] : ST<S>::zero());
        r[i] = ST<S>::scale(D[i], bi - Ax[i]);
    }
}

// forward sweep over one level: y_i = (a_i - b_i - sum L_ij y_j) / L_ii
template <typename S>
__global__ void k_mrtr_fwd(int u0, int u1, const int* __restrict__ rows, const int* __restrict__ Lrp,
                           const int* __restrict__ Lci, const S* __restrict__ Lv, const S* __restrict__ a,
                           const S* __restrict__ b, S* __restrict__ y, const KState* st) {
    if (st && st->done) return;
    const int u = u0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= u1) return;
    const int i = rows[u];
    S s = a[i];
    if (b) s = s - b[i];
    const int ke = Lrp[i + 1] - 1;
    for (int k = Lrp[i]; k < ke; ++k) s = s - Lv[k] * y[Lci[k]];
    y[i] = ST<S>::div(s, Lv[ke]);
}

// backward sweep over one level: y_i = (rhs_i - sum_{j>i} U_ij y_j) / U_ii
template <typename S>
__global__ void k_mrtr_bwd(int u0, int u1, const int* __restrict__ rows, const int* __restrict__ Urp,
                           const int* __restrict__ Uci, const S* __restrict__ Uv, const S* __restrict__ rhs,
                           S* __restrict__ y, const KState* st) {
    if (st && st->done) return;
    const int u = u0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= u1) return;
    const int i = rows[u];
    const int rs = Urp[i], re = Urp[i + 1];
    if (rs >= re) { y[i] = ST<S>::zero(); return; }
    S s = rhs[i];
    for (int k = rs + 1; k < re; ++k) s = s - Uv[k] * y[Uci[k]];
    y[i] = ST<S>::div(s, Uv[rs]);
}

template <typename S>
__device__ __forceinline__ S dotc(S a, S b, bool conj) {
    return (conj ? ST<S>::conj(a) : a) * b;
}

// Ard += u, then (Ard, rd), (Ard, Ard), (Ard, y); last block: MRTR scalars
// (sgs_mrtr_solver.hpp:182-211).
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_mrtr_dots(int n, S* __restrict__ Ard, const S* __restrict__ u, const S* __restrict__ rd,
            const S* __restrict__ y, KState* st, double2* partials, unsigned int* ticket) {
    if (st->done) return;
    const bool conj = st->conj != 0;
    double2 p0 = make_double2(0, 0), p1 = p0, p2 = p0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const S a = Ard[i] + u[i];
        Ard[i] = a;
        p0 = add2(p0, s_to2<S>(dotc(a, rd[i], conj)));
        p1 = add2(p1, s_to2<S>(dotc(a, a, conj)));
        p2 = add2(p2, s_to2<S>(dotc(a, y[i], conj)));
    }
    __shared__ bool am_last;
    p0 = block_sum2(p0);
    p1 = block_sum2(p1);
    p2 = block_sum2(p2);
    const int G = gridDim.x;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = p0;
        partials[G + blockIdx.x] = p1;
        partials[2 * G + blockIdx.x] = p2;
        __threadfence();
        am_last = (atomicAdd(ticket, 1u) == (unsigned)G - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    double2 s0 = make_double2(0, 0), s1 = s0, s2 = s0;
    for (int b = threadIdx.x; b < G; b += blockDim.x) {
        s0 = add2(s0, __ldcg(&partials[b]));
        s1 = add2(s1, __ldcg(&partials[G + b]));
        s2 = add2(s2, __ldcg(&partials[2 * G + b]));
    }
    s0 = block_sum2(s0);
    s1 = block_sum2(s1);
    s2 = block_sum2(s2);
    if (threadIdx.x != 0) return;
    *ticket = 0u;
    const S Ar_r = s_from2<S>(s0), Ar_Ar = s_from2<S>(s1), Ar_y = s_from2<S>(s2);
    // st->rho = zeta_old, st->rho_new = nu, st->alpha = zeta, st->beta = eta, st->denom = coeff
    S zeta, eta, zeta_old = s_from2<S>(st->rho), nu = s_from2<S>(st->rho_new);
    if (st->it == 0) {
        zeta = ST<S>::div(Ar_r, Ar_Ar);
        zeta_old = zeta;
        eta = ST<S>::zero();
    } else {
        S denom = nu * Ar_Ar - Ar_y * Ar_y;
        if (ST<S>::abs(denom) < 1e-60)
            denom = ST<S>::real(denom) >= 0 ? ST<S>::from(1e-60) : ST<S>::from(-1e-60);
        const S inv = ST<S>::div(ST<S>::one(), denom);
        zeta = nu * Ar_r * inv;
        eta = (ST<S>::zero() - Ar_y) * Ar_r * inv;
    }
    nu = zeta * Ar_r;
    const S coeff = ST<S>::div(eta * zeta_old, zeta);
    st->alpha = s_to2<S>(zeta);
    st->beta = s_to2<S>(eta);
    st->denom = s_to2<S>(coeff);
    st->rho = s_to2<S>(zeta);  // zeta_old for the next iteration
    st->rho_new = s_to2<S>(nu);
}

// p = u + coeff p ; x2 += zeta p ; y = eta y + zeta Ard ; rd -= y ; ||rd||
template <typename S>
__global__ void __launch_bounds__(kBlock)
k_mrtr_update(int n, S* xb0, S* xb1, S* xb2, const S* __restrict__ u, const S* __restrict__ Ard,
              S* __restrict__ p, S* __restrict__ y, S* __restrict__ rd, KState* st, RedBuf red) {
    if (st->done) return;
    const int cur = st->cur;
    int nxt = cur;
    if (st->save_best) {
        const int best = st->best;
        for (int c = 0; c < 3; ++c) if (c != cur && c != best) { nxt = c; break; }
    }
    S* xs[3] = {xb0, xb1, xb2};
    const S* xc = xs[cur];
    S* xn = xs[nxt];
    const S zeta = s_from2<S>(st->alpha), eta = s_from2<S>(st->beta), coeff = s_from2<S>(st->denom);
    double2 part = make_double2(0.0, 0.0);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const S pi = u[i] + coeff * p[i];
        p[i] = pi;
        xn[i] = xc[i] + zeta * pi;
        const S yi = eta * y[i] + zeta * Ard[i];
        y[i] = yi;
        const S ri = rd[i] - yi;
        rd[i] = ri;
        part.x += ST<S>::norm2(ri);
    }
    double2 total;
    if (grid_reduce2(part, red.partials, red.ticket, total)) dev_check(st, sqrt(total.x), 0, nxt);
}

template <typename S>
__global__ void k_neg(int n, const S* __restrict__ a, S* __restrict__ b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        b[i] = ST<S>::zero() - a[i];
}

// x_i = D_i x2_i on free entries (convert_x2_to_x + the free-DOF copy-back)
template <typename S>
__global__ void k_mrtr_out(int n, const double* __restrict__ D, const S* __restrict__ x2,
                           const uint8_t* __restrict__ fd, S* __restrict__ x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (!fd || fd[i]) x[i] = ST<S>::scale(D[i], x2[i]);
}

template <typename S>
struct MrtrPattern {
    bool built = false;
    std::vector<std::pair<int, int>> fwd, bwd;
    DevBuf<int> Lrp, Lci, Lsrc, Urp, Uci, Usrc, rows_f, rows_b;
    DevBuf<S> Lv, Uv, u, Ard, y, rd;
    DevBuf<double> D, iD;
};

template <typename S> MrtrPattern<S>& mrtr_of(ssv_solver* s);

template <typename S>
void run_mrtr(ssv_solver* sv, const ssv_config& cfg, const S* d_b, S* d_x, ssv_result* res, double* hist,
              int hist_cap);

}  // namespace ssv

// The pattern objects hang off the solver handle through a side table keyed
// by the handle (kept here so objects.cuh stays small).
#include <map>
#include <memory>
namespace ssv {
template <typename S>
static std::map<const ssv_solver*, std::unique_ptr<MrtrPattern<S>>>& mrtr_table() {
    static std::map<const ssv_solver*, std::unique_ptr<MrtrPattern<S>>> t;
    return t;
}
void mrtr_forget(const ssv_solver* s) {
    mrtr_table<double>().erase(s);
    mrtr_table<zdouble>().erase(s);
}
template <typename S>
MrtrPattern<S>& mrtr_of(ssv_solver* s) {
    auto& t = mrtr_table<S>();
    auto& p = t[s];
    if (!p) p.reset(new MrtrPattern<S>());
    return *p;
}

template <typename S> KrylovWork<S>& mwork_of(ssv_solver* s);
template <> KrylovWork<double>& mwork_of<double>(ssv_solver* s) { return s->w_d; }
template <> KrylovWork<zdouble>& mwork_of<zdouble>(ssv_solver* s) { return s->w_z; }

template <typename S>
void run_mrtr(ssv_solver* sv, const ssv_config& cfg, const S* d_b, S* d_x, ssv_result* res, double* hist,
              int hist_cap) {
    cudaStream_t s = stream();
    ssv_matrix* A = sv->A;
    const int n = A->rows;
    const double t0 = wall_seconds();
    const uint8_t* fd = sv->has_fd ? sv->fd.get() : nullptr;
    const S* vals = reinterpret_cast<const S*>(A->val.get());
    if (fd) {
        sv->vals_bc.alloc(A->val.size());
        k_bc_values<S><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, A->rp.get(), A->ci.get(), vals, fd,
                                                             reinterpret_cast<S*>(sv->vals_bc.get()));
        vals = reinterpret_cast<const S*>(sv->vals_bc.get());
    }
    MrtrPattern<S>& P = mrtr_of<S>(sv);
    if (!P.built) {
        std::vector<int> lrp, lci, lsrc, urp, uci, usrc, lev, rws, off;
        lower_pattern(n, A->h_rp.data(), A->h_ci.data(), lrp, lci, lsrc);
        transpose_pattern(n, lrp, lci, urp, uci, usrc);
        P.fwd.clear();
        P.bwd.clear();
        int nl = build_levels(n, lrp.data(), lci.data(), false, lev);
        group_by_level(lev, nl, rws, off);
        P.rows_f.upload(rws.data(), rws.size(), s);
        for (int l = 0; l < nl; ++l) P.fwd.push_back({off[l], off[l + 1]});
        nl = build_levels(n, urp.data(), uci.data(), true, lev);
        group_by_level(lev, nl, rws, off);
        P.rows_b.upload(rws.data(), rws.size(), s);
        for (int l = 0; l < nl; ++l) P.bwd.push_back({off[l], off[l + 1]});
        P.Lrp.upload(lrp.data(), lrp.size(), s);
        P.Lci.upload(lci.data(), lci.size(), s);
        P.Lsrc.upload(lsrc.data(), lsrc.size(), s);
        P.Urp.upload(urp.data(), urp.size(), s);
        P.Uci.upload(uci.data(), uci.size(), s);
        P.Usrc.upload(usrc.data(), usrc.size(), s);
        P.Lv.alloc(lci.size());
        P.Uv.alloc(uci.size());
        P.u.alloc(n); P.Ard.alloc(n); P.y.alloc(n); P.rd.alloc(n);
        P.D.alloc(n); P.iD.alloc(n);
        P.built = true;
    }
    const int g = grid_for(n, kBlock);
    KrylovWork<S>& w = mwork_of<S>(sv);
    const int dev_hist = cfg.save_residual_history ? std::max(cfg.max_iterations, 0) + 2 : 1;
    w.ensure(n, dev_hist);
    if (w.partials.size() < (size_t)sm_count() * 8 * 3 + 64) w.partials.alloc((size_t)sm_count() * 8 * 3 + 64);
    const RedBuf red = w.red();
    k_mrtr_diag<S><<<g, kBlock, 0, s>>>(n, A->rp.get(), A->ci.get(), vals, P.D.get(), P.iD.get());
    k_mrtr_lvals<S><<<g, kBlock, 0, s>>>(n, P.Lrp.get(), P.Lci.get(), P.Lsrc.get(), vals, P.D.get(), P.Lv.get());
    k_gather_values<S><<<grid_for(P.Usrc.size(), kBlock), kBlock, 0, s>>>((int64_t)P.Usrc.size(), P.Usrc.get(),
                                                                         P.Lv.get(), P.Uv.get());
    SSV_LAUNCH_CHECK();
    SSV_CUDA(cudaStreamSynchronize(s));
    const double t1 = wall_seconds();
    // x_mod with constrained entries zeroed, Ax = A x_mod
    S* xm = w.t.get();
    k_gather_perm<S><<<g, kBlock, 0, s>>>(n, nullptr, d_x, xm, fd, 1);
    launch_spmv<S, S, 0>(A->lanes, n, A->rp.get(), A->ci.get(), vals, xm, w.Ap.get(), nullptr, nullptr, nullptr,
                         RED_STORE, red, nullptr, s);
    S* b2 = w.bw.get();
    k_mrtr_prep<S><<<g, kBlock, 0, s>>>(n, P.D.get(), P.iD.get(), d_b, xm, w.Ap.get(), fd, b2, w.xb[0].get(),
                                       w.r.get());
    // normalizer = ||L b2|| (lower incl. diagonal)
    launch_spmv<S, S, 0>(pick_lanes(n ? (double)P.Lci.size() / n : 1.0), n, P.Lrp.get(), P.Lci.get(),
                         P.Lv.get(), b2, w.qt.get(), nullptr, nullptr, nullptr, RED_STORE, red, nullptr, s);
    k_norm2<S><<<g, kBlock, 0, s>>>(n, w.qt.get(), red, w.scal.get());
    k_norm2<S><<<g, kBlock, 0, s>>>(n, w.r.get(), red, w.scal.get() + 1);
    k_norm2<S><<<g, kBlock, 0, s>>>(n, b2, red, w.scal.get() + 2);
    SSV_LAUNCH_CHECK();
    double2 nrm[3];
    SSV_CUDA(cudaMemcpyAsync(nrm, w.scal.get(), sizeof(nrm), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    const double nLb = std::sqrt(nrm[0].x), norm_r0 = std::sqrt(nrm[1].x);
    double nb2 = std::sqrt(nrm[2].x);
    const double normalizer = nLb > 1e-15 ? nLb : 1.0;
    if (nb2 < 1e-30) nb2 = 1.0;

    // rd = L^{-1} r ; y = -rd ; p = 0
    for (const auto& lv : P.fwd)
        k_mrtr_fwd<S><<<(lv.second - lv.first + 127) / 128, 128, 0, s>>>(lv.first, lv.second, P.rows_f.get(),
                                                                         P.Lrp.get(), P.Lci.get(), P.Lv.get(),
                                                                         w.r.get(), nullptr, P.rd.get(), nullptr);
    k_neg<S><<<g, kBlock, 0, s>>>(n, P.rd.get(), P.y.get());
    w.p.zero(s);
    SSV_LAUNCH_CHECK();

    KState h;
    std::memset(&h, 0, sizeof(h));
    h.cur = 0;
    h.best = -1;
    h.normalizer = normalizer;
    h.best_residual = DBL_MAX;
    h.norm_r = norm_r0;
    h.final_norm = norm_r0;
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
    h.rho = make_double2(1.0, 0.0);      // zeta_old
    h.rho_new = make_double2(1.0, 0.0);  // nu
    if (cfg.save_residual_history) {
        const double h0 = norm_r0 / normalizer;
        SSV_CUDA(cudaMemcpyAsync(w.hist.get(), &h0, sizeof(double), cudaMemcpyHostToDevice, s));
        h.hist_len = 1;
    }
    bool early = false;
    if (norm_r0 / nb2 < cfg.tolerance * 0.1) {  // do_iterate :155-163
        h.done = 1; h.converged = 1; h.iters = 0; h.final_norm = norm_r0;
        early = true;
    } else if (cfg.max_iterations <= 0) {
        h.done = 1; h.iters = 0;
    }
    KState* dst = w.st.get();
    SSV_CUDA(cudaMemcpyAsync(dst, &h, sizeof(h), cudaMemcpyHostToDevice, s));
    const std::string key = "mrtr;" + std::to_string(n) + ";" + std::to_string((size_t)P.Lv.get()) + ";" +
                            std::to_string((size_t)dst) + ";" + std::to_string((size_t)w.r.get()) + ";" +
                            std::to_string((size_t)w.partials.get()) + ";" + std::to_string(fd != nullptr);
    build_graph_loop(sv->loop, key, [&](cudaGraphConditionalHandle hc, int use_cond) {
        for (const auto& lv : P.bwd)
            k_mrtr_bwd<S><<<(lv.second - lv.first + 127) / 128, 128, 0, s>>>(
                lv.first, lv.second, P.rows_b.get(), P.Urp.get(), P.Uci.get(), P.Uv.get(), P.rd.get(), P.u.get(),
                dst);
        for (const auto& lv : P.fwd)
            k_mrtr_fwd<S><<<(lv.second - lv.first + 127) / 128, 128, 0, s>>>(
                lv.first, lv.second, P.rows_f.get(), P.Lrp.get(), P.Lci.get(), P.Lv.get(), P.rd.get(), P.u.get(),
                P.Ard.get(), dst);
        k_mrtr_dots<S><<<g, kBlock, 0, s>>>(n, P.Ard.get(), P.u.get(), P.rd.get(), P.y.get(), dst, w.partials.get(),
                                           w.ticket.get());
        k_mrtr_update<S><<<g, kBlock, 0, s>>>(n, w.xb[0].get(), w.xb[1].get(), w.xb[2].get(), P.u.get(),
                                             P.Ard.get(), w.p.get(), P.y.get(), P.rd.get(), dst, red);
        k_loop_ctl<<<1, 32, 0, s>>>(dst, hc, use_cond);
        SSV_LAUNCH_CHECK();
    });
    if (!h.done) run_graph_loop(sv->loop, dst, cfg.max_iterations);
    SSV_CUDA(cudaMemcpyAsync(&h, dst, sizeof(h), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    if (h.status == SSV_ERR_TIMEOUT) fail(SSV_ERR_TIMEOUT, "SGS-MRTR loop guard fired");
    res->converged = h.converged;
    res->iterations = h.iters;
    res->final_residual = h.final_norm / h.normalizer;
    int xbuf = h.cur;
    if (!h.converged && cfg.save_best_result && !early) {
        res->final_residual = h.best_residual;
        xbuf = h.best;
    }
    const S* x2;
    if (xbuf < 0) { w.Ap.zero(s); x2 = w.Ap.get(); }
    else x2 = w.xb[xbuf].get();
    k_mrtr_out<S><<<g, kBlock, 0, s>>>(n, P.D.get(), x2, fd, d_x);
    SSV_LAUNCH_CHECK();
    res->history_total = cfg.save_residual_history ? h.hist_len : 0;
    res->history_len = std::min(std::min(res->history_total, dev_hist), std::max(hist_cap, 0));
    if (hist && res->history_len > 0)
        SSV_CUDA(cudaMemcpyAsync(hist, w.hist.get(), sizeof(double) * res->history_len, cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    res->setup_seconds = t1 - t0;
    res->solve_seconds = wall_seconds() - t1;
}

template void run_mrtr<double>(ssv_solver*, const ssv_config&, const double*, double*, ssv_result*, double*, int);
template void run_mrtr<zdouble>(ssv_solver*, const ssv_config&, const zdouble*, zdouble*, ssv_result*, double*,
                                int);

}  // namespace ssv
