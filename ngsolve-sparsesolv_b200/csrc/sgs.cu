// SGSPreconditioner (include/sparsesolv/preconditioners/sgs_preconditioner.hpp
// and its NGSolve wrapper ngsolve/sparsesolv_precond.hpp:230-250):
// M^{-1} = (D + U)^{-1} D (D + L)^{-1} on the FreeDofs view of A (constrained
// rows identity, constrained columns zero), output zeroed on constrained DOFs.
// Both sweeps run level set by level set (the reference's LevelSchedule built
// from the full pattern, entries j < i forward and j > i backward), one
// launch per level, one thread per row; the arithmetic of a row is the
// reference's, in its order.
#include "objects.cuh"
#include "solver_api.hpp"

namespace ssv {

// 1 / a_ii, or 1 where |a_ii| <= 1e-15 (constants.hpp:30, sgs_preconditioner.hpp:76-85)
template <typename S>
__global__ void k_sgs_inv_diag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                               const S* __restrict__ v, S* __restrict__ inv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        S d = ST<S>::zero();
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) {
                d = v[k];
                break;
            }
        inv[i] = ST<S>::abs(d) > 1e-15 ? ST<S>::div(ST<S>::one(), d) : ST<S>::one();
    }
}

// one level of a sweep: y_i = (x_i - sum_{j<i (fwd) / j>i (bwd)} a_ij y_j) / a_ii
template <typename S, bool FWD>
__global__ void __launch_bounds__(128)
k_sgs_sweep(int q0, int q1, const int* __restrict__ rows, const int* __restrict__ rp, const int* __restrict__ ci,
            const S* __restrict__ v, const S* __restrict__ inv, const S* __restrict__ x, S* y, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int q = q0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= q1) return;
    const int i = rows[q];
    S sum = x[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int j = ci[k];
        if (FWD ? j < i : j > i) sum = sum - v[k] * y[j];
    }
    y[i] = sum * inv[i];
}

// scaled = temp / inv (sgs_preconditioner.hpp:119-123: D = 1 / inv_diag)
template <typename S>
__global__ void k_sgs_scale(int n, const S* __restrict__ inv, S* __restrict__ t, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        t[i] = ST<S>::div(t[i], inv[i]);
}

template <typename S> SgsDevice<S>& sgs_of(ssv_precond* p);
template <> SgsDevice<double>& sgs_of<double>(ssv_precond* p) { return p->sgs_d; }
template <> SgsDevice<zdouble>& sgs_of<zdouble>(ssv_precond* p) { return p->sgs_z; }

static void levels_of(int n, const std::vector<int>& rp, const std::vector<int>& ci, bool upper,
                      std::vector<std::pair<int, int>>& ranges, DevBuf<int>& rows_d, cudaStream_t s) {
    std::vector<int> lev, rows, off;
    const int nl = build_levels(n, rp.data(), ci.data(), upper, lev);
    group_by_level(lev, nl, rows, off);
    ranges.clear();
    for (int l = 0; l < nl; ++l) ranges.push_back({off[l], off[l + 1]});
    rows_d.upload(rows.data(), rows.size(), s);
}

template <typename S>
static void sgs_update_t(ssv_precond* p) {
    cudaStream_t s = stream();
    ssv_matrix* A = p->A;
    const int n = A->rows;
    SgsDevice<S>& g = sgs_of<S>(p);
    const S* vals = reinterpret_cast<const S*>(A->val.get());
    if (p->has_fd) {  // BuildSparseMatrixView (sparsesolv_precond.hpp:35-90)
        p->vals_bc.alloc(A->val.size());
        k_bc_values<S><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, A->rp.get(), A->ci.get(), vals, p->fd.get(),
                                                             reinterpret_cast<S*>(p->vals_bc.get()));
        SSV_LAUNCH_CHECK();
        vals = reinterpret_cast<const S*>(p->vals_bc.get());
    }
    if (!g.built) {
        levels_of(n, A->h_rp, A->h_ci, false, g.fwd_lev, g.rows_f, s);
        levels_of(n, A->h_rp, A->h_ci, true, g.bwd_lev, g.rows_b, s);
        g.inv.alloc(n);
        g.tmp.alloc(n);
        g.built = true;
        ++g.gen;
    }
    k_sgs_inv_diag<S><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, A->rp.get(), A->ci.get(), vals, g.inv.get());
    SSV_LAUNCH_CHECK();
    SSV_CUDA(cudaStreamSynchronize(s));
    p->ready = true;
}

void sgs_update(ssv_precond* p) {
    if (p->A->dtype == SSV_F64) sgs_update_t<double>(p);
    else sgs_update_t<zdouble>(p);
}

template <typename S>
void sgs_apply_dev(ssv_precond* p, const S* x, S* y, const KState* st, cudaStream_t s) {
    ssv_matrix* A = p->A;
    const int n = A->rows;
    SgsDevice<S>& g = sgs_of<S>(p);
    const S* v = p->has_fd ? reinterpret_cast<const S*>(p->vals_bc.get()) : reinterpret_cast<const S*>(A->val.get());
    const int* rp = A->rp.get();
    const int* ci = A->ci.get();
    S* t = g.tmp.get();
    for (const auto& r : g.fwd_lev)
        launch_k(k_sgs_sweep<S, true>, (r.second - r.first + 127) / 128, 128, s, r.first, r.second,
                 (const int*)g.rows_f.get(), rp, ci, v, (const S*)g.inv.get(), x, t, st);
    launch_k(k_sgs_scale<S>, grid_for(n, kBlock), kBlock, s, n, (const S*)g.inv.get(), t, st);
    for (const auto& r : g.bwd_lev)
        launch_k(k_sgs_sweep<S, false>, (r.second - r.first + 127) / 128, 128, s, r.first, r.second,
                 (const int*)g.rows_b.get(), rp, ci, v, (const S*)g.inv.get(), (const S*)t, y, st);
    if (p->has_fd) launch_k(k_mask_zero<S>, grid_for(n, kBlock), kBlock, s, n, y, (const uint8_t*)p->fd.get());
    SSV_LAUNCH_CHECK();
}

template void sgs_apply_dev<double>(ssv_precond*, const double*, double*, const KState*, cudaStream_t);
template void sgs_apply_dev<zdouble>(ssv_precond*, const zdouble*, zdouble*, const KState*, cudaStream_t);

}  // namespace ssv
