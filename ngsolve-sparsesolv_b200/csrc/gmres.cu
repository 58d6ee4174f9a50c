// GMRESSolver (include/sparsesolv/ngsolve/sparsesolv_solvers.hpp:409-584,
// factory sparsesolv_python_export.hpp:643-697): right-preconditioned GMRES
// with restarts, modified Gram-Schmidt and Givens rotations on the FreeDofs
// projection, x0 = 0, stop when |g_{j+1}| / ||P b|| < tol. Vectors, the
// Hessenberg columns, rotations and the rotated right-hand side live on the
// device; the host drives the iteration (the Gram-Schmidt of step j has j+1
// dependent dot/update pairs) and reads two scalars per step to stop.
#include <cmath>

#include "objects.cuh"
#include "solver_api.hpp"

namespace ssv {

// y = s x (s a host scalar), or y = 0 when zero != 0
template <typename S>
__global__ void k_gm_scale(int n, double s, int zero, const S* __restrict__ x, S* __restrict__ y) {
    pdl_gate();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = zero ? ST<S>::zero() : ST<S>::scale(s, x[i]);
}

// w -= h v with h = H[j][i] on the device (the Gram-Schmidt update)
template <typename S>
__global__ void k_gm_axpy(int n, const double2* __restrict__ h, const S* __restrict__ v, S* __restrict__ w) {
    pdl_gate();
    const S hv = s_from2<S>(*h);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] = w[i] - hv * v[i];
}

template <typename S>
__device__ inline S gm_conj(S a) { return ST<S>::conj(a); }

// complex / real divides each component (std::complex<double> / double)
__device__ inline double gm_div_real(double a, double d) { return a / d; }
__device__ inline zdouble gm_div_real(zdouble a, double d) { return {a.x / d, a.y / d}; }

// compute_givens (:547-562): [c s; -conj(s) c] [a; b] = [r; 0]
template <typename S>
__device__ inline void gm_givens(S a, S b, double& c, S& s) {
    if (ST<S>::abs(b) < 1e-30) {
        c = 1.0;
        s = ST<S>::zero();
    } else if (ST<S>::abs(a) < 1e-30) {
        c = 0.0;
        s = ST<S>::one();
    } else {
        const double denom = sqrt(ST<S>::norm2(a) + ST<S>::norm2(b));
        c = ST<S>::abs(a) / denom;
        s = gm_div_real(a * gm_conj(b), ST<S>::abs(a) * denom);
    }
}

// Step j after the Gram-Schmidt: H[j][j+1] = ||w||, earlier rotations, the new
// rotation, g; out = (|g_{j+1}| / ||P b||, ||w||). Column j of H at H2 + j*(m+1).
template <typename S>
__global__ void k_gm_rotate(int j, int m, double2* H2, double* cs, double2* sn2, double2* g2, const double2* wn2,
                            double rhs_norm, double2* out) {
    pdl_gate();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double2* h = H2 + (size_t)j * (m + 1);
    const double h_next = sqrt(fabs(wn2->x));
    h[j + 1] = s_to2<S>(ST<S>::from(h_next));
    for (int i = 0; i < j; ++i) {
        const S hi = s_from2<S>(h[i]), hi1 = s_from2<S>(h[i + 1]);
        const S si = s_from2<S>(sn2[i]);
        h[i] = s_to2<S>(ST<S>::from(cs[i]) * hi + si * hi1);
        h[i + 1] = s_to2<S>(ST<S>::from(-1.0) * gm_conj(si) * hi + ST<S>::from(cs[i]) * hi1);
    }
    double c;
    S s;
    gm_givens<S>(s_from2<S>(h[j]), s_from2<S>(h[j + 1]), c, s);
    cs[j] = c;
    sn2[j] = s_to2<S>(s);
    h[j] = s_to2<S>(ST<S>::from(c) * s_from2<S>(h[j]) + s * s_from2<S>(h[j + 1]));
    h[j + 1] = make_double2(0.0, 0.0);
    const S gj = s_from2<S>(g2[j]);
    g2[j] = s_to2<S>(ST<S>::from(c) * gj);
    const S gn = ST<S>::from(-1.0) * gm_conj(s) * gj;
    g2[j + 1] = s_to2<S>(gn);
    *out = make_double2(ST<S>::abs(gn) / rhs_norm, h_next);
}

// back substitution H y = g (:566-573), y in yv
template <typename S>
__global__ void k_gm_backsolve(int dim, int m, const double2* H2, const double2* g2, double2* yv) {
    pdl_gate();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = dim - 1; i >= 0; --i) {
        S yi = s_from2<S>(g2[i]);
        for (int k = i + 1; k < dim; ++k) yi = yi - s_from2<S>(H2[(size_t)k * (m + 1) + i]) * s_from2<S>(yv[k]);
        const S hii = s_from2<S>(H2[(size_t)i * (m + 1) + i]);
        if (ST<S>::abs(hii) > 1e-30) yi = ST<S>::div(yi, hii);
        yv[i] = s_to2<S>(yi);
    }
}

// x += sum_i y_i Z_i, the terms added in the order i = 0 .. dim-1 (:576-578)
template <typename S>
__global__ void k_gm_update(int n, int dim, const S* __restrict__ Z, const double2* __restrict__ yv, S* __restrict__ x) {
    pdl_gate();
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        S acc = x[r];
        for (int i = 0; i < dim; ++i) acc = acc + s_from2<S>(yv[i]) * Z[(size_t)i * n + r];
        x[r] = acc;
    }
}

template <typename S>
static void run_gmres(ssv_matrix* A, ssv_precond* pre, const uint8_t* fd, int maxiter, double tol, int restart,
                      const S* d_b, S* d_x, int* iterations) {
    cudaStream_t s = stream();
    const int n = A->rows;
    const int g = grid_for(n, kBlock);
    const S* v = reinterpret_cast<const S*>(A->val.get());
    const int m = std::max(1, std::min(maxiter, restart > 0 ? restart : maxiter));
    DevBuf<S> V((size_t)(m + 1) * n), Z((size_t)m * n), w(n), r(n), rhs(n);
    DevBuf<double2> H2((size_t)m * (m + 1)), sn2(m), g2(m + 1), yv(m), scal(4);
    DevBuf<double> cs(m);
    DevBuf<double2> partials((size_t)sm_count() * 8 + 64);
    DevBuf<unsigned int> ticket(4);
    SSV_CUDA(cudaMemsetAsync(ticket.get(), 0, sizeof(unsigned int) * 4, s));
    const RedBuf red{partials.get(), ticket.get()};
    auto vcol = [&](int i) { return V.get() + (size_t)i * n; };
    auto zcol = [&](int i) { return Z.get() + (size_t)i * n; };
    auto read2 = [&](const double2* p) {
        double2 h;
        SSV_CUDA(cudaMemcpyAsync(&h, p, sizeof(h), cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
        return h;
    };
    auto norm = [&](const S* a) {
        launch_k(k_norm2<S>, g, kBlock, s, n, a, red, scal.get());
        return std::sqrt(std::fabs(read2(scal.get()).x));
    };
    const int conj = ST<S>::cplx ? 1 : 0;
    SSV_CUDA(cudaMemsetAsync(d_x, 0, sizeof(S) * n, s));  // sol = 0
    launch_k(k_gather_perm<S>, g, kBlock, s, n, (const int*)nullptr, d_b, rhs.get(), fd, 1);  // r = P rhs
    const double rhs_norm = norm(rhs.get());
    int total = 0;
    if (rhs_norm >= 1e-30) {
        double beta = rhs_norm;
        for (int cycle = 0; total < maxiter; ++cycle) {
            const S* rv = rhs.get();
            if (cycle > 0) {  // r = P rhs - P (A sol)
                launch_spmv<S, S, 2>(A->lanes, n, A->rp.get(), A->ci.get(), v, d_x, r.get(), rhs.get(), fd, nullptr,
                                     RED_STORE, red, nullptr, s);
                beta = norm(r.get());
                if (beta / rhs_norm < tol) break;
                rv = r.get();
            }
            launch_k(k_gm_scale<S>, g, kBlock, s, n, 1.0 / beta, 0, rv, vcol(0));
            std::vector<double2> g0(m + 1, make_double2(0.0, 0.0));
            g0[0] = make_double2(beta, 0.0);
            g2.upload(g0.data(), g0.size(), s);
            SSV_CUDA(cudaMemsetAsync(cs.get(), 0, sizeof(double) * m, s));
            SSV_CUDA(cudaMemsetAsync(sn2.get(), 0, sizeof(double2) * m, s));
            int j = 0;
            double2 last = make_double2(1.0, 1.0);
            while (j < m && total < maxiter) {
                if (pre) precond_apply_any<S>(pre, vcol(j), zcol(j), nullptr, s);
                else launch_k(k_copy<S>, g, kBlock, s, n, (const S*)vcol(j), zcol(j));
                launch_spmv<S, S, 0>(A->lanes, n, A->rp.get(), A->ci.get(), v, zcol(j), w.get(), nullptr, fd, nullptr,
                                     RED_STORE, red, nullptr, s);
                double2* hcol = H2.get() + (size_t)j * (m + 1);
                for (int i = 0; i <= j; ++i) {  // modified Gram-Schmidt
                    launch_k(k_dot<S>, g, kBlock, s, n, (const S*)vcol(i), (const S*)w.get(), conj, (KState*)nullptr,
                             (int)RED_STORE, red, hcol + i);
                    launch_k(k_gm_axpy<S>, g, kBlock, s, n, (const double2*)(hcol + i), (const S*)vcol(i), w.get());
                }
                launch_k(k_norm2<S>, g, kBlock, s, n, (const S*)w.get(), red, scal.get());
                launch_k(k_gm_rotate<S>, 1, 32, s, j, m, H2.get(), cs.get(), sn2.get(), g2.get(),
                         (const double2*)scal.get(), rhs_norm, scal.get() + 1);
                last = read2(scal.get() + 1);  // (res, h_next)
                const double h_next = last.y;
                launch_k(k_gm_scale<S>, g, kBlock, s, n, h_next > 1e-30 ? 1.0 / h_next : 0.0, h_next > 1e-30 ? 0 : 1,
                         (const S*)w.get(), vcol(j + 1));
                ++j;
                ++total;
                if (last.x < tol || h_next < 1e-30) break;
            }
            launch_k(k_gm_backsolve<S>, 1, 32, s, j, m, (const double2*)H2.get(), (const double2*)g2.get(), yv.get());
            launch_k(k_gm_update<S>, g, kBlock, s, n, j, (const S*)Z.get(), (const double2*)yv.get(), d_x);
            const double2 gd = read2(g2.get() + j);
            if (std::sqrt(gd.x * gd.x + gd.y * gd.y) / rhs_norm < tol) break;
        }
    }
    SSV_CUDA(cudaStreamSynchronize(s));
    SSV_LAUNCH_CHECK();
    *iterations = total;
}

void gmres_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* d_fd, int maxiter, double tol, int restart,
                     const void* d_b, void* d_x, int* iterations) {
    if (pre && pre->vdtype != A->dtype)
        fail(SSV_ERR_TYPE, A->dtype == SSV_F64 ? "preconditioner is complex; the matrix is real"
                                               : "preconditioner is real; the matrix is complex");
    if (A->dtype == SSV_F64)
        run_gmres<double>(A, pre, d_fd, maxiter, tol, restart, static_cast<const double*>(d_b),
                          static_cast<double*>(d_x), iterations);
    else
        run_gmres<zdouble>(A, pre, d_fd, maxiter, tol, restart, static_cast<const zdouble*>(d_b),
                           static_cast<zdouble*>(d_x), iterations);
}

}  // namespace ssv
