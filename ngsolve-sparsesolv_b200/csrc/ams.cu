// ams.cu -- Compact AMS (compact_ams.hpp) and ComplexCompactAMS
// (complex_compact_ams.hpp) applied on the device.
//
// Every vector is a block of NV real columns stored row-interleaved
// ([row][column]): NV = 1 is CompactAMS on a real vector, NV = 2 is
// ComplexCompactAMS on a complex vector (Re/Im interleaved exactly as
// std::complex<double> stores them), larger NV serve several right-hand sides
// at once. One pass over a matrix row feeds all NV columns, which is the
// reference's fused Re/Im idea taken to its end (DualSpMV, FusedResidual ...).
// RECIP selects the l1 update of the fused complex operators, x += r * (1/l1)
// (complex_compact_ams.hpp:197-201, compact_amg.hpp:724-728), instead of the
// real one, x += r / l1 (compact_ams.hpp:538-540, compact_amg.hpp:654-656).
#include <algorithm>
#include <cstring>

#include "amg_setup.hpp"
#include "objects.cuh"
#include "solver_api.hpp"

namespace ssv {

// ---------------------------------------------------------------------------
// Multi-vector kernels
// ---------------------------------------------------------------------------
enum MvMode : int { MV_AX = 0, MV_RES = 1, MV_ADD = 2, MV_JAC = 3 };

template <int NV>
struct Acc {
    double a[NV];
};

template <int NV, int LANES, int MODE, bool RECIP>
__global__ void __launch_bounds__(kBlock)
k_mv_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
          const double* __restrict__ x, double* __restrict__ y, const double* __restrict__ b,
          const double* __restrict__ d, double w, const KState* st) {
    if (st && st->done) return;
    const int sub = threadIdx.x % LANES;
    const int rpb = kBlock / LANES;
    const int lane_row = (threadIdx.x & 31) / LANES;  // warp-uniform trip count
    for (int row = blockIdx.x * rpb + threadIdx.x / LANES; row - lane_row < n; row += gridDim.x * rpb) {
        const bool valid = row < n;
        double acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = 0.0;
        if (valid) {
            const int k1 = rp[row + 1];
            for (int k = rp[row] + sub; k < k1; k += LANES) {
                const double a = v[k];
                const double* xr = x + (size_t)ci[k] * NV;
                if constexpr (NV == 2) {
                    const double2 xv = *reinterpret_cast<const double2*>(xr);
                    acc[0] += a * xv.x;
                    acc[1] += a * xv.y;
                } else {
#pragma unroll
                    for (int c = 0; c < NV; ++c) acc[c] += a * xr[c];
                }
            }
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o, LANES);
        if (valid && sub == 0) {
            const size_t base = (size_t)row * NV;
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                if constexpr (MODE == MV_AX) {
                    y[base + c] = acc[c];
                } else if constexpr (MODE == MV_RES) {
                    y[base + c] = b[base + c] - acc[c];
                } else if constexpr (MODE == MV_ADD) {
                    y[base + c] += w * acc[c];
                } else {
                    const double r = b[base + c] - acc[c];
                    y[base + c] = RECIP ? x[base + c] + r * d[row] : x[base + c] + r / d[row];
                }
            }
        }
    }
}

// rx/ry/rz = Pi_{x,y,z}^T r over the shared pattern of G^T (one pass over r)
template <int NV, int LANES>
__global__ void __launch_bounds__(kBlock)
k_mv_pi_restrict(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ px,
                 const double* __restrict__ py, const double* __restrict__ pz, const double* __restrict__ r,
                 double* __restrict__ ox, double* __restrict__ oy, double* __restrict__ oz, const KState* st) {
    if (st && st->done) return;
    const int sub = threadIdx.x % LANES;
    const int rpb = kBlock / LANES;
    const int lane_row = (threadIdx.x & 31) / LANES;
    for (int row = blockIdx.x * rpb + threadIdx.x / LANES; row - lane_row < n; row += gridDim.x * rpb) {
        const bool valid = row < n;
        double ax[NV], ay[NV], az[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) ax[c] = ay[c] = az[c] = 0.0;
        if (valid)
            for (int k = rp[row] + sub; k < rp[row + 1]; k += LANES) {
                const double* rr = r + (size_t)ci[k] * NV;
                const double vx = px[k], vy = py[k], vz = pz[k];
#pragma unroll
                for (int c = 0; c < NV; ++c) {
                    const double t = rr[c];
                    ax[c] += vx * t;
                    ay[c] += vy * t;
                    az[c] += vz * t;
                }
            }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                ax[c] += __shfl_down_sync(0xffffffffu, ax[c], o, LANES);
                ay[c] += __shfl_down_sync(0xffffffffu, ay[c], o, LANES);
                az[c] += __shfl_down_sync(0xffffffffu, az[c], o, LANES);
            }
        if (valid && sub == 0)
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                ox[(size_t)row * NV + c] = ax[c];
                oy[(size_t)row * NV + c] = ay[c];
                oz[(size_t)row * NV + c] = az[c];
            }
    }
}

// x += w Pix gx; x += w Piy gy; x += w Piz gz (in this order per row, as the
// reference's three MultAdd calls) over the shared pattern of G
template <int NV, int LANES>
__global__ void __launch_bounds__(kBlock)
k_mv_pi_prolong(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ px,
                const double* __restrict__ py, const double* __restrict__ pz, const double* __restrict__ gx,
                const double* __restrict__ gy, const double* __restrict__ gz, double* __restrict__ x, double w,
                const KState* st) {
    if (st && st->done) return;
    const int sub = threadIdx.x % LANES;
    const int rpb = kBlock / LANES;
    const int lane_row = (threadIdx.x & 31) / LANES;
    for (int row = blockIdx.x * rpb + threadIdx.x / LANES; row - lane_row < n; row += gridDim.x * rpb) {
        const bool valid = row < n;
        double sx[NV], sy[NV], sz[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) sx[c] = sy[c] = sz[c] = 0.0;
        if (valid)
            for (int k = rp[row] + sub; k < rp[row + 1]; k += LANES) {
                const size_t j = (size_t)ci[k] * NV;
                const double vx = px[k], vy = py[k], vz = pz[k];
#pragma unroll
                for (int c = 0; c < NV; ++c) {
                    sx[c] += vx * gx[j + c];
                    sy[c] += vy * gy[j + c];
                    sz[c] += vz * gz[j + c];
                }
            }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                sx[c] += __shfl_down_sync(0xffffffffu, sx[c], o, LANES);
                sy[c] += __shfl_down_sync(0xffffffffu, sy[c], o, LANES);
                sz[c] += __shfl_down_sync(0xffffffffu, sz[c], o, LANES);
            }
        if (valid && sub == 0)
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                double t = x[(size_t)row * NV + c];
                t += w * sx[c];
                t += w * sy[c];
                t += w * sz[c];
                x[(size_t)row * NV + c] = t;
            }
    }
}

// x = b (/ or *) d  -- the first Jacobi sweep from x = 0
template <int NV, bool RECIP>
__global__ void k_mv_first_sweep(int n, const double* __restrict__ b, const double* __restrict__ d,
                                 double* __restrict__ x, const KState* st) {
    if (st && st->done) return;
    const int64_t total = (int64_t)n * NV;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q / NV);
        x[q] = RECIP ? b[q] * d[i] : b[q] / d[i];
    }
}

// out = mask ? in : 0
template <int NV>
__global__ void k_mv_mask_copy(int n, const double* __restrict__ in, const uint8_t* __restrict__ fd,
                               double* __restrict__ out, const KState* st) {
    if (st && st->done) return;
    const int64_t total = (int64_t)n * NV;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q / NV);
        out[q] = (!fd || fd[i]) ? in[q] : 0.0;
    }
}

// y = X b, X dense n x n row-major (coarsest pseudo-inverse); warp per row
template <int NV>
__global__ void __launch_bounds__(kBlock)
k_mv_gemv(int n, const double* __restrict__ X, const double* __restrict__ b, double* __restrict__ y,
          const KState* st) {
    if (st && st->done) return;
    const int lane = threadIdx.x & 31;
    for (int row = blockIdx.x * (kBlock / 32) + threadIdx.x / 32; row < n; row += gridDim.x * (kBlock / 32)) {
        double acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = 0.0;
        const double* xr = X + (size_t)row * n;
        for (int k = lane; k < n; k += 32) {
            const double a = xr[k];
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += a * b[(size_t)k * NV + c];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o);
        if (lane == 0)
#pragma unroll
            for (int c = 0; c < NV; ++c) y[(size_t)row * NV + c] = acc[c];
    }
}

__global__ void k_recip(int n, const double* __restrict__ a, double* __restrict__ b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = 1.0 / a[i];
}

// ---------------------------------------------------------------------------
// Device hierarchy
// ---------------------------------------------------------------------------
struct DevCsr {
    int n = 0, m = 0;
    int64_t nnz = 0;
    int lanes = 8;
    DevBuf<int> rp, ci;
    DevBuf<double> v;
    void upload(const HostCsr& A, cudaStream_t s) {
        n = A.n;
        m = A.m;
        nnz = A.nnz();
        rp.upload(A.rp.data(), A.rp.size(), s);
        ci.upload(A.ci.data(), A.ci.size(), s);
        v.upload(A.v.data(), A.v.size(), s);
        lanes = pick_lanes(n > 0 ? (double)nnz / n : 1.0);
    }
};

struct AmgDevLevel {
    DevCsr A, P, Pt;
    DevBuf<double> l1, il1;
    bool direct = false;
    DevBuf<double> X;
    DevBuf<double> b, xa, xb, r;  // NV-column work vectors of this level
};

struct AmsState {
    int nhc = 0, nh1 = 0, cycle_type = 1, num_smooth = 1, nv_alloc = 0;
    double w = 1.0;
    bool complex_form = false;
    int ndof_complex = 0;
    AmsHost host;
    DevCsr A_bc, G, Gt;
    DevBuf<double> fine_l1, fine_il1, Piv[3], Pitv[3];
    std::vector<AmgDevLevel> amg[4];
    DevBuf<double> b0, xa, xb, r, rs[4];
    DevBuf<uint8_t> fd;
    bool has_fd = false;
    std::vector<uint8_t> h_fd;
    unsigned gen = 0;
};

void ams_free(AmsState* a) { delete a; }

template <int NV, int MODE, bool RECIP>
static void mv_spmv(const DevCsr& A, const double* x, double* y, const double* b, const double* d, double w,
                    const KState* st, cudaStream_t s) {
    const int lanes = A.lanes;
    const int rpb = kBlock / lanes;
    const int grid = std::max(1, std::min((A.n + rpb - 1) / rpb, sm_count() * 8));
    switch (lanes) {
        case 2: k_mv_spmv<NV, 2, MODE, RECIP><<<grid, kBlock, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), x, y, b, d, w, st); break;
        case 4: k_mv_spmv<NV, 4, MODE, RECIP><<<grid, kBlock, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), x, y, b, d, w, st); break;
        case 8: k_mv_spmv<NV, 8, MODE, RECIP><<<grid, kBlock, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), x, y, b, d, w, st); break;
        case 16: k_mv_spmv<NV, 16, MODE, RECIP><<<grid, kBlock, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), x, y, b, d, w, st); break;
        default: k_mv_spmv<NV, 32, MODE, RECIP><<<grid, kBlock, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), x, y, b, d, w, st); break;
    }
}

template <int NV, bool RECIP>
static void first_sweep(int n, const double* b, const double* d, double* x, const KState* st, cudaStream_t s) {
    k_mv_first_sweep<NV, RECIP><<<grid_for((int64_t)n * NV, kBlock), kBlock, 0, s>>>(n, b, d, x, st);
}

// One AMG V-cycle (VCycle / DualVCycle, compact_amg.hpp:662-706,801-841) on
// level l: b -> x (x starts at zero). Returns the buffer holding x.
template <int NV, bool RECIP>
static double* vcycle(std::vector<AmgDevLevel>& L, int l, const double* b, int num_smooth, const KState* st,
                      cudaStream_t s) {
    AmgDevLevel& lv = L[l];
    const double* d = RECIP ? lv.il1.get() : lv.l1.get();
    double* cur = lv.xa.get();
    double* alt = lv.xb.get();
    auto sweep = [&](int count) {
        for (int k = 0; k < count; ++k) {
            mv_spmv<NV, MV_JAC, RECIP>(lv.A, cur, alt, b, d, 0.0, st, s);
            std::swap(cur, alt);
        }
    };
    if (l == (int)L.size() - 1) {
        if (lv.direct) {
            k_mv_gemv<NV><<<std::max(1, std::min((lv.A.n + 7) / 8, sm_count() * 4)), kBlock, 0, s>>>(
                lv.A.n, lv.X.get(), b, cur, st);
        } else {  // 10 l1-Jacobi sweeps from x = 0
            first_sweep<NV, RECIP>(lv.A.n, b, d, cur, st, s);
            sweep(9);
        }
        return cur;
    }
    // pre-smoothing from x = 0: the first sweep is x = b / l1
    first_sweep<NV, RECIP>(lv.A.n, b, d, cur, st, s);
    sweep(num_smooth - 1);
    mv_spmv<NV, MV_RES, RECIP>(lv.A, cur, lv.r.get(), b, nullptr, 0.0, st, s);
    AmgDevLevel& nx = L[l + 1];
    mv_spmv<NV, MV_AX, RECIP>(lv.Pt, lv.r.get(), nx.b.get(), nullptr, nullptr, 0.0, st, s);
    double* ec = vcycle<NV, RECIP>(L, l + 1, nx.b.get(), num_smooth, st, s);
    mv_spmv<NV, MV_ADD, RECIP>(lv.P, ec, cur, nullptr, nullptr, 1.0, st, s);
    sweep(num_smooth);
    return cur;
}

template <int NV, int LANES>
static void pi_restrict_l(const AmsState& a, const double* r, double* ox, double* oy, double* oz, const KState* st,
                          cudaStream_t s) {
    const int rpb = kBlock / LANES;
    const int grid = std::max(1, std::min((a.Gt.n + rpb - 1) / rpb, sm_count() * 8));
    k_mv_pi_restrict<NV, LANES><<<grid, kBlock, 0, s>>>(a.Gt.n, a.Gt.rp.get(), a.Gt.ci.get(), a.Pitv[0].get(),
                                                        a.Pitv[1].get(), a.Pitv[2].get(), r, ox, oy, oz, st);
}

template <int NV, int LANES>
static void pi_prolong_l(const AmsState& a, const double* gx, const double* gy, const double* gz, double* x,
                         const KState* st, cudaStream_t s) {
    const int rpb = kBlock / LANES;
    const int grid = std::max(1, std::min((a.G.n + rpb - 1) / rpb, sm_count() * 8));
    k_mv_pi_prolong<NV, LANES><<<grid, kBlock, 0, s>>>(a.G.n, a.G.rp.get(), a.G.ci.get(), a.Piv[0].get(),
                                                       a.Piv[1].get(), a.Piv[2].get(), gx, gy, gz, x, a.w, st);
}

template <int NV>
static void pi_restrict(const AmsState& a, const double* r, double* ox, double* oy, double* oz, const KState* st,
                        cudaStream_t s) {
    switch (a.Gt.lanes) {
        case 2: pi_restrict_l<NV, 2>(a, r, ox, oy, oz, st, s); break;
        case 4: pi_restrict_l<NV, 4>(a, r, ox, oy, oz, st, s); break;
        case 8: pi_restrict_l<NV, 8>(a, r, ox, oy, oz, st, s); break;
        case 16: pi_restrict_l<NV, 16>(a, r, ox, oy, oz, st, s); break;
        default: pi_restrict_l<NV, 32>(a, r, ox, oy, oz, st, s); break;
    }
}

template <int NV>
static void pi_prolong(const AmsState& a, const double* gx, const double* gy, const double* gz, double* x,
                       const KState* st, cudaStream_t s) {
    switch (a.G.lanes) {
        case 2: pi_prolong_l<NV, 2>(a, gx, gy, gz, x, st, s); break;
        case 4: pi_prolong_l<NV, 4>(a, gx, gy, gz, x, st, s); break;
        case 8: pi_prolong_l<NV, 8>(a, gx, gy, gz, x, st, s); break;
        case 16: pi_prolong_l<NV, 16>(a, gx, gy, gz, x, st, s); break;
        default: pi_prolong_l<NV, 32>(a, gx, gy, gz, x, st, s); break;
    }
}

// One AMS cycle (CompactAMS::Mult, compact_ams.hpp:136-195, or the fused
// ComplexCompactAMS::Mult, complex_compact_ams.hpp:112-154): in -> out.
template <int NV, bool RECIP>
static void ams_cycle(AmsState& a, const double* in, double* out, const KState* st, cudaStream_t s) {
    const int n = a.nhc;
    const uint8_t* fd = a.has_fd ? a.fd.get() : nullptr;
    const double* d = RECIP ? a.fine_il1.get() : a.fine_l1.get();
    double* b0 = a.b0.get();
    double* cur = a.xa.get();
    double* alt = a.xb.get();
    double* r = a.r.get();
    const int gm = grid_for((int64_t)n * NV, kBlock);
    k_mv_mask_copy<NV><<<gm, kBlock, 0, s>>>(n, in, fd, b0, st);
    bool fresh = true;  // x == 0
    auto fine_smooth = [&]() {
        for (int k = 0; k < a.num_smooth; ++k) {
            if (fresh) {
                first_sweep<NV, RECIP>(n, b0, d, cur, st, s);
                fresh = false;
            } else {
                mv_spmv<NV, MV_JAC, RECIP>(a.A_bc, cur, alt, b0, d, 0.0, st, s);
                std::swap(cur, alt);
            }
        }
    };
    auto ensure_x = [&]() {
        if (fresh) {
            SSV_CUDA(cudaMemsetAsync(cur, 0, sizeof(double) * (size_t)n * NV, s));
            fresh = false;
        }
    };
    auto gradient = [&]() {
        ensure_x();
        mv_spmv<NV, MV_RES, RECIP>(a.A_bc, cur, r, b0, nullptr, 0.0, st, s);
        mv_spmv<NV, MV_AX, RECIP>(a.Gt, r, a.rs[0].get(), nullptr, nullptr, 0.0, st, s);
        double* g = vcycle<NV, RECIP>(a.amg[0], 0, a.rs[0].get(), 1, st, s);
        mv_spmv<NV, MV_ADD, RECIP>(a.G, g, cur, nullptr, nullptr, a.w, st, s);
    };
    auto nodal = [&]() {
        ensure_x();
        mv_spmv<NV, MV_RES, RECIP>(a.A_bc, cur, r, b0, nullptr, 0.0, st, s);
        pi_restrict<NV>(a, r, a.rs[1].get(), a.rs[2].get(), a.rs[3].get(), st, s);
        double* gx = vcycle<NV, RECIP>(a.amg[1], 0, a.rs[1].get(), 1, st, s);
        double* gy = vcycle<NV, RECIP>(a.amg[2], 0, a.rs[2].get(), 1, st, s);
        double* gz = vcycle<NV, RECIP>(a.amg[3], 0, a.rs[3].get(), 1, st, s);
        pi_prolong<NV>(a, gx, gy, gz, cur, st, s);
    };
    if (a.cycle_type == 7) {
        fine_smooth(); gradient(); fine_smooth(); nodal(); fine_smooth(); gradient(); fine_smooth();
    } else {
        fine_smooth(); gradient(); nodal(); gradient(); fine_smooth();
    }
    ensure_x();
    k_mv_mask_copy<NV><<<gm, kBlock, 0, s>>>(n, cur, fd, out, st);
    SSV_LAUNCH_CHECK();
}

static HostCsr host_csr_of(const ssv_matrix* M) {
    HostCsr H;
    H.n = M->rows;
    H.m = M->cols;
    H.rp = M->h_rp;
    H.ci = M->h_ci;
    H.v.resize(M->nnz);
    SSV_CUDA(cudaMemcpy(H.v.data(), M->val.get(), sizeof(double) * M->nnz, cudaMemcpyDeviceToHost));
    return H;
}

static void upload_level_work(AmsState& a, int nv) {
    for (int s = 0; s < 4; ++s)
        for (auto& lv : a.amg[s]) {
            const size_t m = (size_t)lv.A.n * nv;
            lv.b.alloc(m);
            lv.xa.alloc(m);
            lv.xb.alloc(m);
            lv.r.alloc(m);
        }
    const size_t mh = (size_t)a.nhc * nv, m1 = (size_t)a.nh1 * nv;
    a.b0.alloc(mh);
    a.xa.alloc(mh);
    a.xb.alloc(mh);
    a.r.alloc(mh);
    for (int s = 0; s < 4; ++s) a.rs[s].alloc(m1);
    a.nv_alloc = nv;
}

// Rebuild the matrix-dependent part (RebuildMatrix) and upload it.
static void ams_rebuild(AmsState& a, const ssv_matrix* A) {
    cudaStream_t s = stream();
    HostCsr H = host_csr_of(A);
    a.host.rebuild(H, a.has_fd ? a.h_fd.data() : nullptr);
    a.A_bc.upload(a.host.A_bc, s);
    a.fine_l1.upload(a.host.fine_l1.data(), a.host.fine_l1.size(), s);
    a.fine_il1.alloc(a.nhc);
    k_recip<<<grid_for(a.nhc, kBlock), kBlock, 0, s>>>(a.nhc, a.fine_l1.get(), a.fine_il1.get());
    for (int sub = 0; sub < 4; ++sub) {
        const auto& hl = a.host.amg[sub].levels;
        a.amg[sub].clear();
        a.amg[sub].resize(hl.size());
        for (size_t l = 0; l < hl.size(); ++l) {
            AmgDevLevel& dl = a.amg[sub][l];
            dl.A.upload(hl[l].A, s);
            dl.l1.upload(hl[l].l1.data(), hl[l].l1.size(), s);
            dl.il1.alloc(hl[l].A.n);
            k_recip<<<grid_for(hl[l].A.n, kBlock), kBlock, 0, s>>>(hl[l].A.n, dl.l1.get(), dl.il1.get());
            if (l + 1 < hl.size()) {
                dl.P.upload(hl[l].P, s);
                dl.Pt.upload(hl[l].Pt, s);
            }
            dl.direct = hl[l].direct;
            if (dl.direct) dl.X.upload(hl[l].inv.data(), hl[l].inv.size(), s);
        }
    }
    SSV_LAUNCH_CHECK();
    upload_level_work(a, a.complex_form ? 2 : 1);
    ++a.gen;
    SSV_CUDA(cudaStreamSynchronize(s));
}

AmsState* ams_create(const ssv_matrix* A, const ssv_matrix* G, const uint8_t* fd, const double* cx,
                     const double* cy, const double* cz, int cycle_type, int num_smooth, double theta, double w,
                     int complex_form, int ndof_complex) {
    auto* a = new AmsState();
    try {
        cudaStream_t s = stream();
        a->nhc = A->rows;
        a->nh1 = G->cols;
        a->cycle_type = cycle_type;
        a->num_smooth = std::max(1, num_smooth);
        a->w = w;
        a->complex_form = complex_form != 0;
        a->ndof_complex = ndof_complex > 0 ? ndof_complex : A->rows;
        a->host.theta = theta;
        if (fd) {
            a->has_fd = true;
            a->h_fd.assign(fd, fd + a->nhc);
            for (auto& v : a->h_fd) v = v ? 1 : 0;
            a->fd.upload(a->h_fd.data(), a->h_fd.size(), s);
        }
        HostCsr Gh = host_csr_of(G);
        a->host.setup_geometry(Gh, cx, cy, cz);
        a->G.upload(a->host.G, s);
        a->Gt.upload(a->host.Gt, s);
        for (int d = 0; d < 3; ++d) {
            a->Piv[d].upload(a->host.Pi[d].v.data(), a->host.Pi[d].v.size(), s);
            a->Pitv[d].upload(a->host.Pit[d].v.data(), a->host.Pit[d].v.size(), s);
        }
        ams_rebuild(*a, A);
        if (a->w <= 0.0) a->w = 1.0;  // Setup (:260-262)
    } catch (...) {
        delete a;
        throw;
    }
    return a;
}

void ams_update(AmsState* a, const ssv_matrix* A) { ams_rebuild(*a, A); }

// y = M^{-1} x for the preconditioner p, stream-ordered and capturable.
template <>
void precond_apply_any<double>(ssv_precond* p, const double* x, double* y, const KState* st, cudaStream_t s) {
    if (p->kind == 1) ic_apply_dev<double>(p, x, y, st, s);
    else if (p->kind == 2) ams_cycle<1, false>(*p->ams, x, y, st, s);
    else fail(SSV_ERR_TYPE, "preconditioner is complex; the matrix is real");
}

template <>
void precond_apply_any<zdouble>(ssv_precond* p, const zdouble* x, zdouble* y, const KState* st, cudaStream_t s) {
    if (p->kind == 1) ic_apply_dev<zdouble>(p, x, y, st, s);
    else if (p->kind == 3)
        ams_cycle<2, true>(*p->ams, reinterpret_cast<const double*>(x), reinterpret_cast<double*>(y), st, s);
    else fail(SSV_ERR_TYPE, "preconditioner is real; the matrix is complex");
}

unsigned precond_generation(const ssv_precond* p) {
    if (p->kind == 1) return p->A->dtype == SSV_F64 ? p->ic_d.gen : p->ic_z.gen;
    return p->ams ? p->ams->gen : 0;
}

int ams_levels(const AmsState* a, int sub, int* sizes, int cap) {
    const auto& hl = a->host.amg[sub].levels;
    for (size_t l = 0; l < hl.size() && 2 * (int)l + 1 < cap; ++l) {
        sizes[2 * l] = hl[l].A.n;
        sizes[2 * l + 1] = hl[l].A.nnz();
    }
    return (int)hl.size();
}

}  // namespace ssv
