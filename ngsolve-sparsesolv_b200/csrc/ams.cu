// ams.cu -- Compact AMS (compact_ams.hpp) and ComplexCompactAMS
// (complex_compact_ams.hpp) applied on the device.
//
// Every vector is a block of NV real columns stored row-interleaved
// ([row][column]): NV = 1 is CompactAMS on a real vector, NV = 2 is
// ComplexCompactAMS on a complex vector (Re/Im interleaved exactly as
// std::complex<double> stores them), larger NV serve several right-hand sides
// at once (NV = 4 real, NV = 8 = four complex). One pass over a matrix row
// feeds all NV columns, which is the reference's fused Re/Im idea taken to its
// end (DualSpMV, FusedResidual ...).
// RECIP selects the l1 update of the fused complex operators, x += r * (1/l1)
// (complex_compact_ams.hpp:197-201, compact_amg.hpp:724-728), instead of the
// real one, x += r / l1 (compact_ams.hpp:538-540, compact_amg.hpp:654-656).
//
// T is the storage and arithmetic type of the four subspace AMG hierarchies:
// double is the drop-in form; float is the FP32-preconditioner form, where the
// hierarchies' matrices (A_l, P_l, P_l^T), their l1 norms and vectors are FP32
// while the fine level (A_bc, its l1 norms, the HCurl vectors, the G and Pi
// transfers) and the coarsest LDL^T solves stay FP64. The fine level cannot be
// FP32 on the systems this serves: an entry of K + 1e-6 nu M (and the iron's
// nu = 1e-3) carries its mass part below FP32 resolution, so an FP32 residual
// has no gradient-space content left and the gradient correction diverges.
// Kernels that cross between the two accumulate in FP64. The cycle's input
// and output are FP64 in both forms.

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <thread>
#include <type_traits>

#include "amg_device.hpp"
#include "amg_setup.hpp"
#include "objects.cuh"
#include "sell.cuh"
#include "solver_api.hpp"

namespace ssv {

// ---------------------------------------------------------------------------
// Multi-vector kernels
// ---------------------------------------------------------------------------
// MV_TWO: y = A [x; z] with z passed in the b slot -- columns below the row
// count read x, the rest read z at (column - rows) (the fused up-sweep
// matrix of a V-cycle level: its own right-hand side and the coarse
// correction)
enum MvMode : int { MV_AX = 0, MV_RES = 1, MV_ADD = 2, MV_JAC = 3, MV_TWO = 4 };

// One row of NV columns in the widest aligned accesses the row allows (work
// vectors come from cudaMalloc, so row r starts at r * NV * sizeof(T)).
template <int NV>
__device__ __forceinline__ void load_row(const double* __restrict__ p, double (&o)[NV]) {
    if constexpr (NV % 2 == 0) {
#pragma unroll
        for (int i = 0; i < NV / 2; ++i) {
            const double2 t = reinterpret_cast<const double2*>(p)[i];
            o[2 * i] = t.x;
            o[2 * i + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int c = 0; c < NV; ++c) o[c] = p[c];
    }
}
template <int NV>
__device__ __forceinline__ void load_row(const float* __restrict__ p, float (&o)[NV]) {
    if constexpr (NV % 4 == 0) {
#pragma unroll
        for (int i = 0; i < NV / 4; ++i) {
            const float4 t = reinterpret_cast<const float4*>(p)[i];
            o[4 * i] = t.x;
            o[4 * i + 1] = t.y;
            o[4 * i + 2] = t.z;
            o[4 * i + 3] = t.w;
        }
    } else if constexpr (NV % 2 == 0) {
#pragma unroll
        for (int i = 0; i < NV / 2; ++i) {
            const float2 t = reinterpret_cast<const float2*>(p)[i];
            o[2 * i] = t.x;
            o[2 * i + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int c = 0; c < NV; ++c) o[c] = p[c];
    }
}

template <typename A, typename B>
using wider_t = std::conditional_t<(sizeof(A) >= sizeof(B)), A, B>;

// y (op)= A x with matrix values TV, input TX, output TY; accumulation in the
// wider of TV and TX. Each LANES-wide row group handles U rows per pass of the
// row loop and issues the loads of all U rows before using any of them, so a
// warp keeps U times as many HBM requests in flight (a cold fine-level pass
// is bound by requests in flight, not by bandwidth, at U = 1). The sum of each
// row runs in the same order for every U.
template <typename TV, typename TX, typename TY, int NV, int LANES, int MODE, bool RECIP, int U = 1>
__global__ void __launch_bounds__(kBlock)
k_mv_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const TV* __restrict__ v,
          const TX* __restrict__ x, TY* __restrict__ y, const TY* __restrict__ b, const TY* __restrict__ d, TY w,
          const KState* st) {
    using TA = wider_t<TV, TX>;
    pdl_gate();
    if (st && st->done) return;
    const int sub = threadIdx.x % LANES;
    const int rpb = kBlock / LANES;
    const int lane_row = (threadIdx.x & 31) / LANES;  // warp-uniform trip count
    for (int row0 = blockIdx.x * rpb * U + threadIdx.x / LANES; row0 - lane_row < n; row0 += gridDim.x * rpb * U) {
        int kk[U], ke[U];
        TA acc[U][NV];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int row = row0 + u * rpb;
            kk[u] = row < n ? rp[row] + sub : 0;
            ke[u] = row < n ? rp[row + 1] : 0;
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[u][c] = TA(0);
        }
        while (true) {
            TA a[U];
            int col[U];
            bool any = false;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const bool on = kk[u] < ke[u];
                a[u] = on ? (TA)v[kk[u]] : TA(0);
                col[u] = on ? ci[kk[u]] : -1;
                any |= on;
            }
            if (!any) break;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (col[u] >= 0) {
                    TX xv[NV];
                    if constexpr (MODE == MV_TWO)
                        load_row<NV>(col[u] < n ? x + (size_t)col[u] * NV
                                                : reinterpret_cast<const TX*>(b) + (size_t)(col[u] - n) * NV,
                                     xv);
                    else
                        load_row<NV>(x + (size_t)col[u] * NV, xv);
#pragma unroll
                    for (int c = 0; c < NV; ++c) acc[u][c] += a[u] * (TA)xv[c];
                    kk[u] += LANES;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int o = LANES / 2; o > 0; o >>= 1)
#pragma unroll
                for (int c = 0; c < NV; ++c) acc[u][c] += __shfl_down_sync(0xffffffffu, acc[u][c], o, LANES);
            const int row = row0 + u * rpb;
            if (row < n && sub == 0) {
                const size_t base = (size_t)row * NV;
#pragma unroll
                for (int c = 0; c < NV; ++c) {
                    const TY ac = (TY)acc[u][c];
                    if constexpr (MODE == MV_AX || MODE == MV_TWO) {
                        y[base + c] = ac;
                    } else if constexpr (MODE == MV_RES) {
                        y[base + c] = b[base + c] - ac;
                    } else if constexpr (MODE == MV_ADD) {
                        y[base + c] += w * ac;
                    } else {
                        const TY r = b[base + c] - ac;
                        const TY xo = (TY)x[base + c];
                        y[base + c] = RECIP ? xo + r * d[row] : xo + r / d[row];
                    }
                }
            }
        }
    }
}

// Sliced-ELL form of the same product (FP64 values): one warp per slice of 32
// rows, slice entries stored column-major, so step k of the slice's 32 rows
// is one coalesced load of 32 values and one of 32 column indices, with no
// row-pointer load in front of them. Padding entries carry column -1 and are
// skipped. The steps go in rounds of R: the values and columns of round j+1
// are loaded before the gathers of round j are issued, so each warp keeps two
// rounds of requests in flight. With P = 2 a warp walks two neighbouring
// slices side by side (a lane per row of each), which doubles the requests a
// warp keeps in flight and halves the warp count, so a matrix of about 1.5
// waves of slices runs in one. Each row is summed in its CSR column order for
// every R and P. A slice's entry count is a multiple of 32, so the loop
// conditions are warp-uniform.
// the output of one row of a sliced-ELL product, by mode
template <typename TX, typename TY, int NV, int MODE, bool RECIP, typename TA>
__device__ __forceinline__ void sell_store(int row, const TA (&acc)[NV], const TX* __restrict__ x, TY* __restrict__ y,
                                           const TY* __restrict__ b, const TY* __restrict__ d, TY w) {
    const size_t base = (size_t)row * NV;
#pragma unroll
    for (int c = 0; c < NV; ++c) {
        const TY ac = (TY)acc[c];
        if constexpr (MODE == MV_AX || MODE == MV_TWO) {
            y[base + c] = ac;
        } else if constexpr (MODE == MV_RES) {
            y[base + c] = b[base + c] - ac;
        } else if constexpr (MODE == MV_ADD) {
            y[base + c] += w * ac;
        } else {
            const TY r = b[base + c] - ac;
            const TY xo = (TY)x[base + c];
            y[base + c] = RECIP ? xo + r * d[row] : xo + r / d[row];
        }
    }
}

template <typename TX, typename TY, int NV, int MODE, bool RECIP, int R, int P = 1>
__global__ void __launch_bounds__(kBlock)
k_sell_spmv(int slices, const int* __restrict__ off, const int* __restrict__ rows, const int* __restrict__ ci,
            const double* __restrict__ v, const TX* __restrict__ x, TY* __restrict__ y, const TY* __restrict__ b,
            const TY* __restrict__ d, TY w, const KState* st, int n) {
    using TA = wider_t<double, TX>;
    pdl_gate();
    if (st && st->done) return;
    const int lane = threadIdx.x & 31;
    const int wpb = kBlock / 32;
    for (int sl0 = (blockIdx.x * wpb + threadIdx.x / 32) * P; sl0 < slices; sl0 += gridDim.x * wpb * P) {
        int e[P], e1[P], row[P];
        TA acc[P][NV];
        double a[P][R];
        int col[P][R];
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const int sl = sl0 + q;
            const bool on = sl < slices;
            e1[q] = on ? off[sl + 1] : 0;
            e[q] = on ? off[sl] + lane : 32;  // past e1 = 0: no steps
            row[q] = on ? rows[(size_t)sl * 32 + lane] : -1;
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[q][c] = TA(0);
#pragma unroll
            for (int u = 0; u < R; ++u) {
                const int k = e[q] + 32 * u;
                a[q][u] = k < e1[q] ? v[k] : 0.0;
                col[q][u] = k < e1[q] ? ci[k] : -1;
            }
        }
        while (true) {
            bool any = false;
#pragma unroll
            for (int q = 0; q < P; ++q) any |= e[q] < e1[q];
            if (!any) break;
            double an[P][R];
            int cn[P][R];
#pragma unroll
            for (int q = 0; q < P; ++q)
#pragma unroll
                for (int u = 0; u < R; ++u) {
                    const int k = e[q] + 32 * R + 32 * u;
                    an[q][u] = k < e1[q] ? v[k] : 0.0;
                    cn[q][u] = k < e1[q] ? ci[k] : -1;
                }
#pragma unroll
            for (int q = 0; q < P; ++q)
#pragma unroll
                for (int u = 0; u < R; ++u) {
                    if (col[q][u] >= 0) {
                        TX xv[NV];
                        if constexpr (MODE == MV_TWO)  // columns past the row count read the b slot
                            load_row<NV>(col[q][u] < n ? x + (size_t)col[q][u] * NV
                                                       : reinterpret_cast<const TX*>(b) + (size_t)(col[q][u] - n) * NV,
                                         xv);
                        else
                            load_row<NV>(x + (size_t)col[q][u] * NV, xv);
#pragma unroll
                        for (int c = 0; c < NV; ++c) acc[q][c] += (TA)a[q][u] * (TA)xv[c];
                    }
                }
#pragma unroll
            for (int q = 0; q < P; ++q) {
#pragma unroll
                for (int u = 0; u < R; ++u) {
                    a[q][u] = an[q][u];
                    col[q][u] = cn[q][u];
                }
                e[q] += 32 * R;
            }
        }
#pragma unroll
        for (int q = 0; q < P; ++q)
            if (row[q] >= 0) sell_store<TX, TY, NV, MODE, RECIP>(row[q], acc[q], x, y, b, d, w);
    }
}

// Column-split form for block vectors (NV = 4 or 8): NV / 2 lanes share a
// row and each sums two of its columns, so a warp covers 32 / (NV / 2) rows of
// its slice per pass and walks the slice in NV / 2 passes. The x rows of a
// step are then gathered as 64- or 32-byte pieces of few rows instead of 32
// whole rows (a fourth of the L1 wavefronts at NV = 8, where the lane-per-row
// form is bound by the L1/TEX pipeline); the slice's values and columns are
// still read once. Each column is summed in its CSR column order, as in
// k_sell_spmv.
template <typename TX, typename TY, int NV, int MODE, bool RECIP, int R>
__global__ void __launch_bounds__(kBlock)
k_sell_spmv_cs(int slices, const int* __restrict__ off, const int* __restrict__ rows, const int* __restrict__ ci,
               const double* __restrict__ v, const TX* __restrict__ x, TY* __restrict__ y, const TY* __restrict__ b,
               const TY* __restrict__ d, TY w, const KState* st, int n) {
    static_assert(NV == 4 || NV == 8, "column-split form: 4 or 8 columns");
    constexpr int CS = 2;       // columns per lane
    constexpr int G = NV / CS;  // lanes per row
    constexpr int RP = 32 / G;  // rows per pass
    using TA = wider_t<double, TX>;
    pdl_gate();
    if (st && st->done) return;
    const int lane = threadIdx.x & 31;
    const int cg = lane % G, rl = lane / G;
    const int wpb = kBlock / 32;
    for (int sl = blockIdx.x * wpb + threadIdx.x / 32; sl < slices; sl += gridDim.x * wpb) {
        const int o0 = off[sl], e1 = off[sl + 1];
#pragma unroll 1
        for (int ps = 0; ps < G; ++ps) {
            const int t = ps * RP + rl;  // this lane's row of the slice
            const int row = rows[(size_t)sl * 32 + t];
            int e = o0 + t;
            TA acc[CS];
#pragma unroll
            for (int c = 0; c < CS; ++c) acc[c] = TA(0);
            double a[R];
            int col[R];
#pragma unroll
            for (int u = 0; u < R; ++u) {
                const int k = e + 32 * u;
                a[u] = k < e1 ? v[k] : 0.0;
                col[u] = k < e1 ? ci[k] : -1;
            }
            while (e < e1) {  // a slice's entry count is a multiple of 32: warp-uniform
                double an[R];
                int cn[R];
#pragma unroll
                for (int u = 0; u < R; ++u) {
                    const int k = e + 32 * R + 32 * u;
                    an[u] = k < e1 ? v[k] : 0.0;
                    cn[u] = k < e1 ? ci[k] : -1;
                }
#pragma unroll
                for (int u = 0; u < R; ++u) {
                    if (col[u] >= 0) {
                        TX xv[CS];
                        if constexpr (MODE == MV_TWO)  // columns past the row count read the b slot
                            load_row<CS>(col[u] < n ? x + (size_t)col[u] * NV + cg * CS
                                                    : reinterpret_cast<const TX*>(b) + (size_t)(col[u] - n) * NV +
                                                          cg * CS,
                                         xv);
                        else
                            load_row<CS>(x + (size_t)col[u] * NV + cg * CS, xv);
#pragma unroll
                        for (int c = 0; c < CS; ++c) acc[c] += (TA)a[u] * (TA)xv[c];
                    }
                }
#pragma unroll
                for (int u = 0; u < R; ++u) {
                    a[u] = an[u];
                    col[u] = cn[u];
                }
                e += 32 * R;
            }
            if (row >= 0) {
                const size_t base = (size_t)row * NV + cg * CS;
#pragma unroll
                for (int c = 0; c < CS; ++c) {
                    const TY ac = (TY)acc[c];
                    if constexpr (MODE == MV_AX || MODE == MV_TWO) {
                        y[base + c] = ac;
                    } else if constexpr (MODE == MV_RES) {
                        y[base + c] = b[base + c] - ac;
                    } else if constexpr (MODE == MV_ADD) {
                        y[base + c] += w * ac;
                    } else {
                        const TY r = b[base + c] - ac;
                        const TY xo = (TY)x[base + c];
                        y[base + c] = RECIP ? xo + r * d[row] : xo + r / d[row];
                    }
                }
            }
        }
    }
}

// Three-stage form of the one-slice product (NV <= 2): in each round the
// values and columns of round j+2 are loaded and the x entries of round j+1
// gathered before the products of round j are summed, so the gather no longer
// waits behind the column load of its own round: a warp has one HBM round
// trip per round on its critical path instead of two. Same summation order
// as k_sell_spmv.
template <typename TX, typename TY, int NV, int MODE, bool RECIP, int R>
__global__ void __launch_bounds__(kBlock)
k_sell_spmv_deep(int slices, const int* __restrict__ off, const int* __restrict__ rows, const int* __restrict__ ci,
                 const double* __restrict__ v, const TX* __restrict__ x, TY* __restrict__ y, const TY* __restrict__ b,
                 const TY* __restrict__ d, TY w, const KState* st, int n) {
    using TA = wider_t<double, TX>;
    pdl_gate();
    if (st && st->done) return;
    const int lane = threadIdx.x & 31;
    const int wpb = kBlock / 32;
    auto gather = [&](int c, TX (&o)[NV]) {
        if constexpr (MODE == MV_TWO)  // columns past the row count read the b slot
            load_row<NV>(c < n ? x + (size_t)c * NV : reinterpret_cast<const TX*>(b) + (size_t)(c - n) * NV, o);
        else
            load_row<NV>(x + (size_t)c * NV, o);
    };
    for (int sl = blockIdx.x * wpb + threadIdx.x / 32; sl < slices; sl += gridDim.x * wpb) {
        const int e1 = off[sl + 1];
        int e = off[sl] + lane;
        const int row = rows[(size_t)sl * 32 + lane];
        TA acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = TA(0);
        double a[R], an[R];
        int cn[R];
        bool on[R];
        TX xv[R][NV];
#pragma unroll
        for (int u = 0; u < R; ++u) {  // round 0: values, columns, gathers; round 1: values, columns
            const int k = e + 32 * u;
            a[u] = k < e1 ? v[k] : 0.0;
            const int c0 = k < e1 ? ci[k] : -1;
            on[u] = c0 >= 0;
            if (on[u]) gather(c0, xv[u]);
            const int k1 = k + 32 * R;
            an[u] = k1 < e1 ? v[k1] : 0.0;
            cn[u] = k1 < e1 ? ci[k1] : -1;
        }
        while (e < e1) {
            double a2[R];
            int c2[R];
#pragma unroll
            for (int u = 0; u < R; ++u) {
                const int k = e + 64 * R + 32 * u;
                a2[u] = k < e1 ? v[k] : 0.0;
                c2[u] = k < e1 ? ci[k] : -1;
            }
            TX xn[R][NV];
            bool onn[R];
#pragma unroll
            for (int u = 0; u < R; ++u) {
                onn[u] = cn[u] >= 0;
                if (onn[u]) gather(cn[u], xn[u]);
            }
#pragma unroll
            for (int u = 0; u < R; ++u)
                if (on[u])
#pragma unroll
                    for (int c = 0; c < NV; ++c) acc[c] += (TA)a[u] * (TA)xv[u][c];
#pragma unroll
            for (int u = 0; u < R; ++u) {
                a[u] = an[u];
                on[u] = onn[u];
#pragma unroll
                for (int c = 0; c < NV; ++c) xv[u][c] = xn[u][c];
                an[u] = a2[u];
                cn[u] = c2[u];
            }
            e += 32 * R;
        }
        if (row >= 0) sell_store<TX, TY, NV, MODE, RECIP>(row, acc, x, y, b, d, w);
    }
}

// rx/ry/rz = Pi_{x,y,z}^T r over the shared pattern of G^T (one pass over r);
// FP64 values and accumulation, outputs in the hierarchy type TO
template <typename TO, int NV, int LANES>
__global__ void __launch_bounds__(kBlock)
k_mv_pi_restrict(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ px,
                 const double* __restrict__ py, const double* __restrict__ pz, const double* __restrict__ r,
                 TO* __restrict__ ox, TO* __restrict__ oy, TO* __restrict__ oz, const KState* st) {
    pdl_gate();
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
                double rr[NV];
                load_row<NV>(r + (size_t)ci[k] * NV, rr);
                const double vx = px[k], vy = py[k], vz = pz[k];
#pragma unroll
                for (int c = 0; c < NV; ++c) {
                    ax[c] += vx * rr[c];
                    ay[c] += vy * rr[c];
                    az[c] += vz * rr[c];
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
                ox[(size_t)row * NV + c] = (TO)ax[c];
                oy[(size_t)row * NV + c] = (TO)ay[c];
                oz[(size_t)row * NV + c] = (TO)az[c];
            }
    }
}

// x += w Pix gx; x += w Piy gy; x += w Piz gz (in this order per row, as the
// reference's three MultAdd calls) over the shared pattern of G; x FP64,
// corrections in the hierarchy type TG, FP64 accumulation
template <typename TG, int NV, int LANES>
__global__ void __launch_bounds__(kBlock)
k_mv_pi_prolong(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ px,
                const double* __restrict__ py, const double* __restrict__ pz, const TG* __restrict__ gx,
                const TG* __restrict__ gy, const TG* __restrict__ gz, double* __restrict__ x, double w,
                const KState* st) {
    pdl_gate();
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
                TG vgx[NV], vgy[NV], vgz[NV];
                load_row<NV>(gx + j, vgx);
                load_row<NV>(gy + j, vgy);
                load_row<NV>(gz + j, vgz);
                const double vx = px[k], vy = py[k], vz = pz[k];
#pragma unroll
                for (int c = 0; c < NV; ++c) {
                    sx[c] += vx * (double)vgx[c];
                    sy[c] += vy * (double)vgy[c];
                    sz[c] += vz * (double)vgz[c];
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
template <typename T, int NV, bool RECIP>
__global__ void k_mv_first_sweep(int n, const T* __restrict__ b, const T* __restrict__ d, T* __restrict__ x,
                                 const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int64_t total = (int64_t)n * NV;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q / NV);
        x[q] = RECIP ? b[q] * d[i] : b[q] / d[i];
    }
}

// The first Jacobi sweep from x = 0 fused with the residual that follows it:
// x = b (/ or *) l1 and r = b - A x, the neighbours' x formed on the fly from
// b and l1 (the same values the two separate passes would store and read).
template <typename T, int NV, int LANES, bool RECIP>
__global__ void __launch_bounds__(kBlock)
k_mv_first_res(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
               const T* __restrict__ b, const T* __restrict__ d, T* __restrict__ x, T* __restrict__ r,
               const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int sub = threadIdx.x % LANES;
    const int rpb = kBlock / LANES;
    const int lane_row = (threadIdx.x & 31) / LANES;  // warp-uniform trip count
    for (int row = blockIdx.x * rpb + threadIdx.x / LANES; row - lane_row < n; row += gridDim.x * rpb) {
        const bool valid = row < n;
        T acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = T(0);
        if (valid) {
            const int k1 = rp[row + 1];
            for (int k = rp[row] + sub; k < k1; k += LANES) {
                const int j = ci[k];
                const T a = v[k];
                const T dj = d[j];
                T bj[NV];
                load_row<NV>(b + (size_t)j * NV, bj);
#pragma unroll
                for (int c = 0; c < NV; ++c) acc[c] += a * (RECIP ? bj[c] * dj : bj[c] / dj);
            }
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o, LANES);
        if (valid && sub == 0) {
            const size_t base = (size_t)row * NV;
            const T di = d[row];
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                const T bi = b[base + c];
                x[base + c] = RECIP ? bi * di : bi / di;
                r[base + c] = bi - acc[c];
            }
        }
    }
}

// out = mask ? in : 0, converting between the Krylov type (FP64) and the
// cycle's type at the two ends of the cycle
template <typename TI, typename TO, int NV>
__global__ void k_mv_mask_copy(int n, const TI* __restrict__ in, const uint8_t* __restrict__ fd,
                               TO* __restrict__ out, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int64_t total = (int64_t)n * NV;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q / NV);
        out[q] = (!fd || fd[i]) ? (TO)in[q] : TO(0);
    }
}

// Coarsest solve x = L^{-T} (D^+ (L^{-1} b)) (the LDL^T pseudo-inverse kept
// factored), FP64 factors and FP64 accumulation in both forms; warp per row.
// Forward part: z_i = (sum_{k<=i} Linv[i][k] b_k) / d_i, or 0 for a dropped
// pivot; z is FP64 scratch.
template <typename T, int NV>
__global__ void __launch_bounds__(kBlock)
k_mv_coarse_fwd(int n, const double* __restrict__ Li, const double* __restrict__ piv, const T* __restrict__ b,
                double* __restrict__ z, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int lane = threadIdx.x & 31;
    for (int row = blockIdx.x * (kBlock / 32) + threadIdx.x / 32; row < n; row += gridDim.x * (kBlock / 32)) {
        double acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = 0.0;
        const double* lr = Li + (size_t)row * n;
        for (int k = lane; k <= row; k += 32) {
            const double a = lr[k];
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += a * (double)b[(size_t)k * NV + c];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o);
        if (lane == 0) {
            const double d = piv[row];
#pragma unroll
            for (int c = 0; c < NV; ++c) z[(size_t)row * NV + c] = d != 0.0 ? acc[c] / d : 0.0;
        }
    }
}

// Backward part: x_i = sum_{k>=i} Linv[k][i] z_k, read from the transposed copy.
template <typename T, int NV>
__global__ void __launch_bounds__(kBlock)
k_mv_coarse_bwd(int n, const double* __restrict__ LiT, const double* __restrict__ z, T* __restrict__ x,
                const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int lane = threadIdx.x & 31;
    for (int row = blockIdx.x * (kBlock / 32) + threadIdx.x / 32; row < n; row += gridDim.x * (kBlock / 32)) {
        double acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = 0.0;
        const double* lr = LiT + (size_t)row * n;
        for (int k = row + lane; k < n; k += 32) {
            const double a = lr[k];
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += a * z[(size_t)k * NV + c];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o);
        if (lane == 0)
#pragma unroll
            for (int c = 0; c < NV; ++c) x[(size_t)row * NV + c] = (T)acc[c];
    }
}

// ---------------------------------------------------------------------------
// V-cycles in lockstep: one launch carries the same step of up to K
// hierarchies (blockIdx.y picks the hierarchy) -- the x, y and z nodal
// hierarchies of one AMS (K = 3), or the hierarchies of several AMS
// preconditioners applied together -- so K chains of small per-level
// launches become one chain with K times the work per launch. Same
// arithmetic per hierarchy as the single-hierarchy kernels above.
// ---------------------------------------------------------------------------
template <typename T, int K = 3>
struct Tri {
    int n[K];
    const int* rp[K];
    const int* ci[K];
    const T* v[K];
    const T* x[K];
    T* y[K];
    const T* b[K];
    const T* d[K];
    T* r[K];
};

template <typename T, int NV, int LANES, int MODE, bool RECIP, int K = 3>
__global__ void __launch_bounds__(kBlock)
k_mv3_spmv(Tri<T, K> t, T w, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int q = blockIdx.y;
    const int n = t.n[q];
    const int* __restrict__ rp = t.rp[q];
    const int* __restrict__ ci = t.ci[q];
    const T* __restrict__ v = t.v[q];
    const T* __restrict__ x = t.x[q];
    T* __restrict__ y = t.y[q];
    const T* __restrict__ b = t.b[q];
    const T* __restrict__ d = t.d[q];
    const int sub = threadIdx.x % LANES;
    const int rpb = kBlock / LANES;
    const int lane_row = (threadIdx.x & 31) / LANES;
    for (int row = blockIdx.x * rpb + threadIdx.x / LANES; row - lane_row < n; row += gridDim.x * rpb) {
        const bool valid = row < n;
        T acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = T(0);
        if (valid) {
            const int k1 = rp[row + 1];
            for (int k = rp[row] + sub; k < k1; k += LANES) {
                const T a = v[k];
                const int j = ci[k];
                T xv[NV];
                if constexpr (MODE == MV_TWO)
                    load_row<NV>(j < n ? x + (size_t)j * NV : b + (size_t)(j - n) * NV, xv);
                else
                    load_row<NV>(x + (size_t)j * NV, xv);
#pragma unroll
                for (int c = 0; c < NV; ++c) acc[c] += a * xv[c];
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
                if constexpr (MODE == MV_AX || MODE == MV_TWO) {
                    y[base + c] = acc[c];
                } else if constexpr (MODE == MV_ADD) {
                    y[base + c] += w * acc[c];
                } else {  // MV_JAC
                    const T rr = b[base + c] - acc[c];
                    const T xo = x[base + c];
                    y[base + c] = RECIP ? xo + rr * d[row] : xo + rr / d[row];
                }
            }
        }
    }
}

template <typename T, int NV, int LANES, bool RECIP, int K = 3>
__global__ void __launch_bounds__(kBlock)
k_mv3_first_res(Tri<T, K> t, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int q = blockIdx.y;
    const int n = t.n[q];
    const int* __restrict__ rp = t.rp[q];
    const int* __restrict__ ci = t.ci[q];
    const T* __restrict__ v = t.v[q];
    const T* __restrict__ b = t.b[q];
    const T* __restrict__ d = t.d[q];
    T* __restrict__ x = t.y[q];
    T* __restrict__ r = t.r[q];
    const int sub = threadIdx.x % LANES;
    const int rpb = kBlock / LANES;
    const int lane_row = (threadIdx.x & 31) / LANES;
    for (int row = blockIdx.x * rpb + threadIdx.x / LANES; row - lane_row < n; row += gridDim.x * rpb) {
        const bool valid = row < n;
        T acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = T(0);
        if (valid) {
            const int k1 = rp[row + 1];
            for (int k = rp[row] + sub; k < k1; k += LANES) {
                const int j = ci[k];
                const T a = v[k];
                const T dj = d[j];
                T bj[NV];
                load_row<NV>(b + (size_t)j * NV, bj);
#pragma unroll
                for (int c = 0; c < NV; ++c) acc[c] += a * (RECIP ? bj[c] * dj : bj[c] / dj);
            }
        }
#pragma unroll
        for (int o = LANES / 2; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o, LANES);
        if (valid && sub == 0) {
            const size_t base = (size_t)row * NV;
            const T di = d[row];
#pragma unroll
            for (int c = 0; c < NV; ++c) {
                const T bi = b[base + c];
                x[base + c] = RECIP ? bi * di : bi / di;
                r[base + c] = bi - acc[c];
            }
        }
    }
}

// coarsest LDL^T solves of the three hierarchies: Li/LiT/piv/cz per subspace
template <int K = 3>
struct TriCoarse {
    int n[K];
    const double* M[K];    // L^{-1} (forward) or its transpose (backward)
    const double* piv[K];
    double* cz[K];
    const void* io[K];     // forward: b (hierarchy type); backward: x output
};

template <typename T, int NV, bool FWD, int K = 3>
__global__ void __launch_bounds__(kBlock)
k_mv3_coarse(TriCoarse<K> t, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int q = blockIdx.y;
    const int n = t.n[q];
    const int lane = threadIdx.x & 31;
    for (int row = blockIdx.x * (kBlock / 32) + threadIdx.x / 32; row < n; row += gridDim.x * (kBlock / 32)) {
        double acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = 0.0;
        const double* lr = t.M[q] + (size_t)row * n;
        if constexpr (FWD) {
            const T* b = (const T*)t.io[q];
            for (int k = lane; k <= row; k += 32) {
                const double a = lr[k];
#pragma unroll
                for (int c = 0; c < NV; ++c) acc[c] += a * (double)b[(size_t)k * NV + c];
            }
        } else {
            const double* z = t.cz[q];
            for (int k = row + lane; k < n; k += 32) {
                const double a = lr[k];
#pragma unroll
                for (int c = 0; c < NV; ++c) acc[c] += a * z[(size_t)k * NV + c];
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o);
        if (lane == 0) {
            if constexpr (FWD) {
                const double dd = t.piv[q][row];
#pragma unroll
                for (int c = 0; c < NV; ++c) t.cz[q][(size_t)row * NV + c] = dd != 0.0 ? acc[c] / dd : 0.0;
            } else {
                T* x = (T*)t.io[q];
#pragma unroll
                for (int c = 0; c < NV; ++c) x[(size_t)row * NV + c] = (T)acc[c];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Dense V-cycle tails. Below a level of at most tail_rows() rows, the fused
// V-cycle from x = 0 is one fixed linear map b_l -> x_l: T = L^{-T} D^+ L^{-1}
// on the coarsest level and T_l = M_l + Q_l T_{l+1} R_l above it, where
// U_l = [M_l | Q_l] and R_l are the level's two fused products. The set-up
// forms T (FP64, dense) at the first level with at most tail_rows() rows, and
// the cycle applies it as one dense product in place of the two launches per
// level below: the same operator up to the order of the roundings, for the
// small levels where launch latency, not bytes, sets the time.
// ---------------------------------------------------------------------------
template <typename T, int K>
struct TailSet {
    int n[K];
    const double* M[K];
    const T* b[K];
    T* y[K];
};

// y = T b for K hierarchies (blockIdx.y), warp per row, FP64 accumulation
template <typename T, int NV, int K>
__global__ void __launch_bounds__(kBlock) k_tail_apply(TailSet<T, K> t, const KState* st) {
    pdl_gate();
    if (st && st->done) return;
    const int q = blockIdx.y;
    const int n = t.n[q];
    const double* __restrict__ M = t.M[q];
    const T* __restrict__ b = t.b[q];
    const int lane = threadIdx.x & 31;
    for (int row = blockIdx.x * (kBlock / 32) + threadIdx.x / 32; row < n; row += gridDim.x * (kBlock / 32)) {
        double acc[NV];
#pragma unroll
        for (int c = 0; c < NV; ++c) acc[c] = 0.0;
        const double* mr = M + (size_t)row * n;
        for (int j = lane; j < n; j += 32) {
            const double a = mr[j];
            T bv[NV];
            load_row<NV>(b + (size_t)j * NV, bv);
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += a * (double)bv[c];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int c = 0; c < NV; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o);
        if (lane == 0)
#pragma unroll
            for (int c = 0; c < NV; ++c) t.y[q][(size_t)row * NV + c] = (T)acc[c];
    }
}

template <typename T, int NV, int K>
static void tail_apply(const TailSet<T, K>& t, int parts, const KState* st, cudaStream_t s) {
    int nmax = 0;
    for (int k = 0; k < parts; ++k) nmax = std::max(nmax, t.n[k]);
    const dim3 grid(std::max(1, std::min((nmax + 7) / 8, std::max(1, sm_count() * 4 / parts))), parts);
    launch_k(k_tail_apply<T, NV, K>, grid, kBlock, s, t, st);
}

// set-up: T[i][j] = sum_{k >= max(i,j)} LiT[i][k] Li[k][j] / piv_k (0 for a
// dropped pivot), one block per row i
__global__ void k_tail_coarsest(int n, const double* __restrict__ Li, const double* __restrict__ LiT,
                                const double* __restrict__ piv, double* __restrict__ T) {
    extern __shared__ double arow[];
    const int i = blockIdx.x;
    for (int k = threadIdx.x; k < n; k += blockDim.x)
        arow[k] = (k >= i && piv[k] != 0.0) ? LiT[(size_t)i * n + k] / piv[k] : 0.0;
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double acc = 0.0;
        for (int k = max(i, j); k < n; ++k) acc += arow[k] * Li[(size_t)k * n + j];
        T[(size_t)i * n + j] = acc;
    }
}

// set-up: W = T R (T n1 x n1, R n1 x n0 given as its transpose Rt, n0 rows),
// one block per row i of T
__global__ void k_tail_w(int n1, int n0, const double* __restrict__ T, const int* __restrict__ rtp,
                         const int* __restrict__ rti, const double* __restrict__ rtv, double* __restrict__ W) {
    extern __shared__ double trow[];
    const int i = blockIdx.x;
    for (int k = threadIdx.x; k < n1; k += blockDim.x) trow[k] = T[(size_t)i * n1 + k];
    __syncthreads();
    for (int j = threadIdx.x; j < n0; j += blockDim.x) {
        double acc = 0.0;
        for (int e = rtp[j]; e < rtp[j + 1]; ++e) acc += trow[rti[e]] * rtv[e];
        W[(size_t)i * n0 + j] = acc;
    }
}

// set-up: T0 = M + Q W with U = [M | Q] (rows n0, columns n0 + n1), one
// block per row i
template <typename TV>
__global__ void k_tail_t(int n0, const int* __restrict__ up, const int* __restrict__ uci, const TV* __restrict__ uv,
                         const double* __restrict__ W, double* __restrict__ T0) {
    const int i = blockIdx.x;
    const int e0 = up[i], e1 = up[i + 1];
    for (int j = threadIdx.x; j < n0; j += blockDim.x) {
        double acc = 0.0;
        for (int e = e0; e < e1; ++e) {
            const int c = uci[e];
            const double v = (double)uv[e];
            if (c < n0) {
                if (c == j) acc += v;
            } else {
                acc += v * W[(size_t)(c - n0) * n0 + j];
            }
        }
        T0[(size_t)i * n0 + j] = acc;
    }
}

// set-up: T = (T + T^T) / 2. The V-cycle from x = 0 is a symmetric map
// (R_l^T = Q_l, M_l symmetric), which COCR's recurrence relies on; the dense
// formation rounds T[i][j] and T[j][i] along different sums, and symmetrising
// removes that difference.
__global__ void k_tail_sym(int n, double* __restrict__ T) {
    const int64_t total = (int64_t)n * n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / n), j = (int)(e % n);
        if (j <= i) continue;
        const double a = 0.5 * (T[(size_t)i * n + j] + T[(size_t)j * n + i]);
        T[(size_t)i * n + j] = a;
        T[(size_t)j * n + i] = a;
    }
}

__global__ void k_widen(int64_t n, const float* __restrict__ in, double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[i];
}

template <typename T>
static void widen_to(const T* in, int64_t n, double* out, cudaStream_t s) {
    if constexpr (std::is_same_v<T, double>) {
        if (n) SSV_CUDA(cudaMemcpyAsync(out, in, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    } else {
        if (n) k_widen<<<grid_for(n, 256), 256, 0, s>>>(n, in, out);
        SSV_LAUNCH_CHECK();
    }
}

// rows of the largest level a tail may start at (SSV_AMS_TAIL=<rows>; 0: no tails)
static int tail_rows() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("SSV_AMS_TAIL");
        v = e ? std::max(0, std::atoi(e)) : 2048;
    }
    return v;
}

// ---------------------------------------------------------------------------
// Device hierarchy
// ---------------------------------------------------------------------------
static std::vector<float> to_float(const std::vector<double>& h) { return std::vector<float>(h.begin(), h.end()); }

// A real array held in exactly one of the two forms.
struct DualVec {
    DevBuf<double> d;
    DevBuf<float> f;
    void set(const std::vector<double>& h, bool fp32, cudaStream_t s) {
        if (fp32) {
            d.release();
            const std::vector<float> t = to_float(h);
            f.upload(t.data(), t.size(), s);  // pageable source: staged before return
        } else {
            f.release();
            d.upload(h.data(), h.size(), s);
        }
    }
    // the same from a device FP64 array
    void set_dev(const double* src, size_t n, bool fp32, cudaStream_t s) {
        if (fp32) {
            d.release();
            f.alloc(std::max<size_t>(n, 1));
            d_to_float((int64_t)n, src, f.get(), s);
        } else {
            f.release();
            d.alloc(std::max<size_t>(n, 1));
            if (n) SSV_CUDA(cudaMemcpyAsync(d.get(), src, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        }
    }
    template <typename T> const T* get() const;
};
template <> inline const double* DualVec::get<double>() const { return d.get(); }
template <> inline const float* DualVec::get<float>() const { return f.get(); }

// Sliced-ELL copy (sell.cuh) of a fine-level FP64 matrix for k_sell_spmv.
struct DevSell : SellPattern {
    DevBuf<double> v;
    // the same values on the same pattern: v from the CSR values (device)
    void refresh(const double* csr_v, cudaStream_t s) { sell_gather(*this, csr_v, 1, v.get(), s); }
    // the layout built on the device from a device CSR (a_rp, a_ci, a_v)
    void build_dev(int n, int64_t nnz, const int* a_rp, const int* a_ci, const double* a_v, cudaStream_t s) {
        if (!build_pattern(n, nnz, a_rp, a_ci, s)) return;
        try {
            v.alloc((size_t)std::max<int64_t>(entries, 1));
            sell_gather(*this, a_v, 1, v.get(), s);
            SSV_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            invalidate();  // a layout without its values is no layout
            throw;
        }
    }
    void build(const HostCsr& A, cudaStream_t s) {
        invalidate();
        try {
            build_host(A, s);
        } catch (...) {
            invalidate();
            throw;
        }
    }

private:
    void build_host(const HostCsr& A, cudaStream_t s) {
        const int n = A.n;
        int slices = (n + 31) / 32;  // the members are set once everything is on the device
        std::vector<int> order(n);
        for (int i = 0; i < n; ++i) order[i] = i;
        auto len = [&](int r) { return A.rp[r + 1] - A.rp[r]; };
        for (int w0 = 0; w0 < n; w0 += kSellWindow) {
            const int w1 = std::min(n, w0 + kSellWindow);
            std::stable_sort(order.begin() + w0, order.begin() + w1, [&](int p, int q) { return len(p) > len(q); });
        }
        std::vector<int> h_off(slices + 1, 0), h_rows((size_t)slices * 32, -1);
        for (int sl = 0; sl < slices; ++sl) {
            int wmax = 0;
            for (int t = 0; t < 32 && sl * 32 + t < n; ++t) {
                const int r = order[sl * 32 + t];
                h_rows[(size_t)sl * 32 + t] = r;
                wmax = std::max(wmax, len(r));
            }
            if ((int64_t)h_off[sl] + 32 * (int64_t)wmax > (int64_t)INT32_MAX - 4096) return;  // int offsets: no copy
            h_off[sl + 1] = h_off[sl] + 32 * wmax;
        }
        const int64_t entries = h_off[slices];
        std::vector<int> h_ci((size_t)entries, -1), h_src((size_t)entries, -1);
        std::vector<double> h_v((size_t)entries, 0.0);
        for (int sl = 0; sl < slices; ++sl)
            for (int t = 0; t < 32; ++t) {
                const int r = h_rows[(size_t)sl * 32 + t];
                if (r < 0) continue;
                for (int k = 0; k < len(r); ++k) {
                    const size_t e = (size_t)h_off[sl] + 32 * (size_t)k + t;
                    h_ci[e] = A.ci[A.rp[r] + k];
                    h_v[e] = A.v[A.rp[r] + k];
                    h_src[e] = A.rp[r] + k;
                }
            }
        off.upload(h_off.data(), h_off.size(), s);
        rows.upload(h_rows.data(), h_rows.size(), s);
        ci.upload(h_ci.data(), h_ci.size(), s);
        src.upload(h_src.data(), h_src.size(), s);
        v.upload(h_v.data(), h_v.size(), s);
        SSV_CUDA(cudaStreamSynchronize(s));  // pageable sources
        this->slices = slices;
        this->entries = entries;
        pat_n = A.n;
        pat_nnz = A.nnz();
    }
};

struct DevCsr {
    int n = 0, m = 0;
    int64_t nnz = 0;
    int lanes = 8;               // from the mean row length until tuned
    int tuned[4] = {0, 0, 0, 0}; // lanes chosen by timing for NV = 1, 2, 4, 8 (0 = not tuned)
    int tuned_u[4] = {1, 1, 1, 1};  // rows per row group and pass chosen with them
    static int nv_slot(int nv) { return nv == 1 ? 0 : nv == 2 ? 1 : nv == 4 ? 2 : 3; }
    int lanes_for(int nv) const {
        const int i = nv_slot(nv);
        return tuned[i] ? tuned[i] : lanes;
    }
    int unroll_for(int nv) const { return tuned[nv_slot(nv)] ? tuned_u[nv_slot(nv)] : 1; }
    bool sell_for(int nv) const { return sell.slices > 0 && tuned_sell[nv_slot(nv)] > 0; }
    int tuned_sell[4] = {0, 0, 0, 0};  // launch shape of the sliced-ELL copy when it timed fastest (0 = CSR)
    DevBuf<int> rp, ci;
    DualVec v;
    DevSell sell;  // built for the fine-level FP64 matrices only (A_bc, G, G^T)
    void upload(const HostCsr& A, bool fp32, cudaStream_t s) {
        n = A.n;
        m = A.m;
        nnz = A.nnz();
        rp.upload(A.rp.data(), A.rp.size(), s);
        ci.upload(A.ci.data(), A.ci.size(), s);
        v.set(A.v, fp32, s);
        lanes = pick_lanes(n > 0 ? (double)nnz / n : 1.0);
    }
    template <typename T> const T* val() const { return v.get<T>(); }
};

// Work vector: raw FP64-sized storage, used as T.
struct WorkVec {
    DevBuf<double> raw;
    void alloc(size_t elems) { raw.alloc(elems); }
    template <typename T> T* as() const { return reinterpret_cast<T*>(raw.get()); }
};

struct AmgDevLevel {
    DevCsr A, P, Pt;
    DevCsr R, U;  // fused down / up matrices (fused_level; non-coarsest levels, SSV_AMS_FUSED)
    DualVec l1, il1;
    bool direct = false;
    DevBuf<double> Li, LiT, piv;  // coarsest: LDL^T factors (FP64 in both forms)
    DevBuf<double> cz;            // coarsest: FP64 scratch between the two triangular products
    DevBuf<double> tail;          // tail level: the V-cycle from here down as one dense FP64 map x = T b
    double piv_min = 1.0;         // coarsest: smallest kept |pivot| / |diagonal| of the factors held
    WorkVec b, xa, xb, r;  // NV-column work vectors of this level
};

// the level holding the hierarchy's dense tail, or -1
static int tail_level(const std::vector<AmgDevLevel>& L) {
    for (size_t l = 0; l < L.size(); ++l)
        if (L[l].tail.get()) return (int)l;
    return -1;
}

// The hierarchy as the device set-up builds it (FP64, unscaled): the input of
// the cycle's arrays in either form, kept so that a precision switch needs no
// new set-up.
struct AmsDev {
    bool on = false;                 // this state was set up on the device
    const ssv_matrix* src = nullptr;  // the HCurl matrix the fine layouts were built for
    DCsr A_bc, G, Gt, Pi[3], Pit[3];
    DevBuf<double> fine_l1;
    std::vector<DAmgLevel> amg[4];
};

struct AmsState {
    int nhc = 0, nh1 = 0, cycle_type = 1, num_smooth = 1, nv_alloc = 0;
    double w = 1.0;
    bool complex_form = false;
    bool fp32 = false;    // some subspace hierarchy in FP32
    bool grad64 = false;  // with fp32: the gradient hierarchy stays FP64, the three nodal ones FP32
    int ndof_complex = 0;
    AmsHost host;
    DevCsr A_bc, G, Gt;                          // FP64 in both forms
    DevBuf<double> fine_l1, fine_il1, Piv[3], Pitv[3];
    std::vector<AmgDevLevel> amg[4];
    DevBuf<double> b0, xa, xb, r;                // fine level, FP64
    WorkVec rs[4];                               // subspace right-hand sides, hierarchy type
    DevBuf<uint8_t> fd;
    bool has_fd = false;
    std::vector<uint8_t> h_fd;
    unsigned gen = 0;
    ForkSet forks;  // the y and z nodal V-cycles run beside the x one
    bool tri = true;  // nodal V-cycles in lockstep launches (SSV_AMS_TRI=0: three branches)
    int pi_lanes[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};  // Pi restrict / prolong lanes by NV slot (0 = untuned)
    // wall seconds of the last set-up (create, Update or precision switch):
    // total, hierarchy, fused level products, shape tuner (the rest is uploads)
    double t_total = 0, t_host = 0, t_fused = 0, t_tune = 0;
    AmsDev dev;
};

void ams_free(AmsState* a) { delete a; }

// the (lanes, rows per group and pass) shapes the tuner tries; U > 1 only where
// the matrix is large enough to fill the GPU several times over
constexpr int kShapeL[] = {2, 4, 8, 16, 32, 4, 8, 16, 8, 16};
constexpr int kShapeU[] = {1, 1, 1, 1, 1, 2, 2, 2, 4, 4};
constexpr int kShapes = 10;
constexpr int kUnrollMinRows = 65536;
// sliced-ELL launch shapes: steps per round R (2, 4, 8), | kSellPair for two
// slices per warp (R = 2, 4), | kSellDeep for the three-stage form (R = 2, 4;
// one or two columns), | kSellCols for the column-split form (R = 4, 8; four
// or eight columns)
constexpr int kSellPair = 16;
constexpr int kSellDeep = 32;
constexpr int kSellCols = 64;  // the column-split form (R = 4, 8; four or eight columns)
constexpr int kSellShapes[] = {2, 4, 8, kSellPair | 2, kSellPair | 4, kSellDeep | 2, kSellDeep | 4,
                               kSellCols | 4, kSellCols | 8};

template <typename TV, typename TX, typename TY, int NV, int MODE, bool RECIP>
static void launch_mv(int lanes, int u, int grid, cudaStream_t s, int n, const int* rp, const int* ci, const TV* v,
                      const TX* x, TY* y, const TY* b, const TY* d, TY w, const KState* st) {
#define SSV_MV_CASE(L, UU)                                                                                          \
    if (lanes == L && u == UU) {                                                                                   \
        launch_k(k_mv_spmv<TV, TX, TY, NV, L, MODE, RECIP, UU>, grid, kBlock, s, n, rp, ci, v, x, y, b, d, w, st); \
        return;                                                                                                    \
    }
    SSV_MV_CASE(2, 1)
    SSV_MV_CASE(4, 1)
    SSV_MV_CASE(8, 1)
    SSV_MV_CASE(16, 1)
    SSV_MV_CASE(4, 2)
    SSV_MV_CASE(8, 2)
    SSV_MV_CASE(16, 2)
    SSV_MV_CASE(8, 4)
    SSV_MV_CASE(16, 4)
#undef SSV_MV_CASE
    launch_k(k_mv_spmv<TV, TX, TY, NV, 32, MODE, RECIP, 1>, grid, kBlock, s, n, rp, ci, v, x, y, b, d, w, st);
}

static int mv_grid(int n, int lanes, int u) {
    const int rpb = kBlock / lanes * u;
    return std::max(1, std::min((n + rpb - 1) / rpb, sm_count() * 8));
}

template <typename TX, typename TY, int NV, int MODE, bool RECIP>
static void launch_sell(const DevSell& S, int shape, cudaStream_t s, const TX* x, TY* y, const TY* b, const TY* d,
                        TY w, const KState* st) {
    const int pairs = shape & kSellPair;  // two slices per warp
    const int per_block = (kBlock / 32) * (pairs ? 2 : 1);
    const int grid = std::max(1, (S.slices + per_block - 1) / per_block);
#define SSV_SELL_ARGS grid, kBlock, s, S.slices, S.off.get(), S.rows.get(), S.ci.get(), S.v.get(), x, y, b, d, w, st, \
                      S.pat_n
    if constexpr (NV <= 2) {
        if (shape == (kSellDeep | 2)) {
            launch_k(k_sell_spmv_deep<TX, TY, NV, MODE, RECIP, 2>, SSV_SELL_ARGS);
            return;
        }
        if (shape == (kSellDeep | 4)) {
            launch_k(k_sell_spmv_deep<TX, TY, NV, MODE, RECIP, 4>, SSV_SELL_ARGS);
            return;
        }
    }
    if constexpr (NV == 4 || NV == 8) {
        if (shape == (kSellCols | 4)) {
            launch_k(k_sell_spmv_cs<TX, TY, NV, MODE, RECIP, 4>, SSV_SELL_ARGS);
            return;
        }
        if (shape == (kSellCols | 8)) {
            launch_k(k_sell_spmv_cs<TX, TY, NV, MODE, RECIP, 8>, SSV_SELL_ARGS);
            return;
        }
    }
    shape &= ~(kSellDeep | kSellCols);  // (the three-stage and column-split forms exist for some NV only)
    if (shape == (kSellPair | 2)) launch_k(k_sell_spmv<TX, TY, NV, MODE, RECIP, 2, 2>, SSV_SELL_ARGS);
    else if (shape == (kSellPair | 4)) launch_k(k_sell_spmv<TX, TY, NV, MODE, RECIP, 4, 2>, SSV_SELL_ARGS);
    else if (shape == 2) launch_k(k_sell_spmv<TX, TY, NV, MODE, RECIP, 2>, SSV_SELL_ARGS);
    else if (shape == 4) launch_k(k_sell_spmv<TX, TY, NV, MODE, RECIP, 4>, SSV_SELL_ARGS);
    else launch_k(k_sell_spmv<TX, TY, NV, MODE, RECIP, 8>, SSV_SELL_ARGS);
#undef SSV_SELL_ARGS
}

template <typename TV, typename TX, typename TY, int NV, int MODE, bool RECIP>
static void mv_spmv(const DevCsr& A, const TX* x, TY* y, const TY* b, const TY* d, TY w, const KState* st,
                    cudaStream_t s) {
    if constexpr (std::is_same_v<TV, double>) {
        if (A.sell_for(NV)) {
            launch_sell<TX, TY, NV, MODE, RECIP>(A.sell, A.tuned_sell[DevCsr::nv_slot(NV)], s, x, y, b, d, w, st);
            return;
        }
    }
    const int lanes = A.lanes_for(NV);
    const int u = A.unroll_for(NV);
    launch_mv<TV, TX, TY, NV, MODE, RECIP>(lanes, u, mv_grid(A.n, lanes, u), s, A.n, A.rp.get(), A.ci.get(),
                                           A.val<TV>(), x, y, b, d, w, st);
}

template <typename T, int NV, bool RECIP>
static void first_sweep(int n, const T* b, const T* d, T* x, const KState* st, cudaStream_t s) {
    launch_k(k_mv_first_sweep<T, NV, RECIP>, grid_for((int64_t)n * NV, kBlock), kBlock, s, n, b, d, x, st);
}

template <typename T, int NV, bool RECIP>
static void first_res(const DevCsr& A, const T* b, const T* d, T* x, T* r, const KState* st, cudaStream_t s) {
    const int lanes = A.lanes_for(NV);
    const int rpb = kBlock / lanes;
    const int grid = std::max(1, std::min((A.n + rpb - 1) / rpb, sm_count() * 8));
    const T* v = A.val<T>();
    switch (lanes) {
        case 2: launch_k(k_mv_first_res<T, NV, 2, RECIP>, grid, kBlock, s, A.n, A.rp.get(), A.ci.get(), v, b, d, x, r, st); break;
        case 4: launch_k(k_mv_first_res<T, NV, 4, RECIP>, grid, kBlock, s, A.n, A.rp.get(), A.ci.get(), v, b, d, x, r, st); break;
        case 8: launch_k(k_mv_first_res<T, NV, 8, RECIP>, grid, kBlock, s, A.n, A.rp.get(), A.ci.get(), v, b, d, x, r, st); break;
        case 16: launch_k(k_mv_first_res<T, NV, 16, RECIP>, grid, kBlock, s, A.n, A.rp.get(), A.ci.get(), v, b, d, x, r, st); break;
        default: launch_k(k_mv_first_res<T, NV, 32, RECIP>, grid, kBlock, s, A.n, A.rp.get(), A.ci.get(), v, b, d, x, r, st); break;
    }
}

template <typename T, bool RECIP>
static const T* l1_of(const AmgDevLevel& lv) {
    return RECIP ? lv.il1.get<T>() : lv.l1.get<T>();
}

// SSV_AMS_FUSED=0: V-cycles run the four per-level passes (fused first sweep +
// residual, restriction, prolongation, post sweep) instead of the two fused
// products R and U
static bool fused_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("SSV_AMS_FUSED");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v != 0;
}

// a hierarchy the fused V-cycle can run: R and U on every non-coarsest level,
// a direct coarsest solve
static bool fused_ready(const std::vector<AmgDevLevel>& L) {
    if (L.empty() || !L.back().direct) return false;
    for (size_t l = 0; l + 1 < L.size(); ++l)
        if (L[l].U.n == 0 || L[l].R.n == 0) return false;
    return true;
}

template <typename T, int NV, bool RECIP>
static void coarse_direct(AmgDevLevel& lv, const T* b, T* x, const KState* st, cudaStream_t s) {
    const int g = std::max(1, std::min((lv.A.n + 7) / 8, sm_count() * 4));
    launch_k(k_mv_coarse_fwd<T, NV>, g, kBlock, s, lv.A.n, lv.Li.get(), lv.piv.get(), b, lv.cz.get(), st);
    launch_k(k_mv_coarse_bwd<T, NV>, g, kBlock, s, lv.A.n, lv.LiT.get(), lv.cz.get(), x, st);
}

// The V-cycle of `vcycle` (num_smooth = 1, direct coarsest) through the fused
// level matrices: the down sweep is one product b_{l+1} = R_l b_l per level,
// the up sweep one product x_l = U_l [b_l; e_{l+1}] per level -- two launches
// per level instead of four. Same arithmetic up to rounding.
template <typename T, int NV, bool RECIP>
static T* vcycle_fused(std::vector<AmgDevLevel>& L, const T* b0, const KState* st, cudaStream_t s) {
    const int tl = tail_level(L);
    const int n = tl >= 0 ? tl + 1 : (int)L.size();  // levels run one by one (the last: coarsest or tail)
    auto rhs = [&](int l) -> const T* { return l == 0 ? b0 : L[l].b.template as<T>(); };
    for (int l = 0; l + 1 < n; ++l)
        mv_spmv<T, T, T, NV, MV_AX, RECIP>(L[l].R, rhs(l), L[l + 1].b.template as<T>(), nullptr, nullptr, T(0), st,
                                           s);
    if (tl >= 0) {
        TailSet<T, 1> t{};
        t.n[0] = L[tl].A.n;
        t.M[0] = L[tl].tail.get();
        t.b[0] = rhs(tl);
        t.y[0] = L[tl].xa.template as<T>();
        tail_apply<T, NV, 1>(t, 1, st, s);
    } else {
        coarse_direct<T, NV, RECIP>(L[n - 1], rhs(n - 1), L[n - 1].xa.template as<T>(), st, s);
    }
    for (int l = n - 2; l >= 0; --l) {
        const T* e = (l + 1 == n - 1) ? L[l + 1].xa.template as<T>() : L[l + 1].xb.template as<T>();
        mv_spmv<T, T, T, NV, MV_TWO, RECIP>(L[l].U, rhs(l), L[l].xb.template as<T>(), e, nullptr, T(0), st, s);
    }
    return n == 1 ? L[0].xa.template as<T>() : L[0].xb.template as<T>();
}

// One AMG V-cycle (VCycle / DualVCycle, compact_amg.hpp:662-706,801-841) on
// level l: b -> x (x starts at zero). Returns the buffer holding x.
template <typename T, int NV, bool RECIP>
static T* vcycle(std::vector<AmgDevLevel>& L, int l, const T* b, int num_smooth, const KState* st, cudaStream_t s) {
    if (l == 0 && num_smooth == 1 && fused_ready(L)) return vcycle_fused<T, NV, RECIP>(L, b, st, s);
    AmgDevLevel& lv = L[l];
    const T* d = l1_of<T, RECIP>(lv);
    T* cur = lv.xa.as<T>();
    T* alt = lv.xb.as<T>();
    auto sweep = [&](int count) {
        for (int k = 0; k < count; ++k) {
            mv_spmv<T, T, T, NV, MV_JAC, RECIP>(lv.A, cur, alt, b, d, T(0), st, s);
            std::swap(cur, alt);
        }
    };
    if (l == (int)L.size() - 1) {
        if (lv.direct) {
            const int g = std::max(1, std::min((lv.A.n + 7) / 8, sm_count() * 4));
            launch_k(k_mv_coarse_fwd<T, NV>, g, kBlock, s, lv.A.n, lv.Li.get(), lv.piv.get(), b, lv.cz.get(), st);
            launch_k(k_mv_coarse_bwd<T, NV>, g, kBlock, s, lv.A.n, lv.LiT.get(), lv.cz.get(), cur, st);
        } else {  // 10 l1-Jacobi sweeps from x = 0
            first_sweep<T, NV, RECIP>(lv.A.n, b, d, cur, st, s);
            sweep(9);
        }
        return cur;
    }
    // pre-smoothing from x = 0: the first sweep is x = b / l1 (fused with the
    // residual when it is the only sweep)
    if (num_smooth == 1) {
        first_res<T, NV, RECIP>(lv.A, b, d, cur, lv.r.as<T>(), st, s);
    } else {
        first_sweep<T, NV, RECIP>(lv.A.n, b, d, cur, st, s);
        sweep(num_smooth - 1);
        mv_spmv<T, T, T, NV, MV_RES, RECIP>(lv.A, cur, lv.r.as<T>(), b, nullptr, T(0), st, s);
    }
    AmgDevLevel& nx = L[l + 1];
    mv_spmv<T, T, T, NV, MV_AX, RECIP>(lv.Pt, lv.r.as<T>(), nx.b.as<T>(), nullptr, nullptr, T(0), st, s);
    T* ec = vcycle<T, NV, RECIP>(L, l + 1, nx.b.as<T>(), num_smooth, st, s);
    mv_spmv<T, T, T, NV, MV_ADD, RECIP>(lv.P, ec, cur, nullptr, nullptr, T(1), st, s);
    sweep(num_smooth);
    return cur;
}

// ---- the three nodal V-cycles in lockstep --------------------------------
static bool tri_ok(const AmsState& a) {
    if (!a.tri) return false;
    for (int k = 1; k < 4; ++k) {
        if (a.amg[k].empty() || !a.amg[k].back().direct) return false;
    }
    return true;
}

template <typename T, int K>
static int parts_nmax(const Tri<T, K>& t, int parts) {
    int m = 0;
    for (int k = 0; k < parts; ++k) m = std::max(m, t.n[k]);
    return m;
}

template <typename T, int NV, int MODE, bool RECIP, int K>
static void spmv3(const Tri<T, K>& t, int parts, int lanes, T w, const KState* st, cudaStream_t s) {
    const int rpb = kBlock / lanes;
    const dim3 grid(std::max(1, std::min((parts_nmax(t, parts) + rpb - 1) / rpb, sm_count() * 8 / parts)), parts);
    switch (lanes) {
        case 2: launch_k(k_mv3_spmv<T, NV, 2, MODE, RECIP, K>, grid, kBlock, s, t, w, st); break;
        case 4: launch_k(k_mv3_spmv<T, NV, 4, MODE, RECIP, K>, grid, kBlock, s, t, w, st); break;
        case 8: launch_k(k_mv3_spmv<T, NV, 8, MODE, RECIP, K>, grid, kBlock, s, t, w, st); break;
        case 16: launch_k(k_mv3_spmv<T, NV, 16, MODE, RECIP, K>, grid, kBlock, s, t, w, st); break;
        default: launch_k(k_mv3_spmv<T, NV, 32, MODE, RECIP, K>, grid, kBlock, s, t, w, st); break;
    }
}

template <typename T, int NV, bool RECIP, int K>
static void first_res3(const Tri<T, K>& t, int parts, int lanes, const KState* st, cudaStream_t s) {
    const int rpb = kBlock / lanes;
    const dim3 grid(std::max(1, std::min((parts_nmax(t, parts) + rpb - 1) / rpb, sm_count() * 8 / parts)), parts);
    switch (lanes) {
        case 2: launch_k(k_mv3_first_res<T, NV, 2, RECIP, K>, grid, kBlock, s, t, st); break;
        case 4: launch_k(k_mv3_first_res<T, NV, 4, RECIP, K>, grid, kBlock, s, t, st); break;
        case 8: launch_k(k_mv3_first_res<T, NV, 8, RECIP, K>, grid, kBlock, s, t, st); break;
        case 16: launch_k(k_mv3_first_res<T, NV, 16, RECIP, K>, grid, kBlock, s, t, st); break;
        default: launch_k(k_mv3_first_res<T, NV, 32, RECIP, K>, grid, kBlock, s, t, st); break;
    }
}

// Hierarchies H[0..parts) (direct coarsest, num_smooth 1, level counts may
// differ) in lockstep from right-hand sides rhs0[k]; out[k] = each level 0's
// result. Every hierarchy keeps its own order of steps -- its down levels,
// its coarsest solve, its up levels -- and a launch carries the hierarchies
// that have a step at that level: the down sweep of level l those with more
// than l+1 levels, then one pair of launches for all coarsest solves, then
// the up sweep of level l those with more than l+1 levels.
template <typename T, int NV, bool RECIP, int K>
static void vcycleM(std::vector<AmgDevLevel>* const* H, const T* const* rhs0, int parts, const KState* st,
                    cudaStream_t s, T** out) {
    int Lmax = 0;
    for (int k = 0; k < parts; ++k) Lmax = std::max(Lmax, (int)H[k]->size());
    auto L = [&](int k) { return (int)H[k]->size(); };
    auto rhs = [&](int k, int l) -> const T* { return l == 0 ? rhs0[k] : (*H[k])[l].b.template as<T>(); };
    auto lv = [&](int k, int l) -> AmgDevLevel& { return (*H[k])[l]; };
    bool fused = true;
    for (int k = 0; k < parts; ++k) fused = fused && fused_ready(*H[k]);
    if (fused) {  // the dense tails end the level-by-level part (vcycle_fused)
        int lt[K];
        for (int k = 0; k < parts; ++k) lt[k] = tail_level(*H[k]);
        auto Lt = [&](int k) { return lt[k] >= 0 ? lt[k] + 1 : L(k); };
        Lmax = 0;
        for (int k = 0; k < parts; ++k) Lmax = std::max(Lmax, Lt(k));
        // a level whose products all have a chosen sliced-ELL copy (the large FP64 levels) runs
        // them one by one on it; the rest in one lockstep launch
        auto all_sell = [&](int l, bool up) {
            bool any = false;
            for (int k = 0; k < parts; ++k) {
                if (l >= Lt(k) - 1) continue;
                const DevCsr& M = up ? lv(k, l).U : lv(k, l).R;
                if (!M.sell_for(NV)) return false;
                any = true;
            }
            return any;
        };
        for (int l = 0; l < Lmax - 1; ++l) {
            if (all_sell(l, false)) {
                for (int k = 0; k < parts; ++k)
                    if (l < Lt(k) - 1)
                        mv_spmv<T, T, T, NV, MV_AX, RECIP>(lv(k, l).R, rhs(k, l), lv(k, l + 1).b.template as<T>(),
                                                           nullptr, nullptr, T(0), st, s);
                continue;
            }
            Tri<T, K> rs{};
            int q = 0, k0 = -1;
            for (int k = 0; k < parts; ++k) {
                if (l >= Lt(k) - 1) continue;
                if (k0 < 0) k0 = k;
                const DevCsr& R = lv(k, l).R;
                rs.n[q] = R.n; rs.rp[q] = R.rp.get(); rs.ci[q] = R.ci.get(); rs.v[q] = R.val<T>();
                rs.x[q] = rhs(k, l); rs.y[q] = lv(k, l + 1).b.template as<T>();
                ++q;
            }
            if (q) spmv3<T, NV, MV_AX, RECIP, K>(rs, q, lv(k0, l).R.lanes_for(NV), T(0), st, s);
        }
        {  // the last level of each: its dense tail, or the LDL^T solve of the coarsest
            TailSet<T, K> ts{};
            TriCoarse<K> f{}, b{};
            int qt = 0, qc = 0, nmax = 0;
            for (int k = 0; k < parts; ++k) {
                AmgDevLevel& v = lv(k, Lt(k) - 1);
                if (lt[k] >= 0) {
                    ts.n[qt] = v.A.n; ts.M[qt] = v.tail.get();
                    ts.b[qt] = rhs(k, Lt(k) - 1); ts.y[qt] = v.xa.template as<T>();
                    ++qt;
                } else {
                    nmax = std::max(nmax, v.A.n);
                    f.n[qc] = b.n[qc] = v.A.n;
                    f.M[qc] = v.Li.get(); b.M[qc] = v.LiT.get();
                    f.piv[qc] = b.piv[qc] = v.piv.get();
                    f.cz[qc] = b.cz[qc] = v.cz.get();
                    f.io[qc] = rhs(k, Lt(k) - 1);
                    b.io[qc] = v.xa.raw.get();
                    ++qc;
                }
            }
            if (qt) tail_apply<T, NV, K>(ts, qt, st, s);
            if (qc) {
                const dim3 grid(std::max(1, std::min((nmax + 7) / 8, std::max(1, sm_count() * 4 / qc))), qc);
                launch_k(k_mv3_coarse<T, NV, true, K>, grid, kBlock, s, f, st);
                launch_k(k_mv3_coarse<T, NV, false, K>, grid, kBlock, s, b, st);
            }
        }
        for (int l = Lmax - 2; l >= 0; --l) {
            if (all_sell(l, true)) {
                for (int k = 0; k < parts; ++k) {
                    if (l > Lt(k) - 2) continue;
                    AmgDevLevel& nx = lv(k, l + 1);
                    const T* e = (l + 1 == Lt(k) - 1) ? nx.xa.template as<T>() : nx.xb.template as<T>();
                    mv_spmv<T, T, T, NV, MV_TWO, RECIP>(lv(k, l).U, rhs(k, l), lv(k, l).xb.template as<T>(), e,
                                                        nullptr, T(0), st, s);
                }
                continue;
            }
            Tri<T, K> up{};
            int q = 0, k0 = -1;
            for (int k = 0; k < parts; ++k) {
                if (l > Lt(k) - 2) continue;
                if (k0 < 0) k0 = k;
                AmgDevLevel& v = lv(k, l);
                AmgDevLevel& nx = lv(k, l + 1);
                up.n[q] = v.U.n; up.rp[q] = v.U.rp.get(); up.ci[q] = v.U.ci.get(); up.v[q] = v.U.val<T>();
                up.x[q] = rhs(k, l);
                up.b[q] = (l + 1 == Lt(k) - 1) ? nx.xa.template as<T>() : nx.xb.template as<T>();
                up.y[q] = v.xb.template as<T>();
                ++q;
            }
            if (q) spmv3<T, NV, MV_TWO, RECIP, K>(up, q, lv(k0, l).U.lanes_for(NV), T(0), st, s);
        }
        for (int k = 0; k < parts; ++k)
            out[k] = (Lt(k) == 1) ? lv(k, 0).xa.template as<T>() : lv(k, 0).xb.template as<T>();
        return;
    }
    for (int l = 0; l < Lmax - 1; ++l) {
        Tri<T, K> fr{}, rs{};
        int q = 0, k0 = -1;
        for (int k = 0; k < parts; ++k) {
            if (l >= L(k) - 1) continue;
            if (k0 < 0) k0 = k;
            AmgDevLevel& v = lv(k, l);
            fr.n[q] = v.A.n; fr.rp[q] = v.A.rp.get(); fr.ci[q] = v.A.ci.get(); fr.v[q] = v.A.val<T>();
            fr.b[q] = rhs(k, l); fr.d[q] = l1_of<T, RECIP>(v); fr.y[q] = v.xa.as<T>(); fr.r[q] = v.r.as<T>();
            rs.n[q] = v.Pt.n; rs.rp[q] = v.Pt.rp.get(); rs.ci[q] = v.Pt.ci.get(); rs.v[q] = v.Pt.val<T>();
            rs.x[q] = v.r.as<T>(); rs.y[q] = lv(k, l + 1).b.template as<T>();
            ++q;
        }
        if (q == 0) continue;
        first_res3<T, NV, RECIP, K>(fr, q, lv(k0, l).A.lanes_for(NV), st, s);
        spmv3<T, NV, MV_AX, RECIP, K>(rs, q, lv(k0, l).Pt.lanes_for(NV), T(0), st, s);
    }
    {   // coarsest levels: LDL^T pseudo-inverse, FP64
        TriCoarse<K> f{}, b{};
        int nmax = 0;
        for (int k = 0; k < parts; ++k) {
            AmgDevLevel& v = lv(k, L(k) - 1);
            nmax = std::max(nmax, v.A.n);
            f.n[k] = b.n[k] = v.A.n;
            f.M[k] = v.Li.get(); b.M[k] = v.LiT.get();
            f.piv[k] = b.piv[k] = v.piv.get();
            f.cz[k] = b.cz[k] = v.cz.get();
            f.io[k] = rhs(k, L(k) - 1);
            b.io[k] = v.xa.raw.get();
        }
        const dim3 grid(std::max(1, std::min((nmax + 7) / 8, std::max(1, sm_count() * 4 / parts))), parts);
        launch_k(k_mv3_coarse<T, NV, true, K>, grid, kBlock, s, f, st);
        launch_k(k_mv3_coarse<T, NV, false, K>, grid, kBlock, s, b, st);
    }
    for (int l = Lmax - 2; l >= 0; --l) {
        Tri<T, K> pa{}, js{};
        int q = 0, k0 = -1;
        for (int k = 0; k < parts; ++k) {
            if (l > L(k) - 2) continue;
            if (k0 < 0) k0 = k;
            AmgDevLevel& v = lv(k, l);
            AmgDevLevel& nx = lv(k, l + 1);
            const T* e = (l + 1 == L(k) - 1) ? nx.xa.as<T>() : nx.xb.as<T>();
            pa.n[q] = v.P.n; pa.rp[q] = v.P.rp.get(); pa.ci[q] = v.P.ci.get(); pa.v[q] = v.P.val<T>();
            pa.x[q] = e; pa.y[q] = v.xa.as<T>();
            js.n[q] = v.A.n; js.rp[q] = v.A.rp.get(); js.ci[q] = v.A.ci.get(); js.v[q] = v.A.val<T>();
            js.x[q] = v.xa.as<T>(); js.y[q] = v.xb.as<T>(); js.b[q] = rhs(k, l); js.d[q] = l1_of<T, RECIP>(v);
            ++q;
        }
        if (q == 0) continue;
        spmv3<T, NV, MV_ADD, RECIP, K>(pa, q, lv(k0, l).P.lanes_for(NV), T(1), st, s);
        spmv3<T, NV, MV_JAC, RECIP, K>(js, q, lv(k0, l).A.lanes_for(NV), T(0), st, s);
    }
    for (int k = 0; k < parts; ++k)
        out[k] = (L(k) == 1) ? lv(k, 0).xa.template as<T>() : lv(k, 0).xb.template as<T>();
}

// V-cycles of subspaces 1..3 from their right-hand sides a.rs[1..3]
template <typename T, int NV, bool RECIP>
static void vcycle3(AmsState& a, const KState* st, cudaStream_t s, T* out[3]) {
    std::vector<AmgDevLevel>* H[3] = {&a.amg[1], &a.amg[2], &a.amg[3]};
    const T* rhs0[3] = {a.rs[1].as<T>(), a.rs[2].as<T>(), a.rs[3].as<T>()};
    vcycleM<T, NV, RECIP, 3>(H, rhs0, 3, st, s, out);
}

template <typename T, int NV, int LANES>
static void pi_restrict_l(const AmsState& a, const double* r, T* ox, T* oy, T* oz, const KState* st,
                          cudaStream_t s) {
    const int rpb = kBlock / LANES;
    const int grid = std::max(1, std::min((a.Gt.n + rpb - 1) / rpb, sm_count() * 8));
    launch_k(k_mv_pi_restrict<T, NV, LANES>, grid, kBlock, s, a.Gt.n, a.Gt.rp.get(), a.Gt.ci.get(), a.Pitv[0].get(),
                                                           a.Pitv[1].get(), a.Pitv[2].get(), r, ox, oy, oz, st);
}

template <typename T, int NV, int LANES>
static void pi_prolong_l(const AmsState& a, const T* gx, const T* gy, const T* gz, double* x, const KState* st,
                         cudaStream_t s) {
    const int rpb = kBlock / LANES;
    const int grid = std::max(1, std::min((a.G.n + rpb - 1) / rpb, sm_count() * 8));
    launch_k(k_mv_pi_prolong<T, NV, LANES>, grid, kBlock, s, a.G.n, a.G.rp.get(), a.G.ci.get(), a.Piv[0].get(),
                                                          a.Piv[1].get(), a.Piv[2].get(), gx, gy, gz, x, a.w, st);
}

template <typename T, int NV>
static void pi_restrict(const AmsState& a, const double* r, T* ox, T* oy, T* oz, const KState* st,
                        cudaStream_t s) {
    const int tuned = a.pi_lanes[0][DevCsr::nv_slot(NV)];
    switch (tuned ? tuned : a.Gt.lanes) {
        case 2: pi_restrict_l<T, NV, 2>(a, r, ox, oy, oz, st, s); break;
        case 4: pi_restrict_l<T, NV, 4>(a, r, ox, oy, oz, st, s); break;
        case 8: pi_restrict_l<T, NV, 8>(a, r, ox, oy, oz, st, s); break;
        case 16: pi_restrict_l<T, NV, 16>(a, r, ox, oy, oz, st, s); break;
        default: pi_restrict_l<T, NV, 32>(a, r, ox, oy, oz, st, s); break;
    }
}

template <typename T, int NV>
static void pi_prolong(const AmsState& a, const T* gx, const T* gy, const T* gz, double* x, const KState* st,
                       cudaStream_t s) {
    const int tuned = a.pi_lanes[1][DevCsr::nv_slot(NV)];
    switch (tuned ? tuned : a.G.lanes) {
        case 2: pi_prolong_l<T, NV, 2>(a, gx, gy, gz, x, st, s); break;
        case 4: pi_prolong_l<T, NV, 4>(a, gx, gy, gz, x, st, s); break;
        case 8: pi_prolong_l<T, NV, 8>(a, gx, gy, gz, x, st, s); break;
        case 16: pi_prolong_l<T, NV, 16>(a, gx, gy, gz, x, st, s); break;
        default: pi_prolong_l<T, NV, 32>(a, gx, gy, gz, x, st, s); break;
    }
}

// One AMS cycle (CompactAMS::Mult, compact_ams.hpp:136-195, or the fused
// ComplexCompactAMS::Mult, complex_compact_ams.hpp:112-154): in -> out, both
// FP64 with NV columns.
static void ams_reserve(AmsState& a, int nv);

// The work vectors of NV columns before a cycle: missing only after an
// allocation that failed; outside a capture they are allocated again here,
// inside one the cycle refuses to run (no kernel may see a released buffer).
static void ams_need_columns(AmsState& a, int nv, cudaStream_t s) {
    if (nv <= a.nv_alloc) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    SSV_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone)
        fail(SSV_ERR_RUNTIME, "AMS cycle: work vectors missing after a failed allocation (call Update())");
    ams_reserve(a, nv);
}

template <typename TG, typename TN, int NV, bool RECIP>
static void ams_cycle(AmsState& a, const double* in, double* out, const KState* st, cudaStream_t s) {
    ams_need_columns(a, NV, s);
    const int n = a.nhc;
    const uint8_t* fd = a.has_fd ? a.fd.get() : nullptr;
    const double* d = RECIP ? a.fine_il1.get() : a.fine_l1.get();
    double* b0 = a.b0.get();
    double* cur = a.xa.get();
    double* alt = a.xb.get();
    double* r = a.r.get();
    const int gm = grid_for((int64_t)n * NV, kBlock);
    launch_k(k_mv_mask_copy<double, double, NV>, gm, kBlock, s, n, in, fd, b0, st);
    // (the fused first sweep + residual is not used on the fine level: with
    // 7.4M nonzeros its second gather, of l1, costs more than the separate
    // elementwise sweep saves)
    bool fresh = true;      // x == 0
    bool deferred = false;  // a lone first sweep waiting to be fused with the next residual
    auto fine_smooth = [&]() {
        for (int k = 0; k < a.num_smooth; ++k) {
            if (fresh) {
                first_sweep<double, NV, RECIP>(n, b0, d, cur, st, s);
                fresh = false;
            } else {
                mv_spmv<double, double, double, NV, MV_JAC, RECIP>(a.A_bc, cur, alt, b0, d, 0.0, st, s);
                std::swap(cur, alt);
            }
        }
    };
    auto ensure_x = [&]() {
        if (deferred) {
            first_sweep<double, NV, RECIP>(n, b0, d, cur, st, s);
            deferred = false;
        }
        if (fresh) {
            SSV_CUDA(cudaMemsetAsync(cur, 0, sizeof(double) * (size_t)n * NV, s));
            fresh = false;
        }
    };
    auto residual = [&]() {  // r = b0 - A_bc x
        if (deferred) {
            first_res<double, NV, RECIP>(a.A_bc, b0, d, cur, r, st, s);
            deferred = false;
            return;
        }
        ensure_x();
        mv_spmv<double, double, double, NV, MV_RES, RECIP>(a.A_bc, cur, r, b0, nullptr, 0.0, st, s);
    };
    auto gradient = [&]() {
        residual();
        mv_spmv<double, double, TG, NV, MV_AX, RECIP>(a.Gt, r, a.rs[0].as<TG>(), nullptr, nullptr, TG(0), st, s);
        TG* g = vcycle<TG, NV, RECIP>(a.amg[0], 0, a.rs[0].as<TG>(), 1, st, s);
        mv_spmv<double, TG, double, NV, MV_ADD, RECIP>(a.G, g, cur, nullptr, nullptr, a.w, st, s);
    };
    auto nodal = [&]() {
        residual();
        pi_restrict<TN, NV>(a, r, a.rs[1].as<TN>(), a.rs[2].as<TN>(), a.rs[3].as<TN>(), st, s);
        TN* g3[3];
        if (tri_ok(a)) {  // one chain of launches carrying all three hierarchies
            vcycle3<TN, NV, RECIP>(a, st, s, g3);
        } else {  // the three V-cycles are independent (own hierarchies and vectors)
            a.forks.fork(s, 2);
            g3[0] = vcycle<TN, NV, RECIP>(a.amg[1], 0, a.rs[1].as<TN>(), 1, st, s);
            g3[1] = vcycle<TN, NV, RECIP>(a.amg[2], 0, a.rs[2].as<TN>(), 1, st, a.forks.side[0]);
            g3[2] = vcycle<TN, NV, RECIP>(a.amg[3], 0, a.rs[3].as<TN>(), 1, st, a.forks.side[1]);
            a.forks.join(s, 2);
        }
        pi_prolong<TN, NV>(a, g3[0], g3[1], g3[2], cur, st, s);
    };
    if (a.cycle_type == 7) {
        fine_smooth(); gradient(); fine_smooth(); nodal(); fine_smooth(); gradient(); fine_smooth();
    } else {
        fine_smooth(); gradient(); nodal(); gradient(); fine_smooth();
    }
    ensure_x();
    launch_k(k_mv_mask_copy<double, double, NV>, gm, kBlock, s, n, cur, fd, out, st);
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

// ---------------------------------------------------------------------------
// Lanes autotuner: for every CSR of the cycle and every column count in use,
// time y = A x for 2..32 lanes per row on the actual matrix (work vectors as
// operands) and keep the fastest. Runs when work vectors are (re)allocated,
// outside any capture.
// ---------------------------------------------------------------------------
// Evicts the 126 MB L2 by reading a 256 MiB buffer (allocated and zeroed on
// first use, kept until exit), which leaves L2 holding clean lines of that
// buffer: the measurements below that stand for HBM-bound passes time each
// launch after an eviction. (Writing the buffer instead leaves up to 126 MB of
// dirty lines, whose write-back the timed launch would then pay for while it
// streams its own data -- which no pass of the cycle meets in a solve, where
// the preceding passes write only vectors. SSV_PROFILE_FLUSH=write selects
// that form, for comparison.)
__global__ void k_l2_evict(const uint4* __restrict__ p, size_t n, unsigned* sink) {
    unsigned acc = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint4 v = p[i];
        acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;  // the buffer is zero: never taken, keeps the loads
}

static void l2_flush(cudaStream_t s) {
    static DevBuf<uint8_t> buf;
    static DevBuf<unsigned> sink;
    static const bool write_form = [] {
        const char* e = std::getenv("SSV_PROFILE_FLUSH");
        return e && std::strcmp(e, "write") == 0;
    }();
    static bool zeroed = false;  // each step is retried by the next call after a failure
    if (!sink.get()) sink.alloc(1);
    if (!buf.get()) {
        zeroed = false;
        buf.alloc((size_t)256 << 20);
    }
    if (!zeroed) {
        buf.zero(s);
        zeroed = true;
    }
    if (write_form) {
        SSV_CUDA(cudaMemsetAsync(buf.get(), 0, buf.size(), s));
        return;
    }
    k_l2_evict<<<sm_count() * 8, 256, 0, s>>>(reinterpret_cast<const uint4*>(buf.get()), buf.size() / 16, sink.get());
    SSV_LAUNCH_CHECK();
}

// Device time of `reps` launches: back to back (warm), or each after an L2
// flush and timed alone (cold; `median` returns reps x the median launch,
// which ranks candidate shapes with less noise than the sum).
template <typename F>
static float time_launches(F&& launch, int reps, bool cold, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1,
                           bool median = false) {
    float total = 0.f;
    if (!cold) {
        SSV_CUDA(cudaEventRecord(e0, s));
        for (int k = 0; k < reps; ++k) launch();
        SSV_CUDA(cudaEventRecord(e1, s));
        SSV_CUDA(cudaEventSynchronize(e1));
        SSV_LAUNCH_CHECK();
        SSV_CUDA(cudaEventElapsedTime(&total, e0, e1));
        return total;
    }
    float each[16];
    for (int k = 0; k < reps; ++k) {
        l2_flush(s);
        SSV_CUDA(cudaEventRecord(e0, s));
        launch();
        SSV_CUDA(cudaEventRecord(e1, s));
        SSV_CUDA(cudaEventSynchronize(e1));
        SSV_LAUNCH_CHECK();
        float ms = 0.f;
        SSV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        total += ms;
        if (k < 16) each[k] = ms;
    }
    if (median && reps <= 16) {
        std::sort(each, each + reps);
        return each[reps / 2] * reps;
    }
    return total;
}

// matrices larger than this are tuned cold (SSV_AMS_COLD_TUNE_MB, default 32;
// 0.5 and 2 measured the same cycle time at 40^3)
static double cold_tune_bytes() {
    static double v = -1.0;
    if (v < 0.0) {
        const char* e = std::getenv("SSV_AMS_COLD_TUNE_MB");
        v = (e ? std::max(0.0, std::atof(e)) : 32.0) * (1 << 20);
    }
    return v;
}

// The fine-level matrices' sliced-ELL copies (A_bc, G, G^T; SSV_AMS_SELL):
// 1 (default) = a tuner candidate beside the CSR shapes on matrices of at
// least kUnrollMinRows rows, 0 = off, 2 = always used, on any size
static int sell_mode() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("SSV_AMS_SELL");
        v = (e && (e[0] == '0' || e[0] == '2')) ? e[0] - '0' : 1;
    }
    return v;
}
static bool sell_enabled() { return sell_mode() != 0; }
// SSV_AMS_SELL_SHAPE=<shape> (one of kSellShapes): the tuner offers that
// sliced-ELL launch shape alone
static int sell_shape_forced() {
    static int v = -1;
    if (v < 0) {
        v = 0;
        if (const char* e = std::getenv("SSV_AMS_SELL_SHAPE")) {
            const int k = std::atoi(e);
            for (int c : kSellShapes)
                if (c == k) v = k;
        }
    }
    return v;
}

// largest rows-per-group the tuner may pick (SSV_AMS_MAX_UNROLL, default 4)
static int max_unroll() {
    static int v = 0;
    if (v == 0) {
        const char* e = std::getenv("SSV_AMS_MAX_UNROLL");
        v = e ? std::max(1, std::atoi(e)) : 4;
    }
    return v;
}

// Tuner record and replay. SSV_AMS_TUNE_SAVE=<file> appends every choice of
// the tuners below, in call order, one line each ("csr n nnz nv lanes rows
// sliced" / "pi dir nv lanes"); SSV_AMS_TUNE_LOAD=<file> replays such a file
// instead of timing, as long as each line names the matrix (size, nonzeros,
// columns) the tuner is at -- on the first mismatch it says so on stderr and
// times from there on. A tuning cache for repeated runs, and what keeps a
// profiled run (where every launch is serialised and the timings say nothing)
// on the shapes of the plain run it profiles.
struct TuneReplay {
    std::vector<std::vector<long long>> rows;
    size_t next = 0;
    bool live = false;
    FILE* save = nullptr;
    TuneReplay() {
        if (const char* f = std::getenv("SSV_AMS_TUNE_LOAD")) {
            if (FILE* in = std::fopen(f, "r")) {
                char kind[8];
                while (std::fscanf(in, "%7s", kind) == 1) {
                    std::vector<long long> r(1, kind[0] == 'c' ? 0 : 1);
                    const int cnt = kind[0] == 'c' ? 6 : 3;
                    long long v;
                    for (int i = 0; i < cnt && std::fscanf(in, "%lld", &v) == 1; ++i) r.push_back(v);
                    if ((int)r.size() == cnt + 1) rows.push_back(r);
                }
                std::fclose(in);
                live = !rows.empty();
            } else {
                std::fprintf(stderr, "ams tune: cannot read %s, timing instead\n", f);
            }
        }
        if (const char* f = std::getenv("SSV_AMS_TUNE_SAVE")) save = std::fopen(f, "a");
    }
    // the next recorded row if it matches `want` (kind and key fields), else stop replaying
    const std::vector<long long>* take(const std::vector<long long>& want) {
        if (!live) return nullptr;
        if (next < rows.size() && rows[next].size() >= want.size() &&
            std::equal(want.begin(), want.end(), rows[next].begin()))
            return &rows[next++];
        std::fprintf(stderr, "ams tune: replay stops at entry %zu (matrix differs), timing from here on\n", next);
        live = false;
        return nullptr;
    }
    void record(const char* line) {
        if (save) {
            std::fputs(line, save);
            std::fflush(save);
        }
    }
};
static TuneReplay& tune_replay() {
    static TuneReplay r;
    return r;
}

// Shapes already timed in this process, by matrix (rows, nonzeros, columns
// per pass, value type, kind): a later Update() of the same preconditioner,
// whose fine level and often several coarse levels keep their sizes, and the
// other preconditioners of a frequency family reuse them instead of timing
// again (SSV_AMS_TUNE_MEMO=0 times every matrix).
struct TuneMemo {
    std::mutex mu;
    std::map<std::array<long long, 6>, std::array<int, 3>> m;
    static bool on() {
        static const bool v = [] {
            const char* e = std::getenv("SSV_AMS_TUNE_MEMO");
            return !(e && e[0] == '0');
        }();
        return v;
    }
};
static TuneMemo& tune_memo() {
    static TuneMemo t;
    return t;
}

// Shapes of square level matrices are timed as residuals r = b - A x (b given),
// the form the cycle runs them in (smoothing reads the same streams); the
// transfers as y = A x.
template <typename TV, typename TX, typename TY, int NV>
static void tune_csr(DevCsr& A, const TX* x, TY* y, const TY* b, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1,
                     bool force_cold = false, bool two = false) {
    if (A.n == 0 || A.nnz == 0) return;
    if (const auto* r = tune_replay().take({0, A.n, A.nnz, NV})) {
        const int slot = DevCsr::nv_slot(NV);
        A.tuned[slot] = (int)(*r)[4];
        A.tuned_u[slot] = (int)(*r)[5];
        A.tuned_sell[slot] = (A.sell.slices > 0 && std::is_same_v<TV, double>) ? (int)(*r)[6] : 0;
        return;
    }
    const std::array<long long, 6> memo_key = {A.n, A.nnz, NV, (long long)sizeof(TV),
                                               (two ? 2 : 0) + (b ? 1 : 0) + (force_cold ? 4 : 0),
                                               A.sell.slices > 0 ? 1 : 0};
    if (TuneMemo::on()) {
        std::lock_guard<std::mutex> lk(tune_memo().mu);
        auto it = tune_memo().m.find(memo_key);
        if (it != tune_memo().m.end()) {
            const int slot = DevCsr::nv_slot(NV);
            A.tuned[slot] = it->second[0];
            A.tuned_u[slot] = it->second[1];
            A.tuned_sell[slot] = it->second[2];
            char line[128];  // the record lists every choice in call order, memo hits included
            std::snprintf(line, sizeof(line), "csr %d %lld %d %d %d %d\n", A.n, (long long)A.nnz, NV, A.tuned[slot],
                          A.tuned_u[slot], A.tuned_sell[slot]);
            tune_replay().record(line);
            return;
        }
    }
    const TV* v = A.val<TV>();
    // A matrix much larger than a quarter of L2 streams from HBM in the cycle:
    // time it cold; the rest back to back.
    const bool cold = force_cold || (double)A.nnz * (4 + sizeof(TV)) > (double)(cold_tune_bytes());
    float best = 1e30f;
    int pick = A.lanes, pick_u = 1;
    for (int i = 0; i < kShapes; ++i) {
        const int L = kShapeL[i], U = kShapeU[i];
        if (U > 1 && (A.n < kUnrollMinRows || U > max_unroll())) continue;
        const int grid = mv_grid(A.n, L, U);
        auto launch = [&] {
            if (two)
                launch_mv<TV, TX, TY, NV, MV_TWO, false>(L, U, grid, s, A.n, A.rp.get(), A.ci.get(), v, x, y, b,
                                                         nullptr, TY(0), nullptr);
            else if (b)
                launch_mv<TV, TX, TY, NV, MV_RES, false>(L, U, grid, s, A.n, A.rp.get(), A.ci.get(), v, x, y, b,
                                                         nullptr, TY(0), nullptr);
            else
                launch_mv<TV, TX, TY, NV, MV_AX, false>(L, U, grid, s, A.n, A.rp.get(), A.ci.get(), v, x, y, nullptr,
                                                        nullptr, TY(0), nullptr);
        };
        launch();
        const float ms = time_launches(launch, cold ? 5 : 4, cold, s, e0, e1, true);
        if (ms < best) {
            best = ms;
            pick = L;
            pick_u = U;
        }
    }
    A.tuned[DevCsr::nv_slot(NV)] = pick;
    A.tuned_u[DevCsr::nv_slot(NV)] = pick_u;
    const int slot = DevCsr::nv_slot(NV);
    A.tuned_sell[slot] = 0;
    float sell_best = 1e30f;
    int sell_pick = 0;
    if constexpr (std::is_same_v<TV, double>) {
        if (A.sell.slices > 0 && sell_enabled()) {
            for (int R : kSellShapes) {
                if (sell_shape_forced() && R != sell_shape_forced()) continue;
                if ((R & kSellDeep) && NV > 2) continue;
                if ((R & kSellCols) && NV != 4 && NV != 8) continue;
                auto launch = [&] {
                    if (two)
                        launch_sell<TX, TY, NV, MV_TWO, false>(A.sell, R, s, x, y, b, nullptr, TY(0), nullptr);
                    else if (b)
                        launch_sell<TX, TY, NV, MV_RES, false>(A.sell, R, s, x, y, b, nullptr, TY(0), nullptr);
                    else
                        launch_sell<TX, TY, NV, MV_AX, false>(A.sell, R, s, x, y, nullptr, nullptr, TY(0), nullptr);
                };
                launch();
                const float ms = time_launches(launch, cold ? 5 : 4, cold, s, e0, e1, true);
                if (ms < sell_best) {
                    sell_best = ms;
                    sell_pick = R;
                }
            }
            if (sell_best < best || sell_mode() == 2) A.tuned_sell[slot] = sell_pick;
        }
    }
    {
        char line[128];
        std::snprintf(line, sizeof(line), "csr %d %lld %d %d %d %d\n", A.n, (long long)A.nnz, NV, pick, pick_u,
                      A.tuned_sell[slot]);
        tune_replay().record(line);
    }
    if (TuneMemo::on()) {
        std::lock_guard<std::mutex> lk(tune_memo().mu);
        tune_memo().m[memo_key] = {pick, pick_u, A.tuned_sell[slot]};
    }
    static const bool log = std::getenv("SSV_AMS_TUNE_LOG") != nullptr;
    if (log) {
        std::fprintf(stderr, "ams tune: n=%d nnz=%lld nv=%d %s -> lanes %d rows/group %d (%.2f us)", A.n,
                     (long long)A.nnz, NV, cold ? "cold" : "warm", pick, pick_u, 1e3 * best / (cold ? 5 : 4));
        if (sell_pick)
            std::fprintf(stderr, "; sliced-ELL %d steps/round%s %.2f us%s", sell_pick & 15,
                         (sell_pick & kSellPair)   ? " two slices/warp"
                         : (sell_pick & kSellDeep) ? " three-stage"
                         : (sell_pick & kSellCols) ? " column-split"
                                                   : "",
                         1e3 * sell_best / (cold ? 5 : 4),
                         A.tuned_sell[slot] ? " -> sliced-ELL" : "");
        std::fprintf(stderr, "\n");
    }
}

// lanes of the Pi transfers (one pass over G's pattern, three coefficient
// arrays), timed cold like the other fine-level transfers
template <typename T, int NV>
static void tune_pi(AmsState& a, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    const int slot = DevCsr::nv_slot(NV);
    const int cand[5] = {2, 4, 8, 16, 32};
    T* o1 = a.rs[1].as<T>();
    T* o2 = a.rs[2].as<T>();
    T* o3 = a.rs[3].as<T>();
    for (int dir = 0; dir < 2; ++dir) {
        if (const auto* r = tune_replay().take({1, dir, NV})) {
            a.pi_lanes[dir][slot] = (int)(*r)[3];
            continue;
        }
        const std::array<long long, 6> memo_key = {-1, a.G.n, a.G.nnz, NV, (long long)sizeof(T), dir};
        if (TuneMemo::on()) {
            std::lock_guard<std::mutex> lk(tune_memo().mu);
            auto it = tune_memo().m.find(memo_key);
            if (it != tune_memo().m.end()) {
                a.pi_lanes[dir][slot] = it->second[0];
                char line[64];
                std::snprintf(line, sizeof(line), "pi %d %d %d\n", dir, NV, a.pi_lanes[dir][slot]);
                tune_replay().record(line);
                continue;
            }
        }
        float best = 1e30f;
        int pick = 0;
        for (int L : cand) {
            auto launch = [&] {
                if (dir == 0) {
                    switch (L) {
                        case 2: pi_restrict_l<T, NV, 2>(a, a.r.get(), o1, o2, o3, nullptr, s); break;
                        case 4: pi_restrict_l<T, NV, 4>(a, a.r.get(), o1, o2, o3, nullptr, s); break;
                        case 8: pi_restrict_l<T, NV, 8>(a, a.r.get(), o1, o2, o3, nullptr, s); break;
                        case 16: pi_restrict_l<T, NV, 16>(a, a.r.get(), o1, o2, o3, nullptr, s); break;
                        default: pi_restrict_l<T, NV, 32>(a, a.r.get(), o1, o2, o3, nullptr, s); break;
                    }
                } else {
                    switch (L) {
                        case 2: pi_prolong_l<T, NV, 2>(a, o1, o2, o3, a.xb.get(), nullptr, s); break;
                        case 4: pi_prolong_l<T, NV, 4>(a, o1, o2, o3, a.xb.get(), nullptr, s); break;
                        case 8: pi_prolong_l<T, NV, 8>(a, o1, o2, o3, a.xb.get(), nullptr, s); break;
                        case 16: pi_prolong_l<T, NV, 16>(a, o1, o2, o3, a.xb.get(), nullptr, s); break;
                        default: pi_prolong_l<T, NV, 32>(a, o1, o2, o3, a.xb.get(), nullptr, s); break;
                    }
                }
            };
            launch();
            const float ms = time_launches(launch, 5, true, s, e0, e1, true);
            if (ms < best) {
                best = ms;
                pick = L;
            }
        }
        a.pi_lanes[dir][slot] = pick;
        if (TuneMemo::on()) {
            std::lock_guard<std::mutex> lk(tune_memo().mu);
            tune_memo().m[memo_key] = {pick, 0, 0};
        }
        {
            char line[64];
            std::snprintf(line, sizeof(line), "pi %d %d %d\n", dir, NV, pick);
            tune_replay().record(line);
        }
        if (std::getenv("SSV_AMS_TUNE_LOG"))
            std::fprintf(stderr, "ams tune: Pi %s nv=%d cold -> lanes %d (%.2f us)\n", dir ? "prolong" : "restrict", NV,
                         pick, 1e3 * best / 5);
    }
}

// The hierarchy types of the current form: FP64 for every subspace, FP32 for
// every subspace, or the gradient hierarchy FP64 with the nodal ones FP32.
template <typename F>
static void with_forms(const AmsState& a, F&& fn) {
    if (!a.fp32) fn(double{}, double{});
    else if (a.grad64) fn(double{}, float{});
    else fn(float{}, float{});
}

template <typename T, int NV>
static void tune_levels(std::vector<AmgDevLevel>& L, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    for (size_t l = 0; l < L.size(); ++l) {
        tune_csr<T, T, T, NV>(L[l].A, L[l].xa.as<T>(), L[l].xb.as<T>(), L[l].b.as<T>(), s, e0, e1);
        if (l + 1 < L.size()) {
            tune_csr<T, T, T, NV>(L[l].P, L[l + 1].xa.as<T>(), L[l].r.as<T>(), nullptr, s, e0, e1);
            tune_csr<T, T, T, NV>(L[l].Pt, L[l].r.as<T>(), L[l + 1].b.as<T>(), nullptr, s, e0, e1);
            if (L[l].R.n) {  // fused down: b_{l+1} = R b_l; fused up: x_l = U [b_l; e]
                tune_csr<T, T, T, NV>(L[l].R, L[l].b.as<T>(), L[l + 1].b.as<T>(), nullptr, s, e0, e1);
                tune_csr<T, T, T, NV>(L[l].U, L[l].b.as<T>(), L[l].xb.as<T>(), L[l + 1].xa.as<T>(), s, e0, e1,
                                      false, true);
            }
        }
    }
}

template <typename TG, typename TN, int NV>
static void tune_all_nv(AmsState& a, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    tune_csr<double, double, double, NV>(a.A_bc, a.xa.get(), a.xb.get(), a.r.get(), s, e0, e1);
    tune_csr<double, double, TG, NV>(a.Gt, a.r.get(), a.rs[0].as<TG>(), nullptr, s, e0, e1, true);
    tune_csr<double, TG, double, NV>(a.G, a.rs[0].as<TG>(), a.xb.get(), nullptr, s, e0, e1, true);
    tune_pi<TN, NV>(a, s, e0, e1);
    tune_levels<TG, NV>(a.amg[0], s, e0, e1);
    for (int sub = 1; sub < 4; ++sub) tune_levels<TN, NV>(a.amg[sub], s, e0, e1);
}

template <typename TG, typename TN>
static void tune_lanes_t(AmsState& a, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
    if (a.complex_form) {
        tune_all_nv<TG, TN, 2>(a, s, e0, e1);
        if (a.nv_alloc >= 8) tune_all_nv<TG, TN, 8>(a, s, e0, e1);
    } else {
        tune_all_nv<TG, TN, 1>(a, s, e0, e1);
        if (a.nv_alloc >= 4) tune_all_nv<TG, TN, 4>(a, s, e0, e1);
    }
}

static void tune_lanes(AmsState& a) {
    cudaStream_t s = stream();
    cudaEvent_t e0, e1;
    SSV_CUDA(cudaEventCreate(&e0));
    SSV_CUDA(cudaEventCreate(&e1));
    with_forms(a, [&](auto g, auto n) { tune_lanes_t<decltype(g), decltype(n)>(a, s, e0, e1); });
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// Work vectors for blocks of up to nv real columns (allocation only, so the
// cycle itself never allocates and can be captured).
static void ams_reserve(AmsState& a, int nv) {
    if (nv <= a.nv_alloc) return;
    try {
        for (int s = 0; s < 4; ++s)
            for (auto& lv : a.amg[s]) {
                const size_t m = (size_t)lv.A.n * nv;
                lv.b.alloc(m);
                lv.xa.alloc(m);
                lv.xb.alloc(m);
                lv.r.alloc(m);
                if (lv.direct) lv.cz.alloc(m);
            }
        const size_t mh = (size_t)a.nhc * nv, m1 = (size_t)a.nh1 * nv;
        a.b0.alloc(mh);
        a.xa.alloc(mh);
        a.xb.alloc(mh);
        a.r.alloc(mh);
        for (int s = 0; s < 4; ++s) a.rs[s].alloc(m1);
    } catch (...) {
        // some buffers were released and not replaced: no column count is
        // usable until a later reserve succeeds
        a.nv_alloc = 0;
        ++a.gen;
        throw;
    }
    a.nv_alloc = nv;
    ++a.gen;  // new work buffers: graphs that captured the old ones must be rebuilt
    const double t0 = wall_seconds();
    tune_lanes(a);
    a.t_tune += wall_seconds() - t0;
    {
        const char* e = std::getenv("SSV_AMS_TRI");
        a.tri = !(e && e[0] == '0');
    }
}

static std::vector<double> reciprocal(const std::vector<double>& v) {
    std::vector<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i) r[i] = 1.0 / v[i];
    return r;
}

// Uploads a fine-level FP64 matrix (A_bc, G, G^T) and, where the shape tuner
// may use it, its sliced-ELL copy.
static void upload_fine(DevCsr& M, const HostCsr& H, cudaStream_t s) {
    M.upload(H, false, s);
    if (sell_mode() == 2 || (sell_mode() == 1 && M.n >= kUnrollMinRows)) M.sell.build(H, s);
}

// Geometry part (G, G^T, Pi): FP64 in both forms. (The FP32 form replaces
// the values by scaled ones in ams_upload_matrix.)
static void ams_upload_geometry(AmsState& a, cudaStream_t s) {
    upload_fine(a.G, a.host.G, s);
    upload_fine(a.Gt, a.host.Gt, s);
    for (int d = 0; d < 3; ++d) {
        a.Piv[d].upload(a.host.Pi[d].v.data(), a.host.Pi[d].v.size(), s);
        a.Pitv[d].upload(a.host.Pit[d].v.data(), a.host.Pit[d].v.size(), s);
    }
}

// ---------------------------------------------------------------------------
// FP32 form: every subspace hierarchy is stored diagonally scaled,
// A^_l = S_l^{-1} A_l S_l^{-1} with s_i = sqrt|a_ii| (1 for a zero diagonal),
// P^_l = S_l P_l S_{l+1}^{-1}, P^_l^T its transpose, l1^ = l1 / s^2, the
// coarsest factors L^{-1} -> S^{-1} L^{-1} S and D -> S^{-1} D S^{-1} (the
// same pivots dropped), and the level-0 scaling folded into the transfers
// (G^T and Pi^T rows times 1/s, G and Pi columns times 1/s). In exact
// arithmetic this is the same cycle; in FP32 every row is stored and
// rounded relative to its own scale, which the eddy-current hierarchies
// (conductor |omega| sigma M next to the 1e-6 mass weight of air: diagonals
// 13 decades apart) need.
// ---------------------------------------------------------------------------
static std::vector<double> diag_scale(const HostCsr& A) {
    std::vector<double> sc(A.n, 1.0);
    for (int i = 0; i < A.n; ++i)
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
            if (A.ci[k] == i && A.v[k] != 0.0) sc[i] = std::sqrt(std::fabs(A.v[k]));
    return sc;
}

// v_k *= rmul[row] * cmul[col] (either may be null = 1)
static HostCsr scaled_csr(const HostCsr& A, const std::vector<double>* rmul, const std::vector<double>* cmul) {
    HostCsr B = A;
    for (int i = 0; i < A.n; ++i)
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
            double f = 1.0;
            if (rmul) f *= (*rmul)[i];
            if (cmul) f *= (*cmul)[A.ci[k]];
            B.v[k] = A.v[k] * f;
        }
    return B;
}

static std::vector<double> inverted(const std::vector<double>& v) {
    std::vector<double> r(v.size());
    for (size_t i = 0; i < v.size(); ++i) r[i] = 1.0 / v[i];
    return r;
}

// whether subspace sub's hierarchy is held in FP32 (diagonally scaled)
static bool sub_lo(const AmsState& a, int sub) { return a.fp32 && !(a.grad64 && sub == 0); }

// Coarsest factors of an FP32 hierarchy. Its solve reads FP32 right-hand
// sides, whose rounding (6e-8 relative) a kept pivot of relative size rho =
// |d_j| / |a_jj| amplifies by 1/rho along that pivot's direction. The
// reference's factorization keeps every pivot above 1e-13 of its diagonal, so
// a near-null mode (rho 1e-13..1e-9: the nodal hierarchies that are one level
// deep, whose coarsest matrix is the subspace's fine Galerkin matrix) turns
// one FP32 rounding into an O(1) error of the correction, and COCR diverges
// (the FP64 form is unaffected: its inputs round at 1e-16). Such a matrix is
// factored again with pivots at or below kLoPivotDrop of their diagonal
// dropped (their direction is left to the other subspaces, as a dropped
// pivot of the reference's). Out: the factors of the FP32 form, unscaled.
constexpr double kLoPivotDrop = 1e-6;

static double lo_coarse_factors(const HostCsr& A, double piv_min, const std::vector<double>& linv,
                                const std::vector<double>& linvt, const std::vector<double>& piv,
                                std::vector<double>& li, std::vector<double>& lt, std::vector<double>& pv) {
    if (piv_min > kLoPivotDrop) {
        li = linv;
        lt = linvt;
        pv = piv;
        return piv_min;
    }
    return dense_ldlt_pseudo(A, li, lt, pv, kLoPivotDrop);
}

// The dense tail of one hierarchy (see k_tail_apply) from its fused level
// products (values TV, as the cycle holds them) and its coarsest factors: none
// unless every level above the coarsest has R and U and some level has at
// most tail_rows() rows.
constexpr double kTailPivot = 1e-6;

template <typename TV>
static void build_tail(std::vector<AmgDevLevel>& L, cudaStream_t s) {
    for (auto& lv : L) lv.tail.release();
    const int rows = tail_rows();
    // an explicit inverse of a coarsest matrix with a kept pivot of relative size
    // rho carries entries of size 1/rho, whose rounding (1e-16 / rho relative)
    // the factored solve does not have: no tail below kTailPivot. (Holding such
    // near-null modes apart in factored form, T = T_reg + sum u w^T / d, was
    // measured on the 64^3 gradient hierarchy: 2% faster cycles, but COCR then
    // ended at a true residual of 2e-9 instead of 1.4e-10.)
    if (rows <= 0 || !fused_ready(L) || L.back().piv_min < kTailPivot) return;
    const int nl = (int)L.size();
    int cut = -1;
    for (int l = 0; l < nl; ++l)
        if (L[l].A.n <= rows) {
            cut = l;
            break;
        }
    if (cut < 0) return;
    const AmgDevLevel& co = L[nl - 1];
    const int nc = co.A.n;
    DevBuf<double> T((size_t)std::max(nc, 1) * std::max(nc, 1));
    if (nc)
        k_tail_coarsest<<<nc, 256, sizeof(double) * nc, s>>>(nc, co.Li.get(), co.LiT.get(), co.piv.get(), T.get());
    SSV_LAUNCH_CHECK();
    for (int l = nl - 2; l >= cut; --l) {
        const int n0 = L[l].A.n, n1 = L[l + 1].A.n;
        const DevCsr& R = L[l].R;
        DCsr Rd, Rt;
        Rd.n = R.n;
        Rd.m = R.m;
        Rd.nnz = R.nnz;
        Rd.rp.alloc(R.n + 1);
        Rd.ci.alloc(std::max<int64_t>(R.nnz, 1));
        Rd.v.alloc(std::max<int64_t>(R.nnz, 1));
        SSV_CUDA(cudaMemcpyAsync(Rd.rp.get(), R.rp.get(), sizeof(int) * (R.n + 1), cudaMemcpyDeviceToDevice, s));
        if (R.nnz) SSV_CUDA(cudaMemcpyAsync(Rd.ci.get(), R.ci.get(), sizeof(int) * R.nnz, cudaMemcpyDeviceToDevice, s));
        widen_to<TV>(R.val<TV>(), R.nnz, Rd.v.get(), s);
        d_transpose(Rd, Rt, s);
        DevBuf<double> W((size_t)std::max(n1, 1) * std::max(n0, 1)), T0((size_t)std::max(n0, 1) * std::max(n0, 1));
        if (n1 && n0)
            k_tail_w<<<n1, 256, sizeof(double) * n1, s>>>(n1, n0, T.get(), Rt.rp.get(), Rt.ci.get(), Rt.v.get(),
                                                           W.get());
        if (n0)
            k_tail_t<TV><<<n0, 256, 0, s>>>(n0, L[l].U.rp.get(), L[l].U.ci.get(), L[l].U.val<TV>(), W.get(), T0.get());
        SSV_LAUNCH_CHECK();
        SSV_CUDA(cudaStreamSynchronize(s));  // this level's temporaries go out of scope
        T = std::move(T0);
    }
    if (L[cut].A.n)
        k_tail_sym<<<grid_for((int64_t)L[cut].A.n * L[cut].A.n, 256), 256, 0, s>>>(L[cut].A.n, T.get());
    SSV_LAUNCH_CHECK();
    SSV_CUDA(cudaStreamSynchronize(s));
    L[cut].tail = std::move(T);
}

static void build_tails(AmsState& a, cudaStream_t s) {
    SetupLog log(s);
    for (int sub = 0; sub < 4; ++sub) {
        if (a.num_smooth != 1) {
            for (auto& lv : a.amg[sub]) lv.tail.release();
            continue;
        }
        if (sub_lo(a, sub)) build_tail<float>(a.amg[sub], s);
        else build_tail<double>(a.amg[sub], s);
        const int tl = tail_level(a.amg[sub]);
        if (tl >= 0)
            log.mark("  subspace %d: dense tail at level %d (%d rows, %zu levels below)", sub, tl, a.amg[sub][tl].A.n,
                     a.amg[sub].size() - 1 - tl);
        else
            log.mark("  subspace %d: no dense tail (coarsest pivot ratio %.1e)", sub,
                     a.amg[sub].empty() ? 0.0 : a.amg[sub].back().piv_min);
    }
}

// Matrix part: A_bc and its l1 norms (FP64), the four AMG hierarchies (in the
// chosen form; the coarsest factors FP64), and in the FP32 form the scaled
// transfer values.
static void ams_upload_matrix(AmsState& a, cudaStream_t s) {
    const int nv = std::max(a.nv_alloc, a.complex_form ? 2 : 1);
    upload_fine(a.A_bc, a.host.A_bc, s);
    a.fine_l1.upload(a.host.fine_l1.data(), a.host.fine_l1.size(), s);
    const std::vector<double> il1 = reciprocal(a.host.fine_l1);
    a.fine_il1.upload(il1.data(), il1.size(), s);
    // fused down / up matrices of every non-coarsest level, from the matrices in
    // the form the device holds them (diagonally scaled in the FP32 form); the
    // subspaces on their own host threads. In the FP32 form only the three
    // nodal hierarchies take them: fused in FP32, the gradient hierarchy costs
    // the preconditioner its quality (144 instead of 34 PCG iterations on the
    // 40^3 magnetostatic system; with every hierarchy fused, no convergence in
    // 500), while the fused nodal ones change nothing (34).
    std::vector<FusedLevel> fused[4];
    const double tf0 = wall_seconds();
    if (fused_enabled()) {
        run_threads(4, [&a, &fused](int sub) {
                if (sub_lo(a, sub) && sub == 0) return;  // FP32 gradient hierarchies keep the four passes
                const bool lo = sub_lo(a, sub);
                const auto& hl = a.host.amg[sub].levels;
                fused[sub].resize(hl.empty() ? 0 : hl.size() - 1);
                std::vector<std::vector<double>> sc(hl.size()), isc(hl.size());
                if (lo)
                    for (size_t l = 0; l < hl.size(); ++l) {
                        sc[l] = diag_scale(hl[l].A);
                        isc[l] = inverted(sc[l]);
                    }
                for (size_t l = 0; l + 1 < hl.size(); ++l) {
                    if (!lo) {
                        fused[sub][l] = fused_level(hl[l].A, hl[l].P, hl[l].Pt, hl[l].l1);
                        continue;
                    }
                    std::vector<double> l1s(hl[l].A.n);
                    for (int i = 0; i < hl[l].A.n; ++i) l1s[i] = hl[l].l1[i] * isc[l][i] * isc[l][i];
                    fused[sub][l] =
                        fused_level(scaled_csr(hl[l].A, &isc[l], &isc[l]), scaled_csr(hl[l].P, &sc[l], &isc[l + 1]),
                                    scaled_csr(hl[l].Pt, &isc[l + 1], &sc[l]), l1s);
                }
        });
    }
    a.t_fused = wall_seconds() - tf0;
    for (int sub = 0; sub < 4; ++sub) {
        const bool lo = sub_lo(a, sub);
        const auto& hl = a.host.amg[sub].levels;
        a.amg[sub].clear();
        a.amg[sub].resize(hl.size());
        std::vector<std::vector<double>> sc(hl.size()), isc(hl.size());
        for (size_t l = 0; l < hl.size(); ++l) {
            sc[l] = lo ? diag_scale(hl[l].A) : std::vector<double>(hl[l].A.n, 1.0);
            isc[l] = inverted(sc[l]);
        }
        for (size_t l = 0; l < hl.size(); ++l) {
            AmgDevLevel& dl = a.amg[sub][l];
            const int nl = hl[l].A.n;
            if (lo) {
                dl.A.upload(scaled_csr(hl[l].A, &isc[l], &isc[l]), true, s);
                std::vector<double> l1s(nl);
                for (int i = 0; i < nl; ++i) l1s[i] = hl[l].l1[i] * isc[l][i] * isc[l][i];
                dl.l1.set(l1s, true, s);
                dl.il1.set(reciprocal(l1s), true, s);
                if (l + 1 < hl.size()) {
                    dl.P.upload(scaled_csr(hl[l].P, &sc[l], &isc[l + 1]), true, s);
                    dl.Pt.upload(scaled_csr(hl[l].Pt, &isc[l + 1], &sc[l]), true, s);
                }
            } else {
                dl.A.upload(hl[l].A, false, s);
                dl.l1.set(hl[l].l1, false, s);
                dl.il1.set(reciprocal(hl[l].l1), false, s);
                if (l + 1 < hl.size()) {
                    dl.P.upload(hl[l].P, false, s);
                    dl.Pt.upload(hl[l].Pt, false, s);
                }
            }
            dl.direct = hl[l].direct;
            if (dl.direct) {  // FP64 in both forms
                if (lo) {
                    std::vector<double> li, lt, pv;
                    dl.piv_min =
                        lo_coarse_factors(hl[l].A, hl[l].piv_min, hl[l].linv, hl[l].linvt, hl[l].piv, li, lt, pv);
                    for (int i = 0; i < nl; ++i)
                        for (int k = 0; k < nl; ++k) {
                            li[(size_t)i * nl + k] *= isc[l][i] * sc[l][k];
                            lt[(size_t)i * nl + k] *= sc[l][i] * isc[l][k];
                        }
                    for (int i = 0; i < nl; ++i) pv[i] *= isc[l][i] * isc[l][i];
                    dl.Li.upload(li.data(), li.size(), s);
                    dl.LiT.upload(lt.data(), lt.size(), s);
                    dl.piv.upload(pv.data(), pv.size(), s);
                } else {
                    dl.Li.upload(hl[l].linv.data(), hl[l].linv.size(), s);
                    dl.LiT.upload(hl[l].linvt.data(), hl[l].linvt.size(), s);
                    dl.piv.upload(hl[l].piv.data(), hl[l].piv.size(), s);
                    dl.piv_min = hl[l].piv_min;
                }
            }
        }
        for (size_t l = 0; l < fused[sub].size(); ++l) {
            a.amg[sub][l].R.upload(fused[sub][l].R, lo, s);
            a.amg[sub][l].U.upload(fused[sub][l].U, lo, s);
            // sliced-ELL copies of the large FP64 level products (timed by the tuner against CSR)
            if (!lo && sell_enabled() && fused[sub][l].R.n >= kUnrollMinRows)
                a.amg[sub][l].R.sell.build(fused[sub][l].R, s);
            if (!lo && sell_enabled() && fused[sub][l].U.n >= kUnrollMinRows)
                a.amg[sub][l].U.sell.build(fused[sub][l].U, s);
        }
        // level-0 scaling folded into this subspace's transfers
        if (sub == 0) {
            upload_fine(a.G, lo ? scaled_csr(a.host.G, nullptr, &isc[0]) : a.host.G, s);
            upload_fine(a.Gt, lo ? scaled_csr(a.host.Gt, &isc[0], nullptr) : a.host.Gt, s);
        } else {
            const int d = sub - 1;
            const HostCsr pi = lo ? scaled_csr(a.host.Pi[d], nullptr, &isc[0]) : a.host.Pi[d];
            const HostCsr pit = lo ? scaled_csr(a.host.Pit[d], &isc[0], nullptr) : a.host.Pit[d];
            a.Piv[d].upload(pi.v.data(), pi.v.size(), s);
            a.Pitv[d].upload(pit.v.data(), pit.v.size(), s);
        }
    }
    build_tails(a, s);
    a.nv_alloc = 0;
    ams_reserve(a, nv);
}

// ---------------------------------------------------------------------------
// Set-up on the device (the default; SSV_AMS_SETUP=host runs the host set-up
// of amg_setup.cpp instead, which gives the same hierarchy bit for bit): the
// BC matrix, the four Galerkin products and the four AMG hierarchies come
// from amg_device.cu; the cycle's arrays (FP64, or diagonally scaled FP32) and
// the fused level products are derived from them on the device.
// ---------------------------------------------------------------------------
static bool device_setup_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("SSV_AMS_SETUP");
        v = (e && std::strcmp(e, "host") == 0) ? 0 : 1;
    }
    return v != 0;
}

// the cycle's CSR from a device FP64 CSR: an FP64 copy, or FP32 values
static void devcsr_from(DevCsr& M, const DCsr& D, bool fp32, cudaStream_t s) {
    M.n = D.n;
    M.m = D.m;
    M.nnz = D.nnz;
    M.rp.alloc(D.n + 1);
    M.ci.alloc(std::max<int64_t>(D.nnz, 1));
    SSV_CUDA(cudaMemcpyAsync(M.rp.get(), D.rp.get(), sizeof(int) * (D.n + 1), cudaMemcpyDeviceToDevice, s));
    if (D.nnz) SSV_CUDA(cudaMemcpyAsync(M.ci.get(), D.ci.get(), sizeof(int) * D.nnz, cudaMemcpyDeviceToDevice, s));
    M.v.set_dev(D.v.get(), (size_t)D.nnz, fp32, s);
    M.lanes = pick_lanes(D.n > 0 ? (double)D.nnz / D.n : 1.0);
}

// a fine-level FP64 matrix and its sliced-ELL copy: the layout (a function of
// the pattern) is kept while the pattern is the same, and only its values
// are gathered again
static void fine_from(DevCsr& M, const DCsr& D, bool layout_valid, cudaStream_t s) {
    devcsr_from(M, D, false, s);
    const bool want = sell_mode() == 2 || (sell_mode() == 1 && M.n >= kUnrollMinRows);
    if (!want) return;
    if (layout_valid && M.sell.slices > 0 && M.sell.pat_n == D.n && M.sell.pat_nnz == D.nnz)
        M.sell.refresh(D.v.get(), s);
    else
        M.sell.build_dev(D.n, D.nnz, D.rp.get(), D.ci.get(), D.v.get(), s);
}

// The four subspaces' set-up steps on host threads, each on its own stream with
// stream-ordered temporaries (AllocScope), so their latency-bound launch chains
// and host syncs overlap. The caller's stream s is drained first (buffers a job
// frees may have been in use there) and each job's stream before its thread
// ends; errors are rethrown on the calling thread. SSV_AMS_SETUP_THREADS=0
// runs the jobs in turn on s.
static bool setup_threads_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("SSV_AMS_SETUP_THREADS");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v != 0;
}

static cudaStream_t setup_stream(int k) {
    static cudaStream_t st[4] = {};
    static std::once_flag once;
    std::call_once(once, [] {
        for (auto& x : st) SSV_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
        // the pool keeps up to 4 GB of freed temporaries for the next set-up
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = 4ull << 30;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    });
    return st[k];
}

template <typename F>
static void for_subspaces(cudaStream_t s, F&& job) {
    if (!setup_threads_enabled()) {
        for (int sub = 0; sub < 4; ++sub) job(sub, s);
        return;
    }
    SSV_CUDA(cudaStreamSynchronize(s));
    int dev = 0;
    SSV_CUDA(cudaGetDevice(&dev));
    std::exception_ptr err[4];
    std::vector<std::thread> th;
    for (int sub = 0; sub < 4; ++sub) {
        try {
            th.emplace_back([&, sub] {
                try {
                    SSV_CUDA(cudaSetDevice(dev));
                    cudaStream_t ss = setup_stream(sub);
                    {
                        AllocScope scope(ss);
                        job(sub, ss);
                    }
                    SSV_CUDA(cudaStreamSynchronize(ss));
                } catch (...) {
                    err[sub] = std::current_exception();
                }
            });
        } catch (...) {
            err[sub] = std::current_exception();
        }
    }
    for (auto& t : th) t.join();
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

// BC matrix, Galerkin products (FixZeroRows) and AMG hierarchies of the four
// subspaces, fine l1 norms; false (nothing replaced) if a product row is too
// long for the device symbolic step
static bool ams_device_setup(AmsState& a, const ssv_matrix* A, cudaStream_t s) {
    AmsDev& D = a.dev;
    SetupLog log(s);
    DCsr Abc;
    d_bc_matrix(A->rows, A->cols, A->nnz, A->rp.get(), A->ci.get(), A->val.get(), a.has_fd ? a.fd.get() : nullptr,
                Abc, s);
    log.mark("BC matrix");
    std::vector<DAmgLevel> amg[4];
    WorkerThread coarse[4];  // the coarsest factorisations, on host threads while the device goes on
    bool ok[4] = {true, true, true, true};
    auto wait = [&] {
        for (auto& t : coarse) t.wait();
    };
    try {
        for_subspaces(s, [&](int sub, cudaStream_t ss) {
            SetupLog slog(ss);
            const DCsr& P0 = sub == 0 ? D.G : D.Pi[sub - 1];
            const DCsr& P0t = sub == 0 ? D.Gt : D.Pit[sub - 1];
            DCsr A0;
            if (!d_rap(Abc, P0, P0t, A0, ss)) {
                ok[sub] = false;
                return;
            }
            d_fix_zero_rows(A0, ss);
            slog.mark("subspace %d Galerkin product (%d rows, %lld nnz)", sub, A0.n, (long long)A0.nnz);
            ok[sub] = d_amg_setup(A0, a.host.theta, 25, 500, amg[sub], ss, &coarse[sub]);
            slog.mark("subspace %d hierarchy (%zu levels)", sub, amg[sub].size());
        });
    } catch (...) {
        wait();
        throw;
    }
    for (auto& t : coarse) t.join();  // rethrows a factorisation's exception
    log.mark("subspace hierarchies and coarsest factorisations");
    for (bool o : ok)
        if (!o) return false;
    D.A_bc = std::move(Abc);
    for (int sub = 0; sub < 4; ++sub) D.amg[sub] = std::move(amg[sub]);
    d_fine_l1(D.A_bc, D.fine_l1, s);
    SSV_CUDA(cudaStreamSynchronize(s));
    return true;
}

// The cycle's arrays from the device hierarchy (ams_upload_matrix's device
// counterpart, the same values): fine level FP64, every subspace level in the
// current form, the fused level products, the coarsest factors, the scaled
// transfers of the FP32 form.
static void ams_build_cycle(AmsState& a, bool layout_valid, cudaStream_t s) {
    AmsDev& D = a.dev;
    const int nv = std::max(a.nv_alloc, a.complex_form ? 2 : 1);
    SetupLog log(s);
    fine_from(a.A_bc, D.A_bc, layout_valid, s);
    log.mark("fine A_bc and its sliced-ELL copy");
    a.fine_l1.alloc(std::max(a.nhc, 1));
    SSV_CUDA(cudaMemcpyAsync(a.fine_l1.get(), D.fine_l1.get(), sizeof(double) * a.nhc, cudaMemcpyDeviceToDevice, s));
    a.fine_il1.alloc(std::max(a.nhc, 1));
    d_reciprocal(a.nhc, a.fine_l1.get(), a.fine_il1.get(), s);
    (void)fused_enabled();  // the switches are read once, before the jobs' threads
    (void)sell_enabled();
    (void)tail_rows();
    double t_fused_sub[4] = {0, 0, 0, 0};
    auto job = [&](int sub, cudaStream_t s) {
        SetupLog log(s);
        double& t_fused = t_fused_sub[sub];
        const auto& hl = D.amg[sub];
        const size_t L = hl.size();
        a.amg[sub].clear();
        a.amg[sub].resize(L);
        const bool lo = sub_lo(a, sub);
        std::vector<DevBuf<double>> sc(L), isc(L);
        if (lo)
            for (size_t l = 0; l < L; ++l) d_diag_scale(hl[l].A, sc[l], isc[l], s);
        // FP32 gradient hierarchies keep the four passes (fused, they lose too much)
        const bool fuse = fused_enabled() && !(lo && sub == 0);
        for (size_t l = 0; l < L; ++l) {
            AmgDevLevel& dl = a.amg[sub][l];
            const int nl = hl[l].A.n;
            const bool last = l + 1 == L;
            DCsr As, Ps, Pts;
            DevBuf<double> l1s, il1(std::max(nl, 1));
            const DCsr* Al = &hl[l].A;
            const DCsr* Pl = last ? nullptr : &hl[l].P;
            const DCsr* Ptl = last ? nullptr : &hl[l].Pt;
            const double* l1p = hl[l].l1.get();
            if (lo) {
                d_scaled(hl[l].A, isc[l].get(), isc[l].get(), As, s);
                Al = &As;
                l1s.alloc(std::max(nl, 1));
                d_scale_vec(nl, hl[l].l1.get(), isc[l].get(), isc[l].get(), l1s.get(), s);
                l1p = l1s.get();
                if (!last) {
                    d_scaled(hl[l].P, sc[l].get(), isc[l + 1].get(), Ps, s);
                    d_scaled(hl[l].Pt, isc[l + 1].get(), sc[l].get(), Pts, s);
                    Pl = &Ps;
                    Ptl = &Pts;
                }
            }
            devcsr_from(dl.A, *Al, lo, s);
            dl.l1.set_dev(l1p, nl, lo, s);
            d_reciprocal(nl, l1p, il1.get(), s);
            dl.il1.set_dev(il1.get(), nl, lo, s);
            if (!last) {
                devcsr_from(dl.P, *Pl, lo, s);
                devcsr_from(dl.Pt, *Ptl, lo, s);
            }
            dl.direct = hl[l].direct;
            if (dl.direct) {  // FP64 in both forms; in the FP32 form scaled like the level
                if (lo) {
                    std::vector<double> hs(nl), his(nl);
                    SSV_CUDA(cudaMemcpyAsync(hs.data(), sc[l].get(), sizeof(double) * nl, cudaMemcpyDeviceToHost, s));
                    SSV_CUDA(cudaMemcpyAsync(his.data(), isc[l].get(), sizeof(double) * nl, cudaMemcpyDeviceToHost, s));
                    SSV_CUDA(cudaStreamSynchronize(s));
                    std::vector<double> li, lt, pv;
                    if (hl[l].piv_min > kLoPivotDrop) {
                        li = hl[l].linv;
                        lt = hl[l].linvt;
                        pv = hl[l].piv;
                        dl.piv_min = hl[l].piv_min;
                    } else {
                        dl.piv_min = lo_coarse_factors(hl[l].A.to_host(s), hl[l].piv_min, hl[l].linv, hl[l].linvt,
                                                       hl[l].piv, li, lt, pv);
                    }
                    for (int i = 0; i < nl; ++i)
                        for (int k = 0; k < nl; ++k) {
                            li[(size_t)i * nl + k] *= his[i] * hs[k];
                            lt[(size_t)i * nl + k] *= hs[i] * his[k];
                        }
                    for (int i = 0; i < nl; ++i) pv[i] *= his[i] * his[i];
                    dl.Li.upload(li.data(), li.size(), s);
                    dl.LiT.upload(lt.data(), lt.size(), s);
                    dl.piv.upload(pv.data(), pv.size(), s);
                    SSV_CUDA(cudaStreamSynchronize(s));
                } else {
                    dl.Li.upload(hl[l].linv.data(), hl[l].linv.size(), s);
                    dl.LiT.upload(hl[l].linvt.data(), hl[l].linvt.size(), s);
                    dl.piv.upload(hl[l].piv.data(), hl[l].piv.size(), s);
                    dl.piv_min = hl[l].piv_min;
                }
            }
            if (fuse && !last) {
                const double tf0 = wall_seconds();
                DCsr R, U;
                if (d_fused_level(*Al, *Pl, *Ptl, l1p, R, U, s)) {
                    devcsr_from(dl.R, R, lo, s);
                    devcsr_from(dl.U, U, lo, s);
                    if (!lo && sell_enabled() && R.n >= kUnrollMinRows)
                        dl.R.sell.build_dev(R.n, R.nnz, R.rp.get(), R.ci.get(), R.v.get(), s);
                    if (!lo && sell_enabled() && U.n >= kUnrollMinRows)
                        dl.U.sell.build_dev(U.n, U.nnz, U.rp.get(), U.ci.get(), U.v.get(), s);
                }
                SSV_CUDA(cudaStreamSynchronize(s));
                t_fused += wall_seconds() - tf0;
            }
            SSV_CUDA(cudaStreamSynchronize(s));  // this level's temporaries go out of scope
        }
        log.mark("subspace %d cycle arrays (%s%s)", sub, lo ? "FP32" : "FP64", fuse ? ", fused products" : "");
        // level-0 scaling folded into this subspace's transfers
        if (sub == 0) {
            if (lo) {
                DCsr Gs, Gts;
                d_scaled(D.G, nullptr, isc[0].get(), Gs, s);
                d_scaled(D.Gt, isc[0].get(), nullptr, Gts, s);
                fine_from(a.G, Gs, true, s);
                fine_from(a.Gt, Gts, true, s);
                SSV_CUDA(cudaStreamSynchronize(s));
            } else {
                fine_from(a.G, D.G, true, s);
                fine_from(a.Gt, D.Gt, true, s);
            }
        } else {
            const int d = sub - 1;
            const int64_t nz = D.Pi[d].nnz;
            a.Piv[d].alloc(std::max<int64_t>(nz, 1));
            a.Pitv[d].alloc(std::max<int64_t>(nz, 1));
            if (lo) {
                DCsr pi, pit;
                d_scaled(D.Pi[d], nullptr, isc[0].get(), pi, s);
                d_scaled(D.Pit[d], isc[0].get(), nullptr, pit, s);
                SSV_CUDA(cudaMemcpyAsync(a.Piv[d].get(), pi.v.get(), sizeof(double) * nz, cudaMemcpyDeviceToDevice, s));
                SSV_CUDA(cudaMemcpyAsync(a.Pitv[d].get(), pit.v.get(), sizeof(double) * nz, cudaMemcpyDeviceToDevice, s));
                SSV_CUDA(cudaStreamSynchronize(s));
            } else {
                SSV_CUDA(cudaMemcpyAsync(a.Piv[d].get(), D.Pi[d].v.get(), sizeof(double) * nz, cudaMemcpyDeviceToDevice,
                                         s));
                SSV_CUDA(cudaMemcpyAsync(a.Pitv[d].get(), D.Pit[d].v.get(), sizeof(double) * nz,
                                         cudaMemcpyDeviceToDevice, s));
            }
        }
        if (a.num_smooth == 1) {
            if (lo) build_tail<float>(a.amg[sub], s);
            else build_tail<double>(a.amg[sub], s);
        } else {
            for (auto& lv : a.amg[sub]) lv.tail.release();
        }
        const int tl = tail_level(a.amg[sub]);
        log.mark("subspace %d transfers and %s", sub, tl >= 0 ? "dense tail" : "no dense tail");
    };
    for_subspaces(s, job);
    log.mark("subspace cycle arrays, transfers, dense tails");
    a.t_fused = t_fused_sub[0] + t_fused_sub[1] + t_fused_sub[2] + t_fused_sub[3];
    a.nv_alloc = 0;
    ams_reserve(a, nv);
    log.mark("work vectors + shape tuner");
}

// Rebuild the matrix-dependent part (RebuildMatrix) and upload it.
static void ams_rebuild(AmsState& a, const ssv_matrix* A) {
    cudaStream_t s = stream();
    const double t0 = wall_seconds();
    a.t_tune = 0;
    a.t_fused = 0;
    if (A->dtype != SSV_F64) fail(SSV_ERR_TYPE, "CompactAMS: the HCurl matrix must be real");
    if (device_setup_enabled() && ams_device_setup(a, A, stream())) {
        a.t_host = wall_seconds() - t0;
        const bool same = a.dev.on && a.dev.src == A;
        a.dev.on = true;
        a.dev.src = A;
        ams_build_cycle(a, same, s);
    } else {
        a.dev.on = false;
        HostCsr H = host_csr_of(A);
        a.host.rebuild(H, a.has_fd ? a.h_fd.data() : nullptr);
        a.t_host = wall_seconds() - t0;
        ams_upload_matrix(a, s);
    }
    ++a.gen;
    SSV_CUDA(cudaStreamSynchronize(s));
    a.t_total = wall_seconds() - t0;
}

void ams_setup_times(const AmsState* a, double* t) {
    t[0] = a->t_total;
    t[1] = a->t_host;
    t[2] = a->t_fused;
    t[3] = a->t_tune;
}

AmsState* ams_create(const ssv_matrix* A, const ssv_matrix* G, const uint8_t* fd, const double* cx,
                     const double* cy, const double* cz, int cycle_type, int num_smooth, double theta, double w,
                     int complex_form, int ndof_complex) {
    auto* a = new AmsState();
    try {
        cudaStream_t s = stream();
        a->forks.ensure(2);
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
        ams_upload_geometry(*a, s);
        if (device_setup_enabled()) {  // the geometry in FP64 for the device set-up (kept)
            a->dev.G.from_host(a->host.G, s);
            a->dev.Gt.from_host(a->host.Gt, s);
            for (int d = 0; d < 3; ++d) {
                a->dev.Pi[d].from_host(a->host.Pi[d], s);
                a->dev.Pit[d].from_host(a->host.Pit[d], s);
            }
            SSV_CUDA(cudaStreamSynchronize(s));
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

// Switch between the FP64 and FP32 forms: the host keeps the hierarchy, so
// this is a re-upload, no new set-up.
void ams_set_precision(AmsState* a, int precision) {
    const bool lo = precision == SSV_PREC_FP32 || precision == SSV_PREC_FP32_NODAL;
    const bool g64 = precision == SSV_PREC_FP32_NODAL;
    if (lo == a->fp32 && g64 == a->grad64) return;
    cudaStream_t s = stream();
    const double t0 = wall_seconds();
    a->fp32 = lo;
    a->grad64 = g64;
    a->t_tune = 0;
    a->t_host = 0;
    if (a->dev.on) ams_build_cycle(*a, true, s);
    else ams_upload_matrix(*a, s);
    ++a->gen;
    SSV_CUDA(cudaStreamSynchronize(s));
    a->t_total = wall_seconds() - t0;
}

int ams_precision(const AmsState* a) {
    return !a->fp32 ? SSV_PREC_FP64 : a->grad64 ? SSV_PREC_FP32_NODAL : SSV_PREC_FP32;
}

void ams_reserve_block(AmsState* a, int nrhs) {
    ams_reserve(*a, nrhs * (a->complex_form ? 2 : 1));
    SSV_CUDA(cudaStreamSynchronize(stream()));
}

template <typename TG, typename TN>
static void ams_block_t(AmsState& a, const double* in, double* out, int nrhs, const KState* st, cudaStream_t s) {
    if (a.complex_form) {
        switch (nrhs) {
            case 1: ams_cycle<TG, TN, 2, true>(a, in, out, st, s); return;
            case 4: ams_cycle<TG, TN, 8, true>(a, in, out, st, s); return;
        }
    } else {
        switch (nrhs) {
            case 1: ams_cycle<TG, TN, 1, false>(a, in, out, st, s); return;
            case 4: ams_cycle<TG, TN, 4, false>(a, in, out, st, s); return;
        }
    }
    fail(SSV_ERR_INVALID_ARG, "AMS block apply: nrhs must be 1 or 4");
}

// One subspace correction of the cycle on its own (parity hook): the
// restriction b_s = P_s^T r (G^T for the gradient subspace, the scaled Pi_s^T
// for a nodal one), the subspace V-cycle x_s, and the prolonged correction
// c = w P_s x_s -- each in the types of the current form, returned as FP64
// (b_s and x_s in the hierarchy's own, diagonally scaled in the FP32 forms,
// coordinates).
template <typename TG, typename TN, int NV>
static void ams_subspace_t(AmsState& a, int sub, const double* r, double* bs, double* xs, double* corr,
                           cudaStream_t s) {
    const int64_t m1 = (int64_t)a.nh1 * NV;
    SSV_CUDA(cudaMemsetAsync(corr, 0, sizeof(double) * (size_t)a.nhc * NV, s));
    if (sub == 0) {
        mv_spmv<double, double, TG, NV, MV_AX, true>(a.Gt, r, a.rs[0].as<TG>(), nullptr, nullptr, TG(0), nullptr, s);
        widen_to<TG>(a.rs[0].as<TG>(), m1, bs, s);
        TG* g = vcycle<TG, NV, true>(a.amg[0], 0, a.rs[0].as<TG>(), 1, nullptr, s);
        widen_to<TG>(g, m1, xs, s);
        mv_spmv<double, TG, double, NV, MV_ADD, true>(a.G, g, corr, nullptr, nullptr, a.w, nullptr, s);
    } else {
        pi_restrict<TN, NV>(a, r, a.rs[1].as<TN>(), a.rs[2].as<TN>(), a.rs[3].as<TN>(), nullptr, s);
        widen_to<TN>(a.rs[sub].as<TN>(), m1, bs, s);
        TN* g = vcycle<TN, NV, true>(a.amg[sub], 0, a.rs[sub].as<TN>(), 1, nullptr, s);
        widen_to<TN>(g, m1, xs, s);
        DevBuf<TN> zero((size_t)std::max<int64_t>(m1, 1));
        zero.zero(s);
        pi_prolong<TN, NV>(a, sub == 1 ? g : zero.get(), sub == 2 ? g : zero.get(), sub == 3 ? g : zero.get(), corr,
                           nullptr, s);
        SSV_CUDA(cudaStreamSynchronize(s));
    }
}

void ams_subspace_apply(AmsState* a, int sub, const double* r, double* bs, double* xs, double* corr) {
    if (sub < 0 || sub > 3) fail(SSV_ERR_INVALID_ARG, "ssv_ams_subspace_apply: subspace must be 0..3");
    cudaStream_t s = stream();
    const int nv = a->complex_form ? 2 : 1;
    const size_t nh = (size_t)a->nhc * nv, n1 = (size_t)a->nh1 * nv;
    DevBuf<double> dr(nh), db(n1), dx(n1), dc(nh);
    SSV_CUDA(cudaMemcpyAsync(dr.get(), r, sizeof(double) * nh, cudaMemcpyHostToDevice, s));
    with_forms(*a, [&](auto g, auto n) {
        if (nv == 2) ams_subspace_t<decltype(g), decltype(n), 2>(*a, sub, dr.get(), db.get(), dx.get(), dc.get(), s);
        else ams_subspace_t<decltype(g), decltype(n), 1>(*a, sub, dr.get(), db.get(), dx.get(), dc.get(), s);
    });
    SSV_CUDA(cudaMemcpyAsync(bs, db.get(), sizeof(double) * n1, cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaMemcpyAsync(xs, dx.get(), sizeof(double) * n1, cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaMemcpyAsync(corr, dc.get(), sizeof(double) * nh, cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
}

// nrhs right-hand sides, row-interleaved ([row][rhs], complex as Re/Im pairs).
void ams_apply_block(AmsState* a, const double* in, double* out, int nrhs, const KState* st, cudaStream_t s) {
    if (nrhs * (a->complex_form ? 2 : 1) > a->nv_alloc) fail(SSV_ERR_INVALID_ARG, "AMS block apply: reserve first");
    with_forms(*a, [&](auto g, auto n) { ams_block_t<decltype(g), decltype(n)>(*a, in, out, nrhs, st, s); });
}

// ---------------------------------------------------------------------------
// Per-phase profile of one cycle (measurement hook, no reference counterpart):
// every phase is re-launched `reps` times between CUDA events on the
// library's stream; bytes are the algorithmic bytes of one execution (CSR
// with int32 indices, values of the stored type, every vector entry read or
// written once, gathered x counted once).
// ---------------------------------------------------------------------------
static double csr_pass_bytes(const DevCsr& A, int vb) { return (double)A.nnz * (4 + vb) + 4.0 * (A.n + 1); }

// one V-cycle from level l: matrix passes and vector streams
static double vcycle_bytes(const std::vector<AmgDevLevel>& L, int l, int NV, int tb) {
    const AmgDevLevel& lv = L[l];
    const double n = lv.A.n, v = (double)NV * tb;
    if (l == (int)L.size() - 1) {
        if (lv.direct) return 8.0 * n * n + n * 8.0 + n * (2 * v + 2 * 8.0 * NV);
        return n * (2 * v + tb) + 9 * (csr_pass_bytes(lv.A, tb) + n * (3 * v + tb));
    }
    const double nc = L[l + 1].A.n;
    double b = n * (2 * v + tb);                            // first sweep x = b / l1
    b += csr_pass_bytes(lv.A, tb) + 3 * n * v;              // residual
    b += csr_pass_bytes(lv.Pt, tb) + (n + nc) * v;          // restriction
    b += vcycle_bytes(L, l + 1, NV, tb);
    b += csr_pass_bytes(lv.P, tb) + (nc + 2 * n) * v;       // prolongation add
    b += csr_pass_bytes(lv.A, tb) + n * (3 * v + tb);       // post sweep
    return b;
}

template <typename TG, typename TN, int NV, bool RECIP>
static void ams_profile_t(AmsState& a, int reps, bool cold, ssv_phase_profile* out) {
    cudaStream_t s = stream();
    const int n = a.nhc, n1 = a.nh1;
    const int tg = (int)sizeof(TG), tn = (int)sizeof(TN);
    DevBuf<double> pin((size_t)n * NV), pout((size_t)n * NV);
    pin.zero(s);
    double* cur = a.xa.get();
    double* alt = a.xb.get();
    double* r = a.r.get();
    const double* d = RECIP ? a.fine_il1.get() : a.fine_l1.get();
    cudaEvent_t e0, e1;
    SSV_CUDA(cudaEventCreate(&e0));
    SSV_CUDA(cudaEventCreate(&e1));
    std::memset(out, 0, sizeof(*out));
    auto timed = [&](const char* name, double bytes, int kernels, auto&& launch) {
        for (int k = 0; k < 2; ++k) launch();
        const float ms = time_launches(launch, reps, cold, s, e0, e1);
        const int i = out->num_phases++;
        std::snprintf(out->names[i], sizeof(out->names[i]), "%s", name);
        out->ms[i] = (double)ms / reps;
        out->bytes[i] = bytes;
        out->kernels[i] = kernels;
    };
    const double N = n, N1 = n1, V = 8.0 * NV, Vg = (double)tg * NV, Vn = (double)tn * NV;
    const double fine_res = csr_pass_bytes(a.A_bc, 8) + 3 * N * V;
    const double fine_jac = csr_pass_bytes(a.A_bc, 8) + N * (3 * V + 8);
    const double grad_vc = vcycle_bytes(a.amg[0], 0, NV, tg);
    double nod_vc = 0;
    for (int k = 1; k < 4; ++k) nod_vc += vcycle_bytes(a.amg[k], 0, NV, tn);
    const double g_tr = csr_pass_bytes(a.Gt, 8) + N * V + N1 * Vg + csr_pass_bytes(a.G, 8) + N1 * Vg + 2 * N * V;
    const double pi_tr = (double)a.Gt.nnz * (4 + 24) + 4.0 * (n1 + 1) + N * V + 3 * N1 * Vn +
                         (double)a.G.nnz * (4 + 24) + 4.0 * (n + 1) + 3 * N1 * Vn + 2 * N * V;
    // cycle 1 (01210): 2 masks, first sweep, 3 residuals, 2 + 1 corrections, one final sweep
    const double cyc = 2 * (2 * N * V + N) + N * (2 * V + 8) + 3 * fine_res + 2 * grad_vc + nod_vc + 2 * g_tr + pi_tr +
                       fine_jac;
    timed("ams_cycle", cyc, 0, [&] { ams_cycle<TG, TN, NV, RECIP>(a, pin.get(), pout.get(), nullptr, s); });
    timed("fine_residual", fine_res, 1, [&] {
        mv_spmv<double, double, double, NV, MV_RES, RECIP>(a.A_bc, cur, r, a.b0.get(), nullptr, 0.0, nullptr, s);
    });
    timed("fine_smooth", fine_jac, 1, [&] {
        mv_spmv<double, double, double, NV, MV_JAC, RECIP>(a.A_bc, cur, alt, a.b0.get(), d, 0.0, nullptr, s);
    });
    timed("grad_vcycle", grad_vc, 0, [&] { vcycle<TG, NV, RECIP>(a.amg[0], 0, a.rs[0].as<TG>(), 1, nullptr, s); });
    timed("nodal_vcycles", nod_vc, 0, [&] {
        if (tri_ok(a)) {
            TN* g3[3];
            vcycle3<TN, NV, RECIP>(a, nullptr, s, g3);
            return;
        }
        a.forks.fork(s, 2);
        vcycle<TN, NV, RECIP>(a.amg[1], 0, a.rs[1].as<TN>(), 1, nullptr, s);
        vcycle<TN, NV, RECIP>(a.amg[2], 0, a.rs[2].as<TN>(), 1, nullptr, a.forks.side[0]);
        vcycle<TN, NV, RECIP>(a.amg[3], 0, a.rs[3].as<TN>(), 1, nullptr, a.forks.side[1]);
        a.forks.join(s, 2);
    });
    timed("grad_transfers", g_tr, 2, [&] {
        mv_spmv<double, double, TG, NV, MV_AX, RECIP>(a.Gt, r, a.rs[0].as<TG>(), nullptr, nullptr, TG(0), nullptr, s);
        mv_spmv<double, TG, double, NV, MV_ADD, RECIP>(a.G, a.rs[0].as<TG>(), alt, nullptr, nullptr, a.w, nullptr, s);
    });
    timed("pi_transfers", pi_tr, 2, [&] {
        pi_restrict<TN, NV>(a, r, a.rs[1].as<TN>(), a.rs[2].as<TN>(), a.rs[3].as<TN>(), nullptr, s);
        pi_prolong<TN, NV>(a, a.rs[1].as<TN>(), a.rs[2].as<TN>(), a.rs[3].as<TN>(), alt, nullptr, s);
    });
    SSV_CUDA(cudaEventDestroy(e0));
    SSV_CUDA(cudaEventDestroy(e1));
    SSV_CUDA(cudaStreamSynchronize(s));
}

// Per-level device time of one subspace V-cycle (measurement hook): the down
// product R_l and the up product U_l of every level run one by one (warm,
// back to back, reps times), then the last step (the dense tail or the
// coarsest solve); shape = lanes * 10 + rows per group, as the tuner chose.
template <typename T, int NV>
static int profile_levels_t(std::vector<AmgDevLevel>& L, int reps, double* ms_r, double* ms_u, int* shape_r,
                            int* shape_u, int cap, double* last_ms, cudaStream_t s) {
    cudaEvent_t e0, e1;
    SSV_CUDA(cudaEventCreate(&e0));
    SSV_CUDA(cudaEventCreate(&e1));
    const int tl = tail_level(L);
    const int n = tl >= 0 ? tl + 1 : (int)L.size();
    auto time = [&](auto&& launch) {
        launch();
        return (double)time_launches(launch, reps, false, s, e0, e1) / reps;
    };
    for (int l = 0; l + 1 < n && l < cap; ++l) {
        if (!L[l].R.n) {
            ms_r[l] = ms_u[l] = 0;
            shape_r[l] = shape_u[l] = 0;
            continue;
        }
        const T* e = (l + 1 == n - 1) ? L[l + 1].xa.template as<T>() : L[l + 1].xb.template as<T>();
        ms_r[l] = time([&] {
            mv_spmv<T, T, T, NV, MV_AX, true>(L[l].R, L[l].b.template as<T>(), L[l + 1].b.template as<T>(), nullptr,
                                              nullptr, T(0), nullptr, s);
        });
        ms_u[l] = time([&] {
            mv_spmv<T, T, T, NV, MV_TWO, true>(L[l].U, L[l].b.template as<T>(), L[l].xb.template as<T>(), e, nullptr,
                                               T(0), nullptr, s);
        });
        shape_r[l] = L[l].R.lanes_for(NV) * 10 + L[l].R.unroll_for(NV);
        shape_u[l] = L[l].U.lanes_for(NV) * 10 + L[l].U.unroll_for(NV);
    }
    *last_ms = time([&] {
        if (tl >= 0) {
            TailSet<T, 1> t{};
            t.n[0] = L[tl].A.n;
            t.M[0] = L[tl].tail.get();
            t.b[0] = L[tl].b.template as<T>();
            t.y[0] = L[tl].xa.template as<T>();
            tail_apply<T, NV, 1>(t, 1, nullptr, s);
        } else {
            coarse_direct<T, NV, true>(L[n - 1], L[n - 1].b.template as<T>(), L[n - 1].xa.template as<T>(), nullptr,
                                       s);
        }
    });
    SSV_CUDA(cudaEventDestroy(e0));
    SSV_CUDA(cudaEventDestroy(e1));
    return n;
}

int ams_profile_levels(AmsState* a, int sub, int reps, double* ms_r, double* ms_u, int* shape_r, int* shape_u,
                       int cap, double* last_ms) {
    if (sub < 0 || sub > 3) fail(SSV_ERR_INVALID_ARG, "ssv_ams_profile_levels: subspace must be 0..3");
    const int nv = a->complex_form ? 2 : 1;
    ams_reserve(*a, nv);
    cudaStream_t s = stream();
    int n = 0;
    auto run = [&](auto tag) {
        using T = decltype(tag);
        if (nv == 2)
            n = profile_levels_t<T, 2>(a->amg[sub], std::max(reps, 1), ms_r, ms_u, shape_r, shape_u, cap, last_ms, s);
        else
            n = profile_levels_t<T, 1>(a->amg[sub], std::max(reps, 1), ms_r, ms_u, shape_r, shape_u, cap, last_ms, s);
    };
    if (sub_lo(*a, sub)) run(float{});
    else run(double{});
    SSV_CUDA(cudaStreamSynchronize(s));
    return n;
}

template <typename TG, typename TN>
static void ams_profile_nrhs(AmsState& a, int nrhs, int reps, bool cold, ssv_phase_profile* out) {
    if (a.complex_form) {
        if (nrhs == 1) ams_profile_t<TG, TN, 2, true>(a, reps, cold, out);
        else ams_profile_t<TG, TN, 8, true>(a, reps, cold, out);
    } else {
        if (nrhs == 1) ams_profile_t<TG, TN, 1, false>(a, reps, cold, out);
        else ams_profile_t<TG, TN, 4, false>(a, reps, cold, out);
    }
}

void ams_profile(AmsState* a, int nrhs, int reps, int flags, ssv_phase_profile* out) {
    if (nrhs != 1 && nrhs != 4) fail(SSV_ERR_INVALID_ARG, "ssv_ams_profile: nrhs must be 1 or 4");
    ams_reserve(*a, nrhs * (a->complex_form ? 2 : 1));
    const bool cold = (flags & SSV_PROFILE_COLD) != 0;
    with_forms(*a, [&](auto g, auto n) {
        ams_profile_nrhs<decltype(g), decltype(n)>(*a, nrhs, std::max(reps, 1), cold, out);
    });
}

// ---------------------------------------------------------------------------
// CompactAMGPreconditioner (compact_amg.hpp:49-183, factory
// sparsesolv_python_export.hpp:359-404): one AMG hierarchy of a scalar H1
// matrix (FreeDofs view), set up on the host like the AMS subspaces, and
// Mult = x = 0, one V-cycle, constrained outputs zeroed, FP64 on the device.
// ---------------------------------------------------------------------------
struct AmgOnly {
    AmgHost host;
    std::vector<AmgDevLevel> lev;
    bool has_fd = false;
    std::vector<uint8_t> h_fd;
    DevBuf<uint8_t> fd;
    int n = 0, num_smooth = 1;
    unsigned gen = 0;
};

void amg_free(AmgOnly* g) { delete g; }

static void amg_rebuild(AmgOnly& g, const ssv_matrix* A) {
    cudaStream_t s = stream();
    HostCsr H = host_csr_of(A);
    if (g.has_fd)  // CreateBCModifiedMatrix (compact_amg.hpp:252-287)
        for (int i = 0; i < H.n; ++i)
            for (int k = H.rp[i]; k < H.rp[i + 1]; ++k) {
                const int j = H.ci[k];
                if (!g.h_fd[i]) H.v[k] = (j == i) ? 1.0 : 0.0;
                else if (!g.h_fd[j]) H.v[k] = 0.0;
            }
    g.host.setup(H);
    const auto& hl = g.host.levels;
    g.lev.clear();
    g.lev.resize(hl.size());
    for (size_t l = 0; l < hl.size(); ++l) {
        AmgDevLevel& dl = g.lev[l];
        const int nl = hl[l].A.n;
        dl.A.upload(hl[l].A, false, s);
        dl.l1.set(hl[l].l1, false, s);
        dl.il1.set(reciprocal(hl[l].l1), false, s);
        if (l + 1 < hl.size()) {
            dl.P.upload(hl[l].P, false, s);
            dl.Pt.upload(hl[l].Pt, false, s);
            if (fused_enabled() && g.num_smooth == 1) {  // the two fused level products (vcycle_fused)
                const FusedLevel F = fused_level(hl[l].A, hl[l].P, hl[l].Pt, hl[l].l1);
                dl.R.upload(F.R, false, s);
                dl.U.upload(F.U, false, s);
            }
        }
        dl.direct = hl[l].direct;
        if (dl.direct) {
            dl.Li.upload(hl[l].linv.data(), hl[l].linv.size(), s);
            dl.LiT.upload(hl[l].linvt.data(), hl[l].linvt.size(), s);
            dl.piv.upload(hl[l].piv.data(), hl[l].piv.size(), s);
            dl.cz.alloc(nl);
        }
        dl.b.alloc(nl);
        dl.xa.alloc(nl);
        dl.xb.alloc(nl);
        dl.r.alloc(nl);
    }
    cudaEvent_t e0, e1;
    SSV_CUDA(cudaEventCreate(&e0));
    SSV_CUDA(cudaEventCreate(&e1));
    for (size_t l = 0; l < g.lev.size(); ++l) {
        AmgDevLevel& L = g.lev[l];
        tune_csr<double, double, double, 1>(L.A, L.xa.as<double>(), L.xb.as<double>(), L.b.as<double>(), s, e0, e1);
        if (l + 1 < g.lev.size()) {
            tune_csr<double, double, double, 1>(L.P, g.lev[l + 1].xa.as<double>(), L.r.as<double>(), nullptr, s, e0,
                                                e1);
            tune_csr<double, double, double, 1>(L.Pt, L.r.as<double>(), g.lev[l + 1].b.as<double>(), nullptr, s, e0,
                                                e1);
            if (L.R.n) {
                tune_csr<double, double, double, 1>(L.R, L.b.as<double>(), g.lev[l + 1].b.as<double>(), nullptr, s,
                                                    e0, e1);
                tune_csr<double, double, double, 1>(L.U, L.b.as<double>(), L.xb.as<double>(),
                                                    g.lev[l + 1].xa.as<double>(), s, e0, e1, false, true);
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ++g.gen;
    SSV_CUDA(cudaStreamSynchronize(s));
}

AmgOnly* amg_create(const ssv_matrix* A, const uint8_t* fd, double theta, int max_levels, int min_coarse,
                    int num_smooth) {
    auto* g = new AmgOnly();
    try {
        g->n = A->rows;
        g->num_smooth = std::max(1, num_smooth);
        g->host.theta = theta;
        g->host.max_levels = std::max(1, max_levels);
        g->host.min_coarse = min_coarse;
        g->host.num_smooth = g->num_smooth;
        if (fd) {
            g->has_fd = true;
            g->h_fd.assign(fd, fd + g->n);
            for (auto& v : g->h_fd) v = v ? 1 : 0;
            g->fd.upload(g->h_fd.data(), g->h_fd.size(), stream());
        }
        amg_rebuild(*g, A);
    } catch (...) {
        delete g;
        throw;
    }
    return g;
}

void amg_update(AmgOnly* g, const ssv_matrix* A) { amg_rebuild(*g, A); }

int amg_levels(const AmgOnly* g, int* sizes, int cap) {
    const auto& hl = g->host.levels;
    for (size_t l = 0; l < hl.size() && 2 * (int)l + 1 < cap; ++l) {
        sizes[2 * l] = hl[l].A.n;
        sizes[2 * l + 1] = hl[l].A.nnz();
    }
    return (int)hl.size();
}

// Mult (compact_amg.hpp:166-183): x = 0, VCycle(0, b, x), constrained x = 0
static void amg_apply(AmgOnly& g, const double* x, double* y, const KState* st, cudaStream_t s) {
    const double* res = vcycle<double, 1, false>(g.lev, 0, x, g.num_smooth, st, s);
    launch_k(k_mv_mask_copy<double, double, 1>, grid_for(g.n, kBlock), kBlock, s, g.n, res,
             (const uint8_t*)(g.has_fd ? g.fd.get() : nullptr), y, st);
    SSV_LAUNCH_CHECK();
}

// y = M^{-1} x for the preconditioner p, stream-ordered and capturable.
template <>
void precond_apply_any<double>(ssv_precond* p, const double* x, double* y, const KState* st, cudaStream_t s) {
    if (p->kind == 1) ic_apply_dev<double>(p, x, y, st, s);
    else if (p->kind == 4) sgs_apply_dev<double>(p, x, y, st, s);
    else if (p->kind == 5) amg_apply(*p->amg, x, y, st, s);
    else if (p->kind == 2) {
        with_forms(*p->ams, [&](auto g, auto n) { ams_cycle<decltype(g), decltype(n), 1, false>(*p->ams, x, y, st, s); });
    } else fail(SSV_ERR_TYPE, "preconditioner is complex; the matrix is real");
}

template <>
void precond_apply_any<zdouble>(ssv_precond* p, const zdouble* x, zdouble* y, const KState* st, cudaStream_t s) {
    if (p->kind == 1) ic_apply_dev<zdouble>(p, x, y, st, s);
    else if (p->kind == 4) sgs_apply_dev<zdouble>(p, x, y, st, s);
    else if (p->kind == 3) {
        const double* xi = reinterpret_cast<const double*>(x);
        double* yo = reinterpret_cast<double*>(y);
        with_forms(*p->ams, [&](auto g, auto n) { ams_cycle<decltype(g), decltype(n), 2, true>(*p->ams, xi, yo, st, s); });
    } else fail(SSV_ERR_TYPE, "preconditioner is real; the matrix is complex");
}

unsigned precond_generation(const ssv_precond* p) {
    if (p->kind == 1) return p->A->dtype == SSV_F64 ? p->ic_d.gen : p->ic_z.gen;
    if (p->kind == 4) return p->A->dtype == SSV_F64 ? p->sgs_d.gen : p->sgs_z.gen;
    if (p->kind == 5) return p->amg ? p->amg->gen : 0;
    return p->ams ? p->ams->gen : 0;
}

// Level matrix of the hierarchy as set up (FP64, unscaled): what = 0 A_l,
// 1 P_l; returns nnz (arrays filled only when cap >= nnz)
int ams_level_matrix(const AmsState* a, int sub, int l, int what, int* rp, int* ci, double* v, int cap) {
    if (sub < 0 || sub > 3) fail(SSV_ERR_INVALID_ARG, "ssv_ams_level_matrix: subspace must be 0..3");
    HostCsr H;
    if (a->dev.on) {
        const auto& dl = a->dev.amg[sub];
        if (l < 0 || l >= (int)dl.size() || (what == 1 && l + 1 >= (int)dl.size()))
            fail(SSV_ERR_INVALID_ARG, "ssv_ams_level_matrix: no such level");
        H = (what == 0 ? dl[l].A : dl[l].P).to_host(stream());
    } else {
        const auto& hl = a->host.amg[sub].levels;
        if (l < 0 || l >= (int)hl.size() || (what == 1 && l + 1 >= (int)hl.size()))
            fail(SSV_ERR_INVALID_ARG, "ssv_ams_level_matrix: no such level");
        H = what == 0 ? hl[l].A : hl[l].P;
    }
    const int nnz = H.nnz();
    if (cap >= nnz && rp && ci && v) {
        std::copy(H.rp.begin(), H.rp.end(), rp);
        std::copy(H.ci.begin(), H.ci.begin() + nnz, ci);
        std::copy(H.v.begin(), H.v.begin() + nnz, v);
    }
    return nnz;
}

bool ams_on_device(const AmsState* a) { return a->dev.on; }

int ams_levels(const AmsState* a, int sub, int* sizes, int cap) {
    if (a->dev.on) {
        const auto& dl = a->dev.amg[sub];
        for (size_t l = 0; l < dl.size() && 2 * (int)l + 1 < cap; ++l) {
            sizes[2 * l] = dl[l].A.n;
            sizes[2 * l + 1] = (int)dl[l].A.nnz;
        }
        return (int)dl.size();
    }
    const auto& hl = a->host.amg[sub].levels;
    for (size_t l = 0; l < hl.size() && 2 * (int)l + 1 < cap; ++l) {
        sizes[2 * l] = hl[l].A.n;
        sizes[2 * l + 1] = hl[l].A.nnz();
    }
    return (int)hl.size();
}

}  // namespace ssv
