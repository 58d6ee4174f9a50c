// assembly.cu -- on-device assembly of the lowest-order Nedelec (Whitney)
// curl-curl and mass matrices and the discrete gradient of a tetrahedral mesh
// (the step before the solve path; NGSolve assembles the reference's matrices).
//
// Element matrices: w_ab = l_a grad l_b - l_b grad l_a on the local edge (a,b),
// curl w_ab = 2 grad l_a x grad l_b, int l_p l_q = vol (1 + delta_pq) / 20,
// each local edge signed by its orientation against the global edge. The
// global matrices sum coef_t E_t over the elements; every CSR row is built by
// one thread that visits the row's elements in increasing element order, so
// each entry is summed in element order (the order of the element-wise COO
// sum it replaces) and the result does not depend on the launch.
#include <algorithm>
#include <memory>
#include <vector>

#include "objects.cuh"
#include "solver_api.hpp"

namespace ssv {
namespace {

__device__ __constant__ int kLE[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
constexpr int kMaxCand = 384;  // candidate columns of one row (6 per incident element)

// Ke (curl-curl per unit coefficient) and Me (mass) of element t, 36 entries each
__global__ void k_element_matrices(int nt, const double* __restrict__ xyz, const int* __restrict__ tets,
                                   const int8_t* __restrict__ sgn, double* __restrict__ Ke, double* __restrict__ Me) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        double P[4][3];
        for (int v = 0; v < 4; ++v)
            for (int d = 0; d < 3; ++d) P[v][d] = xyz[(size_t)tets[(size_t)t * 4 + v] * 3 + d];
        // J = [P1-P0 | P2-P0 | P3-P0] (columns); rows of J^{-1} = grad l1..l3
        double J[3][3];
        for (int d = 0; d < 3; ++d)
            for (int c = 0; c < 3; ++c) J[d][c] = P[c + 1][d] - P[0][d];
        const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                           J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        double g[4][3];
        // inverse by the adjugate: (J^{-1})[r][c] = cof(J)[c][r] / det
        g[1][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
        g[1][1] = -(J[0][1] * J[2][2] - J[0][2] * J[2][1]) / det;
        g[1][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
        g[2][0] = -(J[1][0] * J[2][2] - J[1][2] * J[2][0]) / det;
        g[2][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
        g[2][2] = -(J[0][0] * J[1][2] - J[0][2] * J[1][0]) / det;
        g[3][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
        g[3][1] = -(J[0][0] * J[2][1] - J[0][1] * J[2][0]) / det;
        g[3][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
        for (int d = 0; d < 3; ++d) g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
        const double vol = fabs(det) / 6.0;
        double curl[6][3], s[6];
        for (int a = 0; a < 6; ++a) {
            const double* ga = g[kLE[a][0]];
            const double* gb = g[kLE[a][1]];
            s[a] = (double)sgn[(size_t)t * 6 + a];
            curl[a][0] = 2.0 * (ga[1] * gb[2] - ga[2] * gb[1]) * s[a];
            curl[a][1] = 2.0 * (ga[2] * gb[0] - ga[0] * gb[2]) * s[a];
            curl[a][2] = 2.0 * (ga[0] * gb[1] - ga[1] * gb[0]) * s[a];
        }
        double G[4][4];
        for (int p = 0; p < 4; ++p)
            for (int q = 0; q < 4; ++q) G[p][q] = g[p][0] * g[q][0] + g[p][1] * g[q][1] + g[p][2] * g[q][2];
        auto I = [](int p, int q) { return (p == q ? 2.0 : 1.0) / 20.0; };
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b) {
                const int i = kLE[a][0], j = kLE[a][1], k = kLE[b][0], l = kLE[b][1];
                Ke[(size_t)t * 36 + a * 6 + b] =
                    (curl[a][0] * curl[b][0] + curl[a][1] * curl[b][1] + curl[a][2] * curl[b][2]) * vol;
                const double m = I(i, k) * G[j][l] - I(i, l) * G[j][k] - I(j, k) * G[i][l] + I(j, l) * G[i][k];
                Me[(size_t)t * 36 + a * 6 + b] = m * vol * (s[a] * s[b]);
            }
    }
}

// incidence: cnt[e] = elements holding edge e
__global__ void k_inc_count(int nt, const int* __restrict__ te, int* __restrict__ cnt) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nt * 6; q += gridDim.x * blockDim.x)
        atomicAdd(&cnt[te[q]], 1);
}

__global__ void k_inc_fill(int nt, const int* __restrict__ te, const int* __restrict__ irp, int* __restrict__ fill,
                           int* __restrict__ inc) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nt * 6; q += gridDim.x * blockDim.x) {
        const int e = te[q];
        inc[irp[e] + atomicAdd(&fill[e], 1)] = q;  // q = 6 t + local edge
    }
}

// each edge's incidences in increasing element order (the fill order is not fixed)
__global__ void k_inc_sort(int ne, const int* __restrict__ irp, int* __restrict__ inc) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x)
        for (int k = irp[e] + 1; k < irp[e + 1]; ++k) {
            const int v = inc[k];
            int j = k - 1;
            while (j >= irp[e] && inc[j] > v) {
                inc[j + 1] = inc[j];
                --j;
            }
            inc[j + 1] = v;
        }
}

// row e's distinct columns (the edges of its elements), counted (out == null)
// or written sorted at rp[e]; *ovf = 1 when a row has too many candidates
__global__ void k_row_pattern(int ne, const int* __restrict__ irp, const int* __restrict__ inc,
                              const int* __restrict__ te, int* __restrict__ cnt, const int* __restrict__ rp,
                              int* __restrict__ out, int* __restrict__ ovf) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        int cand[kMaxCand];
        int m = 0;
        bool over = false;
        for (int k = irp[e]; k < irp[e + 1]; ++k) {
            const int t = inc[k] / 6;
            for (int b = 0; b < 6; ++b) {
                const int c = te[(size_t)t * 6 + b];
                int j = m - 1;  // insertion into the sorted list, duplicates dropped
                while (j >= 0 && cand[j] > c) --j;
                if (j >= 0 && cand[j] == c) continue;
                if (m == kMaxCand) {
                    over = true;
                    continue;
                }
                for (int q = m; q > j + 1; --q) cand[q] = cand[q - 1];
                cand[j + 1] = c;
                ++m;
            }
        }
        if (over) atomicExch(ovf, 1);
        if (!out) {
            cnt[e] = m;
        } else {
            for (int q = 0; q < m; ++q) out[rp[e] + q] = cand[q];
        }
    }
}

// K and M values of row e: its elements in increasing order, each local row
// a of the element's matrices scattered by column (binary search in the row)
__global__ void k_row_values(int ne, const int* __restrict__ irp, const int* __restrict__ inc,
                             const int* __restrict__ te, const double* __restrict__ Ke,
                             const double* __restrict__ Me, const double* __restrict__ nu,
                             const double* __restrict__ kappa, const int* __restrict__ rp,
                             const int* __restrict__ ci, double* __restrict__ kv, double* __restrict__ mv) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const int r0 = rp[e], r1 = rp[e + 1];
        for (int q = r0; q < r1; ++q) kv[q] = mv[q] = 0.0;
        for (int k = irp[e]; k < irp[e + 1]; ++k) {
            const int t = inc[k] / 6, a = inc[k] % 6;
            const double cn = nu ? nu[t] : 1.0, ck = kappa ? kappa[t] : 1.0;
            for (int b = 0; b < 6; ++b) {
                const int c = te[(size_t)t * 6 + b];
                int lo = r0, hi = r1 - 1;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (ci[mid] < c) lo = mid + 1;
                    else hi = mid;
                }
                kv[lo] += cn * Ke[(size_t)t * 36 + a * 6 + b];
                mv[lo] += ck * Me[(size_t)t * 36 + a * 6 + b];
            }
        }
    }
}

// G: row e = (lo, hi) holds -1 at lo and +1 at hi
__global__ void k_gradient(int ne, const int* __restrict__ ev, int* __restrict__ rp, int* __restrict__ ci,
                           double* __restrict__ v) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        rp[e] = 2 * e;
        if (e == ne - 1) rp[ne] = 2 * ne;
        ci[2 * e] = ev[2 * e];
        ci[2 * e + 1] = ev[2 * e + 1];
        v[2 * e] = -1.0;
        v[2 * e + 1] = 1.0;
    }
}

// an ssv_matrix handle around device CSR arrays (the pattern also kept on the host)
ssv_matrix* wrap_matrix(int rows, int cols, int64_t nnz, DevBuf<int>&& rp, DevBuf<int>&& ci, DevBuf<double>&& v,
                        cudaStream_t s) {
    auto* M = new ssv_matrix();
    M->rows = rows;
    M->cols = cols;
    M->nnz = nnz;
    M->dtype = SSV_F64;
    M->h_rp.resize(rows + 1);
    M->h_ci.resize(nnz);
    SSV_CUDA(cudaMemcpyAsync(M->h_rp.data(), rp.get(), sizeof(int) * (rows + 1), cudaMemcpyDeviceToHost, s));
    if (nnz) SSV_CUDA(cudaMemcpyAsync(M->h_ci.data(), ci.get(), sizeof(int) * nnz, cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    M->rp = std::move(rp);
    M->ci = std::move(ci);
    M->val = std::move(v);
    M->lanes = pick_shape(rows, rows > 0 ? (double)nnz / rows : 1.0);
    return M;
}

}  // namespace

void hcurl_assemble(int nv, const double* xyz, int nt, const int* tets, const int* tet_edges, const int8_t* signs,
                    int ne, const int* edge_verts, const double* nu, const double* kappa, ssv_matrix** K,
                    ssv_matrix** M, ssv_matrix** G) {
    cudaStream_t s = stream();
    DevBuf<double> d_xyz((size_t)nv * 3), Ke((size_t)std::max(nt, 1) * 36), Me((size_t)std::max(nt, 1) * 36);
    DevBuf<int> d_tets((size_t)std::max(nt, 1) * 4), d_te((size_t)std::max(nt, 1) * 6), d_ev((size_t)std::max(ne, 1) * 2);
    DevBuf<int8_t> d_sg((size_t)std::max(nt, 1) * 6);
    DevBuf<double> d_nu, d_ka;
    d_xyz.upload(xyz, (size_t)nv * 3, s);
    d_tets.upload(tets, (size_t)nt * 4, s);
    d_te.upload(tet_edges, (size_t)nt * 6, s);
    d_sg.upload(signs, (size_t)nt * 6, s);
    d_ev.upload(edge_verts, (size_t)ne * 2, s);
    if (nu) d_nu.upload(nu, nt, s);
    if (kappa) d_ka.upload(kappa, nt, s);
    if (nt) k_element_matrices<<<grid_for(nt, 128), 128, 0, s>>>(nt, d_xyz.get(), d_tets.get(), d_sg.get(), Ke.get(),
                                                                  Me.get());
    // edge -> (element, local edge) incidence in element order
    DevBuf<int> cnt(std::max(ne, 1)), fill(std::max(ne, 1)), irp(ne + 1), inc((size_t)std::max(nt, 1) * 6);
    cnt.zero(s);
    fill.zero(s);
    if (nt) k_inc_count<<<grid_for((int64_t)nt * 6, 256), 256, 0, s>>>(nt, d_te.get(), cnt.get());
    if (sell_offsets(ne, cnt.get(), irp.get(), s) < 0)  // exclusive scan (sell.cuh)
        fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: too many element-edge incidences");
    if (nt) k_inc_fill<<<grid_for((int64_t)nt * 6, 256), 256, 0, s>>>(nt, d_te.get(), irp.get(), fill.get(), inc.get());
    if (ne) k_inc_sort<<<grid_for(ne, 128), 128, 0, s>>>(ne, irp.get(), inc.get());
    SSV_LAUNCH_CHECK();
    // pattern: count, scan, fill
    DevBuf<int> ovf(1), rcnt(std::max(ne, 1)), rp(ne + 1);
    ovf.zero(s);
    if (ne)
        k_row_pattern<<<grid_for(ne, 128), 128, 0, s>>>(ne, irp.get(), inc.get(), d_te.get(), rcnt.get(), nullptr,
                                                         nullptr, ovf.get());
    const int64_t nnz = sell_offsets(ne, rcnt.get(), rp.get(), s);
    int h_ovf = 0;
    SSV_CUDA(cudaMemcpyAsync(&h_ovf, ovf.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    if (h_ovf) fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: an edge has more than 384 neighbour candidates");
    if (nnz < 0) fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: more than 2^31 nonzeros");
    DevBuf<int> ci((size_t)std::max<int64_t>(nnz, 1)), ci2((size_t)std::max<int64_t>(nnz, 1)), rp2(ne + 1);
    DevBuf<double> kv((size_t)std::max<int64_t>(nnz, 1)), mv((size_t)std::max<int64_t>(nnz, 1));
    if (ne)
        k_row_pattern<<<grid_for(ne, 128), 128, 0, s>>>(ne, irp.get(), inc.get(), d_te.get(), nullptr, rp.get(),
                                                         ci.get(), ovf.get());
    if (ne)
        k_row_values<<<grid_for(ne, 128), 128, 0, s>>>(ne, irp.get(), inc.get(), d_te.get(), Ke.get(), Me.get(),
                                                        nu ? d_nu.get() : nullptr, kappa ? d_ka.get() : nullptr,
                                                        rp.get(), ci.get(), kv.get(), mv.get());
    SSV_LAUNCH_CHECK();
    SSV_CUDA(cudaMemcpyAsync(rp2.get(), rp.get(), sizeof(int) * (ne + 1), cudaMemcpyDeviceToDevice, s));
    if (nnz) SSV_CUDA(cudaMemcpyAsync(ci2.get(), ci.get(), sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
    DevBuf<int> grp(ne + 1), gci((size_t)std::max(ne, 1) * 2);
    DevBuf<double> gv((size_t)std::max(ne, 1) * 2);
    if (ne) k_gradient<<<grid_for(ne, 256), 256, 0, s>>>(ne, d_ev.get(), grp.get(), gci.get(), gv.get());
    else SSV_CUDA(cudaMemsetAsync(grp.get(), 0, sizeof(int), s));
    SSV_LAUNCH_CHECK();
    SSV_CUDA(cudaStreamSynchronize(s));
    std::unique_ptr<ssv_matrix> k(wrap_matrix(ne, ne, nnz, std::move(rp), std::move(ci), std::move(kv), s));
    std::unique_ptr<ssv_matrix> m(wrap_matrix(ne, ne, nnz, std::move(rp2), std::move(ci2), std::move(mv), s));
    std::unique_ptr<ssv_matrix> g(wrap_matrix(ne, nv, 2 * (int64_t)ne, std::move(grp), std::move(gci), std::move(gv), s));
    *K = k.release();
    *M = m.release();
    *G = g.release();
}

}  // namespace ssv
