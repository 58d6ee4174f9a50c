// sell.cu -- see sell.cuh: the sliced-ELL layout built on the device.
#include <algorithm>

#include "sell.cuh"

namespace ssv {
namespace {

// in each window of kSellWindow rows, the rows sorted by length, longest
// first, ties in row order (a stable rank per row)
__global__ void __launch_bounds__(kSellWindow) k_sell_order(int n, const int* __restrict__ rp, int* __restrict__ order) {
    __shared__ int len[kSellWindow];
    const int w0 = blockIdx.x * kSellWindow, t = threadIdx.x;
    const int m = min(kSellWindow, n - w0);
    if (t < m) len[t] = rp[w0 + t + 1] - rp[w0 + t];
    __syncthreads();
    if (t < m) {
        int r = 0;
        for (int j = 0; j < m; ++j) r += (len[j] > len[t]) || (len[j] == len[t] && j < t);
        order[w0 + r] = w0 + t;
    }
}

// rows of each slice and its padded width (32 x its longest row)
__global__ void k_sell_width(int n, int slices, const int* __restrict__ rp, const int* __restrict__ order,
                             int* __restrict__ rows, int* __restrict__ width) {
    for (int sl = blockIdx.x * blockDim.x + threadIdx.x; sl < slices; sl += gridDim.x * blockDim.x) {
        int w = 0;
        for (int t = 0; t < 32; ++t) {
            const int q = sl * 32 + t;
            const int r = q < n ? order[q] : -1;
            rows[q] = r;
            if (r >= 0) w = max(w, rp[r + 1] - rp[r]);
        }
        width[sl] = 32 * w;
    }
}

__global__ void k_sell_fill(int slices, const int* __restrict__ rp, const int* __restrict__ ci,
                            const int* __restrict__ rows, const int* __restrict__ off, int* __restrict__ sci,
                            int* __restrict__ src) {
    const int64_t total = (int64_t)slices * 32;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int r = rows[q];
        if (r < 0) continue;
        const int sl = (int)(q / 32), t = (int)(q % 32);
        const int k0 = rp[r], len = rp[r + 1] - k0;
        for (int k = 0; k < len; ++k) {
            const size_t e = (size_t)off[sl] + 32 * (size_t)k + t;
            sci[e] = ci[k0 + k];
            src[e] = k0 + k;
        }
    }
}

template <int W>
__global__ void k_sell_gather(int64_t entries, const int* __restrict__ src, const double* __restrict__ csr_v,
                              double* __restrict__ v) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < entries; e += (int64_t)gridDim.x * blockDim.x) {
        const int k = src[e];
#pragma unroll
        for (int w = 0; w < W; ++w) v[(size_t)e * W + w] = k >= 0 ? csr_v[(size_t)k * W + w] : 0.0;
    }
}

}  // namespace

bool SellPattern::build_pattern(int n, int64_t nnz, const int* rp, const int* a_ci, cudaStream_t s) {
    invalidate();  // until every array below is in place
    const int nsl = (n + 31) / 32;
    DevBuf<int> order(std::max(n, 1)), width(std::max(nsl, 1));
    off.alloc(nsl + 1);
    rows.alloc((size_t)std::max(nsl, 1) * 32);
    if (n) {
        k_sell_order<<<(n + kSellWindow - 1) / kSellWindow, kSellWindow, 0, s>>>(n, rp, order.get());
        k_sell_width<<<grid_for(nsl, 128), 128, 0, s>>>(n, nsl, rp, order.get(), rows.get(), width.get());
        SSV_LAUNCH_CHECK();
    }
    const int total = sell_offsets(nsl, width.get(), off.get(), s);
    if (total < 0) return false;  // int offsets would overflow: no copy
    const size_t cap = (size_t)std::max(total, 1);
    ci.alloc(cap);
    src.alloc(cap);
    SSV_CUDA(cudaMemsetAsync(ci.get(), 0xff, sizeof(int) * cap, s));  // -1: padding
    SSV_CUDA(cudaMemsetAsync(src.get(), 0xff, sizeof(int) * cap, s));
    if (nsl)
        k_sell_fill<<<grid_for((int64_t)nsl * 32, 256), 256, 0, s>>>(nsl, rp, a_ci, rows.get(), off.get(), ci.get(),
                                                                     src.get());
    SSV_LAUNCH_CHECK();
    SSV_CUDA(cudaStreamSynchronize(s));  // the temporaries go out of scope
    slices = nsl;
    entries = total;
    pat_n = n;
    pat_nnz = nnz;
    return true;
}

void sell_gather(const SellPattern& P, const double* csr_v, int words, double* v, cudaStream_t s) {
    if (P.slices <= 0 || P.entries <= 0) return;
    if (words == 2)
        k_sell_gather<2><<<grid_for(P.entries, 256), 256, 0, s>>>(P.entries, P.src.get(), csr_v, v);
    else
        k_sell_gather<1><<<grid_for(P.entries, 256), 256, 0, s>>>(P.entries, P.src.get(), csr_v, v);
    SSV_LAUNCH_CHECK();
}

}  // namespace ssv
