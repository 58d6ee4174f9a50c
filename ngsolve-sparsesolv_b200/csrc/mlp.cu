// mlp.cu -- the learned initial-guess predictor (new: no reference
// counterpart): a 2-layer per-edge MLP, out = w2 . relu(W1 x + b1) + b2,
// FP32, trained and evaluated by the kernels below.
//
// Parameters live in one FP32 array: W1 (H x D, row-major), b1 (H), w2 (H),
// b2 (1). Training minimises the mean squared error over a minibatch with
// Adam. Gradients are summed deterministically: each block writes its partial
// gradient, a second kernel adds the partials in block order.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "objects.cuh"
#include "solver_api.hpp"

namespace ssv {

constexpr int kMlpBlock = 256;
constexpr int kMlpMaxD = 32;
constexpr int kMlpMaxH = 128;

struct MlpDims {
    int D, H;
    __host__ __device__ int nw1() const { return H * D; }
    __host__ __device__ int nparams() const { return H * D + 2 * H + 1; }
};

// out[i] = MLP(X[i]) for n samples (X row-major n x D)
__global__ void __launch_bounds__(kMlpBlock)
k_mlp_forward(MlpDims dm, const float* __restrict__ P, const float* __restrict__ X, int64_t n, float* __restrict__ out) {
    extern __shared__ float sp[];
    const int np = dm.nparams();
    for (int k = threadIdx.x; k < np; k += blockDim.x) sp[k] = P[k];
    __syncthreads();
    const float* W1 = sp;
    const float* b1 = sp + dm.nw1();
    const float* w2 = b1 + dm.H;
    const float b2 = w2[dm.H];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float x[kMlpMaxD];
        for (int d = 0; d < dm.D; ++d) x[d] = X[i * dm.D + d];
        float o = b2;
        for (int j = 0; j < dm.H; ++j) {
            float a = b1[j];
            const float* wr = W1 + j * dm.D;
            for (int d = 0; d < dm.D; ++d) a = fmaf(wr[d], x[d], a);
            o = fmaf(w2[j], fmaxf(a, 0.f), o);
        }
        out[i] = o;
    }
}

// Per-block partial gradient of L = (1/m) sum_i (MLP(x_i) - y_i)^2 over the
// samples idx[0..m) (or 0..m when idx is null), plus the partial loss.
// partial: gridDim.x rows of (nparams + 1) floats. One sample per thread and
// pass; each warp folds its 32 samples with shuffles into its own shared row,
// the rows are added in warp order at the end (no atomics: deterministic).
__global__ void __launch_bounds__(kMlpBlock)
k_mlp_grad_partial(MlpDims dm, const float* __restrict__ P, const float* __restrict__ X, const float* __restrict__ Y,
                   const int64_t* __restrict__ idx, int64_t m, float* __restrict__ partial) {
    extern __shared__ float sh[];
    const int np = dm.nparams();
    const int np1 = np + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    float* sp = sh;                  // parameters
    float* rows = sh + np;           // nwarps rows of np + 1 (last = loss)
    for (int k = threadIdx.x; k < np; k += blockDim.x) sp[k] = P[k];
    for (int k = threadIdx.x; k < nwarps * np1; k += blockDim.x) rows[k] = 0.f;
    __syncthreads();
    const float* W1 = sp;
    const float* b1 = sp + dm.nw1();
    const float* w2 = b1 + dm.H;
    const float b2 = w2[dm.H];
    float* my = rows + warp * np1;
    float* gW1 = my;
    float* gb1 = my + dm.nw1();
    float* gw2 = gb1 + dm.H;
    float* gb2 = gw2 + dm.H;
    float* gl = gb2 + 1;
    const float inv_m = 1.0f / (float)m;
    auto wsum = [](float v) {
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        return v;
    };
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < m; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = base + threadIdx.x;
        const bool valid = t < m;
        float x[kMlpMaxD];
        float pre[kMlpMaxH];
        float o = b2, y = 0.f;
        if (valid) {
            const int64_t i = idx ? idx[t] : t;
            for (int d = 0; d < dm.D; ++d) x[d] = X[i * dm.D + d];
            y = Y[i];
            for (int j = 0; j < dm.H; ++j) {
                float a = b1[j];
                const float* wr = W1 + j * dm.D;
                for (int d = 0; d < dm.D; ++d) a = fmaf(wr[d], x[d], a);
                pre[j] = a;
                o = fmaf(w2[j], fmaxf(a, 0.f), o);
            }
        } else {
            for (int d = 0; d < dm.D; ++d) x[d] = 0.f;
            for (int j = 0; j < dm.H; ++j) pre[j] = 0.f;
        }
        const float e = valid ? (o - y) : 0.f;
        const float g = 2.f * e * inv_m;  // dL/dout
        float sv = wsum(e * e * inv_m);
        if (lane == 0) gl[0] += sv;
        sv = wsum(g);
        if (lane == 0) gb2[0] += sv;
        for (int j = 0; j < dm.H; ++j) {
            sv = wsum(g * fmaxf(pre[j], 0.f));
            if (lane == 0) gw2[j] += sv;
            const float gh = (pre[j] > 0.f) ? g * w2[j] : 0.f;
            sv = wsum(gh);
            if (lane == 0) gb1[j] += sv;
            for (int d = 0; d < dm.D; ++d) {
                sv = wsum(gh * x[d]);
                if (lane == 0) gW1[j * dm.D + d] += sv;
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < np1; k += blockDim.x) {
        float acc = 0.f;
        for (int w = 0; w < nwarps; ++w) acc += rows[w * np1 + k];
        partial[(size_t)blockIdx.x * np1 + k] = acc;
    }
}

// grad[k] = sum over blocks of partial[b][k], in block order
__global__ void k_mlp_grad_reduce(int np1, int blocks, const float* __restrict__ partial, float* __restrict__ grad) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np1; k += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int b = 0; b < blocks; ++b) s += partial[(size_t)b * np1 + k];
        grad[k] = s;
    }
}

// Adam (Kingma & Ba 2015) with bias correction
__global__ void k_mlp_adam(int np, float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M,
                           float* __restrict__ V, float lr, float b1, float b2, float eps, int t) {
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
        const float g = G[k];
        const float m = b1 * M[k] + (1.f - b1) * g;
        const float v = b2 * V[k] + (1.f - b2) * g * g;
        M[k] = m;
        V[k] = v;
        P[k] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    }
}

}  // namespace ssv

using ssv::DevBuf;

struct ssv_mlp {
    ssv::MlpDims dm{0, 0};
    DevBuf<float> P, G, M, V, partial;
    DevBuf<int64_t> idx;
    int step = 0;
    int grad_blocks = 0;
};

namespace ssv {

static size_t grad_smem(const MlpDims& dm) {
    return sizeof(float) * ((size_t)dm.nparams() + (size_t)(kMlpBlock / 32) * (dm.nparams() + 1));
}

ssv_mlp* mlp_create(int D, int H, uint64_t seed) {
    if (D < 1 || D > kMlpMaxD || H < 1 || H > kMlpMaxH)
        fail(SSV_ERR_INVALID_ARG, "mlp: input width must be 1..32 and hidden width 1..128");
    auto* m = new ssv_mlp();
    try {
        m->dm = MlpDims{D, H};
        const int np = m->dm.nparams();
        // He-uniform first layer, small second layer, zero biases
        std::mt19937_64 rng(seed);
        std::uniform_real_distribution<float> u1(-std::sqrt(6.f / D), std::sqrt(6.f / D));
        std::uniform_real_distribution<float> u2(-1.f / std::sqrt((float)H), 1.f / std::sqrt((float)H));
        std::vector<float> p(np, 0.f);
        for (int k = 0; k < H * D; ++k) p[k] = u1(rng);
        for (int j = 0; j < H; ++j) p[H * D + H + j] = u2(rng);
        cudaStream_t s = stream();
        m->P.upload(p.data(), np, s);
        m->G.alloc(np + 1);
        m->M.alloc(np);
        m->V.alloc(np);
        m->M.zero(s);
        m->V.zero(s);
        m->grad_blocks = sm_count() * 2;
        m->partial.alloc((size_t)m->grad_blocks * (np + 1));
        const size_t smem = grad_smem(m->dm);
        if (smem > 48 * 1024)
            SSV_CUDA(cudaFuncSetAttribute(k_mlp_grad_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        SSV_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        delete m;
        throw;
    }
    return m;
}

void mlp_destroy(ssv_mlp* m) { delete m; }

int mlp_nparams(const ssv_mlp* m) { return m->dm.nparams(); }

void mlp_get_params(const ssv_mlp* m, float* p) {
    SSV_CUDA(cudaMemcpy(p, m->P.get(), sizeof(float) * m->dm.nparams(), cudaMemcpyDeviceToHost));
}

void mlp_set_params(ssv_mlp* m, const float* p) {
    m->P.upload(p, m->dm.nparams(), stream());
    m->M.zero(stream());
    m->V.zero(stream());
    m->step = 0;
    SSV_CUDA(cudaStreamSynchronize(stream()));
}

// gradient (and loss) of the mean squared error over samples idx (or all)
static void grad_dev(ssv_mlp* m, const float* X, const float* Y, const int64_t* idx, int64_t cnt, cudaStream_t s) {
    const int np = m->dm.nparams();
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(m->grad_blocks, (cnt + kMlpBlock - 1) / kMlpBlock));
    k_mlp_grad_partial<<<blocks, kMlpBlock, grad_smem(m->dm), s>>>(m->dm, m->P.get(), X, Y, idx, cnt,
                                                                   m->partial.get());
    k_mlp_grad_reduce<<<(np + 1 + 255) / 256, 256, 0, s>>>(np + 1, blocks, m->partial.get(), m->G.get());
    SSV_LAUNCH_CHECK();
}

void mlp_gradients_host(ssv_mlp* m, const float* X, const float* Y, int64_t n, float* grad, float* loss) {
    cudaStream_t s = stream();
    const int D = m->dm.D, np = m->dm.nparams();
    DevBuf<float> dX, dY;
    dX.upload(X, (size_t)n * D, s);
    dY.upload(Y, (size_t)n, s);
    grad_dev(m, dX.get(), dY.get(), nullptr, n, s);
    std::vector<float> g(np + 1);
    SSV_CUDA(cudaMemcpyAsync(g.data(), m->G.get(), sizeof(float) * (np + 1), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    std::memcpy(grad, g.data(), sizeof(float) * np);
    if (loss) *loss = g[np];
}

// Minibatch Adam over (X, Y) resident on the device: `epochs` passes, each a
// fresh permutation (host mt19937_64(seed + epoch)) cut into batches.
void mlp_train_dev(ssv_mlp* m, const float* X, const float* Y, int64_t n, int epochs, int batch, float lr,
                   uint64_t seed, float* last_loss) {
    if (n <= 0 || batch <= 0 || epochs < 0) fail(SSV_ERR_INVALID_ARG, "mlp train: empty data or bad batch");
    cudaStream_t s = stream();
    const int np = m->dm.nparams();
    m->idx.alloc((size_t)n);
    std::vector<int64_t> perm(n);
    float loss = 0.f;
    for (int e = 0; e < epochs; ++e) {
        for (int64_t i = 0; i < n; ++i) perm[i] = i;
        std::mt19937_64 rng(seed + (uint64_t)e);
        std::shuffle(perm.begin(), perm.end(), rng);
        SSV_CUDA(cudaMemcpyAsync(m->idx.get(), perm.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice, s));
        for (int64_t b0 = 0; b0 < n; b0 += batch) {
            const int64_t cnt = std::min<int64_t>(batch, n - b0);
            grad_dev(m, X, Y, m->idx.get() + b0, cnt, s);
            ++m->step;
            k_mlp_adam<<<(np + 255) / 256, 256, 0, s>>>(np, m->P.get(), m->G.get(), m->M.get(), m->V.get(), lr, 0.9f,
                                                        0.999f, 1e-8f, m->step);
            SSV_LAUNCH_CHECK();
        }
        // host copy of perm must outlive the async copy: wait before the next shuffle
        SSV_CUDA(cudaMemcpyAsync(&loss, m->G.get() + np, sizeof(float), cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
    }
    if (last_loss) *last_loss = loss;
}

void mlp_predict_dev(ssv_mlp* m, const float* X, int64_t n, float* out) {
    cudaStream_t s = stream();
    const size_t smem = sizeof(float) * m->dm.nparams();
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + kMlpBlock - 1) / kMlpBlock, sm_count() * 8));
    k_mlp_forward<<<grid, kMlpBlock, smem, s>>>(m->dm, m->P.get(), X, n, out);
    SSV_LAUNCH_CHECK();
    SSV_CUDA(cudaStreamSynchronize(s));
}

}  // namespace ssv
