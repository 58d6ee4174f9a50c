// noalloc.cu -- ssv_spmv_dot_noalloc: y = A x and x^T y without any device
// allocation, for callers that must not allocate device memory.
//
// Some callers can't call cudaMalloc: code that runs inside another
// framework's memory pool or under a strict memory budget, real-time
// loops where an allocation could block or fail mid-run, and host code that
// has handed all of the device's memory to its own allocator. This entry
// point takes every input and output from the caller and keeps its only
// scratch -- the per-CTA partial sums of the x^T y reduction and the counter
// that elects the CTA which adds them up -- in a fixed array compiled into
// the library.
//
// The scratch is a file-scope __device__ array: every GPU that loads this
// library holds it (about 512 KB) until the process exits, and every call on
// a device shares it. Calls whose kernels overlap on the GPU (e.g. from two
// host threads or two streams at once) race on it and give wrong results;
// serialise them. The array keeps the last call's contents, so the counter
// is cleared at the start of each call.
//
// Host code may not dereference or pass the array's name to a kernel: there
// it names a host-side stand-in, not device memory. Its device address is
// looked up with cudaGetSymbolAddress once per device, on the first call made
// with that device current (that first call should therefore come before any
// stream capture that includes this entry point). The address is kept for the
// life of the process: calls must not span a cudaDeviceReset (or any other
// teardown of the device's primary context), after which the module is
// reloaded elsewhere and the kept address is stale.
//
// Every pointer argument is checked to be device (or managed) memory with
// cudaPointerGetAttributes before anything is launched, as in the library's
// other _dev calls: a host pointer is refused with SSV_ERR_INVALID_ARG
// instead of reaching the kernel.
//
// The kernel runs on the legacy default stream and the call synchronises it
// before returning. A caller whose inputs were produced on a non-blocking
// stream must synchronise that stream (or the device) before the call.
#include <mutex>

#include "kernels.cuh"

namespace {

constexpr int kLanes = 8;                          // lanes per CSR row
constexpr int kRowsPerCta = ssv::kBlock / kLanes;  // 32 rows per CTA
constexpr int kMaxCtas = 65536;                    // one partial sum per CTA
constexpr long long kMaxRows = (long long)kMaxCtas * kRowsPerCta;  // 2,097,152 rows

// [0, kMaxCtas): per-CTA partial sums; [kMaxCtas]: completion counter.
static __device__ __align__(256) double g_noalloc_scratch[kMaxCtas + 32];

// One CTA per 32 rows (no grid-stride loop: CTA b owns partial b), 8 lanes
// per row; the last CTA to finish sums the partials in CTA order.
__global__ void __launch_bounds__(ssv::kBlock)
k_spmv_dot_noalloc(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                   const double* __restrict__ x, double* __restrict__ y, double* scratch, double* dot) {
    const int sub = threadIdx.x % kLanes;
    const int row = blockIdx.x * kRowsPerCta + threadIdx.x / kLanes;
    const bool valid = row < n;
    double acc = 0.0;
    if (valid)
        for (int k = rp[row] + sub; k < rp[row + 1]; k += kLanes) acc += v[k] * x[ci[k]];
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, kLanes);
    double2 part = make_double2(0.0, 0.0);
    if (sub == 0 && valid) {
        y[row] = acc;
        part.x = x[row] * acc;
    }
    unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + kMaxCtas);
    __shared__ bool am_last;
    part = ssv::block_sum2(part);
    if (threadIdx.x == 0) {
        scratch[blockIdx.x] = part.x;
        __threadfence();
        am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    double2 s = make_double2(0.0, 0.0);
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s.x += __ldcg(&scratch[b]);
    s = ssv::block_sum2(s);
    if (threadIdx.x == 0) {
        *dot = s.x;
        *ticket = 0u;
    }
}

std::mutex g_mu;
double* g_addr[64] = {};

}  // namespace

extern "C" int ssv_spmv_dot_noalloc(int32_t rows, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                    const double* d_values, const double* d_x, double* d_y, double* d_dot);

namespace ssv {
const char* noalloc_set_error(const std::string& m);
}

namespace {
// true when p is device or managed memory (cudaPointerGetAttributes
// allocates nothing)
bool is_device_ptr(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}
}  // namespace

extern "C" int ssv_spmv_dot_noalloc(int32_t rows, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                    const double* d_values, const double* d_x, double* d_y, double* d_dot) {
    if (rows < 0 || !d_row_ptr || !d_x || !d_y || !d_dot || (rows > 0 && (!d_col_idx || !d_values))) {
        ssv::noalloc_set_error("ssv_spmv_dot_noalloc: negative size or NULL pointer");
        return SSV_ERR_INVALID_ARG;
    }
    if ((long long)rows > kMaxRows) {
        ssv::noalloc_set_error("ssv_spmv_dot_noalloc: " + std::to_string(rows) +
                               " rows exceed the maximum of 2097152 (the fixed scratch holds 65536 CTA "
                               "partial sums of 32 rows each); use ssv_matrix_spmv_dev instead");
        return SSV_ERR_INVALID_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        ssv::noalloc_set_error(std::string("ssv_spmv_dot_noalloc: no usable CUDA device: ") + cudaGetErrorString(e));
        return SSV_ERR_NO_DEVICE;
    }
    {
        const void* ptrs[6] = {d_row_ptr, d_col_idx, d_values, d_x, d_y, d_dot};
        const char* names[6] = {"d_row_ptr", "d_col_idx", "d_values", "d_x", "d_y", "d_dot"};
        for (int k = 0; k < 6; ++k) {
            if (!ptrs[k]) continue;  // NULL col_idx / values are allowed for rows == 0
            if (!is_device_ptr(ptrs[k])) {
                ssv::noalloc_set_error(std::string("ssv_spmv_dot_noalloc: ") + names[k] +
                                       " is not device memory (every pointer must be a device address)");
                return SSV_ERR_INVALID_ARG;
            }
        }
    }
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {  // set-up: once per device, with that device current
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                ssv::noalloc_set_error(std::string("ssv_spmv_dot_noalloc: cudaGetSymbolAddress failed: ") +
                                       cudaGetErrorString(e));
                return SSV_ERR_CUDA;
            }
            g_addr[dev] = static_cast<double*>(p);
        }
        scratch = g_addr[dev];
    }
    // the array keeps the previous call's contents: clear the counter
    e = cudaMemsetAsync(scratch + kMaxCtas, 0, sizeof(unsigned int), 0);
    if (e == cudaSuccess && rows > 0) {
        const int grid = (rows + kRowsPerCta - 1) / kRowsPerCta;
        k_spmv_dot_noalloc<<<grid, ssv::kBlock, 0, 0>>>(rows, d_row_ptr, d_col_idx, d_values, d_x, d_y, scratch,
                                                        d_dot);
        e = cudaGetLastError();
    } else if (e == cudaSuccess) {
        e = cudaMemsetAsync(d_dot, 0, sizeof(double), 0);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        ssv::noalloc_set_error(std::string("ssv_spmv_dot_noalloc: ") + cudaGetErrorString(e));
        return SSV_ERR_CUDA;
    }
    ssv::noalloc_set_error("");
    return SSV_OK;
}
