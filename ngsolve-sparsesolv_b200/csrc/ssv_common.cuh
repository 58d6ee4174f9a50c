// ssv_common.cuh -- shared definitions of the B200 solve path: scalar types,
// error plumbing, device buffers and the launch geometry of B200 (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sparsesolv_b200.h"

namespace ssv {

// ---------------------------------------------------------------------------
// Errors: C++ exceptions inside the library, status codes at the C ABI.
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        int code = (e == cudaErrorMemoryAllocation) ? SSV_ERR_ALLOC
                 : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? SSV_ERR_NO_DEVICE
                 : SSV_ERR_CUDA;
        fail(code, std::string("CUDA error in ") + what + " (" + file + ":" + std::to_string(line) +
                       "): " + cudaGetErrorString(e));
    }
}
#define SSV_CUDA(call) ::ssv::cuda_check((call), #call, __FILE__, __LINE__)
#define SSV_LAUNCH_CHECK() ::ssv::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// ---------------------------------------------------------------------------
// Scalars. zdouble has the layout of std::complex<double> (two doubles,
// 16-byte aligned so a pair moves in one 128-bit load).
// ---------------------------------------------------------------------------
struct __align__(16) zdouble {
    double x, y;
};
struct __align__(8) zfloat {
    float x, y;
};

__host__ __device__ inline zdouble operator+(zdouble a, zdouble b) { return {a.x + b.x, a.y + b.y}; }
__host__ __device__ inline zdouble operator-(zdouble a, zdouble b) { return {a.x - b.x, a.y - b.y}; }
__host__ __device__ inline zdouble operator-(zdouble a) { return {-a.x, -a.y}; }
__host__ __device__ inline zdouble operator*(zdouble a, zdouble b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__host__ __device__ inline zdouble operator*(double s, zdouble a) { return {s * a.x, s * a.y}; }
__host__ __device__ inline zdouble& operator+=(zdouble& a, zdouble b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ inline zdouble& operator-=(zdouble& a, zdouble b) { a.x -= b.x; a.y -= b.y; return a; }
__host__ __device__ inline zfloat operator+(zfloat a, zfloat b) { return {a.x + b.x, a.y + b.y}; }
__host__ __device__ inline zfloat operator-(zfloat a, zfloat b) { return {a.x - b.x, a.y - b.y}; }
__host__ __device__ inline zfloat operator*(zfloat a, zfloat b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__host__ __device__ inline zfloat& operator+=(zfloat& a, zfloat b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ inline zfloat& operator-=(zfloat& a, zfloat b) { a.x -= b.x; a.y -= b.y; return a; }

// Complex division with the scaling of Smith's method (numerically safe for
// the magnitudes met in Krylov recurrences).
__host__ __device__ inline zdouble zdiv(zdouble a, zdouble b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return {(a.x + a.y * r) / d, (a.y - a.x * r) / d};
    } else {
        double r = b.x / b.y, d = b.x * r + b.y;
        return {(a.x * r + a.y) / d, (a.y * r - a.x) / d};
    }
}

// Scalar traits: one code path for double and complex<double>.
template <typename S> struct ST;
template <> struct ST<double> {
    using lo = float;  // storage type of the FP32 preconditioner form
    static constexpr bool cplx = false;
    __host__ __device__ static double zero() { return 0.0; }
    __host__ __device__ static double one() { return 1.0; }
    __host__ __device__ static double real(double a) { return a; }
    __host__ __device__ static double from(double a) { return a; }
    __host__ __device__ static double conj(double a) { return a; }
    __host__ __device__ static double norm2(double a) { return a * a; }
    __host__ __device__ static double abs(double a) { return fabs(a); }
    __host__ __device__ static double div(double a, double b) { return a / b; }
    __host__ __device__ static double scale(double s, double a) { return s * a; }
    __host__ __device__ static double fma(double a, double b, double c) { return a * b + c; }
    __host__ __device__ static double to_d2_x(double a) { return a; }
};
template <> struct ST<zdouble> {
    using lo = zfloat;
    static constexpr bool cplx = true;
    __host__ __device__ static zdouble zero() { return {0.0, 0.0}; }
    __host__ __device__ static zdouble one() { return {1.0, 0.0}; }
    __host__ __device__ static double real(zdouble a) { return a.x; }
    __host__ __device__ static zdouble from(double a) { return {a, 0.0}; }
    __host__ __device__ static zdouble conj(zdouble a) { return {a.x, -a.y}; }
    __host__ __device__ static double norm2(zdouble a) { return a.x * a.x + a.y * a.y; }
    __host__ __device__ static double abs(zdouble a) { return hypot(a.x, a.y); }
    __host__ __device__ static zdouble div(zdouble a, zdouble b) { return zdiv(a, b); }
    __host__ __device__ static zdouble scale(double s, zdouble a) { return {s * a.x, s * a.y}; }
    __host__ __device__ static zdouble fma(zdouble a, zdouble b, zdouble c) { return a * b + c; }
};

// Conversions between the FP64 and FP32 forms.
__host__ __device__ inline float lo_of(double a) { return (float)a; }
__host__ __device__ inline zfloat lo_of(zdouble a) { return {(float)a.x, (float)a.y}; }
__host__ __device__ inline double hi_of(float a) { return (double)a; }
__host__ __device__ inline zdouble hi_of(zfloat a) { return {(double)a.x, (double)a.y}; }
// Widen a stored coefficient (FP64 or FP32 form) to the arithmetic type.
__host__ __device__ inline double hi_of_any(double a) { return a; }
__host__ __device__ inline double hi_of_any(float a) { return (double)a; }
__host__ __device__ inline zdouble hi_of_any(zdouble a) { return a; }
__host__ __device__ inline zdouble hi_of_any(zfloat a) { return {(double)a.x, (double)a.y}; }

// ---------------------------------------------------------------------------
// Device memory
// ---------------------------------------------------------------------------
// While a thread has an allocation stream set (AllocScope), its DevBuf
// allocations are stream-ordered on it (cudaMallocAsync / cudaFreeAsync from
// the device's default pool): no device-wide synchronisation per free, so
// host threads that each build one part of a set-up on their own stream do
// not serialise on their temporaries. A buffer allocated that way and freed
// outside such a scope is freed by cudaFree (which waits for the device).
inline cudaStream_t& alloc_stream() {
    thread_local cudaStream_t s = nullptr;
    return s;
}
struct AllocScope {
    cudaStream_t prev;
    explicit AllocScope(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
    ~AllocScope() { alloc_stream() = prev; }
    AllocScope(const AllocScope&) = delete;
    AllocScope& operator=(const AllocScope&) = delete;
};

// Device-allocation budget (the test hook ssv_set_alloc_budget): negative =
// no limit; otherwise every device allocation is charged against it, and one
// that does not fit fails with SSV_ERR_ALLOC before cudaMalloc is called, so
// the failure paths of set-up and solves run without exhausting the GPU.
inline std::atomic<long long>& alloc_budget() {
    static std::atomic<long long> b{-1};
    return b;
}
inline void charge_alloc(size_t bytes) {
    std::atomic<long long>& b = alloc_budget();
    long long cur = b.load(std::memory_order_relaxed);
    while (cur >= 0) {
        if ((long long)bytes > cur)
            fail(SSV_ERR_ALLOC, "device allocation of " + std::to_string(bytes) +
                                    " bytes refused: over the allocation budget (ssv_set_alloc_budget)");
        if (b.compare_exchange_weak(cur, cur - (long long)bytes, std::memory_order_relaxed)) return;
    }
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    bool pooled = false;  // from cudaMallocAsync
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), pooled(o.pooled) { o.p = nullptr; o.n = 0; o.pooled = false; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p; n = o.n; pooled = o.pooled;
            o.p = nullptr; o.n = 0; o.pooled = false;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count) {
        if (count == n && p) return;
        release();
        if (!count) return;
        charge_alloc(sizeof(T) * count);
        T* q = nullptr;
        if (cudaStream_t as = alloc_stream()) {
            SSV_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&q), sizeof(T) * count, as));
            pooled = true;
        } else {
            SSV_CUDA(cudaMalloc(&q, sizeof(T) * count));
        }
        p = q;
        n = count;  // only once the memory is there: a failed alloc leaves an empty buffer
    }
    void release() {
        if (p) {
            if (pooled && alloc_stream()) cudaFreeAsync(p, alloc_stream());
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
        pooled = false;
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        alloc(count);
        if (count) SSV_CUDA(cudaMemcpyAsync(p, h, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    }
    void zero(cudaStream_t s) {
        if (n) SSV_CUDA(cudaMemsetAsync(p, 0, sizeof(T) * n, s));
    }
    T* get() const { return p; }
    size_t size() const { return n; }
};

// Launch geometry: 148 SMs on B200; grids are sized in multiples of the SM
// count (queried once) for grid-stride kernels.
int sm_count();
inline int grid_for(int64_t work, int block, int per_sm = 8) {
    int64_t g = (work + block - 1) / block;
    int64_t cap = (int64_t)sm_count() * per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

double wall_seconds();

}  // namespace ssv
