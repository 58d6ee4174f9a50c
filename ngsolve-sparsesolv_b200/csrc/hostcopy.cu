// Host -> device copies of large pageable host arrays (matrix values re-read
// on every Solve, as the reference re-reads them): the copy runs through
// pinned staging buffers, several host threads filling them in parallel while
// the copy engine drains the previous chunk of each thread. A single pageable
// cudaMemcpy is bound by one thread's memcpy into the driver's own staging.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "objects.cuh"

namespace ssv {
namespace {

constexpr int kCopyThreads = 8;
constexpr size_t kChunk = size_t(4) << 20;
constexpr size_t kStagedMin = size_t(16) << 20;  // smaller copies go straight to cudaMemcpyAsync

struct PinnedPool {
    std::mutex mu;
    bool ready = false;
    void* buf[kCopyThreads][2] = {};
    cudaStream_t st[kCopyThreads] = {};
    cudaEvent_t ev[kCopyThreads][2] = {};
    cudaEvent_t start = nullptr;

    void init() {
        if (ready) return;
        for (int t = 0; t < kCopyThreads; ++t) {
            SSV_CUDA(cudaStreamCreateWithFlags(&st[t], cudaStreamNonBlocking));
            for (int k = 0; k < 2; ++k) {
                SSV_CUDA(cudaHostAlloc(&buf[t][k], kChunk, cudaHostAllocDefault));
                SSV_CUDA(cudaEventCreateWithFlags(&ev[t][k], cudaEventDisableTiming));
            }
        }
        SSV_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
        ready = true;
    }
};

PinnedPool& pool() {
    static PinnedPool* p = new PinnedPool();  // never destroyed: it may outlive the CUDA context at exit
    return *p;
}

}  // namespace

void h2d_staged(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    if (bytes < kStagedMin) {
        SSV_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return;
    }
    PinnedPool& P = pool();
    std::lock_guard<std::mutex> lock(P.mu);
    P.init();
    // the copies follow the work already queued on s
    SSV_CUDA(cudaEventRecord(P.start, s));
    for (int t = 0; t < kCopyThreads; ++t) SSV_CUDA(cudaStreamWaitEvent(P.st[t], P.start, 0));
    std::atomic<int> err{0};
    std::vector<std::thread> th;
    th.reserve(kCopyThreads);
    for (int t = 0; t < kCopyThreads; ++t) {
        th.emplace_back([&, t] {
            const size_t a = bytes * t / kCopyThreads, b = bytes * (t + 1) / kCopyThreads;
            int k = 0;
            for (size_t off = a; off < b; off += kChunk, ++k) {
                const size_t len = std::min(kChunk, b - off);
                const int slot = k & 1;
                cudaError_t e = cudaSuccess;
                if (k >= 2) e = cudaEventSynchronize(P.ev[t][slot]);  // this slot's previous copy is done
                if (e == cudaSuccess) {
                    std::memcpy(P.buf[t][slot], static_cast<const char*>(src) + off, len);
                    e = cudaMemcpyAsync(static_cast<char*>(dst) + off, P.buf[t][slot], len, cudaMemcpyHostToDevice,
                                        P.st[t]);
                }
                if (e == cudaSuccess) e = cudaEventRecord(P.ev[t][slot], P.st[t]);
                if (e != cudaSuccess) {
                    err.store((int)e);
                    return;
                }
            }
        });
    }
    for (auto& x : th) x.join();
    // the staging buffers are reused by the next call: wait for every copy
    for (int t = 0; t < kCopyThreads; ++t) SSV_CUDA(cudaStreamSynchronize(P.st[t]));
    if (err.load() != 0) SSV_CUDA((cudaError_t)err.load());
}

}  // namespace ssv
