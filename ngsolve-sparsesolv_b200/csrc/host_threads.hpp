// host_threads.hpp -- host worker threads whose exceptions reach the caller.
// A C++ exception that leaves a std::thread's function ends the process
// (std::terminate); the set-up's worker threads instead hand theirs to the
// thread that joins them, so a failed allocation or a refused input inside a
// worker becomes the status code of the C-ABI call like anywhere else.
#pragma once

#include <exception>
#include <system_error>
#include <thread>
#include <utility>
#include <vector>

namespace ssv {

// Runs job(i) for i in [0, n) on n host threads and joins them all; then the
// exception of the lowest i whose job threw, if any, is rethrown here. A job
// whose thread cannot be started runs on the calling thread instead.
template <typename F>
void run_threads(int n, F&& job) {
    std::vector<std::exception_ptr> err(n > 0 ? n : 0);
    std::vector<std::thread> th;
    th.reserve(err.size());
    auto guarded = [&](int i) {
        try {
            job(i);
        } catch (...) {
            err[i] = std::current_exception();
        }
    };
    for (int i = 0; i < n; ++i) {
        try {
            th.emplace_back(guarded, i);
        } catch (const std::system_error&) {
            guarded(i);
        }
    }
    for (auto& t : th) t.join();
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

// A single background thread whose exception is kept for the joiner:
// start(f) runs f on a new thread, join() waits and rethrows what f threw.
class WorkerThread {
public:
    WorkerThread() = default;
    WorkerThread(const WorkerThread&) = delete;
    WorkerThread& operator=(const WorkerThread&) = delete;
    ~WorkerThread() {
        if (t_.joinable()) t_.join();
    }
    template <typename F>
    void start(F&& f) {
        wait();
        err_ = nullptr;
        t_ = std::thread([this, g = std::forward<F>(f)]() mutable {
            try {
                g();
            } catch (...) {
                err_ = std::current_exception();
            }
        });
    }
    bool joinable() const { return t_.joinable(); }
    // waits for the thread; does not rethrow (for clean-up paths)
    void wait() {
        if (t_.joinable()) t_.join();
    }
    // waits for the thread and rethrows the exception its function threw
    void join() {
        wait();
        if (err_) {
            std::exception_ptr e = err_;
            err_ = nullptr;
            std::rethrow_exception(e);
        }
    }

private:
    std::thread t_;
    std::exception_ptr err_;
};

}  // namespace ssv
