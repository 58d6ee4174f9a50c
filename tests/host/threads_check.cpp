// Host check of csrc/host_threads.hpp: every job of run_threads runs, the
// exception of the lowest failing index reaches the caller after all threads
// joined, and WorkerThread hands its function's exception to join() (wait()
// does not rethrow). Prints "ok" and returns 0 on success.
#include <atomic>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "host_threads.hpp"

static int fails = 0;
#define CHECK(c)                                                         \
    do {                                                                 \
        if (!(c)) {                                                      \
            std::printf("check failed: %s (line %d)\n", #c, __LINE__);   \
            ++fails;                                                     \
        }                                                                \
    } while (0)

int main() {
    {  // no exception: every job ran once
        std::atomic<int> ran{0};
        ssv::run_threads(8, [&](int) { ran++; });
        CHECK(ran == 8);
    }
    {  // two jobs throw: all jobs still ran, the lowest index's exception is rethrown
        std::atomic<int> ran{0};
        std::string what;
        try {
            ssv::run_threads(6, [&](int i) {
                ran++;
                if (i == 4) throw std::runtime_error("job 4");
                if (i == 2) throw std::runtime_error("job 2");
            });
        } catch (const std::runtime_error& e) {
            what = e.what();
        }
        CHECK(ran == 6);
        CHECK(what == "job 2");
    }
    {  // a non-std exception type passes through unchanged
        bool caught = false;
        try {
            ssv::run_threads(3, [](int i) {
                if (i == 1) throw 7;
            });
        } catch (int v) {
            caught = v == 7;
        }
        CHECK(caught);
    }
    {  // WorkerThread: join rethrows, a second join does not
        ssv::WorkerThread t;
        t.start([] { throw std::runtime_error("worker"); });
        std::string what;
        try {
            t.join();
        } catch (const std::runtime_error& e) {
            what = e.what();
        }
        CHECK(what == "worker");
        bool second = false;
        try {
            t.join();
        } catch (...) {
            second = true;
        }
        CHECK(!second);
    }
    {  // WorkerThread: a clean run joins quietly; wait() does not rethrow
        ssv::WorkerThread t;
        int v = 0;
        t.start([&] { v = 42; });
        t.join();
        CHECK(v == 42);
        ssv::WorkerThread u;
        u.start([] { throw std::runtime_error("late"); });
        u.wait();  // clean-up path: no rethrow here
        CHECK(!u.joinable());
    }
    if (fails) return 1;
    std::printf("ok\n");
    return 0;
}
