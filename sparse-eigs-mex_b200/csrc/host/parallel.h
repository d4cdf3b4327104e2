// Host fork-join helpers for the per-call setup work (pattern checks,
// symbolic analysis, task lists): static ranges on short-lived threads, used
// only where the work is large enough to pay for starting them.
#pragma once

#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <exception>
#include <mutex>
#include <thread>
#include <utility>
#include <vector>

namespace spx {

inline unsigned host_threads() {
    const unsigned hw = std::thread::hardware_concurrency();
    return std::max(1u, std::min(hw, 32u));
}

// Threads started with run() and joined by wait(), which rethrows the first
// exception any of them raised (std::bad_alloc from a side thread reaches
// the caller's handler as if the work had run on the calling thread).  The
// destructor joins whatever is still running.  A group made with
// threads = false runs each callable at once on the calling thread (small
// inputs, where starting a thread costs more than the work).
class TaskGroup {
public:
    explicit TaskGroup(bool threads = true) : threads_(threads) {}
    template <class F>
    void run(F &&f) {
        if (!threads_) {
            f();
            return;
        }
        th_.emplace_back([this, fn = std::forward<F>(f)]() mutable {
            try {
                fn();
            } catch (...) {
                std::lock_guard<std::mutex> lk(mu_);
                if (!err_) err_ = std::current_exception();
            }
        });
    }
    void wait() {
        for (auto &x : th_)
            if (x.joinable()) x.join();
        th_.clear();
        if (err_) {
            std::exception_ptr e = err_;
            err_ = nullptr;
            std::rethrow_exception(e);
        }
    }
    ~TaskGroup() {
        for (auto &x : th_)
            if (x.joinable()) x.join();
    }

private:
    bool threads_;
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::exception_ptr err_;
};

// f(lo, hi) over [0, n) in contiguous ranges of at least `grain` items, one
// range per thread (the calling thread takes the first).
template <class F>
void parallel_ranges(int64_t n, int64_t grain, F &&f) {
    if (n <= 0) return;
    const int64_t want = std::max<int64_t>(1, n / std::max<int64_t>(1, grain));
    const int nt = (int)std::min<int64_t>(want, host_threads());
    if (nt <= 1) {
        f((int64_t)0, n);
        return;
    }
    TaskGroup g;
    for (int t = 1; t < nt; t++) {
        const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
        g.run([&f, lo, hi] { f(lo, hi); });
    }
    f((int64_t)0, n / nt);
    g.wait();
}

// Items [0, count) taken in order from a shared counter by `nthreads`
// threads, the calling thread among them.  Every thread runs enter() once
// before its first item: a new std::thread starts on CUDA device 0, so a
// pool whose items launch GPU work passes a callable that makes the
// caller's device current.  A thread stops taking items once stop() is true.
template <class Enter, class Work, class Stop>
void run_pool(int64_t count, int nthreads, Enter &&enter, Work &&work, Stop &&stop) {
    std::atomic<int64_t> next{0};
    auto body = [&] {
        enter();
        for (;;) {
            const int64_t it = next.fetch_add(1);
            if (it >= count || stop()) break;
            work(it);
        }
    };
    std::vector<std::thread> th;
    for (int i = 1; i < nthreads; i++) th.emplace_back(body);
    body();
    for (auto &t : th) t.join();
}

}  // namespace spx
