// Host check of spx::run_pool (sparse-eigs-mex_b200/csrc/host/parallel.h):
// every worker thread runs the pool's enter() before its first item, so a
// per-thread setting made there (the library passes "make the caller's CUDA
// device current") is the one each item sees.  A thread-local integer
// stands in for the CUDA runtime's per-thread current device.
#include "parallel.h"

#include <cstdio>
#include <vector>

static thread_local int current = 0;   // new threads start at 0, as CUDA's device does

int main() {
    current = 5;                        // the caller's setting
    const int caller = current;
    const int64_t count = 4000;
    std::vector<int> seen(count, -1), runs(count, 0);
    spx::run_pool(count, 8, [caller] { current = caller; },
                  [&](int64_t i) { seen[i] = current; runs[i]++; }, [] { return false; });
    for (int64_t i = 0; i < count; i++)
        if (seen[i] != caller || runs[i] != 1) {
            std::printf("item %lld ran %d times on setting %d (caller %d)\n", (long long)i, runs[i],
                        seen[i], caller);
            return 1;
        }
    // stop(): no item starts once it is true
    std::atomic<int64_t> done{0};
    spx::run_pool(count, 8, [] {}, [&](int64_t) { done++; }, [&] { return done.load() >= 10; });
    if (done.load() > 10 + 8) {
        std::printf("stop() ignored: %lld items ran\n", (long long)done.load());
        return 1;
    }
    std::printf("ok\n");
    return 0;
}
