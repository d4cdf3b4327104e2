// Process-wide diagnostic counters: kernels launched by this library and
// bytes it copied between host and device.  Relaxed atomics, read through
// speigs_b200_counters().
#pragma once

#include <atomic>
#include <cstdint>

namespace spx {
struct Counters {
    std::atomic<long long> launches{0};
    std::atomic<long long> h2d{0};
    std::atomic<long long> d2h{0};
};
Counters &counters();
inline void note_launch(long long n = 1) { counters().launches.fetch_add(n, std::memory_order_relaxed); }
inline void note_h2d(long long b) { counters().h2d.fetch_add(b, std::memory_order_relaxed); }
inline void note_d2h(long long b) { counters().d2h.fetch_add(b, std::memory_order_relaxed); }
}  // namespace spx
