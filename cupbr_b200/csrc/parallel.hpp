// Host-side parallel loops on std::thread.  The library deliberately does
// not use OpenMP: it is loaded next to PyTorch, which ships its own
// libgomp.so.1 with the same soname, and two OpenMP runtimes in one process
// are not safe.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

namespace cupbr_b200 {

inline unsigned hw_threads() {
    unsigned n = std::thread::hardware_concurrency();
    return n == 0 ? 1u : std::min(n, 64u);
}

// fn(begin, end) over [0, n) in chunks of `grain`, dynamically scheduled.
template <typename F>
void parallel_for(int64_t n, int64_t grain, F&& fn, unsigned threads = 0) {
    if (n <= 0) return;
    unsigned nt = threads ? threads : hw_threads();
    nt = (unsigned)std::min<int64_t>(nt, (n + grain - 1) / grain);
    if (nt <= 1) {
        fn((int64_t)0, n);
        return;
    }
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            int64_t b = next.fetch_add(grain);
            if (b >= n) break;
            fn(b, std::min(n, b + grain));
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(nt - 1);
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
}

}  // namespace cupbr_b200
