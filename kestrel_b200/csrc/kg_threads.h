// kg_threads.h — a fork-join loop over host threads (VCF parsing, the CLI's
// output formatting).
#pragma once

#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace kg {

// Threads for a request: n <= 0 means every hardware thread.
inline int host_threads(int n) {
    return n > 0 ? n : (int)std::max(1u, std::thread::hardware_concurrency());
}

// f(thread, begin, end) over [0, n) cut into at most n_threads contiguous
// ranges; the caller's thread runs the first.
template <class F>
void parallel_for(int n_threads, int64_t n, F&& f) {
    if (n <= 0) return;
    const int t = (int)std::max<int64_t>(1, std::min<int64_t>(n_threads, n));
    std::vector<std::thread> pool;
    pool.reserve((size_t)t - 1);
    for (int i = 1; i < t; i++) {
        const int64_t b = n * i / t, e = n * (i + 1) / t;
        pool.emplace_back([&f, i, b, e] { f(i, b, e); });
    }
    f(0, (int64_t)0, n / t);
    for (auto& th : pool) th.join();
}

}  // namespace kg
