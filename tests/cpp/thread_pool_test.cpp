// Host worker pool: concurrent parallel_for calls from several threads each
// run every index exactly once, exceptions reach the caller, and the pool
// keeps working after one.
#include <atomic>
#include <cstdio>
#include <stdexcept>
#include <thread>
#include <vector>

#include "thread_pool.hpp"

int main()
{
    cctagb::ThreadPool pool(7);
    constexpr int kCallers = 6, kRounds = 200;
    std::atomic<int> bad{0};
    std::vector<std::thread> callers;
    for (int c = 0; c < kCallers; ++c)
        callers.emplace_back([&, c] {
            for (int r = 0; r < kRounds; ++r) {
                const int n = 1 + (c * 37 + r * 11) % 97;
                std::vector<std::atomic<int>> hit(static_cast<size_t>(n));
                for (auto& h : hit) h = 0;
                pool.parallel_for(n, [&](int i) { hit[size_t(i)]++; });
                for (auto& h : hit)
                    if (h != 1) ++bad;
            }
        });
    for (auto& t : callers) t.join();
    bool thrown = false;
    try {
        pool.parallel_for(50, [](int i) {
            if (i == 17) throw std::runtime_error("task 17");
        });
    } catch (const std::runtime_error&) {
        thrown = true;
    }
    std::atomic<int> after{0};
    pool.parallel_for(100, [&](int) { after++; });
    std::printf("bad=%d thrown=%d after=%d\n", bad.load(), int(thrown), after.load());
    return (bad == 0 && thrown && after == 100) ? 0 : 1;
}
