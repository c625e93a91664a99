// Stress check of lmie_b200/csrc/host_pool.h (built and run by
// tests/test_host_pool.py): many parallel loops of varying width on one
// caller, then several caller threads at once; every loop must cover its
// index range exactly once and every call must return.
#include <atomic>
#include <cstdio>

#include "host_pool.h"

static bool loop(int width, int n) {
    std::atomic<int> next(0);
    std::atomic<long long> sum(0);
    const std::function<void()> body = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            sum += i;
        }
    };
    host_pool().run(width, body);
    return sum == (long long) n * (n - 1) / 2;
}

int main() {
    for (int rep = 0; rep < 3000; ++rep)
        if (!loop(1 + rep % 33, 1 + rep % 997)) {
            std::printf("wrong sum at %d\n", rep);
            return 1;
        }
    std::atomic<int> bad(0);
    std::vector<std::thread> callers;
    for (int t = 0; t < 6; ++t)
        callers.emplace_back([&bad, t] {
            for (int rep = 0; rep < 500; ++rep)
                if (!loop(2 + (rep + t) % 15, 700)) ++bad;
        });
    for (auto &c : callers) c.join();
    std::printf("%s\n", bad == 0 ? "ok" : "wrong sums from concurrent callers");
    return bad != 0;
}
