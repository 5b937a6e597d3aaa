// Test program for dasha_b200/csrc/host_pool.h (tests/test_host_pool.py): every row of every
// job is visited exactly once, across many jobs, job sizes and concurrent callers.
#include "host_pool.h"

#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>

int main() {
    using dasha::HostPool;
    int bad = 0;
    for (long n : {0L, 1L, 255L, 256L, 257L, 1000L, 4097L, 100000L}) {
        for (int rep = 0; rep < 200; ++rep) {
            std::vector<std::atomic<int>> hit(n > 0 ? n : 1);
            for (auto& h : hit) h = 0;
            HostPool::get().run(n, [&](long r0, long r1) {
                for (long r = r0; r < r1; ++r) hit[r].fetch_add(1);
            });
            for (long r = 0; r < n; ++r) bad += hit[r] != 1;
        }
    }
    // concurrent callers take turns
    std::atomic<long> total{0};
    std::vector<std::thread> callers;
    for (int c = 0; c < 4; ++c)
        callers.emplace_back([&] {
            for (int rep = 0; rep < 100; ++rep)
                HostPool::get().run(5000, [&](long r0, long r1) { total.fetch_add(r1 - r0); });
        });
    for (auto& t : callers) t.join();
    bad += total != 4L * 100 * 5000;
    std::printf("host_pool bad=%d\n", bad);
    return bad != 0;
}
