// Host check of the slab group's barrier (dasha_b200/csrc/halo.h, GroupBarrier): n threads pass
// many generations in step; a member that fails releases every waiter (false, no hang); a member
// that never arrives makes the others give up after the time limit; reset() makes the barrier
// usable again.  Prints "bad=<count of violated checks>".
#include "halo.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <thread>
#include <vector>

using dasha::GroupBarrier;

int main() {
    int bad = 0;
    {   // 4 threads, 2000 generations: nobody runs ahead of a generation
        const int n = 4, gens = 2000;
        GroupBarrier b(n);
        std::atomic<int> arrived[gens] = {};
        std::atomic<int> early{0}, fails{0};
        std::vector<std::thread> th;
        for (int t = 0; t < n; ++t)
            th.emplace_back([&] {
                for (int g = 0; g < gens; ++g) {
                    arrived[g].fetch_add(1);
                    if (!b.arrive(30.0)) fails.fetch_add(1);
                    if (arrived[g].load() != n) early.fetch_add(1);
                }
            });
        for (auto& x : th) x.join();
        bad += early.load() != 0;
        bad += fails.load() != 0;
        std::printf("generations early=%d fails=%d\n", early.load(), fails.load());
    }
    {   // one member fails while three wait: all three return false at once
        GroupBarrier b(4);
        std::atomic<int> released{0};
        std::vector<std::thread> th;
        const auto t0 = std::chrono::steady_clock::now();
        for (int t = 0; t < 3; ++t)
            th.emplace_back([&] { if (!b.arrive(60.0)) released.fetch_add(1); });
        std::this_thread::sleep_for(std::chrono::milliseconds(50));
        b.fail();
        for (auto& x : th) x.join();
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        bad += released.load() != 3;
        bad += s > 5.0;
        bad += b.arrive(1.0);   // a failed barrier refuses at once
        b.reset();
        std::atomic<int> ok{0};
        std::vector<std::thread> th2;
        for (int t = 0; t < 4; ++t) th2.emplace_back([&] { if (b.arrive(30.0)) ok.fetch_add(1); });
        for (auto& x : th2) x.join();
        bad += ok.load() != 4;
        std::printf("release released=%d seconds=%.3f after_reset=%d\n", released.load(), s, ok.load());
    }
    {   // a member never arrives: the waiters give up after the limit and the barrier is failed
        GroupBarrier b(3);
        std::atomic<int> gave_up{0};
        std::vector<std::thread> th;
        const auto t0 = std::chrono::steady_clock::now();
        for (int t = 0; t < 2; ++t)
            th.emplace_back([&] { if (!b.arrive(0.2)) gave_up.fetch_add(1); });
        for (auto& x : th) x.join();
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        bad += gave_up.load() != 2;
        bad += s < 0.15 || s > 5.0;
        bad += !b.failed();
        std::printf("limit gave_up=%d seconds=%.3f\n", gave_up.load(), s);
    }
    {   // the partition and the exchange ranges: neighbours send what the other receives
        for (int mz : {16, 41, 1028, 1031})
            for (int n = 1; n <= 8; ++n) {
                dasha::SlabPart prev{}, p{};
                int covered = 0;
                for (int s = 0; s < n; ++s) {
                    if (!dasha::slab_partition(mz, n, s, p)) { if ((mz - 4) >= 3 * n) ++bad; break; }
                    if (s == 0) bad += p.first != 2;
                    else bad += p.first != prev.first + prev.count;
                    covered += p.count;
                    prev = p;
                }
                if ((mz - 4) >= 3 * n) bad += covered != mz - 4;
            }
    }
    std::printf("bad=%d\n", bad);
    return bad != 0;
}
