// host_pool.h -- a fixed set of host threads for the row gathers and scatters of the chunked
// host transfers.  One job at a time: run(n, f) splits the rows [0, n) into as many parts as
// there are workers plus the calling thread, runs f(r0, r1) on each and returns when all are
// done.  The workers start on first use and wait on a condition variable between jobs, so a
// transfer of many chunks does not create threads per chunk.  Concurrent callers (contexts
// driven from several host threads) take turns.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace dasha {

class HostPool {
public:
    static HostPool& get() {
        static HostPool pool;
        return pool;
    }

    template <class F>
    void run(long n, F f) {
        const long parts = (long)workers_.size() + 1;
        if (n < 256 || parts == 1) { f(0L, n); return; }
        std::lock_guard<std::mutex> turn(turn_);
        const long per = (n + parts - 1) / parts;
        {
            std::lock_guard<std::mutex> lk(m_);
            job_ = [&](long t) {
                const long a0 = t * per, a1 = std::min(n, a0 + per);
                if (a0 < a1) f(a0, a1);
            };
            pending_ = (int)workers_.size();
            ++gen_;
        }
        go_.notify_all();
        job_(parts - 1);                      // the caller's own part
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return pending_ == 0; });
        job_ = nullptr;
    }

    ~HostPool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
            ++gen_;
        }
        go_.notify_all();
        for (auto& t : workers_) t.join();
    }

private:
    HostPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        const int nw = (int)std::min<unsigned>(16, std::max<unsigned>(1, hw)) - 1;
        for (int w = 0; w < nw; ++w) workers_.emplace_back([this, w] { loop(w); });
    }
    void loop(int w) {
        unsigned long seen = 0;
        for (;;) {
            std::function<void(long)> job;
            {
                std::unique_lock<std::mutex> lk(m_);
                go_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
                job = job_;
            }
            job(w);
            std::lock_guard<std::mutex> lk(m_);
            if (--pending_ == 0) done_.notify_one();
        }
    }

    std::vector<std::thread> workers_;
    std::mutex turn_, m_;
    std::condition_variable go_, done_;
    std::function<void(long)> job_;
    unsigned long gen_ = 0;
    int pending_ = 0;
    bool stop_ = false;
};

}  // namespace dasha
