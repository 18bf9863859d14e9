// A small persistent pool of host threads for the per-step host loops of the engine
// (packing the cells into the upload buffers, adding the downloaded forces into the cells).
//
// run(n, grain, fn) splits [0, n) into at most threads() contiguous ranges of at least
// `grain` items, calls fn(part, begin, end) for each (the calling thread takes part 0) and
// returns when every range is done.  Idle workers block on a
// condition variable, so they take no CPU time between steps.  The thread count is
// MDB_HOST_THREADS if set, else the number of CPUs this process may run on, at most 16.
#pragma once
#include <sched.h>
#include <cstdlib>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace nb {

class HostPool {
public:
    static HostPool& get() {
        static HostPool pool;
        return pool;
    }

    int threads() const { return (int)workers_.size() + 1; }

    void run(int n, int grain, const std::function<void(int, int, int)>& fn) {
        int parts = threads();
        if (grain < 1) grain = 1;
        if (parts > n / grain) parts = n / grain;
        if (parts <= 1) {
            if (n > 0) fn(0, 0, n);
            return;
        }
        {
            std::unique_lock<std::mutex> lk(m_);
            job_ = &fn;
            n_ = n;
            parts_ = parts;
            pending_ = parts - 1;
            ++generation_;
        }
        cv_.notify_all();
        fn(0, 0, range_end(0));
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return pending_ == 0; });
        job_ = nullptr;
    }

    ~HostPool() {
        {
            std::unique_lock<std::mutex> lk(m_);
            stop_ = true;
            ++generation_;
        }
        cv_.notify_all();
        for (std::thread& t : workers_) t.join();
    }

private:
    HostPool() {
        int n = 0;
        if (const char* env = std::getenv("MDB_HOST_THREADS")) n = std::atoi(env);
        if (n <= 0) {
#ifdef __linux__
            cpu_set_t set;
            CPU_ZERO(&set);
            if (sched_getaffinity(0, sizeof(set), &set) == 0) n = CPU_COUNT(&set);
#endif
            if (n <= 0) n = (int)std::thread::hardware_concurrency();
            if (n > 16) n = 16;
        }
        if (n < 1) n = 1;
        for (int k = 1; k < n; k++) workers_.emplace_back([this, k] { loop(k); });
    }

    int range_begin(int part) const { return (int)((long long)n_ * part / parts_); }
    int range_end(int part) const { return (int)((long long)n_ * (part + 1) / parts_); }

    void loop(int id) {
        long long seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(m_);
            cv_.wait(lk, [&] { return generation_ != seen; });
            seen = generation_;
            if (stop_) return;
            if (id >= parts_ || job_ == nullptr) continue;
            const std::function<void(int, int, int)>* job = job_;
            const int b = range_begin(id), e = range_end(id);
            lk.unlock();
            (*job)(id, b, e);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }

    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    const std::function<void(int, int, int)>* job_ = nullptr;
    int n_ = 0, parts_ = 1, pending_ = 0;
    long long generation_ = 0;
    bool stop_ = false;
};

}  // namespace nb
