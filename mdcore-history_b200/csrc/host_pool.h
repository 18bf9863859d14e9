// A small persistent pool of host threads for the per-step host loops of the engine
// (packing the cells into the upload buffers, adding the downloaded forces into the cells).
//
// run(n, grain, fn) splits [0, n) into at most threads() contiguous ranges of at least
// `grain` items, calls fn(part, begin, end) for each (the calling thread takes part 0) and
// returns when every range is done.  The thread count is MDB_HOST_THREADS if set, else the
// number of CPUs this process may run on, at most 16.
//
// Waiting is spin-then-block: an idle worker polls for the next job for MDB_HOST_SPIN_US
// microseconds (default 2000) after its last one, then blocks on a condition variable, so
// that the several loops of one step (and of steps issued back to back) start without a
// thread wake-up each, and an idle pool takes no CPU time.  The caller waits for the
// workers the same way.  MDB_HOST_SPIN_US=0 blocks at once.
#pragma once
#include <sched.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>
#if defined(__x86_64__) || defined(__i386__)
#include <immintrin.h>
#endif

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
            std::lock_guard<std::mutex> lk(m_);
            job_ = &fn;
            n_ = n;
            parts_ = parts;
            pending_.store(parts - 1, std::memory_order_relaxed);
            gen_.fetch_add(1, std::memory_order_release);
        }
        if (sleepers_.load(std::memory_order_acquire) > 0) cv_.notify_all();
        fn(0, 0, range_end(0, n, parts));
        if (!spin_until([&] { return pending_.load(std::memory_order_acquire) == 0; })) {
            std::unique_lock<std::mutex> lk(m_);
            done_.wait(lk, [&] { return pending_.load(std::memory_order_acquire) == 0; });
        }
        std::lock_guard<std::mutex> lk(m_);
        job_ = nullptr;
    }

    ~HostPool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
            gen_.fetch_add(1, std::memory_order_release);
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
        if (const char* env = std::getenv("MDB_HOST_SPIN_US")) spin_us_ = std::max(0, std::atoi(env));
        for (int k = 1; k < n; k++) workers_.emplace_back([this, k] { loop(k); });
    }

    static int range_end(int part, int n, int parts) { return (int)((long long)n * (part + 1) / parts); }

    static void relax() {
#if defined(__x86_64__) || defined(__i386__)
        _mm_pause();
#else
        std::this_thread::yield();
#endif
    }

    // Polls `ready` for at most spin_us_ microseconds; true once it holds.
    template <class F>
    bool spin_until(F ready) const {
        if (ready()) return true;
        if (spin_us_ <= 0) return false;
        const auto t_end = std::chrono::steady_clock::now() + std::chrono::microseconds(spin_us_);
        for (int it = 1;; ++it) {
            relax();
            if (ready()) return true;
            if ((it & 63) == 0 && std::chrono::steady_clock::now() >= t_end) return ready();
        }
    }

    void loop(int id) {
        long long seen = 0;
        for (;;) {
            spin_until([&] { return gen_.load(std::memory_order_acquire) != seen; });
            std::unique_lock<std::mutex> lk(m_);
            if (gen_.load(std::memory_order_acquire) == seen) {
                sleepers_.fetch_add(1, std::memory_order_acq_rel);
                cv_.wait(lk, [&] { return gen_.load(std::memory_order_acquire) != seen; });
                sleepers_.fetch_sub(1, std::memory_order_acq_rel);
            }
            seen = gen_.load(std::memory_order_acquire);
            if (stop_) return;
            if (id >= parts_ || job_ == nullptr) continue;
            const std::function<void(int, int, int)>* job = job_;
            const int b = range_end(id - 1, n_, parts_), e = range_end(id, n_, parts_);
            lk.unlock();
            (*job)(id, b, e);
            if (pending_.fetch_sub(1, std::memory_order_acq_rel) == 1) {
                std::lock_guard<std::mutex> g(m_);
                done_.notify_one();
            }
        }
    }

    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    const std::function<void(int, int, int)>* job_ = nullptr;   // guarded by m_
    int n_ = 0, parts_ = 1;                                       // guarded by m_
    std::atomic<int> pending_{0};
    std::atomic<long long> gen_{0};
    std::atomic<int> sleepers_{0};
    bool stop_ = false;                                           // guarded by m_
    int spin_us_ = 2000;
};

}  // namespace nb
