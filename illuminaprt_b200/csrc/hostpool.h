// Host threads for the copies between a caller's pageable arrays and the
// library's page-locked staging slots (plain C++: no CUDA in this file).
//
// A query from pageable memory moves every ray and hit through host memory
// twice; one core copies about 10 GB/s, so the copies are split over a fixed
// set of threads made once per context instead of threads started per copy.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace ilg {

// Runs the parts of one job at a time: part 0 on the calling thread, the
// others on the pool's threads. Threads are added on demand up to the number
// a job asks for; if none can be made, the calling thread runs every part.
class HostPool {
public:
    HostPool() = default;
    HostPool(const HostPool &) = delete;
    HostPool &operator=(const HostPool &) = delete;
    ~HostPool()
    {
        {
            std::lock_guard<std::mutex> l(m_);
            stop_ = true;
        }
        go_.notify_all();
        for (auto &t : th_) t.join();
    }

    unsigned threads() const { return (unsigned)th_.size(); }

    // f(k) for every k in [0, parts); returns when all parts have run
    void run(unsigned parts, const std::function<void(unsigned)> &f)
    {
        if (parts == 0) return;
        grow(parts - 1);
        const unsigned on_pool = std::min<unsigned>(parts - 1, (unsigned)th_.size());
        if (on_pool > 0) {
            {
                std::lock_guard<std::mutex> l(m_);
                job_ = &f;
                parts_ = on_pool + 1;
                left_ = on_pool;
                gen_++;
            }
            go_.notify_all();
        }
        f(0);
        // parts that found no thread run here, after part 0
        for (unsigned k = on_pool + 1; k < parts; k++) f(k);
        if (on_pool > 0) {
            std::unique_lock<std::mutex> l(m_);
            done_.wait(l, [&] { return left_ == 0; });
            job_ = nullptr;
        }
    }

private:
    void grow(unsigned n)
    {
        while (th_.size() < n) {
            // a new thread waits for the job after the current generation
            const unsigned id = (unsigned)th_.size() + 1u, seen = gen_;
            try {
                th_.emplace_back(&HostPool::worker, this, id, seen);
            } catch (...) {
                return;
            }
        }
    }

    void worker(unsigned id, unsigned seen)
    {
        for (;;) {
            const std::function<void(unsigned)> *f;
            {
                std::unique_lock<std::mutex> l(m_);
                go_.wait(l, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                if (id >= parts_) continue;
                f = job_;
            }
            (*f)(id);
            std::lock_guard<std::mutex> l(m_);
            if (--left_ == 0) done_.notify_one();
        }
    }

    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable go_, done_;
    const std::function<void(unsigned)> *job_ = nullptr;
    unsigned parts_ = 0, left_ = 0, gen_ = 0;
    bool stop_ = false;
};

struct CopySeg {
    void *dst;
    const void *src;
    size_t bytes;
};

// The segments' bytes, taken as one run, split evenly over up to max_parts
// parts of at least min_part bytes each; one memcpy per part and segment.
inline void pool_copy(HostPool &pool, const CopySeg *seg, int nseg, unsigned max_parts,
                      size_t min_part = size_t(1) << 20)
{
    size_t total = 0;
    for (int i = 0; i < nseg; i++) total += seg[i].bytes;
    if (total == 0) return;
    const unsigned parts = (unsigned)std::max<size_t>(
        1, std::min<size_t>(std::max(1u, max_parts), (total + min_part - 1) / min_part));
    pool.run(parts, [&](unsigned k) {
        const size_t lo = total * k / parts, hi = total * (k + 1) / parts;
        size_t base = 0;
        for (int i = 0; i < nseg && base < hi; base += seg[i].bytes, i++) {
            const size_t a = std::max(lo, base), b = std::min(hi, base + seg[i].bytes);
            if (a < b)
                memcpy(static_cast<char *>(seg[i].dst) + (a - base), static_cast<const char *>(seg[i].src) + (a - base),
                       b - a);
        }
    });
}

}  // namespace ilg
