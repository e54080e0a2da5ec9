// oracle/tbb/parallel_for.h -- project-written stand-in for the two oneTBB names the reference's
// CPU path uses (tbb::blocked_range, tbb::parallel_for; Redzone_CPU.hxx:3,164,186,227,236 and
// std_parallel_remove.hxx:276). oneTBB is not installed on this image. TEST INFRASTRUCTURE ONLY.
//
// The reference indexes its per-thread state by r.begin() and so assumes every body call gets a
// unit range. This shim honours that: parallel_for(range(b, e), body) calls body(range(i, i+1))
// exactly once for every i in [b, e), spread over a persistent pool of worker threads (one per
// hardware thread, created on first use, like TBB's own arena) with the caller participating.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace tbb {

template <typename T>
class blocked_range {
public:
    blocked_range(T b, T e) : b_(b), e_(e) {}
    T begin() const { return b_; }
    T end() const { return e_; }
    bool empty() const { return !(b_ < e_); }

private:
    T b_, e_;
};

namespace shim {

// One parallel_for invocation. Workers hold a shared_ptr to the run they joined, so a worker
// that is late leaving one run can never take an index of the next.
struct run_state {
    const std::function<void(size_t)>* job;
    size_t count;
    std::atomic<size_t> next{0};
    std::atomic<size_t> done{0};
    std::mutex mu;
    std::condition_variable cv;

    void work() {
        for (;;) {
            const size_t i = next.fetch_add(1);
            if (i >= count) return;
            (*job)(i);
            if (done.fetch_add(1) + 1 == count) {
                std::lock_guard<std::mutex> g(mu);
                cv.notify_all();
            }
        }
    }
};

class pool {
public:
    static pool& get() {
        static pool p;
        return p;
    }
    void run(size_t count, const std::function<void(size_t)>& job) {
        if (count == 0) return;
        std::lock_guard<std::mutex> serial(run_mu_);
        auto rs = std::make_shared<run_state>();
        rs->job = &job;
        rs->count = count;
        {
            std::lock_guard<std::mutex> g(mu_);
            current_ = rs;
            ++epoch_;
        }
        cv_.notify_all();
        rs->work();
        {
            std::unique_lock<std::mutex> g(rs->mu);
            rs->cv.wait(g, [&] { return rs->done.load() == rs->count; });
        }
        std::lock_guard<std::mutex> g(mu_);
        current_.reset();
    }
    size_t workers() const { return threads_.size() + 1; }
    ~pool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
            ++epoch_;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }

private:
    pool() {
        unsigned hw = std::thread::hardware_concurrency();
        if (hw < 1) hw = 1;
        for (unsigned i = 0; i + 1 < hw; ++i) threads_.emplace_back([this] { loop(); });
    }
    void loop() {
        unsigned long seen = 0;
        for (;;) {
            std::shared_ptr<run_state> rs;
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return stop_ || epoch_ != seen; });
                if (stop_) return;
                seen = epoch_;
                rs = current_;
            }
            if (rs) rs->work();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex mu_, run_mu_;
    std::condition_variable cv_;
    std::shared_ptr<run_state> current_;
    unsigned long epoch_ = 0;
    bool stop_ = false;
};

}  // namespace shim

template <typename Range, typename Body>
void parallel_for(const Range& r, const Body& body) {
    using T = decltype(r.begin());
    const T b = r.begin();
    const size_t count = r.empty() ? 0 : size_t(r.end() - b);
    std::function<void(size_t)> job = [&](size_t i) { body(Range(T(b + i), T(b + i + 1))); };
    shim::pool::get().run(count, job);
}

}  // namespace tbb
