// Small persistent worker pool for the host stages (one per handle).
#pragma once

#include <algorithm>
#include <condition_variable>
#include <exception>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace cctagb {

class ThreadPool {
public:
    explicit ThreadPool(int n) : active_(n)
    {
        for (int i = 0; i < n; ++i) workers_.emplace_back([this, i] { loop(i); });
    }
    ~ThreadPool()
    {
        {
            std::lock_guard<std::mutex> l(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    int size() const { return int(workers_.size()); }
    // Only the first n workers take part in later parallel_for calls (the
    // others stay idle); n is clamped to [0, size()].
    void set_active(int n)
    {
        std::lock_guard<std::mutex> l(mu_);
        active_ = std::max(0, std::min(n, size()));
    }

    // Runs fn(i) for i in [0, n) on the workers and the calling thread; the
    // first exception thrown by a task is rethrown here.
    void parallel_for(int n, const std::function<void(int)>& fn)
    {
        if (n <= 0) return;
        if (n == 1 || workers_.empty() || active_ == 0) {
            for (int i = 0; i < n; ++i) fn(i);
            return;
        }
        {
            std::lock_guard<std::mutex> l(mu_);
            fn_ = &fn;
            next_ = 0;
            total_ = n;
            done_ = 0;
            err_ = nullptr;
            ++gen_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> l(mu_);
        done_cv_.wait(l, [&] { return done_ == total_; });
        fn_ = nullptr;
        if (err_) std::rethrow_exception(err_);
    }

private:
    void work()
    {
        for (;;) {
            int i;
            const std::function<void(int)>* f;
            {
                std::lock_guard<std::mutex> l(mu_);
                if (!fn_ || next_ >= total_) return;
                i = next_++;
                f = fn_;
            }
            try {
                (*f)(i);
            } catch (...) {
                std::lock_guard<std::mutex> l(mu_);
                if (!err_) err_ = std::current_exception();
            }
            {
                std::lock_guard<std::mutex> l(mu_);
                if (++done_ == total_) done_cv_.notify_all();
            }
        }
    }
    void loop(int index)
    {
        unsigned seen = 0;
        for (;;) {
            bool take_part;
            {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait(l, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                take_part = index < active_;
            }
            if (take_part) work();
        }
    }

    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* fn_ = nullptr;
    int next_ = 0, total_ = 0, done_ = 0;
    int active_ = 0;
    unsigned gen_ = 0;
    bool stop_ = false;
    std::exception_ptr err_;
};

}  // namespace cctagb
