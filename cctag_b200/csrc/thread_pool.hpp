// Persistent worker pool for the host stages, shared by all detection slots
// of a handle.  Several threads may run parallel_for at once: each call is a
// job, its caller works on it, and idle workers take tasks from any job that
// still has some (round robin), so a frame with more work left gets more
// threads while other frames wait on the GPU.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace cctagb {

class ThreadPool {
public:
    explicit ThreadPool(int n)
    {
        for (int i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
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
    ThreadPool(const ThreadPool&) = delete;
    ThreadPool& operator=(const ThreadPool&) = delete;
    int size() const { return int(workers_.size()); }

    // Runs fn(i) for i in [0, n) on the calling thread and idle workers; the
    // first exception thrown by a task is rethrown here.  Tasks must not call
    // parallel_for themselves.
    void parallel_for(int n, const std::function<void(int)>& fn)
    {
        if (n <= 0) return;
        if (n == 1 || workers_.empty()) {
            for (int i = 0; i < n; ++i) fn(i);
            return;
        }
        Job job;
        job.fn = &fn;
        job.total = n;
        {
            std::lock_guard<std::mutex> l(mu_);
            jobs_.push_back(&job);
        }
        cv_.notify_all();
        for (;;) {
            int i;
            {
                std::lock_guard<std::mutex> l(mu_);
                if (job.next >= job.total) break;
                i = job.next++;
            }
            run(&job, i);
        }
        std::unique_lock<std::mutex> l(mu_);
        job.cv.wait(l, [&] { return job.done == job.total; });
        jobs_.erase(std::find(jobs_.begin(), jobs_.end(), &job));
        if (job.err) std::rethrow_exception(job.err);
    }

private:
    struct Job {
        const std::function<void(int)>* fn = nullptr;
        int next = 0, total = 0, done = 0;
        std::exception_ptr err;
        std::condition_variable cv;
    };

    // Under the lock: a job with tasks left, starting after the last one
    // served.
    Job* pick()
    {
        const size_t n = jobs_.size();
        for (size_t k = 0; k < n; ++k) {
            Job* j = jobs_[(rr_ + k) % n];
            if (j->next < j->total) {
                rr_ = (rr_ + k + 1) % n;
                return j;
            }
        }
        return nullptr;
    }

    void run(Job* job, int i)
    {
        std::exception_ptr err;
        try {
            (*job->fn)(i);
        } catch (...) {
            err = std::current_exception();
        }
        std::lock_guard<std::mutex> l(mu_);
        if (err && !job->err) job->err = err;
        if (++job->done == job->total) job->cv.notify_all();
    }

    void loop()
    {
        for (;;) {
            Job* job;
            int i;
            {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait(l, [&] { return stop_ || (job = pick()) != nullptr; });
                if (stop_) return;
                i = job->next++;
            }
            run(job, i);
        }
    }

    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<Job*> jobs_;
    size_t rr_ = 0;
    bool stop_ = false;
};

// Physical cores available to the process: the logical CPUs scaled by
// "cpu cores" / "siblings" of /proc/cpuinfo (two hardware threads of one core
// share its floating-point units, and the host stages are FP-bound); the
// logical count when that is unknown.
inline int physical_cores()
{
    const int logical = int(std::max(1u, std::thread::hardware_concurrency()));
    std::ifstream f("/proc/cpuinfo");
    std::string line;
    int cores = 0, siblings = 0;
    while (std::getline(f, line) && (!cores || !siblings)) {
        const auto colon = line.find(':');
        if (colon == std::string::npos) continue;
        const std::string key = line.substr(0, line.find_last_not_of(" \t", colon - 1) + 1);
        if (key == "cpu cores") cores = std::atoi(line.c_str() + colon + 1);
        if (key == "siblings") siblings = std::atoi(line.c_str() + colon + 1);
    }
    if (cores <= 0 || siblings <= 0 || cores > siblings) return logical;
    return std::max(1, logical * cores / siblings);
}

// A pool of `threads` host threads counting the caller (0: one per physical
// core), that is threads - 1 workers, at most 63.
inline std::shared_ptr<ThreadPool> make_host_pool(int threads = 0)
{
    if (threads <= 0) threads = physical_cores();
    return std::make_shared<ThreadPool>(std::min(63, threads - 1));
}

}  // namespace cctagb
