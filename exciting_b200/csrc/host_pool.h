// A small persistent pool of host threads for the host side of the
// host-pointer calls (rebuilding full Hermitian matrices from packed upper
// triangles).  parallel_for(n, f) runs f(0..n-1) on the workers and the
// calling thread and returns when all are done.
#pragma once
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace exs {

class HostPool {
public:
    explicit HostPool(int nworkers)
    {
        for (int i = 0; i < nworkers; i++) th_.emplace_back([this] { worker(); });
    }
    ~HostPool()
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
    }
    HostPool(const HostPool &) = delete;
    HostPool &operator=(const HostPool &) = delete;

    void parallel_for(int n, const std::function<void(int)> &f)
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            fn_ = &f;
            ntasks_ = n;
            next_ = 0;
            active_ = (int)th_.size();
            gen_++;
        }
        cv_.notify_all();
        run_tasks();
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return active_ == 0; });
        fn_ = nullptr;
    }

private:
    void run_tasks()
    {
        for (;;) {
            const int t = next_.fetch_add(1);
            if (t >= ntasks_) break;
            (*fn_)(t);
        }
    }
    void worker()
    {
        unsigned seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(m_);
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            lk.unlock();
            run_tasks();
            lk.lock();
            if (--active_ == 0) done_.notify_all();
        }
    }

    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    const std::function<void(int)> *fn_ = nullptr;
    int ntasks_ = 0;
    std::atomic<int> next_{0};
    int active_ = 0;
    unsigned gen_ = 0;
    bool stop_ = false;
};

}  // namespace exs
