// host_pool.h -- host worker threads of liblmie_b200, started once and kept.
//
// The packing and unpacking of every sub-batch, and the case preparation of
// the C host layer, run many short parallel loops; starting threads for each
// of them cost more than the loops themselves.
#pragma once

#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include <unistd.h>

class HostPool {
  public:
    // body() on the caller and on n - 1 pool threads; returns when all are done.
    // body must share its work out dynamically: a nested call, or one made
    // while another caller thread holds the pool, runs it on the caller alone.
    void run(int n, const std::function<void()> &body) {
        std::unique_lock<std::mutex> use(use_mu_, std::try_to_lock);
        if (n <= 1 || t_in_pool || !use.owns_lock()) {
            body();
            return;
        }
        std::unique_lock<std::mutex> lk(mu_);
        // a new worker starts out having seen the generation before this job's
        const long long prev = gen_;
        while ((int) th_.size() < n - 1) th_.emplace_back([this, prev] { work(prev); });
        job_ = &body;
        want_ = n - 1;
        taken_ = 0;
        active_ = n - 1;
        ++gen_;
        cv_.notify_all();
        lk.unlock();
        body();
        lk.lock();
        done_.wait(lk, [this] { return active_ == 0; });
        job_ = nullptr;
    }

  private:
    void work(long long seen) {
        t_in_pool = true;
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&] { return gen_ != seen && taken_ < want_; });
            seen = gen_;
            ++taken_;
            const std::function<void()> *job = job_;
            lk.unlock();
            (*job)();
            lk.lock();
            if (--active_ == 0) done_.notify_all();
        }
    }
    static thread_local bool t_in_pool;
    std::mutex use_mu_, mu_;
    std::condition_variable cv_, done_;
    std::vector<std::thread> th_;
    const std::function<void()> *job_ = nullptr;
    long long gen_ = 0;
    int want_ = 0, taken_ = 0, active_ = 0;
};
inline thread_local bool HostPool::t_in_pool = false;

// The pool is never destroyed (its threads wait until the process exits); a
// process forked from this one starts a pool of its own.
inline HostPool &host_pool() {
    static std::mutex m;
    static HostPool *pool = nullptr;
    static pid_t owner = 0;
    std::lock_guard<std::mutex> lock(m);
    if (!pool || owner != getpid()) {
        pool = new HostPool();
        owner = getpid();
    }
    return *pool;
}

