// Stand-in for the subset of oneTBB that the reference k-NN graph builder uses
// (TEST INFRASTRUCTURE ONLY: it lets the reference's own, unmodified headers be
// compiled into the oracle under oracle/_ref; nothing in the product links it).
//
// Used API (reference src/SolutionKmeans.hpp:226-309, :401-550):
//   tbb::blocked_range<T>(begin, end[, grain])  .begin() .end()
//   tbb::parallel_for(range, body)
//   tbb::parallel_invoke(f1, f2)
//   tbb::combinable<T>(init)  .local()  .combine(f)
//
// Two builds:
//   KNNG_SHIM_THREADS == 0  serial and deterministic: parallel_for runs the body
//                           once over the whole range, parallel_invoke runs f1
//                           then f2, combinable holds a single value.  With this
//                           build the reference consumes its thread_local
//                           std::mt19937 in depth-first order and its large-node
//                           partition is stable, which is what parity is pinned to.
//   KNNG_SHIM_THREADS != 0  a persistent std::thread pool (size from the
//                           environment variable KNNG_REF_THREADS, else
//                           hardware_concurrency) with help-while-waiting task
//                           groups.  Worker threads live for the whole process,
//                           so each keeps its own thread_local RNG stream as TBB
//                           workers do.  Used only to time the reference on the
//                           host cores.
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdlib>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

#ifndef KNNG_SHIM_THREADS
#define KNNG_SHIM_THREADS 0
#endif

namespace oneapi {
namespace tbb {

template <class T>
class blocked_range {
public:
    blocked_range(T b, T e, std::size_t grain = 1) : b_(b), e_(e), grain_(grain ? grain : 1) {}
    T begin() const { return b_; }
    T end() const { return e_; }
    std::size_t size() const { return static_cast<std::size_t>(e_ - b_); }
    std::size_t grainsize() const { return grain_; }
    bool empty() const { return !(b_ < e_); }

private:
    T b_, e_;
    std::size_t grain_;
};

#if KNNG_SHIM_THREADS == 0

template <class T, class Body>
void parallel_for(const blocked_range<T>& r, const Body& body) {
    if (!r.empty()) body(r);
}

template <class F1, class F2>
void parallel_invoke(const F1& f1, const F2& f2) {
    f1();
    f2();
}

template <class T>
class combinable {
public:
    explicit combinable(const T& init) : init_(init), has_(false) {}
    T& local() {
        if (!has_) {
            value_ = init_;
            has_ = true;
        }
        return value_;
    }
    template <class F>
    T combine(F f) {
        (void)f;
        if (!has_) return init_;
        return value_;
    }

private:
    T init_;
    T value_;
    bool has_;
};

#else  // threaded stand-in

namespace shim_detail {

class Pool {
public:
    static Pool& get() {
        static Pool pool;
        return pool;
    }
    void submit(std::function<void()> task) {
        {
            std::lock_guard<std::mutex> lk(m_);
            q_.push_back(std::move(task));
        }
        cv_.notify_one();
    }
    bool try_run_one() {
        std::function<void()> task;
        {
            std::lock_guard<std::mutex> lk(m_);
            if (q_.empty()) return false;
            task = std::move(q_.front());
            q_.pop_front();
        }
        task();
        return true;
    }
    unsigned size() const { return nthreads_; }

private:
    Pool() {
        unsigned n = std::thread::hardware_concurrency();
        if (const char* s = std::getenv("KNNG_REF_THREADS")) {
            int v = std::atoi(s);
            if (v > 0) n = static_cast<unsigned>(v);
        }
        if (n == 0) n = 1;
        nthreads_ = n;
        // The calling thread also works while it waits, so n-1 workers give n
        // busy threads.
        for (unsigned i = 1; i < n; ++i) {
            workers_.emplace_back([this] { loop(); });
        }
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    void loop() {
        for (;;) {
            std::function<void()> task;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [this] { return stop_ || !q_.empty(); });
                if (stop_ && q_.empty()) return;
                task = std::move(q_.front());
                q_.pop_front();
            }
            task();
        }
    }
    std::vector<std::thread> workers_;
    std::deque<std::function<void()>> q_;
    std::mutex m_;
    std::condition_variable cv_;
    bool stop_ = false;
    unsigned nthreads_ = 1;
};

class TaskGroup {
public:
    template <class F>
    void run(F&& f) {
        pending_.fetch_add(1);
        Pool::get().submit([this, f]() {
            f();
            pending_.fetch_sub(1);
        });
    }
    void wait() {
        while (pending_.load() > 0) {
            if (!Pool::get().try_run_one()) std::this_thread::yield();
        }
    }

private:
    std::atomic<long> pending_{0};
};

}  // namespace shim_detail

template <class T, class Body>
void parallel_for(const blocked_range<T>& r, const Body& body) {
    if (r.empty()) return;
    const std::size_t n = r.size();
    const std::size_t nthreads = shim_detail::Pool::get().size();
    std::size_t chunk = std::max<std::size_t>(r.grainsize(), (n + 4 * nthreads - 1) / (4 * nthreads));
    if (chunk >= n || nthreads == 1) {
        body(r);
        return;
    }
    shim_detail::TaskGroup g;
    for (std::size_t off = 0; off < n; off += chunk) {
        T b = static_cast<T>(r.begin() + off);
        T e = static_cast<T>(r.begin() + std::min(n, off + chunk));
        g.run([&body, b, e]() { body(blocked_range<T>(b, e)); });
    }
    g.wait();
}

template <class F1, class F2>
void parallel_invoke(const F1& f1, const F2& f2) {
    shim_detail::TaskGroup g;
    g.run([&f1]() { f1(); });
    f2();
    g.wait();
}

template <class T>
class combinable {
public:
    explicit combinable(const T& init) : init_(init) {}
    T& local() {
        std::lock_guard<std::mutex> lk(m_);
        auto it = per_thread_.find(std::this_thread::get_id());
        if (it == per_thread_.end()) {
            it = per_thread_.emplace(std::this_thread::get_id(), init_).first;
        }
        return it->second;
    }
    template <class F>
    T combine(F f) {
        std::lock_guard<std::mutex> lk(m_);
        if (per_thread_.empty()) return init_;
        auto it = per_thread_.begin();
        T acc = it->second;
        for (++it; it != per_thread_.end(); ++it) acc = f(acc, it->second);
        return acc;
    }

private:
    T init_;
    std::mutex m_;
    std::unordered_map<std::thread::id, T> per_thread_;
};

#endif

}  // namespace tbb
}  // namespace oneapi

namespace tbb = oneapi::tbb;
