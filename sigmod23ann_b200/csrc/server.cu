// Serving form: a request loop for graph-build jobs of different sizes.
//
// The reference builds one graph per process (constructResult,
// src/SolutionKmeans.hpp:558, called once by main, src/main.cpp:59); it has no
// serving counterpart.  Here a server owns a device and an HBM budget.  Jobs
// are queued as they are submitted; worker threads admit them in arrival
// order while the sum of the admitted jobs' reservations stays within the
// budget and fewer than `max_running` run, and each admitted job builds on its
// own context and stream, so the work of concurrent jobs overlaps on the
// device.  A job's points and neighbour sets stay resident in HBM from
// admission until its result has been copied out; its memory is stream-
// ordered, so a finishing job does not synchronise the device under the
// others.  Every job runs the same build as knng_build with the same
// parameters, so its result does not depend on what else runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "admission.hpp"
#include "knng.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Job {
    uint64_t id = 0;
    const float* points = nullptr;
    uint32_t n = 0, d = 0;
    uint64_t ld_bytes = 0;
    knng_params params{};
    uint32_t* out_ids = nullptr;
    float* out_dists = nullptr;
    uint64_t need = 0;
    uint32_t state = KNNG_JOB_QUEUED;
    knng_status status = KNNG_OK;
    std::string error;
    Clock::time_point t_submit, t_start, t_done;
    knng_stats stats{};
};

}  // namespace

struct knng_server {
    int device = 0;
    uint64_t budget = 0;
    uint64_t in_use = 0;
    uint32_t max_running = 1;
    uint32_t running = 0;
    std::mutex mu;
    std::condition_variable cv_work;  // a job was queued, or memory / a slot freed up
    std::condition_variable cv_done;  // a job ended
    std::deque<Job*> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Job>> jobs;
    uint64_t next_id = 1;
    bool stopping = false;
    std::vector<std::thread> workers;
};

namespace {

// Runs one admitted job on a fresh context whose budget is the job's
// reservation; returns with the job's outputs written.
void run_job(knng_server* s, Job* j) {
    knng_context* ctx = nullptr;
    knng_status st = knng_create(s->device, j->need, &ctx);
    std::string err;
    if (st == KNNG_OK) {
        st = knng_build(ctx, j->points, j->n, j->d, j->ld_bytes, &j->params, j->out_ids, j->out_dists, &j->stats);
        if (st != KNNG_OK) err = knng_last_error(ctx);
        knng_destroy(ctx);
    } else {
        err = knng_status_string(st);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    j->status = st;
    j->error = err;
    j->state = st == KNNG_OK ? KNNG_JOB_DONE : KNNG_JOB_FAILED;
    j->t_done = Clock::now();
    s->in_use -= j->need;
    s->running -= 1;
    s->cv_done.notify_all();
    s->cv_work.notify_all();
}

void worker_loop(knng_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // Strict arrival order: the head of the queue is admitted once its
        // reservation fits and a running slot is free.
        s->cv_work.wait(lk, [s] {
            if (s->stopping) return true;
            if (s->queue.empty()) return false;
            return knng::admits(s->in_use, s->queue.front()->need, s->budget, s->running, s->max_running);
        });
        if (s->stopping) return;
        Job* j = s->queue.front();
        s->queue.pop_front();
        s->in_use += j->need;
        s->running += 1;
        j->state = KNNG_JOB_RUNNING;
        j->t_start = Clock::now();
        // Another worker may admit the next job now.
        s->cv_work.notify_all();
        lk.unlock();
        run_job(s, j);
        lk.lock();
    }
}

void fill_info(const Job& j, knng_job_info* info) {
    if (!info) return;
    std::memset(info, 0, sizeof(*info));
    info->state = j.state;
    info->status = static_cast<int32_t>(j.status);
    info->n = j.n;
    info->d = j.d;
    info->k = j.params.k;
    info->reserved_bytes = j.need;
    const Clock::time_point now = Clock::now();
    const bool started = j.state != KNNG_JOB_QUEUED;
    const bool ended = j.state == KNNG_JOB_DONE || j.state == KNNG_JOB_FAILED;
    info->ms_queued = ms_between(j.t_submit, started ? j.t_start : now);
    info->ms_run = started ? ms_between(j.t_start, ended ? j.t_done : now) : 0.0;
    info->ms_latency = ms_between(j.t_submit, ended ? j.t_done : now);
    info->stats = j.stats;
}

}  // namespace

extern "C" {

uint64_t knng_job_reservation(uint32_t n, uint32_t d, uint32_t k) {
    const uint64_t N = n, K = k, ld = (static_cast<uint64_t>(d) + 3) / 4 * 4;
    const uint64_t points = N * ld * 4;
    const uint64_t order = N * 8;                   // permutation + scatter buffer
    const uint64_t sets = N * (K * 8 + 12);         // distances, ids, size, max slot, bound
    const uint64_t refine = N * K * 8 + N * 40;     // snapshot, reverse lists, counts and offsets
    const uint64_t survivors = N * K * 96;          // per-point slots and pool of the join
    const uint64_t fixed = 256ull << 20;            // split, leaf and scan scratch
    return points + order + sets + refine + survivors + fixed;
}

knng_status knng_server_create(int device, uint64_t hbm_budget_bytes, uint32_t max_running, knng_server** out) {
    if (!out || max_running == 0) return KNNG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return KNNG_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return KNNG_ERR_INVALID_ARGUMENT;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return KNNG_ERR_CUDA;
    if (prop.major != 10) return KNNG_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return KNNG_ERR_CUDA;
    auto* s = new (std::nothrow) knng_server();
    if (!s) return KNNG_ERR_OUT_OF_MEMORY;
    s->device = device;
    s->budget = hbm_budget_bytes ? hbm_budget_bytes : static_cast<uint64_t>(prop.totalGlobalMem * 0.8);
    s->max_running = max_running;
    // Jobs allocate and free stream-ordered memory from the device's default
    // pool: keep up to the budget cached there between jobs instead of
    // returning it to the driver at every synchronisation.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = s->budget;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    try {
        for (uint32_t i = 0; i < max_running; ++i) s->workers.emplace_back(worker_loop, s);
    } catch (...) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stopping = true;
        }
        s->cv_work.notify_all();
        for (auto& t : s->workers) t.join();
        delete s;
        return KNNG_ERR_OUT_OF_MEMORY;
    }
    *out = s;
    return KNNG_OK;
}

knng_status knng_server_submit(knng_server* s, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                               const knng_params* params, uint32_t* out_ids, float* out_dists, uint64_t* out_job) {
    if (!s || !points || !params || !out_ids || !out_job || n == 0) return KNNG_ERR_INVALID_ARGUMENT;
    if (d != 64 && d != 100 && d != 128) return KNNG_ERR_UNSUPPORTED;
    if (params->k == 0 || params->k > 128) return KNNG_ERR_UNSUPPORTED;
    if (ld_bytes < 4ull * d || ld_bytes % 4 != 0) return KNNG_ERR_INVALID_ARGUMENT;
    auto j = std::make_unique<Job>();
    j->points = points;
    j->n = n;
    j->d = d;
    j->ld_bytes = ld_bytes;
    j->params = *params;
    j->out_ids = out_ids;
    j->out_dists = out_dists;
    j->need = knng_job_reservation(n, d, params->k);
    if (j->need > s->budget) return KNNG_ERR_BUDGET;
    j->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return KNNG_ERR_STATE;
    j->id = s->next_id++;
    *out_job = j->id;
    s->queue.push_back(j.get());
    s->jobs.emplace(j->id, std::move(j));
    s->cv_work.notify_all();
    return KNNG_OK;
}

knng_status knng_server_poll(knng_server* s, uint64_t job, knng_job_info* info) {
    if (!s) return KNNG_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job);
    if (it == s->jobs.end()) return KNNG_ERR_INVALID_ARGUMENT;
    fill_info(*it->second, info);
    return KNNG_OK;
}

knng_status knng_server_wait(knng_server* s, uint64_t job, int64_t timeout_ms, knng_job_info* info) {
    if (!s) return KNNG_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job);
    if (it == s->jobs.end()) return KNNG_ERR_INVALID_ARGUMENT;
    Job* j = it->second.get();
    auto ended = [j] { return j->state == KNNG_JOB_DONE || j->state == KNNG_JOB_FAILED; };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, ended);
    else
        s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ended);
    fill_info(*j, info);
    return ended() ? KNNG_OK : KNNG_ERR_PENDING;
}

const char* knng_server_job_error(knng_server* s, uint64_t job) {
    if (!s) return "null server";
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job);
    if (it == s->jobs.end()) return "unknown job";
    return it->second->error.c_str();
}

knng_status knng_server_release(knng_server* s, uint64_t job) {
    if (!s) return KNNG_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job);
    if (it == s->jobs.end()) return KNNG_ERR_INVALID_ARGUMENT;
    const uint32_t st = it->second->state;
    if (st != KNNG_JOB_DONE && st != KNNG_JOB_FAILED) return KNNG_ERR_PENDING;
    s->jobs.erase(it);
    return KNNG_OK;
}

knng_status knng_server_destroy(knng_server* s) {
    if (!s) return KNNG_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        // New submissions are refused and queued jobs cancelled; running jobs
        // finish before their workers exit.
        s->stopping = true;
        for (Job* j : s->queue) {
            j->state = KNNG_JOB_FAILED;
            j->status = KNNG_ERR_STATE;
            j->error = "server destroyed before the job was admitted";
            j->t_done = Clock::now();
        }
        s->queue.clear();
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    // Hand the memory the jobs cached in the device's default pool back.
    cudaSetDevice(s->device);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
        uint64_t keep = 0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        cudaMemPoolTrimTo(pool, 0);
    }
    delete s;
    return KNNG_OK;
}

}  // extern "C"
