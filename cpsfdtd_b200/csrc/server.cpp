// server.cpp -- the serving loop behind cps_server_*: simulation jobs arrive
// over time, are admitted by device-memory footprint against a budget, run
// together in one batch (continuous batching: a job admitted while others are
// running joins them at the next chunk), and retire when they reach their
// step count.  No counterpart exists in the reference, whose main.cpp runs one
// simulation per process.
//
// Scheduling is first come, first served.  A job is admitted when a slot is
// free and used + footprint <= budget (the footprint is reserved then); a job
// larger than the whole budget is rejected (CPS_E_BUDGET).  Admitted jobs are
// built on a builder thread (the caller's build callback creates and sets up
// the grid) while chunks keep running on the device.  Each poll:
//   1. moves built jobs into the batch and hands queued jobs that fit to the
//      builder;
//   2. waits for the chunk in flight, credits its steps to the jobs that were
//      in it and retires the finished, cancelled or failed ones (done
//      callback on the polling thread, then the grid is destroyed);
//   3. admits again into the freed room and launches the next chunk for all
//      live jobs: min(chunk, fewest steps any live job still needs), so every
//      job stops exactly at its step count.
// A job's results depend only on its own grid: the batch runs each cell with
// the same arithmetic whatever the other jobs are.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "grid.h"

using namespace cps;

extern "C" {
cps_status cps_batch_create(int32_t precision, cps_batch **out);
cps_status cps_batch_destroy(cps_batch *b);
cps_status cps_batch_add(cps_batch *b, cps_grid *g);
cps_status cps_batch_remove(cps_batch *b, cps_grid *g);
cps_status cps_batch_step(cps_batch *b, int32_t nsteps);
cps_status cps_batch_synchronize(cps_batch *b);
cps_status cps_batch_set_tile(cps_batch *b, int32_t rows, int32_t planes, int32_t persistent);
cps_status cps_batch_get_stream(const cps_batch *b, void **stream);
cps_status cps_grid_destroy(cps_grid *g);
cps_status cps_grid_bytes(const cps_grid *g, int64_t *bytes);
}

namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Job {
    int64_t id = 0;
    int64_t footprint = 0;   // admission estimate
    int64_t charged = 0;     // what the budget carries for it (max of estimate and actual)
    int32_t nsteps = 0, done_steps = 0;
    cps_job_build_fn build = nullptr;
    cps_job_done_fn done = nullptr;
    void *user = nullptr;
    cps_grid *g = nullptr;
    cps_status build_status = CPS_OK;
    int64_t cells = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    std::atomic<bool> cancel{false};  // set by cps_server_cancel on the caller's thread, read by the poll and builder threads
};

double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t lo = (size_t)floor(pos), hi = std::min(v.size() - 1, lo + 1);
    return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

struct cps_server {
    cps_server_config cfg{};
    cps_batch *batch = nullptr;
    int device = 0;
    // builder thread: admitted jobs wait in to_build, come back in built
    std::thread builder;
    std::mutex mu;
    std::condition_variable cv, cv_built;
    bool stop = false;
    std::deque<Job *> to_build;
    Job *building = nullptr;  // the job the builder holds
    std::vector<Job *> built;
    int pending = 0;  // admitted jobs not yet collected from the builder
    int64_t used = 0;
    int64_t next_id = 1;
    std::deque<Job *> queue;
    std::vector<Job *> live;
    std::vector<Job *> inflight;  // jobs of the chunk in flight
    int32_t inflight_steps = 0;
    std::vector<double> latency, wait, run;
    int64_t done_ok = 0, failed = 0, rejected = 0, cancelled = 0;
    double cell_updates = 0;
    double t_first = -1, t_last = 0;
    int64_t chunks = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // around the chunk in flight
    double gpu_ms = 0;
};

namespace {

void finish(cps_server *s, Job *j, cps_status status)
{
    j->t_done = now_s();
    if (j->g) {
        if (j->done) j->done(j->user, j->id, j->g, status);
        cps_grid_destroy(j->g);
        j->g = nullptr;
    } else if (j->done) {
        j->done(j->user, j->id, nullptr, status);
    }
    s->used -= j->charged;
    if (status == CPS_OK) {
        s->done_ok++;
        s->latency.push_back(1e3 * (j->t_done - j->t_submit));
        s->wait.push_back(1e3 * (j->t_admit - j->t_submit));
        s->run.push_back(1e3 * (j->t_done - j->t_admit));
        s->t_last = j->t_done;
    } else if (status == CPS_E_CANCELLED) {
        s->cancelled++;
    } else if (status == CPS_E_BUDGET) {
        s->rejected++;
    } else {
        s->failed++;
    }
    delete j;
}

void builder_main(cps_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        Job *j = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [s] { return s->stop || !s->to_build.empty(); });
            if (s->to_build.empty()) return;  // stopping
            j = s->to_build.front();
            s->to_build.pop_front();
            s->building = j;
        }
        cps_grid *g = nullptr;
        cps_status st = CPS_E_CANCELLED;
        if (!j->cancel) {
            st = j->build ? j->build(j->user, j->id, &g) : CPS_E_INVALID;
            if (st == CPS_OK && !g) st = CPS_E_INVALID;
        }
        j->g = g;
        j->build_status = st;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->built.push_back(j);
            s->building = nullptr;
        }
        s->cv_built.notify_all();
    }
}

// built jobs join the batch (or end, when the build failed or they were cancelled)
void collect(cps_server *s)
{
    std::vector<Job *> ready;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        ready.swap(s->built);
    }
    for (Job *j : ready) {
        s->pending--;
        cps_status st = j->build_status;
        if (st == CPS_OK && j->cancel) st = CPS_E_CANCELLED;
        if (st == CPS_OK) {
            int64_t actual = 0;
            cps_grid_bytes(j->g, &actual);
            if (actual > j->charged) {
                s->used += actual - j->charged;
                j->charged = actual;
            }
            st = cps_batch_add(s->batch, j->g);
            if (st == CPS_OK) {
                j->cells = (int64_t)j->g->d.nx * j->g->d.ny * j->g->d.nz;
                s->live.push_back(j);
                continue;
            }
        }
        finish(s, j, st);  // a failed build or add ends this job only
    }
}

// hand queued jobs to the builder while a slot and budget room are free
void admit(cps_server *s)
{
    std::vector<Job *> go;
    while (!s->queue.empty()) {
        Job *j = s->queue.front();
        if (j->cancel) {
            s->queue.pop_front();
            finish(s, j, CPS_E_CANCELLED);
            continue;
        }
        if (j->footprint > s->cfg.budget_bytes) {
            s->queue.pop_front();
            set_error("job " + std::to_string(j->id) + " footprint exceeds the admission budget");
            finish(s, j, CPS_E_BUDGET);
            continue;
        }
        if ((int)s->live.size() + s->pending >= s->cfg.max_jobs || s->used + j->footprint > s->cfg.budget_bytes)
            break;
        s->queue.pop_front();
        j->t_admit = now_s();
        j->charged = j->footprint;
        s->used += j->charged;
        s->pending++;
        go.push_back(j);
    }
    if (go.empty()) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Job *j : go) s->to_build.push_back(j);
    }
    s->cv.notify_one();
}

// wait for the chunk in flight; credit its steps; retire what is finished
cps_status complete(cps_server *s)
{
    if (s->inflight.empty()) return CPS_OK;
    const cps_status st = cps_batch_synchronize(s->batch);
    float ms = 0;
    if (cudaEventElapsedTime(&ms, s->ev0, s->ev1) == cudaSuccess) s->gpu_ms += ms;
    else cudaGetLastError();
    for (Job *j : s->inflight) {
        j->done_steps += s->inflight_steps;
        s->cell_updates += (double)j->cells * s->inflight_steps;
    }
    s->inflight.clear();
    s->inflight_steps = 0;
    std::vector<Job *> keep;
    for (Job *j : s->live) {
        const bool fin = j->done_steps >= j->nsteps;
        if (st != CPS_OK || fin || j->cancel) {
            cps_batch_remove(s->batch, j->g);
            finish(s, j, st != CPS_OK ? st : (fin ? CPS_OK : CPS_E_CANCELLED));
        } else {
            keep.push_back(j);
        }
    }
    s->live.swap(keep);
    return st;
}

cps_status launch(cps_server *s)
{
    if (s->live.empty()) return CPS_OK;
    int32_t S = s->cfg.chunk_steps;
    for (Job *j : s->live) S = std::min(S, j->nsteps - j->done_steps);
    if (S <= 0) return CPS_OK;
    void *stream = nullptr;
    cps_batch_get_stream(s->batch, &stream);
    cudaEventRecord(s->ev0, (cudaStream_t)stream);
    const cps_status st = cps_batch_step(s->batch, S);
    cudaEventRecord(s->ev1, (cudaStream_t)stream);
    if (st != CPS_OK) {
        for (Job *j : s->live) {
            cps_batch_remove(s->batch, j->g);
            finish(s, j, st);
        }
        s->live.clear();
        return st;
    }
    s->inflight = s->live;
    s->inflight_steps = S;
    s->chunks++;
    return CPS_OK;
}

}  // namespace

// ================================================================ C ABI

extern "C" cps_status cps_server_create(const cps_server_config *cfg, cps_server **out)
{
    REQUIRE(cfg && out, CPS_E_INVALID, "cps_server_create: NULL argument");
    REQUIRE(cfg->precision == CPS_FP32 || cfg->precision == CPS_FP64, CPS_E_INVALID, "cps_server_create: precision");
    REQUIRE(cfg->budget_bytes > 0 && cfg->max_jobs >= 1 && cfg->chunk_steps >= 1 && cfg->chunk_steps <= 64,
            CPS_E_INVALID, "cps_server_create: budget > 0, max_jobs >= 1, chunk_steps in [1, 64]");
    *out = nullptr;
    cps_server *s = new cps_server();
    s->cfg = *cfg;
    cps_status st = cps_batch_create(cfg->precision, &s->batch);
    if (st == CPS_OK && cfg->tile_rows)
        st = cps_batch_set_tile(s->batch, cfg->tile_rows, cfg->tile_planes, cfg->tile_persistent);
    if (st != CPS_OK) {
        if (s->batch) cps_batch_destroy(s->batch);
        delete s;
        return st;
    }
    cudaGetDevice(&s->device);
    cudaEventCreate(&s->ev0);
    cudaEventCreate(&s->ev1);
    s->builder = std::thread(builder_main, s);
    *out = s;
    return CPS_OK;
}

extern "C" cps_status cps_server_submit(cps_server *s, int64_t footprint_bytes, int32_t nsteps,
                                        cps_job_build_fn build, cps_job_done_fn done, void *user, int64_t *job_id)
{
    REQUIRE(s && build, CPS_E_INVALID, "cps_server_submit: NULL argument");
    REQUIRE(nsteps >= 1 && footprint_bytes >= 0, CPS_E_INVALID, "cps_server_submit: nsteps >= 1, footprint >= 0");
    Job *j = new Job();
    j->id = s->next_id++;
    j->footprint = footprint_bytes;
    j->nsteps = nsteps;
    j->build = build;
    j->done = done;
    j->user = user;
    j->t_submit = now_s();
    if (s->t_first < 0) s->t_first = j->t_submit;
    s->queue.push_back(j);
    if (job_id) *job_id = j->id;
    return CPS_OK;
}

extern "C" cps_status cps_server_poll(cps_server *s, int32_t *live, int32_t *queued)
{
    REQUIRE(s, CPS_E_INVALID, "cps_server_poll: NULL server");
    collect(s);
    admit(s);
    cps_status st = complete(s);
    collect(s);
    admit(s);
    if (s->live.empty() && s->inflight.empty() && s->pending > 0) {
        // nothing to run until a build finishes: wait for one (bounded)
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_built.wait_for(lk, std::chrono::milliseconds(20), [s] { return !s->built.empty(); });
        lk.unlock();
        collect(s);
    }
    cps_status st2 = launch(s);
    if (live) *live = (int32_t)s->live.size();
    if (queued) *queued = (int32_t)s->queue.size();
    return st != CPS_OK ? st : st2;
}

extern "C" cps_status cps_server_drain(cps_server *s)
{
    REQUIRE(s, CPS_E_INVALID, "cps_server_drain: NULL server");
    cps_status first = CPS_OK;
    while (!s->queue.empty() || s->pending > 0 || !s->live.empty() || !s->inflight.empty()) {
        cps_status st = cps_server_poll(s, nullptr, nullptr);
        if (st != CPS_OK && first == CPS_OK) first = st;
        if (s->live.empty() && s->inflight.empty() && s->pending == 0 && !s->queue.empty()) {
            // nothing live or building and the head job was not admitted: it never will be
            set_error("cps_server_drain: queued job cannot be admitted");
            return CPS_E_BUDGET;
        }
    }
    return first;
}

extern "C" cps_status cps_server_cancel(cps_server *s, int64_t job_id)
{
    REQUIRE(s, CPS_E_INVALID, "cps_server_cancel: NULL server");
    for (Job *j : s->queue)
        if (j->id == job_id) { j->cancel = true; return CPS_OK; }
    for (Job *j : s->live)
        if (j->id == job_id) { j->cancel = true; return CPS_OK; }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Job *j : s->to_build)
            if (j->id == job_id) { j->cancel = true; return CPS_OK; }
        if (s->building && s->building->id == job_id) { s->building->cancel = true; return CPS_OK; }
        for (Job *j : s->built)
            if (j->id == job_id) { j->cancel = true; return CPS_OK; }
    }
    set_error("cps_server_cancel: no such job");
    return CPS_E_NOTFOUND;
}

extern "C" cps_status cps_server_get_stats(const cps_server *s, cps_server_stats *out)
{
    REQUIRE(s && out, CPS_E_INVALID, "cps_server_get_stats: NULL argument");
    memset(out, 0, sizeof(*out));
    out->jobs_done = s->done_ok;
    out->jobs_failed = s->failed;
    out->jobs_rejected = s->rejected;
    out->jobs_cancelled = s->cancelled;
    out->jobs_live = (int64_t)s->live.size();
    out->jobs_queued = (int64_t)s->queue.size();
    out->bytes_in_use = s->used;
    out->chunks = s->chunks;
    out->latency_p50_ms = percentile(s->latency, 0.50);
    out->latency_p99_ms = percentile(s->latency, 0.99);
    out->wait_p50_ms = percentile(s->wait, 0.50);
    out->wait_p99_ms = percentile(s->wait, 0.99);
    out->run_p50_ms = percentile(s->run, 0.50);
    out->cell_updates = s->cell_updates;
    out->span_s = s->t_first >= 0 && s->t_last > s->t_first ? s->t_last - s->t_first : 0.0;
    out->gpu_busy_s = s->gpu_ms / 1e3;
    return CPS_OK;
}

extern "C" cps_status cps_server_destroy(cps_server *s)
{
    if (!s) return CPS_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Job *j : s->to_build) j->cancel = true;
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->builder.joinable()) s->builder.join();
    collect(s);  // cancelled and finished builds end here
    if (!s->inflight.empty()) cps_batch_synchronize(s->batch);
    s->inflight.clear();
    for (Job *j : s->live) {
        cps_batch_remove(s->batch, j->g);
        finish(s, j, CPS_E_CANCELLED);
    }
    s->live.clear();
    while (!s->queue.empty()) {
        Job *j = s->queue.front();
        s->queue.pop_front();
        finish(s, j, CPS_E_CANCELLED);
    }
    cps_batch_destroy(s->batch);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    delete s;
    return CPS_OK;
}
