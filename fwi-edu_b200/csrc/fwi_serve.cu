// fwi_serve.cu -- the request loop: modeling and gradient requests of any grid size, admitted
// by device-memory footprint and batched continuously on one GPU.
//
// Requests arrive through fwi_server_submit from any host thread.  The server keeps them in
// arrival order and admits the oldest one as soon as fewer than `max_active` requests are in
// flight and its footprint (fwi_estimate_bytes) fits into the budget left by the requests
// already admitted (strictly first come, first served: a request that does not fit waits at
// the head, so none starves; one larger than the whole budget is rejected at submission).
//
// An admitted request goes through three stages, each on its own threads:
//  * set-up (two threads): a context of its own, the model's coefficients on the host, shots
//    and observed data uploaded on the context's stream, the run's state allocated -- then the
//    run is added to the server's executor (fwi_exec_add);
//  * the batch (one thread): the executor's step launches advance every run in the batch at
//    once, one program item each (continuous batching: a run set up while others are on the
//    GPU joins at the next launch, and a modeling request of one shot shares every launch with
//    the runs around it instead of filling the GPU with one small grid);
//  * hand-back (one thread): results copied into the caller's buffers on the context's own
//    stream, the context released, the request's memory returned to the budget.
// Each request's result depends on its inputs only (the executor's runs are bit-identical to
// their runs alone), so it is the same alone and in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fwi_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    long long id = 0;
    fwi_request req{};
    fwi_ctx *ctx = nullptr;
    size_t bytes = 0;
    int state = FWI_REQ_QUEUED;
    int status = FWI_OK;
    std::string error;
    Clock::time_point t_submit, t_start, t_end;
    double cell_updates = 0.0, objective = 0.0;
};

double ms(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); }

double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

struct fwi_server {
    int device = 0;
    size_t budget = 0;
    int max_active = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_batch, cv_back;
    std::deque<Job *> queue;          // submitted, not admitted
    std::deque<Job *> to_setup;       // admitted, waiting for a set-up thread
    std::vector<Job *> in_batch;      // added to the executor
    std::deque<Job *> to_hand_back;   // handed back by the executor
    std::map<long long, Job *> jobs;
    std::vector<std::thread> workers;
    fwi_exec *ex = nullptr;
    int setting_up = 0;
    size_t in_use = 0, peak_bytes = 0;
    int active = 0, peak_active = 0;
    long long next_id = 1, submitted = 0, completed = 0, failed = 0, rejected = 0;
    bool stop = false, any = false, batch_done = false;
    Clock::time_point t_first, t_last;
    std::vector<double> lat_ms, queue_ms;
    double cell_updates = 0.0, shots_modeled = 0.0, shot_gradients = 0.0;
};

namespace {

// stage 1: a context for the request, its inputs, and the run added to the executor
int set_up(fwi_server *s, Job *j)
{
    const fwi_request &r = j->req;
    int rc = fwi_ctx_create(&j->ctx, s->device, 0);
    if (rc == FWI_OK)
        rc = fwi_ctx_set_model(j->ctx, r.vp, r.rho, r.nz, r.nx, r.dx, r.dz, r.dt, r.nt, r.pml, r.fs);
    if (rc == FWI_OK) rc = fwi_ctx_set_shots(j->ctx, r.shots, r.nshot);
    if (rc == FWI_OK && r.kind == FWI_REQ_GRADIENT) rc = fwi_ctx_set_observed(j->ctx, r.obs);
    if (rc == FWI_OK)
        rc = fwi_exec_add(s->ex, j->ctx, r.kind == FWI_REQ_GRADIENT ? 1 : 0, r.freq, r.filter, r.precondition);
    return rc;
}

// stage 3: results into the caller's buffers (the context's stream is ordered after the run)
int hand_back(Job *j)
{
    const fwi_request &r = j->req;
    fwi_ctx *c = j->ctx;
    int rc = j->status;
    if (rc == FWI_OK && r.traces)
        for (int i = 0; i < r.nshot && rc == FWI_OK; i++)
            if (r.traces[i]) rc = fwi_ctx_get_traces(c, i, r.traces[i]);
    if (rc == FWI_OK && r.kind == FWI_REQ_GRADIENT) {
        if (r.grad) rc = fwi_ctx_get_gradient(c, r.grad);
        if (rc == FWI_OK) rc = fwi_ctx_objective(c, &j->objective);
    }
    if (rc == FWI_OK) {
        fwi_stats st;
        if (fwi_ctx_stats(c, &st) == FWI_OK) j->cell_updates = st.cell_updates;
    }
    return rc;
}

// the request leaves the server (any stage): context released, memory and slot returned
void finish(fwi_server *s, Job *j, int rc, std::unique_lock<std::mutex> &lk)
{
    if (rc != FWI_OK && j->error.empty()) j->error = fwi_last_error();
    fwi_ctx *c = j->ctx;
    j->ctx = nullptr;
    lk.unlock();
    if (c) fwi_ctx_destroy(c);
    lk.lock();
    j->status = rc;
    j->t_end = Clock::now();
    j->state = rc == FWI_OK ? FWI_REQ_DONE : FWI_REQ_FAILED;
    s->in_use -= j->bytes;
    s->active--;
    s->t_last = j->t_end;
    if (rc == FWI_OK) {
        s->completed++;
        s->lat_ms.push_back(ms(j->t_submit, j->t_end));
        s->queue_ms.push_back(ms(j->t_submit, j->t_start));
        s->cell_updates += j->cell_updates;
        if (j->req.kind == FWI_REQ_GRADIENT) s->shot_gradients += j->req.nshot;
        else s->shots_modeled += j->req.nshot;
    } else {
        s->failed++;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();   // memory and a slot were released
    s->cv_batch.notify_all();  // the batch thread may be waiting to shut down
}

// admission: the oldest request, once a slot is free and its footprint fits (caller holds mu)
void admit(fwi_server *s)
{
    while (!s->queue.empty() && s->active < s->max_active && s->in_use + s->queue.front()->bytes <= s->budget) {
        Job *j = s->queue.front();
        s->queue.pop_front();
        s->in_use += j->bytes;
        s->peak_bytes = std::max(s->peak_bytes, s->in_use);
        s->active++;
        s->peak_active = std::max(s->peak_active, s->active);
        j->state = FWI_REQ_RUNNING;
        j->t_start = Clock::now();
        s->to_setup.push_back(j);
    }
}

void setup_main(fwi_server *s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        admit(s);
        s->cv_work.wait(lk, [&] {
            admit(s);
            return !s->to_setup.empty() || (s->stop && s->queue.empty());
        });
        if (s->to_setup.empty()) return;  // shutting down, nothing left to set up
        Job *j = s->to_setup.front();
        s->to_setup.pop_front();
        s->setting_up++;
        lk.unlock();
        const int rc = set_up(s, j);
        if (rc != FWI_OK) j->error = fwi_last_error();
        lk.lock();
        s->setting_up--;
        if (rc == FWI_OK) {
            s->in_batch.push_back(j);
            s->cv_batch.notify_all();
        } else {
            finish(s, j, rc, lk);
        }
    }
}

// stage 2: the executor's launches while any run is in the batch; runs it hands back move on
void batch_main(fwi_server *s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_batch.wait(lk, [&] {
            return !s->in_batch.empty() || (s->stop && s->queue.empty() && s->to_setup.empty() && s->setting_up == 0);
        });
        if (s->in_batch.empty()) {
            s->batch_done = true;
            s->cv_back.notify_all();
            return;
        }
        lk.unlock();
        int active = 0;
        const int rc = fwi_exec_step(s->ex, 16, &active);
        lk.lock();
        for (size_t i = 0; i < s->in_batch.size();) {
            Job *j = s->in_batch[i];
            int done = 0, st = FWI_OK;
            fwi_exec_poll(s->ex, j->ctx, &done, &st);
            if (!done && rc != FWI_OK && active == 0) done = 1, st = rc;  // the executor failed its runs
            if (done) {
                j->status = st;
                s->to_hand_back.push_back(j);
                s->in_batch.erase(s->in_batch.begin() + i);
                s->cv_back.notify_all();
            } else {
                i++;
            }
        }
    }
}

void back_main(fwi_server *s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_back.wait(lk, [&] { return !s->to_hand_back.empty() || s->batch_done; });
        if (s->to_hand_back.empty()) return;
        Job *j = s->to_hand_back.front();
        s->to_hand_back.pop_front();
        lk.unlock();
        const int rc = hand_back(j);
        lk.lock();
        finish(s, j, rc, lk);
    }
}

}  // namespace

extern "C" int fwi_server_create(fwi_server **out, int device, size_t hbm_budget, int max_active)
{
    if (!out || max_active < 1) return FWI_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return FWI_ERR_NODEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return FWI_ERR_CUDA;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return FWI_ERR_CUDA;
    fwi_server *s = new fwi_server();
    s->device = device;
    s->budget = hbm_budget ? std::min(hbm_budget, free_b) : free_b - free_b / 10;
    s->max_active = max_active;
    // the server owns the device's stream-ordered pool: keep released blocks for the next
    // requests instead of returning them (returning them synchronises the device)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = (uint64_t)s->budget;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (fwi_exec_create(&s->ex, device) != FWI_OK) {
        delete s;
        return FWI_ERR_CUDA;
    }
    for (int i = 0; i < 2; i++) s->workers.emplace_back(setup_main, s);
    s->workers.emplace_back(batch_main, s);
    s->workers.emplace_back(back_main, s);
    *out = s;
    return FWI_OK;
}

extern "C" size_t fwi_request_bytes(const fwi_request *r)
{
    if (!r) return 0;
    return fwi_estimate_bytes(r->shots, r->nshot, r->nz, r->nx, r->nt, r->pml, r->kind == FWI_REQ_GRADIENT ? 1 : 0,
                              r->filter);
}

extern "C" int fwi_server_submit(fwi_server *s, const fwi_request *r, long long *id)
{
    if (!s || !r || !id) return FWI_ERR_ARG;
    if ((r->kind != FWI_REQ_MODEL && r->kind != FWI_REQ_GRADIENT) || !r->vp || !r->rho || !r->shots || r->nshot <= 0)
        return FWI_ERR_ARG;
    if (r->kind == FWI_REQ_GRADIENT && !r->obs) return FWI_ERR_ARG;
    const size_t bytes = fwi_request_bytes(r);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return FWI_ERR_STATE;
    if (bytes == 0 || bytes > s->budget) {
        s->rejected++;
        return FWI_ERR_NOMEM;
    }
    Job *j = new Job();
    j->id = s->next_id++;
    j->req = *r;
    j->bytes = bytes;
    j->t_submit = Clock::now();
    if (!s->any) {
        s->t_first = j->t_submit;
        s->any = true;
    }
    s->jobs[j->id] = j;
    s->queue.push_back(j);
    s->submitted++;
    *id = j->id;
    s->cv_work.notify_all();
    return FWI_OK;
}

extern "C" int fwi_server_wait(fwi_server *s, long long id, double timeout_s, fwi_request_info *info)
{
    if (!s) return FWI_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return FWI_ERR_ARG;
    Job *j = it->second;
    auto done = [&] { return j->state == FWI_REQ_DONE || j->state == FWI_REQ_FAILED; };
    if (timeout_s < 0) s->cv_done.wait(lk, done);
    else s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
    if (info) {
        memset(info, 0, sizeof(*info));
        info->state = j->state;
        info->status = j->status;
        info->bytes = j->bytes;
        info->objective = j->objective;
        info->cell_updates = j->cell_updates;
        if (done()) {
            info->queue_ms = ms(j->t_submit, j->t_start);
            info->run_ms = ms(j->t_start, j->t_end);
            info->total_ms = ms(j->t_submit, j->t_end);
            snprintf(info->error, sizeof(info->error), "%s", j->error.c_str());
        }
    }
    return done() ? FWI_OK : FWI_ERR_STATE;
}

extern "C" int fwi_server_stats(fwi_server *s, fwi_server_report *out)
{
    if (!s || !out) return FWI_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->rejected = s->rejected;
    out->p50_ms = percentile(s->lat_ms, 0.50);
    out->p99_ms = percentile(s->lat_ms, 0.99);
    out->max_ms = s->lat_ms.empty() ? 0.0 : *std::max_element(s->lat_ms.begin(), s->lat_ms.end());
    out->p50_queue_ms = percentile(s->queue_ms, 0.50);
    out->p99_queue_ms = percentile(s->queue_ms, 0.99);
    out->wall_s = s->any ? ms(s->t_first, s->t_last) / 1e3 : 0.0;
    out->cell_updates = s->cell_updates;
    out->shots_modeled = s->shots_modeled;
    out->shot_gradients = s->shot_gradients;
    out->budget = s->budget;
    out->peak_bytes = s->peak_bytes;
    out->max_active = s->max_active;
    out->peak_active = s->peak_active;
    return FWI_OK;
}

extern "C" int fwi_server_destroy(fwi_server *s)
{
    if (!s) return FWI_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;  // the workers finish every request already submitted, then exit
    }
    s->cv_work.notify_all();
    s->cv_batch.notify_all();
    for (auto &t : s->workers) t.join();
    fwi_exec_destroy(s->ex);
    for (auto &kv : s->jobs) delete kv.second;
    delete s;
    return FWI_OK;
}
