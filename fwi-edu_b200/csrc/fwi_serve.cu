// fwi_serve.cu -- the request loop: modeling and gradient requests of any grid size, admitted
// by device-memory footprint and run concurrently on one GPU.
//
// Requests arrive through fwi_server_submit from any host thread.  The server keeps them in
// arrival order and admits the oldest one as soon as a worker is free and its footprint
// (fwi_estimate_bytes) fits into the budget left by the requests already running; requests
// that arrive while others are on the GPU are therefore admitted as slots and memory free up
// (continuous admission, not a queue drained one at a time).  Every worker owns a CUDA stream
// through its own engine context, so admitted requests overlap on the device; the engine's
// allocations are stream-ordered, so one request growing or releasing its state never stalls
// the others.  Each request's result depends on its inputs only (the engine is deterministic
// and contexts share nothing), so it is the same alone and in any mix.
//
// Admission is strictly first come, first served: a request that does not fit waits at the
// head until enough memory is released (no later request overtakes it, so none starves).  A
// request larger than the whole budget is rejected at submission.
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
    std::condition_variable cv_work, cv_done;
    std::deque<Job *> queue;
    std::map<long long, Job *> jobs;
    std::vector<std::thread> workers;
    size_t in_use = 0, peak_bytes = 0;
    int active = 0, peak_active = 0;
    long long next_id = 1, submitted = 0, completed = 0, failed = 0, rejected = 0;
    bool stop = false, any = false;
    Clock::time_point t_first, t_last;
    std::vector<double> lat_ms, queue_ms;
    double cell_updates = 0.0, shots_modeled = 0.0, shot_gradients = 0.0;
};

namespace {

// one request on a fresh engine context of this worker's thread
void run_job(fwi_server *s, Job *j)
{
    const fwi_request &r = j->req;
    fwi_ctx *c = nullptr;
    int rc = fwi_ctx_create(&c, s->device, 0);
    if (rc == FWI_OK) rc = fwi_ctx_set_graphs(c, 0);  // one-off launch sequences: capturing them does not pay
    if (rc == FWI_OK)
        rc = fwi_ctx_set_model(c, r.vp, r.rho, r.nz, r.nx, r.dx, r.dz, r.dt, r.nt, r.pml, r.fs);
    if (rc == FWI_OK) rc = fwi_ctx_set_shots(c, r.shots, r.nshot);
    if (rc == FWI_OK && r.kind == FWI_REQ_GRADIENT) rc = fwi_ctx_set_observed(c, r.obs);
    if (rc == FWI_OK) {
        const int problem = r.kind == FWI_REQ_GRADIENT ? 1 : 0;
        rc = fwi_ctx_run(c, problem, r.freq, r.filter, r.precondition, FWI_PATH_BATCHED);
    }
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
    if (rc != FWI_OK) j->error = fwi_last_error();
    if (c) fwi_ctx_destroy(c);
    j->status = rc;
}

void worker_main(fwi_server *s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // admit the oldest request once it fits next to the running ones
        s->cv_work.wait(lk, [&] {
            return (!s->queue.empty() && s->in_use + s->queue.front()->bytes <= s->budget) ||
                   (s->stop && s->queue.empty());
        });
        if (s->queue.empty()) return;  // shutting down, nothing left to run
        Job *j = s->queue.front();
        s->queue.pop_front();
        s->in_use += j->bytes;
        s->peak_bytes = std::max(s->peak_bytes, s->in_use);
        s->active++;
        s->peak_active = std::max(s->peak_active, s->active);
        j->state = FWI_REQ_RUNNING;
        j->t_start = Clock::now();
        lk.unlock();
        run_job(s, j);
        lk.lock();
        j->t_end = Clock::now();
        j->state = j->status == FWI_OK ? FWI_REQ_DONE : FWI_REQ_FAILED;
        s->in_use -= j->bytes;
        s->active--;
        s->t_last = j->t_end;
        if (j->status == FWI_OK) {
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
        s->cv_work.notify_all();  // memory and a slot were released
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
    for (int i = 0; i < max_active; i++) s->workers.emplace_back(worker_main, s);
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
    for (auto &t : s->workers) t.join();
    for (auto &kv : s->jobs) delete kv.second;
    delete s;
    return FWI_OK;
}
