// fwi_exec.cuh -- continuous batching: several independent runs advanced by the same step
// launches.  Included at the end of fwi_engine.cu (it drives the engine's internals).
//
// A run (one context: its model, shots and, for a gradient, observed data) joins the
// executor's batch at a launch boundary: from then on every step launch -- one k_tile_groups
// launch on the executor's stream -- advances each shot group of every run in the batch by the
// next item of that group's own program (forward steps, or replay + adjoint steps), whatever
// its grid size, record length or progress.  Between the passes of a run the executor issues
// that run's own work (gathers, adjoint sources, finalisation, stacking) on the same stream, and
// a run whose last work is issued leaves the batch and is handed back to its context's stream.
// Runs therefore overlap on the GPU step by step, and one that arrives while others are in
// flight starts at the next launch, not when they finish.
//
// Every run's arithmetic is the single-run engine's (same kernel body, same programs, same
// per-shot state), so its results are bit-identical alone and in any mix.
//
// The host keeps at most 64 launches in flight ahead of the device (an event every 8
// launches).  A step kernel that gave up waiting for a tile copy sets the executor's error
// word; every run in flight at that point fails with FWI_ERR_CUDA.

struct ExecGroup {
    int shot_base = 0, nshot = 0, chunk = 1, ntx = 0, zt = 0;
    ShotRun *r0 = nullptr;
    CUtensorMap p1, p0, cf;
    const Program *prog = nullptr;
    long long L0 = 0;
    int *flags = nullptr;  // the group's TileSync flags in its context's flag array, or null
    size_t nflags = 0;
};

struct ExecRun {
    fwi_ctx *c = nullptr;
    int problem = 0, filter = 2, precondition = 1;
    float freq = 0.f;
    int phase = 0;  // 0 forward pass, 1 adjoint pass, 2 handed back
    std::vector<ExecGroup> groups;
    cudaStream_t own = nullptr;  // the context's stream while it is out of the batch
    cudaEvent_t done = nullptr;
    long long end_launch = 0;  // launch index at which the current pass ends
    int status = FWI_OK;
    double cells = 0.0;
};

struct fwi_exec {
    int device = 0;
    int math = 0;  // arithmetic of the step kernel (FWI_MATH when the executor was created)
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::vector<ExecRun *> runs;      // in the batch
    std::vector<ExecRun *> finished;  // handed back, not yet polled
    TileGroup *d_groups = nullptr;  // the group table in global memory (more than GROUPS_PARAM groups)
    int groups_cap = 0;
    GroupTable ptab;                  // the group table passed as a kernel parameter (at most GROUPS_PARAM)
    bool use_param = false;
    bool dirty = true;
    int ngroups = 0;
    dim3 grid;
    long long L = 0;  // step launches issued
    int *d_err = nullptr, *h_err = nullptr;
    std::deque<cudaEvent_t> inflight, spare;
    long long launches_total = 0;
};

// 16-column tiles, a ring of three stages (measured on one 60-shot gradient run: 163 ms against
// 168 with four)
static const int EXEC_TX = 16, EXEC_NST = 3;

// the batched path's set-up of a run without waves: per-shot runs, groups of consecutive shots
// sharing a model window, their frame pools and descriptors; initial frames zeroed
static int exec_setup(fwi_ctx *c, ExecRun *er)
{
    const bool gradient = er->problem == 1;
    const int ns = (int)c->shots.size();
    if ((int)c->runs.size() != ns) {
        free_runs(c);
        for (int i = 0; i < ns; i++) c->runs.emplace_back(new ShotRun());
    }
    for (int i = 0; i < ns; i++) {
        TRY(prepare_run(c, c->runs[i].get(), i, gradient));
        c->runs[i]->d.hessian = gradient && er->precondition == 1;
    }
    std::vector<std::pair<int, int>> gs;
    for (int i = 0; i < ns; i++) {
        if (gs.empty() || c->runs[i]->plan != c->runs[gs.back().first]->plan) gs.push_back({i, 1});
        else gs.back().second++;
    }
    std::vector<ShotDesc> descs(ns);
    for (auto &g : gs) {
        std::vector<ShotRun *> rs;
        for (int i = g.first; i < g.first + g.second; i++) rs.push_back(c->runs[i].get());
        TRY(assign_pool(c, g.first, rs));
    }
    for (int i = 0; i < ns; i++) descs[i] = c->runs[i]->d;
    TRY(upload_descs(c, descs));
    TRY(ensure_red(c));
    void *scr;
    TRY(scratch(c, 64 * 1024, &scr));
    for (auto &r : c->runs) TRY(zero_initial(c, r.get(), gradient));
    Program *pf, *pa;
    TRY(get_program(c, gradient ? "fwd1" : "fwd0", program_forward(c->nt, gradient ? K_FWD1 : K_FWD0), &pf));
    if (gradient) TRY(get_program(c, "adj/overlap", program_adjoint(c->nt, true), &pa));
    er->groups.clear();
    for (auto &g : gs) {
        ExecGroup eg;
        eg.shot_base = g.first;
        eg.nshot = g.second;
        eg.r0 = c->runs[g.first].get();
        const Plan *p = eg.r0->plan;
        eg.ntx = (p->Nx + EXEC_TX - 1) / EXEC_TX;
        eg.zt = (p->G + TG - 1) / TG;
        eg.chunk = std::min(eg.nshot, pick_chunk(eg.ntx * eg.zt, eg.nshot, 3));
        TRY(encode_group_maps<EXEC_TX>(eg.r0->d, eg.nshot, p->d_coef, &eg.p1, &eg.p0, &eg.cf));
        eg.prog = pf;
        er->groups.push_back(eg);
    }
    // Neighbour waits between the launches (TileSync) would need the group's flags here, zeroed
    // at the start of each pass; they are left off: measured on one 60-shot gradient run they made
    // the executor slower (166 -> 172 ms) and the serving mix too, while the single-run launches
    // gain 8 % from them.  The groups wait for the whole launch before (flags null).
    // cell updates of the run, as fwi_ctx_run counts them
    er->cells = 0.0;
    for (int i = 0; i < ns; i++) {
        const fwi_shot &s = c->shots[i].s;
        const double cellsz = (double)(c->nz + 2 * c->pml) * (s.ix_max - s.ix_min + 1 + 2 * c->pml);
        er->cells += cellsz * (gradient ? (double)c->nt * 2 + (c->nt - fwi_ck_count(c->nt)) : (double)c->nt);
    }
    return FWI_OK;
}

// the work of a run between its passes, issued on the executor's stream (the context's stream
// is the executor's while the run is in the batch)
static int exec_forward_done(fwi_exec *ex, ExecRun *er)
{
    fwi_ctx *c = er->c;
    for (auto &g : er->groups) {
        std::vector<ShotRun *> rs;
        for (int i = g.shot_base; i < g.shot_base + g.nshot; i++) rs.push_back(c->runs[i].get());
        if (er->problem == 0) {
            TRY(gather(c, rs, 0, false));
        } else if (er->problem == 2) {
            for (ShotRun *r : rs) TRY(prepare_taper(c, r, er->freq));
            if (er->filter == 0 || er->filter == 1) TRY(adjoint_source_filtered(c, rs, er->filter, false));
            else TRY(gather(c, rs, 1, false));
        } else {
            if (er->precondition == 1) TRY(finalize(c, rs, 0));
            for (ShotRun *r : rs) TRY(prepare_taper(c, r, er->freq));
            bool interp = false;
            for (ShotRun *r : rs) interp = interp || r->d.sr > 1;
            if (er->filter == 2 && !interp) TRY(gather(c, rs, 1, true));
            else TRY(adjoint_source_filtered(c, rs, er->filter, true));
            TRY(dump_shot_traces(c, rs));
            TRY(adj_init(c, rs, g.shot_base));
            g.prog = &c->progs.at("adj/overlap");
            g.L0 = ex->L;
            if (g.flags) CK(cudaMemsetAsync(g.flags, 0, g.nflags * sizeof(int), ex->stream));
        }
    }
    return FWI_OK;
}

static int exec_adjoint_done(ExecRun *er)
{
    fwi_ctx *c = er->c;
    std::vector<ShotRun *> all;
    for (auto &g : er->groups) {
        std::vector<ShotRun *> rs;
        for (int i = g.shot_base; i < g.shot_base + g.nshot; i++) rs.push_back(c->runs[i].get());
        TRY(finalize(c, rs, 1));
        TRY(dump_shot_gradients(c, rs));
        if (er->precondition == 1) TRY(shot_precondition(c, rs));
        all.insert(all.end(), rs.begin(), rs.end());
    }
    return stack_and_precondition(c, all, er->precondition);
}

// the run leaves the batch: its context gets its own stream back, ordered after the run's work
static int exec_hand_back(fwi_exec *ex, ExecRun *er)
{
    fwi_ctx *c = er->c;
    CK(cudaEventRecord(er->done, ex->stream));
    c->stream = er->own;
    CK(cudaStreamWaitEvent(er->own, er->done, 0));
    c->stats.cell_updates = er->cells;
    er->phase = 2;
    return FWI_OK;
}

static long long exec_pass_end(const ExecRun *er)
{
    long long e = 0;
    for (const auto &g : er->groups) e = std::max(e, g.L0 + (long long)g.prog->items.size());
    return e;
}

extern "C" int fwi_exec_create(fwi_exec **out, int device)
{
    if (!out) return fail(FWI_ERR_ARG, "NULL output");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
        return fail(FWI_ERR_NODEVICE, "no CUDA device %d: this engine runs on the GPU only", device);
    CK(cudaSetDevice(device));
    fwi_exec *ex = new fwi_exec();
    ex->device = device;
    if (const char *e = getenv("FWI_MATH")) ex->math = atoi(e) ? 1 : 0;
    CK(cudaStreamCreateWithFlags(&ex->stream, cudaStreamNonBlocking));
    CK(cudaMalloc(&ex->d_err, sizeof(int)));
    CK(cudaMemset(ex->d_err, 0, sizeof(int)));
    CK(cudaMallocHost(&ex->h_err, sizeof(int)));
    *ex->h_err = 0;
    *out = ex;
    return FWI_OK;
}

extern "C" int fwi_exec_add(fwi_exec *ex, fwi_ctx *c, int problem, float freq, int filter, int precondition)
{
    if (!ex || !c) return fail(FWI_ERR_ARG, "NULL executor or context");
    if (problem < 0 || problem > 2) return fail(FWI_ERR_ARG, "problem must be 0, 1 or 2 (got %d)", problem);
    if (filter < 0 || filter > 2) return fail(FWI_ERR_ARG, "residual filter %d (0 lowpass, 1 bandpass, 2 none)", filter);
    if (c->shots.empty()) return fail(FWI_ERR_STATE, "no shots");
    if (c->device != ex->device) return fail(FWI_ERR_ARG, "context and executor on different devices");
    if (c->dump.verbose > 1) return fail(FWI_ERR_UNSUPPORTED, "snapshots (verbose > 1) need fwi_ctx_run");
    if (c->math != ex->math) return fail(FWI_ERR_ARG, "context and executor differ in arithmetic (FWI_MATH)");
    CK(cudaSetDevice(c->device));
    ExecRun *er = new ExecRun();
    er->c = c;
    er->problem = problem;
    er->freq = freq;
    er->filter = filter;
    er->precondition = precondition;
    // set-up on the context's own stream (allocations synchronise that stream only)
    int rc = exec_setup(c, er);
    if (rc == FWI_OK && cudaEventCreateWithFlags(&er->done, cudaEventDisableTiming) != cudaSuccess)
        rc = fail(FWI_ERR_CUDA, "cudaEventCreate failed");
    if (rc != FWI_OK) {
        delete er;
        return rc;
    }
    er->own = c->stream;
    std::lock_guard<std::mutex> lk(ex->mu);
    CK(cudaEventRecord(er->done, er->own));
    CK(cudaStreamWaitEvent(ex->stream, er->done, 0));  // the batch waits for the set-up
    c->stream = ex->stream;
    for (auto &g : er->groups) g.L0 = ex->L;
    er->end_launch = exec_pass_end(er);
    ex->runs.push_back(er);
    ex->dirty = true;
    return FWI_OK;
}

// the launch table: every group of every run in the batch, one flat block range each
static int exec_table(fwi_exec *ex)
{
    std::vector<TileGroup> t;
    long long nb = 0;
    for (ExecRun *er : ex->runs)
        for (auto &g : er->groups) {
            TileGroup T;
            memset(&T, 0, sizeof(T));
            T.p1 = g.p1;
            T.p0 = g.p0;
            T.cf = g.cf;
            T.shots = er->c->d_desc;
            T.prog = g.prog->d;
            T.L0 = g.L0;
            T.nprog = (int)g.prog->items.size();
            T.shot_base = g.shot_base;
            T.nshot = g.nshot;
            T.chunk = g.chunk;
            T.ntx = g.ntx;
            T.zt = g.zt;
            T.halves = er->phase == 1 ? 2 : 1;  // the adjoint program pairs replay and adjoint items
            T.flags = g.flags;
            T.b0 = (int)nb;
            T.nblk = (g.flags ? g.ntx : g.ntx + 1) * g.zt * T.halves * ((g.nshot + g.chunk - 1) / g.chunk);
            nb += T.nblk;
            t.push_back(T);
        }
    if (nb > 0x7fffffff) return fail(FWI_ERR_UNSUPPORTED, "too many blocks in one launch of the batch");
    ex->use_param = (int)t.size() <= GROUPS_PARAM;
    if (ex->use_param) {
        memset(&ex->ptab, 0, sizeof(ex->ptab));
        for (size_t i = 0; i < t.size(); i++) ex->ptab.g[i] = t[i];
        ex->ngroups = (int)t.size();
        ex->grid = dim3((unsigned)std::max<long long>(nb, 1), 1, 1);
        ex->dirty = false;
        return FWI_OK;
    }
    if ((int)t.size() > ex->groups_cap) {
        if (ex->d_groups) {
            CK(cudaStreamSynchronize(ex->stream));
            cudaFree(ex->d_groups);
        }
        ex->groups_cap = std::max<int>((int)t.size(), 16);
        CK(cudaMalloc(&ex->d_groups, ex->groups_cap * sizeof(TileGroup)));
    }
    if (!t.empty())  // pageable source: staged before the call returns, ordered after the last launch
        CK(cudaMemcpyAsync(ex->d_groups, t.data(), t.size() * sizeof(TileGroup), cudaMemcpyHostToDevice, ex->stream));
    ex->ngroups = (int)t.size();
    ex->grid = dim3((unsigned)std::max<long long>(nb, 1), 1, 1);
    ex->dirty = false;
    return FWI_OK;
}

static int exec_fail_all(fwi_exec *ex, int code, const char *why)
{
    cudaStreamSynchronize(ex->stream);  // nothing of the failed runs may still be in flight
    for (ExecRun *er : ex->runs) {
        er->status = code;
        er->c->stream = er->own;
        er->phase = 2;
        ex->finished.push_back(er);
    }
    ex->runs.clear();
    ex->dirty = true;
    return fail(code, "%s", why);
}

// keep at most 128 launches in flight; read the error word as the device catches up.  The copy
// and the event between two launches end the programmatic overlap of that pair, so they come
// once per 32 launches.
static int exec_throttle(fwi_exec *ex)
{
    if (ex->L % 32 != 0) return FWI_OK;
    cudaEvent_t e;
    if (!ex->spare.empty()) {
        e = ex->spare.back();
        ex->spare.pop_back();
    } else {
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    CK(cudaMemcpyAsync(ex->h_err, ex->d_err, sizeof(int), cudaMemcpyDeviceToHost, ex->stream));
    CK(cudaEventRecord(e, ex->stream));
    ex->inflight.push_back(e);
    while (ex->inflight.size() > 4) {
        CK(cudaEventSynchronize(ex->inflight.front()));
        ex->spare.push_back(ex->inflight.front());
        ex->inflight.pop_front();
    }
    if (*ex->h_err) return exec_fail_all(ex, FWI_ERR_CUDA, "step kernel: a tile copy did not complete within 2 s");
    return FWI_OK;
}

extern "C" int fwi_exec_step(fwi_exec *ex, int launches, int *active)
{
    if (!ex) return fail(FWI_ERR_ARG, "NULL executor");
    std::lock_guard<std::mutex> lk(ex->mu);
    CK(cudaSetDevice(ex->device));
    for (int k = 0; (launches <= 0 || k < launches) && !ex->runs.empty(); k++) {
        if (ex->dirty) TRY(exec_table(ex));
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t lc = {};
        lc.gridDim = ex->grid;
        lc.blockDim = dim3(TG, EXEC_TX + 32 / TG);
        lc.dynamicSmemBytes = TileGeom<EXEC_TX>::smem(EXEC_NST);
        lc.stream = ex->stream;
        lc.attrs = attr;
        lc.numAttrs = 1;
        const bool math = ex->math != 0;
        static std::once_flag attr_once[2];
        std::call_once(attr_once[math ? 1 : 0], [&] {
            const int sm = TileGeom<EXEC_TX>::smem(EXEC_NST);
            cudaFuncSetAttribute(math ? (const void *)k_tile_groups<EXEC_TX, EXEC_NST, 1>
                                      : (const void *)k_tile_groups<EXEC_TX, EXEC_NST, 0>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
            cudaFuncSetAttribute(math ? (const void *)k_tile_groups_p<EXEC_TX, EXEC_NST, 1>
                                      : (const void *)k_tile_groups_p<EXEC_TX, EXEC_NST, 0>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        });
        if (ex->use_param) {
            auto fn = math ? k_tile_groups_p<EXEC_TX, EXEC_NST, 1> : k_tile_groups_p<EXEC_TX, EXEC_NST, 0>;
            CK(cudaLaunchKernelEx(&lc, fn, ex->ptab, ex->ngroups, ex->L, ex->d_err));
        } else {
            auto fn = math ? k_tile_groups<EXEC_TX, EXEC_NST, 1> : k_tile_groups<EXEC_TX, EXEC_NST, 0>;
            CK(cudaLaunchKernelEx(&lc, fn, (const TileGroup *)ex->d_groups, ex->ngroups, ex->L, ex->d_err));
        }
        ex->L++;
        ex->launches_total++;
        // runs whose pass ended with this launch: their work between passes, or hand-back
        for (size_t i = 0; i < ex->runs.size();) {
            ExecRun *er = ex->runs[i];
            if (ex->L < er->end_launch) {
                i++;
                continue;
            }
            int rc = FWI_OK;
            if (er->phase == 0 && er->problem == 1) {
                rc = exec_forward_done(ex, er);
                if (rc == FWI_OK) {
                    er->phase = 1;
                    er->end_launch = exec_pass_end(er);
                    ex->dirty = true;
                    i++;
                    continue;
                }
            } else if (er->phase == 0) {
                rc = exec_forward_done(ex, er);
            } else {
                rc = exec_adjoint_done(er);
            }
            if (rc == FWI_OK) rc = exec_hand_back(ex, er);
            if (rc != FWI_OK) {
                er->status = rc;
                er->c->stream = er->own;
                er->phase = 2;
            }
            ex->finished.push_back(er);
            ex->runs.erase(ex->runs.begin() + i);
            ex->dirty = true;
        }
        TRY(exec_throttle(ex));
    }
    if (active) *active = (int)ex->runs.size();
    return FWI_OK;
}

extern "C" int fwi_exec_poll(fwi_exec *ex, fwi_ctx *c, int *done, int *status)
{
    if (!ex || !c || !done) return fail(FWI_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(ex->mu);
    *done = 0;
    for (size_t i = 0; i < ex->finished.size(); i++)
        if (ex->finished[i]->c == c) {
            ExecRun *er = ex->finished[i];
            *done = 1;
            if (status) *status = er->status;
            if (er->done) cudaEventDestroy(er->done);
            delete er;
            ex->finished.erase(ex->finished.begin() + i);
            return FWI_OK;
        }
    return FWI_OK;
}

extern "C" int fwi_exec_launches(fwi_exec *ex, long long *launches)
{
    if (!ex || !launches) return fail(FWI_ERR_ARG, "NULL argument");
    *launches = ex->launches_total;
    return FWI_OK;
}

extern "C" int fwi_exec_destroy(fwi_exec *ex)
{
    if (!ex) return FWI_OK;
    cudaSetDevice(ex->device);
    cudaStreamSynchronize(ex->stream);
    for (ExecRun *er : ex->runs) {  // runs never finished: hand their contexts back
        er->c->stream = er->own;
        if (er->done) cudaEventDestroy(er->done);
        delete er;
    }
    for (ExecRun *er : ex->finished) {
        if (er->done) cudaEventDestroy(er->done);
        delete er;
    }
    for (cudaEvent_t e : ex->inflight) cudaEventDestroy(e);
    for (cudaEvent_t e : ex->spare) cudaEventDestroy(e);
    if (ex->d_groups) cudaFree(ex->d_groups);
    cudaFree(ex->d_err);
    cudaFreeHost(ex->h_err);
    cudaStreamDestroy(ex->stream);
    delete ex;
    return FWI_OK;
}
