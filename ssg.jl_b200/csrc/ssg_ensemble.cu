// ssg_ensemble.cu -- several contexts on one GPU advanced together (no
// counterpart in SSG.jl, which runs one problem per process).
//
// Two ways, chosen at creation:
//  - SSG_ENSEMBLE_THREADS: every member steps as in ssg_step (whole steps as
//    cached CUDA graphs on the member's own stream, iteration loops as
//    conditional while nodes); worker threads issue the members' graph
//    launches in parallel, so the host keeps the streams fed.
//  - SSG_ENSEMBLE_ONE_GRAPH: one graph captured from an ensemble stream that
//    forks into every member's stream and joins back, each member's steps an
//    independent branch; one launch advances every member by a chunk of steps
//    (the least common multiple of the members' predictor-ring periods, after
//    which every member's buffer assignment repeats and the same graph serves
//    the next chunk).
// On the 80-member 128^2/256^2 workload the one-graph form is the faster of
// the two (1287 ensemble steps/s, 1400 with tuned kernels, against 1130 for
// the threaded form, which depends on host thread scheduling).  Members of one
// grid do better still as the members of one context (ssg_config.nmembers,
// moved there by ssg_members_gather below): 1942 ensemble steps/s, with the two
// batched contexts advanced by one one-graph ensemble.
#include "ctx.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <thread>

namespace {

int gcd(int a, int b) {
    while (b) {
        const int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

int member_period(const ssg_ctx* c) {
    const int spp = c->cfg.ma_per_stage ? (c->cfg.scheme == SSG_SCHEME_RK3 ? 3 : 1) : 0;
    const int pred = c->cfg.ma_predictor;
    if (spp == 0 || pred == 0) return 1;
    const int cap = pred + 1;
    return cap / gcd(cap, spp);
}

bool member_warm(const ssg_ctx* c) {
    const int cap = c->cfg.ma_predictor >= 1 ? c->cfg.ma_predictor + 1 : 1;
    return c->cfg.ma_predictor == 0 || !c->cfg.ma_per_stage || c->nhist >= cap;
}

}  // namespace

struct ssg_ensemble {
    std::vector<ssg_ctx*> m;
    int device = 0;
    int mode = SSG_ENSEMBLE_THREADS;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> fork, join;
    struct Cached {
        std::vector<uint64_t> key;
        cudaGraphExec_t exec;
    };
    std::vector<Cached> graphs;
    int chunk = 1;
    std::string err;
};

static int efail(ssg_ensemble* e, int code, const std::string& msg) {
    if (e) e->err = msg;
    else set_global_error(msg.c_str());
    return code;
}

#define ECU(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return efail(e, SSG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

static void ensemble_release(ssg_ensemble* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (auto& g : e->graphs) cudaGraphExecDestroy(g.exec);
    e->graphs.clear();
    for (auto ev : e->fork) cudaEventDestroy(ev);
    for (auto ev : e->join) cudaEventDestroy(ev);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->stream) cudaStreamDestroy(e->stream);
}

extern "C" int ssg_ensemble_create(ssg_ctx* const* members, int32_t n, int32_t mode, ssg_ensemble** out) {
    if (!members || n < 1 || !out) return efail(nullptr, SSG_ERR_ARG, "ensemble_create: need members");
    if (mode != SSG_ENSEMBLE_THREADS && mode != SSG_ENSEMBLE_ONE_GRAPH)
        return efail(nullptr, SSG_ERR_ARG, "ensemble_create: unknown mode");
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (!members[i]) return efail(nullptr, SSG_ERR_ARG, "ensemble_create: null member");
        if (members[i]->device != members[0]->device)
            return efail(nullptr, SSG_ERR_ARG, "ensemble_create: members must share one device");
        for (int j = 0; j < i; ++j)
            if (members[j] == members[i]) return efail(nullptr, SSG_ERR_ARG, "ensemble_create: repeated member");
    }
    ssg_ensemble* e = new ssg_ensemble();
    e->mode = mode;
    e->m.assign(members, members + n);
    e->device = members[0]->device;
    int chunk = 1;
    for (ssg_ctx* c : e->m) {
        const int p = member_period(c);
        chunk = chunk / gcd(chunk, p) * p;
    }
    e->chunk = chunk;
    auto bail = [&](const char* what) {
        std::string msg = std::string("ensemble_create: ") + what;
        ensemble_release(e);
        delete e;
        set_global_error(msg.c_str());
        return SSG_ERR_CUDA;
    };
    if (cudaSetDevice(e->device) != cudaSuccess) return bail("cudaSetDevice");
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) return bail("stream");
    if (cudaEventCreate(&e->ev0) != cudaSuccess || cudaEventCreate(&e->ev1) != cudaSuccess) return bail("events");
    e->fork.resize(n, nullptr);
    e->join.resize(n, nullptr);
    for (int i = 0; i < n; ++i)
        if (cudaEventCreateWithFlags(&e->fork[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming) != cudaSuccess)
            return bail("events");
    *out = e;
    return SSG_OK;
}

extern "C" int ssg_ensemble_destroy(ssg_ensemble* e) {
    if (!e) return SSG_OK;
    ensemble_release(e);
    delete e;
    return SSG_OK;
}

extern "C" const char* ssg_ensemble_last_error(const ssg_ensemble* e) { return e ? e->err.c_str() : ""; }

// ensemble stream waits for every member's stream, or every member's stream
// waits for the ensemble stream
static int ensemble_order(ssg_ensemble* e, bool members_first) {
    for (size_t i = 0; i < e->m.size(); ++i) {
        ssg_ctx* c = e->m[i];
        if (members_first) {
            ECU(cudaEventRecord(e->join[i], c->stream));
            ECU(cudaStreamWaitEvent(e->stream, e->join[i], 0));
        } else {
            ECU(cudaEventRecord(e->fork[i], e->stream));
            ECU(cudaStreamWaitEvent(c->stream, e->fork[i], 0));
        }
    }
    return SSG_OK;
}

// Capture `chunk` steps of every member into one graph: fork from the ensemble
// stream into the member streams, each member captures its steps on its own
// stream, join back.  Member host state is put back afterwards (the chunk
// returns every ring to its assignment).
static int capture_chunk(ssg_ensemble* e, cudaGraphExec_t* out) {
    const size_t n = e->m.size();
    struct Saved {
        double2* ring[4];
        double t;
        int64_t step;
        int nhist;
    };
    std::vector<Saved> saved(n);
    for (size_t i = 0; i < n; ++i) {
        ssg_ctx* c = e->m[i];
        saved[i] = Saved{{c->Phat, c->hist[0], c->hist[1], c->hist[2]}, c->t, c->step, c->nhist};
    }
    ECU(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed));
    int r = SSG_OK;
    for (size_t i = 0; i < n && r == SSG_OK; ++i) {
        if (cudaEventRecord(e->fork[i], e->stream) != cudaSuccess ||
            cudaStreamWaitEvent(e->m[i]->stream, e->fork[i], 0) != cudaSuccess)
            r = efail(e, SSG_ERR_CUDA, "ensemble capture: fork");
    }
    for (size_t i = 0; i < n && r == SSG_OK; ++i) {
        ssg_ctx* c = e->m[i];
        c->capturing = true;
        SolveAcc acc;
        for (int k = 0; k < e->chunk && r == SSG_OK; ++k) {
            r = advance_step(c, c->cfg.dt, acc, nullptr);
            if (r) r = efail(e, r, std::string("ensemble capture: ") + ssg_last_error(c));
        }
        c->capturing = false;
        if (r == SSG_OK && (cudaEventRecord(e->join[i], c->stream) != cudaSuccess ||
                            cudaStreamWaitEvent(e->stream, e->join[i], 0) != cudaSuccess))
            r = efail(e, SSG_ERR_CUDA, "ensemble capture: join");
    }
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    for (size_t i = 0; i < n; ++i) {
        ssg_ctx* c = e->m[i];
        c->capturing = false;
        c->Phat = saved[i].ring[0];
        for (int k = 0; k < 3; ++k) c->hist[k] = saved[i].ring[1 + k];
        c->t = saved[i].t;
        c->step = saved[i].step;
        c->nhist = saved[i].nhist;
    }
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (ce != cudaSuccess) return efail(e, SSG_ERR_CUDA, std::string("ensemble capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return efail(e, SSG_ERR_CUDA, std::string("ensemble instantiate: ") + cudaGetErrorString(ce));
    return SSG_OK;
}

extern "C" int ssg_ensemble_step(ssg_ensemble* e, int32_t nsteps, ssg_step_stats* stats) {
    if (!e) return SSG_ERR_ARG;
    if (nsteps < 0) return efail(e, SSG_ERR_ARG, "nsteps < 0");
    ECU(cudaSetDevice(e->device));
    const size_t n = e->m.size();
    std::vector<SolveAcc> acc(n);
    int r;
    for (ssg_ctx* c : e->m) {
        if (c->profiling) return efail(e, SSG_ERR_ARG, "ensemble_step: a member has kernel profiling on");
        if ((r = reset_device_stats(c))) return efail(e, r, ssg_last_error(c));
    }
    ECU(cudaEventRecord(e->ev0, e->m[0]->stream));
    // members start where they are: each steps alone until its predictor
    // history is full, then all advance together chunk by chunk
    std::vector<int> done(n, 0);
    for (size_t i = 0; i < n; ++i) {
        ssg_ctx* c = e->m[i];
        while (done[i] < nsteps && !member_warm(c)) {
            if ((r = advance_step(c, c->cfg.dt, acc[i], nullptr))) return efail(e, r, ssg_last_error(c));
            done[i] += 1;
        }
    }
    int common = nsteps;
    for (size_t i = 0; i < n; ++i) common = std::min(common, nsteps - done[i]);
    const int chunks = (e->chunk > 0 && e->mode == SSG_ENSEMBLE_ONE_GRAPH) ? common / e->chunk : 0;
    if (chunks > 0) {
        std::vector<uint64_t> key;
        for (ssg_ctx* c : e->m) {
            key.push_back((uint64_t)c->Phat);
            for (int k = 0; k < 3; ++k) key.push_back((uint64_t)c->hist[k]);
            key.push_back((uint64_t)c->nhist);
            key.push_back(bits_of(c->cfg.dt));
        }
        cudaGraphExec_t ge = nullptr;
        for (auto& g : e->graphs)
            if (g.key == key) ge = g.exec;
        if ((r = ensemble_order(e, true))) return r;
        if (!ge) {
            if (e->graphs.size() >= 8) {
                ECU(cudaStreamSynchronize(e->stream));
                for (auto& g : e->graphs) cudaGraphExecDestroy(g.exec);
                e->graphs.clear();
            }
            if ((r = capture_chunk(e, &ge))) return r;
            e->graphs.push_back({key, ge});
        }
        for (int k = 0; k < chunks; ++k) ECU(cudaGraphLaunch(ge, e->stream));
        if ((r = ensemble_order(e, false))) return r;
        for (size_t i = 0; i < n; ++i) {
            ssg_ctx* c = e->m[i];
            for (int k = 0; k < chunks * e->chunk; ++k) c->t += c->cfg.dt;
            c->step += (int64_t)chunks * e->chunk;
            done[i] += chunks * e->chunk;
        }
    }
    // the remaining steps (all of them in threaded mode): each member as in
    // ssg_step, worker threads issuing in parallel
    {
        // the workers mostly wait in the driver's launch path: as many as
        // members, up to 32
        const size_t nw = std::min<size_t>(n, 32);
        std::vector<int> rc(n, SSG_OK);
        auto work = [&](size_t w) {
            cudaSetDevice(e->device);
            for (size_t i = w; i < n; i += nw) {
                ssg_ctx* c = e->m[i];
                rc[i] = run_steps(c, c->cfg.dt, nsteps - done[i], acc[i]);
            }
        };
        if (nw <= 1) {
            work(0);
        } else {
            std::vector<std::thread> th;
            for (size_t w = 0; w < nw; ++w) th.emplace_back(work, w);
            for (auto& t : th) t.join();
        }
        for (size_t i = 0; i < n; ++i)
            if (rc[i]) return efail(e, rc[i], ssg_last_error(e->m[i]));
    }
    for (size_t i = 1; i < n; ++i) {
        ECU(cudaEventRecord(e->join[i], e->m[i]->stream));
        ECU(cudaStreamWaitEvent(e->m[0]->stream, e->join[i], 0));
    }
    ECU(cudaEventRecord(e->ev1, e->m[0]->stream));
    int status = SSG_OK;
    for (size_t i = 0; i < n; ++i) {
        ssg_ctx* c = e->m[i];
        ECU(cudaMemcpyAsync(c->h_flag, c->nonfinite, sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream));
        if ((r = merge_device_stats(c, acc[i])) && status == SSG_OK) status = efail(e, r, ssg_last_error(c));
        if (*c->h_flag && status == SSG_OK) status = efail(e, SSG_ERR_NONFINITE, "a member's buoyancy became non-finite");
        if (stats) {
            ssg_step_stats& s = stats[i];
            s.steps = nsteps;
            s.ma_solves = acc[i].solves;
            s.ma_iterations = acc[i].iters;
            s.ma_iterations_max = acc[i].itmax;
            s.ma_unconverged = acc[i].unconv;
            s.pad0 = 0;
            s.ma_update_max = acc[i].updmax;
            s.t = c->t;
            s.step = c->step;
        }
    }
    ECU(cudaEventSynchronize(e->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    for (ssg_ctx* c : e->m) c->last_ms = ms;
    return status;
}

// ---------------------------------------------------------------------------
// State transfer between one-member contexts and the members of one context
// (ssg_config.nmembers): device-to-device copies of each member's buoyancy,
// AB2 history / RK3 stage buffers and potential history, in the predictor
// ring's logical order (newest first).
// ---------------------------------------------------------------------------
// equal apart from nmembers and filter_type (the transfer table itself is
// compared and copied: ssg_set_filter_table marks a context's type custom)
static bool same_config(ssg_config a, ssg_config b) {
    a.nmembers = b.nmembers = 0;
    a.filter_type = b.filter_type = 0;
    return std::memcmp(&a, &b, sizeof(a)) == 0;
}

// checks that solo[0..n) can be the members of batch; the clock, predictor
// history length and the device tables must agree
static int check_members(ssg_ctx* batch, ssg_ctx* const* solo, int32_t n, bool gather) {
    if (!batch || !solo) return SSG_ERR_ARG;
    if (n != batch->d.members) return fail(batch, SSG_ERR_ARG, "members: n must equal the context's nmembers");
    ssg_ctx* ctx = batch;  // CU's error slot
    const size_t c2 = batch->d.c2();
    std::vector<double> sig0(c2), sig(c2);
    ZOps z0{}, z{};
    for (int i = 0; i < n; ++i) {
        ssg_ctx* s = solo[i];
        if (!s || s == batch) return fail(batch, SSG_ERR_ARG, "members: null or repeated context");
        if (s->d.members != 1) return fail(batch, SSG_ERR_ARG, "members: one-member contexts only");
        if (s->device != batch->device) return fail(batch, SSG_ERR_ARG, "members: contexts on different devices");
        if (!same_config(s->cfg, batch->cfg))
            return fail(batch, SSG_ERR_ARG, "members: configurations differ (apart from nmembers)");
        if (gather && i > 0 &&
            (s->step != solo[0]->step || bits_of(s->t) != bits_of(solo[0]->t) || s->nhist != solo[0]->nhist))
            return fail(batch, SSG_ERR_ARG, "members: clocks or predictor histories differ");
        CU(cudaStreamSynchronize(s->stream));
        if (gather) {
            // the vertical operator and filter table of every member equal solo[0]'s
            CU(cudaMemcpy(i == 0 ? sig0.data() : sig.data(), s->sigma, c2 * sizeof(double), cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(i == 0 ? &z0 : &z, s->zops, sizeof(ZOps), cudaMemcpyDeviceToHost));
            if (i > 0 && (std::memcmp(sig0.data(), sig.data(), c2 * sizeof(double)) != 0 ||
                          std::memcmp(&z0, &z, sizeof(ZOps)) != 0))
                return fail(batch, SSG_ERR_ARG, "members: filter tables or vertical grids differ");
        }
    }
    return SSG_OK;
}

extern "C" int ssg_members_gather(ssg_ctx* batch, ssg_ctx* const* solo, int32_t n) {
    int r = check_members(batch, solo, n, true);
    if (r) return r;
    ssg_ctx* ctx = batch;
    CU(cudaSetDevice(ctx->device));
    CU(cudaStreamSynchronize(ctx->stream));
    const Dims& d = ctx->d;
    const size_t c2 = d.c2(), c3 = c2 * d.nz, b2 = c2 * sizeof(double2), b3 = c3 * sizeof(double2);
    cudaStream_t st = ctx->stream;
    // tables of solo[0]: filter transfer, vertical operator and its pivots
    CU(cudaMemcpyAsync(ctx->sigma, solo[0]->sigma, c2 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CU(cudaMemcpyAsync(ctx->zops, solo[0]->zops, sizeof(ZOps), cudaMemcpyDeviceToDevice, st));
    CU(cudaMemcpyAsync(ctx->tinv, solo[0]->tinv, (size_t)(d.nz - 2) * pivot_plane(d.Mx, d.My) * sizeof(double),
                       cudaMemcpyDeviceToDevice, st));
    reset_ring(ctx);
    for (int i = 0; i < n; ++i) {
        const ssg_ctx* s = solo[i];
        CU(cudaMemcpyAsync(ctx->bh + c2 * i, s->bh, b2, cudaMemcpyDeviceToDevice, st));
        CU(cudaMemcpyAsync(ctx->fold + c2 * i, s->fold, b2, cudaMemcpyDeviceToDevice, st));
        CU(cudaMemcpyAsync(ctx->bstage + c2 * i, s->bstage, b2, cudaMemcpyDeviceToDevice, st));
        CU(cudaMemcpyAsync(ctx->Phat + c3 * i, s->Phat, b3, cudaMemcpyDeviceToDevice, st));
        for (int k = 0; k < 3; ++k)
            CU(cudaMemcpyAsync(ctx->hist[k] + c3 * i, s->hist[k], b3, cudaMemcpyDeviceToDevice, st));
    }
    ctx->nhist = solo[0]->nhist;
    ctx->last_ma_iterations = solo[0]->last_ma_iterations;
    ctx->cfg.filter_type = solo[0]->cfg.filter_type;
    return set_clock(ctx, solo[0]->t, solo[0]->step);
}

extern "C" int ssg_members_scatter(ssg_ctx* batch, ssg_ctx* const* solo, int32_t n) {
    int r = check_members(batch, solo, n, false);
    if (r) return r;
    ssg_ctx* ctx = batch;
    CU(cudaSetDevice(ctx->device));
    CU(cudaStreamSynchronize(ctx->stream));
    const Dims& d = ctx->d;
    const size_t c2 = d.c2(), c3 = c2 * d.nz, b2 = c2 * sizeof(double2), b3 = c3 * sizeof(double2);
    cudaStream_t st = ctx->stream;
    for (int i = 0; i < n; ++i) {
        ssg_ctx* s = solo[i];
        reset_ring(s);
        CU(cudaMemcpyAsync(s->bh, ctx->bh + c2 * i, b2, cudaMemcpyDeviceToDevice, st));
        CU(cudaMemcpyAsync(s->fold, ctx->fold + c2 * i, b2, cudaMemcpyDeviceToDevice, st));
        CU(cudaMemcpyAsync(s->bstage, ctx->bstage + c2 * i, b2, cudaMemcpyDeviceToDevice, st));
        CU(cudaMemcpyAsync(s->Phat, ctx->Phat + c3 * i, b3, cudaMemcpyDeviceToDevice, st));
        for (int k = 0; k < 3; ++k)
            CU(cudaMemcpyAsync(s->hist[k], ctx->hist[k] + c3 * i, b3, cudaMemcpyDeviceToDevice, st));
    }
    CU(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) {
        ssg_ctx* s = solo[i];
        s->nhist = ctx->nhist;
        s->last_ma_iterations = ctx->last_ma_iterations;
        if ((r = set_clock(s, ctx->t, ctx->step))) return fail(ctx, r, "members: " + s->err);
    }
    return SSG_OK;
}
