// ssg_adjoint.cu -- discrete adjoint of the time step (no counterpart in SSG.jl).
//
// Record: set_b!(b0), then nsteps steps, with a device checkpoint of the whole
// step state (b_hat, AB2 history / RK3 buffers, Phi_hat and the predictor's
// previous solution, clock) every ckpt_every steps, and one of the final state.
//
// Reverse: the cotangent lam_b = P_V dL/db_T (compact coordinates of its
// projection on the kept modes) runs backwards one segment at a time: restore
// the segment's checkpoint, recompute its steps while recording the buoyancy
// entering every tendency stage and the potential solved from it (StepTape),
// then apply the transposed stages in reverse order.  The recording itself
// tapes the last segment, which therefore needs no recomputation (with
// ckpt_every >= nsteps nothing is recomputed).  The recomputation
// reproduces the recorded trajectory bit for bit: same kernels, same predictor
// history, deterministic reductions.
//
// Transposed stage at (b, Phi(b)) with cotangent lam on its tendency f:
//   lam_b += P_V[u dx(mu) + v dy(mu)] + S'(b)^T gphi,   mu = D lam,
//   gphi   = P_V[dy(b dx(mu)) - dx(b dy(mu))]   (cotangent on phi_s),
// where S'(b)^T is the transposed derivative of the converged Monge-Ampere
// solution (implicit-function theorem): with G the per-mode vertical solve and
// F(Phi) = P_V FFT(Phi_xx Phi_yy - Phi_xy^2) on the interior planes, the
// forward fixed point Phi = G(eps F(Phi), b) gives
//   y = G^T (gphi e_top + eps F'(Phi)^T y),   S'(b)^T gphi = (d G / d b)^T(...)
// solved by fixed-point iteration (the transpose of the forward iteration's
// linearisation, so the same contraction rate), started from the cubic
// extrapolation of the previous adjoint solutions of the same stage.
#include "ctx.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace {

struct CkptMeta {
    double t = 0.0;
    int64_t step = 0;
    int nhist = 0;
};

}  // namespace

struct AdjointState {
    // the recorded run
    bool recorded = false;
    int nsteps = 0, every = 0, nseg = 0, stages = 1;
    double h = 0.0;
    std::vector<CkptMeta> meta;  // nseg + 1 entries; the last is the final state
    double2* ck = nullptr;       // checkpoint slots: [bh, fold, bstage, Phat, hist[0..2] (nz each)]
    int ck_slots = 0;
    // tapes of one segment each: every * stages * (b: c2, Phi: c2 nz).  With
    // two, the recomputation of segment s-1 (on rstream) runs while segment s
    // is reversed (on the context's stream); tape points at the one in use.
    double2* tape = nullptr;
    double2* tapes[2] = {};
    int tape_held[2] = {-1, -1}; // segment whose stages each tape holds (-1: none)
    int ntapes = 0;
    int tape_steps = 0;
    int tape_seg = -1;           // segment whose stages the recording left in tapes[0] (-1: none)
    cudaStream_t rstream = nullptr;
    cudaEvent_t ev_done[2] = {}, ev_free[2] = {};
    // adjoint workspace
    bool ws = false;
    double2 *lb = nullptr, *lf = nullptr, *lk1 = nullptr, *lk2 = nullptr, *ly = nullptr;
    double2 *gphi = nullptr, *gb = nullptr;
    // adjoint solutions (interior planes) and their predictor history, one per
    // tendency stage: a stage's cotangent varies smoothly from step to step,
    // while consecutive stages of one step carry different stage weights
    double2* Y[3][4] = {};       // [stage][ring slot], slot 0 the newest
    double2* Y_base[3][4] = {};  // the same buffers in allocation order
    double2* G[3][4] = {};       // the top cotangents the ring's solutions were solved for
    double2* G_base[3][4] = {};
    int yhist[3] = {0, 0, 0};
    double2 *Hxx = nullptr, *Hyy = nullptr, *Hxy = nullptr;
    // the transposed solves' own transform workspace and norm reduction, so
    // that they may run while a recomputation uses the context's
    double2 *A = nullptr, *B = nullptr, *C = nullptr, *Dt = nullptr, *Dh = nullptr;
    double* partials = nullptr;
    unsigned int* ticket = nullptr;
    double* norms = nullptr;
    double2* P[5] = {};
    double2* Q[3] = {};
    std::vector<void*> mem_ws, mem_ck, mem_tape;
    int64_t bytes_ws = 0, bytes_ck = 0, bytes_tape = 0;
    // counters of the current call (host loop), and the device counters of
    // solves that ran inside graphs
    int solves = 0, iters = 0, itmax = 0, unconv = 0;
    double updmax = 0.0;
    SolveDev* sdev = nullptr;
    SolveDev* h_sdev = nullptr;  // pinned
};

static void free_list(std::vector<void*>& l, int64_t& bytes) {
    for (void* p : l) cudaFree(p);
    l.clear();
    bytes = 0;
}

void adjoint_release(ssg_ctx* ctx) {
    if (!ctx || !ctx->adj) return;
    release_graphs(ctx);
    AdjointState* st = ctx->adj;
    if (st->rstream) cudaStreamSynchronize(st->rstream);
    if (st->h_sdev) cudaFreeHost(st->h_sdev);
    for (int i = 0; i < 2; ++i) {
        if (st->ev_done[i]) cudaEventDestroy(st->ev_done[i]);
        if (st->ev_free[i]) cudaEventDestroy(st->ev_free[i]);
    }
    if (st->rstream) cudaStreamDestroy(st->rstream);
    free_list(st->mem_ws, st->bytes_ws);
    free_list(st->mem_ck, st->bytes_ck);
    free_list(st->mem_tape, st->bytes_tape);
    delete st;
    ctx->adj = nullptr;
}

template <typename T>
static int amalloc(ssg_ctx* ctx, std::vector<void*>& list, int64_t& bytes, T** p, size_t count) {
    void* q = nullptr;
    const size_t n = count * sizeof(T);
    cudaError_t e = cudaMalloc(&q, n + 256);
    if (e != cudaSuccess)
        return fail(ctx, SSG_ERR_OOM, std::string("cudaMalloc (adjoint): ") + cudaGetErrorString(e));
    list.push_back(q);
    bytes += (int64_t)n;
    *p = static_cast<T*>(q);
    return SSG_OK;
}

static size_t slot_elems(const Dims& d) { return (3 + 4 * (size_t)d.nz) * d.c2(); }
static size_t tape_step_elems(const Dims& d, int stages) { return (size_t)stages * (1 + (size_t)d.nz) * d.c2(); }

static int ensure_ws(ssg_ctx* ctx, AdjointState* st) {
    if (st->ws) return SSG_OK;
    const Dims& d = ctx->d;
    const size_t c2 = d.c2(), nzi = (size_t)d.nz - 2, hplane = d.r2() / 2;
    int r;
    for (double2** p : {&st->lb, &st->lf, &st->lk1, &st->lk2, &st->ly, &st->gphi, &st->gb})
        if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, p, c2))) return r;
    for (int s = 0; s < 3; ++s)
        for (int k = 0; k < 4; ++k) {
            if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, &st->Y[s][k], c2 * nzi))) return r;
            st->Y_base[s][k] = st->Y[s][k];
            if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, &st->G[s][k], c2))) return r;
            st->G_base[s][k] = st->G[s][k];
        }
    for (double2** p : {&st->Hxx, &st->Hyy, &st->Hxy})
        if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, p, hplane * nzi))) return r;
    for (int i = 0; i < 5; ++i)
        if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, &st->P[i], d.m2()))) return r;
    for (int i = 0; i < 3; ++i)
        if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, &st->Q[i], d.m2()))) return r;
    for (double2** p : {&st->A, &st->B, &st->C, &st->Dt})
        if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, p, d.m2() * nzi))) return r;
    if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, &st->Dh, c2 * nzi))) return r;
    const size_t nblk = (c2 + 31) / 32 + 1;
    if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, &st->partials, 2 * nblk))) return r;
    if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, &st->ticket, 1))) return r;
    if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, &st->norms, 2))) return r;
    CU(cudaMemsetAsync(st->ticket, 0, sizeof(unsigned int), ctx->stream));
    if ((r = amalloc(ctx, st->mem_ws, st->bytes_ws, &st->sdev, 1))) return r;
    if (cudaMallocHost(&st->h_sdev, sizeof(SolveDev)) != cudaSuccess)
        return fail(ctx, SSG_ERR_OOM, "cudaMallocHost (adjoint) failed");
    CU(cudaStreamCreateWithFlags(&st->rstream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
        CU(cudaEventCreateWithFlags(&st->ev_done[i], cudaEventDisableTiming));
        CU(cudaEventCreateWithFlags(&st->ev_free[i], cudaEventDisableTiming));
    }
    st->ws = true;
    return SSG_OK;
}

static int ensure_ck(ssg_ctx* ctx, AdjointState* st, int slots) {
    if (st->ck_slots >= slots) return SSG_OK;
    // (checkpoints are copied by the host between graph launches; no graph
    // bakes in their address)
    CU(cudaStreamSynchronize(ctx->stream));
    free_list(st->mem_ck, st->bytes_ck);
    st->ck_slots = 0;
    int r;
    if ((r = amalloc(ctx, st->mem_ck, st->bytes_ck, &st->ck, slot_elems(ctx->d) * (size_t)slots))) return r;
    st->ck_slots = slots;
    return SSG_OK;
}

// ntapes tapes of `steps` steps (two when segments are recomputed, so that a
// recomputation can run while the previous segment is reversed)
static int ensure_tape(ssg_ctx* ctx, AdjointState* st, int steps, int ntapes) {
    if (st->tape_steps >= steps && st->ntapes >= ntapes) return SSG_OK;
    CU(cudaStreamSynchronize(ctx->stream));
    if (st->rstream) CU(cudaStreamSynchronize(st->rstream));
    // keep what was there: graphs bake in tape addresses, so the tapes only grow
    const int nt = std::max(ntapes, st->ntapes);
    steps = std::max(steps, st->tape_steps);
    release_graphs(ctx);
    free_list(st->mem_tape, st->bytes_tape);
    st->tape_steps = 0;
    st->ntapes = 0;
    st->tapes[0] = st->tapes[1] = st->tape = nullptr;
    st->tape_held[0] = st->tape_held[1] = -1;
    int r;
    for (int i = 0; i < nt; ++i)
        if ((r = amalloc(ctx, st->mem_tape, st->bytes_tape, &st->tapes[i],
                         tape_step_elems(ctx->d, st->stages) * (size_t)steps)))
            return r;
    st->tape = st->tapes[0];
    st->tape_steps = steps;
    st->ntapes = nt;
    return SSG_OK;
}

static StepTape tape_of(const ssg_ctx* ctx, const AdjointState* st, int i) {
    const Dims& d = ctx->d;
    const size_t c2 = d.c2();
    double2* base = st->tape + tape_step_elems(d, st->stages) * (size_t)i;
    StepTape tp{};
    for (int s = 0; s < st->stages; ++s) {
        tp.b[s] = base + (size_t)s * (1 + d.nz) * c2;
        tp.phi[s] = tp.b[s] + c2;
    }
    return tp;
}

static int save_ckpt(ssg_ctx* ctx, AdjointState* st, int i) {
    const Dims& d = ctx->d;
    const size_t c2 = d.c2(), cb = c2 * sizeof(double2);
    double2* p = st->ck + slot_elems(d) * (size_t)i;
    const auto D2D = cudaMemcpyDeviceToDevice;
    CU(cudaMemcpyAsync(p, ctx->bh, cb, D2D, ctx->stream));
    CU(cudaMemcpyAsync(p + c2, ctx->fold, cb, D2D, ctx->stream));
    CU(cudaMemcpyAsync(p + 2 * c2, ctx->bstage, cb, D2D, ctx->stream));
    CU(cudaMemcpyAsync(p + 3 * c2, ctx->Phat, cb * d.nz, D2D, ctx->stream));
    for (int h = 0; h < 3; ++h)
        CU(cudaMemcpyAsync(p + (3 + (1 + h) * d.nz) * c2, ctx->hist[h], cb * d.nz, D2D, ctx->stream));
    st->meta[i].t = ctx->t;
    st->meta[i].step = ctx->step;
    st->meta[i].nhist = ctx->nhist;
    return SSG_OK;
}

// the forward state of checkpoint i, copied on stream s (the clock's device
// copy included)
static int restore_ckpt(ssg_ctx* ctx, AdjointState* st, int i, cudaStream_t s) {
    const Dims& d = ctx->d;
    const size_t c2 = d.c2(), cb = c2 * sizeof(double2);
    const double2* p = st->ck + slot_elems(d) * (size_t)i;
    const auto D2D = cudaMemcpyDeviceToDevice;
    CU(cudaMemcpyAsync(ctx->bh, p, cb, D2D, s));
    CU(cudaMemcpyAsync(ctx->fold, p + c2, cb, D2D, s));
    CU(cudaMemcpyAsync(ctx->bstage, p + 2 * c2, cb, D2D, s));
    CU(cudaMemcpyAsync(ctx->Phat, p + 3 * c2, cb * d.nz, D2D, s));
    for (int h = 0; h < 3; ++h)
        CU(cudaMemcpyAsync(ctx->hist[h], p + (3 + (1 + h) * d.nz) * c2, cb * d.nz, D2D, s));
    ctx->nhist = st->meta[i].nhist;
    if (s == ctx->stream) return set_clock(ctx, st->meta[i].t, st->meta[i].step);
    ctx->t = st->meta[i].t;
    ctx->step = st->meta[i].step;
    CU(cudaMemcpyAsync(ctx->step_dev, &ctx->step, sizeof(int64_t), cudaMemcpyHostToDevice, s));
    CU(cudaStreamSynchronize(s));
    return SSG_OK;
}

// S'(b)^T: the cotangent on b of the Monge-Ampere solution at potential phat,
// for the cotangent st->gphi on its top plane, written to st->gb.  stage
// selects the predictor history.
static int adj_ma_solve(ssg_ctx* ctx, AdjointState* st, const double2* phat, int stage) {
    const Dims& d = ctx->d;
    const Tables tb = ctx->tables();
    const size_t nzi = (size_t)d.nz - 2, ny = d.c2() * nzi;
    const int volume = ctx->cfg.ma_rhs_mode == SSG_MA_RHS_VOLUME ? 1 : 0;
    // the linearisation's fixed fields: Phi_xx, Phi_yy, Phi_xy of this potential
    KLC(KC_ADJ_XINV, launch_ma_xinv3(d, tb, phat, st->A, st->B, st->C, ctx->stream));
    KLC(KC_ADJ_Y, launch_ma_hess_y(d, tb, st->A, st->B, st->C, st->Hxx, st->Hyy, st->Hxy, ctx->stream));
    // predictor: cubic extrapolation through this stage's last four solutions
    // (ring as in the forward solve; on the 256^2 x 16 RK3 adjoint workload it
    // takes 5.4 iterations per solve against 6.4 for the quadratic one)
    // With ma_bc_guess the guess is also corrected for this solve's top
    // cotangent (launch_adj_predict_bc); the ring G of the cotangents the
    // history was solved for rotates with Y.
    {
        double2** S = st->Y[stage];
        double2** Gr = st->G[stage];
        const bool bc = ctx->cfg.ma_bc_guess != 0;
        const int pred = 3;
        const int cap = pred + 1, h = st->yhist[stage];
        if (h >= 1) {
            const int t = h < cap ? h : cap - 1;
            const int order = pred < h - 1 ? pred : h - 1;
            if (bc)
                KL(launch_adj_predict_bc(d, S, S[t], order, Gr, Gr[t], st->gphi, ctx->tinv, ctx->zops, ctx->stream));
            else
                KL(launch_predict(S[0], S[1], S[2], S[3], S[t], order, ny, ctx->stream));
            double2* y = S[t];
            double2* g = Gr[t];
            for (int i = t; i > 0; --i) {
                S[i] = S[i - 1];
                Gr[i] = Gr[i - 1];
            }
            S[0] = y;
            Gr[0] = g;
        } else if (bc) {
            CU(cudaMemcpyAsync(Gr[0], st->gphi, d.c2() * sizeof(double2), cudaMemcpyDeviceToDevice, ctx->stream));
        }
        st->yhist[stage] = h < cap ? h + 1 : cap;
    }
    double2* Y = st->Y[stage][0];
    auto iteration = [&](cudaStream_t s) -> int {
        KLC(KC_ADJ_XINV, launch_x_inv_compact(d, tb, Y, st->Dt, (int)nzi, 0, s));
        KLC(KC_ADJ_Y, launch_adj_ma_y(d, tb, st->Dt, st->Hxx, st->Hyy, st->Hxy, st->A, st->B, st->C, ctx->cfg.eps,
                                      s));
        KLC(KC_ADJ_XFWD, launch_adj_ma_xfwd(d, tb, st->A, st->B, st->C, st->Dh, s));
        KLC(KC_ADJ_THOMAS, launch_adj_thomas(d, tb, ctx->zops, ctx->tinv, st->Dh, st->gphi, Y, st->gb, volume,
                                             st->partials, st->ticket, st->norms, ctx->thomas_staged, s));
        return SSG_OK;
    };
    if (ctx->capturing) {
        // inside a graph: the iterations as a conditional while node, stop
        // rule on the device (statistics into st->sdev)
        KL(launch_solve_begin(st->sdev, nullptr, 1, ctx->stream));
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        CU(cudaStreamGetCaptureInfo(ctx->stream, &cs, nullptr, &g, &deps, &ndeps));
        cudaGraphConditionalHandle hdl;
        CU(cudaGraphConditionalHandleCreate(&hdl, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = hdl;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        CU(cudaGraphAddNode(&node, g, deps, ndeps, &np));
        CU(cudaStreamBeginCaptureToGraph(ctx->side, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeRelaxed));
        int r = iteration(ctx->side);
        if (!r && launch_solve_check(st->sdev, st->norms, nullptr, 1, ctx->cfg.ma_tol, ctx->cfg.ma_maxiter, 0, 0.0,
                                     (unsigned long long)hdl, nullptr, ctx->side))
            r = fail(ctx, SSG_ERR_CUDA, "solve_check launch failed");
        cudaGraph_t body = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->side, &body);
        if (r) return r;
        if (e != cudaSuccess)
            return fail(ctx, SSG_ERR_CUDA, std::string("capture of an adjoint iteration: ") + cudaGetErrorString(e));
        CU(cudaStreamUpdateCaptureDependencies(ctx->stream, &node, 1, cudaStreamSetCaptureDependencies));
        return SSG_OK;
    }
    double upd = 0.0;
    int it;
    bool conv = false;
    for (it = 1; it <= ctx->cfg.ma_maxiter; ++it) {
        int r = iteration(ctx->stream);
        if (r) return r;
        CU(cudaMemcpyAsync(ctx->h_norms, st->norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        if (ctx->profiling) drain_profile(ctx);
        const double ds = ctx->h_norms[0], ns = ctx->h_norms[1];
        upd = ns > 0 ? std::sqrt(ds / ns) : std::sqrt(ds);
        if (!(upd == upd) || std::isinf(upd))
            return fail(ctx, SSG_ERR_NONFINITE, "adjoint Monge-Ampere iteration produced a non-finite update");
        if (upd <= ctx->cfg.ma_tol) {
            conv = true;
            break;
        }
    }
    if (it > ctx->cfg.ma_maxiter) it = ctx->cfg.ma_maxiter;
    st->solves += 1;
    st->iters += it;
    st->itmax = std::max(st->itmax, it);
    st->updmax = std::max(st->updmax, upd);
    if (!conv) st->unconv += 1;
    return SSG_OK;
}

// Transposed tendency stage at (b, Phi): out = base + (cotangent on b of the
// stage tendency for cotangent lam).  base may be null or alias out.
static int adj_stage(ssg_ctx* ctx, AdjointState* st, int stage, const double2* bh, const double2* phat,
                     const double2* lam, const double2* base, double2* out) {
    const Dims& d = ctx->d;
    const Tables tb = ctx->tables();
    const double2* phih = phat + d.c2() * (d.nz - 1);
    KLC(KC_ADJ_SURF, launch_adj_surf_xinv5(d, tb, phih, bh, lam, st->P, ctx->stream));
    KLC(KC_ADJ_SURF, launch_adj_surf_y(d, tb, st->P, st->Q, ctx->stream));
    KLC(KC_ADJ_SURF, launch_adj_surf_xfwd(d, tb, st->Q, base, out, st->gphi, ctx->stream));
    int r = adj_ma_solve(ctx, st, phat, stage);
    if (r) return r;
    KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, out, out, 1.0, st->gb, 1.0, 0, ctx->stream));
    return SSG_OK;
}

// Transpose of step k (its clock step before the update) recorded in tp.
static int reverse_step(ssg_ctx* ctx, AdjointState* st, const StepTape& tp, int64_t k) {
    const Dims& d = ctx->d;
    const Tables tb = ctx->tables();
    cudaStream_t s = ctx->stream;
    const double h = st->h;
    const int ff = ctx->cfg.filter_freq;
    int r;
    // the filter acts on the updated buoyancy (diagonal, so its own transpose)
    if (ff > 0 && (k + 1) % ff == 0) KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, st->lb, st->lb, 1.0, nullptr, 0.0, 1, s));
    if (ctx->cfg.scheme == SSG_SCHEME_AB2) {
        // b+ = b + h f (first step) or b + h (1.5 f - 0.5 f_old); f_old <- f
        const bool first = k == 0;
        KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, st->lk1, st->lb, first ? h : 1.5 * h, st->lf, 1.0, 0, s));
        KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, st->lf, st->lb, first ? 0.0 : -0.5 * h, nullptr, 0.0, 0, s));
        if ((r = adj_stage(ctx, st, 0, tp.b[0], tp.phi[0], st->lk1, st->lb, st->lb))) return r;
    } else {
        // k1 = f(b); y1 = b + h/3 k1; k2 = f(y1); y2 = b + 2h/3 k2; k3 = f(y2);
        // b+ = b + h/4 (k1 + 3 k3)
        KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, st->lk1, st->lb, 0.25 * h, nullptr, 0.0, 0, s));
        KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, st->lk2, st->lb, 0.75 * h, nullptr, 0.0, 0, s));
        if ((r = adj_stage(ctx, st, 2, tp.b[2], tp.phi[2], st->lk2, nullptr, st->ly))) return r;
        KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, st->lb, st->lb, 1.0, st->ly, 1.0, 0, s));
        KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, st->lk2, st->ly, 2.0 * h / 3.0, nullptr, 0.0, 0, s));
        if ((r = adj_stage(ctx, st, 1, tp.b[1], tp.phi[1], st->lk2, nullptr, st->ly))) return r;
        KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, st->lb, st->lb, 1.0, st->ly, 1.0, 0, s));
        KLC(KC_ADJ_SURF, launch_adj_axpby(d, tb, st->lk1, st->lk1, 1.0, st->ly, h / 3.0, 0, s));
        if ((r = adj_stage(ctx, st, 0, tp.b[0], tp.phi[0], st->lk1, st->lb, st->lb))) return r;
    }
    return SSG_OK;
}

// len steps from the current state, taping step i into tape slot i: as one
// cached graph (the tape buffer, the ring assignment and the history count are
// baked in, and the state the steps leave behind is recorded with it), or
// step by step when graphs are off.
static int run_taped(ssg_ctx* ctx, AdjointState* st, int len, SolveAcc& acc, cudaStream_t launch_stream = nullptr) {
    int r;
    const double h = st->h;
    if (!launch_stream) launch_stream = ctx->stream;
    if (!ctx->graphs || ctx->profiling) {
        for (int i = 0; i < len; ++i) {
            const StepTape tp = tape_of(ctx, st, i);
            if ((r = advance_step(ctx, h, acc, &tp))) return r;
        }
        return SSG_OK;
    }
    const std::vector<uint64_t> key = {2, (uint64_t)ctx->Phat, (uint64_t)ctx->hist[0], (uint64_t)ctx->hist[1],
                                       (uint64_t)ctx->hist[2], bits_of(h), (uint64_t)len, (uint64_t)ctx->nhist,
                                       (uint64_t)st->tape};
    GraphEntry* ge = find_graph(ctx, key);
    if (!ge) {
        double2* ring[4] = {ctx->Phat, ctx->hist[0], ctx->hist[1], ctx->hist[2]};
        const double t0 = ctx->t;
        const int64_t s0 = ctx->step;
        const int nh0 = ctx->nhist;
        SolveAcc cap_acc;
        r = add_graph(ctx, key, [&] {
            int rr = SSG_OK;
            for (int i = 0; i < len && rr == SSG_OK; ++i) {
                const StepTape tp = tape_of(ctx, st, i);
                rr = advance_step(ctx, h, cap_acc, &tp);
            }
            return rr;
        }, &ge);
        if (!r)
            ge->post = {(uint64_t)ctx->Phat, (uint64_t)ctx->hist[0], (uint64_t)ctx->hist[1], (uint64_t)ctx->hist[2],
                        (uint64_t)ctx->nhist};
        ctx->Phat = ring[0];
        for (int i = 0; i < 3; ++i) ctx->hist[i] = ring[1 + i];
        ctx->t = t0;
        ctx->step = s0;
        ctx->nhist = nh0;
        if (r) return r;
    }
    CU(cudaGraphLaunch(ge->exec, launch_stream));
    ctx->Phat = reinterpret_cast<double2*>(ge->post[0]);
    for (int i = 0; i < 3; ++i) ctx->hist[i] = reinterpret_cast<double2*>(ge->post[1 + i]);
    ctx->nhist = (int)ge->post[4];
    for (int i = 0; i < len; ++i) ctx->t += h;
    ctx->step += len;
    return SSG_OK;
}

// The transposes of steps s1-1 .. s0 of the tape (clock steps k0 + i), as one
// cached graph (key: the adjoint predictor rings and counts, the segment
// length, and what the clock decides: the filter phase and AB2's first step).
static int run_reverse(ssg_ctx* ctx, AdjointState* st, int s0, int s1, int64_t k0) {
    int r;
    if (!ctx->graphs || ctx->profiling) {
        for (int s = s1 - 1; s >= s0; --s)
            if ((r = reverse_step(ctx, st, tape_of(ctx, st, s - s0), k0 + (s - s0)))) return r;
        return SSG_OK;
    }
    const int ff = ctx->cfg.filter_freq;
    std::vector<uint64_t> key = {3, (uint64_t)(s1 - s0), (uint64_t)(ff > 0 ? k0 % ff : 0), (uint64_t)(k0 == 0),
                                 (uint64_t)st->tape, bits_of(st->h)};
    for (int g = 0; g < 3; ++g) {
        key.push_back((uint64_t)st->yhist[g]);
        for (int k = 0; k < 4; ++k) key.push_back((uint64_t)st->Y[g][k]);
        for (int k = 0; k < 4; ++k) key.push_back((uint64_t)st->G[g][k]);
    }
    GraphEntry* ge = find_graph(ctx, key);
    if (!ge) {
        double2* ring[3][4];
        double2* gring[3][4];
        int yh[3];
        std::memcpy(ring, st->Y, sizeof(ring));
        std::memcpy(gring, st->G, sizeof(gring));
        std::memcpy(yh, st->yhist, sizeof(yh));
        r = add_graph(ctx, key, [&] {
            int rr = SSG_OK;
            for (int s = s1 - 1; s >= s0 && rr == SSG_OK; --s)
                rr = reverse_step(ctx, st, tape_of(ctx, st, s - s0), k0 + (s - s0));
            return rr;
        }, &ge);
        if (!r) {
            ge->post.clear();
            for (int g = 0; g < 3; ++g) {
                ge->post.push_back((uint64_t)st->yhist[g]);
                for (int k = 0; k < 4; ++k) ge->post.push_back((uint64_t)st->Y[g][k]);
                for (int k = 0; k < 4; ++k) ge->post.push_back((uint64_t)st->G[g][k]);
            }
        }
        std::memcpy(st->Y, ring, sizeof(ring));
        std::memcpy(st->G, gring, sizeof(gring));
        std::memcpy(st->yhist, yh, sizeof(yh));
        if (r) return r;
    }
    CU(cudaGraphLaunch(ge->exec, ctx->stream));
    for (int g = 0, p = 0; g < 3; ++g) {
        st->yhist[g] = (int)ge->post[p++];
        for (int k = 0; k < 4; ++k) st->Y[g][k] = reinterpret_cast<double2*>(ge->post[p++]);
        for (int k = 0; k < 4; ++k) st->G[g][k] = reinterpret_cast<double2*>(ge->post[p++]);
    }
    return SSG_OK;
}

static void fill_stats(const AdjointState* st, const SolveAcc& acc, double ms, ssg_adjoint_stats* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->steps = st->nsteps;
    out->checkpoints = st->nseg + 1;
    out->forward_solves = acc.solves;
    out->forward_iterations = acc.iters;
    out->adjoint_solves = st->solves;
    out->adjoint_iterations = st->iters;
    out->adjoint_iterations_max = st->itmax;
    out->adjoint_unconverged = st->unconv;
    out->adjoint_update_max = st->updmax;
    out->ms = ms;
    out->device_bytes = st->bytes_ws + st->bytes_ck + st->bytes_tape;
}

static int check_adjoint_config(ssg_ctx* ctx) {
    if (ctx->cfg.precision != 0)
        return fail(ctx, SSG_ERR_UNSUPPORTED, "adjoint: FP64 contexts only (precision 0)");
    if (!ctx->cfg.ma_per_stage)
        return fail(ctx, SSG_ERR_UNSUPPORTED, "adjoint: the potential must be re-solved every stage (ma_per_stage 1)");
    if (ctx->cfg.ab2_literal_alias && ctx->cfg.scheme == SSG_SCHEME_AB2)
        return fail(ctx, SSG_ERR_UNSUPPORTED, "adjoint: the conservative Jacobian only (ab2_literal_alias 0)");
    if (ctx->d.members > 1) return fail(ctx, SSG_ERR_UNSUPPORTED, "adjoint: one member per context (nmembers 1)");
    return SSG_OK;
}

extern "C" int ssg_adjoint_record(ssg_ctx* ctx, const double* b0, int64_t n, int32_t nsteps, int32_t ckpt_every,
                                  ssg_adjoint_stats* stats) {
    if (!ctx) return SSG_ERR_ARG;
    if (!b0 || n != (int64_t)ctx->d.r2()) return fail(ctx, SSG_ERR_ARG, "adjoint_record: expected nx*ny values");
    if (nsteps < 1 || ckpt_every < 1)
        return fail(ctx, SSG_ERR_ARG, "adjoint_record: nsteps and ckpt_every must be >= 1");
    int r;
    if ((r = check_adjoint_config(ctx))) return r;
    CU(cudaSetDevice(ctx->device));
    if (!ctx->adj) ctx->adj = new AdjointState();
    AdjointState* st = ctx->adj;
    st->recorded = false;
    st->nsteps = nsteps;
    st->every = std::min<int>(ckpt_every, nsteps);
    st->nseg = (nsteps + st->every - 1) / st->every;
    st->h = ctx->cfg.dt;
    st->stages = ctx->cfg.scheme == SSG_SCHEME_RK3 ? 3 : 1;
    st->meta.assign((size_t)st->nseg + 1, CkptMeta{});
    st->solves = st->iters = st->itmax = st->unconv = 0;
    st->updmax = 0.0;
    if ((r = ensure_ck(ctx, st, st->nseg + 1))) return r;
    // the last segment's stages are taped during the recording, so the
    // reverse sweep starts without a recomputation
    st->tape_seg = -1;
    if ((r = ensure_tape(ctx, st, st->every, st->nseg > 1 ? 2 : 1))) return r;
    st->tape = st->tapes[0];
    st->tape_held[0] = st->tape_held[1] = -1;
    const int s_last = (st->nseg - 1) * st->every;
    const int64_t l0 = launch_counter();
    CU(cudaEventRecord(ctx->ev0, ctx->stream));
    // set_b!: projection, fresh potential
    if ((r = upload_surface(ctx, b0, ctx->bh, 1))) return r;
    reset_ring(ctx);
    CU(cudaMemsetAsync(ctx->Phat, 0, ctx->d.c2() * ctx->d.nz * sizeof(double2), ctx->stream));
    SolveAcc acc;
    if ((r = solve_counted(ctx, acc))) return r;
    if ((r = reset_device_stats(ctx))) return r;
    for (int seg = 0; seg < st->nseg; ++seg) {
        const int s0 = seg * st->every, len = std::min(st->every, nsteps - s0);
        if ((r = save_ckpt(ctx, st, seg))) return r;
        if (s0 == s_last) r = run_taped(ctx, st, len, acc);
        else r = run_steps(ctx, st->h, len, acc);
        if (r) return r;
    }
    st->tape_seg = st->nseg - 1;
    st->tape_held[0] = st->nseg - 1;
    if ((r = save_ckpt(ctx, st, st->nseg))) return r;
    CU(cudaEventRecord(ctx->ev1, ctx->stream));
    CU(cudaMemcpyAsync(ctx->h_flag, ctx->nonfinite, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    if ((r = merge_device_stats(ctx, acc))) return r;
    if (ctx->profiling) drain_profile(ctx);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_ms = ms;
    ctx->last_launches = launch_counter() - l0;
    fill_stats(st, acc, ms, stats);
    if (*ctx->h_flag) return fail(ctx, SSG_ERR_NONFINITE, "surface buoyancy became non-finite");
    st->recorded = true;
    return SSG_OK;
}

extern "C" int ssg_adjoint(ssg_ctx* ctx, const double* dL_dbT, double* dL_db0, int64_t n, ssg_adjoint_stats* stats) {
    if (!ctx) return SSG_ERR_ARG;
    AdjointState* st = ctx->adj;
    if (!st || !st->recorded) return fail(ctx, SSG_ERR_ARG, "adjoint: no recorded run (call ssg_adjoint_record)");
    if (!dL_dbT || !dL_db0 || n != (int64_t)ctx->d.r2()) return fail(ctx, SSG_ERR_ARG, "adjoint: expected nx*ny values");
    int r;
    if ((r = check_adjoint_config(ctx))) return r;
    CU(cudaSetDevice(ctx->device));
    if ((r = ensure_ws(ctx, st))) return r;
    const Dims& d = ctx->d;
    st->solves = st->iters = st->itmax = st->unconv = 0;
    st->updmax = 0.0;
    const int64_t l0 = launch_counter();
    CU(cudaEventRecord(ctx->ev0, ctx->stream));
    // lam_b = coordinates of P_V dL/db_T; no AB2-history cotangent after the last step
    if ((r = upload_surface(ctx, dL_dbT, st->lb, 0))) return r;
    CU(cudaMemsetAsync(st->lf, 0, d.c2() * sizeof(double2), ctx->stream));
    std::memcpy(st->Y, st->Y_base, sizeof(st->Y));
    std::memcpy(st->G, st->G_base, sizeof(st->G));
    for (int s = 0; s < 3; ++s) {
        CU(cudaMemsetAsync(st->Y[s][0], 0, d.c2() * (d.nz - 2) * sizeof(double2), ctx->stream));
        st->yhist[s] = 0;
    }
    SolveAcc acc;
    if ((r = reset_device_stats(ctx))) return r;
    CU(cudaMemsetAsync(st->sdev, 0, sizeof(SolveDev), ctx->stream));
    // Segments from the last to the first.  With two tapes (and CUDA graphs),
    // segment s-1 is recomputed on rstream into one tape while segment s is
    // reversed from the other on the context's stream: the two share no
    // buffer (the transposed solves have their own workspace), and events
    // order each tape's reuse.  Otherwise recomputation and reversal alternate
    // on the context's stream.
    const bool overlap = st->ntapes == 2 && ctx->graphs && !ctx->profiling;
    cudaStream_t R = overlap ? st->rstream : ctx->stream;
    auto recompute = [&](int seg, int buf) -> int {
        const int a0 = seg * st->every, a1 = std::min(a0 + st->every, st->nsteps);
        int rr;
        if (overlap && st->tape_held[buf] >= 0) CU(cudaStreamWaitEvent(R, st->ev_free[buf], 0));
        if ((rr = restore_ckpt(ctx, st, seg, R))) return rr;
        st->tape = st->tapes[buf];
        st->tape_held[buf] = -1;
        if ((rr = run_taped(ctx, st, a1 - a0, acc, R))) return rr;
        st->tape_held[buf] = seg;
        if (overlap) CU(cudaEventRecord(st->ev_done[buf], R));
        return SSG_OK;
    };
    if (overlap) {
        // rstream's work follows the set-up above (statistics reset, cotangent upload)
        CU(cudaEventRecord(st->ev_done[1], ctx->stream));
        CU(cudaStreamWaitEvent(R, st->ev_done[1], 0));
    }
    int cur = st->tape_held[0] == st->nseg - 1 ? 0 : st->tape_held[1] == st->nseg - 1 ? 1 : -1;
    bool pending = false;  // the tape in use was recomputed on R
    if (cur < 0) {
        cur = 0;
        if ((r = recompute(st->nseg - 1, cur))) return r;
        pending = overlap;
    }
    for (int seg = st->nseg - 1; seg >= 0; --seg) {
        const int s0 = seg * st->every, s1 = std::min(s0 + st->every, st->nsteps);
        const int64_t k0 = st->meta[seg].step;
        if (pending) CU(cudaStreamWaitEvent(ctx->stream, st->ev_done[cur], 0));
        st->tape = st->tapes[cur];
        if ((r = run_reverse(ctx, st, s0, s1, k0))) return r;
        if (seg == 0) break;
        const int nxt = overlap ? (cur ^ 1) : cur;
        if (overlap) CU(cudaEventRecord(st->ev_free[cur], ctx->stream));
        if ((r = recompute(seg - 1, nxt))) return r;
        pending = overlap;
        cur = nxt;
    }
    if (overlap) {
        // the context's stream continues after rstream's last work
        CU(cudaEventRecord(st->ev_done[0], R));
        CU(cudaStreamWaitEvent(ctx->stream, st->ev_done[0], 0));
    }
    st->tape_seg = -1;
    // through set_b!'s projection
    KLC(KC_ADJ_SURF, launch_adj_setb(d, st->lb, st->ly, ctx->stream));
    CU(cudaEventRecord(ctx->ev1, ctx->stream));
    if ((r = merge_device_stats(ctx, acc))) return r;
    CU(cudaMemcpyAsync(st->h_sdev, st->sdev, sizeof(SolveDev), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    {
        const SolveDev& sd = *st->h_sdev;
        st->solves += sd.solves;
        st->iters += sd.iters;
        st->itmax = std::max(st->itmax, sd.itmax);
        st->unconv += sd.unconv;
        st->updmax = std::max(st->updmax, sd.updmax);
        if (sd.flags & 1u) return fail(ctx, SSG_ERR_NONFINITE, "adjoint Monge-Ampere iteration produced a non-finite update");
    }
    if ((r = download_planes(ctx, st->ly, 1, 0, dL_db0))) return r;
    if ((r = restore_ckpt(ctx, st, st->nseg, ctx->stream))) return r;
    CU(cudaStreamSynchronize(ctx->stream));
    if (ctx->profiling) drain_profile(ctx);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_ms = ms;
    ctx->last_launches = launch_counter() - l0;
    fill_stats(st, acc, ms, stats);
    for (size_t i = 0; i < d.r2(); ++i)
        if (!std::isfinite(dL_db0[i])) return fail(ctx, SSG_ERR_NONFINITE, "adjoint gradient is non-finite");
    return SSG_OK;
}
