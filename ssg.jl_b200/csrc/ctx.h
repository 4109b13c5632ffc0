// ctx.h -- the context object behind the C ABI and the internal interface
// shared by the files that drive it (time loop, adjoint).
#pragma once
#include "../../include/ssg_b200.h"
#include "kernels.cuh"

#include <cstring>
#include <functional>
#include <string>
#include <utility>
#include <vector>

// internal header: the context code uses the kernel interface unqualified
using namespace ssg;

struct ssg_ctx {
    ssg_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    Dims d{};
    // tables
    double2* tw = nullptr;
    float2* tw32 = nullptr;
    double* kxc = nullptr;
    double* kyc = nullptr;
    double* sigma = nullptr;
    ZOps* zops = nullptr;
    double* tinv = nullptr;          // pivot reciprocals of the vertical solve [nz-2][pivot_plane]
    // state
    double2* Phat = nullptr;    // nz compact planes
    double2* hist[3] = {};      // earlier solutions, newest first (predictor history)
    double2* ring_base[4] = {}; // the four buffers of Phat and hist in allocation order
    int nhist = 0;              // solutions held in Phat and hist
    double2* bh = nullptr;      // compact surface buoyancy
    double2* bstage = nullptr;  // RK3 stage start
    double2* fold = nullptr;    // AB2 history / RK3 k1
    // Monge-Ampere workspace
    double2 *A = nullptr, *B = nullptr, *C = nullptr, *Dt = nullptr, *Dh = nullptr;
    double* partials = nullptr;
    unsigned int* ticket = nullptr;
    double* norms = nullptr;
    unsigned int* nonfinite = nullptr;
    double* h_norms = nullptr;       // pinned
    unsigned int* h_flag = nullptr;  // pinned
    unsigned int* errflag = nullptr; // device: kernel-side wait timeouts
    unsigned int* h_err = nullptr;   // pinned
    MixedTmaps ytm{};                // TMA descriptors of A, B, C, Dt (FP64 y-pass)
    bool use_tma = false;
    MixedTmaps ytm32{};              // the same arrays viewed as FP32 (mixed y-pass)
    bool use_tma32 = false;
    MixedTmaps ytm32w{};             // 16-column FP32 tiles (warp-transform y-pass, N = 1024)
    bool use_warp32 = false;
    bool use_xwarp32 = false;        // FP32 row passes with one warp per row (N = 1024)
    bool thomas_staged = false;      // shared-memory staged vertical solve at every depth
    float2* tww32 = nullptr;         // W1024^(n1 k1) at [k1][n1], FP32
    int num_sms = 148;
    // surface workspace
    double2 *P1 = nullptr, *P2 = nullptr, *P3 = nullptr, *Q1 = nullptr, *Q2 = nullptr;
    // staging for field I/O
    double* phys = nullptr;
    double2* mixed = nullptr;
    // clock
    double t = 0.0;
    int64_t step = 0;
    int last_ma_iterations = 0;
    // diagnostics
    std::string err;
    double last_ms = 0.0;
    int64_t last_launches = 0;
    std::vector<void*> allocations;
    // per-class kernel timing
    bool profiling = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
    double kc_ms[KC_COUNT] = {0};
    int64_t kc_n[KC_COUNT] = {0};

    // discrete adjoint: checkpoints, tape and workspace (ssg_adjoint.cu)
    struct AdjointState* adj = nullptr;
    // CUDA graphs of whole steps (ssg_step): the device copy of the step
    // counter, the device state of the iteration loop, a stream on which the
    // while-node bodies are captured, and the instantiated graphs
    int64_t* step_dev = nullptr;
    SolveDev* sdev = nullptr;    // one per member
    SolveDev* h_sdev = nullptr;  // pinned, one per member
    // members > 1: the members whose solve goes on, and the device's answer
    // to "does any go on" for the host loop of a solve
    unsigned int* active = nullptr;
    unsigned int* going = nullptr;
    unsigned int* h_going = nullptr;  // pinned
    cudaStream_t side = nullptr;
    bool capturing = false;
    bool graphs = true;
    std::vector<struct GraphEntry> graph_cache;

    Tables tables() const { return Tables{tw, tw32, kxc, kyc, sigma}; }
};

// frees the adjoint's device memory (context destruction)
void adjoint_release(ssg_ctx* ctx);



// record an error message on the context (or the global slot when ctx is null)
int fail(ssg_ctx* c, int code, const std::string& msg);
cudaEvent_t pool_event(ssg_ctx* ctx);
// accumulate the pending per-kernel event pairs (after a stream sync)
void drain_profile(ssg_ctx* ctx);

#define CU(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? SSG_ERR_OOM : SSG_ERR_CUDA,      \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                  \
    } while (0)

// Launch with optional per-class event bracketing.
#define KLC(cls, call)                                                              \
    do {                                                                            \
        cudaEvent_t e0_ = nullptr, e1_ = nullptr;                                   \
        if (ctx->profiling) {                                                       \
            e0_ = pool_event(ctx);                                                  \
            e1_ = pool_event(ctx);                                                  \
            cudaEventRecord(e0_, ctx->stream);                                      \
        }                                                                           \
        int r_ = (call);                                                            \
        if (ctx->profiling) {                                                       \
            cudaEventRecord(e1_, ctx->stream);                                      \
            ctx->ev_pending.push_back({(cls), {e0_, e1_}});                         \
        }                                                                           \
        if (r_ == -6) return fail(ctx, SSG_ERR_UNSUPPORTED, "grid size not supported"); \
        if (r_ != 0) return fail(ctx, SSG_ERR_CUDA, std::string("kernel launch: ") + #call + ": " + cudaGetErrorString(cudaGetLastError())); \
    } while (0)
#define KL(call) KLC(KC_IO, call)

template <typename T>
inline int dalloc(ssg_ctx* ctx, T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 256);
    if (e != cudaSuccess) return fail(ctx, SSG_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    ctx->allocations.push_back(q);
    *p = static_cast<T*>(q);
    return SSG_OK;
}

// physical (nx*ny) host array -> compact spectrum (zero_mean: set_b!'s
// projection, else the plain restriction to the kept modes)
int upload_surface(ssg_ctx* ctx, const double* host, double2* dst, int zero_mean);
// compact planes -> physical host array (mult as launch_x_inv_compact); synchronises
int download_planes(ssg_ctx* ctx, const double2* src, int nplanes, int mult, double* host);

// Monge-Ampere solve for the current b_hat (predictor, fixed-point iterations);
// while the context's stream is being captured the iterations become a
// conditional while node with the stop rule on the device
int ma_solve(ssg_ctx* ctx, ssg_ma_stats* st);
// set the clock (host value and the device step counter)
int set_clock(ssg_ctx* ctx, double t, int64_t step);
// forget the predictor history and give Phat and hist their allocation order
// back (so that identical runs capture and replay identical graphs)
void reset_ring(ssg_ctx* ctx);
// one surface-tendency stage with its time-stage epilogue
int tendency_stage(ssg_ctx* ctx, int mode, int filter, double dt);

struct SolveAcc {
    int solves = 0, iters = 0, itmax = 0, unconv = 0;
    double updmax = 0.0;
};
int solve_counted(ssg_ctx* ctx, SolveAcc& acc);

// Per-step record for the adjoint: the buoyancy entering each tendency stage
// and the potential solved from it (one stage for AB2, three for RK3).
struct StepTape {
    double2* b[3];
    double2* phi[3];
};
// one time step (timestep! followed by the solve for the new buoyancy); when
// tape is non-null the stage inputs are copied into it
int advance_step(ssg_ctx* ctx, double h, SolveAcc& acc, const StepTape* tape);

// An instantiated graph of captured work, cached under a key that holds
// everything the capture baked in (buffer pointers, step length, counts), with
// the host-side state the captured work leaves behind (post).
struct GraphEntry {
    std::vector<uint64_t> key, post;
    cudaGraphExec_t exec = nullptr;
};
GraphEntry* find_graph(ssg_ctx* ctx, const std::vector<uint64_t>& key);
// destroy every cached graph (before a buffer that graphs bake in is freed)
void release_graphs(ssg_ctx* ctx);
// capture fn (work launched on ctx->stream, iteration loops as while nodes)
// into a new entry under key; the caller saves and restores the host state fn
// advances and fills entry->post
int add_graph(ssg_ctx* ctx, const std::vector<uint64_t>& key, const std::function<int()>& fn, GraphEntry** out);
// solve statistics of graph work accumulate in ctx->sdev: reset, and merge into acc (synchronises)
int reset_device_stats(ssg_ctx* ctx);
int merge_device_stats(ssg_ctx* ctx, SolveAcc& acc);
// n steps of length h, as cached graphs of whole steps where the predictor
// history allows it, else step by step (ssg_step's loop)
int run_steps(ssg_ctx* ctx, double h, int n, SolveAcc& acc);
uint64_t bits_of(double x);
