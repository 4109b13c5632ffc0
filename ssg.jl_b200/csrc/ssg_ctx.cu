// ssg_ctx.cu -- context, time loop and the C ABI of libssg_b200.so.
//
// A context is one SemiGeostrophicProblem on one GPU (src/timestep.jl:348-399
// in SSG.jl): the device tables of Domain, the device fields of Fields, the
// TimeState clock, and the drivers timestep!/set_b!/solve_monge_ampere_fields!.
//
// State is kept spectral and compact (only the modes the 2/3 mask keeps): the
// surface buoyancy b_hat, the AB2 history / RK3 stage buffers, and the 3-D
// potential Phi_hat on all nz planes.  Physical fields are produced only when a
// caller asks for them.  In exact arithmetic this is the reference's state: its
// buoyancy stays inside the mask (the initial field is dealiased, every
// tendency is dealiased, the filter is diagonal), and its potential is
// dealiased by the solver.
#include "ctx.h"
#include "fft.cuh"
#include "fft_warp.cuh"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <initializer_list>
#include <vector>

using namespace ssg;

static thread_local std::string g_create_error;

// interior planes of the Monge-Ampere workspace over all members
static int ma_planes(const Dims& d) { return (d.nz - 2) * d.members; }

void ssg::set_global_error(const char* msg) { g_create_error = msg ? msg : ""; }

int fail(ssg_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg; else g_create_error = msg;
    return code;
}

cudaEvent_t pool_event(ssg_ctx* ctx) {
    if (!ctx->ev_pool.empty()) {
        cudaEvent_t e = ctx->ev_pool.back();
        ctx->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Accumulate the pending per-kernel event pairs (after a stream sync).
void drain_profile(ssg_ctx* ctx) {
    for (auto& pe : ctx->ev_pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, pe.second.first, pe.second.second) == cudaSuccess) {
            ctx->kc_ms[pe.first] += ms;
            ctx->kc_n[pe.first] += 1;
        }
        ctx->ev_pool.push_back(pe.second.first);
        ctx->ev_pool.push_back(pe.second.second);
    }
    ctx->ev_pending.clear();
}

extern "C" int ssg_abi_version(void) { return SSG_ABI_VERSION; }

extern "C" void ssg_config_init(ssg_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->abi_version = SSG_ABI_VERSION;
    c->lx = 2.0 * M_PI;
    c->ly = 2.0 * M_PI;
    c->lz = 1.0;
    c->eps = 0.01;
    c->dt = 1e-3;
    c->scheme = SSG_SCHEME_AB2;
    c->filter_freq = 10;
    c->filter_order = 4;
    c->ma_maxiter = 50;
    c->filter_strength = 0.1;
    c->filter_cutoff = 0.65;
    c->ma_tol = 1e-10;
    c->ma_per_stage = 1;
    c->ma_rhs_mode = SSG_MA_RHS_SURFACE;
    c->precision = 0;
    c->ma_predictor = 3;
    c->ma_bc_guess = 1;
}

static int validate(const ssg_config* c, std::string& why) {
    if (c->abi_version != SSG_ABI_VERSION) { why = "abi_version mismatch"; return SSG_ERR_ARG; }
    if (c->nx != c->ny) { why = "nx != ny is not supported"; return SSG_ERR_UNSUPPORTED; }
    const int n = c->nx;
    if (n < 32 || n > 1024 || (n & (n - 1))) { why = "nx must be a power of two in [32, 1024]"; return SSG_ERR_UNSUPPORTED; }
    if (c->nz < 4 || c->nz > 64) { why = "nz must be in [4, 64]"; return SSG_ERR_UNSUPPORTED; }
    if (!(c->lx > 0 && c->ly > 0 && c->lz > 0)) { why = "domain lengths must be positive"; return SSG_ERR_ARG; }
    if (c->scheme != SSG_SCHEME_AB2 && c->scheme != SSG_SCHEME_RK3) { why = "unknown scheme"; return SSG_ERR_ARG; }
    if (c->filter_freq < 0 || c->filter_order < 1) { why = "bad filter parameters"; return SSG_ERR_ARG; }
    if (c->filter_freq > 0 && !(c->filter_cutoff > 0 && c->filter_cutoff <= 1)) { why = "filter_cutoff must be in (0, 1]"; return SSG_ERR_ARG; }
    if (c->ma_maxiter < 1) { why = "ma_maxiter must be >= 1"; return SSG_ERR_ARG; }
    if (c->ma_rhs_mode != SSG_MA_RHS_SURFACE && c->ma_rhs_mode != SSG_MA_RHS_VOLUME) { why = "bad ma_rhs_mode"; return SSG_ERR_ARG; }
    if (c->precision != 0 && c->precision != 1) { why = "precision must be 0 (FP64) or 1 (mixed)"; return SSG_ERR_ARG; }
    if (c->ma_predictor < 0 || c->ma_predictor > 3) { why = "bad ma_predictor"; return SSG_ERR_ARG; }
    if (c->filter_type < SSG_FILTER_EXPONENTIAL || c->filter_type > SSG_FILTER_CUSTOM) { why = "bad filter_type"; return SSG_ERR_ARG; }
    if (c->ab2_literal_alias != 0 && c->ab2_literal_alias != 1) { why = "ab2_literal_alias must be 0 or 1"; return SSG_ERR_ARG; }
    if (c->ma_bc_guess != 0 && c->ma_bc_guess != 1) { why = "ma_bc_guess must be 0 or 1"; return SSG_ERR_ARG; }
    if (c->nmembers < 0 || c->nmembers > 1024) { why = "nmembers must be in [0, 1024]"; return SSG_ERR_ARG; }
    if (c->nmembers > 1 && c->ma_rhs_mode != SSG_MA_RHS_SURFACE) {
        why = "ensemble members (nmembers > 1) need the surface right-hand side";
        return SSG_ERR_UNSUPPORTED;
    }
    return SSG_OK;
}

// Transfer functions of src/filter.jl:119-169 (exponential, hyperviscosity,
// sharp cutoff, Cesaro), evaluated on the host for the sigma table.
static double transfer(int type, double knorm, double kmag, double strength, int order, double cutoff, double dt) {
    switch (type) {
        case SSG_FILTER_HYPERVISCOSITY: {
            double p = 1.0;
            for (int q = 0; q < 2 * order; ++q) p *= kmag;
            return std::exp(-strength * p * dt);
        }
        case SSG_FILTER_CUTOFF: return knorm <= cutoff ? 1.0 : 0.0;
        case SSG_FILTER_CESARO: {
            if (knorm <= cutoff) return 1.0;
            if (knorm >= 1.0) return 0.0;
            const double ratio = (knorm - cutoff) / (1.0 - cutoff);
            double p = 1.0;
            for (int q = 0; q < order; ++q) p *= (1.0 - ratio);
            return p;
        }
        default: {
            if (knorm <= cutoff) return 1.0;
            const double ratio = (knorm - cutoff) / (1.0 - cutoff);
            double p = 1.0;
            for (int q = 0; q < order; ++q) p *= ratio;
            return std::exp(-strength * p);
        }
    }
}

// The vertical operator for the spacing vector dz (length nz, as Domain.dz):
// d2dz2! rows of the interior planes (src/transforms.jl:812-818) and the
// one-sided Neumann rows (src/poisson.jl:309-364), with the reference's indexing
// of dz (plane k uses dz[k-1] and dz[k]; the top row dz[nz-2] and dz[nz-3]; the
// bottom row dz[0] and dz[1]).
static ZOps vertical_ops(const std::vector<double>& dz) {
    const int nz = (int)dz.size();
    ZOps z{};
    for (int k = 1; k < nz - 1; ++k) {
        const double dzm = dz[k - 1], dzp = dz[k];
        z.al[k] = 2.0 / (dzm * (dzm + dzp));
        z.be[k] = -2.0 / (dzm * dzp);
        z.ga[k] = 2.0 / (dzp * (dzm + dzp));
    }
    {
        const double h1 = dz[0], h2 = dz[1], a = h1 + h2;
        z.ab = -(2 * h1 + h2) / (h1 * a);
        z.bb = a / (h1 * h2);
        z.cb = -h1 / (h2 * a);
    }
    {
        const int k = nz - 1;
        const double h1 = dz[k - 1], h2 = dz[k - 2], a = h1 + h2;
        z.at = (2 * h1 + h2) / (h1 * a);
        z.bt = -a / (h1 * h2);
        z.ct = h1 / (h2 * a);
    }
    return z;
}

static int build_tables(ssg_ctx* ctx) {
    const ssg_config& c = ctx->cfg;
    const Dims& d = ctx->d;
    const int N = d.N;
    // twiddles W_N^e in long double, in the FFT's pass order
    std::vector<double2> tw(N, make_double2(1.0, 0.0));
    std::vector<float2> tw32(N, make_float2(1.f, 0.f));
    const long double PI_L = 3.141592653589793238462643383279502884L;
    pass_twiddle_exponents(N, [&](int i, int e) {
        long double a = -2.0L * PI_L * (long double)e / (long double)N;
        tw[i] = make_double2((double)cosl(a), (double)sinl(a));
        tw32[i] = make_float2((float)cosl(a), (float)sinl(a));
    });
    // kx = 2pi .* fftfreq(Nx, 1/dx), ky = 2pi .* rfftfreq(Ny, 1/dy)  (src/domain.jl:143-162)
    const double dx = c.lx / c.nx, dy = c.ly / c.ny;
    const double mulx = (1.0 / dx) / c.nx, muly = (1.0 / dy) / c.ny;
    const int nnx = (c.nx - 1) / 2 + 1;
    std::vector<double> kxfull(N), kyfull(d.nyc);
    for (int i = 0; i < N; ++i) kxfull[i] = 2.0 * M_PI * ((double)(i < nnx ? i : i - N) * mulx);
    for (int j = 0; j < d.nyc; ++j) kyfull[j] = 2.0 * M_PI * ((double)j * muly);
    std::vector<double> kxc(d.Mx), kyc(d.My);
    for (int cc = 0; cc < d.Mx; ++cc) kxc[cc] = kxfull[cc < d.Kp ? cc : cc + (N - 2 * d.Kp)];
    for (int j = 0; j < d.My; ++j) kyc[j] = kyfull[j];
    // exponential filter transfer per compact mode (src/filter.jl:283-309)
    const double kmx = M_PI / dx, kmy = M_PI / dy;
    const double kmax = std::sqrt(kmx * kmx + kmy * kmy);
    std::vector<double> sig(d.c2());
    for (int j = 0; j < d.My; ++j)
        for (int cc = 0; cc < d.Mx; ++cc) {
            const double kmag = std::sqrt(kxc[cc] * kxc[cc] + kyc[j] * kyc[j]);
            sig[cc + (size_t)d.Mx * j] =
                transfer(c.filter_type, kmag / kmax, kmag, c.filter_strength, c.filter_order, c.filter_cutoff, c.dt);
        }
    // vertical operator on the uniform non-periodic grid dz = Lz/(Nz-1)
    // (src/domain.jl:245-248); ssg_set_vertical_grid replaces it
    const ZOps z = vertical_ops(std::vector<double>(c.nz, c.lz / (c.nz - 1)));
    int r;
    if ((r = dalloc(ctx, &ctx->tw, N))) return r;
    if ((r = dalloc(ctx, &ctx->tw32, N))) return r;
    if ((r = dalloc(ctx, &ctx->kxc, d.Mx))) return r;
    if ((r = dalloc(ctx, &ctx->kyc, d.My))) return r;
    if ((r = dalloc(ctx, &ctx->sigma, d.c2()))) return r;
    if ((r = dalloc(ctx, &ctx->zops, 1))) return r;
    CU(cudaMemcpy(ctx->tw, tw.data(), N * sizeof(double2), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(ctx->tw32, tw32.data(), N * sizeof(float2), cudaMemcpyHostToDevice));
    if (N == 1024) {
        std::vector<float2> tww(1024);
        warp_twiddle_exponents([&](int i, int e) {
            long double a = -2.0L * PI_L * (long double)e / (long double)N;
            tww[i] = make_float2((float)cosl(a), (float)sinl(a));
        });
        if ((r = dalloc(ctx, &ctx->tww32, 1024))) return r;
        CU(cudaMemcpy(ctx->tww32, tww.data(), 1024 * sizeof(float2), cudaMemcpyHostToDevice));
    }
    CU(cudaMemcpy(ctx->kxc, kxc.data(), d.Mx * sizeof(double), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(ctx->kyc, kyc.data(), d.My * sizeof(double), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(ctx->sigma, sig.data(), d.c2() * sizeof(double), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(ctx->zops, &z, sizeof(ZOps), cudaMemcpyHostToDevice));
    return SSG_OK;
}

static void release(ssg_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drain_profile(ctx);
    adjoint_release(ctx);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    ctx->ev_pool.clear();
    for (void* p : ctx->allocations) cudaFree(p);
    ctx->allocations.clear();
    if (ctx->h_norms) cudaFreeHost(ctx->h_norms);
    if (ctx->h_flag) cudaFreeHost(ctx->h_flag);
    if (ctx->h_err) cudaFreeHost(ctx->h_err);
    if (ctx->h_sdev) cudaFreeHost(ctx->h_sdev);
    if (ctx->h_going) cudaFreeHost(ctx->h_going);
    release_graphs(ctx);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
}

extern "C" int ssg_ctx_create(const ssg_config* cfg, int device, ssg_ctx** out) {
    if (!cfg || !out) return fail(nullptr, SSG_ERR_ARG, "null argument");
    *out = nullptr;
    std::string why;
    int v = validate(cfg, why);
    if (v != SSG_OK) return fail(nullptr, v, why);
    ssg_ctx* ctx = new ssg_ctx();
    ctx->cfg = *cfg;
    ctx->device = device;
    Dims& d = ctx->d;
    d.N = cfg->nx;
    d.nyc = d.N / 2 + 1;
    d.Kp = d.N / 3;
    d.Mx = 2 * d.Kp;
    d.My = (2 * d.nyc) / 3;
    d.nz = cfg->nz;
    d.members = cfg->nmembers > 1 ? cfg->nmembers : 1;
    auto bail = [&](int code) {
        std::string msg = ctx->err;
        release(ctx);
        delete ctx;
        g_create_error = msg;
        return code;
    };
    int r;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { ctx->err = std::string("cudaSetDevice: ") + cudaGetErrorString(e); return bail(SSG_ERR_CUDA); }
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { ctx->err = std::string("cudaStreamCreate: ") + cudaGetErrorString(e); return bail(SSG_ERR_CUDA); }
    if (cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
        ctx->err = "cudaEventCreate failed";
        return bail(SSG_ERR_CUDA);
    }
    if ((r = build_tables(ctx))) return bail(r);
    if ((r = dalloc(ctx, &ctx->tinv, (size_t)(d.nz - 2) * pivot_plane(d.Mx, d.My)))) return bail(r);
    // the tables went up by cudaMemcpy on the legacy stream; the factorisation
    // runs on this context's non-blocking stream
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { ctx->err = std::string("init: ") + cudaGetErrorString(e); return bail(SSG_ERR_CUDA); }
    if (launch_ma_thomas_factor(d, ctx->tables(), ctx->zops, ctx->tinv, ctx->stream)) {
        ctx->err = "vertical solve factorisation failed";
        return bail(SSG_ERR_CUDA);
    }
    // every member's state and workspace one after another (members = 1: the
    // one problem)
    const size_t nm = (size_t)d.members;
    const size_t c2 = d.c2() * nm, m2 = d.m2() * nm, nzi = (size_t)d.nz - 2;
    if ((r = dalloc(ctx, &ctx->Phat, c2 * d.nz))) return bail(r);
    for (int i = 0; i < 3; ++i)
        if ((r = dalloc(ctx, &ctx->hist[i], c2 * d.nz))) return bail(r);
    ctx->ring_base[0] = ctx->Phat;
    for (int i = 0; i < 3; ++i) ctx->ring_base[1 + i] = ctx->hist[i];
    if ((r = dalloc(ctx, &ctx->bh, c2))) return bail(r);
    if ((r = dalloc(ctx, &ctx->bstage, c2))) return bail(r);
    if ((r = dalloc(ctx, &ctx->fold, c2))) return bail(r);
    if ((r = dalloc(ctx, &ctx->A, m2 * nzi))) return bail(r);
    if ((r = dalloc(ctx, &ctx->B, m2 * nzi))) return bail(r);
    if ((r = dalloc(ctx, &ctx->C, m2 * nzi))) return bail(r);
    if ((r = dalloc(ctx, &ctx->Dt, m2 * nzi))) return bail(r);
    if ((r = dalloc(ctx, &ctx->Dh, c2 * nzi))) return bail(r);
    const size_t nblk = (d.c2() + 31) / 32 + 1;   // blocks of 32 or more threads per member
    if ((r = dalloc(ctx, &ctx->partials, 2 * nblk * nm))) return bail(r);
    if ((r = dalloc(ctx, &ctx->ticket, nm))) return bail(r);
    if ((r = dalloc(ctx, &ctx->norms, 2 * nm))) return bail(r);
    if ((r = dalloc(ctx, &ctx->nonfinite, 1))) return bail(r);
    if ((r = dalloc(ctx, &ctx->errflag, 1))) return bail(r);
    if ((r = dalloc(ctx, &ctx->step_dev, 1))) return bail(r);
    if ((r = dalloc(ctx, &ctx->sdev, nm))) return bail(r);
    if (nm > 1) {
        if ((r = dalloc(ctx, &ctx->active, nm))) return bail(r);
        if ((r = dalloc(ctx, &ctx->going, 1))) return bail(r);
    }
    if ((r = dalloc(ctx, &ctx->P1, m2))) return bail(r);
    if ((r = dalloc(ctx, &ctx->P2, m2))) return bail(r);
    if ((r = dalloc(ctx, &ctx->P3, m2))) return bail(r);
    if ((r = dalloc(ctx, &ctx->Q1, m2))) return bail(r);
    if ((r = dalloc(ctx, &ctx->Q2, m2))) return bail(r);
    // field I/O stages one member at a time
    if ((r = dalloc(ctx, &ctx->phys, d.r2() * d.nz))) return bail(r);
    if ((r = dalloc(ctx, &ctx->mixed, d.m2() * d.nz))) return bail(r);
    if (cudaMallocHost(&ctx->h_norms, 2 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_flag, sizeof(unsigned int)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_err, sizeof(unsigned int)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_going, sizeof(unsigned int)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_sdev, nm * sizeof(SolveDev)) != cudaSuccess) {
        ctx->err = "cudaMallocHost failed";
        return bail(SSG_ERR_OOM);
    }
    // zero state (allocate_fields leaves memory undefined; the solver starts from zeros)
    cudaMemsetAsync(ctx->Phat, 0, c2 * d.nz * sizeof(double2), ctx->stream);
    cudaMemsetAsync(ctx->bh, 0, c2 * sizeof(double2), ctx->stream);
    cudaMemsetAsync(ctx->bstage, 0, c2 * sizeof(double2), ctx->stream);
    cudaMemsetAsync(ctx->fold, 0, c2 * sizeof(double2), ctx->stream);
    cudaMemsetAsync(ctx->ticket, 0, nm * sizeof(unsigned int), ctx->stream);
    cudaMemsetAsync(ctx->nonfinite, 0, sizeof(unsigned int), ctx->stream);
    cudaMemsetAsync(ctx->errflag, 0, sizeof(unsigned int), ctx->stream);
    cudaMemsetAsync(ctx->step_dev, 0, sizeof(int64_t), ctx->stream);
    cudaMemsetAsync(ctx->sdev, 0, nm * sizeof(SolveDev), ctx->stream);
    if (cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess) {
        ctx->err = "cudaStreamCreate failed";
        return bail(SSG_ERR_CUDA);
    }
    {
        const char* g = getenv("SSG_B200_GRAPHS");
        ctx->graphs = !(g && g[0] == '0');
    }
    {
        const char* ts = getenv("SSG_B200_THOMAS_STAGED");
        ctx->thomas_staged = ts && ts[0] == '1';
    }
    // FP64 y-pass: the persistent TMA-pipelined kernel for N >= 512, where it
    // was measured faster than the plain-load one (0.0495 against 0.068 ms at
    // 512^2 x 16, 0.527 against 0.577 ms at 1024^2 x 32).  SSG_B200_TMA=0 or 1
    // forces either kernel.
    {
        const char* tma = getenv("SSG_B200_TMA");
        const bool want = tma ? tma[0] == '1' : d.N >= 512;
        ctx->use_tma = want && mixed_tma_supported(d) &&
                       make_mixed_tmaps(d, ctx->A, ctx->B, ctx->C, ctx->Dt, ma_planes(d), &ctx->ytm) == 0;
    }
    // mixed precision: persistent TMA-pipelined y-pass unless SSG_B200_MP_PLAIN=1
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    {
        const char* plain = getenv("SSG_B200_MP_PLAIN");
        ctx->use_tma32 = !(plain && plain[0] == '1') && mixed_tma_supported(d) &&
                         make_mixed32_tmaps(d, reinterpret_cast<float2*>(ctx->A), reinterpret_cast<float2*>(ctx->B),
                                            reinterpret_cast<float2*>(ctx->C), reinterpret_cast<float2*>(ctx->Dt),
                                            ma_planes(d), &ctx->ytm32) == 0;
    }
    // N = 1024: the y-pass with one warp per transform (SSG_B200_MP_WARP=0
    // selects the team-transform kernel instead; SSG_B200_MP_WARP=2, 4 or 8
    // sets the warps per block)
    {
        const char* wv = getenv("SSG_B200_MP_WARP");
        // four warps per block (two blocks per SM): 0.160 ms against 0.172 (eight)
        // and 0.165 (two) at 1024^2 x 32
        int warps = 4;
        if (wv && (wv[0] == '2' || wv[0] == '4' || wv[0] == '8')) warps = wv[0] - '0';
        ctx->use_warp32 = ctx->use_tma32 && d.N == 1024 && ctx->tww32 && !(wv && wv[0] == '0') &&
                          make_mixed32w_tmaps(d, reinterpret_cast<float2*>(ctx->A), reinterpret_cast<float2*>(ctx->B),
                                              reinterpret_cast<float2*>(ctx->C), reinterpret_cast<float2*>(ctx->Dt),
                                              ma_planes(d), warps, &ctx->ytm32w) == 0;
    }
    // N = 1024: FP32 row passes with one warp per row when SSG_B200_MP_XWARP=1;
    // the team-transform row passes are the default, measured faster at
    // 1024^2 x 32 (x-inverse 0.112 against 0.132 ms, x-forward 0.041 against
    // 0.046 ms)
    {
        const char* xw = getenv("SSG_B200_MP_XWARP");
        ctx->use_xwarp32 = d.N == 1024 && ctx->tww32 && xw && xw[0] == '1';
    }
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { ctx->err = std::string("init: ") + cudaGetErrorString(e); return bail(SSG_ERR_CUDA); }
    *out = ctx;
    return SSG_OK;
}

extern "C" int ssg_ctx_destroy(ssg_ctx* ctx) {
    if (!ctx) return SSG_OK;
    release(ctx);
    delete ctx;
    return SSG_OK;
}

// ---------------------------------------------------------------------------
// Monge-Ampere solve (documented problem of src/poisson.jl:1-12, fixed-point
// iteration with the exact per-mode linear inverse; see spectral_kernels.cu)
// ---------------------------------------------------------------------------
// relative update at which a mixed-precision solve has converged: 12 FP32
// ulps.  Measured on 1024^2 x 32, AB2, steps 100-1000 (iterations per step,
// relative b_s error against the FP64 path after 1000 steps): 4 ulps 2.00 and
// 2.8e-8, 8 ulps 1.63 and 8.9e-8, 12 ulps 1.41 and 2.6e-7, 16 ulps 1.23 and
// 5.0e-7, 64 ulps 1.23 and 2.5e-6; 12 keeps the error a factor ~4 under 1e-6.
static const double kMixedUpdateFloor = 12.0 / 16777216.0;

// One fixed-point iteration of the Monge-Ampere solve on stream s: the three
// transform passes (FP64 or FP32) and the per-mode vertical solve, which
// leaves the update norms in ctx->norms.
static int ma_iteration(ssg_ctx* ctx, cudaStream_t s) {
    const Dims& d = ctx->d;
    const Tables tb = ctx->tables();
    const bool surface = ctx->cfg.ma_rhs_mode == SSG_MA_RHS_SURFACE;
    // Mixed precision, surface right-hand side, register-form vertical solve:
    // the x-forward pass stores its FP32 transform (in Dh's memory) and the
    // solve forms eps times it in FP64 as it loads it -- the same values, half
    // the bytes written and read between the two
    const bool rhs32 = ctx->cfg.precision == 1 && surface && !ctx->use_xwarp32 && !ctx->thomas_staged &&
                       thomas_reg_depth(d.nz);
    float2* Dh32 = reinterpret_cast<float2*>(ctx->Dh);
    if (ctx->cfg.precision == 1) {
        float2* A32 = reinterpret_cast<float2*>(ctx->A);
        float2* B32 = reinterpret_cast<float2*>(ctx->B);
        float2* C32 = reinterpret_cast<float2*>(ctx->C);
        float2* D32 = reinterpret_cast<float2*>(ctx->Dt);
        if (ctx->use_xwarp32)
            KLC(KC_MA_XINV, launch_ma_xinv3_mp_warp(d, tb, ctx->tww32, ctx->Phat, A32, B32, C32, s));
        else
            KLC(KC_MA_XINV, launch_ma_xinv3_mp(d, tb, ctx->Phat, A32, B32, C32, s));
        if (ctx->use_tma32)
            KLC(KC_MA_Y, ctx->use_warp32
                             ? launch_ma_y_mp_warp(d, tb, ctx->tww32, ctx->ytm32w, ctx->num_sms, ctx->errflag, s)
                             : launch_ma_y_mp_tma(d, tb, ctx->ytm32, ctx->num_sms, ctx->errflag, s));
        else
            KLC(KC_MA_Y, launch_ma_y_mp(d, tb, A32, B32, C32, D32, s));
        if (ctx->use_xwarp32)
            KLC(KC_MA_XFWD, launch_ma_xfwd_mp_warp(d, tb, ctx->tww32, D32, ctx->Dh, ctx->cfg.eps,
                                                   surface ? nullptr : ctx->bh, s));
        else
            KLC(KC_MA_XFWD, launch_ma_xfwd_mp(d, tb, D32, ctx->Dh, ctx->cfg.eps, surface ? nullptr : ctx->bh,
                                              rhs32 ? Dh32 : nullptr, s));
    } else {
        KLC(KC_MA_XINV, launch_ma_xinv3(d, tb, ctx->Phat, ctx->A, ctx->B, ctx->C, s));
        if (ctx->use_tma)
            KLC(KC_MA_Y, launch_ma_y_tma(d, tb, ctx->ytm, ctx->num_sms, ctx->errflag, s));
        else
            KLC(KC_MA_Y, launch_ma_y(d, tb, ctx->A, ctx->B, ctx->C, ctx->Dt, s));
        KLC(KC_MA_XFWD, launch_ma_xfwd(d, tb, ctx->Dt, ctx->Dh, ctx->cfg.eps, surface ? nullptr : ctx->bh, s));
    }
    KLC(KC_MA_THOMAS, launch_ma_thomas(d, ctx->zops, ctx->tinv, ctx->Dh, rhs32 ? Dh32 : nullptr, ctx->cfg.eps,
                                       surface ? ctx->bh : nullptr, ctx->Phat, ctx->partials, ctx->ticket, ctx->norms,
                                       ctx->thomas_staged, ctx->active, s));
    return SSG_OK;
}

int ma_solve(ssg_ctx* ctx, ssg_ma_stats* st) {
    const Dims& d = ctx->d;
    // initial guess: the polynomial extrapolation of order ma_predictor
    // (1 linear, 2 quadratic, 3 cubic) through the last solutions; solves come
    // at equally spaced times: every step for AB2, every stage of dt/3 for RK3.
    // History ring S[0] = Phat (newest), S[1..3] = hist; the guess is written
    // into the slot after the newest kept solution (the oldest once the ring is
    // full) and rotated to the front, where the solve refines it in place.
    const int pred = ctx->cfg.ma_predictor;
    if (pred >= 1) {
        const size_t n = d.c2() * d.nz * d.members;
        double2** S[4] = {&ctx->Phat, &ctx->hist[0], &ctx->hist[1], &ctx->hist[2]};
        const int cap = pred + 1, h = ctx->nhist;
        if (h >= 1) {
            const int t = h < cap ? h : cap - 1;
            const int order = pred < h - 1 ? pred : h - 1;
            if (ctx->cfg.ma_bc_guess)
                KL(launch_predict_bc(d, *S[0], *S[1], *S[2], *S[3], *S[t], order,
                                     ctx->cfg.ma_rhs_mode == SSG_MA_RHS_SURFACE ? ctx->bh : nullptr, ctx->tinv,
                                     ctx->zops, ctx->stream));
            else
                KL(launch_predict(*S[0], *S[1], *S[2], *S[3], *S[t], order, n, ctx->stream));
            double2* g = *S[t];
            for (int i = t; i > 0; --i) *S[i] = *S[i - 1];
            *S[0] = g;
        }
        ctx->nhist = h < cap ? h + 1 : cap;
    }
    const bool mixed = ctx->cfg.precision == 1;
    if (ctx->capturing) {
        // device-side loop: a conditional while node whose body is one
        // iteration followed by the stop rule (solve_check_kernel)
        KL(launch_solve_begin(ctx->sdev, ctx->active, d.members, ctx->stream));
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
        cudaGraph_t body = np.conditional.phGraph_out[0];
        CU(cudaStreamBeginCaptureToGraph(ctx->side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        int r = ma_iteration(ctx, ctx->side);
        if (!r)
            r = launch_solve_check(ctx->sdev, ctx->norms, ctx->active, d.members, ctx->cfg.ma_tol,
                                   ctx->cfg.ma_maxiter, mixed ? 1 : 0, kMixedUpdateFloor, (unsigned long long)hdl,
                                   nullptr, ctx->side) == 0
                    ? SSG_OK
                    : fail(ctx, SSG_ERR_CUDA, "solve_check launch failed");
        cudaGraph_t captured = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->side, &captured);
        if (r) return r;
        if (e != cudaSuccess) return fail(ctx, SSG_ERR_CUDA, std::string("capture of an iteration: ") + cudaGetErrorString(e));
        CU(cudaStreamUpdateCaptureDependencies(ctx->stream, &node, 1, cudaStreamSetCaptureDependencies));
        if (st) { st->iterations = 0; st->converged = 1; st->update = 0.0; }
        return SSG_OK;
    }
    if (d.members > 1) {
        // every member's stop rule on the device (solve_check_kernel); the
        // host reads whether any member goes on after each iteration
        KL(launch_solve_begin(ctx->sdev, ctx->active, d.members, ctx->stream));
        int it = 0;
        for (it = 1; it <= ctx->cfg.ma_maxiter; ++it) {
            int r = ma_iteration(ctx, ctx->stream);
            if (r) return r;
            KL(launch_solve_check(ctx->sdev, ctx->norms, ctx->active, d.members, ctx->cfg.ma_tol,
                                  ctx->cfg.ma_maxiter, mixed ? 1 : 0, kMixedUpdateFloor, 0, ctx->going, ctx->stream));
            CU(cudaMemcpyAsync(ctx->h_going, ctx->going, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
            CU(cudaMemcpyAsync(ctx->h_err, ctx->errflag, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
            CU(cudaStreamSynchronize(ctx->stream));
            if (ctx->profiling) drain_profile(ctx);
            if (*ctx->h_err) return fail(ctx, SSG_ERR_CUDA, "a kernel's bounded wait for a TMA tile timed out");
            if (!*ctx->h_going) break;
        }
        CU(cudaMemcpyAsync(ctx->h_sdev, ctx->sdev, d.members * sizeof(SolveDev), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        // the solve's outcome over the members: the most iterations, the
        // largest final update, converged when every member converged
        bool conv = true, nonfinite = false;
        double upd = 0.0;
        int itmax = 0;
        for (int m = 0; m < d.members; ++m) {
            const SolveDev& sd = ctx->h_sdev[m];
            itmax = sd.last_it > itmax ? sd.last_it : itmax;
            upd = sd.upd > upd ? sd.upd : upd;
            conv = conv && sd.last_conv;
            nonfinite = nonfinite || (sd.flags & 1u);
        }
        ctx->last_ma_iterations = itmax;
        if (st) { st->iterations = itmax; st->converged = conv ? 1 : 0; st->update = upd; }
        if (nonfinite) return fail(ctx, SSG_ERR_NONFINITE, "Monge-Ampere iteration produced a non-finite update");
        return conv ? SSG_OK : SSG_ERR_NOT_CONVERGED;
    }
    double upd = 0.0, prev = 0.0;
    int it = 0;
    bool conv = false;
    for (it = 1; it <= ctx->cfg.ma_maxiter; ++it) {
        int r = ma_iteration(ctx, ctx->stream);
        if (r) return r;
        CU(cudaMemcpyAsync(ctx->h_norms, ctx->norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaMemcpyAsync(ctx->h_err, ctx->errflag, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        if (ctx->profiling) drain_profile(ctx);
        if (*ctx->h_err) return fail(ctx, SSG_ERR_CUDA, "a kernel's bounded wait for a TMA tile timed out");
        const double ds = ctx->h_norms[0], ns = ctx->h_norms[1];
        upd = ns > 0 ? std::sqrt(ds / ns) : std::sqrt(ds);
        if (!(upd == upd) || std::isinf(upd)) {
            if (st) { st->iterations = it; st->converged = 0; st->update = upd; }
            return fail(ctx, SSG_ERR_NONFINITE, "Monge-Ampere iteration produced a non-finite update");
        }
        if (upd <= ctx->cfg.ma_tol) { conv = true; break; }
        // FP32 transforms put a floor of a few FP32 ulps under the relative
        // update: the solve has converged once the update is within that floor
        // (12 * 2^-24), or when it stops contracting (counted as converged
        // below 1e-5)
        if (mixed && upd <= kMixedUpdateFloor) { conv = true; break; }
        if (mixed && it > 1 && upd > 0.5 * prev) { conv = upd <= 1e-5; break; }
        prev = upd;
    }
    if (it > ctx->cfg.ma_maxiter) it = ctx->cfg.ma_maxiter;
    ctx->last_ma_iterations = it;
    if (st) { st->iterations = it; st->converged = conv ? 1 : 0; st->update = upd; }
    return conv ? SSG_OK : SSG_ERR_NOT_CONVERGED;
}

int tendency_stage(ssg_ctx* ctx, int mode, int filter, double dt) {
    const Dims& d = ctx->d;
    const Tables tb = ctx->tables();
    const double2* phih = ctx->Phat + d.c2() * (d.nz - 1);
    KLC(KC_SURF_XINV, launch_surf_xinv3(d, tb, phih, ctx->bh, ctx->P1, ctx->P2, ctx->P3, ctx->stream));
    KLC(KC_SURF_Y, launch_surf_y(d, tb, ctx->P1, ctx->P2, ctx->P3, ctx->Q1, ctx->Q2, ctx->stream));
    StageArgs a{};
    a.mode = mode;
    a.filter = filter;
    a.dt = dt;
    a.bh = ctx->bh;
    a.bstage = ctx->bstage;
    a.fold = ctx->fold;
    a.fout = nullptr;
    a.nonfinite = ctx->nonfinite;
    a.step_dev = ctx->step_dev;
    a.filter_freq = ctx->cfg.filter_freq;
    a.ab2_alias = ctx->cfg.ab2_literal_alias;
    KLC(KC_SURF_XFWD, launch_surf_xfwd_stage(d, tb, ctx->Q1, ctx->Q2, a, ctx->stream));
    return SSG_OK;
}

int solve_counted(ssg_ctx* ctx, SolveAcc& acc) {
    ssg_ma_stats s{};
    int r = ma_solve(ctx, &s);
    if (ctx->d.members > 1 && (r == SSG_OK || r == SSG_ERR_NOT_CONVERGED)) {
        // one solve per member (the host copy of the members' last solves)
        for (int m = 0; m < ctx->d.members; ++m) {
            const SolveDev& sd = ctx->h_sdev[m];
            acc.solves += 1;
            acc.iters += sd.last_it;
            acc.itmax = sd.last_it > acc.itmax ? sd.last_it : acc.itmax;
            acc.updmax = sd.upd > acc.updmax ? sd.upd : acc.updmax;
            if (!sd.last_conv) acc.unconv += 1;
        }
        return SSG_OK;
    }
    acc.solves += 1;
    acc.iters += s.iterations;
    acc.itmax = s.iterations > acc.itmax ? s.iterations : acc.itmax;
    acc.updmax = s.update > acc.updmax ? s.update : acc.updmax;
    if (r == SSG_ERR_NOT_CONVERGED) { acc.unconv += 1; return SSG_OK; }
    return r;
}

int advance_step(ssg_ctx* ctx, double h, SolveAcc& acc, const StepTape* tape) {
    const Dims& d = ctx->d;
    const size_t cb = d.c2() * sizeof(double2);
    auto rec = [&](int s) -> int {
        if (!tape) return SSG_OK;
        CU(cudaMemcpyAsync(tape->b[s], ctx->bh, cb, cudaMemcpyDeviceToDevice, ctx->stream));
        CU(cudaMemcpyAsync(tape->phi[s], ctx->Phat, cb * d.nz, cudaMemcpyDeviceToDevice, ctx->stream));
        return SSG_OK;
    };
    const bool per_stage = ctx->cfg.ma_per_stage != 0;
    // the stage kernels read the device step counter: forward Euler at step 0,
    // the filter when (step + 1) % filter_freq == 0 (timestep!, src/timestep.jl:280)
    const int filt = 1;
    int r;
    if ((r = rec(0))) return r;
    if (ctx->cfg.scheme == SSG_SCHEME_AB2) {
        // timestep_ab2_ls! (src/timestep.jl:152-190)
        if ((r = tendency_stage(ctx, STAGE_AB2, filt, h))) return r;
    } else {
        // timestep_rk3! (src/timestep.jl:195-242)
        if ((r = tendency_stage(ctx, STAGE_RK3_1, 0, h))) return r;
        if (per_stage && (r = solve_counted(ctx, acc))) return r;
        if ((r = rec(1))) return r;
        if ((r = tendency_stage(ctx, STAGE_RK3_2, 0, h))) return r;
        if (per_stage && (r = solve_counted(ctx, acc))) return r;
        if ((r = rec(2))) return r;
        if ((r = tendency_stage(ctx, STAGE_RK3_3, filt, h))) return r;
    }
    KL(launch_step_bump(ctx->step_dev, ctx->stream));
    ctx->t += h;
    ctx->step += 1;
    if (per_stage && (r = solve_counted(ctx, acc))) return r;
    return SSG_OK;
}

void reset_ring(ssg_ctx* ctx) {
    ctx->Phat = ctx->ring_base[0];
    for (int i = 0; i < 3; ++i) ctx->hist[i] = ctx->ring_base[1 + i];
    ctx->nhist = 0;
}

int set_clock(ssg_ctx* ctx, double t, int64_t step) {
    ctx->t = t;
    ctx->step = step;
    CU(cudaMemcpyAsync(ctx->step_dev, &ctx->step, sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return SSG_OK;
}

// Steps one graph of whole steps covers: the predictor ring returns to the same
// buffer assignment after cap solves, i.e. after cap / gcd(cap, solves per step)
// steps (1 when nothing rotates).
static int graph_period(const ssg_ctx* ctx) {
    const int spp = ctx->cfg.ma_per_stage ? (ctx->cfg.scheme == SSG_SCHEME_RK3 ? 3 : 1) : 0;
    const int pred = ctx->cfg.ma_predictor;
    if (spp == 0 || pred == 0) return 1;
    const int cap = pred + 1;
    int a = cap, b = spp;
    while (b) { const int t = a % b; a = b; b = t; }
    return cap / a;
}

uint64_t bits_of(double x) {
    uint64_t u;
    std::memcpy(&u, &x, sizeof(u));
    return u;
}

GraphEntry* find_graph(ssg_ctx* ctx, const std::vector<uint64_t>& key) {
    for (auto& g : ctx->graph_cache)
        if (g.key == key) return &g;
    return nullptr;
}

void release_graphs(ssg_ctx* ctx) {
    for (auto& g : ctx->graph_cache) cudaGraphExecDestroy(g.exec);
    ctx->graph_cache.clear();
}

int add_graph(ssg_ctx* ctx, const std::vector<uint64_t>& key, const std::function<int()>& fn, GraphEntry** out) {
    if (ctx->graph_cache.size() >= 32) release_graphs(ctx);
    CU(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
    ctx->capturing = true;
    int r = fn();
    ctx->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(ctx, SSG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    GraphEntry ent;
    ent.key = key;
    e = cudaGraphInstantiate(&ent.exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(ctx, SSG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    ctx->graph_cache.push_back(ent);
    *out = &ctx->graph_cache.back();
    return SSG_OK;
}

int reset_device_stats(ssg_ctx* ctx) {
    CU(cudaMemsetAsync(ctx->sdev, 0, ctx->d.members * sizeof(SolveDev), ctx->stream));
    return SSG_OK;
}

int merge_device_stats(ssg_ctx* ctx, SolveAcc& acc) {
    const int nm = ctx->d.members;
    CU(cudaMemcpyAsync(ctx->h_sdev, ctx->sdev, nm * sizeof(SolveDev), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(ctx->h_err, ctx->errflag, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    unsigned int flags = 0;
    int last = 0;
    bool any = false;
    for (int m = 0; m < nm; ++m) {
        const SolveDev& sd = ctx->h_sdev[m];
        acc.solves += sd.solves;
        acc.iters += sd.iters;
        acc.itmax = sd.itmax > acc.itmax ? sd.itmax : acc.itmax;
        acc.unconv += sd.unconv;
        acc.updmax = sd.updmax > acc.updmax ? sd.updmax : acc.updmax;
        if (sd.solves > 0) any = true, last = sd.last_it > last ? sd.last_it : last;
        flags |= sd.flags;
    }
    if (any) ctx->last_ma_iterations = last;
    if (*ctx->h_err) return fail(ctx, SSG_ERR_CUDA, "a kernel's bounded wait for a TMA tile timed out");
    if (flags & 1u) return fail(ctx, SSG_ERR_NONFINITE, "Monge-Ampere iteration produced a non-finite update");
    return SSG_OK;
}

int run_steps(ssg_ctx* ctx, double h, int n, SolveAcc& acc) {
    int r;
    const int period = graph_period(ctx);
    const int cap = ctx->cfg.ma_predictor >= 1 ? ctx->cfg.ma_predictor + 1 : 1;
    const bool use_graphs = ctx->graphs && !ctx->profiling;
    for (int s = 0; s < n;) {
        const bool warm = ctx->cfg.ma_predictor == 0 || ctx->nhist >= cap || !ctx->cfg.ma_per_stage;
        if (use_graphs && warm) {
            // A graph of L steps: a whole period (after which the predictor
            // ring is back in this assignment), or the steps that remain.
            // Graphs are keyed by the assignment they start from and carry
            // the one they leave, so short calls (one step at a time, as
            // timestep! makes them) replay a graph per phase of the ring.
            const int L = n - s >= period ? period : n - s;
            const std::vector<uint64_t> key = {1, (uint64_t)ctx->Phat, (uint64_t)ctx->hist[0],
                                               (uint64_t)ctx->hist[1], (uint64_t)ctx->hist[2], bits_of(h),
                                               (uint64_t)period, (uint64_t)ctx->nhist, (uint64_t)L};
            GraphEntry* ge = find_graph(ctx, key);
            if (!ge) {
                double2* ring[4] = {ctx->Phat, ctx->hist[0], ctx->hist[1], ctx->hist[2]};
                const double t0 = ctx->t;
                const int64_t s0 = ctx->step;
                const int nh0 = ctx->nhist;
                SolveAcc cap_acc;
                r = add_graph(ctx, key, [&] {
                    int rr = SSG_OK;
                    for (int k = 0; k < L && rr == SSG_OK; ++k) rr = advance_step(ctx, h, cap_acc, nullptr);
                    return rr;
                }, &ge);
                if (!r)
                    ge->post = {(uint64_t)ctx->Phat, (uint64_t)ctx->hist[0], (uint64_t)ctx->hist[1],
                                (uint64_t)ctx->hist[2], (uint64_t)ctx->nhist};
                ctx->Phat = ring[0];
                for (int i = 0; i < 3; ++i) ctx->hist[i] = ring[1 + i];
                ctx->t = t0;
                ctx->step = s0;
                ctx->nhist = nh0;
                if (r) return r;
            }
            CU(cudaGraphLaunch(ge->exec, ctx->stream));
            ctx->Phat = reinterpret_cast<double2*>(ge->post[0]);
            for (int i = 0; i < 3; ++i) ctx->hist[i] = reinterpret_cast<double2*>(ge->post[1 + i]);
            ctx->nhist = (int)ge->post[4];
            for (int k = 0; k < L; ++k) ctx->t += h;
            ctx->step += L;
            s += L;
        } else {
            if ((r = advance_step(ctx, h, acc, nullptr))) return r;
            s += 1;
        }
    }
    return SSG_OK;
}

extern "C" int ssg_step(ssg_ctx* ctx, int32_t nsteps, double dt, ssg_step_stats* stats) {
    if (!ctx) return SSG_ERR_ARG;
    if (nsteps < 0) return fail(ctx, SSG_ERR_ARG, "nsteps < 0");
    CU(cudaSetDevice(ctx->device));
    const double h = dt > 0 ? dt : ctx->cfg.dt;
    const int64_t l0 = launch_counter();
    CU(cudaEventRecord(ctx->ev0, ctx->stream));
    SolveAcc acc;
    int r;
    // Whole steps run as CUDA graphs once the predictor history is full: the
    // iteration loops become conditional while nodes, so no step waits for the
    // host.  The solve statistics of graph steps accumulate on the device.
    if ((r = reset_device_stats(ctx))) return r;
    if ((r = run_steps(ctx, h, nsteps, acc))) return r;
    CU(cudaEventRecord(ctx->ev1, ctx->stream));
    CU(cudaMemcpyAsync(ctx->h_flag, ctx->nonfinite, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    if ((r = merge_device_stats(ctx, acc))) return r;
    if (ctx->profiling) drain_profile(ctx);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_ms = ms;
    ctx->last_launches = launch_counter() - l0;
    if (stats) {
        stats->steps = nsteps;
        stats->ma_solves = acc.solves;
        stats->ma_iterations = acc.iters;
        stats->ma_iterations_max = acc.itmax;
        stats->ma_unconverged = acc.unconv;
        stats->pad0 = 0;
        stats->ma_update_max = acc.updmax;
        stats->t = ctx->t;
        stats->step = ctx->step;
    }
    if (*ctx->h_flag) return fail(ctx, SSG_ERR_NONFINITE, "surface buoyancy became non-finite");
    return SSG_OK;
}

extern "C" int ssg_solve_ma(ssg_ctx* ctx, ssg_ma_stats* stats) {
    if (!ctx) return SSG_ERR_ARG;
    CU(cudaSetDevice(ctx->device));
    const int64_t l0 = launch_counter();
    CU(cudaEventRecord(ctx->ev0, ctx->stream));
    int r = ma_solve(ctx, stats);
    CU(cudaEventRecord(ctx->ev1, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    ctx->last_ms = ms;
    ctx->last_launches = launch_counter() - l0;
    return r;
}

// physical (nx*ny) host array -> compact spectrum dst
int upload_surface(ssg_ctx* ctx, const double* host, double2* dst, int zero_mean) {
    const Dims& d = ctx->d;
    const Tables tb = ctx->tables();
    CU(cudaMemcpyAsync(ctx->phys, host, d.r2() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    KL(launch_y_r2c(d, tb, ctx->phys, ctx->mixed, 1, ctx->stream));
    KL(launch_x_fwd_compact(d, tb, ctx->mixed, dst, 1, 1.0, zero_mean, ctx->stream));
    return SSG_OK;
}

// compact planes -> physical host array
int download_planes(ssg_ctx* ctx, const double2* src, int nplanes, int mult, double* host) {
    const Dims& d = ctx->d;
    const Tables tb = ctx->tables();
    KL(launch_x_inv_compact(d, tb, src, ctx->mixed, nplanes, mult, ctx->stream));
    KL(launch_y_c2r(d, tb, ctx->mixed, ctx->phys, nplanes, ctx->stream));
    CU(cudaMemcpyAsync(host, ctx->phys, d.r2() * nplanes * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return SSG_OK;
}

extern "C" int ssg_set_b(ssg_ctx* ctx, const double* b, int64_t n, ssg_ma_stats* stats) {
    if (!ctx) return SSG_ERR_ARG;
    const Dims& d = ctx->d;
    if (!b || n != (int64_t)d.r2() * d.members) return fail(ctx, SSG_ERR_ARG, "set_b: expected nmembers*nx*ny values");
    CU(cudaSetDevice(ctx->device));
    for (int m = 0; m < d.members; ++m) {
        int r = upload_surface(ctx, b + d.r2() * m, ctx->bh + d.c2() * m, 1);
        if (r) return r;
    }
    reset_ring(ctx);
    CU(cudaMemsetAsync(ctx->Phat, 0, d.c2() * d.nz * d.members * sizeof(double2), ctx->stream));
    return ssg_solve_ma(ctx, stats);
}

extern "C" int ssg_set_field(ssg_ctx* ctx, int32_t field, const double* host, int64_t n) {
    if (!ctx) return SSG_ERR_ARG;
    CU(cudaSetDevice(ctx->device));
    const Dims& d = ctx->d;
    if (!host || n != (int64_t)d.r2() * d.members)
        return fail(ctx, SSG_ERR_ARG, "set_field: expected nmembers*nx*ny values");
    double2* dst;
    switch (field) {
        case SSG_FIELD_B_S: dst = ctx->bh; break;
        case SSG_FIELD_DBDT_OLD: dst = ctx->fold; break;
        default: return fail(ctx, SSG_ERR_ARG, "set_field: field is read-only or unknown");
    }
    for (int m = 0; m < d.members; ++m) {
        int r = upload_surface(ctx, host + d.r2() * m, dst + d.c2() * m, 0);
        if (r) return r;
    }
    CU(cudaStreamSynchronize(ctx->stream));
    return SSG_OK;
}

extern "C" int ssg_get_field(ssg_ctx* ctx, int32_t field, double* host, int64_t n) {
    if (!ctx || !host) return SSG_ERR_ARG;
    CU(cudaSetDevice(ctx->device));
    const Dims& d = ctx->d;
    const size_t c2 = d.c2(), c3 = c2 * d.nz;
    // per member: its first compact plane, its member stride, planes, multiplier
    const double2* src = nullptr;
    size_t stride = c2;
    int planes = 1, mult = 0;
    switch (field) {
        case SSG_FIELD_B_S: src = ctx->bh; break;
        case SSG_FIELD_PHI_S: src = ctx->Phat + c2 * (d.nz - 1), stride = c3; break;
        case SSG_FIELD_PHI: src = ctx->Phat, stride = c3, planes = d.nz; break;
        case SSG_FIELD_DBDT_OLD: src = ctx->fold; break;
        case SSG_FIELD_U_S: src = ctx->Phat + c2 * (d.nz - 1), stride = c3, mult = 1; break;
        case SSG_FIELD_V_S: src = ctx->Phat + c2 * (d.nz - 1), stride = c3, mult = 2; break;
        default: return fail(ctx, SSG_ERR_ARG, "get_field: unknown field");
    }
    const int64_t per = (int64_t)d.r2() * planes;
    if (n != per * d.members) return fail(ctx, SSG_ERR_ARG, "get_field: wrong element count");
    for (int m = 0; m < d.members; ++m) {
        int r = download_planes(ctx, src + stride * m, planes, mult, host + per * m);
        if (r) return r;
    }
    return SSG_OK;
}

extern "C" int ssg_apply_filter(ssg_ctx* ctx) {
    if (!ctx) return SSG_ERR_ARG;
    CU(cudaSetDevice(ctx->device));
    KL(launch_filter(ctx->d, ctx->tables(), ctx->bh, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return SSG_OK;
}

extern "C" int ssg_set_filter_table(ssg_ctx* ctx, const double* sigma, int64_t n) {
    if (!ctx) return SSG_ERR_ARG;
    const Dims& d = ctx->d;
    if (!sigma || n != (int64_t)d.N * d.nyc) return fail(ctx, SSG_ERR_ARG, "set_filter_table: expected nx*(ny/2+1) values");
    CU(cudaSetDevice(ctx->device));
    std::vector<double> sig(d.c2());
    for (int j = 0; j < d.My; ++j)
        for (int c = 0; c < d.Mx; ++c) {
            const int i = c < d.Kp ? c : c + (d.N - 2 * d.Kp);
            sig[c + (size_t)d.Mx * j] = sigma[i + (size_t)d.N * j];
        }
    CU(cudaMemcpy(ctx->sigma, sig.data(), d.c2() * sizeof(double), cudaMemcpyHostToDevice));
    ctx->cfg.filter_type = SSG_FILTER_CUSTOM;
    return SSG_OK;
}

extern "C" int ssg_get_diagnostics(ssg_ctx* ctx, ssg_diagnostics* out) {
    if (!ctx || !out) return SSG_ERR_ARG;
    if (ctx->d.members > 1) return fail(ctx, SSG_ERR_UNSUPPORTED, "get_diagnostics: one member per context");
    CU(cudaSetDevice(ctx->device));
    const Dims& d = ctx->d;
    const double2* top = ctx->Phat + d.c2() * (d.nz - 1);
    KL(launch_diagnostics(d, ctx->tables(), top, ctx->bh, ctx->partials, ctx->ticket, ctx->norms, ctx->stream));
    double2 b00;
    CU(cudaMemcpyAsync(ctx->h_norms, ctx->norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(&b00, ctx->bh, sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    const double N2 = (double)d.N * (double)d.N;
    const double area = ctx->cfg.lx * ctx->cfg.ly;
    out->t = ctx->t;
    out->step = ctx->step;
    out->kinetic_energy = 0.5 * area / (N2 * N2) * ctx->h_norms[0];
    out->buoyancy_variance = area / (N2 * N2) * ctx->h_norms[1];
    out->total_buoyancy = area / N2 * b00.x;
    out->ma_last_iterations = ctx->last_ma_iterations;
    out->pad0 = 0;
    return SSG_OK;
}

// ---- checkpoint blob: header + bh, fold, bstage, Phat, hist[0..2] -----------
// (version 1 blobs hold one history plane set, version 2 two, version 3 three)
struct CkptHeader {
    char magic[8];
    int32_t version, nx, ny, nz, nhist, precision;
    double t;
    int64_t step;
    int64_t payload;
};
static const char kCkptMagic[8] = {'S', 'S', 'G', 'B', '2', '0', '0', 0};

static int ckpt_hist_sets(int version) { return version >= 3 ? 3 : version; }
static int64_t ckpt_payload(const ssg_ctx* ctx, int version = 3) {
    return (int64_t)((3 + (size_t)(1 + ckpt_hist_sets(version)) * ctx->d.nz) * ctx->d.c2() * ctx->d.members *
                     sizeof(double2));
}

extern "C" int ssg_checkpoint_size(const ssg_ctx* ctx, int64_t* bytes) {
    if (!ctx || !bytes) return SSG_ERR_ARG;
    *bytes = (int64_t)sizeof(CkptHeader) + ckpt_payload(ctx);
    return SSG_OK;
}

extern "C" int ssg_checkpoint(ssg_ctx* ctx, void* blob, int64_t bytes) {
    if (!ctx || !blob) return SSG_ERR_ARG;
    const int64_t need = (int64_t)sizeof(CkptHeader) + ckpt_payload(ctx);
    if (bytes < need) return fail(ctx, SSG_ERR_ARG, "checkpoint: buffer too small");
    CU(cudaSetDevice(ctx->device));
    CkptHeader h{};
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = 3;
    h.nx = ctx->cfg.nx;
    h.ny = ctx->cfg.ny;
    h.nz = ctx->cfg.nz;
    h.nhist = ctx->nhist;
    h.precision = ctx->cfg.precision;
    h.t = ctx->t;
    h.step = ctx->step;
    h.payload = ckpt_payload(ctx);
    unsigned char* p = static_cast<unsigned char*>(blob);
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    // every member's buffers (members one after another within each)
    const size_t c2 = ctx->d.c2() * ctx->d.members * sizeof(double2), c3 = c2 * ctx->d.nz;
    CU(cudaMemcpyAsync(p, ctx->bh, c2, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(p + c2, ctx->fold, c2, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(p + 2 * c2, ctx->bstage, c2, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaMemcpyAsync(p + 3 * c2, ctx->Phat, c3, cudaMemcpyDeviceToHost, ctx->stream));
    for (int i = 0; i < 3; ++i)
        CU(cudaMemcpyAsync(p + 3 * c2 + (1 + i) * c3, ctx->hist[i], c3, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return SSG_OK;
}

extern "C" int ssg_restore(ssg_ctx* ctx, const void* blob, int64_t bytes) {
    if (!ctx || !blob) return SSG_ERR_ARG;
    if (bytes < (int64_t)sizeof(CkptHeader)) return fail(ctx, SSG_ERR_ARG, "restore: blob too small");
    CkptHeader h;
    std::memcpy(&h, blob, sizeof(h));
    if (std::memcmp(h.magic, kCkptMagic, 8) != 0 || h.version < 1 || h.version > 3)
        return fail(ctx, SSG_ERR_ARG, "restore: not a checkpoint of this library");
    if (h.nx != ctx->cfg.nx || h.ny != ctx->cfg.ny || h.nz != ctx->cfg.nz)
        return fail(ctx, SSG_ERR_ARG, "restore: checkpoint grid differs from the context's");
    if (h.payload != ckpt_payload(ctx, h.version))
        return fail(ctx, SSG_ERR_ARG, "restore: checkpoint of another member count (nmembers) or corrupt header");
    if (bytes < (int64_t)sizeof(h) + h.payload) return fail(ctx, SSG_ERR_ARG, "restore: truncated checkpoint");
    if (h.nhist < 0 || h.nhist > 1 + ckpt_hist_sets(h.version) || h.step < 0)
        return fail(ctx, SSG_ERR_ARG, "restore: corrupt header");
    CU(cudaSetDevice(ctx->device));
    // the predictor ring goes back to allocation order before the solutions
    // are copied in, so that every restored run meets the same buffer
    // assignment (and the step graphs cached for it)
    reset_ring(ctx);
    const unsigned char* p = static_cast<const unsigned char*>(blob) + sizeof(h);
    const size_t c2 = ctx->d.c2() * ctx->d.members * sizeof(double2), c3 = c2 * ctx->d.nz;
    CU(cudaMemcpyAsync(ctx->bh, p, c2, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->fold, p + c2, c2, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->bstage, p + 2 * c2, c2, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaMemcpyAsync(ctx->Phat, p + 3 * c2, c3, cudaMemcpyHostToDevice, ctx->stream));
    for (int i = 0; i < ckpt_hist_sets(h.version); ++i)
        CU(cudaMemcpyAsync(ctx->hist[i], p + 3 * c2 + (1 + i) * c3, c3, cudaMemcpyHostToDevice, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->nhist = h.nhist;
    return set_clock(ctx, h.t, h.step);
}

extern "C" int ssg_set_vertical_grid(ssg_ctx* ctx, const double* dz, int32_t n) {
    if (!ctx) return SSG_ERR_ARG;
    if (!dz || n != ctx->cfg.nz) return fail(ctx, SSG_ERR_ARG, "set_vertical_grid: expected nz spacings");
    std::vector<double> v(dz, dz + n);
    for (int k = 0; k < n; ++k)
        if (!std::isfinite(v[k]) || v[k] == 0.0) return fail(ctx, SSG_ERR_ARG, "set_vertical_grid: spacings must be finite and non-zero");
    for (int k = 1; k < n; ++k)
        if (v[k - 1] + v[k] == 0.0) return fail(ctx, SSG_ERR_ARG, "set_vertical_grid: adjacent spacings cancel");
    const ZOps z = vertical_ops(v);
    CU(cudaSetDevice(ctx->device));
    CU(cudaStreamSynchronize(ctx->stream));
    CU(cudaMemcpyAsync(ctx->zops, &z, sizeof(ZOps), cudaMemcpyHostToDevice, ctx->stream));
    if (launch_ma_thomas_factor(ctx->d, ctx->tables(), ctx->zops, ctx->tinv, ctx->stream))
        return fail(ctx, SSG_ERR_CUDA, "set_vertical_grid: factorisation launch failed");
    CU(cudaStreamSynchronize(ctx->stream));
    return SSG_OK;
}

extern "C" int ssg_get_time(const ssg_ctx* ctx, double* t, int64_t* step) {
    if (!ctx) return SSG_ERR_ARG;
    if (t) *t = ctx->t;
    if (step) *step = ctx->step;
    return SSG_OK;
}

extern "C" int ssg_set_time(ssg_ctx* ctx, double t, int64_t step) {
    if (!ctx) return SSG_ERR_ARG;
    if (step < 0) return fail(ctx, SSG_ERR_ARG, "step < 0");
    CU(cudaSetDevice(ctx->device));
    return set_clock(ctx, t, step);
}

extern "C" int ssg_last_timing(const ssg_ctx* ctx, double* ms, int64_t* launches) {
    if (!ctx) return SSG_ERR_ARG;
    if (ms) *ms = ctx->last_ms;
    if (launches) *launches = ctx->last_launches;
    return SSG_OK;
}

extern "C" int ssg_profile_kernels(ssg_ctx* ctx, int enable) {
    if (!ctx) return SSG_ERR_ARG;
    CU(cudaSetDevice(ctx->device));
    CU(cudaStreamSynchronize(ctx->stream));
    drain_profile(ctx);
    ctx->profiling = enable != 0;
    for (int i = 0; i < KC_COUNT; ++i) {
        ctx->kc_ms[i] = 0.0;
        ctx->kc_n[i] = 0;
    }
    return SSG_OK;
}

extern "C" int ssg_kernel_times(ssg_ctx* ctx, double* ms, int64_t* launches, int32_t nclass) {
    if (!ctx || nclass < 0) return SSG_ERR_ARG;
    CU(cudaSetDevice(ctx->device));
    CU(cudaStreamSynchronize(ctx->stream));
    drain_profile(ctx);
    for (int i = 0; i < nclass && i < KC_COUNT; ++i) {
        if (ms) ms[i] = ctx->kc_ms[i];
        if (launches) launches[i] = ctx->kc_n[i];
    }
    return SSG_OK;
}

// ---------------------------------------------------------------------------
// Block shapes of the step's transform passes (tunable for 64 <= N <= 512)
// ---------------------------------------------------------------------------
static bool tile_candidate(const int (&cands)[3], int bt) {
    if (bt == 0) return true;
    for (int c : cands)
        if (c == bt) return true;
    return false;
}

static bool tiles_tunable(const ssg_ctx* ctx) { return ctx->d.N >= 64 && ctx->d.N <= 512; }

// The Monge-Ampere y-pass kernel of this context (SSG_YPASS_*).
static int current_y_variant(const ssg_ctx* ctx) {
    if (ctx->cfg.precision == 1) {
        if (!ctx->use_tma32) return SSG_YPASS_PLAIN;
        return ctx->use_warp32 ? ctx->ytm32w.warps : SSG_YPASS_TMA;
    }
    return ctx->use_tma ? SSG_YPASS_TMA : SSG_YPASS_PLAIN;
}

// Selects y-pass kernel v, building its tensor maps; SSG_ERR_UNSUPPORTED
// (nothing changed) when the kernel does not exist for this grid/precision.
static int apply_y_variant(ssg_ctx* ctx, int v) {
    const Dims& d = ctx->d;
    float2* A32 = reinterpret_cast<float2*>(ctx->A);
    float2* B32 = reinterpret_cast<float2*>(ctx->B);
    float2* C32 = reinterpret_cast<float2*>(ctx->C);
    float2* D32 = reinterpret_cast<float2*>(ctx->Dt);
    if (v == SSG_YPASS_PLAIN) {
        if (ctx->cfg.precision == 1) ctx->use_tma32 = false;
        else ctx->use_tma = false;
        return SSG_OK;
    }
    if (!mixed_tma_supported(d)) return SSG_ERR_UNSUPPORTED;
    if (ctx->cfg.precision == 0) {
        if (v != SSG_YPASS_TMA) return SSG_ERR_UNSUPPORTED;
        if (make_mixed_tmaps(d, ctx->A, ctx->B, ctx->C, ctx->Dt, ma_planes(d), &ctx->ytm)) return SSG_ERR_UNSUPPORTED;
        ctx->use_tma = true;
        return SSG_OK;
    }
    if (v == SSG_YPASS_TMA) {
        if (make_mixed32_tmaps(d, A32, B32, C32, D32, ma_planes(d), &ctx->ytm32)) return SSG_ERR_UNSUPPORTED;
        ctx->use_tma32 = true;
        ctx->use_warp32 = false;
        return SSG_OK;
    }
    if (v == SSG_YPASS_WARP2 || v == SSG_YPASS_WARP4 || v == SSG_YPASS_WARP8) {
        if (d.N != 1024 || !ctx->tww32) return SSG_ERR_UNSUPPORTED;
        if (make_mixed32_tmaps(d, A32, B32, C32, D32, ma_planes(d), &ctx->ytm32)) return SSG_ERR_UNSUPPORTED;
        if (make_mixed32w_tmaps(d, A32, B32, C32, D32, ma_planes(d), v, &ctx->ytm32w)) return SSG_ERR_UNSUPPORTED;
        ctx->use_tma32 = true;
        ctx->use_warp32 = true;
        return SSG_OK;
    }
    return SSG_ERR_UNSUPPORTED;
}

extern "C" int ssg_set_variants(ssg_ctx* ctx, int32_t y_pass, int32_t thomas_staged) {
    if (!ctx) return SSG_ERR_ARG;
    if (thomas_staged != 0 && thomas_staged != 1) return fail(ctx, SSG_ERR_ARG, "set_variants: thomas_staged is 0 or 1");
    CU(cudaSetDevice(ctx->device));
    CU(cudaStreamSynchronize(ctx->stream));
    const int y0 = current_y_variant(ctx);
    if (y_pass != y0 || (thomas_staged != 0) != ctx->thomas_staged) release_graphs(ctx);  // graphs bake in kernels
    if (y_pass != y0 && apply_y_variant(ctx, y_pass) != SSG_OK) {
        apply_y_variant(ctx, y0);
        return fail(ctx, SSG_ERR_UNSUPPORTED, "set_variants: y-pass kernel not available for this grid and precision");
    }
    ctx->thomas_staged = thomas_staged != 0;
    return SSG_OK;
}

extern "C" int ssg_get_variants(const ssg_ctx* ctx, int32_t* y_pass, int32_t* thomas_staged) {
    if (!ctx) return SSG_ERR_ARG;
    if (y_pass) *y_pass = current_y_variant(ctx);
    if (thomas_staged) *thomas_staged = ctx->thomas_staged ? 1 : 0;
    return SSG_OK;
}

extern "C" int ssg_set_tiles(ssg_ctx* ctx, int32_t x_threads, int32_t y_threads) {
    if (!ctx) return SSG_ERR_ARG;
    if (!tile_candidate(kTileThreadsX, x_threads) || !tile_candidate(kTileThreadsY, y_threads))
        return fail(ctx, SSG_ERR_ARG, "set_tiles: x_threads in {0, 64, 128, 256}, y_threads in {0, 128, 256, 512}");
    if (!tiles_tunable(ctx) && (x_threads || y_threads))
        return fail(ctx, SSG_ERR_UNSUPPORTED, "set_tiles: block shapes are tunable for 64 <= N <= 512");
    CU(cudaSetDevice(ctx->device));
    CU(cudaStreamSynchronize(ctx->stream));
    if (x_threads != ctx->d.xbt || y_threads != ctx->d.ybt) release_graphs(ctx);  // graphs bake in launch shapes
    ctx->d.xbt = x_threads;
    ctx->d.ybt = y_threads;
    return SSG_OK;
}

extern "C" int ssg_get_tiles(const ssg_ctx* ctx, int32_t* x_threads, int32_t* y_threads) {
    if (!ctx) return SSG_ERR_ARG;
    if (x_threads) *x_threads = ctx->d.xbt;
    if (y_threads) *y_threads = ctx->d.ybt;
    return SSG_OK;
}

// Times each candidate block shape on this context's grid and precision over
// `reps` rounds of one Monge-Ampere iteration and one tendency pass (CUDA
// events per kernel class), keeps the fastest shape for the row passes, then
// for the column-pair passes, and restores the state the context had.
extern "C" int ssg_autotune(ssg_ctx* ctx, int32_t reps, int32_t* x_threads, int32_t* y_threads) {
    if (!ctx || reps < 1) return SSG_ERR_ARG;
    CU(cudaSetDevice(ctx->device));
    int64_t nb = 0;
    int r;
    if ((r = ssg_checkpoint_size(ctx, &nb))) return r;
    std::vector<unsigned char> blob((size_t)nb);
    if ((r = ssg_checkpoint(ctx, blob.data(), nb))) return r;
    const bool was_profiling = ctx->profiling;
    const int x0 = ctx->d.xbt, y0 = ctx->d.ybt;
    // every member's vertical solve runs while the passes are timed
    KL(launch_solve_begin(ctx->sdev, ctx->active, ctx->d.members, ctx->stream));
    auto round = [&]() -> int {
        int rr = ma_iteration(ctx, ctx->stream);
        return rr ? rr : tendency_stage(ctx, STAGE_AB2, 0, 0.0);
    };
    // summed time of the given kernel classes over `reps` rounds
    auto measure = [&](std::initializer_list<int> classes, double& ms) -> int {
        int rr;
        if ((rr = round())) return rr;  // first launches of this shape (attributes, caches)
        if ((rr = ssg_profile_kernels(ctx, 1))) return rr;
        for (int i = 0; i < reps; ++i)
            if ((rr = round())) return rr;
        CU(cudaStreamSynchronize(ctx->stream));
        drain_profile(ctx);
        ms = 0.0;
        for (int c : classes) ms += ctx->kc_ms[c];
        return SSG_OK;
    };
    int best_x = x0, best_y = y0;
    double best = 1e300;
    release_graphs(ctx);
    r = SSG_OK;
    if (tiles_tunable(ctx)) {
        for (int bt : kTileThreadsX) {
            ctx->d.xbt = bt;
            double ms = 0.0;
            if ((r = measure({KC_MA_XINV, KC_MA_XFWD, KC_SURF_XINV, KC_SURF_XFWD}, ms))) break;
            if (ms < best) best = ms, best_x = bt;
        }
        ctx->d.xbt = best_x;
        best = 1e300;
        for (int bt : kTileThreadsY) {
            if (r) break;
            ctx->d.ybt = bt;
            double ms = 0.0;
            if ((r = measure({KC_MA_Y, KC_SURF_Y}, ms))) break;
            if (ms < best) best = ms, best_y = bt;
        }
        ctx->d.ybt = best_y;
    }
    // kernel variants of the y-pass (plain loads, TMA tiles, one warp per
    // transform with 2, 4 or 8 warps per block) and of the vertical solve
    // (column in registers or staged through shared memory)
    const int yv0 = current_y_variant(ctx);
    const bool ts0 = ctx->thomas_staged;
    if (!r) {
        int best_v = yv0;
        best = 1e300;
        for (int v : {SSG_YPASS_PLAIN, SSG_YPASS_TMA, SSG_YPASS_WARP2, SSG_YPASS_WARP4, SSG_YPASS_WARP8}) {
            if (apply_y_variant(ctx, v) != SSG_OK) continue;
            double ms = 0.0;
            if ((r = measure({KC_MA_Y}, ms))) break;
            if (ms < best) best = ms, best_v = v;
        }
        if (!r) r = apply_y_variant(ctx, best_v);
    }
    if (!r) {
        bool best_s = ts0;
        best = 1e300;
        for (bool staged : {false, true}) {
            ctx->thomas_staged = staged;
            double ms = 0.0;
            if ((r = measure({KC_MA_THOMAS}, ms))) break;
            if (ms < best) best = ms, best_s = staged;
        }
        ctx->thomas_staged = best_s;
    }
    if (r) {
        ctx->d.xbt = x0;
        ctx->d.ybt = y0;
        apply_y_variant(ctx, yv0);
        ctx->thomas_staged = ts0;
    }
    release_graphs(ctx);
    // back to the state (and profiling mode) the context had
    const int rs = ssg_restore(ctx, blob.data(), nb);
    ssg_profile_kernels(ctx, was_profiling ? 1 : 0);
    if (r) return r;
    if (rs) return rs;
    if (x_threads) *x_threads = ctx->d.xbt;
    if (y_threads) *y_threads = ctx->d.ybt;
    return SSG_OK;
}

extern "C" const char* ssg_last_error(const ssg_ctx* ctx) {
    return ctx ? ctx->err.c_str() : g_create_error.c_str();
}
