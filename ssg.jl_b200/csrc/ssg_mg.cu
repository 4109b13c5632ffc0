// ssg_mg.cu -- the reference's own Monge-Ampere multigrid on the GPU.
//
// SSG.jl's solve_ssg_equation (src/poisson.jl:869-959) builds an
// SSGMultigridSolver over SSGLevels (src/poisson.jl:33-127) and V-cycles with
// a spectral or red-black SOR smoother.  As shipped that solver diverges
// (spectral smoother) or stays inert (SOR ignores the right-hand side), so the
// time step does not use it (the time step solves the documented equations in
// ssg_ctx.cu).  These entry points reproduce the reference's functions as they
// are, on physical 3-D fields, so that each is available and checked against
// its CPU restatement:
//   compute_ssg_residual!           src/poisson.jl:228-253 (+ :143-223, d2dz2!)
//   apply_ssg_boundary_conditions!  src/poisson.jl:262-364
//   ssg_spectral_smoother!          src/poisson.jl:635-697
//   ssg_sor_smoother! / _enhanced! / _adaptive!  src/poisson.jl:402-630
//   restrict_ssg_3d!, prolongate_ssg_3d!  src/poisson.jl:706-793 (injection)
//   ssg_v_cycle!                    src/poisson.jl:802-860
//   norm_field                      src/poisson.jl:986-995
// Horizontal derivatives use full (unmasked) spectra, as rfft!/ddx!/irfft! do.
#include "../../include/ssg_b200.h"
#include "kernels.cuh"
#include "fft.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

using namespace ssg;

namespace {

// ---- full-spectrum x-passes -------------------------------------------------

template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    x_fwd_full_kernel(const double2* __restrict__ in, double2* __restrict__ out, const double2* __restrict__ tw,
                      int rows) {
    constexpr int T = N / 8;
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int row = blockIdx.x * ROWS + team;
    const bool active = row < rows;
    const size_t o = (size_t)N * (row + (size_t)rows * blockIdx.y);
    double2 v[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = active ? in[o + t + p * T] : make_double2(0.0, 0.0);
    fft_team<N, -1>(v, t, buf, tw);
    if (active) {
#pragma unroll
        for (int p = 0; p < 8; ++p) out[o + t + p * T] = v[p];
    }
}

// mult: 0 none, 1 ddx(ddx), 2 ddy(ddy), 3 ddy(ddx); scale = 1/(nx ny)
template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    x_inv_full_kernel(const double2* __restrict__ in, double2* __restrict__ out, const double2* __restrict__ tw,
                      const double* __restrict__ kxf, const double* __restrict__ kyf, int rows, int mult,
                      double scale) {
    constexpr int T = N / 8;
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int row = blockIdx.x * ROWS + team;
    const bool active = row < rows;
    const size_t o = (size_t)N * (row + (size_t)rows * blockIdx.y);
    const double ky = active ? kyf[row] : 0.0;
    double2 v[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        double2 x = make_double2(0.0, 0.0);
        if (active) {
            x = cscale(in[o + t + p * T], scale);
            const double kx = kxf[t + p * T];
            if (mult == 1) x = cmul_is(cmul_is(x, kx), kx);
            else if (mult == 2) x = cmul_is(cmul_is(x, ky), ky);
            else if (mult == 3) x = cmul_is(cmul_is(x, kx), ky);
        }
        v[p] = x;
    }
    fft_team<N, +1>(v, t, buf, tw);
    if (active) {
#pragma unroll
        for (int p = 0; p < 8; ++p) out[o + t + p * T] = v[p];
    }
}

// ---- pointwise pieces --------------------------------------------------------

struct ZRows {
    double al[64], be[64], ga[64], dz[64];
    double at, bt, ct, ab, bb, cb;
    // rows and relaxation factors of ssg_sor_smoother_enhanced! with metrics
    double ma[64], mb[64], mc[64], mw[64];
};

// r = (Phi_xx + Phi_yy + Phi_zz) - eps (Phi_xx Phi_yy - Phi_xy^2) - b, with
// Phi_zz from d2dz2! on interior planes and 0 on planes 1 and nz (the
// reference's Phi_zz array keeps its initial zeros there)
__global__ void mg_combine_kernel(const double* __restrict__ xx, const double* __restrict__ yy,
                                  const double* __restrict__ xy, const double* __restrict__ Phi,
                                  const double* __restrict__ b, double* __restrict__ r, const ZRows* __restrict__ z,
                                  size_t n2, int nz, double eps) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n2 * nz) return;
    const int k = (int)(idx / n2);
    double zz = 0.0;
    if (k > 0 && k < nz - 1) zz = z->al[k] * Phi[idx - n2] + z->be[k] * Phi[idx] + z->ga[k] * Phi[idx + n2];
    const double a = xx[idx], c = yy[idx], d = xy[idx];
    const double lap = a + c + zz;
    const double D = a * c - d * d;
    r[idx] = lap - eps * D - b[idx];
}

__global__ void mg_bc_kernel(double* __restrict__ Phi, double* __restrict__ r, const double* __restrict__ bs,
                             const ZRows* __restrict__ z, size_t n2, int nz) {
    const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n2) return;
    const int k = nz - 1;
    Phi[m + n2 * k] = (bs[m] - z->bt * Phi[m + n2 * (k - 1)] - z->ct * Phi[m + n2 * (k - 2)]) / z->at;
    r[m + n2 * k] = 0.0;
    Phi[m] = -(z->bb * Phi[m + n2] + z->cb * Phi[m + 2 * n2]) / z->ab;
    r[m] = 0.0;
}

// Phi_hat += omega r_hat / (k^2 + eps k^2 + 1e-12) for k^2 > 1e-14, then the
// 2/3 mask (dealias!)
__global__ void mg_spectral_update_kernel(double2* __restrict__ Ph, const double2* __restrict__ Rh,
                                          const double* __restrict__ kxf, const double* __restrict__ kyf, int N,
                                          int nyc, int nz, double omega, double eps) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)N * nyc * nz) return;
    const int i = (int)(idx % N), j = (int)((idx / N) % nyc);
    const int kxm = N / 3, kym = (2 * nyc) / 3;
    const bool keep = (i < kxm || i >= N - kxm) && j < kym;
    if (!keep) {
        Ph[idx] = make_double2(0.0, 0.0);
        return;
    }
    const double ksq = kxf[i] * kxf[i] + kyf[j] * kyf[j];
    if (ksq > 1e-14) {
        const double epsf = eps * ksq;
        const double pre = 1.0 / (ksq + epsf + 1e-12);
        const double2 r = Rh[idx];
        const double2 p = Ph[idx];
        Ph[idx] = make_double2(p.x + omega * (r.x * pre), p.y + omega * (r.y * pre));
    }
}

// one colour of the red-black sweep; (i, j, k) are 1-based as in the reference.
// plain: ssg_sor_smoother! (diagonal carries -0.1 eps); otherwise the enhanced
// smoother, with the metric rows and relaxation factors when metrics is set.
__global__ void mg_sor_color_kernel(double* __restrict__ Phi, const ZRows* __restrict__ z, int nx, int ny, int nz,
                                    double idx2, double idy2, double omega, double eps, int plain, int metrics,
                                    int color) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int j = blockIdx.y + 2;
    const int k = blockIdx.z + 2;
    if (i > nx - 1 || j > ny - 1 || k > nz - 1) return;
    if ((i + j + k) % 2 != color) return;
    const size_t n2 = (size_t)nx * ny;
    const size_t at = (size_t)(i - 1) + (size_t)nx * (j - 1) + n2 * (k - 1);
    const double c = Phi[at];
    const double e = Phi[at + 1], w = Phi[at - 1], nn = Phi[at + nx], ss = Phi[at - nx];
    const double u = Phi[at + n2], d = Phi[at - n2];
    double a, bta, gm, relax = omega;
    if (metrics) {
        a = z->ma[k - 1];
        bta = z->mb[k - 1];
        gm = z->mc[k - 1];
        relax = omega * z->mw[k - 1];
    } else {
        const double hb = z->dz[k - 2], ha = z->dz[k - 1], ht = hb + ha;
        a = 2.0 / (hb * ht);
        bta = -2.0 / (hb * ha);
        gm = 2.0 / (ha * ht);
    }
    const double diag = plain ? (-2 * idx2 - 2 * idy2 + bta - eps * 0.1) : (-2 * idx2 - 2 * idy2 + bta);
    const double off = (e + w) * idx2 + (nn + ss) * idy2 + a * d + gm * u;
    if (fabs(diag) > 1e-14) {
        const double nv = -off / diag;
        Phi[at] = c + relax * (nv - c);
    }
}

__global__ void mg_restrict_kernel(double* __restrict__ C, const double* __restrict__ F, int cx, int cy, int fx,
                                   int fy, int nz) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)cx * cy * nz) return;
    const int i = (int)(idx % cx), j = (int)((idx / cx) % cy), k = (int)(idx / ((size_t)cx * cy));
    if (2 * i < fx && 2 * j < fy) C[idx] = F[(size_t)2 * i + (size_t)fx * 2 * j + (size_t)fx * fy * k];
}

__global__ void mg_prolong_kernel(double* __restrict__ F, const double* __restrict__ C, int cx, int cy, int fx,
                                  int fy, int nz) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)cx * cy * nz) return;
    const int i = (int)(idx % cx), j = (int)((idx / cx) % cy), k = (int)(idx / ((size_t)cx * cy));
    if (2 * i < fx && 2 * j < fy) F[(size_t)2 * i + (size_t)fx * 2 * j + (size_t)fx * fy * k] += C[idx];
}

__global__ void mg_sub_kernel(double* __restrict__ a, const double* __restrict__ b, size_t n) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < n) a[idx] -= b[idx];
}

// sum of squares: per-block partials (fixed order), then one block sums them
__global__ void mg_sumsq_partial_kernel(const double* __restrict__ x, size_t n, double* __restrict__ part) {
    __shared__ double red[256];
    double s = 0.0;
    for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (size_t)gridDim.x * 256) s += x[i] * x[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void mg_sum_final_kernel(const double* __restrict__ part, int nparts, double* __restrict__ out) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < nparts; i += 256) s += part[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

template <int N>
int x_full_impl(int dir, const double2* in, double2* out, const double2* tw, const double* kxf, const double* kyf,
                int rows, int nplanes, int mult, double scale, cudaStream_t s) {
    constexpr int T = N / 8;
    constexpr int R = (128 / T) > 1 ? (128 / T) : 1;
    const size_t sm = (size_t)R * FftShape<N>::BUF * sizeof(double2);
    dim3 grid((rows + R - 1) / R, nplanes), block(T, R);
    if (dir < 0) {
        auto k = x_fwd_full_kernel<N, R>;
        if (sm > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k<<<grid, block, sm, s>>>(in, out, tw, rows);
    } else {
        auto k = x_inv_full_kernel<N, R>;
        if (sm > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k<<<grid, block, sm, s>>>(in, out, tw, kxf, kyf, rows, mult, scale);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

int launch_x_full(int N, int dir, const double2* in, double2* out, const double2* tw, const double* kxf,
                  const double* kyf, int rows, int nplanes, int mult, double scale, cudaStream_t s) {
    switch (N) {
        case 8: return x_full_impl<8>(dir, in, out, tw, kxf, kyf, rows, nplanes, mult, scale, s);
        case 16: return x_full_impl<16>(dir, in, out, tw, kxf, kyf, rows, nplanes, mult, scale, s);
        case 32: return x_full_impl<32>(dir, in, out, tw, kxf, kyf, rows, nplanes, mult, scale, s);
        case 64: return x_full_impl<64>(dir, in, out, tw, kxf, kyf, rows, nplanes, mult, scale, s);
        case 128: return x_full_impl<128>(dir, in, out, tw, kxf, kyf, rows, nplanes, mult, scale, s);
        case 256: return x_full_impl<256>(dir, in, out, tw, kxf, kyf, rows, nplanes, mult, scale, s);
        case 512: return x_full_impl<512>(dir, in, out, tw, kxf, kyf, rows, nplanes, mult, scale, s);
        case 1024: return x_full_impl<1024>(dir, in, out, tw, kxf, kyf, rows, nplanes, mult, scale, s);
        default: return -6;
    }
}

int coarsen(int n) {
    int c = n / 2 > 5 ? n / 2 : 5;
    return c % 2 == 0 ? c : c + 1;
}

}  // namespace

struct MgLevelDev {
    Dims d{};          // My = N/2 + 1: full spectra
    size_t n2 = 0, n3 = 0, c3 = 0;
    double2* tw = nullptr;
    double *kxf = nullptr, *kyf = nullptr;
    ZRows* z = nullptr;
    double *Phi = nullptr, *b = nullptr, *r = nullptr, *Phi_old = nullptr, *bs = nullptr;
    double *xx = nullptr, *yy = nullptr, *xy = nullptr;
    double2 *spec = nullptr, *rspec = nullptr, *mixed = nullptr;
    double dx = 0, dy = 0;
};

struct ssg_mg {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<MgLevelDev> lv;
    std::vector<void*> allocs;
    double* partials = nullptr;
    double* sum = nullptr;
    double max_stretch = 1.0;  // of the vertical spacing, for the adaptive smoother
    std::string err;
};

static thread_local std::string g_mg_error;

static int mg_fail(ssg_mg* m, int code, const std::string& msg) {
    if (m) m->err = msg; else g_mg_error = msg;
    return code;
}

#define MCU(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return mg_fail(m, e_ == cudaErrorMemoryAllocation ? SSG_ERR_OOM : SSG_ERR_CUDA,           \
                           std::string(#call) + ": " + cudaGetErrorString(e_));                     \
    } while (0)
#define MKL(call)                                                                             \
    do {                                                                                      \
        int r_ = (call);                                                                      \
        if (r_ == -6) return mg_fail(m, SSG_ERR_UNSUPPORTED, "grid size not supported");      \
        if (r_ != 0) return mg_fail(m, SSG_ERR_CUDA, std::string("kernel launch: ") + #call); \
    } while (0)

template <typename T>
static int mg_alloc(ssg_mg* m, T** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T) + 256) != cudaSuccess) return mg_fail(m, SSG_ERR_OOM, "cudaMalloc failed");
    m->allocs.push_back(q);
    *p = static_cast<T*>(q);
    return SSG_OK;
}

static unsigned blocks_for(size_t n, int tb = 256) { return (unsigned)((n + tb - 1) / tb); }

static Tables level_tables(const MgLevelDev& L) { return Tables{L.tw, nullptr, L.kxf, L.kyf, nullptr}; }

// physical planes -> full spectra (rfft!)
static int fwd_full(ssg_mg* m, MgLevelDev& L, const double* phys, double2* spec) {
    MKL(launch_y_r2c(L.d, level_tables(L), phys, L.mixed, L.d.nz, m->stream));
    MKL(launch_x_full(L.d.N, -1, L.mixed, spec, L.tw, L.kxf, L.kyf, L.d.nyc, L.d.nz, 0, 1.0, m->stream));
    return SSG_OK;
}

// full spectra with a derivative multiplier -> physical planes (irfft!)
static int inv_full(ssg_mg* m, MgLevelDev& L, const double2* spec, double* phys, int mult) {
    const double scale = 1.0 / ((double)L.d.N * (double)L.d.N);
    MKL(launch_x_full(L.d.N, +1, spec, L.mixed, L.tw, L.kxf, L.kyf, L.d.nyc, L.d.nz, mult, scale, m->stream));
    MKL(launch_y_c2r(L.d, level_tables(L), L.mixed, phys, L.d.nz, m->stream));
    return SSG_OK;
}

static int mg_bc(ssg_mg* m, MgLevelDev& L) {
    mg_bc_kernel<<<blocks_for(L.n2), 256, 0, m->stream>>>(L.Phi, L.r, L.bs, L.z, L.n2, L.d.nz);
    MCU(cudaGetLastError());
    return SSG_OK;
}

static int mg_residual(ssg_mg* m, MgLevelDev& L, double eps) {
    int r;
    if ((r = fwd_full(m, L, L.Phi, L.spec))) return r;
    if ((r = inv_full(m, L, L.spec, L.xx, 1))) return r;
    if ((r = inv_full(m, L, L.spec, L.yy, 2))) return r;
    if ((r = inv_full(m, L, L.spec, L.xy, 3))) return r;
    mg_combine_kernel<<<blocks_for(L.n3), 256, 0, m->stream>>>(L.xx, L.yy, L.xy, L.Phi, L.b, L.r, L.z, L.n2, L.d.nz,
                                                               eps);
    MCU(cudaGetLastError());
    return mg_bc(m, L);
}

static int mg_smooth(ssg_mg* m, MgLevelDev& L, int smoother, int iters, double omega, double eps) {
    int r;
    for (int it = 0; it < iters; ++it) {
        if (smoother == 0) {
            if ((r = mg_residual(m, L, eps))) return r;
            if ((r = fwd_full(m, L, L.r, L.rspec))) return r;
            if ((r = fwd_full(m, L, L.Phi, L.spec))) return r;
            mg_spectral_update_kernel<<<blocks_for(L.c3), 256, 0, m->stream>>>(L.spec, L.rspec, L.kxf, L.kyf, L.d.N,
                                                                             L.d.nyc, L.d.nz, omega, eps);
            MCU(cudaGetLastError());
            if ((r = inv_full(m, L, L.spec, L.Phi, 0))) return r;
        } else {
            // 1 SOR, 2 enhanced (use_metrics = true, its default), 3 adaptive
            // (src/poisson.jl:597-630: SOR below a spacing ratio of 2, enhanced
            // without metrics at 0.9 omega below 5, with metrics at 0.8 omega)
            int plain = smoother == 1, metrics = smoother == 2;
            double w = omega;
            if (smoother == 3) {
                if (m->max_stretch < 2.0) plain = 1;
                else if (m->max_stretch < 5.0) w = omega * 0.9;
                else w = omega * 0.8, metrics = 1;
            }
            const int nx = L.d.N, nz = L.d.nz;
            if (nx > 2 && nz > 2) {
                dim3 grid((unsigned)((nx - 2 + 127) / 128), nx - 2, nz - 2);
                for (int color = 0; color <= 1; ++color) {
                    mg_sor_color_kernel<<<grid, 128, 0, m->stream>>>(L.Phi, L.z, nx, nx, nz, 1.0 / (L.dx * L.dx),
                                                                     1.0 / (L.dy * L.dy), w, eps, plain, metrics,
                                                                     color);
                    MCU(cudaGetLastError());
                }
            }
        }
        if ((r = mg_bc(m, L))) return r;
    }
    return SSG_OK;
}

static int mg_restrict(ssg_mg* m, MgLevelDev& C, const MgLevelDev& F) {
    mg_restrict_kernel<<<blocks_for(C.n3), 256, 0, m->stream>>>(C.Phi, F.Phi, C.d.N, C.d.N, F.d.N, F.d.N, C.d.nz);
    mg_restrict_kernel<<<blocks_for(C.n2), 256, 0, m->stream>>>(C.bs, F.bs, C.d.N, C.d.N, F.d.N, F.d.N, 1);
    MCU(cudaGetLastError());
    return SSG_OK;
}

static int mg_prolong(ssg_mg* m, MgLevelDev& F, const MgLevelDev& C) {
    mg_prolong_kernel<<<blocks_for(C.n3), 256, 0, m->stream>>>(F.Phi, C.Phi, C.d.N, C.d.N, F.d.N, F.d.N, C.d.nz);
    MCU(cudaGetLastError());
    return SSG_OK;
}

static int mg_v_cycle(ssg_mg* m, size_t level, int smoother, double omega, double eps) {
    int r;
    // coarsest level: :enhanced falls to the plain SOR smoother (src/poisson.jl:802-811)
    if (level + 1 == m->lv.size()) return mg_smooth(m, m->lv[level], smoother == 2 ? 1 : smoother, 50, omega, eps);
    MgLevelDev& cur = m->lv[level];
    MgLevelDev& crs = m->lv[level + 1];
    if ((r = mg_smooth(m, cur, smoother, 3, omega, eps))) return r;
    if ((r = mg_residual(m, cur, eps))) return r;
    if ((r = mg_restrict(m, crs, cur))) return r;
    MCU(cudaMemcpyAsync(crs.Phi_old, crs.Phi, crs.n3 * sizeof(double), cudaMemcpyDeviceToDevice, m->stream));
    MCU(cudaMemsetAsync(crs.Phi, 0, crs.n3 * sizeof(double), m->stream));
    if ((r = mg_v_cycle(m, level + 1, smoother, omega, eps))) return r;
    mg_sub_kernel<<<blocks_for(crs.n3), 256, 0, m->stream>>>(crs.Phi, crs.Phi_old, crs.n3);
    MCU(cudaGetLastError());
    if ((r = mg_prolong(m, cur, crs))) return r;
    return mg_smooth(m, cur, smoother, 3, omega, eps);
}

static int mg_norm(ssg_mg* m, const double* x, size_t n, double* out) {
    const int parts = 296;
    mg_sumsq_partial_kernel<<<parts, 256, 0, m->stream>>>(x, n, m->partials);
    mg_sum_final_kernel<<<1, 256, 0, m->stream>>>(m->partials, parts, m->sum);
    MCU(cudaGetLastError());
    double s = 0.0;
    MCU(cudaMemcpyAsync(&s, m->sum, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    MCU(cudaStreamSynchronize(m->stream));
    *out = std::sqrt(s);
    return SSG_OK;
}

static double* mg_field_ptr(MgLevelDev& L, int field, size_t* n) {
    switch (field) {
        case SSG_MG_PHI: *n = L.n3; return L.Phi;
        case SSG_MG_RHS: *n = L.n3; return L.b;
        case SSG_MG_RESIDUAL: *n = L.n3; return L.r;
        case SSG_MG_BS_SURFACE: *n = L.n2; return L.bs;
        default: *n = 0; return nullptr;
    }
}

// d2dz2! rows (src/transforms.jl:812-818) and the one-sided Neumann rows of
// apply_ssg_boundary_conditions! (src/poisson.jl:309-364) from the spacing
// vector of make_vertical_grid (src/domain.jl:238-280).  Every level has the
// same nz, so every level gets the same rows.
static ZRows mg_zrows(const std::vector<double>& dz) {
    const int nz = (int)dz.size();
    ZRows z{};
    for (int k = 0; k < nz; ++k) z.dz[k] = dz[k];
    for (int k = 1; k < nz - 1; ++k) {
        const double dzm = dz[k - 1], dzp = dz[k];
        z.al[k] = 2.0 / (dzm * (dzm + dzp));
        z.be[k] = -2.0 / (dzm * dzp);
        z.ga[k] = 2.0 / (dzp * (dzm + dzp));
    }
    const double h1 = dz[nz - 2], h2 = dz[nz - 3], a = h1 + h2;
    z.at = (2 * h1 + h2) / (h1 * a);
    z.bt = -a / (h1 * h2);
    z.ct = h1 / (h2 * a);
    const double g1 = dz[0], g2 = dz[1], ga = g1 + g2;
    z.ab = -(2 * g1 + g2) / (g1 * ga);
    z.bb = ga / (g1 * g2);
    z.cb = -g1 / (g2 * ga);
    // ssg_sor_smoother_enhanced! with metrics (src/poisson.jl:500-530, 565-575):
    // rows of 1-based planes 3..Nz-2 scaled by min(0.9, 5/ratio) where the
    // spacing ratio exceeds 5; relaxation of planes 2..Nz-1 by min(1, 3/ratio)
    // where it exceeds 3
    for (int k = 2; k <= nz - 1; ++k) {
        const double hb = dz[k - 2], ha = dz[k - 1], ht = hb + ha;
        double a = 2.0 / (hb * ht), bta = -2.0 / (hb * ha), gm = 2.0 / (ha * ht);
        const double ratio = std::max(ha, hb) / std::min(ha, hb);
        if (k > 2 && k < nz - 1 && ratio > 5.0) {
            const double sf = std::min(0.9, 5.0 / ratio);
            a *= sf;
            bta *= sf;
            gm *= sf;
        }
        z.ma[k - 1] = a;
        z.mb[k - 1] = bta;
        z.mc[k - 1] = gm;
        z.mw[k - 1] = ratio > 3.0 ? std::min(1.0, 3.0 / ratio) : 1.0;
    }
    return z;
}

// largest spacing ratio max(dz[k+1], dz[k]) / min(...) over k = 1..Nz-1
// (ssg_sor_smoother_adaptive!, src/poisson.jl:597-615)
static double mg_max_stretch(const std::vector<double>& dz) {
    double m = -INFINITY;
    for (size_t k = 0; k + 1 < dz.size(); ++k) m = std::max(m, std::max(dz[k + 1], dz[k]) / std::min(dz[k + 1], dz[k]));
    return m;
}

extern "C" int ssg_mg_create(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz, int32_t n_levels,
                             int device, ssg_mg** out) {
    if (!out) return SSG_ERR_ARG;
    *out = nullptr;
    if (nx != ny || nx < 32 || nx > 1024 || (nx & (nx - 1)) || nz < 4 || nz > 64 || n_levels < 1)
        return mg_fail(nullptr, SSG_ERR_UNSUPPORTED, "ssg_mg_create: nx == ny, power of two in [32, 1024], nz in [4, 64]");
    {
        int n = nx;
        for (int l = 1; l < n_levels; ++l) n = coarsen(n);
        if (n < 8 || (n & (n - 1))) return mg_fail(nullptr, SSG_ERR_UNSUPPORTED, "ssg_mg_create: coarsest grid below 8");
    }
    ssg_mg* m = new ssg_mg();
    m->device = device;
    auto bail = [&](int code) {
        std::string msg = m->err;
        ssg_mg_destroy(m);
        g_mg_error = msg;
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
        m->err = "ssg_mg_create: device or stream setup failed";
        return bail(SSG_ERR_CUDA);
    }
    int n = nx, r;
    const long double PI_L = 3.141592653589793238462643383279502884L;
    for (int l = 0; l < n_levels; ++l) {
        MgLevelDev L;
        L.d.N = n;
        L.d.nyc = n / 2 + 1;
        L.d.Kp = n / 3;
        L.d.Mx = 2 * L.d.Kp;
        L.d.My = L.d.nyc;
        L.d.nz = nz;
        L.n2 = (size_t)n * n;
        L.n3 = L.n2 * nz;
        L.c3 = (size_t)n * L.d.nyc * nz;
        L.dx = lx / n;
        L.dy = ly / n;
        std::vector<double2> tw(n, make_double2(1.0, 0.0));
        pass_twiddle_exponents(n, [&](int i, int e) {
            long double a = -2.0L * PI_L * (long double)e / (long double)n;
            tw[i] = make_double2((double)cosl(a), (double)sinl(a));
        });
        std::vector<double> kxf(n), kyf(L.d.nyc);
        const double mulx = (1.0 / L.dx) / n, muly = (1.0 / L.dy) / n;
        const int nnx = (n - 1) / 2 + 1;
        for (int i = 0; i < n; ++i) kxf[i] = 2.0 * M_PI * ((double)(i < nnx ? i : i - n) * mulx);
        for (int j = 0; j < L.d.nyc; ++j) kyf[j] = 2.0 * M_PI * ((double)j * muly);
        const ZRows z = mg_zrows(std::vector<double>(nz, lz / (nz - 1)));
        if ((r = mg_alloc(m, &L.tw, n)) || (r = mg_alloc(m, &L.kxf, n)) || (r = mg_alloc(m, &L.kyf, L.d.nyc)) ||
            (r = mg_alloc(m, &L.z, 1)) || (r = mg_alloc(m, &L.Phi, L.n3)) || (r = mg_alloc(m, &L.b, L.n3)) ||
            (r = mg_alloc(m, &L.r, L.n3)) || (r = mg_alloc(m, &L.Phi_old, L.n3)) || (r = mg_alloc(m, &L.bs, L.n2)) ||
            (r = mg_alloc(m, &L.xx, L.n3)) || (r = mg_alloc(m, &L.yy, L.n3)) || (r = mg_alloc(m, &L.xy, L.n3)) ||
            (r = mg_alloc(m, &L.spec, L.c3)) || (r = mg_alloc(m, &L.rspec, L.c3)) || (r = mg_alloc(m, &L.mixed, L.c3)))
            return bail(r);
        if (cudaMemcpy(L.tw, tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(L.kxf, kxf.data(), n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(L.kyf, kyf.data(), L.d.nyc * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(L.z, &z, sizeof(ZRows), cudaMemcpyHostToDevice) != cudaSuccess) {
            m->err = "ssg_mg_create: table upload failed";
            return bail(SSG_ERR_CUDA);
        }
        // SSGLevel fields start at zero (src/poisson.jl:80-110)
        cudaMemset(L.Phi, 0, L.n3 * sizeof(double));
        cudaMemset(L.b, 0, L.n3 * sizeof(double));
        cudaMemset(L.r, 0, L.n3 * sizeof(double));
        cudaMemset(L.Phi_old, 0, L.n3 * sizeof(double));
        cudaMemset(L.bs, 0, L.n2 * sizeof(double));
        m->lv.push_back(L);
        n = coarsen(n);
    }
    if ((r = mg_alloc(m, &m->partials, 296)) || (r = mg_alloc(m, &m->sum, 1))) return bail(r);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        m->err = "ssg_mg_create: initialisation failed";
        return bail(SSG_ERR_CUDA);
    }
    *out = m;
    return SSG_OK;
}

extern "C" int ssg_mg_destroy(ssg_mg* m) {
    if (!m) return SSG_OK;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (void* p : m->allocs) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return SSG_OK;
}

extern "C" int ssg_mg_level_shape(const ssg_mg* m, int32_t level, int32_t* nx, int32_t* ny, int32_t* nz) {
    if (!m || level < 0 || level >= (int)m->lv.size()) return SSG_ERR_ARG;
    if (nx) *nx = m->lv[level].d.N;
    if (ny) *ny = m->lv[level].d.N;
    if (nz) *nz = m->lv[level].d.nz;
    return SSG_OK;
}

#define MG_LEVEL_CHECK(m, level)                                                              \
    do {                                                                                      \
        if (!(m)) return SSG_ERR_ARG;                                                         \
        if ((level) < 0 || (level) >= (int)(m)->lv.size()) return mg_fail(m, SSG_ERR_ARG, "bad level"); \
        MCU(cudaSetDevice((m)->device));                                                      \
    } while (0)

extern "C" int ssg_mg_set(ssg_mg* m, int32_t level, int32_t field, const double* host, int64_t n) {
    MG_LEVEL_CHECK(m, level);
    size_t cnt = 0;
    double* p = mg_field_ptr(m->lv[level], field, &cnt);
    if (!p || !host || n != (int64_t)cnt) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_set: bad field or size");
    MCU(cudaMemcpyAsync(p, host, cnt * sizeof(double), cudaMemcpyHostToDevice, m->stream));
    MCU(cudaStreamSynchronize(m->stream));
    return SSG_OK;
}

extern "C" int ssg_mg_set_vertical_grid(ssg_mg* m, const double* dz, int32_t n) {
    if (!m) return SSG_ERR_ARG;
    if (!dz || n != m->lv[0].d.nz) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_set_vertical_grid: expected nz spacings");
    std::vector<double> v(dz, dz + n);
    for (int k = 0; k < n; ++k)
        if (!std::isfinite(v[k]) || v[k] == 0.0)
            return mg_fail(m, SSG_ERR_ARG, "ssg_mg_set_vertical_grid: spacings must be finite and non-zero");
    for (int k = 1; k < n; ++k)
        if (v[k - 1] + v[k] == 0.0) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_set_vertical_grid: adjacent spacings cancel");
    const ZRows z = mg_zrows(v);
    m->max_stretch = mg_max_stretch(v);
    MCU(cudaSetDevice(m->device));
    for (auto& L : m->lv) MCU(cudaMemcpyAsync(L.z, &z, sizeof(ZRows), cudaMemcpyHostToDevice, m->stream));
    MCU(cudaStreamSynchronize(m->stream));
    return SSG_OK;
}

extern "C" int ssg_mg_get(ssg_mg* m, int32_t level, int32_t field, double* host, int64_t n) {
    MG_LEVEL_CHECK(m, level);
    size_t cnt = 0;
    double* p = mg_field_ptr(m->lv[level], field, &cnt);
    if (!p || !host || n != (int64_t)cnt) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_get: bad field or size");
    MCU(cudaMemcpyAsync(host, p, cnt * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    MCU(cudaStreamSynchronize(m->stream));
    return SSG_OK;
}

extern "C" int ssg_mg_residual(ssg_mg* m, int32_t level, double eps) {
    MG_LEVEL_CHECK(m, level);
    int r = mg_residual(m, m->lv[level], eps);
    if (r) return r;
    MCU(cudaStreamSynchronize(m->stream));
    return SSG_OK;
}

extern "C" int ssg_mg_boundary(ssg_mg* m, int32_t level) {
    MG_LEVEL_CHECK(m, level);
    int r = mg_bc(m, m->lv[level]);
    if (r) return r;
    MCU(cudaStreamSynchronize(m->stream));
    return SSG_OK;
}

extern "C" int ssg_mg_smooth(ssg_mg* m, int32_t level, int32_t smoother, int32_t iters, double omega, double eps) {
    MG_LEVEL_CHECK(m, level);
    if (smoother < 0 || smoother > 3 || iters < 0) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_smooth: bad smoother");
    int r = mg_smooth(m, m->lv[level], smoother, iters, omega, eps);
    if (r) return r;
    MCU(cudaStreamSynchronize(m->stream));
    return SSG_OK;
}

extern "C" int ssg_mg_restrict(ssg_mg* m, int32_t coarse_level) {
    MG_LEVEL_CHECK(m, coarse_level);
    if (coarse_level < 1) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_restrict: coarse_level >= 1");
    int r = mg_restrict(m, m->lv[coarse_level], m->lv[coarse_level - 1]);
    if (r) return r;
    MCU(cudaStreamSynchronize(m->stream));
    return SSG_OK;
}

extern "C" int ssg_mg_prolongate(ssg_mg* m, int32_t coarse_level) {
    MG_LEVEL_CHECK(m, coarse_level);
    if (coarse_level < 1) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_prolongate: coarse_level >= 1");
    int r = mg_prolong(m, m->lv[coarse_level - 1], m->lv[coarse_level]);
    if (r) return r;
    MCU(cudaStreamSynchronize(m->stream));
    return SSG_OK;
}

extern "C" int ssg_mg_v_cycle(ssg_mg* m, int32_t smoother, double omega, double eps) {
    MG_LEVEL_CHECK(m, 0);
    if (smoother < 0 || smoother > 3) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_v_cycle: bad smoother");
    int r = mg_v_cycle(m, 0, smoother, omega, eps);
    if (r) return r;
    MCU(cudaStreamSynchronize(m->stream));
    return SSG_OK;
}

extern "C" int ssg_mg_norm(ssg_mg* m, int32_t level, int32_t field, double* out) {
    MG_LEVEL_CHECK(m, level);
    size_t cnt = 0;
    double* p = mg_field_ptr(m->lv[level], field, &cnt);
    if (!p || !out) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_norm: bad field");
    return mg_norm(m, p, cnt, out);
}

extern "C" int ssg_mg_solve(ssg_mg* m, double eps, double tol, int32_t maxiter, int32_t smoother, double omega,
                            int32_t* iterations, double* residual, int32_t* converged) {
    MG_LEVEL_CHECK(m, 0);
    if (smoother < 0 || smoother > 3 || maxiter < 1) return mg_fail(m, SSG_ERR_ARG, "ssg_mg_solve: bad arguments");
    double rn = 0.0;
    int r;
    for (int it = 1; it <= maxiter; ++it) {
        if ((r = mg_v_cycle(m, 0, smoother, omega, eps))) return r;
        if ((r = mg_residual(m, m->lv[0], eps))) return r;
        if ((r = mg_norm(m, m->lv[0].r, m->lv[0].n3, &rn))) return r;
        if (iterations) *iterations = it;
        if (residual) *residual = rn;
        if (rn < tol) {
            if (converged) *converged = 1;
            return SSG_OK;
        }
    }
    if (converged) *converged = 0;
    return SSG_ERR_NOT_CONVERGED;
}

extern "C" const char* ssg_mg_last_error(const ssg_mg* m) { return m ? m->err.c_str() : g_mg_error.c_str(); }
