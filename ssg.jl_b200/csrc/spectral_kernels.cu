// spectral_kernels.cu -- the hot kernels of the SSG time step on sm_100a.
//
// Every transform is split into an x-pass (rows of N contiguous complex values,
// one row per team of N/8 threads) and a y-pass (tiles of 2P adjacent
// x-columns; two real columns are packed into one complex transform of length
// N, so a c2r or r2c costs half a complex FFT per column).  The kernels fuse the
// spectral multipliers, the 2/3 mask, pointwise products and the time-stage
// updates into those passes, so every field crosses HBM once per pass.
//
// Reference operations covered (SSG.jl):
//   rfft_2d!/irfft_2d!, rfft!/irfft!   src/transforms.jl:14-56
//   ddx!/ddy!/ddx_2d!/ddy_2d!          src/transforms.jl:90-166
//   dealias!/dealias_2d!               src/domain.jl:364-379, 522-535
//   compute_d_operator!                src/poisson.jl:183-223
//   jacobian_2d!, compute_tendency!    src/transforms.jl:430-465, src/nonlinear.jl:22-56
//   AB2 / RK3 stage updates            src/timestep.jl:152-242
//   exponential filter                 src/timestep.jl:247-260, src/filter.jl:283-309
//   Neumann rows + d2dz2! operator     src/poisson.jl:262-364, src/transforms.jl:798-826
#include "kernels.cuh"
#include "fft.cuh"
#include "fft_warp.cuh"
#include "spectral_common.cuh"

#include <cudaTypedefs.h>

#include <atomic>

namespace ssg {

static std::atomic<int64_t> g_launches{0};
int64_t launch_counter() { return g_launches.load(); }
int record_launch() {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// ============================================================================
// Monge-Ampere iteration
// ============================================================================

// Interior plane zi of the mixed arrays (members one after another, nzi
// interior planes each) -> its plane in the compact spectrum, where every
// member holds nzi + 2 planes (the boundary planes included).
__device__ __forceinline__ int interior_src_plane(int zi, int nzi) {
    const int member = zi / nzi;
    return member * (nzi + 2) + 1 + (zi - member * nzi);
}

template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS, (N / 8 * ROWS) <= 128 ? 3 : 1)
    ma_xinv3_kernel(const double2* __restrict__ Phat, double2* __restrict__ A, double2* __restrict__ B,
                    double2* __restrict__ C, const double2* __restrict__ tw, const double* __restrict__ kxc, int My,
                    double scale, int nzi) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * 3 * FftShape<N>::BUF;
    const int ky = blockIdx.x * ROWS + team;
    const int zi = blockIdx.y;
    const bool active = ky < My;
    const double2* src = Phat + (size_t)Mx * (ky + (size_t)My * interior_src_plane(zi, nzi));
    const size_t o = (size_t)N * (ky + (size_t)My * zi);
    // the row is read once; its three transforms (A, B, C) run together,
    // pass by pass (fft_team_k: one twiddle load and one barrier per pass for
    // the three)
    double2 v[3][8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        bool cj;
        const int c = real_src_col<N>(t + p * T, ky, cj);
        double2 x = make_double2(0.0, 0.0);
        double kx = 0.0;
        if (active && c >= 0) {
            x = cscale(src[c], scale);
            if (cj) x = cconj(x);
            kx = cj ? -__ldg(&kxc[c]) : __ldg(&kxc[c]);
        }
        v[0][p] = cscale(x, -(kx * kx));
        v[1][p] = x;
        v[2][p] = cmul_is(x, kx);
    }
    fft_team_k<N, +1, 3>(v, t, buf, tw);
    if (active) {
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            A[o + t + p * T] = v[0][p];
            B[o + t + p * T] = v[1][p];
            C[o + t + p * T] = v[2][p];
        }
    }
}

// The running product Phi_xx Phi_yy is parked in shared memory (each thread's
// own slots, no barrier needed) rather than registers, which keeps the kernel
// under 128 registers so that four 128-thread blocks share an SM.
template <int N, int P>
__global__ void __launch_bounds__(N / 8 * P, (N / 8 * P) <= 128 ? 4 : 2)
    ma_y_kernel(const double2* __restrict__ A, const double2* __restrict__ B, const double2* __restrict__ C,
                double2* __restrict__ Dt, const double2* __restrict__ tw, const double* __restrict__ kyc, int My) {
    extern __shared__ double2 smem[];
    constexpr int T = N / 8;
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    double2* S = smem + P * FftShape<N>::BUF + (size_t)team * 8 * T;   // [8][T] per team
    const int x0 = 2 * (blockIdx.x * P + team);
    const size_t poff = (size_t)N * My * blockIdx.y;
    double2 v[8];
    // Phi_xx (both columns packed in re/im)
    load_c2r_pair<N, 0>(v, A + poff, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) S[p * T + t] = v[p];
    // Phi_yy
    load_c2r_pair<N, 1>(v, B + poff, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double2 a = S[p * T + t];
        S[p * T + t] = make_double2(a.x * v[p].x, a.y * v[p].y);
    }
    // Phi_xy and D = Phi_xx Phi_yy - Phi_xy^2
    load_c2r_pair<N, 2>(v, C + poff, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double2 a = S[p * T + t];
        v[p] = make_double2(a.x - v[p].x * v[p].x, a.y - v[p].y * v[p].y);
    }
    fft_team<N, -1>(v, t, buf, tw);
    store_r2c_pair<N>(v, buf, Dt + poff, x0, t, My);
}

template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    ma_xfwd_kernel(const double2* __restrict__ Dt, double2* __restrict__ Dh, const double2* __restrict__ tw, int My,
                   double eps, const double2* __restrict__ rhs_vol) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * 2 * FftShape<N>::BUF;
    // two rows per team (ky0, ky0 + 1), transformed together pass by pass
    const int ky0 = 2 * (blockIdx.x * ROWS + team);
    const int zi = blockIdx.y;
    double2 v[2][8];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const bool active = ky0 + r < My;
        const double2* src = Dt + (size_t)N * (ky0 + r + (size_t)My * zi);
#pragma unroll
        for (int p = 0; p < 8; ++p) v[r][p] = active ? src[t + p * T] : make_double2(0.0, 0.0);
    }
    fft_team_k<N, -1, 2>(v, t, buf, tw);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int ky = ky0 + r;
        if (ky >= My) continue;
        double2* dst = Dh + (size_t)Mx * (ky + (size_t)My * zi);
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            const int c = compact_col<N>(t + p * T);
            if (c >= 0) {
                double2 val = cscale(v[r][p], eps);
                if (rhs_vol) val = cadd(val, rhs_vol[c + (size_t)Mx * ky]);
                dst[c] = val;
            }
        }
    }
}


// One thread per compact mode: tridiagonal solve along z of
//   al Phi[k-1] + (be - K^2) Phi[k] + ga Phi[k+1] = R[k]   (interior k)
// with the Neumann rows eliminated (bottom: ab P0 + bb P1 + cb P2 = 0,
// top: at Pn + bt Pn-1 + ct Pn-2 = bc), in the same operation order as the
// CPU restatement.
//
// The matrix of a mode depends only on K^2 and the vertical rows, so its
// pivot reciprocals inv_q = 1 / (dg_q - lo_q c_{q-1}) (c_q = up_q inv_q) are
// computed once per grid by ma_thomas_factor_kernel, with the same
// expressions as the elimination would use, and stored plane-major
// [q][mode].  The solve is then a chain of multiply-adds per level.

// rows of interior level q (0-based, plane q+1) after the Neumann rows are
// eliminated: lower, diagonal without -K^2, upper
__device__ __forceinline__ void thomas_level(const ZOps* __restrict__ zo, int q, int n, double& lo, double& dg0,
                                             double& up) {
    const int k = q + 1;
    lo = zo->al[k];
    dg0 = zo->be[k];
    up = zo->ga[k];
    if (q == 0) {
        lo = 0.0;
        up -= zo->al[k] * zo->cb / zo->ab;
    }
    if (q == n - 1) {
        lo -= zo->ga[k] * zo->ct / zo->at;
        up = 0.0;
    }
}

template <int TB>
__global__ void __launch_bounds__(TB)
    ma_thomas_factor_kernel(const double* __restrict__ kxc, const double* __restrict__ kyc,
                            const ZOps* __restrict__ zo, int Mx, int My, int nz, double* __restrict__ inv_out) {
    const int n = nz - 2;
    // one thread per entry of a level of the pivot table (pivot_of): column
    // c <= Kp of row j, whose K^2 its mirror column shares
    const size_t M = pivot_plane(Mx, My);
    const size_t m = (size_t)blockIdx.x * TB + threadIdx.x;
    if (m >= M || m == 0) return;
    const int c = (int)(m % (Mx / 2 + 1)), j = (int)(m / (Mx / 2 + 1));
    const double kx = kxc[c], ky = kyc[j];
    const double K2 = kx * kx + ky * ky;
    double cprev = 0.0;
    for (int q = 0; q < n; ++q) {
        const int k = q + 1;
        double lo = zo->al[k], dg = zo->be[k] - K2, up = zo->ga[k];
        if (q == 0) {
            dg -= zo->al[k] * zo->bb / zo->ab;
            up -= zo->al[k] * zo->cb / zo->ab;
            lo = 0.0;
        }
        if (q == n - 1) {
            lo -= zo->ga[k] * zo->ct / zo->at;
            dg -= zo->ga[k] * zo->bt / zo->at;
            up = 0.0;
        }
        const double inv = (q == 0) ? 1.0 / dg : 1.0 / (dg - lo * cprev);
        inv_out[m + M * q] = inv;
        cprev = up * inv;
    }
}

// The whole z-column of every mode of the block (right-hand side, pivot
// reciprocals and old solution) is copied to shared memory with cp.async at
// entry, so all of the block's loads are in flight at once; the sweeps then
// run from shared memory.  Each thread only reads back its own column, so the
// copies need no block barrier, only the thread's own wait.
template <int TB>
__global__ void __launch_bounds__(TB)
    ma_thomas_kernel(const double2* __restrict__ Dh, const double2* __restrict__ bc_top, double2* __restrict__ Phat,
                     const double* __restrict__ inv, const ZOps* __restrict__ zo, int Mx, int My, int nz,
                     double* partials, unsigned int* ticket, double* norms, const unsigned int* __restrict__ active) {
    extern __shared__ double2 tsm2[];
    __shared__ double slo[64], sup[64];
    const int n = nz - 2;
    // member blockIdx.y: its planes, buoyancy and norm reduction; a member
    // whose solve has stopped is left as it is
    {
        const size_t mb = blockIdx.y, Mm = (size_t)Mx * My;
        if (active && !active[mb]) return;
        Dh += mb * n * Mm;
        Phat += mb * nz * Mm;
        if (bc_top) bc_top += mb * Mm;
        partials += mb * 2 * gridDim.x;
        ticket += mb;
        norms += 2 * mb;
    }
    double2* sd = tsm2;                                                     // [n][TB]: rhs, then dp, then x
    double2* so = tsm2 + (size_t)n * TB;                                    // [nz][TB]: old solution
    double* si = reinterpret_cast<double*>(tsm2 + (size_t)(n + nz) * TB);  // [n][TB]: pivot reciprocals
    const int tid = threadIdx.x;
    for (int q = tid; q < n; q += TB) {
        double lo, dg0, up;
        thomas_level(zo, q, n, lo, dg0, up);
        slo[q] = lo;
        sup[q] = up;
    }
    __syncthreads();
    const size_t M = (size_t)Mx * My;
    const size_t m = (size_t)blockIdx.x * TB + tid;
    double ds = 0.0, ns = 0.0;
    if (m < M) {
        for (int q = 0; q < n; ++q) {
            cp_async16(&sd[q * TB + tid], &Dh[m + M * q]);
            cp_async8(&si[q * TB + tid], &inv[pivot_of(m, Mx) + pivot_plane(Mx, My) * q]);
        }
        cp_async_commit();
        for (int k = 0; k < nz; ++k) cp_async16(&so[k * TB + tid], &Phat[m + M * k]);
        cp_async_commit();
        const int c = (int)(m % Mx), j = (int)(m / Mx);
        // Parseval weight: modes with ky > 0 and (-N/3, 0) stand for two modes
        const double w = (j == 0 && c != Mx / 2) ? 1.0 : 2.0;
        const double2 bc = bc_top ? bc_top[m] : make_double2(0.0, 0.0);
        const double ab = zo->ab, bb = zo->bb, cb = zo->cb, at = zo->at, bt = zo->bt, ct = zo->ct;
        const double ftop = zo->ga[n];
        cp_async_wait<1>();
        if (m == 0) {
            cp_async_wait<0>();
            for (int k = 0; k < nz; ++k) {
                const double2 old = so[k * TB + tid];
                ds += w * (old.x * old.x + old.y * old.y);
                Phat[m + M * k] = make_double2(0.0, 0.0);
            }
        } else {
            double2 dprev = make_double2(0.0, 0.0);
            for (int q = 0; q < n; ++q) {
                double2 r = sd[q * TB + tid];
                const double iv = si[q * TB + tid];
                if (q == n - 1) r = make_double2(r.x - ftop * bc.x / at, r.y - ftop * bc.y / at);
                double2 dq;
                if (q == 0) {
                    dq = cscale(r, iv);
                } else {
                    const double lo = slo[q];
                    dq = cscale(make_double2(r.x - lo * dprev.x, r.y - lo * dprev.y), iv);
                }
                sd[q * TB + tid] = dq;
                dprev = dq;
            }
            double2 x = dprev;
            for (int q = n - 2; q >= 0; --q) {
                const double cq = sup[q] * si[q * TB + tid];
                const double2 d = sd[q * TB + tid];
                x = make_double2(d.x - cq * x.x, d.y - cq * x.y);
                sd[q * TB + tid] = x;
            }
            const double2 x0 = sd[tid], x1 = sd[TB + tid];
            const double2 xn1 = sd[(n - 1) * TB + tid], xn2 = sd[(n - 2) * TB + tid];
            const double2 p0 = make_double2(-(bb * x0.x + cb * x1.x) / ab, -(bb * x0.y + cb * x1.y) / ab);
            const double2 pt = make_double2((bc.x - bt * xn1.x - ct * xn2.x) / at, (bc.y - bt * xn1.y - ct * xn2.y) / at);
            cp_async_wait<0>();
            for (int k = 0; k < nz; ++k) {
                const double2 nv = (k == 0) ? p0 : (k == nz - 1) ? pt : sd[(k - 1) * TB + tid];
                const double2 old = so[k * TB + tid];
                const double dx = nv.x - old.x, dy = nv.y - old.y;
                ds += w * (dx * dx + dy * dy);
                ns += w * (nv.x * nv.x + nv.y * nv.y);
                Phat[m + M * k] = nv;
            }
        }
    }
    block_reduce_pair<TB>(ds, ns, partials, ticket, norms);
}

// The same solve for a compile-time depth NZ: each thread loads its mode's
// right-hand side and pivot reciprocals into registers with plain loads issued
// at entry, and copies the old solution to shared memory with cp.async (read
// back only for the update norm); the loops unroll.  At NZ = 32 a thread holds
// its column in about 250 registers without spilling, so 8 warps share an SM,
// where the staged kernel's 40 bytes of shared memory per level per thread
// allow 5; the unrolled sweeps also drop the index arithmetic and the
// per-level branches (0.122 -> 0.087 ms at 1024^2 x 32 in one-warp blocks).  Capping the
// registers at 168 for 12 blocks per SM spilled and was slower.  Same
// operations in the same order as ma_thomas_kernel, so the results are
// bit-identical.
// Right-hand side of one level: FP64 as stored, or eps times the FP32 x-forward
// transform -- the same rounded FP64 product ma_xfwd_mp_kernel would have
// stored (__dmul_rn: never contracted into the elimination's multiply-adds).
__device__ __forceinline__ double2 rhs_value(const double2 v, double) { return v; }
__device__ __forceinline__ double2 rhs_value(const float2 v, double eps) {
    return make_double2(__dmul_rn(eps, (double)v.x), __dmul_rn(eps, (double)v.y));
}

template <int TB, int NZ, typename RHS>
__global__ void __launch_bounds__(TB)
    ma_thomas_reg_kernel(const RHS* __restrict__ Dh, const double2* __restrict__ bc_top, double2* __restrict__ Phat,
                         const double* __restrict__ inv, const ZOps* __restrict__ zo, int Mx, int My,
                         double* partials, unsigned int* ticket, double* norms,
                         const unsigned int* __restrict__ active, double eps) {
    constexpr int n = NZ - 2;
    __shared__ double slo[n], sup[n];
    __shared__ double2 so[NZ][TB];
    const int tid = threadIdx.x;
    {
        const size_t mb = blockIdx.y, Mm = (size_t)Mx * My;
        if (active && !active[mb]) return;
        Dh += mb * n * Mm;
        Phat += mb * NZ * Mm;
        if (bc_top) bc_top += mb * Mm;
        partials += mb * 2 * gridDim.x;
        ticket += mb;
        norms += 2 * mb;
    }
    for (int q = tid; q < n; q += TB) {
        double lo, dg0, up;
        thomas_level(zo, q, n, lo, dg0, up);
        slo[q] = lo;
        sup[q] = up;
    }
    const size_t M = (size_t)Mx * My;
    const size_t m = (size_t)blockIdx.x * TB + tid;
    double ds = 0.0, ns = 0.0;
    double2 x[n];
    double iv[n];
    if (m < M) {
#pragma unroll
        for (int k = 0; k < NZ; ++k) cp_async16(&so[k][tid], &Phat[m + M * k]);
        cp_async_commit();
#pragma unroll
        for (int q = 0; q < n; ++q) {
            x[q] = rhs_value(Dh[m + M * q], eps);
            iv[q] = inv[pivot_of(m, Mx) + pivot_plane(Mx, My) * q];
        }
    }
    __syncthreads();
    if (m < M) {
        const int c = (int)(m % Mx), j = (int)(m / Mx);
        const double w = (j == 0 && c != Mx / 2) ? 1.0 : 2.0;
        const double2 bc = bc_top ? bc_top[m] : make_double2(0.0, 0.0);
        if (m == 0) {
            cp_async_wait<0>();
#pragma unroll
            for (int k = 0; k < NZ; ++k) {
                const double2 old = so[k][tid];
                ds += w * (old.x * old.x + old.y * old.y);
                Phat[m + M * k] = make_double2(0.0, 0.0);
            }
        } else {
            const double ab = zo->ab, bb = zo->bb, cb = zo->cb, at = zo->at, bt = zo->bt, ct = zo->ct;
            const double ftop = zo->ga[n];
            x[n - 1] = make_double2(x[n - 1].x - ftop * bc.x / at, x[n - 1].y - ftop * bc.y / at);
            x[0] = cscale(x[0], iv[0]);
#pragma unroll
            for (int q = 1; q < n; ++q) {
                const double lo = slo[q];
                x[q] = cscale(make_double2(x[q].x - lo * x[q - 1].x, x[q].y - lo * x[q - 1].y), iv[q]);
            }
#pragma unroll
            for (int q = n - 2; q >= 0; --q) {
                const double cq = sup[q] * iv[q];
                x[q] = make_double2(x[q].x - cq * x[q + 1].x, x[q].y - cq * x[q + 1].y);
            }
            const double2 p0 = make_double2(-(bb * x[0].x + cb * x[1].x) / ab, -(bb * x[0].y + cb * x[1].y) / ab);
            const double2 pt = make_double2((bc.x - bt * x[n - 1].x - ct * x[n - 2].x) / at,
                                            (bc.y - bt * x[n - 1].y - ct * x[n - 2].y) / at);
            cp_async_wait<0>();
#pragma unroll
            for (int k = 0; k < NZ; ++k) {
                const double2 nv = (k == 0) ? p0 : (k == NZ - 1) ? pt : x[k - 1];
                const double2 old = so[k][tid];
                const double dx = nv.x - old.x, dy = nv.y - old.y;
                ds += w * (dx * dx + dy * dy);
                ns += w * (nv.x * nv.x + nv.y * nv.y);
                Phat[m + M * k] = nv;
            }
        }
    }
    block_reduce_pair<TB>(ds, ns, partials, ticket, norms);
}



// ============================================================================
// Mixed-precision Monge-Ampere passes: the transforms and the product D run in
// FP32 (float2 intermediates, half the bytes); the potential Phat and the
// right-hand side Dh the tridiagonal solve reads stay FP64.
// ============================================================================

template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS, (N / 8 * ROWS) <= 128 ? 4 : 2)
    ma_xinv3_mp_kernel(const double2* __restrict__ Phat, float2* __restrict__ A, float2* __restrict__ B,
                       float2* __restrict__ Cc, const float2* __restrict__ tw, const double* __restrict__ kxc, int My,
                       double scale, int nzi) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    extern __shared__ float2 smem32[];
    const int t = threadIdx.x, team = threadIdx.y;
    float2* buf = smem32 + team * 3 * FftShape<N>::BUF;
    const int ky = blockIdx.x * ROWS + team;
    const int zi = blockIdx.y;
    const bool active = ky < My;
    const double2* src = Phat + (size_t)Mx * (ky + (size_t)My * interior_src_plane(zi, nzi));
    const size_t o = (size_t)N * (ky + (size_t)My * zi);
    // the row is read once; its three transforms (A, B, C) run together, pass
    // by pass, so each pass loads its twiddles and synchronises once for all
    // three (fft_team_k)
    float2 v[3][8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        bool cj;
        const int c = real_src_col<N>(t + p * T, ky, cj);
        double2 x = make_double2(0.0, 0.0);
        double kx = 0.0;
        if (active && c >= 0) {
            x = cscale(src[c], scale);
            if (cj) x = cconj(x);
            kx = cj ? -__ldg(&kxc[c]) : __ldg(&kxc[c]);
        }
        const double2 xa = cscale(x, -(kx * kx)), xc = cmul_is(x, kx);
        v[0][p] = make_float2((float)xa.x, (float)xa.y);
        v[1][p] = make_float2((float)x.x, (float)x.y);
        v[2][p] = make_float2((float)xc.x, (float)xc.y);
    }
    fft_team_k<N, +1, 3>(v, t, buf, tw);
    if (active) {
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            A[o + t + p * T] = v[0][p];
            B[o + t + p * T] = v[1][p];
            Cc[o + t + p * T] = v[2][p];
        }
    }
}

template <int N, int P>
__global__ void __launch_bounds__(N / 8 * P, (N / 8 * P) <= 128 ? 4 : 2)
    ma_y_mp_kernel(const float2* __restrict__ A, const float2* __restrict__ B, const float2* __restrict__ Cc,
                   float2* __restrict__ Dt, const float2* __restrict__ tw, const double* __restrict__ kyc, int My) {
    extern __shared__ float2 smem32[];
    const int t = threadIdx.x, team = threadIdx.y;
    float2* buf = smem32 + team * FftShape<N>::BUF;
    const int x0 = 2 * (blockIdx.x * P + team);
    const size_t poff = (size_t)N * My * blockIdx.y;
    float2 v[8], S[8];
    load_c2r_pair<N, 0>(v, A + poff, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) S[p] = v[p];
    load_c2r_pair<N, 1>(v, B + poff, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) S[p] = make_float2(S[p].x * v[p].x, S[p].y * v[p].y);
    load_c2r_pair<N, 2>(v, Cc + poff, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = make_float2(S[p].x - v[p].x * v[p].x, S[p].y - v[p].y * v[p].y);
    fft_team<N, -1>(v, t, buf, tw);
    store_r2c_pair<N>(v, buf, Dt + poff, x0, t, My);
}

template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    ma_xfwd_mp_kernel(const float2* __restrict__ Dt, double2* __restrict__ Dh, const float2* __restrict__ tw, int My,
                      double eps, const double2* __restrict__ rhs_vol, float2* __restrict__ dh32) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    extern __shared__ float2 smem32[];
    const int t = threadIdx.x, team = threadIdx.y;
    float2* buf = smem32 + team * 2 * FftShape<N>::BUF;
    // two rows per team (ky0, ky0 + 1), transformed together pass by pass
    const int ky0 = 2 * (blockIdx.x * ROWS + team);
    const int zi = blockIdx.y;
    float2 v[2][8];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const bool active = ky0 + r < My;
        const float2* src = Dt + (size_t)N * (ky0 + r + (size_t)My * zi);
#pragma unroll
        for (int p = 0; p < 8; ++p) v[r][p] = active ? src[t + p * T] : make_float2(0.f, 0.f);
    }
    fft_team_k<N, -1, 2>(v, t, buf, tw);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int ky = ky0 + r;
        if (ky >= My) continue;
        if (dh32) {
            // the FP32 transform itself: the vertical solve forms eps * v in
            // FP64 as it loads it (ma_thomas_reg_kernel with a float2 right-hand side)
            float2* dst = dh32 + (size_t)Mx * (ky + (size_t)My * zi);
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                const int c = compact_col<N>(t + p * T);
                if (c >= 0) dst[c] = v[r][p];
            }
        } else {
            double2* dst = Dh + (size_t)Mx * (ky + (size_t)My * zi);
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                const int c = compact_col<N>(t + p * T);
                if (c >= 0) {
                    double2 val = make_double2(eps * (double)v[r][p].x, eps * (double)v[r][p].y);
                    if (rhs_vol) val = cadd(val, rhs_vol[c + (size_t)Mx * ky]);
                    dst[c] = val;
                }
            }
        }
    }
}

// ============================================================================
// TMA / mbarrier helpers (sm_90+ PTX)
// ============================================================================

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// The dynamic shared memory array advanced to the next multiple of A bytes,
// by pointer arithmetic on the array itself: the compiler keeps knowing that
// the result (and every pointer derived from it) is shared memory, so its
// loads and stores are LDS/STS (a round trip through an integer would turn
// them into generic accesses).
template <unsigned A>
__device__ __forceinline__ unsigned char* smem_align(unsigned char* raw) {
    return raw + ((A - (smem_u32(raw) & (A - 1))) & (A - 1));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait: gives up after `limit` polls (each poll may suspend the warp
// for a hardware-defined interval) and reports failure instead of hanging.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int limit) {
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int c0, int c1, int c2, const void* src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(map),
                 "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(src))
                 : "memory");
}
__device__ __forceinline__ void tma_store_commit_wait() {
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}

constexpr int kTmaWaitLimit = 1 << 22;

// ---- persistent, TMA-pipelined FP64 y-pass ----------------------------------
// Tiles are 4 double2 columns x My rows: 64-byte rows, 64B swizzle (the
// 16-byte chunk index is XORed with (row/2) mod 4), so that the 32 lanes of a
// warp reading one column of 32 consecutive rows hit distinct banks.  A block
// is two teams of N/8 threads (one packed column pair each).  At N = 1024 one
// block holds an SM with the full register file (a transform, the staged
// values and the loop state need about 250 registers per thread; at 128 they
// spill, which measured 20% slower); below, two blocks share an SM.  Each block loops over (x-tile, plane) items through two tile slots
// used as a ring: item i reads A from slot s = i mod 2 and B from s^1; C is
// loaded into s as soon as A has been read, and after C has been read slot s
// stages the output tile for the TMA store.  The next item's A goes into s^1
// once B has been read and its B into s once the store has read the tile, so
// every load overlaps at least one transform.  The running product
// Phi_xx Phi_yy is parked in shared memory (each thread's own slots); inside
// the transforms the teams synchronise only among themselves.
__device__ __forceinline__ double2* swz64d(unsigned char* tile, int r, int col) {
    return reinterpret_cast<double2*>(tile + (size_t)r * 64 + ((col ^ ((r >> 1) & 3)) << 4));
}

// Packed spectrum of columns (2*team, 2*team+1) of a staged tile with
// multiplier MULT, Hermitian-extended (see load_c2r_pair).
template <int N, int MULT>
__device__ __forceinline__ void tile_c2r_pair(double2 (&v)[8], unsigned char* tile, int team, int t, int My,
                                              const double* __restrict__ kyc) {
    constexpr int T = N / 8;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int k = t + p * T;
        int kk = -1;
        bool ext = false;
        if (k < My) {
            kk = k;
        } else if (k > N / 2 && N - k < My) {
            kk = N - k;
            ext = true;
        }
        double2 a = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
        if (kk >= 0) {
            a = *swz64d(tile, kk, 2 * team);
            b = *swz64d(tile, kk, 2 * team + 1);
            if constexpr (MULT == 1) {
                const double ky = __ldg(&kyc[kk]);
                const double m = -(ky * ky);
                a = cscale(a, m);
                b = cscale(b, m);
            } else if constexpr (MULT == 2) {
                const double ky = __ldg(&kyc[kk]);
                a = cmul_is(a, ky);
                b = cmul_is(b, ky);
            }
            if (ext) {
                a = cconj(a);
                b = cconj(b);
            }
            if (k == 0) {
                a.y = 0.0;
                b.y = 0.0;
            }
        }
        v[p] = make_double2(a.x - b.y, a.y + b.x);
    }
}

// Tile loads of one block: slot j (0, 1) at base + j*bytes completes one
// phase of full[j] per load; bit j of ph is the parity of the next phase to
// wait for.  (No arrays indexed by the slot number: they would live in local
// memory.)
struct YTiles {
    unsigned char* base;
    uint64_t* full;
    unsigned ph;
    int box_rows, xtiles;
    int rowb;   // bytes per tile row
    int cstep;  // tensor elements per tile row (the x step between items)
    unsigned bytes;
    __device__ __forceinline__ unsigned char* slot(int j) const { return base + (size_t)j * bytes; }
    __device__ __forceinline__ void load(int j, const CUtensorMap* map, int item) const {
        const int c0 = (item % xtiles) * cstep, plane = item / xtiles;
        mbar_expect_tx(full + j, bytes);
        tma_load_3d(slot(j), map, c0, 0, plane, full + j);
        tma_load_3d(slot(j) + (size_t)box_rows * rowb, map, c0, box_rows, plane, full + j);
    }
    // every thread of the block calls this; false when the wait gave up
    __device__ __forceinline__ bool wait(int j) {
        const bool ok = mbar_wait_bounded(full + j, (ph >> j) & 1u, kTmaWaitLimit);
        ph ^= 1u << j;
        return !__syncthreads_or(!ok);
    }
};

template <int N, typename SYNC>
__device__ __forceinline__ bool ma_y_tma_item(YTiles& yt, const CUtensorMap* tA, const CUtensorMap* tB,
                                              const CUtensorMap* tC, const CUtensorMap* tD, double2* buf,
                                              double2* St, int team, int t, int tid, int My, int w, int next,
                                              int nitems, int sa, const double2* __restrict__ tw,
                                              const double* __restrict__ kyc, const SYNC& sync) {
    constexpr int T = N / 8;
    const int sb = sa ^ 1;
    double2 v[8];
    // Phi_xx from slot sa; then C of this item into sa
    if (!yt.wait(sa)) return false;
    tile_c2r_pair<N, 0>(v, yt.slot(sa), team, t, My, kyc);
    __syncthreads();  // both teams hold their values
    if (tid == 0) {
        fence_proxy_async();
        yt.load(sa, tC, w);
    }
    fft_team<N, +1>(v, t, buf, tw, sync);
#pragma unroll
    for (int p = 0; p < 8; ++p) St[p * T + t] = v[p];
    // Phi_yy from slot sb; then A of the next item into sb
    if (!yt.wait(sb)) return false;
    tile_c2r_pair<N, 1>(v, yt.slot(sb), team, t, My, kyc);
    __syncthreads();
    if (tid == 0 && next < nitems) {
        fence_proxy_async();
        yt.load(sb, tA, next);
    }
    fft_team<N, +1>(v, t, buf, tw, sync);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double2 a = St[p * T + t];
        St[p * T + t] = make_double2(a.x * v[p].x, a.y * v[p].y);
    }
    // Phi_xy from slot sa and D = Phi_xx Phi_yy - Phi_xy^2
    if (!yt.wait(sa)) return false;
    tile_c2r_pair<N, 2>(v, yt.slot(sa), team, t, My, kyc);
    __syncthreads();  // slot sa is read: it becomes the output tile
    fft_team<N, +1>(v, t, buf, tw, sync);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double2 a = St[p * T + t];
        v[p] = make_double2(a.x - v[p].x * v[p].x, a.y - v[p].y * v[p].y);
    }
    fft_team<N, -1>(v, t, buf, tw, sync);
    // split the packed transform into the two half spectra, rows ky < My
    sync();
#pragma unroll
    for (int p = 0; p < 8; ++p) buf[fpad<double2>(t + p * T)] = v[p];
    sync();
    unsigned char* out = yt.slot(sa);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int k = t + p * T;
        if (k < My) {
            const double2 z = buf[fpad<double2>(k)];
            const double2 zm = buf[fpad<double2>((N - k) & (N - 1))];
            *swz64d(out, k, 2 * team) = make_double2(0.5 * (z.x + zm.x), 0.5 * (z.y - zm.y));
            *swz64d(out, k, 2 * team + 1) = make_double2(0.5 * (z.y + zm.y), -0.5 * (z.x - zm.x));
        }
    }
    fence_proxy_async();
    __syncthreads();  // the output tile is complete
    if (tid == 0) {
        const int c0 = (w % yt.xtiles) * yt.cstep, plane = w / yt.xtiles;
        tma_store_3d(tD, c0, 0, plane, out);
        if (yt.box_rows < My) tma_store_3d(tD, c0, yt.box_rows, plane, out + (size_t)yt.box_rows * yt.rowb);
        tma_store_commit_wait();  // the tile has been read out: slot sa takes the next item's B
        if (next < nitems) yt.load(sa, tB, next);
    }
    return true;
}

template <int N>
__global__ void __launch_bounds__(N / 4, (N >= 1024 ? 1 : 2))
    ma_y_tma_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB,
                    const __grid_constant__ CUtensorMap tC, const __grid_constant__ CUtensorMap tD,
                    const double2* __restrict__ tw, const double* __restrict__ kyc, int My, int box_rows,
                    int xtiles, int nitems, unsigned int* errflag) {
    constexpr int T = N / 8;
    extern __shared__ unsigned char ysm_raw[];
    unsigned char* base = smem_align<512>(ysm_raw);
    __shared__ __align__(8) uint64_t full[2];
    const int t = threadIdx.x, team = threadIdx.y;
    const int tid = team * T + t;
    YTiles yt;
    yt.bytes = (unsigned)(2 * box_rows * 64);
    yt.base = base;
    yt.full = full;
    yt.ph = 0u;
    yt.box_rows = box_rows;
    yt.xtiles = xtiles;
    yt.rowb = 64;
    yt.cstep = 8;
    double2* buf = reinterpret_cast<double2*>(base + 2 * yt.bytes) + team * FftShape<N>::BUF;
    double2* St = reinterpret_cast<double2*>(base + 2 * yt.bytes) + 2 * FftShape<N>::BUF + (size_t)team * 8 * T;
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0 && (int)blockIdx.x < nitems) {
        yt.load(0, &tA, blockIdx.x);
        yt.load(1, &tB, blockIdx.x);
    }
    int i = 0;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x, ++i) {
        const int next = w + (int)gridDim.x;
        bool ok;
        if constexpr (T >= 32)
            ok = ma_y_tma_item<N>(yt, &tA, &tB, &tC, &tD, buf, St, team, t, tid, My, w, next, nitems, i & 1, tw, kyc,
                                  TeamSync{team + 1, T});
        else
            ok = ma_y_tma_item<N>(yt, &tA, &tB, &tC, &tD, buf, St, team, t, tid, My, w, next, nitems, i & 1, tw, kyc,
                                  BlockSync{});
        if (!ok) {
            if (tid == 0) {
                atomicOr(errflag, 1u);
                asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
            }
            return;
        }
    }
}

// ---- persistent, TMA-pipelined FP32 y-pass (mixed precision) --------------
// Tiles are 8 float2 columns x My rows (64-byte rows, 64B swizzle: the
// 16-byte chunk index is XORed with (row/2) mod 4).  Each block loops over
// (x-tile, plane) items; two tile sets let the three inputs of item i+1 load
// while item i is transformed.  The four teams of a block (one column pair
// each) synchronise only among themselves inside the transforms.
// The 16-byte chunk of row r holding columns (2*pair, 2*pair+1).  A warp
// reading one pair from 32 consecutive rows with 16-byte accesses touches
// every bank group evenly; two 8-byte accesses per row would conflict 4-way.
__device__ __forceinline__ float4* swz64_pair(unsigned char* tile, int r, int pair) {
    return reinterpret_cast<float4*>(tile + (size_t)r * 64 + ((pair ^ ((r >> 1) & 3)) << 4));
}

template <int N, int MULT>
__device__ __forceinline__ void tile64_c2r_pair(float2 (&v)[8], unsigned char* tile, int team, int t, int My,
                                                const double* __restrict__ kyc) {
    constexpr int T = N / 8;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int k = t + p * T;
        int kk = -1;
        bool ext = false;
        if (k < My) {
            kk = k;
        } else if (k > N / 2 && N - k < My) {
            kk = N - k;
            ext = true;
        }
        float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
        if (kk >= 0) {
            const float4 ab = *swz64_pair(tile, kk, team);
            a = make_float2(ab.x, ab.y);
            b = make_float2(ab.z, ab.w);
            if constexpr (MULT == 1) {
                const float ky = (float)__ldg(&kyc[kk]);
                const float m = -(ky * ky);
                a = cscale(a, m);
                b = cscale(b, m);
            } else if constexpr (MULT == 2) {
                const float ky = (float)__ldg(&kyc[kk]);
                a = cmul_is(a, ky);
                b = cmul_is(b, ky);
            }
            if (ext) {
                a = cconj(a);
                b = cconj(b);
            }
            if (k == 0) {
                a.y = 0.f;
                b.y = 0.f;
            }
        }
        v[p] = make_float2(a.x - b.y, a.y + b.x);
    }
}

template <int N, typename SYNC>
__device__ __forceinline__ void ma_y_mp_item(unsigned char* tA, unsigned char* tB, unsigned char* tC,
                                             unsigned char* tout, float2* buf, int team, int t, int My,
                                             const float2* __restrict__ tw, const double* __restrict__ kyc,
                                             const SYNC& sync) {
    constexpr int T = N / 8;
    float2 v[8], S[8];
    tile64_c2r_pair<N, 0>(v, tA, team, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw, sync);
#pragma unroll
    for (int p = 0; p < 8; ++p) S[p] = v[p];
    tile64_c2r_pair<N, 1>(v, tB, team, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw, sync);
#pragma unroll
    for (int p = 0; p < 8; ++p) S[p] = make_float2(S[p].x * v[p].x, S[p].y * v[p].y);
    tile64_c2r_pair<N, 2>(v, tC, team, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw, sync);
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = make_float2(S[p].x - v[p].x * v[p].x, S[p].y - v[p].y * v[p].y);
    fft_team<N, -1>(v, t, buf, tw, sync);
    sync();
#pragma unroll
    for (int p = 0; p < 8; ++p) buf[fpad<float2>(t + p * T)] = v[p];
    sync();
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int k = t + p * T;
        if (k < My) {
            const float2 z = buf[fpad<float2>(k)];
            const float2 zm = buf[fpad<float2>((N - k) & (N - 1))];
            *swz64_pair(tout, k, team) =
                make_float4(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y), 0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
        }
    }
}

// teams per block of the FP32 y-pass: four (one column pair each), or two at
// N = 1024, where each team takes two pairs in turn so that a thread may hold
// the ~200 registers a transform with its staged values needs (four teams of
// 128 threads cap it at 128 registers, which spill)
template <int N>
constexpr int mp_y_teams() { return N >= 1024 ? 2 : 4; }

template <int N>
__global__ void __launch_bounds__(N / 8 * mp_y_teams<N>(), 1)
    ma_y_mp_tma_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB,
                       const __grid_constant__ CUtensorMap tC, const __grid_constant__ CUtensorMap tD,
                       const float2* __restrict__ tw, const double* __restrict__ kyc, int My, int box_rows, int xtiles,
                       int nitems, unsigned int* errflag) {
    constexpr int T = N / 8;
    extern __shared__ unsigned char ysm_raw[];
    unsigned char* base = smem_align<1024>(ysm_raw);
    const size_t tb_bytes = (size_t)2 * box_rows * 64;   // one input tile: two boxes
    unsigned char* tiles = base;                          // [set 0..1][input 0..2]
    unsigned char* tout = base + 6 * tb_bytes;
    float2* bufs = reinterpret_cast<float2*>(tout + tb_bytes);
    __shared__ __align__(8) uint64_t full[2];
    const int t = threadIdx.x, team = threadIdx.y;
    const int tid = team * T + t;
    float2* buf = bufs + team * FftShape<N>::BUF;
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int item, int set) {
        const int c0 = (item % xtiles) * 16, plane = item / xtiles;
        mbar_expect_tx(&full[set], (unsigned)(3 * tb_bytes));
        const CUtensorMap* maps[3] = {&tA, &tB, &tC};
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            unsigned char* dst = tiles + (size_t)(set * 3 + j) * tb_bytes;
            tma_load_3d(dst, maps[j], c0, 0, plane, &full[set]);
            tma_load_3d(dst + (size_t)box_rows * 64, maps[j], c0, box_rows, plane, &full[set]);
        }
    };
    if (tid == 0) {
        if ((int)blockIdx.x < nitems) issue(blockIdx.x, 0);
        if ((int)(blockIdx.x + gridDim.x) < nitems) issue(blockIdx.x + gridDim.x, 1);
    }
    int i = 0;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x, ++i) {
        const int set = i & 1;
        const bool ok = mbar_wait_bounded(&full[set], (unsigned)((i >> 1) & 1), kTmaWaitLimit);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(errflag, 1u);
            return;
        }
        unsigned char* ts = tiles + (size_t)set * 3 * tb_bytes;
#pragma unroll 1
        for (int pair = team; pair < 4; pair += mp_y_teams<N>()) {
            if constexpr (T >= 32) {
                ma_y_mp_item<N>(ts, ts + tb_bytes, ts + 2 * tb_bytes, tout, buf, pair, t, My, tw, kyc,
                                TeamSync{team + 1, T});
            } else {
                ma_y_mp_item<N>(ts, ts + tb_bytes, ts + 2 * tb_bytes, tout, buf, pair, t, My, tw, kyc, BlockSync{});
            }
        }
        fence_proxy_async();
        __syncthreads();  // this set's tiles are consumed and the output tile is complete
        if (tid == 0) {
            const int c0 = (w % xtiles) * 16, plane = w / xtiles;
            tma_store_3d(&tD, c0, 0, plane, tout);
            if (box_rows < My) tma_store_3d(&tD, c0, box_rows, plane, tout + (size_t)box_rows * 64);
            tma_store_commit_wait();
            const int next = w + 2 * gridDim.x;
            if (next < nitems) issue(next, set);
        }
        __syncthreads();  // the output tile may be rewritten
    }
}

// ---- persistent FP32 y-pass with one warp per transform (N = 1024) -------
// Tiles are 16 float2 columns x My rows: 128-byte rows, 128B swizzle (the
// 16-byte chunk index is XORed with row mod 8).  A block is eight warps; warp w
// transforms packed column pair w (columns 2w, 2w+1) with fft_warp1024, so the
// only synchronisation inside a transform is __syncwarp.  Lane l holds the
// rows l + 32 q; reading pair w of 32 consecutive rows with 16-byte accesses
// spreads over all bank groups.  The tiles flow through the two-slot ring of
// the FP64 y-pass (YTiles): A in slot s, B in s^1, C back in s once A has been
// read, the output staged in s for the TMA store, and the next item's A and B
// loaded as soon as their slots are free.  Phi_xx Phi_yy stays in registers.
// The 16-byte chunk of tile row r holding column pair `pair`, for tiles of
// 2W float2 columns (16W-byte rows) with the matching TMA swizzle: 128B for
// W = 8 (chunk ^= r mod 8), 64B for W = 4 (chunk ^= (r/2) mod 4), 32B for
// W = 2 (chunk ^= (r/4) mod 2).  Each is the swizzle mode's XOR of address
// bits [4+] with bits [7+] for that row pitch, so a warp reading one pair of 32
// consecutive rows spreads over all banks (four wavefronts of 128 bytes).
template <int W>
__device__ __forceinline__ float4* swz_pair(unsigned char* tile, int r, int pair) {
    const int x = W == 8 ? (r & 7) : W == 4 ? ((r >> 1) & 3) : ((r >> 2) & 1);
    return reinterpret_cast<float4*>(tile + (size_t)r * (16 * W) + ((pair ^ x) << 4));
}

// My is a compile-time constant of N here, so that the rows of each register
// q that no lane reads (the masked middle of the spectrum) fold to zeros;
// kyf is the ky table rounded to FP32, in shared memory.
template <int N, int MULT, int W>
__device__ __forceinline__ void warp_tile_c2r_pair(float2 (&v)[32], unsigned char* tile, int pair, int lane,
                                                   const float* kyf) {
    constexpr int My = (2 * (N / 2 + 1)) / 3;
#pragma unroll
    for (int q = 0; q < 32; ++q) {
        const int k = lane + 32 * q;
        int kk = -1;
        bool ext = false;
        if (k < My) {
            kk = k;
        } else if (k > N / 2 && N - k < My) {
            kk = N - k;
            ext = true;
        }
        float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
        if (kk >= 0) {
            const float4 ab = *swz_pair<W>(tile, kk, pair);
            a = make_float2(ab.x, ab.y);
            b = make_float2(ab.z, ab.w);
            if constexpr (MULT == 1) {
                const float ky = kyf[kk];
                const float m = -(ky * ky);
                a = cscale(a, m);
                b = cscale(b, m);
            } else if constexpr (MULT == 2) {
                const float ky = kyf[kk];
                a = cmul_is(a, ky);
                b = cmul_is(b, ky);
            }
            if (ext) {
                a = cconj(a);
                b = cconj(b);
            }
            if (k == 0) {
                a.y = 0.f;
                b.y = 0.f;
            }
        }
        v[q] = make_float2(a.x - b.y, a.y + b.x);
    }
}

template <int N, int W>
__device__ __forceinline__ bool ma_y_mp_warp_item(YTiles& yt, const CUtensorMap* tA, const CUtensorMap* tB,
                                                  const CUtensorMap* tC, const CUtensorMap* tD, float2* buf,
                                                  int pair, int lane, int tid, int w, int next, int nitems,
                                                  int sa, const float2* tw, const float* kyf) {
    constexpr int My = (2 * (N / 2 + 1)) / 3;
    const int sb = sa ^ 1;
    float2 v[32], S[32];
    // Phi_xx from slot sa; then C of this item into sa
    if (!yt.wait(sa)) return false;
    warp_tile_c2r_pair<N, 0, W>(v, yt.slot(sa), pair, lane, kyf);
    __syncthreads();
    if (tid == 0) {
        fence_proxy_async();
        yt.load(sa, tC, w);
    }
    fft_warp1024<+1, float2, true>(v, lane, buf, tw);
#pragma unroll
    for (int q = 0; q < 32; ++q) S[q] = v[q];
    // Phi_yy from slot sb; then A of the next item into sb
    if (!yt.wait(sb)) return false;
    warp_tile_c2r_pair<N, 1, W>(v, yt.slot(sb), pair, lane, kyf);
    __syncthreads();
    if (tid == 0 && next < nitems) {
        fence_proxy_async();
        yt.load(sb, tA, next);
    }
    fft_warp1024<+1, float2, true>(v, lane, buf, tw);
#pragma unroll
    for (int q = 0; q < 32; ++q) S[q] = make_float2(S[q].x * v[q].x, S[q].y * v[q].y);
    // Phi_xy from slot sa and D = Phi_xx Phi_yy - Phi_xy^2
    if (!yt.wait(sa)) return false;
    warp_tile_c2r_pair<N, 2, W>(v, yt.slot(sa), pair, lane, kyf);
    __syncthreads();  // slot sa is read: it becomes the output tile
    fft_warp1024<+1, float2, true>(v, lane, buf, tw);
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = make_float2(S[q].x - v[q].x * v[q].x, S[q].y - v[q].y * v[q].y);
    fft_warp1024<-1, float2, true>(v, lane, buf, tw);
    // split the packed transform into the two half spectra, rows ky < My
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 32; ++q) buf[lane + 32 * q] = v[q];
    __syncwarp();
    unsigned char* out = yt.slot(sa);
#pragma unroll
    for (int q = 0; q < 32; ++q) {
        const int k = lane + 32 * q;
        if (k < My) {
            const float2 z = buf[k];
            const float2 zm = buf[(N - k) & (N - 1)];
            *swz_pair<W>(out, k, pair) =
                make_float4(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y), 0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
        }
    }
    fence_proxy_async();
    __syncthreads();  // the output tile is complete
    if (tid == 0) {
        const int c0 = (w % yt.xtiles) * yt.cstep, plane = w / yt.xtiles;
        tma_store_3d(tD, c0, 0, plane, out);
        if (yt.box_rows < My) tma_store_3d(tD, c0, yt.box_rows, plane, out + (size_t)yt.box_rows * yt.rowb);
        tma_store_commit_wait();  // the tile has been read out: slot sa takes the next item's B
        if (next < nitems) yt.load(sa, tB, next);
    }
    return true;
}

// W warps per block (W column pairs per tile): fewer warps per block means
// more independent blocks per SM (8/W at the ~255 registers a warp's
// transform needs), which run their barriers and tile waits out of step.
template <int N, int W>
__global__ void __launch_bounds__(32 * W, 8 / W)
    ma_y_mp_warp_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB,
                        const __grid_constant__ CUtensorMap tC, const __grid_constant__ CUtensorMap tD,
                        const float2* __restrict__ tw, const double* __restrict__ kyc, int My, int box_rows,
                        int xtiles, int nitems, unsigned int* errflag) {
    static_assert(N == 1024, "one warp holds a length-1024 transform");
    static_assert(W == 2 || W == 4 || W == 8, "tiles of 4, 8 or 16 columns");
    extern __shared__ unsigned char ysm_raw[];
    unsigned char* base = smem_align<1024>(ysm_raw);
    __shared__ __align__(8) uint64_t full[2];
    const int tid = threadIdx.x, lane = tid & 31, pair = tid >> 5;
    YTiles yt;
    yt.bytes = (unsigned)(2 * box_rows * 16 * W);
    yt.base = base;
    yt.full = full;
    yt.ph = 0u;
    yt.box_rows = box_rows;
    yt.xtiles = xtiles;
    yt.rowb = 16 * W;
    yt.cstep = 4 * W;
    float2* buf = reinterpret_cast<float2*>(base + 2 * yt.bytes) + pair * kWarpFftBuf;
    // the twiddle table and the FP32 ky table, once per block
    float2* tws = reinterpret_cast<float2*>(base + 2 * yt.bytes) + W * kWarpFftBuf;
    float* kyf = reinterpret_cast<float*>(tws + N);
    for (int j = tid; j < N; j += 32 * W) tws[j] = tw[j];
    for (int j = tid; j < My; j += 32 * W) kyf[j] = (float)kyc[j];
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (tid == 0 && (int)blockIdx.x < nitems) {
        yt.load(0, &tA, blockIdx.x);
        yt.load(1, &tB, blockIdx.x);
    }
    int i = 0;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x, ++i) {
        const int next = w + (int)gridDim.x;
        if (!ma_y_mp_warp_item<N, W>(yt, &tA, &tB, &tC, &tD, buf, pair, lane, tid, w, next, nitems, i & 1, tws,
                                     kyf)) {
            if (tid == 0) {
                atomicOr(errflag, 1u);
                asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
            }
            return;
        }
    }
}

// ============================================================================
// Surface tendency
// ============================================================================

template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    surf_xinv3_kernel(const double2* __restrict__ phih, const double2* __restrict__ bh, double2* __restrict__ P1,
                      double2* __restrict__ P2, double2* __restrict__ P3, const double2* __restrict__ tw,
                      const double* __restrict__ kxc, int My, double scale, size_t phi_stride) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    {  // member blockIdx.y
        const size_t mb = blockIdx.y;
        phih += mb * phi_stride;
        bh += mb * (size_t)Mx * My;
        P1 += mb * (size_t)N * My;
        P2 += mb * (size_t)N * My;
        P3 += mb * (size_t)N * My;
    }
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * 3 * FftShape<N>::BUF;
    const int ky = blockIdx.x * ROWS + team;
    const bool active = ky < My;
    // phi, i kx phi and b of the row, transformed together pass by pass
    double2 v[3][8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        bool cj;
        const int c = real_src_col<N>(t + p * T, ky, cj);
        double2 ph = make_double2(0.0, 0.0), b = make_double2(0.0, 0.0);
        double kx = 0.0;
        if (active && c >= 0) {
            const double2 x = cscale(phih[c + (size_t)Mx * ky], scale);
            const double2 y = cscale(bh[c + (size_t)Mx * ky], scale);
            ph = cj ? cconj(x) : x;
            b = cj ? cconj(y) : y;
            kx = cj ? -__ldg(&kxc[c]) : __ldg(&kxc[c]);
        }
        v[0][p] = ph;
        v[1][p] = cmul_is(ph, kx);
        v[2][p] = b;
    }
    fft_team_k<N, +1, 3>(v, t, buf, tw);
    if (active) {
        const size_t o = (size_t)N * ky;
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            P1[o + t + p * T] = v[0][p];
            P2[o + t + p * T] = v[1][p];
            P3[o + t + p * T] = v[2][p];
        }
    }
}

template <int N, int P>
__global__ void __launch_bounds__(N / 8 * P)
    surf_y_kernel(const double2* __restrict__ P1, const double2* __restrict__ P2, const double2* __restrict__ P3,
                  double2* __restrict__ Q1, double2* __restrict__ Q2, const double2* __restrict__ tw,
                  const double* __restrict__ kyc, int My) {
    {  // member blockIdx.y
        const size_t off = blockIdx.y * (size_t)N * My;
        P1 += off;
        P2 += off;
        P3 += off;
        Q1 += off;
        Q2 += off;
    }
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * 3 * FftShape<N>::BUF;
    const int x0 = 2 * (blockIdx.x * P + team);
    // b, u = -d(phi)/dy and v = d(phi)/dx of the column pair, transformed
    // together pass by pass (one twiddle load and one barrier per pass for
    // the three); then the fluxes u b and v b, transformed back together
    double2 v[3][8];
    load_c2r_pair<N, 0>(v[0], P3, x0, t, My, kyc);
    load_c2r_pair<N, 3>(v[1], P1, x0, t, My, kyc);
    load_c2r_pair<N, 0>(v[2], P2, x0, t, My, kyc);
    fft_team_k<N, +1, 3>(v, t, buf, tw);
    double2 f[2][8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        f[0][p] = make_double2(v[1][p].x * v[0][p].x, v[1][p].y * v[0][p].y);
        f[1][p] = make_double2(v[2][p].x * v[0][p].x, v[2][p].y * v[0][p].y);
    }
    fft_team_k<N, -1, 2>(f, t, buf, tw);
    store_r2c_pair<N>(f[0], buf, Q1, x0, t, My);
    store_r2c_pair<N>(f[1], buf, Q2, x0, t, My);
}

template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    surf_xfwd_stage_kernel(const double2* __restrict__ Q1, const double2* __restrict__ Q2,
                           const double2* __restrict__ tw, const double* __restrict__ kxc,
                           const double* __restrict__ kyc, const double* __restrict__ sigma, int My, StageArgs a) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    {  // member blockIdx.y
        const size_t mb = blockIdx.y, cs = mb * (size_t)Mx * My, ms = mb * (size_t)N * My;
        Q1 += ms;
        Q2 += ms;
        if (a.bh) a.bh += cs;
        if (a.bstage) a.bstage += cs;
        if (a.fold) a.fold += cs;
        if (a.fout) a.fout += cs;
    }
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * 2 * FftShape<N>::BUF;
    const int ky = blockIdx.x * ROWS + team;
    const bool active = ky < My;
    // the two flux rows, transformed together pass by pass
    double2 Fq[2][8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        Fq[0][p] = active ? Q1[(size_t)N * ky + t + p * T] : make_double2(0.0, 0.0);
        Fq[1][p] = active ? Q2[(size_t)N * ky + t + p * T] : make_double2(0.0, 0.0);
    }
    fft_team_k<N, -1, 2>(Fq, t, buf, tw);
    if (!active) return;
    const double2(&F1)[8] = Fq[0];
    const double2(&v)[8] = Fq[1];
    const double kyv = kyc[ky];
    bool bad = false;
    if (a.step_dev) {
        const int64_t st = *a.step_dev;
        if (a.mode == STAGE_AB2 && st == 0) a.mode = STAGE_AB2_FIRST;
        a.filter = a.filter && a.filter_freq > 0 && (st + 1) % a.filter_freq == 0;
    }
    // Gather first: the tendency of each of this thread's modes and the state
    // its stage update reads, all loads issued before any store (the stores
    // to bh/fold/bstage would otherwise keep the next mode's loads waiting).
    const int mode = a.mode;
    const bool hist1 = mode == STAGE_AB2 || mode == STAGE_RK3_3;    // reads fold (f_old / k1)
    const bool hist2 = mode == STAGE_RK3_2 || mode == STAGE_RK3_3;  // reads bstage
    const bool alias = a.ab2_alias && (mode == STAGE_AB2 || mode == STAGE_AB2_FIRST);
    double2 f[8], bv[8], fo[8], bs[8];
    double sg[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int c = compact_col<N>(t + p * T);
        if (c < 0) continue;
        const size_t m = c + (size_t)Mx * ky;
        const double kx = kxc[c];
        const double2 j1 = cmul_is(F1[p], kx), j2 = cmul_is(v[p], kyv);
        // literal AB2: jacobian_2d!'s step 6 overwrites the x-flux derivative
        // and step 7 adds the y-flux derivative to itself
        f[p] = alias ? make_double2(-(j2.x + j2.x), -(j2.y + j2.y)) : make_double2(-(j1.x + j2.x), -(j1.y + j2.y));
        // dealias_2d! then irfft_2d! (src/nonlinear.jl:31-33) keeps (-N/3, 0)
        // without its partner (+N/3, 0); the complex-to-real transform then
        // keeps half of it.
        if (ky == 0 && c == N / 3) f[p] = cscale(f[p], 0.5);
        if (mode == STAGE_TENDENCY) continue;
        bv[p] = a.bh[m];
        if (hist1) fo[p] = a.fold[m];
        if (hist2) bs[p] = a.bstage[m];
        if (a.filter) sg[p] = __ldg(&sigma[m]);
    }
    const double dt = a.dt;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int c = compact_col<N>(t + p * T);
        if (c < 0) continue;
        const size_t m = c + (size_t)Mx * ky;
        if (mode == STAGE_TENDENCY) {
            a.fout[m] = f[p];
            continue;
        }
        double2 b = bv[p];
        switch (mode) {
            case STAGE_AB2_FIRST:
                b = make_double2(b.x + dt * f[p].x, b.y + dt * f[p].y);
                a.fold[m] = f[p];
                break;
            case STAGE_AB2:
                b = make_double2(b.x + dt * (1.5 * f[p].x - 0.5 * fo[p].x), b.y + dt * (1.5 * f[p].y - 0.5 * fo[p].y));
                a.fold[m] = f[p];
                break;
            case STAGE_RK3_1: {
                a.bstage[m] = b;
                a.fold[m] = f[p];
                const double c1 = dt / 3.0;
                b = make_double2(b.x + c1 * f[p].x, b.y + c1 * f[p].y);
                break;
            }
            case STAGE_RK3_2: {
                const double c2 = 2.0 * dt / 3.0;
                b = make_double2(bs[p].x + c2 * f[p].x, bs[p].y + c2 * f[p].y);
                break;
            }
            default: {  // STAGE_RK3_3
                const double c3 = dt / 4.0;
                b = make_double2(bs[p].x + c3 * (fo[p].x + 3.0 * f[p].x), bs[p].y + c3 * (fo[p].y + 3.0 * f[p].y));
                break;
            }
        }
        if (a.filter) b = cscale(b, sg[p]);
        if (!isfinite(b.x) || !isfinite(b.y)) bad = true;
        a.bh[m] = b;
    }
    if (bad) atomicOr(a.nonfinite, 1u);
}

// ============================================================================
// Generic transforms
// ============================================================================

template <int N, int P>
__global__ void __launch_bounds__(N / 8 * P)
    y_r2c_kernel(const double* __restrict__ in, double2* __restrict__ out, const double2* __restrict__ tw, int My) {
    constexpr int T = N / 8;
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int x0 = 2 * (blockIdx.x * P + team);
    const double* src = in + (size_t)N * N * blockIdx.y;
    double2 v[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double* row = src + (size_t)N * (t + p * T) + x0;
        v[p] = make_double2(row[0], row[1]);
    }
    fft_team<N, -1>(v, t, buf, tw);
    store_r2c_pair<N>(v, buf, out + (size_t)N * My * blockIdx.y, x0, t, My);
}

template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    x_fwd_compact_kernel(const double2* __restrict__ in, double2* __restrict__ out, const double2* __restrict__ tw,
                         int My, double scale, int zero_mean) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int ky = blockIdx.x * ROWS + team;
    const bool active = ky < My;
    const double2* src = in + (size_t)N * (ky + (size_t)My * blockIdx.y);
    double2 v[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = active ? src[t + p * T] : make_double2(0.0, 0.0);
    fft_team<N, -1>(v, t, buf, tw);
    if (!active) return;
    double2* dst = out + (size_t)Mx * (ky + (size_t)My * blockIdx.y);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int c = compact_col<N>(t + p * T);
        if (c < 0) continue;
        double2 x = cscale(v[p], scale);
        if (zero_mean && ky == 0) {
            // set_b!: zero the mean, dealias, irfft (src/setICs.jl:34-51); the
            // complex-to-real transform keeps half of the unpartnered (-N/3, 0)
            if (c == 0) x = make_double2(0.0, 0.0);
            else if (c == N / 3) x = cscale(x, 0.5);
        }
        dst[c] = x;
    }
}

template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    x_inv_compact_kernel(const double2* __restrict__ in, double2* __restrict__ out, const double2* __restrict__ tw,
                         const double* __restrict__ kxc, const double* __restrict__ kyc, int My, int mult,
                         double scale) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int ky = blockIdx.x * ROWS + team;
    const bool active = ky < My;
    const double2* src = in + (size_t)Mx * (ky + (size_t)My * blockIdx.y);
    const double kyv = active ? kyc[ky] : 0.0;
    double2 v[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        bool cj;
        const int c = real_src_col<N>(t + p * T, ky, cj);
        double2 x = make_double2(0.0, 0.0);
        if (active && c >= 0) {
            x = cscale(src[c], scale);
            if (cj) x = cconj(x);
            if (mult == 1) x = cmul_is(x, -kyv);
            else if (mult == 2) x = cmul_is(x, cj ? -kxc[c] : kxc[c]);
        }
        v[p] = x;
    }
    fft_team<N, +1>(v, t, buf, tw);
    if (!active) return;
    double2* dst = out + (size_t)N * (ky + (size_t)My * blockIdx.y);
#pragma unroll
    for (int p = 0; p < 8; ++p) dst[t + p * T] = v[p];
}

template <int N, int P>
__global__ void __launch_bounds__(N / 8 * P)
    y_c2r_kernel(const double2* __restrict__ in, double* __restrict__ out, const double2* __restrict__ tw,
                 const double* __restrict__ kyc, int My) {
    constexpr int T = N / 8;
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int x0 = 2 * (blockIdx.x * P + team);
    double2 v[8];
    load_c2r_pair<N, 0>(v, in + (size_t)N * My * blockIdx.y, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
    double* dst = out + (size_t)N * N * blockIdx.y;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        double* row = dst + (size_t)N * (t + p * T) + x0;
        row[0] = v[p].x;
        row[1] = v[p].y;
    }
}

template <int TB>
__global__ void __launch_bounds__(TB) diagnostics_kernel(const double2* __restrict__ phih, const double2* __restrict__ bh,
                                                         const double* __restrict__ kxc, const double* __restrict__ kyc,
                                                         int Mx, int My, double* partials, unsigned int* ticket,
                                                         double* norms) {
    const size_t m = (size_t)blockIdx.x * TB + threadIdx.x;
    double ke = 0.0, var = 0.0;
    if (m < (size_t)Mx * My) {
        const int c = (int)(m % Mx), j = (int)(m / Mx);
        const double w = (j == 0 && c != Mx / 2) ? 1.0 : 2.0;
        const double K2 = kxc[c] * kxc[c] + kyc[j] * kyc[j];
        const double2 p = phih[m], b = bh[m];
        ke = w * K2 * (p.x * p.x + p.y * p.y);
        var = w * (b.x * b.x + b.y * b.y);
    }
    block_reduce_pair<TB>(ke, var, partials, ticket, norms);
}

__global__ void extrapolate_kernel(const double2* __restrict__ P, double2* __restrict__ Q, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double2 a = P[i], b = Q[i];
        Q[i] = make_double2(2.0 * a.x - b.x, 2.0 * a.y - b.y);
    }
}

__global__ void step_bump_kernel(int64_t* s) { *s += 1; }

// One thread per member (one block): iteration counts and stagnation
// history reset, every member's solve marked as going on.
__global__ void solve_begin_kernel(SolveDev* sd, unsigned int* active, int members) {
    for (int i = threadIdx.x; i < members; i += blockDim.x) {
        sd[i].it = 0;
        sd[i].prev = 0.0;
        if (active) active[i] = 1u;
    }
}

// The stop rule of the host loop in ssg_ctx.cu (ma_solve), on the device:
// one thread per member whose solve goes on (one block); the loop goes on
// while any member's does.
__global__ void solve_check_kernel(SolveDev* sdv, const double* norms, unsigned int* active, int members, double tol,
                                   int maxiter, int mixed, double mixed_floor, cudaGraphConditionalHandle handle,
                                   unsigned int* going_out) {
    int going = 0;
    for (int i = threadIdx.x; i < members; i += blockDim.x) {
        if (active && !active[i]) continue;
        SolveDev* sd = sdv + i;
        const double ds = norms[2 * i], ns = norms[2 * i + 1];
        const double upd = ns > 0 ? sqrt(ds / ns) : sqrt(ds);
        const int it = sd->it + 1;
        sd->it = it;
        bool stop = false, conv = false;
        if (!(upd == upd) || isinf(upd)) {
            stop = true;
            sd->flags |= 1u;
        } else if (upd <= tol) {
            stop = conv = true;
        } else if (mixed && upd <= mixed_floor) {
            stop = conv = true;
        } else if (mixed && it > 1 && upd > 0.5 * sd->prev) {
            stop = true;
            conv = upd <= 1e-5;
        } else if (it >= maxiter) {
            stop = true;
        }
        sd->prev = upd;
        sd->upd = upd;
        if (stop) {
            if (!going_out) {
                sd->solves += 1;
                sd->iters += it;
                sd->itmax = it > sd->itmax ? it : sd->itmax;
                sd->updmax = upd > sd->updmax ? upd : sd->updmax;
                if (!conv) sd->unconv += 1;
            }
            sd->last_it = it;
            sd->last_conv = conv ? 1 : 0;
        } else {
            going = 1;
        }
        if (active) active[i] = stop ? 0u : 1u;
    }
    going = __syncthreads_or(going);
    if (threadIdx.x == 0) {
        if (going_out) *going_out = going ? 1u : 0u;
        else cudaGraphSetConditional(handle, going ? 1u : 0u);
    }
}

// Polynomial extrapolation through equally spaced solutions a (newest), b, c,
// e: order 0 a; 1 2a - b; 2 3(a - b) + c; 3 4(a + c) - (6b + e).  out may
// alias an operand.
__global__ void predict_kernel(const double2* a, const double2* b, const double2* c, const double2* e, double2* out,
                               int order, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 x = a[i];
    double2 g;
    if (order == 0) {
        g = x;
    } else if (order == 1) {
        const double2 y = b[i];
        g = make_double2(2.0 * x.x - y.x, 2.0 * x.y - y.y);
    } else if (order == 2) {
        const double2 y = b[i], z = c[i];
        g = make_double2(3.0 * (x.x - y.x) + z.x, 3.0 * (x.y - y.y) + z.y);
    } else {
        const double2 y = b[i], z = c[i], w = e[i];
        g = make_double2(4.0 * (x.x + z.x) - (6.0 * y.x + w.x), 4.0 * (x.y + z.y) - (6.0 * y.y + w.y));
    }
    out[i] = g;
}

// The same extrapolation per mode (one thread per compact mode), followed by
// the boundary correction of the guess: the solution's dependence on the
// surface buoyancy through the top Neumann row is linear, so the part of the
// extrapolation error that comes from extrapolating b_s is removed exactly by
// adding the solution of L x = [0 ; delta], where
// delta = b_hat - (at G[nz-1] + bt G[nz-2] + ct G[nz-3]) is the mismatch of the
// guess G's top row with the current buoyancy.  With zero interior right-hand
// side the elimination leaves only the top level: x[n-1] = -(ga_n delta / at)
// inv[n-1], x[q] = -c_q x[q+1] (c_q = up_q inv_q from the pivot table), and the
// Neumann rows give the boundary planes.  The thread extrapolates the top
// three planes first (for delta), then walks the column from the top down,
// storing each plane's extrapolation plus its correction as it goes, so it
// holds only a few values (every plane is read before it is written, so out
// may alias an operand).  Only the surface right-hand side is corrected; the
// mean mode is left as extrapolated (the solve zeroes it).
// Four blocks per SM (64 registers, a few bytes spilled): more loads in flight
// than at three (80 registers): 0.582 against 0.591 ms per step at 1024^2 x 32
// mixed; five blocks (48 registers) spilled more and measured 0.585.
__global__ void __launch_bounds__(256, 4)
    predict_bc_kernel(const double2* a, const double2* b, const double2* c, const double2* e, double2* out,
                      int order, const double2* __restrict__ bh, const double* __restrict__ inv,
                      const ZOps* __restrict__ zo, int nz, size_t M, int Mx, size_t P) {
    const int n = nz - 2;
    const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    {  // member blockIdx.y
        const size_t off = blockIdx.y * M * nz;
        a += off;
        b += off;
        c += off;
        e += off;
        out += off;
        if (bh) bh += blockIdx.y * M;
    }
    auto extrap = [&](int k) -> double2 {
        const size_t i = m + M * k;
        const double2 x = a[i];
        if (order == 0) return x;
        if (order == 1) {
            const double2 y = b[i];
            return make_double2(2.0 * x.x - y.x, 2.0 * x.y - y.y);
        }
        if (order == 2) {
            const double2 y = b[i], z = c[i];
            return make_double2(3.0 * (x.x - y.x) + z.x, 3.0 * (x.y - y.y) + z.y);
        }
        const double2 y = b[i], z = c[i], w = e[i];
        return make_double2(4.0 * (x.x + z.x) - (6.0 * y.x + w.x), 4.0 * (x.y + z.y) - (6.0 * y.y + w.y));
    };
    if (m == 0 || !bh) {
        for (int k = 0; k < nz; ++k) out[m + M * k] = extrap(k);
        return;
    }
    const double2 g1 = extrap(nz - 1), g2 = extrap(nz - 2), g3 = extrap(nz - 3);
    const double ab = zo->ab, bb = zo->bb, cb = zo->cb, at = zo->at, bt = zo->bt, ct = zo->ct;
    const double2 bc = bh[m];
    const double2 dl = make_double2(bc.x - (at * g1.x + bt * g2.x + ct * g3.x),
                                    bc.y - (at * g1.y + bt * g2.y + ct * g3.y));
    const double ftop = zo->ga[n];
    const size_t pm = pivot_of(m, Mx);
    const double ivt = inv[pm + P * (n - 1)];
    double2 x = make_double2(-ftop * dl.x / at * ivt, -ftop * dl.y / at * ivt);
    const double2 xn1 = x;
    double2 xn2 = x, x0 = x, x1 = x;
    out[m + M * n] = make_double2(g2.x + x.x, g2.y + x.y);  // plane n = level q = n-1
#pragma unroll 2
    for (int q = n - 2; q >= 0; --q) {
        double lo, dg0, up;
        thomas_level(zo, q, n, lo, dg0, up);
        const double cq = up * inv[pm + P * q];
        const double2 v = (q + 1 == nz - 3) ? g3 : extrap(q + 1);
        x = make_double2(-cq * x.x, -cq * x.y);
        if (q == n - 2) xn2 = x;
        if (q == 1) x1 = x;
        if (q == 0) x0 = x;
        out[m + M * (q + 1)] = make_double2(v.x + x.x, v.y + x.y);
    }
    const double2 p0 = make_double2(-(bb * x0.x + cb * x1.x) / ab, -(bb * x0.y + cb * x1.y) / ab);
    const double2 pt = make_double2((dl.x - bt * xn1.x - ct * xn2.x) / at, (dl.y - bt * xn1.y - ct * xn2.y) / at);
    const double2 v0 = extrap(0);
    out[m] = make_double2(v0.x + p0.x, v0.y + p0.y);
    out[m + M * (nz - 1)] = make_double2(g1.x + pt.x, g1.y + pt.y);
}

__global__ void filter_kernel(double2* __restrict__ bh, const double* __restrict__ sigma, size_t M) {
    const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M) bh[m + blockIdx.y * M] = cscale(bh[m + blockIdx.y * M], sigma[m]);
}

// ============================================================================
// Host launchers
// ============================================================================


template <int N, int R>
static int ma_xinv3_run(const Dims& d, const Tables& tb, const double2* Phat, double2* A, double2* B, double2* C,
                         cudaStream_t s) {
    const size_t sm = (size_t)R * 3 * FftShape<N>::BUF * sizeof(double2);
    auto k = ma_xinv3_kernel<N, R>;
    set_smem(k, sm);
    dim3 grid((d.My + R - 1) / R, (d.nz - 2) * d.members), block(N / 8, R);
    k<<<grid, block, sm, s>>>(Phat, A, B, C, tb.tw, tb.kxc, d.My, 1.0 / ((double)N * (double)N), d.nz - 2);
    return check_launch();
}
template <int N>
static int ma_xinv3_impl(const Dims& d, const Tables& tb, const double2* Phat, double2* A, double2* B, double2* C,
                         cudaStream_t s) {
    SSG_DISPATCH_TILE_X(N, d.xbt, XRows<N>::R, return (ma_xinv3_run<N, RR>(d, tb, Phat, A, B, C, s)));
}
int launch_ma_xinv3(const Dims& d, const Tables& tb, const double2* Phat, double2* A, double2* B, double2* C,
                    cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return ma_xinv3_impl<NN>(d, tb, Phat, A, B, C, s));
    return 0;
}

template <int N, int P>
static int ma_y_run(const Dims& d, const Tables& tb, const double2* A, const double2* B, const double2* C,
                     double2* Dt, cudaStream_t s) {
    const size_t sm = (size_t)P * (FftShape<N>::BUF + 8 * (N / 8)) * sizeof(double2);
    auto k = ma_y_kernel<N, P>;
    set_smem(k, sm);
    dim3 grid(N / (2 * P), (d.nz - 2) * d.members), block(N / 8, P);
    k<<<grid, block, sm, s>>>(A, B, C, Dt, tb.tw, tb.kyc, d.My);
    return check_launch();
}
template <int N>
static int ma_y_impl(const Dims& d, const Tables& tb, const double2* A, const double2* B, const double2* C,
                     double2* Dt, cudaStream_t s) {
    SSG_DISPATCH_TILE_Y(N, d.ybt, (YPairs<N, 128>::P), return (ma_y_run<N, RR>(d, tb, A, B, C, Dt, s)));
}
int launch_ma_y(const Dims& d, const Tables& tb, const double2* A, const double2* B, const double2* C, double2* Dt,
                cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return ma_y_impl<NN>(d, tb, A, B, C, Dt, s));
    return 0;
}


// ---- TMA descriptors for the mixed arrays ----------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

bool mixed_tma_supported(const Dims& d) {
    const int box = ((d.My + 1) / 2 + 7) / 8 * 8;
    return d.N >= 32 && d.N <= 1024 && box <= 256 && tensor_map_encoder() != nullptr;
}

// A mixed array [plane][ky < My][x < N] complex as a 3-D FLOAT64 tensor
// {2N, My, nplanes}; box = 8 doubles (4 complex, 64 B) x box_rows x 1,
// 64B swizzle.  box_rows is a multiple of 8 so that the second box of a tile
// starts on a swizzle-atom boundary.
static int encode_mixed(CUtensorMap* m, const double2* base, const Dims& d, int nplanes, int box_rows) {
    auto fn = tensor_map_encoder();
    if (!fn) return -2;
    cuuint64_t dims[3] = {(cuuint64_t)2 * d.N, (cuuint64_t)d.My, (cuuint64_t)nplanes};
    cuuint64_t strides[2] = {(cuuint64_t)d.N * 16, (cuuint64_t)d.N * d.My * 16};
    cuuint32_t box[3] = {8, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double2*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -2;
}

int make_mixed_tmaps(const Dims& d, const double2* A, const double2* B, const double2* C, const double2* Dt,
                     int nplanes, MixedTmaps* out) {
    const int box = ((d.My + 1) / 2 + 7) / 8 * 8;
    out->box_rows = box;
    if (encode_mixed(&out->a, A, d, nplanes, box)) return -2;
    if (encode_mixed(&out->b, B, d, nplanes, box)) return -2;
    if (encode_mixed(&out->c, C, d, nplanes, box)) return -2;
    if (encode_mixed(&out->d, Dt, d, nplanes, box)) return -2;
    return 0;
}

template <int N>
static int ma_y_tma_impl(const Dims& d, const Tables& tb, const MixedTmaps& m, int sm_count, unsigned int* errflag,
                         cudaStream_t s) {
    if (N < 8) return -6;
    const size_t tb_bytes = (size_t)2 * m.box_rows * 64;
    const size_t sm = 512 + 2 * tb_bytes + (size_t)2 * (FftShape<N>::BUF + N) * sizeof(double2);
    auto k = ma_y_tma_kernel<N>;
    set_smem(k, sm);
    cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    const int xtiles = N / 4, nitems = xtiles * (d.nz - 2) * d.members;
    // one wave of resident blocks (looked up once per N)
    static std::atomic<int> wave[11];
    int lg = 0;
    while ((1 << lg) < N) ++lg;
    int resident = wave[lg].load(std::memory_order_relaxed);
    if (resident == 0) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, N / 4, sm);
        resident = (per_sm > 0 ? per_sm : 1) * (sm_count > 0 ? sm_count : 1);
        wave[lg].store(resident, std::memory_order_relaxed);
    }
    const int grid = resident < nitems ? resident : nitems;
    dim3 block(N / 8, 2);
    k<<<grid, block, sm, s>>>(m.a, m.b, m.c, m.d, tb.tw, tb.kyc, d.My, m.box_rows, xtiles, nitems, errflag);
    return check_launch();
}
int launch_ma_y_tma(const Dims& d, const Tables& tb, const MixedTmaps& maps, int sm_count, unsigned int* errflag,
                    cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return ma_y_tma_impl<NN>(d, tb, maps, sm_count, errflag, s));
    return 0;
}


template <int N, int R, int P>
static int ma_mp_run(const Dims& d, const Tables& tb, int pass, const double2* Phat, float2* A, float2* B, float2* C,
                     float2* Dt, double2* Dh, double eps, const double2* rhs_vol, cudaStream_t s,
                     float2* dh32 = nullptr) {
    if (pass == 0) {
        const size_t sm = (size_t)R * 3 * FftShape<N>::BUF * sizeof(float2);
        auto k = ma_xinv3_mp_kernel<N, R>;
        set_smem(k, sm);
        dim3 grid((d.My + R - 1) / R, (d.nz - 2) * d.members), block(N / 8, R);
        k<<<grid, block, sm, s>>>(Phat, A, B, C, tb.tw32, tb.kxc, d.My, 1.0 / ((double)N * (double)N), d.nz - 2);
    } else if (pass == 1) {
        const size_t sm = (size_t)P * FftShape<N>::BUF * sizeof(float2);
        auto k = ma_y_mp_kernel<N, P>;
        set_smem(k, sm);
        dim3 grid(N / (2 * P), (d.nz - 2) * d.members), block(N / 8, P);
        k<<<grid, block, sm, s>>>(A, B, C, Dt, tb.tw32, tb.kyc, d.My);
    } else {
        const size_t sm = (size_t)R * 2 * FftShape<N>::BUF * sizeof(float2);
        auto k = ma_xfwd_mp_kernel<N, R>;
        set_smem(k, sm);
        dim3 grid((d.My + 2 * R - 1) / (2 * R), (d.nz - 2) * d.members), block(N / 8, R);  // two rows per team
        k<<<grid, block, sm, s>>>(Dt, Dh, tb.tw32, d.My, eps, rhs_vol, dh32);
    }
    return check_launch();
}
template <int N>
static int ma_mp_impl(const Dims& d, const Tables& tb, int pass, const double2* Phat, float2* A, float2* B, float2* C,
                      float2* Dt, double2* Dh, double eps, const double2* rhs_vol, cudaStream_t s,
                      float2* dh32 = nullptr) {
    constexpr int R0 = XRows<N>::R, P0 = YPairs<N, 128>::P;
    if (pass == 1) {
        SSG_DISPATCH_TILE_Y(N, d.ybt, P0, return (ma_mp_run<N, R0, RR>(d, tb, pass, Phat, A, B, C, Dt, Dh, eps, rhs_vol, s)));
    }
    SSG_DISPATCH_TILE_X(N, d.xbt, R0,
                        return (ma_mp_run<N, RR, P0>(d, tb, pass, Phat, A, B, C, Dt, Dh, eps, rhs_vol, s, dh32)));
}
int launch_ma_xinv3_mp(const Dims& d, const Tables& tb, const double2* Phat, float2* A, float2* B, float2* C,
                       cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return ma_mp_impl<NN>(d, tb, 0, Phat, A, B, C, nullptr, nullptr, 0.0, nullptr, s));
    return 0;
}
int launch_ma_y_mp(const Dims& d, const Tables& tb, const float2* A, const float2* B, const float2* C, float2* Dt,
                   cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return ma_mp_impl<NN>(d, tb, 1, nullptr, const_cast<float2*>(A), const_cast<float2*>(B),
                                              const_cast<float2*>(C), Dt, nullptr, 0.0, nullptr, s));
    return 0;
}
int launch_ma_xfwd_mp(const Dims& d, const Tables& tb, const float2* Dt, double2* Dh, double eps,
                      const double2* rhs_vol, float2* dh32, cudaStream_t s) {
    if (dh32 && rhs_vol) return -6;  // the FP32 right-hand side carries no volume term
    SSG_DISPATCH_N(d.N, return ma_mp_impl<NN>(d, tb, 2, nullptr, nullptr, nullptr, nullptr, const_cast<float2*>(Dt), Dh,
                                              eps, rhs_vol, s, dh32));
    return 0;
}

// ---- FP32 row passes with one warp per row (N = 1024) ----------------------
// The same operations as ma_xinv3_mp_kernel / ma_xfwd_mp_kernel, with each
// length-1024 transform held by one warp (fft_warp1024: one shared-memory
// exchange per transform, against three block-wide exchanges for the radix-8
// team transform).  Lane l holds the row's entries l + 32 q, so loads and
// stores of a row are 32 consecutive elements per instruction.  A block is
// kXWarps warps, each its own row of the (plane, ky) row index; the three
// transforms of a row run one after the other through a runtime loop (one copy
// of the transform's code).
constexpr int kXWarps = 4;

__global__ void __launch_bounds__(32 * kXWarps)
    ma_xinv3_mp_warp_kernel(const double2* __restrict__ Phat, float2* __restrict__ A, float2* __restrict__ B,
                            float2* __restrict__ Cc, const float2* __restrict__ tw, const double* __restrict__ kxc,
                            int My, int rows, double scale, int nzi) {
    constexpr int N = 1024, Mx = 2 * (N / 3);
    __shared__ float2 bufs[kXWarps][kWarpFftBuf];
    __shared__ float2 tws[N];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = threadIdx.x; j < N; j += 32 * kXWarps) tws[j] = tw[j];
    __syncthreads();
    const int row = blockIdx.x * kXWarps + w;
    if (row >= rows) return;  // the whole warp: transforms synchronise within the warp only
    const int zi = row / My, ky = row - zi * My;
    const double2* src = Phat + (size_t)Mx * (ky + (size_t)My * interior_src_plane(zi, nzi));
    const size_t o = (size_t)N * (ky + (size_t)My * zi);
    float2* buf = bufs[w];
#pragma unroll 1
    for (int which = 0; which < 3; ++which) {
        float2 v[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) {
            bool cj;
            const int c = real_src_col<N>(lane + 32 * q, ky, cj);
            double2 x = make_double2(0.0, 0.0);
            if (c >= 0) {
                x = cscale(src[c], scale);
                if (cj) x = cconj(x);
                if (which != 1) {
                    const double kx = cj ? -__ldg(&kxc[c]) : __ldg(&kxc[c]);
                    x = (which == 0) ? cscale(x, -(kx * kx)) : cmul_is(x, kx);
                }
            }
            v[q] = make_float2((float)x.x, (float)x.y);
        }
        fft_warp1024<+1, float2, true>(v, lane, buf, tws);
        float2* dst = (which == 0) ? A : (which == 1) ? B : Cc;
#pragma unroll
        for (int q = 0; q < 32; ++q) dst[o + lane + 32 * q] = v[q];
    }
}

__global__ void __launch_bounds__(32 * kXWarps)
    ma_xfwd_mp_warp_kernel(const float2* __restrict__ Dt, double2* __restrict__ Dh, const float2* __restrict__ tw,
                           int My, int rows, double eps, const double2* __restrict__ rhs_vol) {
    constexpr int N = 1024, Mx = 2 * (N / 3);
    __shared__ float2 bufs[kXWarps][kWarpFftBuf];
    __shared__ float2 tws[N];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = threadIdx.x; j < N; j += 32 * kXWarps) tws[j] = tw[j];
    __syncthreads();
    const int row = blockIdx.x * kXWarps + w;
    if (row >= rows) return;
    const int zi = row / My, ky = row - zi * My;
    const float2* src = Dt + (size_t)N * (ky + (size_t)My * zi);
    float2 v[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = src[lane + 32 * q];
    fft_warp1024<-1, float2, true>(v, lane, bufs[w], tws);
    double2* dst = Dh + (size_t)Mx * (ky + (size_t)My * zi);
#pragma unroll
    for (int q = 0; q < 32; ++q) {
        const int c = compact_col<N>(lane + 32 * q);
        if (c >= 0) {
            double2 val = make_double2(eps * (double)v[q].x, eps * (double)v[q].y);
            if (rhs_vol) val = cadd(val, rhs_vol[c + (size_t)Mx * ky]);
            dst[c] = val;
        }
    }
}

int launch_ma_xinv3_mp_warp(const Dims& d, const Tables& tb, const float2* tw_warp, const double2* Phat, float2* A,
                            float2* B, float2* C, cudaStream_t s) {
    if (d.N != 1024) return -6;
    const int rows = d.My * (d.nz - 2) * d.members;
    ma_xinv3_mp_warp_kernel<<<(rows + kXWarps - 1) / kXWarps, 32 * kXWarps, 0, s>>>(
        Phat, A, B, C, tw_warp, tb.kxc, d.My, rows, 1.0 / ((double)d.N * (double)d.N), d.nz - 2);
    return check_launch();
}

int launch_ma_xfwd_mp_warp(const Dims& d, const Tables& tb, const float2* tw_warp, const float2* Dt, double2* Dh,
                           double eps, const double2* rhs_vol, cudaStream_t s) {
    if (d.N != 1024) return -6;
    const int rows = d.My * (d.nz - 2) * d.members;
    ma_xfwd_mp_warp_kernel<<<(rows + kXWarps - 1) / kXWarps, 32 * kXWarps, 0, s>>>(Dt, Dh, tw_warp, d.My, rows, eps,
                                                                                   rhs_vol);
    return check_launch();
}


// FP32 mixed arrays for the persistent y-pass: {2N floats, My, nplanes}, box
// 16 floats (8 float2 = 64 B) x box_rows, 64B swizzle.
static int encode_mixed32(CUtensorMap* m, const float2* base, const Dims& d, int nplanes, int box_rows) {
    auto fn = tensor_map_encoder();
    if (!fn) return -2;
    cuuint64_t dims[3] = {(cuuint64_t)2 * d.N, (cuuint64_t)d.My, (cuuint64_t)nplanes};
    cuuint64_t strides[2] = {(cuuint64_t)d.N * 8, (cuuint64_t)d.N * d.My * 8};
    cuuint32_t box[3] = {16, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -2;
}

int make_mixed32_tmaps(const Dims& d, const float2* A, const float2* B, const float2* C, const float2* Dt,
                       int nplanes, MixedTmaps* out) {
    const int box = ((d.My + 1) / 2 + 7) / 8 * 8;
    out->box_rows = box;
    if (encode_mixed32(&out->a, A, d, nplanes, box)) return -2;
    if (encode_mixed32(&out->b, B, d, nplanes, box)) return -2;
    if (encode_mixed32(&out->c, C, d, nplanes, box)) return -2;
    if (encode_mixed32(&out->d, Dt, d, nplanes, box)) return -2;
    return 0;
}

template <int N>
static int ma_y_mp_tma_impl(const Dims& d, const Tables& tb, const MixedTmaps& m, int grid_blocks,
                            unsigned int* errflag, cudaStream_t s) {
    const size_t tb_bytes = (size_t)2 * m.box_rows * 64;
    const size_t sm = 1024 + 7 * tb_bytes + (size_t)mp_y_teams<N>() * FftShape<N>::BUF * sizeof(float2);
    auto k = ma_y_mp_tma_kernel<N>;
    set_smem(k, sm);
    // one wave of resident blocks: below N = 1024 a block is one small team
    // set (N / 8 x 4 threads), several of which fit on an SM
    static std::atomic<int> per_sm_cache{0};
    int per_sm = per_sm_cache.load();
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, N / 8 * mp_y_teams<N>(), sm) != cudaSuccess ||
            per_sm < 1)
            per_sm = 1;
        per_sm_cache.store(per_sm);
    }
    const int xtiles = N / 8, nitems = xtiles * (d.nz - 2) * d.members;
    const int resident = grid_blocks * per_sm;
    const int grid = resident < nitems ? resident : nitems;
    dim3 block(N / 8, mp_y_teams<N>());
    k<<<grid, block, sm, s>>>(m.a, m.b, m.c, m.d, tb.tw32, tb.kyc, d.My, m.box_rows, xtiles, nitems, errflag);
    return check_launch();
}
int launch_ma_y_mp_tma(const Dims& d, const Tables& tb, const MixedTmaps& maps, int grid_blocks, unsigned int* errflag,
                       cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return ma_y_mp_tma_impl<NN>(d, tb, maps, grid_blocks, errflag, s));
    return 0;
}

// FP32 mixed arrays for the warp-transform y-pass: {2N floats, My, nplanes},
// box 4W floats (2W float2 = 16W bytes) x box_rows, with the swizzle of that
// row width (32B, 64B or 128B for W = 2, 4, 8).
static int encode_mixed32w(CUtensorMap* m, const float2* base, const Dims& d, int nplanes, int box_rows, int W) {
    auto fn = tensor_map_encoder();
    if (!fn) return -2;
    cuuint64_t dims[3] = {(cuuint64_t)2 * d.N, (cuuint64_t)d.My, (cuuint64_t)nplanes};
    cuuint64_t strides[2] = {(cuuint64_t)d.N * 8, (cuuint64_t)d.N * d.My * 8};
    cuuint32_t box[3] = {(cuuint32_t)(4 * W), (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapSwizzle sw = W == 8 ? CU_TENSOR_MAP_SWIZZLE_128B
                                         : W == 4 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B;
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -2;
}

int make_mixed32w_tmaps(const Dims& d, const float2* A, const float2* B, const float2* C, const float2* Dt,
                        int nplanes, int warps, MixedTmaps* out) {
    if (d.N != 1024 || (warps != 2 && warps != 4 && warps != 8)) return -6;
    const int box = ((d.My + 1) / 2 + 7) / 8 * 8;
    out->box_rows = box;
    out->warps = warps;
    if (encode_mixed32w(&out->a, A, d, nplanes, box, warps)) return -2;
    if (encode_mixed32w(&out->b, B, d, nplanes, box, warps)) return -2;
    if (encode_mixed32w(&out->c, C, d, nplanes, box, warps)) return -2;
    if (encode_mixed32w(&out->d, Dt, d, nplanes, box, warps)) return -2;
    return 0;
}

template <int W>
static int ma_y_mp_warp_impl(const Dims& d, const Tables& tb, const float2* tw_warp, const MixedTmaps& m,
                             int sm_count, unsigned int* errflag, cudaStream_t s) {
    constexpr int N = 1024;
    const size_t tb_bytes = (size_t)2 * m.box_rows * 16 * W;
    const size_t sm = 1024 + 2 * tb_bytes + (size_t)W * kWarpFftBuf * sizeof(float2) + N * sizeof(float2) +
                      (size_t)d.My * sizeof(float);
    if (d.My != (2 * (N / 2 + 1)) / 3) return -6;
    auto k = ma_y_mp_warp_kernel<N, W>;
    set_smem(k, sm);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * W, sm) != cudaSuccess || per_sm < 1) per_sm = 1;
    const int xtiles = N / (2 * W), nitems = xtiles * (d.nz - 2) * d.members;
    const int resident = sm_count * per_sm;
    const int grid = resident < nitems ? resident : nitems;
    k<<<grid, 32 * W, sm, s>>>(m.a, m.b, m.c, m.d, tw_warp, tb.kyc, d.My, m.box_rows, xtiles, nitems, errflag);
    return check_launch();
}

int launch_ma_y_mp_warp(const Dims& d, const Tables& tb, const float2* tw_warp, const MixedTmaps& m, int sm_count,
                        unsigned int* errflag, cudaStream_t s) {
    if (d.N != 1024) return -6;
    switch (m.warps) {
        case 2: return ma_y_mp_warp_impl<2>(d, tb, tw_warp, m, sm_count, errflag, s);
        case 4: return ma_y_mp_warp_impl<4>(d, tb, tw_warp, m, sm_count, errflag, s);
        default: return ma_y_mp_warp_impl<8>(d, tb, tw_warp, m, sm_count, errflag, s);
    }
}

template <int N, int R>
static int ma_xfwd_run(const Dims& d, const Tables& tb, const double2* Dt, double2* Dh, double eps,
                        const double2* rhs_vol, cudaStream_t s) {
    const size_t sm = (size_t)R * 2 * FftShape<N>::BUF * sizeof(double2);
    auto k = ma_xfwd_kernel<N, R>;
    set_smem(k, sm);
    dim3 grid((d.My + 2 * R - 1) / (2 * R), (d.nz - 2) * d.members), block(N / 8, R);  // two rows per team
    k<<<grid, block, sm, s>>>(Dt, Dh, tb.tw, d.My, eps, rhs_vol);
    return check_launch();
}
template <int N>
static int ma_xfwd_impl(const Dims& d, const Tables& tb, const double2* Dt, double2* Dh, double eps,
                        const double2* rhs_vol, cudaStream_t s) {
    SSG_DISPATCH_TILE_X(N, d.xbt, XRows<N>::R, return (ma_xfwd_run<N, RR>(d, tb, Dt, Dh, eps, rhs_vol, s)));
}
int launch_ma_xfwd(const Dims& d, const Tables& tb, const double2* Dt, double2* Dh, double eps,
                   const double2* rhs_vol, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return ma_xfwd_impl<NN>(d, tb, Dt, Dh, eps, rhs_vol, s));
    return 0;
}

// threads per block of the vertical solve: single-warp blocks for the staged
// kernel, whose shared memory sets how many share an SM; two-warp blocks for
// the register kernel, whose registers set it (8 warps per SM either way at
// nz = 32), halving the blocks that end with the reduction's fence and ticket
// (0.088 -> 0.078 ms at 1024^2 x 32; bit-identical)
constexpr int kThomasBlock = 32;
constexpr int kThomasRegBlock = 64;

int launch_ma_thomas_factor(const Dims& d, const Tables& tb, const ZOps* zops_dev, double* inv, cudaStream_t s) {
    constexpr int TB = 128;
    const size_t M = pivot_plane(d.Mx, d.My);
    ma_thomas_factor_kernel<TB><<<(unsigned)((M + TB - 1) / TB), TB, 0, s>>>(tb.kxc, tb.kyc, zops_dev, d.Mx, d.My, d.nz,
                                                                           inv);
    return check_launch();
}

bool thomas_reg_depth(int nz) { return nz == 8 || nz == 12 || nz == 16 || nz == 24 || nz == 32; }

int launch_ma_thomas(const Dims& d, const ZOps* zops_dev, const double* inv, const double2* Dh, const float2* Dh32,
                     double eps, const double2* bc_top, double2* Phat, double* partials, unsigned int* ticket,
                     double* norms, bool staged, const unsigned int* active, cudaStream_t s) {
    if (Dh32 && (staged || !thomas_reg_depth(d.nz))) return -6;  // the FP32 right-hand side: register form only
    constexpr int TB = kThomasBlock;
    const size_t M = d.c2();
    const int blocks = (int)((M + TB - 1) / TB);
    const size_t n = (size_t)d.nz - 2;
    const size_t sm = (n + d.nz) * TB * sizeof(double2) + n * TB * sizeof(double);
    constexpr int RB = kThomasRegBlock;
#define SSG_THOMAS_REG(Z)                                                                                         \
    if (!staged && d.nz == Z) {                                                                                   \
        dim3 g((unsigned)((M + RB - 1) / RB), d.members);                                                         \
        if (Dh32)                                                                                                 \
            ma_thomas_reg_kernel<RB, Z, float2><<<g, RB, 0, s>>>(Dh32, bc_top, Phat, inv, zops_dev, d.Mx, d.My,     \
                                                                 partials, ticket, norms, active, eps);           \
        else                                                                                                      \
            ma_thomas_reg_kernel<RB, Z, double2><<<g, RB, 0, s>>>(Dh, bc_top, Phat, inv, zops_dev, d.Mx, d.My,      \
                                                                  partials, ticket, norms, active, 0.0);          \
        return check_launch();                                                                                    \
    }
    SSG_THOMAS_REG(8)
    SSG_THOMAS_REG(12)
    SSG_THOMAS_REG(16)
    SSG_THOMAS_REG(24)
    SSG_THOMAS_REG(32)
#undef SSG_THOMAS_REG
    auto k = ma_thomas_kernel<TB>;
    set_smem(k, sm);
    k<<<dim3(blocks, d.members), TB, sm, s>>>(Dh, bc_top, Phat, inv, zops_dev, d.Mx, d.My, d.nz, partials, ticket,
                                               norms, active);
    return check_launch();
}

template <int N, int R>
static int surf_xinv3_run(const Dims& d, const Tables& tb, const double2* phih, const double2* bh, double2* P1,
                           double2* P2, double2* P3, cudaStream_t s) {
    const size_t sm = (size_t)R * 3 * FftShape<N>::BUF * sizeof(double2);
    auto k = surf_xinv3_kernel<N, R>;
    set_smem(k, sm);
    dim3 grid((d.My + R - 1) / R, d.members), block(N / 8, R);
    k<<<grid, block, sm, s>>>(phih, bh, P1, P2, P3, tb.tw, tb.kxc, d.My, 1.0 / ((double)N * (double)N),
                              d.c2() * d.nz);
    return check_launch();
}
template <int N>
static int surf_xinv3_impl(const Dims& d, const Tables& tb, const double2* phih, const double2* bh, double2* P1,
                           double2* P2, double2* P3, cudaStream_t s) {
    SSG_DISPATCH_TILE_X(N, d.xbt, XRows<N>::R, return (surf_xinv3_run<N, RR>(d, tb, phih, bh, P1, P2, P3, s)));
}
int launch_surf_xinv3(const Dims& d, const Tables& tb, const double2* phih, const double2* bh, double2* P1,
                      double2* P2, double2* P3, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return surf_xinv3_impl<NN>(d, tb, phih, bh, P1, P2, P3, s));
    return 0;
}

template <int N, int P>
static int surf_y_run(const Dims& d, const Tables& tb, const double2* P1, const double2* P2, const double2* P3,
                       double2* Q1, double2* Q2, cudaStream_t s) {
    const size_t sm = (size_t)P * 3 * FftShape<N>::BUF * sizeof(double2);
    auto k = surf_y_kernel<N, P>;
    set_smem(k, sm);
    dim3 grid(N / (2 * P), d.members), block(N / 8, P);
    k<<<grid, block, sm, s>>>(P1, P2, P3, Q1, Q2, tb.tw, tb.kyc, d.My);
    return check_launch();
}
template <int N>
static int surf_y_impl(const Dims& d, const Tables& tb, const double2* P1, const double2* P2, const double2* P3,
                       double2* Q1, double2* Q2, cudaStream_t s) {
    SSG_DISPATCH_TILE_Y(N, d.ybt, (YPairs<N, 256>::P), return (surf_y_run<N, RR>(d, tb, P1, P2, P3, Q1, Q2, s)));
}
int launch_surf_y(const Dims& d, const Tables& tb, const double2* P1, const double2* P2, const double2* P3,
                  double2* Q1, double2* Q2, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return surf_y_impl<NN>(d, tb, P1, P2, P3, Q1, Q2, s));
    return 0;
}

template <int N, int R>
static int surf_xfwd_stage_run(const Dims& d, const Tables& tb, const double2* Q1, const double2* Q2,
                                const StageArgs& a, cudaStream_t s) {
    const size_t sm = (size_t)R * 2 * FftShape<N>::BUF * sizeof(double2);
    auto k = surf_xfwd_stage_kernel<N, R>;
    set_smem(k, sm);
    dim3 grid((d.My + R - 1) / R, d.members), block(N / 8, R);
    k<<<grid, block, sm, s>>>(Q1, Q2, tb.tw, tb.kxc, tb.kyc, tb.sigma, d.My, a);
    return check_launch();
}
template <int N>
static int surf_xfwd_stage_impl(const Dims& d, const Tables& tb, const double2* Q1, const double2* Q2,
                                const StageArgs& a, cudaStream_t s) {
    SSG_DISPATCH_TILE_X(N, d.xbt, XRows<N>::R, return (surf_xfwd_stage_run<N, RR>(d, tb, Q1, Q2, a, s)));
}
int launch_surf_xfwd_stage(const Dims& d, const Tables& tb, const double2* Q1, const double2* Q2, const StageArgs& a,
                           cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return surf_xfwd_stage_impl<NN>(d, tb, Q1, Q2, a, s));
    return 0;
}

template <int N>
static int y_r2c_impl(const Dims& d, const Tables& tb, const double* in, double2* out, int nplanes, cudaStream_t s) {
    constexpr int P = YPairs<N, 256>::P;
    const size_t sm = (size_t)P * FftShape<N>::BUF * sizeof(double2);
    auto k = y_r2c_kernel<N, P>;
    set_smem(k, sm);
    dim3 grid(N / (2 * P), nplanes), block(N / 8, P);
    k<<<grid, block, sm, s>>>(in, out, tb.tw, d.My);
    return check_launch();
}
int launch_y_r2c(const Dims& d, const Tables& tb, const double* in, double2* out, int nplanes, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return y_r2c_impl<NN>(d, tb, in, out, nplanes, s));
    return 0;
}

template <int N>
static int x_fwd_compact_impl(const Dims& d, const Tables& tb, const double2* in, double2* out, int nplanes,
                              double scale, int zero_mean, cudaStream_t s) {
    constexpr int R = XRows<N>::R;
    const size_t sm = (size_t)R * FftShape<N>::BUF * sizeof(double2);
    auto k = x_fwd_compact_kernel<N, R>;
    set_smem(k, sm);
    dim3 grid((d.My + R - 1) / R, nplanes), block(N / 8, R);
    k<<<grid, block, sm, s>>>(in, out, tb.tw, d.My, scale, zero_mean);
    return check_launch();
}
int launch_x_fwd_compact(const Dims& d, const Tables& tb, const double2* in, double2* out, int nplanes, double scale,
                         int zero_mean, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return x_fwd_compact_impl<NN>(d, tb, in, out, nplanes, scale, zero_mean, s));
    return 0;
}

template <int N>
static int x_inv_compact_impl(const Dims& d, const Tables& tb, const double2* in, double2* out, int nplanes, int mult,
                              cudaStream_t s) {
    constexpr int R = XRows<N>::R;
    const size_t sm = (size_t)R * FftShape<N>::BUF * sizeof(double2);
    auto k = x_inv_compact_kernel<N, R>;
    set_smem(k, sm);
    dim3 grid((d.My + R - 1) / R, nplanes), block(N / 8, R);
    k<<<grid, block, sm, s>>>(in, out, tb.tw, tb.kxc, tb.kyc, d.My, mult, 1.0 / ((double)N * (double)N));
    return check_launch();
}
int launch_x_inv_compact(const Dims& d, const Tables& tb, const double2* in, double2* out, int nplanes, int mult,
                         cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return x_inv_compact_impl<NN>(d, tb, in, out, nplanes, mult, s));
    return 0;
}

template <int N>
static int y_c2r_impl(const Dims& d, const Tables& tb, const double2* in, double* out, int nplanes, cudaStream_t s) {
    constexpr int P = YPairs<N, 256>::P;
    const size_t sm = (size_t)P * FftShape<N>::BUF * sizeof(double2);
    auto k = y_c2r_kernel<N, P>;
    set_smem(k, sm);
    dim3 grid(N / (2 * P), nplanes), block(N / 8, P);
    k<<<grid, block, sm, s>>>(in, out, tb.tw, tb.kyc, d.My);
    return check_launch();
}
int launch_y_c2r(const Dims& d, const Tables& tb, const double2* in, double* out, int nplanes, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return y_c2r_impl<NN>(d, tb, in, out, nplanes, s));
    return 0;
}

int launch_diagnostics(const Dims& d, const Tables& tb, const double2* phih, const double2* bh, double* partials,
                       unsigned int* ticket, double* norms, cudaStream_t s) {
    constexpr int TB = 256;
    const size_t M = d.c2();
    diagnostics_kernel<TB><<<(unsigned)((M + TB - 1) / TB), TB, 0, s>>>(phih, bh, tb.kxc, tb.kyc, d.Mx, d.My, partials,
                                                                       ticket, norms);
    return check_launch();
}

int launch_extrapolate(const double2* Phat, double2* Pprev, size_t n, cudaStream_t s) {
    extrapolate_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(Phat, Pprev, n);
    return check_launch();
}

int launch_step_bump(int64_t* step_dev, cudaStream_t s) {
    step_bump_kernel<<<1, 1, 0, s>>>(step_dev);
    return check_launch();
}

int launch_solve_begin(SolveDev* sd, unsigned int* active, int members, cudaStream_t s) {
    solve_begin_kernel<<<1, members < 1024 ? ((members + 31) / 32) * 32 : 1024, 0, s>>>(sd, active, members);
    return check_launch();
}

int launch_solve_check(SolveDev* sd, const double* norms, unsigned int* active, int members, double tol, int maxiter,
                       int mixed, double mixed_floor, unsigned long long handle, unsigned int* going,
                       cudaStream_t s) {
    solve_check_kernel<<<1, members < 1024 ? ((members + 31) / 32) * 32 : 1024, 0, s>>>(
        sd, norms, active, members, tol, maxiter, mixed, mixed_floor, (cudaGraphConditionalHandle)handle, going);
    return check_launch();
}

int launch_predict(const double2* a, const double2* b, const double2* c, const double2* e, double2* out, int order,
                   size_t n, cudaStream_t s) {
    predict_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, c, e, out, order, n);
    return check_launch();
}

int launch_predict_bc(const Dims& d, const double2* a, const double2* b, const double2* c, const double2* e,
                      double2* out, int order, const double2* bh, const double* inv, const ZOps* zops_dev,
                      cudaStream_t s) {
    const size_t M = d.c2();
    predict_bc_kernel<<<dim3((unsigned)((M + 255) / 256), d.members), 256, 0, s>>>(a, b, c, e, out, order, bh, inv,
                                                                                   zops_dev, d.nz, M, d.Mx,
                                                                                   pivot_plane(d.Mx, d.My));
    return check_launch();
}

int launch_filter(const Dims& d, const Tables& tb, double2* bh, cudaStream_t s) {
    const size_t M = d.c2();
    filter_kernel<<<dim3((unsigned)((M + 255) / 256), d.members), 256, 0, s>>>(bh, tb.sigma, M);
    return check_launch();
}

}  // namespace ssg
