// adjoint_kernels.cu -- kernels of the discrete adjoint of the time step.
//
// The adjoint works on the same compact spectral coordinates as the forward
// state: a cotangent is stored as the (unnormalised) Fourier coefficients of a
// real field in V, the span of the modes the 2/3 mask keeps (with (+N/3, 0)
// implied as the conjugate of (-N/3, 0)).  In those coordinates every forward
// operator is one of
//   - a real even Fourier multiplier (dealiasing, filter, the vertical solve
//     per mode, second derivatives): its transpose is itself (per mode, the
//     transposed vertical matrix);
//   - an odd imaginary multiplier (first derivatives): transpose = negative;
//   - a pointwise product with a fixed real field: transpose = itself.
// So the transposed tendency and the transposed linearised Monge-Ampere
// operator are again spectral transforms, products and per-mode solves, and
// they reuse the forward passes' structure: x-passes over rows of the compact
// spectrum, y-passes over packed pairs of real columns, one thread per mode for
// the vertical solve.
//
// Forward operators transposed here (SSG.jl):
//   compute_tendency!/jacobian_2d!   src/nonlinear.jl:22-56, src/transforms.jl:430-465
//   compute_d_operator! (linearised) src/poisson.jl:183-223
//   d2dz2! + Neumann rows (per mode) src/transforms.jl:798-826, src/poisson.jl:309-364
#include "spectral_common.cuh"

namespace ssg {

// ============================================================================
// Transposed linearised Monge-Ampere operator
// ============================================================================

// Phi_xx, Phi_yy, Phi_xy of the interior planes as physical fields, from the
// x-pass outputs A, B, C of launch_ma_xinv3.  Stored per column pair:
// H[plane][x/2][y] = (f(x, y), f(x+1, y)) for even x, the layout in which the
// pair transforms of the y-passes read and write them with unit stride.
template <int N, int P>
__global__ void __launch_bounds__(N / 8 * P)
    ma_hess_y_kernel(const double2* __restrict__ A, const double2* __restrict__ B, const double2* __restrict__ C,
                     double2* __restrict__ Hxx, double2* __restrict__ Hyy, double2* __restrict__ Hxy,
                     const double2* __restrict__ tw, const double* __restrict__ kyc, int My) {
    extern __shared__ double2 smem[];
    constexpr int T = N / 8;
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int q = blockIdx.x * P + team;
    const int x0 = 2 * q;
    const size_t poff = (size_t)N * My * blockIdx.y;
    const size_t hoff = (size_t)N * (N / 2) * blockIdx.y + (size_t)N * q;
    double2 v[8];
    load_c2r_pair<N, 0>(v, A + poff, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) Hxx[hoff + t + p * T] = v[p];
    load_c2r_pair<N, 1>(v, B + poff, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) Hyy[hoff + t + p * T] = v[p];
    load_c2r_pair<N, 2>(v, C + poff, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) Hxy[hoff + t + p * T] = v[p];
}

// y-pass of F'(Phi)^T: zeta = eps * c2r(E) (E = x-inverse of the cotangent y,
// scaled 1/N^2), then Z1 = r2c_y(Phi_yy zeta), Z2 = r2c_y(Phi_xx zeta),
// Z3 = r2c_y(Phi_xy zeta), the transposes of the three products of the
// linearised operator dD = Phi_yy dPhi_xx + Phi_xx dPhi_yy - 2 Phi_xy dPhi_xy.
template <int N, int P>
__global__ void __launch_bounds__(N / 8 * P)
    adj_ma_y_kernel(const double2* __restrict__ E, const double2* __restrict__ Hxx, const double2* __restrict__ Hyy,
                    const double2* __restrict__ Hxy, double2* __restrict__ Z1, double2* __restrict__ Z2,
                    double2* __restrict__ Z3, const double2* __restrict__ tw, const double* __restrict__ kyc, int My,
                    double eps) {
    extern __shared__ double2 smem[];
    constexpr int T = N / 8;
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int q = blockIdx.x * P + team;
    const int x0 = 2 * q;
    const size_t poff = (size_t)N * My * blockIdx.y;
    const size_t hoff = (size_t)N * (N / 2) * blockIdx.y + (size_t)N * q;
    double2 z[8], v[8];
    load_c2r_pair<N, 0>(z, E + poff, x0, t, My, kyc);
    fft_team<N, +1>(z, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) z[p] = cscale(z[p], eps);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double2 h = Hyy[hoff + t + p * T];
        v[p] = make_double2(h.x * z[p].x, h.y * z[p].y);
    }
    fft_team<N, -1>(v, t, buf, tw);
    store_r2c_pair<N>(v, buf, Z1 + poff, x0, t, My);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double2 h = Hxx[hoff + t + p * T];
        v[p] = make_double2(h.x * z[p].x, h.y * z[p].y);
    }
    fft_team<N, -1>(v, t, buf, tw);
    store_r2c_pair<N>(v, buf, Z2 + poff, x0, t, My);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double2 h = Hxy[hoff + t + p * T];
        v[p] = make_double2(h.x * z[p].x, h.y * z[p].y);
    }
    fft_team<N, -1>(v, t, buf, tw);
    store_r2c_pair<N>(v, buf, Z3 + poff, x0, t, My);
}

// x-pass of F'(Phi)^T: Qh = -kx^2 X(Z1) - ky^2 X(Z2) + 2 kx ky X(Z3) on the
// kept modes (the second-derivative multipliers are real and even, so each is
// its own transpose).
template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    adj_ma_xfwd_kernel(const double2* __restrict__ Z1, const double2* __restrict__ Z2, const double2* __restrict__ Z3,
                       double2* __restrict__ Qh, const double2* __restrict__ tw, const double* __restrict__ kxc,
                       const double* __restrict__ kyc, int My) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int ky = blockIdx.x * ROWS + team;
    const int zi = blockIdx.y;
    const bool active = ky < My;
    const size_t o = (size_t)N * (ky + (size_t)My * zi);
    const double kyv = active ? kyc[ky] : 0.0;
    double2 acc[8], v[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = active ? Z1[o + t + p * T] : make_double2(0.0, 0.0);
    fft_team<N, -1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int c = compact_col<N>(t + p * T);
        const double kx = c >= 0 ? __ldg(&kxc[c]) : 0.0;
        acc[p] = cscale(v[p], -(kx * kx));
    }
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = active ? Z2[o + t + p * T] : make_double2(0.0, 0.0);
    fft_team<N, -1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) acc[p] = cadd(acc[p], cscale(v[p], -(kyv * kyv)));
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = active ? Z3[o + t + p * T] : make_double2(0.0, 0.0);
    fft_team<N, -1>(v, t, buf, tw);
    if (!active) return;
    double2* dst = Qh + (size_t)Mx * (ky + (size_t)My * zi);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int c = compact_col<N>(t + p * T);
        if (c < 0) continue;
        const double kx = __ldg(&kxc[c]);
        dst[c] = cadd(acc[p], cscale(v[p], 2.0 * kx * kyv));
    }
}

// Row q (plane q+1) of the interior tridiagonal system with the Neumann rows
// eliminated, exactly as the forward solve builds it.
__device__ __forceinline__ void z_row(const ZOps* __restrict__ zo, double K2, int q, int n, double& lo, double& dg,
                                      double& up) {
    const int k = q + 1;
    lo = zo->al[k];
    dg = zo->be[k] - K2;
    up = zo->ga[k];
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
}

// Transposed vertical solve, one thread per compact mode.  The forward solve
// per mode is Phi = E A^{-1} (R - (ga/at) bc e_last) + e_top bc / at, with A
// the interior tridiagonal matrix, E the map from interior unknowns to all
// planes (identity inside, the eliminated Neumann rows at the two ends).  For
// the plane cotangent w = (0, Qh (interior), gtop (top plane)) this computes
//   y  = A^{-T} E^T w                        (written to Y, update norm accumulated)
//   gb = (gtop - ga y_last) / at             (surface right-hand side), or
//   gb = sum_q y_q                           (volume right-hand side).
template <int TB>
__global__ void __launch_bounds__(TB)
    adj_thomas_kernel(const double2* __restrict__ Qh, const double2* __restrict__ gtop, double2* __restrict__ Y,
                      double2* __restrict__ gb, const double* __restrict__ kxc, const double* __restrict__ kyc,
                      const ZOps* __restrict__ zo, int Mx, int My, int nz, int volume, double* partials,
                      unsigned int* ticket, double* norms) {
    extern __shared__ double2 tsm2[];
    const int n = nz - 2;
    double2* sd = tsm2;                                             // [n][TB]: rhs, then d', then y
    double2* so = tsm2 + (size_t)n * TB;                            // [n][TB]: previous y
    double* sc = reinterpret_cast<double*>(tsm2 + (size_t)2 * n * TB);  // [n][TB]: c'
    const int tid = threadIdx.x;
    const size_t M = (size_t)Mx * My;
    const size_t m = (size_t)blockIdx.x * TB + tid;
    double ds = 0.0, ns = 0.0;
    if (m < M) {
        for (int q = 0; q < n; ++q) cp_async16(&sd[q * TB + tid], &Qh[m + M * q]);
        cp_async_commit();
        for (int q = 0; q < n; ++q) cp_async16(&so[q * TB + tid], &Y[m + M * q]);
        cp_async_commit();
        const int c = (int)(m % Mx), j = (int)(m / Mx);
        const double w = (j == 0 && c != Mx / 2) ? 1.0 : 2.0;
        const double2 g = gtop[m];
        cp_async_wait<1>();
        if (m == 0) {
            cp_async_wait<0>();
            for (int q = 0; q < n; ++q) {
                const double2 old = so[q * TB + tid];
                ds += w * (old.x * old.x + old.y * old.y);
                Y[m + M * q] = make_double2(0.0, 0.0);
            }
            gb[m] = make_double2(0.0, 0.0);
        } else {
            const double kx = kxc[c], ky = kyc[j];
            const double K2 = kx * kx + ky * ky;
            const double at = zo->at;
            // E^T w: the top plane's cotangent reaches the last two interior
            // unknowns through the eliminated top Neumann row
            {
                const double ft = -zo->bt / at, fc = -zo->ct / at;
                double2 r1 = sd[(n - 1) * TB + tid], r2 = sd[(n - 2) * TB + tid];
                sd[(n - 1) * TB + tid] = make_double2(r1.x + ft * g.x, r1.y + ft * g.y);
                sd[(n - 2) * TB + tid] = make_double2(r2.x + fc * g.x, r2.y + fc * g.y);
            }
            // A^T: row q has sub-diagonal up_{q-1}, diagonal dg_q, super-diagonal lo_{q+1}
            double lo_q, dg_q, up_q, lo_n, dg_n, up_n;
            z_row(zo, K2, 0, n, lo_q, dg_q, up_q);
            double up_prev = 0.0, cprev = 0.0;
            double2 dprev = make_double2(0.0, 0.0);
            for (int q = 0; q < n; ++q) {
                if (q + 1 < n) z_row(zo, K2, q + 1, n, lo_n, dg_n, up_n);
                else { lo_n = 0.0; dg_n = 0.0; up_n = 0.0; }
                const double subT = q > 0 ? up_prev : 0.0;
                const double supT = q + 1 < n ? lo_n : 0.0;
                const double2 r = sd[q * TB + tid];
                const double inv = 1.0 / (dg_q - subT * cprev);
                const double cq = supT * inv;
                const double2 dq = cscale(make_double2(r.x - subT * dprev.x, r.y - subT * dprev.y), inv);
                sc[q * TB + tid] = cq;
                sd[q * TB + tid] = dq;
                cprev = cq;
                dprev = dq;
                up_prev = up_q;
                lo_q = lo_n;
                dg_q = dg_n;
                up_q = up_n;
            }
            (void)lo_q;
            double2 x = dprev;
            for (int q = n - 2; q >= 0; --q) {
                const double2 dd = sd[q * TB + tid];
                const double cq = sc[q * TB + tid];
                x = make_double2(dd.x - cq * x.x, dd.y - cq * x.y);
                sd[q * TB + tid] = x;
            }
            cp_async_wait<0>();
            double2 sum = make_double2(0.0, 0.0);
            for (int q = 0; q < n; ++q) {
                const double2 nv = sd[q * TB + tid];
                const double2 old = so[q * TB + tid];
                const double dx = nv.x - old.x, dy = nv.y - old.y;
                ds += w * (dx * dx + dy * dy);
                ns += w * (nv.x * nv.x + nv.y * nv.y);
                sum = cadd(sum, nv);
                Y[m + M * q] = nv;
            }
            if (volume) {
                gb[m] = sum;
            } else {
                const double ga = zo->ga[nz - 2];
                const double2 yl = sd[(n - 1) * TB + tid];
                gb[m] = make_double2((g.x - ga * yl.x) / at, (g.y - ga * yl.y) / at);
            }
        }
    }
    block_reduce_pair<TB>(ds, ns, partials, ticket, norms);
}

// The transposed solve for a compile-time depth NZ, from the forward solve's
// pivot table.  The forward elimination factors A = L U with L lower
// bidiagonal (diagonal p_q = 1 / inv_q, sub-diagonal lo_q) and U unit upper
// (super-diagonal c_q = up_q inv_q), so A^T = U^T L^T solves as
//   z_q = r_q - c_{q-1} z_{q-1},   y_{n-1} = z_{n-1} inv_{n-1},
//   y_q = (z_q - lo_{q+1} y_{q+1}) inv_q,
// with no divisions.  Each thread holds its mode's column in registers
// (right-hand side and pivots by plain loads at entry, the previous y by
// cp.async for the update norm); the loops unroll.
template <int TB, int NZ>
__global__ void __launch_bounds__(TB)
    adj_thomas_reg_kernel(const double2* __restrict__ Qh, const double2* __restrict__ gtop, double2* __restrict__ Y,
                          double2* __restrict__ gb, const double* __restrict__ inv, const ZOps* __restrict__ zo,
                          int Mx, int My, int volume, double* partials, unsigned int* ticket, double* norms) {
    constexpr int n = NZ - 2;
    __shared__ double slo[n], sup[n];
    __shared__ double2 so[n][TB];
    const int tid = threadIdx.x;
    for (int q = tid; q < n; q += TB) {
        double lo, dg, up;
        z_row(zo, 0.0, q, n, lo, dg, up);
        slo[q] = lo;
        sup[q] = up;
    }
    const size_t M = (size_t)Mx * My;
    const size_t m = (size_t)blockIdx.x * TB + tid;
    double ds = 0.0, ns = 0.0;
    double2 y[n];
    double iv[n];
    if (m < M) {
#pragma unroll
        for (int q = 0; q < n; ++q) cp_async16(&so[q][tid], &Y[m + M * q]);
        cp_async_commit();
#pragma unroll
        for (int q = 0; q < n; ++q) {
            y[q] = Qh[m + M * q];
            iv[q] = inv[pivot_of(m, Mx) + pivot_plane(Mx, My) * q];
        }
    }
    __syncthreads();
    if (m < M) {
        const int c = (int)(m % Mx), j = (int)(m / Mx);
        const double w = (j == 0 && c != Mx / 2) ? 1.0 : 2.0;
        const double2 g = gtop[m];
        if (m == 0) {
            cp_async_wait<0>();
#pragma unroll
            for (int q = 0; q < n; ++q) {
                const double2 old = so[q][tid];
                ds += w * (old.x * old.x + old.y * old.y);
                Y[m + M * q] = make_double2(0.0, 0.0);
            }
            gb[m] = make_double2(0.0, 0.0);
        } else {
            const double at = zo->at;
            // E^T w: the top plane's cotangent reaches the last two interior
            // unknowns through the eliminated top Neumann row
            {
                const double ft = -zo->bt / at, fc = -zo->ct / at;
                y[n - 1] = make_double2(y[n - 1].x + ft * g.x, y[n - 1].y + ft * g.y);
                y[n - 2] = make_double2(y[n - 2].x + fc * g.x, y[n - 2].y + fc * g.y);
            }
#pragma unroll
            for (int q = 1; q < n; ++q) {
                const double cp = sup[q - 1] * iv[q - 1];
                y[q] = make_double2(y[q].x - cp * y[q - 1].x, y[q].y - cp * y[q - 1].y);
            }
            y[n - 1] = cscale(y[n - 1], iv[n - 1]);
#pragma unroll
            for (int q = n - 2; q >= 0; --q) {
                const double lo = slo[q + 1];
                y[q] = cscale(make_double2(y[q].x - lo * y[q + 1].x, y[q].y - lo * y[q + 1].y), iv[q]);
            }
            cp_async_wait<0>();
            double2 sum = make_double2(0.0, 0.0);
#pragma unroll
            for (int q = 0; q < n; ++q) {
                const double2 old = so[q][tid];
                const double dx = y[q].x - old.x, dy = y[q].y - old.y;
                ds += w * (dx * dx + dy * dy);
                ns += w * (y[q].x * y[q].x + y[q].y * y[q].y);
                sum = cadd(sum, y[q]);
                Y[m + M * q] = y[q];
            }
            if (volume) {
                gb[m] = sum;
            } else {
                const double ga = zo->ga[n];
                gb[m] = make_double2((g.x - ga * y[n - 1].x) / at, (g.y - ga * y[n - 1].y) / at);
            }
        }
    }
    block_reduce_pair<TB>(ds, ns, partials, ticket, norms);
}

// ============================================================================
// Transposed surface tendency
// ============================================================================
// Forward: f = -D[dx(u b) + dy(v b)], u = -dy(phi), v = dx(phi), with D the
// dealiasing of compute_tendency! (which keeps half of the unpartnered
// (-N/3, 0) mode).  For a cotangent lam on f, with mu = D lam:
//   cotangent on b   = P_V[u dx(mu) + v dy(mu)]
//   cotangent on phi = P_V[dy(b dx(mu)) - dx(b dy(mu))]

// x-pass: P1 = X^-1(phi), P2 = X^-1(i kx phi), P3 = X^-1(b), P4 = X^-1(i kx mu),
// P5 = X^-1(mu), all scaled 1/N^2 (ky multipliers follow in the y-pass).
template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    adj_surf_xinv5_kernel(const double2* __restrict__ phih, const double2* __restrict__ bh,
                          const double2* __restrict__ lam, double2* __restrict__ P1, double2* __restrict__ P2,
                          double2* __restrict__ P3, double2* __restrict__ P4, double2* __restrict__ P5,
                          const double2* __restrict__ tw, const double* __restrict__ kxc, int My, double scale) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int ky = blockIdx.x * ROWS + team;
    const bool active = ky < My;
    const size_t o = (size_t)N * ky;
    double2 src[8], v[8];
    double kx[8];
    // phi and its x-derivative
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        bool cj;
        const int c = real_src_col<N>(t + p * T, ky, cj);
        if (active && c >= 0) {
            const double2 x = cscale(phih[c + (size_t)Mx * ky], scale);
            src[p] = cj ? cconj(x) : x;
            kx[p] = cj ? -__ldg(&kxc[c]) : __ldg(&kxc[c]);
        } else {
            src[p] = make_double2(0.0, 0.0);
            kx[p] = 0.0;
        }
        v[p] = src[p];
    }
    fft_team<N, +1>(v, t, buf, tw);
    if (active) {
#pragma unroll
        for (int p = 0; p < 8; ++p) P1[o + t + p * T] = v[p];
    }
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = cmul_is(src[p], kx[p]);
    fft_team<N, +1>(v, t, buf, tw);
    if (active) {
#pragma unroll
        for (int p = 0; p < 8; ++p) P2[o + t + p * T] = v[p];
    }
    // b
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        bool cj;
        const int c = real_src_col<N>(t + p * T, ky, cj);
        double2 x = make_double2(0.0, 0.0);
        if (active && c >= 0) {
            x = cscale(bh[c + (size_t)Mx * ky], scale);
            if (cj) x = cconj(x);
        }
        v[p] = x;
    }
    fft_team<N, +1>(v, t, buf, tw);
    if (active) {
#pragma unroll
        for (int p = 0; p < 8; ++p) P3[o + t + p * T] = v[p];
    }
    // mu = D lam: the (-N/3, 0) coefficient (and its implied partner) halved
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        bool cj;
        const int c = real_src_col<N>(t + p * T, ky, cj);
        double2 x = make_double2(0.0, 0.0);
        if (active && c >= 0) {
            x = cscale(lam[c + (size_t)Mx * ky], (ky == 0 && c == N / 3) ? 0.5 * scale : scale);
            if (cj) x = cconj(x);
        }
        src[p] = x;
        v[p] = cmul_is(x, kx[p]);
    }
    fft_team<N, +1>(v, t, buf, tw);
    if (active) {
#pragma unroll
        for (int p = 0; p < 8; ++p) P4[o + t + p * T] = v[p];
    }
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = src[p];
    fft_team<N, +1>(v, t, buf, tw);
    if (active) {
#pragma unroll
        for (int p = 0; p < 8; ++p) P5[o + t + p * T] = v[p];
    }
}

// y-pass: b = c2r(P3), u = c2r(-i ky P1), v = c2r(P2), mux = c2r(P4),
// muy = c2r(i ky P5); Q1 = r2c_y(u mux + v muy), Q2 = r2c_y(b mux),
// Q3 = r2c_y(b muy).  b is parked in shared memory (each thread's own slots).
template <int N, int P>
__global__ void __launch_bounds__(N / 8 * P)
    adj_surf_y_kernel(const double2* __restrict__ P1, const double2* __restrict__ P2, const double2* __restrict__ P3,
                      const double2* __restrict__ P4, const double2* __restrict__ P5, double2* __restrict__ Q1,
                      double2* __restrict__ Q2, double2* __restrict__ Q3, const double2* __restrict__ tw,
                      const double* __restrict__ kyc, int My) {
    extern __shared__ double2 smem[];
    constexpr int T = N / 8;
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    double2* S = smem + P * FftShape<N>::BUF + (size_t)team * 8 * T;
    const int x0 = 2 * (blockIdx.x * P + team);
    double2 v[8], mu[8], acc[8];
    load_c2r_pair<N, 0>(v, P3, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) S[p * T + t] = v[p];
    // d(mu)/dx
    load_c2r_pair<N, 0>(mu, P4, x0, t, My, kyc);
    fft_team<N, +1>(mu, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double2 b = S[p * T + t];
        v[p] = make_double2(b.x * mu[p].x, b.y * mu[p].y);
    }
    fft_team<N, -1>(v, t, buf, tw);
    store_r2c_pair<N>(v, buf, Q2, x0, t, My);
    // u = -d(phi)/dy
    load_c2r_pair<N, 3>(v, P1, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) acc[p] = make_double2(v[p].x * mu[p].x, v[p].y * mu[p].y);
    // d(mu)/dy
    load_c2r_pair<N, 2>(mu, P5, x0, t, My, kyc);
    fft_team<N, +1>(mu, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const double2 b = S[p * T + t];
        v[p] = make_double2(b.x * mu[p].x, b.y * mu[p].y);
    }
    fft_team<N, -1>(v, t, buf, tw);
    store_r2c_pair<N>(v, buf, Q3, x0, t, My);
    // v = d(phi)/dx
    load_c2r_pair<N, 0>(v, P2, x0, t, My, kyc);
    fft_team<N, +1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) acc[p] = make_double2(acc[p].x + v[p].x * mu[p].x, acc[p].y + v[p].y * mu[p].y);
    fft_team<N, -1>(acc, t, buf, tw);
    store_r2c_pair<N>(acc, buf, Q1, x0, t, My);
}

// x-pass: out = base + X(Q1) (cotangent on b), gphi = i ky X(Q2) - i kx X(Q3)
// (cotangent on phi), on the kept modes.  base may be null (taken as zero) or
// alias out.
template <int N, int ROWS>
__global__ void __launch_bounds__(N / 8 * ROWS)
    adj_surf_xfwd_kernel(const double2* __restrict__ Q1, const double2* __restrict__ Q2,
                         const double2* __restrict__ Q3, const double2* base, double2* out,
                         double2* __restrict__ gphi, const double2* __restrict__ tw, const double* __restrict__ kxc,
                         const double* __restrict__ kyc, int My) {
    constexpr int T = N / 8, Mx = 2 * (N / 3);
    extern __shared__ double2 smem[];
    const int t = threadIdx.x, team = threadIdx.y;
    double2* buf = smem + team * FftShape<N>::BUF;
    const int ky = blockIdx.x * ROWS + team;
    const bool active = ky < My;
    const size_t o = (size_t)N * ky;
    const double kyv = active ? kyc[ky] : 0.0;
    double2 v[8], g[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = active ? Q1[o + t + p * T] : make_double2(0.0, 0.0);
    fft_team<N, -1>(v, t, buf, tw);
    if (active) {
        // out may be base (accumulation in place): read all of base first
        if (base) {
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                const int c = compact_col<N>(t + p * T);
                if (c >= 0) g[p] = base[c + (size_t)Mx * ky];
            }
        }
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            const int c = compact_col<N>(t + p * T);
            if (c < 0) continue;
            const size_t m = c + (size_t)Mx * ky;
            out[m] = base ? cadd(g[p], v[p]) : v[p];
        }
    }
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = active ? Q2[o + t + p * T] : make_double2(0.0, 0.0);
    fft_team<N, -1>(v, t, buf, tw);
#pragma unroll
    for (int p = 0; p < 8; ++p) g[p] = cmul_is(v[p], kyv);
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = active ? Q3[o + t + p * T] : make_double2(0.0, 0.0);
    fft_team<N, -1>(v, t, buf, tw);
    if (!active) return;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int c = compact_col<N>(t + p * T);
        if (c < 0) continue;
        const double kx = __ldg(&kxc[c]);
        gphi[c + (size_t)Mx * ky] = csub(g[p], cmul_is(v[p], kx));
    }
}

// ============================================================================
// Per-mode combinations
// ============================================================================

// out = a * s * x + b * y, s = sigma (filter transfer) when given, else 1;
// y may be null; out may alias x or y.
__global__ void adj_axpby_kernel(double2* out, const double2* x, double a, const double2* y, double b,
                                 const double* __restrict__ sigma, size_t M) {
    const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const double s = sigma ? a * sigma[m] : a;
    double2 r = cscale(x[m], s);
    if (y) r = cadd(r, cscale(y[m], b));
    out[m] = r;
}

// Quadratic extrapolation from three equally spaced solutions:
// Y3 <- 3 Y1 - 3 Y2 + Y3 (Y1 newest).
__global__ void extrapolate3_kernel(const double2* __restrict__ Y1, const double2* __restrict__ Y2, double2* Y3,
                                    size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 a = Y1[i], b = Y2[i], c = Y3[i];
    Y3[i] = make_double2(3.0 * (a.x - b.x) + c.x, 3.0 * (a.y - b.y) + c.y);
}

// Transpose of set_b!'s projection (mean removed, dealiased, complex-to-real):
// the mean mode is dropped and (-N/3, 0) halved.
__global__ void adj_setb_kernel(const double2* __restrict__ lam, double2* __restrict__ out, int Mx, size_t M) {
    const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    double2 v = lam[m];
    if (m == 0) v = make_double2(0.0, 0.0);
    else if (m == (size_t)(Mx / 2)) v = cscale(v, 0.5);
    out[m] = v;
}

// ============================================================================
// Host launchers
// ============================================================================

template <int N>
static int ma_hess_y_impl(const Dims& d, const Tables& tb, const double2* A, const double2* B, const double2* C,
                          double2* Hxx, double2* Hyy, double2* Hxy, cudaStream_t s) {
    constexpr int P = YPairs<N, 128>::P;
    const size_t sm = (size_t)P * FftShape<N>::BUF * sizeof(double2);
    auto k = ma_hess_y_kernel<N, P>;
    set_smem(k, sm);
    dim3 grid(N / (2 * P), d.nz - 2), block(N / 8, P);
    k<<<grid, block, sm, s>>>(A, B, C, Hxx, Hyy, Hxy, tb.tw, tb.kyc, d.My);
    return check_launch();
}
int launch_ma_hess_y(const Dims& d, const Tables& tb, const double2* A, const double2* B, const double2* C,
                     double2* Hxx, double2* Hyy, double2* Hxy, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return ma_hess_y_impl<NN>(d, tb, A, B, C, Hxx, Hyy, Hxy, s));
    return 0;
}

template <int N>
static int adj_ma_y_impl(const Dims& d, const Tables& tb, const double2* E, const double2* Hxx, const double2* Hyy,
                         const double2* Hxy, double2* Z1, double2* Z2, double2* Z3, double eps, cudaStream_t s) {
    constexpr int P = YPairs<N, 128>::P;
    const size_t sm = (size_t)P * FftShape<N>::BUF * sizeof(double2);
    auto k = adj_ma_y_kernel<N, P>;
    set_smem(k, sm);
    dim3 grid(N / (2 * P), d.nz - 2), block(N / 8, P);
    k<<<grid, block, sm, s>>>(E, Hxx, Hyy, Hxy, Z1, Z2, Z3, tb.tw, tb.kyc, d.My, eps);
    return check_launch();
}
int launch_adj_ma_y(const Dims& d, const Tables& tb, const double2* E, const double2* Hxx, const double2* Hyy,
                    const double2* Hxy, double2* Z1, double2* Z2, double2* Z3, double eps, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return adj_ma_y_impl<NN>(d, tb, E, Hxx, Hyy, Hxy, Z1, Z2, Z3, eps, s));
    return 0;
}

template <int N>
static int adj_ma_xfwd_impl(const Dims& d, const Tables& tb, const double2* Z1, const double2* Z2, const double2* Z3,
                            double2* Qh, cudaStream_t s) {
    constexpr int R = XRows<N>::R;
    const size_t sm = (size_t)R * FftShape<N>::BUF * sizeof(double2);
    auto k = adj_ma_xfwd_kernel<N, R>;
    set_smem(k, sm);
    dim3 grid((d.My + R - 1) / R, d.nz - 2), block(N / 8, R);
    k<<<grid, block, sm, s>>>(Z1, Z2, Z3, Qh, tb.tw, tb.kxc, tb.kyc, d.My);
    return check_launch();
}
int launch_adj_ma_xfwd(const Dims& d, const Tables& tb, const double2* Z1, const double2* Z2, const double2* Z3,
                       double2* Qh, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return adj_ma_xfwd_impl<NN>(d, tb, Z1, Z2, Z3, Qh, s));
    return 0;
}

int launch_adj_thomas(const Dims& d, const Tables& tb, const ZOps* zops_dev, const double* inv, const double2* Qh,
                      const double2* gtop, double2* Y, double2* gb, int volume, double* partials,
                      unsigned int* ticket, double* norms, bool staged, cudaStream_t s) {
    constexpr int TB = 64;
    const size_t M = d.c2();
#define SSG_ADJ_THOMAS_REG(Z)                                                                                      \
    if (!staged && d.nz == Z) {                                                                                    \
        adj_thomas_reg_kernel<TB, Z><<<(unsigned)((M + TB - 1) / TB), TB, 0, s>>>(Qh, gtop, Y, gb, inv, zops_dev,  \
                                                                                  d.Mx, d.My, volume, partials,    \
                                                                                  ticket, norms);                  \
        return check_launch();                                                                                     \
    }
    SSG_ADJ_THOMAS_REG(8)
    SSG_ADJ_THOMAS_REG(12)
    SSG_ADJ_THOMAS_REG(16)
    SSG_ADJ_THOMAS_REG(24)
    SSG_ADJ_THOMAS_REG(32)
#undef SSG_ADJ_THOMAS_REG
    const int blocks = (int)((M + TB - 1) / TB);
    const size_t n = (size_t)d.nz - 2;
    const size_t sm = 2 * n * TB * sizeof(double2) + n * TB * sizeof(double);
    auto k = adj_thomas_kernel<TB>;
    set_smem(k, sm);
    k<<<blocks, TB, sm, s>>>(Qh, gtop, Y, gb, tb.kxc, tb.kyc, zops_dev, d.Mx, d.My, d.nz, volume, partials, ticket,
                             norms);
    return check_launch();
}

template <int N>
static int adj_surf_xinv5_impl(const Dims& d, const Tables& tb, const double2* phih, const double2* bh,
                               const double2* lam, double2* const* P, cudaStream_t s) {
    constexpr int R = XRows<N>::R;
    const size_t sm = (size_t)R * FftShape<N>::BUF * sizeof(double2);
    auto k = adj_surf_xinv5_kernel<N, R>;
    set_smem(k, sm);
    dim3 grid((d.My + R - 1) / R), block(N / 8, R);
    k<<<grid, block, sm, s>>>(phih, bh, lam, P[0], P[1], P[2], P[3], P[4], tb.tw, tb.kxc, d.My,
                              1.0 / ((double)N * (double)N));
    return check_launch();
}
int launch_adj_surf_xinv5(const Dims& d, const Tables& tb, const double2* phih, const double2* bh, const double2* lam,
                          double2* const* P, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return adj_surf_xinv5_impl<NN>(d, tb, phih, bh, lam, P, s));
    return 0;
}

template <int N>
static int adj_surf_y_impl(const Dims& d, const Tables& tb, double2* const* P, double2* const* Q, cudaStream_t s) {
    constexpr int PP = YPairs<N, 128>::P;
    const size_t sm = (size_t)PP * (FftShape<N>::BUF + 8 * (N / 8)) * sizeof(double2);
    auto k = adj_surf_y_kernel<N, PP>;
    set_smem(k, sm);
    dim3 grid(N / (2 * PP)), block(N / 8, PP);
    k<<<grid, block, sm, s>>>(P[0], P[1], P[2], P[3], P[4], Q[0], Q[1], Q[2], tb.tw, tb.kyc, d.My);
    return check_launch();
}
int launch_adj_surf_y(const Dims& d, const Tables& tb, double2* const* P, double2* const* Q, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return adj_surf_y_impl<NN>(d, tb, P, Q, s));
    return 0;
}

template <int N>
static int adj_surf_xfwd_impl(const Dims& d, const Tables& tb, double2* const* Q, const double2* base, double2* out,
                              double2* gphi, cudaStream_t s) {
    constexpr int R = XRows<N>::R;
    const size_t sm = (size_t)R * FftShape<N>::BUF * sizeof(double2);
    auto k = adj_surf_xfwd_kernel<N, R>;
    set_smem(k, sm);
    dim3 grid((d.My + R - 1) / R), block(N / 8, R);
    k<<<grid, block, sm, s>>>(Q[0], Q[1], Q[2], base, out, gphi, tb.tw, tb.kxc, tb.kyc, d.My);
    return check_launch();
}
int launch_adj_surf_xfwd(const Dims& d, const Tables& tb, double2* const* Q, const double2* base, double2* out,
                         double2* gphi, cudaStream_t s) {
    SSG_DISPATCH_N(d.N, return adj_surf_xfwd_impl<NN>(d, tb, Q, base, out, gphi, s));
    return 0;
}

int launch_adj_axpby(const Dims& d, const Tables& tb, double2* out, const double2* x, double a, const double2* y,
                     double b, int use_sigma, cudaStream_t s) {
    const size_t M = d.c2();
    adj_axpby_kernel<<<(unsigned)((M + 255) / 256), 256, 0, s>>>(out, x, a, y, b, use_sigma ? tb.sigma : nullptr, M);
    return check_launch();
}

// Predicted guess of a transposed solve, per compact mode: the polynomial
// extrapolation of order `order` through the stage's earlier solutions a..e
// (interior planes), corrected for the current top cotangent.  The solve's
// solution is linear in the cotangent g on the top plane, which enters only
// through E^T (ft g on the last interior unknown, fc g on the one below it);
// the extrapolated guess carries the part belonging to the extrapolated g
// (history ga..ge, same weights), so adding A^-T E^T applied to
// g - extrap(g) makes that part exact.  A^-T applied to a vector with only its
// last two entries non-zero: the forward sweep touches only the last entry,
// the backward sweep fills the column.  gout receives g (it may alias ge or
// the slot of the newest history entry to be); out may alias e.
template <int NZ>
__global__ void __launch_bounds__(128)
    adj_predict_bc_kernel(const double2* a, const double2* b, const double2* c, const double2* e, double2* out,
                          int order, const double2* ga, const double2* gb, const double2* gc, const double2* ge,
                          double2* gout, const double2* __restrict__ gnew, const double* __restrict__ inv,
                          const ZOps* __restrict__ zo, int nz_rt, size_t M, int Mx, size_t P) {
    const int n = (NZ > 0 ? NZ : nz_rt) - 2;
    const size_t m = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const size_t pm = pivot_of(m, Mx);
    auto extrap = [&](const double2* pa, const double2* pb, const double2* pc, const double2* pe, size_t i) -> double2 {
        const double2 x = pa[i];
        if (order == 0) return x;
        if (order == 1) {
            const double2 y = pb[i];
            return make_double2(2.0 * x.x - y.x, 2.0 * x.y - y.y);
        }
        if (order == 2) {
            const double2 y = pb[i], z = pc[i];
            return make_double2(3.0 * (x.x - y.x) + z.x, 3.0 * (x.y - y.y) + z.y);
        }
        const double2 y = pb[i], z = pc[i], w = pe[i];
        return make_double2(4.0 * (x.x + z.x) - (6.0 * y.x + w.x), 4.0 * (x.y + z.y) - (6.0 * y.y + w.y));
    };
    const double2 gx = extrap(ga, gb, gc, ge, m);
    const double2 g = gnew[m];
    gout[m] = g;
    const double2 dg = make_double2(g.x - gx.x, g.y - gx.y);
    constexpr int NR = NZ > 0 ? NZ - 2 : 1;
    double2 y[NR];
    if constexpr (NZ > 0) {
#pragma unroll
        for (int q = 0; q < NZ - 2; ++q) y[q] = extrap(a, b, c, e, m + M * q);
    } else {
        for (int q = 0; q < n; ++q) out[m + M * q] = extrap(a, b, c, e, m + M * q);
    }
    if (m != 0) {
        const double at = zo->at, ft = -zo->bt / at, fc = -zo->ct / at;
        // forward sweep: only the last entry changes
        double lo, dg0, up;
        z_row(zo, 0.0, n - 2, n, lo, dg0, up);
        const double cpn = up * inv[pm + P * (n - 2)];
        const double ivn = inv[pm + P * (n - 1)];
        double2 x = make_double2((ft * dg.x - cpn * fc * dg.x) * ivn, (ft * dg.y - cpn * fc * dg.y) * ivn);
        double2 rhs = make_double2(fc * dg.x, fc * dg.y);  // entry n-2 of the injected vector
        auto add = [&](int q, double2 v) {
            if constexpr (NZ > 0) {
                y[q] = make_double2(y[q].x + v.x, y[q].y + v.y);
            } else {
                const size_t i = m + M * q;
                out[i] = make_double2(out[i].x + v.x, out[i].y + v.y);
            }
        };
        add(n - 1, x);
        // backward sweep: x_q = (r_q - lo_{q+1} x_{q+1}) inv_q
        if constexpr (NZ > 0) {
#pragma unroll
            for (int q = NZ - 4; q >= 0; --q) {
                double lo1, dg1, up1;
                z_row(zo, 0.0, q + 1, n, lo1, dg1, up1);
                const double iv = inv[pm + P * q];
                const double2 r = q == n - 2 ? rhs : make_double2(0.0, 0.0);
                x = make_double2((r.x - lo1 * x.x) * iv, (r.y - lo1 * x.y) * iv);
                add(q, x);
            }
        } else {
            for (int q = n - 2; q >= 0; --q) {
                double lo1, dg1, up1;
                z_row(zo, 0.0, q + 1, n, lo1, dg1, up1);
                const double iv = inv[pm + P * q];
                const double2 r = q == n - 2 ? rhs : make_double2(0.0, 0.0);
                x = make_double2((r.x - lo1 * x.x) * iv, (r.y - lo1 * x.y) * iv);
                add(q, x);
            }
        }
    }
    if constexpr (NZ > 0) {
#pragma unroll
        for (int q = 0; q < NZ - 2; ++q) out[m + M * q] = y[q];
    }
}

int launch_adj_predict_bc(const Dims& d, double2* const* Y, double2* out, int order, double2* const* G, double2* gout,
                          const double2* gnew, const double* inv, const ZOps* zops_dev, cudaStream_t s) {
    const size_t M = d.c2();
    const unsigned g = (unsigned)((M + 127) / 128);
#define SSG_ADJ_PRED(Z)                                                                                       \
    adj_predict_bc_kernel<Z><<<g, 128, 0, s>>>(Y[0], Y[1], Y[2], Y[3], out, order, G[0], G[1], G[2], G[3], gout, \
                                               gnew, inv, zops_dev, d.nz, M, d.Mx, pivot_plane(d.Mx, d.My))
    switch (d.nz) {
        case 8: SSG_ADJ_PRED(8); break;
        case 16: SSG_ADJ_PRED(16); break;
        case 32: SSG_ADJ_PRED(32); break;
        default: SSG_ADJ_PRED(0); break;
    }
#undef SSG_ADJ_PRED
    return check_launch();
}

int launch_extrapolate3(const double2* Y1, const double2* Y2, double2* Y3, size_t n, cudaStream_t s) {
    extrapolate3_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(Y1, Y2, Y3, n);
    return check_launch();
}

int launch_adj_setb(const Dims& d, const double2* lam, double2* out, cudaStream_t s) {
    const size_t M = d.c2();
    adj_setb_kernel<<<(unsigned)((M + 255) / 256), 256, 0, s>>>(lam, out, d.Mx, M);
    return check_launch();
}

}  // namespace ssg
