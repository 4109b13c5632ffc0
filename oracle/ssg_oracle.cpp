// ssg_oracle.cpp -- CPU restatement of the SSG.jl time-step path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker: it is built into
// liboracle_ssg.so and loaded by tests/, by __graft_entry__.smoke() and by the
// CPU-baseline leg of bench.py.  The product library (libssg_b200.so) never
// links, loads or calls it.
//
// Parity status.  The reference is Julia (SSG.jl) and cannot be executed in
// this image (no julia runtime, no network), and its multigrid solver does not
// run as shipped (create_coarse_domain is never included, `maxiter` is
// undefined in solve_monge_ampere_fields!).  This restatement is therefore
// pinned through
//   * numpy.fft (an independent FFT) for every transform, derivative, mask,
//     Jacobian and tendency primitive, and
//   * the known-answer tests mined from the reference's own test scripts
//     (filter transfer values and DC conservation, test/test_filter.jl;
//     analytic Jacobian, geostrophic velocities and buoyancy conservation,
//     test/test_nonlinear.jl; AB2/RK3 on y' = -y, test/test_timestep.jl).
// The full time step has no reference output to compare against: beyond those
// primitives its parity is unpinned.
//
// What it follows (file:line into SSG.jl):
//   grid, wavenumbers, 2/3 mask ........ src/domain.jl:143-173, 238-248, 498-514
//   rfft_2d!/irfft_2d! conventions ..... src/transforms.jl:42-56 (FFT on x,
//                                        RFFT on y, src/domain.jl:124-147)
//   ddx_2d!/ddy_2d! .................... src/transforms.jl:135-166
//   jacobian_2d! (conservative) ........ src/transforms.jl:430-465
//   compute_tendency!/compute_jacobian!  src/nonlinear.jl:22-56
//   AB2 / RK3 updates, timestep! ....... src/timestep.jl:152-242, 267-285
//   exponential filter ................. src/timestep.jl:247-260,
//                                        src/filter.jl:119-126, 283-309
//   set_b! ............................. src/setICs.jl:21-57
//   SSG residual, D operator, d2dz2 .... src/poisson.jl:143-253,
//                                        src/transforms.jl:798-826
//   Neumann boundary rows .............. src/poisson.jl:262-364
//   surface extraction ................. src/poisson.jl:1119-1131
//   geostrophic surface velocities ..... src/setICs.jl:161-192
//
// Monge-Ampere solve (documented equations).  The reference's own V-cycle
// diverges or is inert, so the solve here restates the documented problem of
// src/poisson.jl:1-12: interior planes satisfy
//     Phi_xx + Phi_yy + Phi_zz - eps (Phi_xx Phi_yy - Phi_xy^2) = rhs,
// with horizontal derivatives spectral and Phi_zz the 3-point stencil of
// d2dz2!, and the top/bottom planes satisfy the one-sided Neumann rows of
// apply_neumann_surface!/apply_neumann_bottom! with dPhi/dz = b_s on top and
// 0 at the bottom.  Phi is a real field kept in the 2/3-dealiased spectral
// space (as the reference's spectral smoother does, src/poisson.jl:685),
// closed under conjugate symmetry (mask_ext below), and the mean mode is
// fixed to zero.  The iteration is the fixed point
//     Phi_new = L^{-1} [ P(eps * F(D(Phi)) + rhs) ; Neumann rows ],
// where L is the linear operator (-k^2 + d2dz2 with Neumann rows), inverted
// exactly per horizontal mode by a tridiagonal (Thomas) solve, and P is the
// 2/3 mask.  The GPU library runs the same iteration; both stop when the
// relative update ||Phi_new - Phi|| / ||Phi_new|| falls to ma_tol.

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

namespace {

const long double PI_L = 3.141592653589793238462643383279502884L;

// ---------------------------------------------------------------------------
// 1-D complex FFT: iterative radix-2 (power-of-two lengths), naive DFT
// otherwise.  Twiddles are computed in long double.  Unnormalised in both
// directions; sign = -1 forward, +1 inverse.
// ---------------------------------------------------------------------------
struct Plan1D {
    int n = 0;
    bool pow2 = false;
    std::vector<cd> w;      // w[k] = exp(-2 pi i k / n)
    std::vector<int> rev;
    // per-stage twiddles of the radix-2 passes, stage of half-length h at
    // [h - 1, 2h - 1): exp(-+2 pi i j / 2h), j < h (forward, inverse)
    std::vector<double> tf, ti;
    void init(int n_) {
        n = n_;
        pow2 = n > 0 && (n & (n - 1)) == 0;
        w.resize(n);
        for (int k = 0; k < n; ++k) {
            long double a = -2.0L * PI_L * (long double)k / (long double)n;
            w[k] = cd((double)cosl(a), (double)sinl(a));
        }
        if (pow2) {
            tf.assign(2 * (size_t)std::max(n - 1, 1), 0.0);
            ti.assign(tf.size(), 0.0);
            for (int h = 1; h < n; h <<= 1)
                for (int j = 0; j < h; ++j) {
                    const cd t = w[(size_t)j * (n / (2 * h))];
                    tf[2 * (h - 1 + j)] = t.real();
                    tf[2 * (h - 1 + j) + 1] = t.imag();
                    ti[2 * (h - 1 + j)] = t.real();
                    ti[2 * (h - 1 + j) + 1] = -t.imag();
                }
            rev.assign(n, 0);
            int lg = 0;
            while ((1 << lg) < n) ++lg;
            for (int i = 0; i < n; ++i) {
                int r = 0;
                for (int b = 0; b < lg; ++b)
                    if (i & (1 << b)) r |= 1 << (lg - 1 - b);
                rev[i] = r;
            }
        }
    }
    void run(cd* a, int sign) const {
        if (n <= 1) return;
        if (!pow2) {
            std::vector<cd> out(n);
            for (int k = 0; k < n; ++k) {
                cd s = 0;
                for (int j = 0; j < n; ++j) {
                    long long idx = ((long long)j * k) % n;
                    cd t = w[idx];
                    if (sign > 0) t = std::conj(t);
                    s += a[j] * t;
                }
                out[k] = s;
            }
            std::copy(out.begin(), out.end(), a);
            return;
        }
        for (int i = 0; i < n; ++i)
            if (i < rev[i]) std::swap(a[i], a[rev[i]]);
        // radix-2 decimation in time on interleaved doubles
        double* x = reinterpret_cast<double*>(a);
        const double* T = (sign > 0 ? ti : tf).data();
        for (int i = 0; i < n; i += 2) {
            double ur = x[2 * i], ui = x[2 * i + 1], vr = x[2 * i + 2], vi = x[2 * i + 3];
            x[2 * i] = ur + vr; x[2 * i + 1] = ui + vi;
            x[2 * i + 2] = ur - vr; x[2 * i + 3] = ui - vi;
        }
        for (int half = 2; half < n; half <<= 1) {
            const double* tw = T + 2 * (half - 1);
            for (int i = 0; i < n; i += 2 * half) {
                double* p = x + 2 * i;
                double* q = x + 2 * (i + half);
                for (int j = 0; j < half; ++j) {
                    const double wr = tw[2 * j], wi = tw[2 * j + 1];
                    const double qr = q[2 * j], qi = q[2 * j + 1];
                    const double vr = qr * wr - qi * wi, vi = qr * wi + qi * wr;
                    const double ur = p[2 * j], ui = p[2 * j + 1];
                    p[2 * j] = ur + vr; p[2 * j + 1] = ui + vi;
                    q[2 * j] = ur - vr; q[2 * j + 1] = ui - vi;
                }
            }
        }
    }
};

// ---------------------------------------------------------------------------
// Grid, wavenumbers, mask (src/domain.jl:143-173, 238-248, 498-514)
// ---------------------------------------------------------------------------
struct Grid {
    int nx = 0, ny = 0, nyc = 0, nz = 0;
    double lx = 0, ly = 0, lz = 0, dx = 0, dy = 0;
    std::vector<double> kx, ky, dz;
    std::vector<uint8_t> mask;   // nx * nyc, x fastest
    // mask closed under the conjugate symmetry of a real field: the 2/3 mask
    // keeps kx = -Nx/3 but not +Nx/3, so in the ky = 0 column the partner of
    // (-Nx/3, 0) is added back.  The Monge-Ampere unknown lives on this set.
    std::vector<uint8_t> mask_ext;
    Plan1D px, py;

    void init(int nx_, int ny_, int nz_, double lx_, double ly_, double lz_) {
        nx = nx_; ny = ny_; nz = nz_; lx = lx_; ly = ly_; lz = lz_;
        nyc = ny / 2 + 1;
        dx = lx / nx;
        dy = ly / ny;
        // kx = 2pi .* fftfreq(Nx, 1/dx): (i < n_nonneg ? i : i - n) * (fs / n)
        const double two_pi = 2.0 * M_PI;
        double fsx = 1.0 / dx, fsy = 1.0 / dy;
        double mulx = fsx / nx, muly = fsy / ny;
        int nnx = (nx - 1) / 2 + 1;
        kx.resize(nx);
        for (int i = 0; i < nx; ++i) kx[i] = two_pi * ((double)(i < nnx ? i : i - nx) * mulx);
        ky.resize(nyc);
        for (int j = 0; j < nyc; ++j) ky[j] = two_pi * ((double)j * muly);
        // uniform, non-periodic vertical grid: dz = Lz/(Nz-1), length Nz
        dz.assign(nz, lz / (nz - 1));
        // twothirds_mask(Nx, Nyc)
        mask.assign((size_t)nx * nyc, 1);
        int kxm = nx / 3;
        for (int i = kxm; i < nx - kxm; ++i)
            for (int j = 0; j < nyc; ++j) mask[i + (size_t)nx * j] = 0;
        int kym = (2 * nyc) / 3;
        for (int j = kym; j < nyc; ++j)
            for (int i = 0; i < nx; ++i) mask[i + (size_t)nx * j] = 0;
        mask_ext = mask;
        if (kxm > 0 && mask[nx - kxm]) mask_ext[kxm] = 1;
        px.init(nx);
        py.init(ny);
    }
    size_t n2() const { return (size_t)nx * ny; }
    size_t c2() const { return (size_t)nx * nyc; }
};

// rfft_2d!: RFFT along y then FFT along x, unnormalised.
// par = false runs serially (the caller parallelises over planes).
void rfft2(const Grid& g, const double* in, cd* out, bool par = true) {
#pragma omp parallel if (par)
    {
        // two real columns per complex transform: z = c0 + i c1,
        // C0[k] = (Z[k] + conj Z[-k]) / 2, C1[k] = (Z[k] - conj Z[-k]) / 2i
        // columns are gathered kB pairs at a time, so that rows are read a
        // cache line at a time
        constexpr int kB = 4;
        std::vector<cd> col((size_t)kB * g.ny);
        const int npair = (g.nx + 1) / 2;
        const int nblk = (npair + kB - 1) / kB;
#pragma omp for schedule(static)
        for (int bk = 0; bk < nblk; ++bk) {
            const int p0 = bk * kB, np = std::min(kB, npair - p0);
            for (int y = 0; y < g.ny; ++y) {
                const double* row = in + (size_t)g.nx * y;
                for (int q = 0; q < np; ++q) {
                    const int x0 = 2 * (p0 + q);
                    col[(size_t)q * g.ny + y] = cd(row[x0], x0 + 1 < g.nx ? row[x0 + 1] : 0.0);
                }
            }
            for (int q = 0; q < np; ++q) g.py.run(col.data() + (size_t)q * g.ny, -1);
            for (int j = 0; j < g.nyc; ++j) {
                cd* orow = out + (size_t)g.nx * j;
                for (int q = 0; q < np; ++q) {
                    const cd* c = col.data() + (size_t)q * g.ny;
                    const int x0 = 2 * (p0 + q);
                    const cd zk = c[j], zm = std::conj(c[(g.ny - j) % g.ny]);
                    orow[x0] = 0.5 * (zk + zm);
                    if (x0 + 1 < g.nx) orow[x0 + 1] = cd(0.0, -0.5) * (zk - zm);
                }
            }
        }
#pragma omp for schedule(static)
        for (int j = 0; j < g.nyc; ++j) g.px.run(out + (size_t)g.nx * j, -1);
    }
}

// irfft_2d!: inverse FFT along x, then complex-to-real along y (imaginary parts
// of the ky = 0 and ky = Ny/2 bins ignored), scaled by 1/(Nx*Ny).
void irfft2(const Grid& g, const cd* in, double* out, bool par = true) {
    std::vector<cd> tmp(in, in + g.c2());
    const double scale = 1.0 / ((double)g.nx * (double)g.ny);
#pragma omp parallel if (par)
    {
#pragma omp for schedule(static)
        for (int j = 0; j < g.nyc; ++j) g.px.run(tmp.data() + (size_t)g.nx * j, +1);
        // two columns per complex transform: the Hermitian spectra H0, H1 of
        // real columns combine to Z = H0 + i H1, whose inverse is c0 + i c1
        // kB pairs at a time, so that rows are read and written a cache line
        // at a time
        constexpr int kB = 4;
        const int npair = (g.nx + 1) / 2;
        const int nblk = (npair + kB - 1) / kB;
        std::vector<cd> h((size_t)2 * kB * g.nyc), zc((size_t)kB * g.ny);
#pragma omp for schedule(static)
        for (int bk = 0; bk < nblk; ++bk) {
            const int p0 = bk * kB, np = std::min(kB, npair - p0);
            for (int j = 0; j < g.nyc; ++j) {
                const cd* row = tmp.data() + (size_t)g.nx * j;
                for (int q = 0; q < np; ++q) {
                    const int x0 = 2 * (p0 + q);
                    h[(size_t)(2 * q) * g.nyc + j] = row[x0];
                    h[(size_t)(2 * q + 1) * g.nyc + j] = x0 + 1 < g.nx ? row[x0 + 1] : cd(0.0, 0.0);
                }
            }
            const cd I(0.0, 1.0);
            for (int q = 0; q < np; ++q) {
                cd* h0 = h.data() + (size_t)(2 * q) * g.nyc;
                cd* h1 = h0 + g.nyc;
                cd* c = zc.data() + (size_t)q * g.ny;
                // c2r ignores the imaginary parts of the ky = 0 and ky = Ny/2 bins
                h0[0] = cd(h0[0].real(), 0.0);
                h1[0] = cd(h1[0].real(), 0.0);
                if (g.ny % 2 == 0) {
                    h0[g.ny / 2] = cd(h0[g.ny / 2].real(), 0.0);
                    h1[g.ny / 2] = cd(h1[g.ny / 2].real(), 0.0);
                }
                for (int j = 0; j < g.nyc; ++j) c[j] = h0[j] + I * h1[j];
                for (int j = 1; j < g.nyc; ++j)
                    if (g.ny - j != j && g.ny - j < g.ny) c[g.ny - j] = std::conj(h0[j]) + I * std::conj(h1[j]);
                g.py.run(c, +1);
            }
            for (int y = 0; y < g.ny; ++y) {
                double* orow = out + (size_t)g.nx * y;
                for (int q = 0; q < np; ++q) {
                    const int x0 = 2 * (p0 + q);
                    const cd v = zc[(size_t)q * g.ny + y];
                    orow[x0] = v.real() * scale;
                    if (x0 + 1 < g.nx) orow[x0 + 1] = v.imag() * scale;
                }
            }
        }
    }
}

// ddx_2d!, ddy_2d! (src/transforms.jl:135-166): multiply by i*kx, i*ky
void ddx(const Grid& g, const cd* a, cd* o) {
    for (int j = 0; j < g.nyc; ++j)
        for (int i = 0; i < g.nx; ++i) o[i + (size_t)g.nx * j] = cd(0.0, g.kx[i]) * a[i + (size_t)g.nx * j];
}
void ddy(const Grid& g, const cd* a, cd* o) {
    for (int j = 0; j < g.nyc; ++j)
        for (int i = 0; i < g.nx; ++i) o[i + (size_t)g.nx * j] = cd(0.0, g.ky[j]) * a[i + (size_t)g.nx * j];
}
void dealias(const Grid& g, cd* a) {
    for (size_t m = 0; m < g.c2(); ++m)
        if (!g.mask[m]) a[m] = 0.0;
}

// jacobian_2d! (src/transforms.jl:430-465), literal order of operations.
// tmp_real2 is the caller's scratch array for step 6 (null: a private one).
// timestep_ab2_ls! passes fields.tmp2 both as the output and as tmp_real2
// (src/timestep.jl:159, src/nonlinear.jl:48-50); with tmp_real2 == out, step 6
// overwrites the x-flux term and step 7 doubles the y-flux term, giving
// 2 d/dy(b d(phi)/dx), which the literal AB2 mode reproduces.
void jacobian_2d(const Grid& g, double* out, const double* a, const double* b, double* tmp_real2 = nullptr) {
    std::vector<cd> s1(g.c2()), s2(g.c2());
    std::vector<double> t1(g.n2()), t2own(tmp_real2 ? 0 : g.n2());
    double* t2 = tmp_real2 ? tmp_real2 : t2own.data();
    rfft2(g, a, s1.data());
    ddy(g, s1.data(), s2.data());
    irfft2(g, s2.data(), t1.data());
    for (size_t m = 0; m < g.n2(); ++m) t1[m] *= -1.0;
    for (size_t m = 0; m < g.n2(); ++m) t1[m] *= b[m];
    rfft2(g, t1.data(), s1.data());
    ddx(g, s1.data(), s2.data());
    irfft2(g, s2.data(), out);
    rfft2(g, a, s1.data());
    ddx(g, s1.data(), s2.data());
    irfft2(g, s2.data(), t1.data());
    for (size_t m = 0; m < g.n2(); ++m) t1[m] *= b[m];
    rfft2(g, t1.data(), s1.data());
    ddy(g, s1.data(), s2.data());
    irfft2(g, s2.data(), t2);
    for (size_t m = 0; m < g.n2(); ++m) out[m] += t2[m];
}

// compute_tendency! (src/nonlinear.jl:22-56): -J(phi, b), then dealias.
// alias_tmp2: the output array is also jacobian_2d!'s tmp_real2 (AB2's call).
void tendency(const Grid& g, double* out, const double* phi, const double* b, bool alias_tmp2 = false) {
    jacobian_2d(g, out, phi, b, alias_tmp2 ? out : nullptr);
    for (size_t m = 0; m < g.n2(); ++m) out[m] *= -1.0;
    std::vector<cd> s(g.c2());
    rfft2(g, out, s.data());
    dealias(g, s.data());
    irfft2(g, s.data(), out);
}

// exponential_transfer (src/filter.jl:119-126)
double exp_transfer(double knorm, double strength, int order, double cutoff) {
    if (knorm <= cutoff) return 1.0;
    double ratio = (knorm - cutoff) / (1.0 - cutoff);
    double p = 1.0;
    for (int q = 0; q < order; ++q) p *= ratio;
    return std::exp(-strength * p);
}

// Transfer functions of the other filter types (src/filter.jl:128-169):
// type 1 hyperviscosity exp(-nu k^{2p} dt) on |k|; 2 sharp cutoff; 3 Cesaro.
double filter_transfer(int type, double knorm, double kmag, double strength, int order, double cutoff, double dt) {
    switch (type) {
        case 1: {
            double p = 1.0;
            for (int q = 0; q < 2 * order; ++q) p *= kmag;
            return std::exp(-strength * p * dt);
        }
        case 2: return knorm <= cutoff ? 1.0 : 0.0;
        case 3: {
            if (knorm <= cutoff) return 1.0;
            if (knorm >= 1.0) return 0.0;
            double ratio = (knorm - cutoff) / (1.0 - cutoff);
            double p = 1.0;
            for (int q = 0; q < order; ++q) p *= (1.0 - ratio);
            return p;
        }
        default: return exp_transfer(knorm, strength, order, cutoff);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Solver state: mirrors SemiGeostrophicProblem / Fields / TimeState
// ---------------------------------------------------------------------------
extern "C" {

typedef struct or_config {
    int32_t nx, ny, nz;
    int32_t scheme;          // 0 AB2 (AB2_LowStorage), 1 RK3
    double lx, ly, lz;
    double eps;
    double dt;
    int32_t filter_freq;
    int32_t filter_order;
    double filter_strength;
    double filter_cutoff;
    double ma_tol;
    int32_t ma_maxiter;
    int32_t ma_per_stage;    // 1: solve Monge-Ampere before every tendency
    int32_t ma_rhs_mode;     // 0: dPhi/dz = b_s on top; 1: b_s as a volume RHS
    int32_t ma_predictor;    // 0: previous solution; 1: linear, 2: quadratic, 3: cubic extrapolation
    int32_t filter_type;     // 0 exponential, 1 hyperviscosity, 2 cutoff, 3 Cesaro
    int32_t ab2_literal_alias;  // 1: AB2's tendency with the tmp2 aliasing of src/timestep.jl:159
    int32_t ma_bc_guess;        // 1: the predictor's guess corrected for the current b_s (surface RHS)
    int32_t pad2;
} or_config;

typedef struct or_stats {
    int32_t last_iters;
    int32_t total_iters;
    int32_t max_iters;
    int32_t solves;
    int32_t unconverged;
    int32_t pad0;
    double last_update;
    double max_update;
} or_stats;

}  // extern "C"

namespace {

struct Oracle {
    or_config cfg{};
    Grid g;
    // Fields (src/fields.jl:28-60) -- physical surface fields
    std::vector<double> bs, phis, dbdt_old, b_stage, k1, k2, k3, tmp2;
    // Monge-Ampere unknown, spectral (nx * nyc * nz), 2/3-masked, and the
    // previous solution for the predictor
    std::vector<cd> Phat, Pprev, Pprev2, Pprev3;
    int nhist = 0;
    // TimeState (src/timestep.jl:45-86)
    double t = 0.0;
    long step = 0;
    or_stats st{};
    // vertical stencil coefficients
    std::vector<double> al, be, ga;
    double ab_b = 0, bb_b = 0, cb_b = 0, at_t = 0, bt_t = 0, ct_t = 0;

    void init(const or_config& c) {
        cfg = c;
        g.init(c.nx, c.ny, c.nz, c.lx, c.ly, c.lz);
        size_t n2 = g.n2();
        bs.assign(n2, 0.0); phis.assign(n2, 0.0); dbdt_old.assign(n2, 0.0);
        b_stage.assign(n2, 0.0); k1.assign(n2, 0.0); k2.assign(n2, 0.0); k3.assign(n2, 0.0);
        tmp2.assign(n2, 0.0);
        Phat.assign(g.c2() * g.nz, cd(0, 0));
        Pprev.assign(g.c2() * g.nz, cd(0, 0));
        Pprev2.assign(g.c2() * g.nz, cd(0, 0));
        Pprev3.assign(g.c2() * g.nz, cd(0, 0));
        set_vertical();
    }

    // d2dz2! rows and Neumann rows from g.dz (make_vertical_grid's spacing vector)
    void set_vertical() {
        // d2dz2! coefficients (src/transforms.jl:812-818), 0-based plane k
        al.assign(g.nz, 0); be.assign(g.nz, 0); ga.assign(g.nz, 0);
        for (int k = 1; k < g.nz - 1; ++k) {
            double dzm = g.dz[k - 1], dzp = g.dz[k];
            al[k] = 2.0 / (dzm * (dzm + dzp));
            be[k] = -2.0 / (dzm * dzp);
            ga[k] = 2.0 / (dzp * (dzm + dzp));
        }
        // apply_neumann_bottom! (src/poisson.jl:345-364): h1 = dz[1], h2 = dz[2]
        {
            double h1 = g.dz[0], h2 = g.dz[1], a = h1 + h2;
            ab_b = -(2 * h1 + h2) / (h1 * a);
            bb_b = a / (h1 * h2);
            cb_b = -h1 / (h2 * a);
        }
        // apply_neumann_surface! (src/poisson.jl:309-339): h1 = dz[Nz-1], h2 = dz[Nz-2]
        {
            int k = g.nz - 1;
            double h1 = g.dz[k - 1], h2 = g.dz[k - 2], a = h1 + h2;
            at_t = (2 * h1 + h2) / (h1 * a);
            bt_t = -a / (h1 * h2);
            ct_t = h1 / (h2 * a);
        }
    }

    // Phi_xx Phi_yy - Phi_xy^2 on one plane from its masked spectrum
    // (compute_d_operator!, src/poisson.jl:183-223)
    // Serial within the plane: ma_iteration runs planes in parallel.
    void d_operator_plane(const cd* P, double* D) {
        size_t c2 = g.c2(), n2 = g.n2();
        std::vector<cd> s(c2), s2(c2);
        std::vector<double> xx(n2), yy(n2), xy(n2);
        ddx(g, P, s.data()); ddy(g, s.data(), s2.data()); irfft2(g, s2.data(), xy.data(), false);
        ddx(g, P, s.data()); ddx(g, s.data(), s2.data()); irfft2(g, s2.data(), xx.data(), false);
        ddy(g, P, s.data()); ddy(g, s.data(), s2.data()); irfft2(g, s2.data(), yy.data(), false);
        for (size_t m = 0; m < n2; ++m) D[m] = xx[m] * yy[m] - xy[m] * xy[m];
    }

    // One fixed-point iteration; returns relative update.
    double ma_iteration(const std::vector<cd>& bsh) {
        const int nz = g.nz;
        const size_t c2 = g.c2();
        std::vector<cd> R(c2 * nz, cd(0, 0));
        // the interior planes are independent: one plane per thread at a time
#pragma omp parallel
        {
            std::vector<double> D(g.n2());
#pragma omp for schedule(dynamic, 1)
            for (int k = 1; k < nz - 1; ++k) {
                d_operator_plane(&Phat[c2 * k], D.data());
                rfft2(g, D.data(), &R[c2 * k], false);
                cd* Rk = &R[c2 * k];
                for (size_t m = 0; m < c2; ++m) {
                    Rk[m] = g.mask_ext[m] ? cfg.eps * Rk[m] : cd(0, 0);
                    if (cfg.ma_rhs_mode == 1 && g.mask_ext[m]) Rk[m] += bsh[m];
                }
            }
        }
        double dsum = 0.0, nsum = 0.0;
        const int n = nz - 2;
#pragma omp parallel reduction(+ : dsum, nsum)
        {
            std::vector<double> cp(n);
            std::vector<cd> dp(n), x(n);
#pragma omp for schedule(static)
            for (int j = 0; j < g.nyc; ++j) {
                for (int i = 0; i < g.nx; ++i) {
                    size_t m = i + (size_t)g.nx * j;
                    double w = (j == 0) ? 1.0 : 2.0;
                    if (!g.mask_ext[m] || m == 0) {
                        for (int k = 0; k < nz; ++k) {
                            cd old = Phat[m + c2 * k];
                            dsum += w * std::norm(old);
                            Phat[m + c2 * k] = 0.0;
                        }
                        continue;
                    }
                    double K2 = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j];
                    cd bc = (cfg.ma_rhs_mode == 0) ? bsh[m] : cd(0, 0);
                    // Thomas on interior planes 1..nz-2 with Neumann rows eliminated
                    for (int q = 0; q < n; ++q) {
                        int k = q + 1;
                        double lo = al[k], dg = be[k] - K2, up = ga[k];
                        cd r = R[m + c2 * k];
                        if (q == 0) { dg -= al[k] * bb_b / ab_b; up -= al[k] * cb_b / ab_b; lo = 0.0; }
                        if (q == n - 1) { lo -= ga[k] * ct_t / at_t; dg -= ga[k] * bt_t / at_t; r -= ga[k] * bc / at_t; up = 0.0; }
                        if (q == 0) {
                            double inv = 1.0 / dg;
                            cp[q] = up * inv;
                            dp[q] = r * inv;
                        } else {
                            double inv = 1.0 / (dg - lo * cp[q - 1]);
                            cp[q] = up * inv;
                            dp[q] = (r - lo * dp[q - 1]) * inv;
                        }
                    }
                    x[n - 1] = dp[n - 1];
                    for (int q = n - 2; q >= 0; --q) x[q] = dp[q] - cp[q] * x[q + 1];
                    cd p0 = -(bb_b * x[0] + cb_b * x[1]) / ab_b;
                    cd pt = (bc - bt_t * x[n - 1] - ct_t * x[n - 2]) / at_t;
                    for (int k = 0; k < nz; ++k) {
                        cd nv = (k == 0) ? p0 : (k == nz - 1) ? pt : x[k - 1];
                        cd d = nv - Phat[m + c2 * k];
                        dsum += w * std::norm(d);
                        nsum += w * std::norm(nv);
                        Phat[m + c2 * k] = nv;
                    }
                }
            }
        }
        return nsum > 0 ? std::sqrt(dsum / nsum) : std::sqrt(dsum);
    }

    // Boundary correction of a predicted guess G (not in the reference, whose
    // solves start from the previous potential): the solution depends on b_s
    // only through the top Neumann row, linearly, so the mismatch
    // delta = b_hat - (at G[Nz] + bt G[Nz-1] + ct G[Nz-2]) between the guess's top
    // row and the current buoyancy is removed exactly by adding the solution
    // of L x = [0 ; delta], the same per-mode tridiagonal system as the
    // iteration's with only the top row's right-hand side non-zero.
    void bc_correct(std::vector<cd>& G, const std::vector<cd>& bsh) {
        const int nz = g.nz, n = nz - 2;
        const size_t c2 = g.c2();
#pragma omp parallel for schedule(static)
        for (int j = 0; j < g.nyc; ++j) {
            std::vector<double> cp(n);
            std::vector<cd> x(n);
            for (int i = 0; i < g.nx; ++i) {
                size_t m = i + (size_t)g.nx * j;
                if (!g.mask_ext[m] || m == 0) continue;
                const cd top = at_t * G[m + c2 * (nz - 1)] + bt_t * G[m + c2 * (nz - 2)] + ct_t * G[m + c2 * (nz - 3)];
                const cd dlt = bsh[m] - top;
                const double K2 = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j];
                cd dp_last = 0;
                for (int q = 0; q < n; ++q) {
                    const int k = q + 1;
                    double lo = al[k], dg = be[k] - K2, up = ga[k];
                    cd r = 0;
                    if (q == 0) { dg -= al[k] * bb_b / ab_b; up -= al[k] * cb_b / ab_b; lo = 0.0; }
                    if (q == n - 1) { lo -= ga[k] * ct_t / at_t; dg -= ga[k] * bt_t / at_t; r -= ga[k] * dlt / at_t; up = 0.0; }
                    const double inv = (q == 0) ? 1.0 / dg : 1.0 / (dg - lo * cp[q - 1]);
                    cp[q] = up * inv;
                    if (q == n - 1) dp_last = r * inv;
                }
                x[n - 1] = dp_last;
                for (int q = n - 2; q >= 0; --q) x[q] = -cp[q] * x[q + 1];
                const cd p0 = -(bb_b * x[0] + cb_b * x[1]) / ab_b;
                const cd pt = (dlt - bt_t * x[n - 1] - ct_t * x[n - 2]) / at_t;
                for (int k = 0; k < nz; ++k) G[m + c2 * k] += (k == 0) ? p0 : (k == nz - 1) ? pt : x[k - 1];
            }
        }
    }

    // solve_monge_ampere_fields! with the documented problem; returns converged
    bool ma_solve(int* iters_out, double* upd_out) {
        std::vector<cd> bsh(g.c2());
        rfft2(g, bs.data(), bsh.data());
        for (size_t m = 0; m < g.c2(); ++m)
            if (!g.mask_ext[m]) bsh[m] = 0.0;
        bsh[0] = 0.0;
        // initial guess: polynomial extrapolation of order ma_predictor through
        // the last solutions (equally spaced solves); history newest first
        if (cfg.ma_predictor >= 1) {
            std::vector<cd>* S[4] = {&Phat, &Pprev, &Pprev2, &Pprev3};
            const int cap = cfg.ma_predictor + 1, h = nhist;
            if (h >= 1) {
                const int t = h < cap ? h : cap - 1;
                const int order = std::min(cfg.ma_predictor, h - 1);
                const std::vector<cd>&a = *S[0], &b = *S[1], &c = *S[2], &e = *S[3];
                std::vector<cd> guess(a.size());
                for (size_t m = 0; m < a.size(); ++m) {
                    switch (order) {
                        case 0: guess[m] = a[m]; break;
                        case 1: guess[m] = 2.0 * a[m] - b[m]; break;
                        case 2: guess[m] = 3.0 * (a[m] - b[m]) + c[m]; break;
                        default: guess[m] = 4.0 * (a[m] + c[m]) - (6.0 * b[m] + e[m]); break;
                    }
                }
                if (cfg.ma_bc_guess && cfg.ma_rhs_mode == 0) bc_correct(guess, bsh);
                *S[t] = std::move(guess);
                for (int i = t; i > 0; --i) std::swap(*S[i], *S[i - 1]);
            }
            nhist = h < cap ? h + 1 : cap;
        }
        double upd = 0.0;
        int it = 0;
        bool conv = false;
        for (it = 1; it <= cfg.ma_maxiter; ++it) {
            upd = ma_iteration(bsh);
            if (!(upd == upd)) break;
            if (upd <= cfg.ma_tol) { conv = true; break; }
        }
        if (it > cfg.ma_maxiter) it = cfg.ma_maxiter;
        // extract_surface_to_2d!: phi_s = Phi[:,:,Nz]
        irfft2(g, &Phat[g.c2() * (g.nz - 1)], phis.data());
        st.last_iters = it;
        st.total_iters += it;
        st.max_iters = std::max(st.max_iters, it);
        st.solves += 1;
        st.last_update = upd;
        st.max_update = std::max(st.max_update, upd);
        if (!conv) st.unconverged += 1;
        if (iters_out) *iters_out = it;
        if (upd_out) *upd_out = upd;
        return conv;
    }

    void compute_tendency(std::vector<double>& out, bool alias_tmp2 = false) {
        tendency(g, out.data(), phis.data(), bs.data(), alias_tmp2);
    }

    // timestep_ab2_ls! (src/timestep.jl:152-190); compute_tendency!(fields.tmp2,
    // ...) makes tmp2 the Jacobian's output and its scratch at once (:159)
    void ab2(double dt) {
        compute_tendency(tmp2, cfg.ab2_literal_alias != 0);
        size_t n2 = g.n2();
        if (step == 0) {
            for (size_t m = 0; m < n2; ++m) bs[m] += dt * tmp2[m];
        } else {
            for (size_t m = 0; m < n2; ++m) bs[m] += dt * (1.5 * tmp2[m] - 0.5 * dbdt_old[m]);
        }
        dbdt_old = tmp2;
        t += dt;
        step += 1;
    }

    // timestep_rk3! (src/timestep.jl:195-242); with ma_per_stage the streamfunction
    // is re-solved from each stage buoyancy before its tendency.
    void rk3(double dt) {
        size_t n2 = g.n2();
        b_stage = bs;
        compute_tendency(k1);
        for (size_t m = 0; m < n2; ++m) bs[m] = b_stage[m] + (dt / 3.0) * k1[m];
        if (cfg.ma_per_stage) ma_solve(nullptr, nullptr);
        compute_tendency(k2);
        for (size_t m = 0; m < n2; ++m) bs[m] = b_stage[m] + (2.0 * dt / 3.0) * k2[m];
        if (cfg.ma_per_stage) ma_solve(nullptr, nullptr);
        compute_tendency(k3);
        for (size_t m = 0; m < n2; ++m) bs[m] = b_stage[m] + (dt / 4.0) * (k1[m] + 3.0 * k3[m]);
        t += dt;
        step += 1;
    }

    // apply_spectral_filter! (src/timestep.jl:247-260 -> src/filter.jl:283-309)
    void filter() {
        std::vector<cd> s(g.c2());
        rfft2(g, bs.data(), s.data());
        double kmx = M_PI / g.dx, kmy = M_PI / g.dy;
        double kmax = std::sqrt(kmx * kmx + kmy * kmy);
        for (int j = 0; j < g.nyc; ++j)
            for (int i = 0; i < g.nx; ++i) {
                double kmag = std::sqrt(g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j]);
                s[i + (size_t)g.nx * j] *= filter_transfer(cfg.filter_type, kmag / kmax, kmag, cfg.filter_strength,
                                                           cfg.filter_order, cfg.filter_cutoff, cfg.dt);
            }
        irfft2(g, s.data(), bs.data());
    }

    // timestep! (src/timestep.jl:267-285) followed, when the streamfunction is
    // re-solved per stage, by the solve for the new buoyancy.
    void timestep(double dt) {
        if (cfg.scheme == 0) ab2(dt); else rk3(dt);
        if (cfg.filter_freq > 0 && step % cfg.filter_freq == 0) filter();
        if (cfg.ma_per_stage) ma_solve(nullptr, nullptr);
    }

    // set_b! (src/setICs.jl:21-57): zero mean, dealias, solve.
    bool set_b(const double* b, int* iters, double* upd) {
        std::vector<cd> s(g.c2());
        rfft2(g, b, s.data());
        s[0] = 0.0;
        dealias(g, s.data());
        irfft2(g, s.data(), bs.data());
        std::fill(Phat.begin(), Phat.end(), cd(0, 0));
        nhist = 0;
        return ma_solve(iters, upd);
    }
};

}  // namespace

extern "C" {

// Domain.dz of a stretched or custom vertical grid (src/domain.jl:238-280)
int or_set_dz(void* h, const double* dz) {
    Oracle* o = static_cast<Oracle*>(h);
    o->g.dz.assign(dz, dz + o->g.nz);
    o->set_vertical();
    return 0;
}

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void* or_create(const or_config* c) {
    if (!c || c->nx < 4 || c->ny < 4 || c->nz < 4) return nullptr;
    Oracle* o = new Oracle();
    o->init(*c);
    return o;
}

void or_destroy(void* h) { delete static_cast<Oracle*>(h); }

int or_set_b(void* h, const double* b, int* iters, double* upd) {
    return static_cast<Oracle*>(h)->set_b(b, iters, upd) ? 0 : 1;
}

int or_solve_ma(void* h, int* iters, double* upd) {
    return static_cast<Oracle*>(h)->ma_solve(iters, upd) ? 0 : 1;
}

// nsteps calls of timestep!; dt <= 0 uses the configured dt
int or_step(void* h, int nsteps, double dt) {
    Oracle* o = static_cast<Oracle*>(h);
    double d = dt > 0 ? dt : o->cfg.dt;
    for (int s = 0; s < nsteps; ++s) o->timestep(d);
    return 0;
}

void or_get_stats(void* h, or_stats* s) { *s = static_cast<Oracle*>(h)->st; }

void or_get_time(void* h, double* t, long* step) {
    Oracle* o = static_cast<Oracle*>(h);
    *t = o->t;
    *step = o->step;
}

// field ids: 0 b_s, 1 phi_s, 2 Phi (3-D, physical), 3 db_dt_old, 4 u_s, 5 v_s
int or_get_field(void* h, int id, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    const Grid& g = o->g;
    size_t n2 = g.n2();
    switch (id) {
        case 0: std::memcpy(out, o->bs.data(), n2 * sizeof(double)); return 0;
        case 1: std::memcpy(out, o->phis.data(), n2 * sizeof(double)); return 0;
        case 2:
            for (int k = 0; k < g.nz; ++k) irfft2(g, &o->Phat[g.c2() * k], out + n2 * k);
            return 0;
        case 3: std::memcpy(out, o->dbdt_old.data(), n2 * sizeof(double)); return 0;
        case 4: case 5: {
            // compute_surface_geostrophic_velocities! (src/setICs.jl:161-192)
            std::vector<cd> s(g.c2()), s2(g.c2());
            rfft2(g, o->phis.data(), s.data());
            if (id == 4) {
                ddy(g, s.data(), s2.data());
                irfft2(g, s2.data(), out);
                for (size_t m = 0; m < n2; ++m) out[m] = -out[m];
            } else {
                ddx(g, s.data(), s2.data());
                irfft2(g, s2.data(), out);
            }
            return 0;
        }
        default: return -1;
    }
}

int or_set_field(void* h, int id, const double* in) {
    Oracle* o = static_cast<Oracle*>(h);
    size_t n2 = o->g.n2();
    switch (id) {
        case 0: std::memcpy(o->bs.data(), in, n2 * sizeof(double)); return 0;
        case 1: std::memcpy(o->phis.data(), in, n2 * sizeof(double)); return 0;
        case 3: std::memcpy(o->dbdt_old.data(), in, n2 * sizeof(double)); return 0;
        default: return -1;
    }
}

void or_set_time(void* h, double t, long step) {
    Oracle* o = static_cast<Oracle*>(h);
    o->t = t;
    o->step = step;
}

// ---- primitives for unit tests ------------------------------------------------

// rfft_2d!: out is interleaved complex, nx * (ny/2+1), x fastest
void or_rfft2(int nx, int ny, const double* in, double* out) {
    Grid g; g.init(nx, ny, 4, 2 * M_PI, 2 * M_PI, 1.0);
    rfft2(g, in, reinterpret_cast<cd*>(out));
}

void or_irfft2(int nx, int ny, const double* in, double* out) {
    Grid g; g.init(nx, ny, 4, 2 * M_PI, 2 * M_PI, 1.0);
    irfft2(g, reinterpret_cast<const cd*>(in), out);
}

void or_jacobian(void* h, const double* phi, const double* b, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    jacobian_2d(o->g, out, phi, b);
}

void or_tendency(void* h, const double* phi, const double* b, double* out) {
    Oracle* o = static_cast<Oracle*>(h);
    tendency(o->g, out, phi, b);
}

double or_exponential_transfer(double knorm, double strength, int order, double cutoff) {
    return exp_transfer(knorm, strength, order, cutoff);
}

// apply_spectral_filter! on a caller array (b is filtered in place)
void or_filter(void* h, double* b) {
    Oracle* o = static_cast<Oracle*>(h);
    std::vector<double> save = o->bs;
    std::memcpy(o->bs.data(), b, o->g.n2() * sizeof(double));
    o->filter();
    std::memcpy(b, o->bs.data(), o->g.n2() * sizeof(double));
    o->bs = save;
}

// Grid tables for cross-checks: kx (nx), ky (nyc), mask (nx*nyc bytes)
void or_grid_tables(void* h, double* kx, double* ky, uint8_t* mask) {
    Oracle* o = static_cast<Oracle*>(h);
    std::memcpy(kx, o->g.kx.data(), o->g.nx * sizeof(double));
    std::memcpy(ky, o->g.ky.data(), o->g.nyc * sizeof(double));
    std::memcpy(mask, o->g.mask.data(), o->g.c2());
}

// compute_ssg_residual! in its literal form (src/poisson.jl:228-253 with
// compute_3d_laplacian! :143-178, compute_d_operator! :183-223, d2dz2!
// src/transforms.jl:798-826 and apply_ssg_boundary_conditions! :262-302).
// Phi (3-D physical, modified on planes 1 and Nz by the boundary rows),
// rhs (3-D physical), bs_surface (2-D), r (3-D output).  The horizontal
// derivatives go through rfft/irfft of each plane as the reference does.
void or_ssg_residual_literal(void* h, double* Phi, const double* rhs, const double* bs_surface, double eps, double* r) {
    Oracle* o = static_cast<Oracle*>(h);
    const Grid& g = o->g;
    size_t n2 = g.n2(), c2 = g.c2();
    int nz = g.nz;
    std::vector<cd> P(c2), s(c2), s2(c2);
    std::vector<double> xx(n2), yy(n2), xy(n2), zz(n2 * nz, 0.0);
    for (int k = 1; k < nz - 1; ++k)
        for (size_t m = 0; m < n2; ++m)
            zz[m + n2 * k] = o->al[k] * Phi[m + n2 * (k - 1)] + o->be[k] * Phi[m + n2 * k] + o->ga[k] * Phi[m + n2 * (k + 1)];
    for (int k = 0; k < nz; ++k) {
        rfft2(g, Phi + n2 * k, P.data());
        ddx(g, P.data(), s.data()); ddx(g, s.data(), s2.data()); irfft2(g, s2.data(), xx.data());
        ddy(g, P.data(), s.data()); ddy(g, s.data(), s2.data()); irfft2(g, s2.data(), yy.data());
        std::vector<double> lap(n2);
        for (size_t m = 0; m < n2; ++m) lap[m] = xx[m] + yy[m] + zz[m + n2 * k];
        ddx(g, P.data(), s.data()); ddy(g, s.data(), s2.data()); irfft2(g, s2.data(), xy.data());
        for (size_t m = 0; m < n2; ++m) {
            double D = xx[m] * yy[m] - xy[m] * xy[m];
            r[m + n2 * k] = lap[m] - eps * D - rhs[m + n2 * k];
        }
    }
    // boundary rows on Phi, zero residual there
    for (size_t m = 0; m < n2; ++m) {
        int k = nz - 1;
        Phi[m + n2 * k] = (bs_surface[m] - o->bt_t * Phi[m + n2 * (k - 1)] - o->ct_t * Phi[m + n2 * (k - 2)]) / o->at_t;
        r[m + n2 * k] = 0.0;
        Phi[m] = -(o->bb_b * Phi[m + n2] + o->cb_b * Phi[m + 2 * n2]) / o->ab_b;
        r[m] = 0.0;
    }
}

}  // extern "C"

// ===========================================================================
// The reference's own multigrid (src/poisson.jl:33-959), restated literally:
// SSGLevel fields on physical grids, compute_ssg_residual! with its boundary
// side effects, the spectral and red-black SOR smoothers, injection
// transfers, the V-cycle and solve_ssg_equation.  As algorithms they diverge
// or stay inert; as functions they are what the GPU's ssg_mg_* entry points
// reproduce.
// ===========================================================================
namespace {

struct MgLevel {
    Grid g;
    std::vector<double> Phi, b, r, Phi_old, bs, Phi_zz;  // Phi_zz keeps its boundary planes at 0
    void init(int nx, int ny, int nz, double lx, double ly, double lz) {
        g.init(nx, ny, nz, lx, ly, lz);
        size_t n3 = g.n2() * nz;
        Phi.assign(n3, 0.0); b.assign(n3, 0.0); r.assign(n3, 0.0); Phi_old.assign(n3, 0.0);
        Phi_zz.assign(n3, 0.0); bs.assign(g.n2(), 0.0);
    }
};

// create_coarse_domain (src/coarse_domain.jl:26-32): halve, at least 5, even
int coarsen(int n) {
    int c = std::max(n / 2, 5);
    return c % 2 == 0 ? c : c + 1;
}

struct Mg {
    std::vector<MgLevel> lv;
    double al_[64], be_[64], ga_[64];
};

void mg_zcoefs(const Grid& g, std::vector<double>& al, std::vector<double>& be, std::vector<double>& ga) {
    al.assign(g.nz, 0); be.assign(g.nz, 0); ga.assign(g.nz, 0);
    for (int k = 1; k < g.nz - 1; ++k) {
        double dzm = g.dz[k - 1], dzp = g.dz[k];
        al[k] = 2.0 / (dzm * (dzm + dzp));
        be[k] = -2.0 / (dzm * dzp);
        ga[k] = 2.0 / (dzp * (dzm + dzp));
    }
}

// apply_ssg_boundary_conditions! (src/poisson.jl:262-364), nz >= 3 branch
void mg_bc(MgLevel& L) {
    const Grid& g = L.g;
    size_t n2 = g.n2();
    int nz = g.nz;
    double h1 = g.dz[nz - 2], h2 = g.dz[nz - 3], a = h1 + h2;
    double at = (2 * h1 + h2) / (h1 * a), bt = -a / (h1 * h2), ct = h1 / (h2 * a);
    double g1 = g.dz[0], g2 = g.dz[1], ga2 = g1 + g2;
    double ab = -(2 * g1 + g2) / (g1 * ga2), bb = ga2 / (g1 * g2), cb = -g1 / (g2 * ga2);
    for (size_t m = 0; m < n2; ++m) {
        int k = nz - 1;
        L.Phi[m + n2 * k] = (L.bs[m] - bt * L.Phi[m + n2 * (k - 1)] - ct * L.Phi[m + n2 * (k - 2)]) / at;
        L.r[m + n2 * k] = 0.0;
        L.Phi[m] = -(bb * L.Phi[m + n2] + cb * L.Phi[m + 2 * n2]) / ab;
        L.r[m] = 0.0;
    }
}

// compute_ssg_residual! (src/poisson.jl:228-253): r = lap Phi - eps D Phi - b
void mg_residual(MgLevel& L, double eps) {
    const Grid& g = L.g;
    size_t n2 = g.n2(), c2 = g.c2();
    int nz = g.nz;
    std::vector<double> al, be, ga;
    mg_zcoefs(g, al, be, ga);
    for (int k = 1; k < nz - 1; ++k)
        for (size_t m = 0; m < n2; ++m)
            L.Phi_zz[m + n2 * k] = al[k] * L.Phi[m + n2 * (k - 1)] + be[k] * L.Phi[m + n2 * k] + ga[k] * L.Phi[m + n2 * (k + 1)];
    std::vector<cd> P(c2), s(c2), s2(c2);
    std::vector<double> xx(n2), yy(n2), xy(n2);
    for (int k = 0; k < nz; ++k) {
        rfft2(g, &L.Phi[n2 * k], P.data());
        ddx(g, P.data(), s.data()); ddx(g, s.data(), s2.data()); irfft2(g, s2.data(), xx.data());
        ddy(g, P.data(), s.data()); ddy(g, s.data(), s2.data()); irfft2(g, s2.data(), yy.data());
        ddx(g, P.data(), s.data()); ddy(g, s.data(), s2.data()); irfft2(g, s2.data(), xy.data());
        for (size_t m = 0; m < n2; ++m) {
            double lap = xx[m] + yy[m] + L.Phi_zz[m + n2 * k];
            double D = xx[m] * yy[m] - xy[m] * xy[m];
            L.r[m + n2 * k] = lap - eps * D - L.b[m + n2 * k];
        }
    }
    mg_bc(L);
}

// ssg_spectral_smoother! (src/poisson.jl:635-697)
void mg_spectral(MgLevel& L, int iters, double omega, double eps) {
    const Grid& g = L.g;
    size_t n2 = g.n2(), c2 = g.c2();
    std::vector<cd> rh(c2), ph(c2);
    for (int it = 0; it < iters; ++it) {
        mg_residual(L, eps);
        for (int k = 0; k < g.nz; ++k) {
            rfft2(g, &L.r[n2 * k], rh.data());
            rfft2(g, &L.Phi[n2 * k], ph.data());
            for (int j = 0; j < g.nyc; ++j)
                for (int i = 0; i < g.nx; ++i) {
                    size_t m = i + (size_t)g.nx * j;
                    double ksq = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j];
                    if (ksq > 1e-14) {
                        double epsf = eps * ksq;
                        double pre = 1.0 / (ksq + epsf + 1e-12);
                        ph[m] += omega * (rh[m] * pre);
                    }
                }
            dealias(g, ph.data());
            irfft2(g, ph.data(), &L.Phi[n2 * k]);
        }
        mg_bc(L);
    }
}

// Per-plane rows of the red-black SOR sweeps (0-based plane index).
// ssg_sor_smoother! (src/poisson.jl:402-482) and ssg_sor_smoother_enhanced!
// without metrics (:488-591) use the d2dz2! rows of dz as they are, with a
// relaxation factor of 1; the enhanced smoother with metrics scales the rows
// of planes 3..Nz-2 (1-based) by min(0.9, 5/ratio) where the spacing ratio
// max(dz[k], dz[k-1]) / min(...) exceeds 5, and the relaxation of planes
// 2..Nz-1 by min(1, 3/ratio) where it exceeds 3.
struct SorRows {
    std::vector<double> a, b, c, w;
};

SorRows mg_sor_rows(const Grid& g, bool metrics) {
    int nz = g.nz;
    SorRows R;
    R.a.assign(nz, 0); R.b.assign(nz, 0); R.c.assign(nz, 0); R.w.assign(nz, 1.0);
    const std::vector<double>& dz = g.dz;
    for (int k = 2; k <= nz - 1; ++k) {
        double hb = dz[k - 2], ha = dz[k - 1], ht = hb + ha;
        double a = 2.0 / (hb * ht), bta = -2.0 / (hb * ha), gm = 2.0 / (ha * ht);
        if (metrics && k > 2 && k < nz - 1) {
            double ratio = std::max(dz[k - 1], dz[k - 2]) / std::min(dz[k - 1], dz[k - 2]);
            if (ratio > 5.0) {
                double sf = std::min(0.9, 5.0 / ratio);
                a *= sf;
                bta *= sf;
                gm *= sf;
            }
        }
        if (metrics) {
            double ratio = std::max(dz[k - 1], dz[k - 2]) / std::min(dz[k - 1], dz[k - 2]);
            if (ratio > 3.0) R.w[k - 1] = std::min(1.0, 3.0 / ratio);
        }
        R.a[k - 1] = a; R.b[k - 1] = bta; R.c[k - 1] = gm;
    }
    return R;
}

// Red-black Gauss-Seidel on interior points 2..N-1 (1-based), ignoring the
// RHS.  plain: ssg_sor_smoother! (diagonal carries -0.1 eps); otherwise
// ssg_sor_smoother_enhanced! (no linearisation term) with or without metrics.
void mg_sor(MgLevel& L, int iters, double omega, double eps, bool plain, bool metrics) {
    const Grid& g = L.g;
    int nx = g.nx, ny = g.ny, nz = g.nz;
    size_t n2 = g.n2();
    double dx = g.dx, dy = g.dy;
    double idx2 = 1 / (dx * dx), idy2 = 1 / (dy * dy);
    const SorRows R = mg_sor_rows(g, metrics);
    for (int it = 0; it < iters; ++it) {
        for (int color = 0; color <= 1; ++color) {
            for (int k = 2; k <= nz - 1; ++k)
                for (int j = 2; j <= ny - 1; ++j)
                    for (int i = 2; i <= nx - 1; ++i) {
                        if ((i + j + k) % 2 != color) continue;
                        auto at = [&](int ii, int jj, int kk) -> double& {
                            return L.Phi[(ii - 1) + (size_t)nx * (jj - 1) + n2 * (kk - 1)];
                        };
                        double c = at(i, j, k);
                        double e = at(i + 1, j, k), w = at(i - 1, j, k), nn = at(i, j + 1, k), ss = at(i, j - 1, k);
                        double u = at(i, j, k + 1), d = at(i, j, k - 1);
                        double a = R.a[k - 1], bta = R.b[k - 1], gm = R.c[k - 1];
                        double diag = plain ? (-2 * idx2 - 2 * idy2 + bta - eps * 0.1) : (-2 * idx2 - 2 * idy2 + bta);
                        double off = (e + w) * idx2 + (nn + ss) * idy2 + a * d + gm * u;
                        if (std::fabs(diag) > 1e-14) {
                            double nv = -off / diag;
                            at(i, j, k) = c + omega * R.w[k - 1] * (nv - c);
                        }
                    }
        }
        mg_bc(L);
    }
}

// largest spacing ratio max(dz[k+1], dz[k]) / min(...) over k = 1..Nz-1
// (ssg_sor_smoother_adaptive!, src/poisson.jl:597-615)
double mg_max_stretch(const Grid& g) {
    double m = 1.0;
    if (g.nz > 2) {
        m = -INFINITY;
        for (int k = 0; k + 1 < g.nz; ++k)
            m = std::max(m, std::max(g.dz[k + 1], g.dz[k]) / std::min(g.dz[k + 1], g.dz[k]));
    }
    return m;
}

// smoother: 0 spectral, 1 SOR, 2 enhanced (use_metrics = true, its default),
// 3 adaptive (src/poisson.jl:597-630: SOR below a spacing ratio of 2, the
// enhanced smoother without metrics at 0.9 omega below 5, with metrics at
// 0.8 omega above)
void mg_smooth(MgLevel& L, int smoother, int iters, double omega, double eps) {
    if (smoother == 0) {
        mg_spectral(L, iters, omega, eps);
    } else if (smoother == 1) {
        mg_sor(L, iters, omega, eps, true, false);
    } else if (smoother == 2) {
        mg_sor(L, iters, omega, eps, false, true);
    } else {
        double ms = mg_max_stretch(L.g);
        if (ms < 2.0) mg_sor(L, iters, omega, eps, true, false);
        else if (ms < 5.0) mg_sor(L, iters, omega * 0.9, eps, false, false);
        else mg_sor(L, iters, omega * 0.8, eps, false, true);
    }
}

// restrict_ssg_3d! / prolongate_ssg_3d! (src/poisson.jl:706-793): injection
void mg_restrict(MgLevel& C, const MgLevel& F) {
    int cx = C.g.nx, cy = C.g.ny, fx = F.g.nx, fy = F.g.ny;
    for (int k = 0; k < C.g.nz; ++k)
        for (int j = 0; j < cy; ++j)
            for (int i = 0; i < cx; ++i)
                if (2 * i < fx && 2 * j < fy && k < F.g.nz)
                    C.Phi[i + (size_t)cx * j + C.g.n2() * k] = F.Phi[2 * i + (size_t)fx * 2 * j + F.g.n2() * k];
    for (int j = 0; j < cy; ++j)
        for (int i = 0; i < cx; ++i)
            if (2 * i < fx && 2 * j < fy) C.bs[i + (size_t)cx * j] = F.bs[2 * i + (size_t)fx * 2 * j];
}

void mg_prolongate(MgLevel& F, const MgLevel& C) {
    int cx = C.g.nx, cy = C.g.ny, fx = F.g.nx, fy = F.g.ny;
    for (int k = 0; k < C.g.nz; ++k)
        for (int j = 0; j < cy; ++j)
            for (int i = 0; i < cx; ++i)
                if (2 * i < fx && 2 * j < fy)
                    F.Phi[2 * i + (size_t)fx * 2 * j + F.g.n2() * k] += C.Phi[i + (size_t)cx * j + C.g.n2() * k];
}

// ssg_v_cycle! (src/poisson.jl:802-860)
void mg_v_cycle(Mg& mg, size_t level, int smoother, double omega, double eps) {
    if (level + 1 == mg.lv.size()) {
        // coarsest level: :enhanced falls to the plain SOR smoother (src/poisson.jl:802-811)
        mg_smooth(mg.lv[level], smoother == 2 ? 1 : smoother, 50, omega, eps);
        return;
    }
    MgLevel& cur = mg.lv[level];
    MgLevel& crs = mg.lv[level + 1];
    mg_smooth(cur, smoother, 3, omega, eps);
    mg_residual(cur, eps);
    mg_restrict(crs, cur);
    crs.Phi_old = crs.Phi;
    std::fill(crs.Phi.begin(), crs.Phi.end(), 0.0);
    mg_v_cycle(mg, level + 1, smoother, omega, eps);
    for (size_t m = 0; m < crs.Phi.size(); ++m) crs.Phi[m] -= crs.Phi_old[m];
    mg_prolongate(cur, crs);
    mg_smooth(cur, smoother, 3, omega, eps);
}

double mg_norm(const std::vector<double>& x) {
    long double s = 0.0L;
    for (double v : x) s += (long double)v * v;
    return std::sqrt((double)s);
}

}  // namespace

extern "C" {

void* or_mg_create(int nx, int ny, int nz, double lx, double ly, double lz, int n_levels) {
    if (nx < 4 || ny < 4 || nz < 4 || n_levels < 1) return nullptr;
    Mg* mg = new Mg();
    int cx = nx, cy = ny;
    for (int l = 0; l < n_levels; ++l) {
        MgLevel L;
        L.init(cx, cy, nz, lx, ly, lz);
        mg->lv.push_back(std::move(L));
        cx = coarsen(cx);
        cy = coarsen(cy);
    }
    return mg;
}
void or_mg_destroy(void* h) { delete static_cast<Mg*>(h); }
// the spacing vector of a custom vertical grid on every level (coarse levels
// keep nz and z, src/coarse_domain.jl:55-65)
void or_mg_set_dz(void* h, const double* dz) {
    Mg* mg = static_cast<Mg*>(h);
    for (auto& L : mg->lv) L.g.dz.assign(dz, dz + L.g.nz);
}
int or_mg_level_nx(void* h, int level) { return static_cast<Mg*>(h)->lv[level].g.nx; }

// field: 0 Phi, 1 rhs b, 2 residual r, 3 bs_surface
static std::vector<double>& mg_field(Mg* mg, int level, int field) {
    MgLevel& L = mg->lv[level];
    return field == 0 ? L.Phi : field == 1 ? L.b : field == 2 ? L.r : L.bs;
}
void or_mg_set(void* h, int level, int field, const double* in) {
    auto& v = mg_field(static_cast<Mg*>(h), level, field);
    std::memcpy(v.data(), in, v.size() * sizeof(double));
}
void or_mg_get(void* h, int level, int field, double* out) {
    auto& v = mg_field(static_cast<Mg*>(h), level, field);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void or_mg_residual(void* h, int level, double eps) { mg_residual(static_cast<Mg*>(h)->lv[level], eps); }
void or_mg_boundary(void* h, int level) { mg_bc(static_cast<Mg*>(h)->lv[level]); }
void or_mg_smooth(void* h, int level, int smoother, int iters, double omega, double eps) {
    mg_smooth(static_cast<Mg*>(h)->lv[level], smoother, iters, omega, eps);
}
void or_mg_restrict(void* h, int coarse_level) {
    Mg* mg = static_cast<Mg*>(h);
    mg_restrict(mg->lv[coarse_level], mg->lv[coarse_level - 1]);
}
void or_mg_prolongate(void* h, int coarse_level) {
    Mg* mg = static_cast<Mg*>(h);
    mg_prolongate(mg->lv[coarse_level - 1], mg->lv[coarse_level]);
}
void or_mg_v_cycle(void* h, int smoother, double omega, double eps) {
    mg_v_cycle(*static_cast<Mg*>(h), 0, smoother, omega, eps);
}
double or_mg_norm(void* h, int level, int field) { return mg_norm(mg_field(static_cast<Mg*>(h), level, field)); }

// solve_ssg_equation (src/poisson.jl:869-959) iteration loop
int or_mg_solve(void* h, double eps, double tol, int maxiter, int smoother, double omega, int* iters, double* res) {
    Mg* mg = static_cast<Mg*>(h);
    double rn = 0.0;
    for (int it = 1; it <= maxiter; ++it) {
        mg_v_cycle(*mg, 0, smoother, omega, eps);
        mg_residual(mg->lv[0], eps);
        rn = mg_norm(mg->lv[0].r);
        *iters = it;
        *res = rn;
        if (rn < tol) return 1;
    }
    return 0;
}

}  // extern "C"
