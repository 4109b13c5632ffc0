// kernels.cuh -- launch interface of the spectral kernels (host side).
//
// Device data layout (all FP64):
//   compact spectrum  [plane][ky < My][c < Mx] complex, where the 2/3 mask of
//                     src/domain.jl:498-514 keeps kx index i < Kp or
//                     i >= N - Kp (Kp = N/3, Mx = 2*Kp) and ky index j < My
//                     (My = (2*(N/2+1))/3).  Compact column c maps to
//                     i = c (c < Kp) or i = c + N - 2*Kp.  Only these modes are
//                     ever non-zero, so only they are stored.
//   mixed (x, ky)     [plane][ky < My][x < N] complex: after the x-transform,
//                     before the y-transform.
//   physical          [plane][y][x] real (Julia column-major, x fastest).
#pragma once
#include <cuda.h>  // CUtensorMap (type only; the encoder is fetched through the runtime)
#include <cuda_runtime.h>
#include <cstdint>

namespace ssg {

struct Dims {
    int N;       // nx == ny
    int nyc;     // N/2 + 1
    int Kp;      // N/3
    int Mx;      // 2*Kp
    int My;      // (2*nyc)/3
    int nz;
    // Block shapes of the row (x) and column-pair (y) transform passes of the
    // step, in threads per block (0: the built-in default).  Tunable for
    // 64 <= N <= 512 (ssg_autotune); see kTileThreadsX / kTileThreadsY.
    int xbt = 0;
    int ybt = 0;
    // ensemble members of this grid held one after another in every buffer
    // (each member's planes, spectra and workspace contiguous); every pass
    // covers all members in one launch
    int members = 1;
    size_t c2() const { return (size_t)Mx * My; }          // compact plane
    size_t m2() const { return (size_t)N * My; }           // mixed plane
    size_t r2() const { return (size_t)N * N; }            // physical plane
};

// Candidate block shapes, in threads per block, of the tunable passes.
constexpr int kTileThreadsX[3] = {64, 128, 256};    // row passes (rows of N/8 threads)
constexpr int kTileThreadsY[3] = {128, 256, 512};   // column-pair passes (pairs of N/8 threads)

// Vertical operator: d2dz2! rows for interior planes and the Neumann rows.
struct ZOps {
    double al[64], be[64], ga[64];
    double ab, bb, cb;   // bottom: ab*P0 + bb*P1 + cb*P2 = 0
    double at, bt, ct;   // top:    at*Pn + bt*Pn-1 + ct*Pn-2 = bc
};

// Time-stage epilogues of the fused tendency kernel.
enum StageMode : int {
    STAGE_AB2_FIRST = 0,  // b += dt f;                     f_old = f
    STAGE_AB2 = 1,        // b += dt (1.5 f - 0.5 f_old);   f_old = f
    STAGE_RK3_1 = 2,      // b_stage = b; k1 = f; b = b_stage + dt/3 f
    STAGE_RK3_2 = 3,      // b = b_stage + 2dt/3 f
    STAGE_RK3_3 = 4,      // b = b_stage + dt/4 (k1 + 3 f)
    STAGE_TENDENCY = 5    // f only (written to f_out)
};

struct Tables {
    const double2* tw;     // W_N^e, e < N
    const float2* tw32;    // the same table rounded to FP32 (mixed-precision passes)
    const double* kxc;     // kx per compact column, Mx
    const double* kyc;     // ky per compact row, My
    const double* sigma;   // exponential filter transfer per compact mode
};

// Pivot table of the per-mode vertical solve: the pivots depend on the mode
// only through K^2 = kx^2 + ky^2, and compact column c (kx) and its mirror
// (-kx) give the same K^2, so the table holds one column per |kx|: Kp + 1
// columns per ky row (column Kp is kx = -Kp), levels outermost.
__host__ __device__ __forceinline__ size_t pivot_plane(int Mx, int My) { return (size_t)(Mx / 2 + 1) * My; }
// (m: a compact mode of one member, < 2^31; 32-bit index arithmetic)
__host__ __device__ __forceinline__ size_t pivot_of(size_t m, int Mx) {
    const int mi = (int)m, j = mi / Mx, c = mi - j * Mx, Kp = Mx / 2;
    return (size_t)((Kp + 1) * j + (c <= Kp ? c : Mx - c));
}

// --- Monge-Ampere fixed-point iteration -------------------------------------
// pass 1: compact Phi (interior planes) -> three mixed fields
//         A = IFFT_x(-kx^2 Phi/N^2), B = IFFT_x(Phi/N^2), C = IFFT_x(i kx Phi/N^2)
int launch_ma_xinv3(const Dims& d, const Tables& tb, const double2* Phat, double2* A, double2* B, double2* C, cudaStream_t s);
// pass 2: y-transforms: Phi_xx = c2r(A), Phi_yy = c2r(-ky^2 B), Phi_xy = c2r(i ky C),
//         D = Phi_xx Phi_yy - Phi_xy^2, Dt = r2c_y(D) (ky < My)
int launch_ma_y(const Dims& d, const Tables& tb, const double2* A, const double2* B, const double2* C, double2* Dt, cudaStream_t s);
// pass 2, persistent TMA-pipelined form (nx >= 512): the input tiles and the
// output tile move between HBM and shared memory by cp.async.bulk.tensor
// (64-byte rows of 4 complex values, 64B swizzle) through a two-slot ring.
// maps = {A, B, C, Dt}, built by make_mixed_tmaps; sm_count sizes one wave of
// resident blocks; errflag gets bit 0 if a tile wait times out.
struct MixedTmaps {
    CUtensorMap a, b, c, d;
    int box_rows;
    int warps;   // warp-transform y-pass: warps per block (column pairs per tile)
};
int make_mixed_tmaps(const Dims& d, const double2* A, const double2* B, const double2* C, const double2* Dt,
                     int nplanes, MixedTmaps* out);
bool mixed_tma_supported(const Dims& d);
// grid: one wave of resident blocks on sm_count SMs
int launch_ma_y_tma(const Dims& d, const Tables& tb, const MixedTmaps& maps, int sm_count, unsigned int* errflag,
                    cudaStream_t s);
// mixed-precision forms of passes 1-3: the mixed arrays hold float2, the
// compact Phat read by pass 1 and the Dh written by pass 3 stay FP64
int launch_ma_xinv3_mp(const Dims& d, const Tables& tb, const double2* Phat, float2* A, float2* B, float2* C,
                       cudaStream_t s);
int launch_ma_y_mp(const Dims& d, const Tables& tb, const float2* A, const float2* B, const float2* C, float2* Dt,
                   cudaStream_t s);
// dh32 (surface right-hand side only): store the FP32 transform of the kept
// modes there instead of eps times it in Dh, for launch_ma_thomas's Dh32
int launch_ma_xfwd_mp(const Dims& d, const Tables& tb, const float2* Dt, double2* Dh, double eps,
                      const double2* rhs_vol, float2* dh32, cudaStream_t s);
// mixed-precision pass 2, persistent and TMA-pipelined (FP32 tiles of 8
// columns, 64B swizzle); grid_blocks = the SM count (the grid is that times
// the blocks an SM holds)
int make_mixed32_tmaps(const Dims& d, const float2* A, const float2* B, const float2* C, const float2* Dt,
                       int nplanes, MixedTmaps* out);
int launch_ma_y_mp_tma(const Dims& d, const Tables& tb, const MixedTmaps& maps, int grid_blocks, unsigned int* errflag,
                       cudaStream_t s);
// N = 1024: the same pass with one warp per transform (fft_warp1024), blocks
// of `warps` warps (2, 4 or 8) and tiles of 2*warps FP32 columns; tw_warp is
// the [k1][n1] table of W1024^(n1 k1)
int make_mixed32w_tmaps(const Dims& d, const float2* A, const float2* B, const float2* C, const float2* Dt,
                        int nplanes, int warps, MixedTmaps* out);
int launch_ma_y_mp_warp(const Dims& d, const Tables& tb, const float2* tw_warp, const MixedTmaps& maps, int sm_count,
                        unsigned int* errflag, cudaStream_t s);
// N = 1024: mixed-precision passes 1 and 3 with one warp per row transform
// (fft_warp1024; tw_warp as for launch_ma_y_mp_warp)
int launch_ma_xinv3_mp_warp(const Dims& d, const Tables& tb, const float2* tw_warp, const double2* Phat, float2* A,
                            float2* B, float2* C, cudaStream_t s);
int launch_ma_xfwd_mp_warp(const Dims& d, const Tables& tb, const float2* tw_warp, const float2* Dt, double2* Dh,
                           double eps, const double2* rhs_vol, cudaStream_t s);
// pass 3: Dh = eps * FFT_x(Dt) on kept kx (+ b_s_hat when the RHS is volume)
int launch_ma_xfwd(const Dims& d, const Tables& tb, const double2* Dt, double2* Dh, double eps,
                   const double2* rhs_vol, cudaStream_t s);
// pass 4: per-mode Thomas solve of L Phi = [Dh ; Neumann rows], in place on
//         Phat; accumulates sum w|dPhi|^2 and sum w|Phi|^2 (Parseval weights)
//         into norms[0..1] (deterministic two-level reduction).  inv holds the
//         pivot reciprocals [nz-2][Mx*My] written by launch_ma_thomas_factor
//         for the current vertical rows.  For nz in {8, 12, 16, 24, 32} each
//         column is held in registers; other depths, or staged = true, use the
//         shared-memory staged kernel (bit-identical results).
int launch_ma_thomas_factor(const Dims& d, const Tables& tb, const ZOps* zops_dev, double* inv, cudaStream_t s);
// With d.members > 1 each member (planes, buoyancy, its norms at norms[2 m],
// its partials at partials[2 m nblocks] and ticket[m]) is solved by its own row
// of blocks; active (null: all) marks the members whose solve goes on.  With
// Dh32 (the register form only: thomas_reg_depth(nz) and not staged) the
// right-hand side is eps times the FP32 x-forward transform stored there by
// launch_ma_xfwd_mp, formed in FP64 as it is loaded (the same values as Dh).
bool thomas_reg_depth(int nz);
int launch_ma_thomas(const Dims& d, const ZOps* zops_dev, const double* inv, const double2* Dh, const float2* Dh32,
                     double eps, const double2* bc_top, double2* Phat, double* partials, unsigned int* ticket,
                     double* norms, bool staged, const unsigned int* active, cudaStream_t s);

// --- surface tendency ----------------------------------------------------------
// pass 1: P1 = IFFT_x(phi/N^2), P2 = IFFT_x(i kx phi/N^2), P3 = IFFT_x(b/N^2)
int launch_surf_xinv3(const Dims& d, const Tables& tb, const double2* phih, const double2* bh,
                      double2* P1, double2* P2, double2* P3, cudaStream_t s);
// pass 2: u = c2r(-i ky P1), v = c2r(P2), b = c2r(P3); Q1 = r2c_y(u b), Q2 = r2c_y(v b)
int launch_surf_y(const Dims& d, const Tables& tb, const double2* P1, const double2* P2, const double2* P3,
                  double2* Q1, double2* Q2, cudaStream_t s);
// pass 3: f = -mask(i kx FFT_x(Q1) + i ky FFT_x(Q2)) and the stage update
struct StageArgs {
    int mode;
    int filter;          // multiply b by sigma after the update (with step_dev: this stage
                         // filters when the step counter says so)
    double dt;
    double2* bh;         // current buoyancy (updated)
    double2* bstage;     // RK3 stage start
    double2* fold;       // AB2 history / RK3 k1
    double2* fout;       // STAGE_TENDENCY output
    unsigned int* nonfinite;
    // Device step counter (the clock's step before this step's update), or
    // null.  When set, STAGE_AB2 takes the forward-Euler first step at step 0
    // and a filtering stage filters when (step + 1) % filter_freq == 0, so the
    // same launch serves every step (CUDA graphs).
    const int64_t* step_dev;
    int filter_freq;
    // AB2 stages: the tendency of SSG.jl's AB2 as written, -P[2 i ky FFT(v b)]
    // (its output array doubles as jacobian_2d!'s scratch, src/timestep.jl:159)
    int ab2_alias;
};
int launch_surf_xfwd_stage(const Dims& d, const Tables& tb, const double2* Q1, const double2* Q2,
                           const StageArgs& a, cudaStream_t s);

// --- generic transforms (set/get of fields) -----------------------------------
// physical real planes -> mixed (ky < My), nplanes planes
int launch_y_r2c(const Dims& d, const Tables& tb, const double* in, double2* out, int nplanes, cudaStream_t s);
// mixed -> compact, scaled, optionally zeroing the mean mode
int launch_x_fwd_compact(const Dims& d, const Tables& tb, const double2* in, double2* out, int nplanes,
                         double scale, int zero_mean, cudaStream_t s);
// compact -> mixed with multiplier (0: 1, 1: -i ky, 2: i kx), scaled by 1/N^2
int launch_x_inv_compact(const Dims& d, const Tables& tb, const double2* in, double2* out, int nplanes,
                         int mult, cudaStream_t s);
// mixed (ky < My) -> physical real planes
int launch_y_c2r(const Dims& d, const Tables& tb, const double2* in, double* out, int nplanes, cudaStream_t s);

// advance the device step counter by one
int launch_step_bump(int64_t* step_dev, cudaStream_t s);

// Device-side state of the Monge-Ampere iteration loop when it runs inside a
// CUDA graph (a conditional while node around the iteration's kernels).
struct SolveDev {
    double prev, upd, updmax;
    int it, solves, iters, itmax, unconv, last_it;
    unsigned int flags;  // bit 0: a non-finite update
    int last_conv;       // the last finished solve converged
};
// start of a solve of every member (sd[members]): iteration counts and
// stagnation history reset; active (null with one member) set for all
int launch_solve_begin(SolveDev* sd, unsigned int* active, int members, cudaStream_t s);
// after an iteration: the stop rule of the host loop on each going member's
// norms[2 m .. 2 m + 1], which clears active[m] when member m's solve stops.
// In a graph (going == null) sets the while condition `handle` to whether any
// member goes on and accumulates the solve statistics in sd; otherwise writes
// that answer to *going and records only each member's last solve
// (last_it, upd, last_conv, flags), the host accumulating the statistics.
int launch_solve_check(SolveDev* sd, const double* norms, unsigned int* active, int members, double tol, int maxiter,
                       int mixed, double mixed_floor, unsigned long long handle, unsigned int* going,
                       cudaStream_t s);

// predictor: out = polynomial extrapolation of order 0-3 through the equally
// spaced solutions a (newest), b, c, e (out may alias an operand)
int launch_predict(const double2* a, const double2* b, const double2* c, const double2* e, double2* out, int order,
                   size_t n, cudaStream_t s);
// the same extrapolation per mode over all nz planes of the compact spectrum
// (a..e and out hold nz planes), then, when bh is not null (surface
// right-hand side), the exact linear correction of the guess for the mismatch
// between its top Neumann row and the current buoyancy bh (inv: the pivot
// table of launch_ma_thomas_factor)
int launch_predict_bc(const Dims& d, const double2* a, const double2* b, const double2* c, const double2* e,
                      double2* out, int order, const double2* bh, const double* inv, const ZOps* zops_dev,
                      cudaStream_t s);
// linear extrapolation: guess = 2 Phat - Pprev written into Pprev
int launch_extrapolate(const double2* Phat, double2* Pprev, size_t n, cudaStream_t s);

// surface diagnostics: norms[0] = sum w K^2 |phi_s_hat|^2, norms[1] = sum w |b_hat|^2
int launch_diagnostics(const Dims& d, const Tables& tb, const double2* phih, const double2* bh, double* partials,
                       unsigned int* ticket, double* norms, cudaStream_t s);

// multiply compact modes by sigma (exponential filter) in place
int launch_filter(const Dims& d, const Tables& tb, double2* bh, cudaStream_t s);

// --- discrete adjoint (transposes of the passes above) --------------------------
// Phi_xx, Phi_yy, Phi_xy of the interior planes from ma_xinv3's A, B, C, as
// physical fields in column-pair layout H[plane][x/2][y] (two reals per y)
int launch_ma_hess_y(const Dims& d, const Tables& tb, const double2* A, const double2* B, const double2* C,
                     double2* Hxx, double2* Hyy, double2* Hxy, cudaStream_t s);
// y-pass of F'(Phi)^T: zeta = eps c2r(E); Z1 = r2c_y(Phi_yy zeta), Z2 = r2c_y(Phi_xx zeta), Z3 = r2c_y(Phi_xy zeta)
int launch_adj_ma_y(const Dims& d, const Tables& tb, const double2* E, const double2* Hxx, const double2* Hyy,
                    const double2* Hxy, double2* Z1, double2* Z2, double2* Z3, double eps, cudaStream_t s);
// x-pass of F'(Phi)^T: Qh = -kx^2 X(Z1) - ky^2 X(Z2) + 2 kx ky X(Z3) (interior planes, compact)
int launch_adj_ma_xfwd(const Dims& d, const Tables& tb, const double2* Z1, const double2* Z2, const double2* Z3,
                       double2* Qh, cudaStream_t s);
// transposed per-mode vertical solve: Y = A^-T E^T (0, Qh, gtop); gb = the cotangent on the right-hand side.
// For nz in {8, 12, 16, 24, 32} (unless staged) from the forward pivot table inv, column in registers;
// otherwise the shared-memory kernel that factors A^T itself (results agree to rounding).
int launch_adj_thomas(const Dims& d, const Tables& tb, const ZOps* zops_dev, const double* inv, const double2* Qh,
                      const double2* gtop, double2* Y, double2* gb, int volume, double* partials,
                      unsigned int* ticket, double* norms, bool staged, cudaStream_t s);
// transposed surface tendency: P[0..4] = x-inverses of phi, i kx phi, b, i kx mu, mu (mu = D lam)
int launch_adj_surf_xinv5(const Dims& d, const Tables& tb, const double2* phih, const double2* bh, const double2* lam,
                          double2* const* P, cudaStream_t s);
// Q[0] = r2c_y(u mu_x + v mu_y), Q[1] = r2c_y(b mu_x), Q[2] = r2c_y(b mu_y)
int launch_adj_surf_y(const Dims& d, const Tables& tb, double2* const* P, double2* const* Q, cudaStream_t s);
// out = base + X(Q[0]); gphi = i ky X(Q[1]) - i kx X(Q[2])
int launch_adj_surf_xfwd(const Dims& d, const Tables& tb, double2* const* Q, const double2* base, double2* out,
                         double2* gphi, cudaStream_t s);
// out = a (sigma) x + b y per compact mode (y may be null)
int launch_adj_axpby(const Dims& d, const Tables& tb, double2* out, const double2* x, double a, const double2* y,
                     double b, int use_sigma, cudaStream_t s);
// predicted guess of a transposed solve (Y: the stage's history ring, newest
// first, interior planes; G: the ring of the top cotangents they were solved
// for), extrapolated with `order` and corrected for the current top cotangent
// gnew, which is also stored into gout
int launch_adj_predict_bc(const Dims& d, double2* const* Y, double2* out, int order, double2* const* G, double2* gout,
                          const double2* gnew, const double* inv, const ZOps* zops_dev, cudaStream_t s);
// quadratic predictor: Y3 = 3 Y1 - 3 Y2 + Y3 (Y1 newest of three equally spaced solutions)
int launch_extrapolate3(const double2* Y1, const double2* Y2, double2* Y3, size_t n, cudaStream_t s);
// transpose of set_b!'s projection: mean dropped, (-N/3, 0) halved
int launch_adj_setb(const Dims& d, const double2* lam, double2* out, cudaStream_t s);

// number of kernel launches issued by this library (for the launch-count
// claim of the benchmark)
int64_t launch_counter();

// Message returned by ssg_last_error(NULL) (errors not tied to a context).
void set_global_error(const char* msg);

// Kernel classes for per-class device timing (ssg_kernel_times).
enum KernelClass : int {
    KC_MA_XINV = 0, KC_MA_Y = 1, KC_MA_XFWD = 2, KC_MA_THOMAS = 3,
    KC_SURF_XINV = 4, KC_SURF_Y = 5, KC_SURF_XFWD = 6, KC_IO = 7,
    KC_ADJ_XINV = 8, KC_ADJ_Y = 9, KC_ADJ_XFWD = 10, KC_ADJ_THOMAS = 11, KC_ADJ_SURF = 12, KC_COUNT = 13
};

}  // namespace ssg
