/*
 * ssg_b200.h -- C ABI of libssg_b200.so, the B200 implementation of SSG.jl's
 * time-step path (Monge-Ampere solve, spectral transforms, Jacobian tendency,
 * exponential filter, AB2/RK3 update).
 *
 * Conventions
 *   - Every function returns an ssg_status (0 = SSG_OK, negative = error);
 *     no C++ exception crosses this boundary.  ssg_last_error() gives text.
 *   - Host arrays use SSG.jl's Julia layout: column-major, x fastest.  A 2-D
 *     field b[i,j] sits at b[i + nx*j]; a 3-D field Phi[i,j,k] at
 *     Phi[i + nx*(j + ny*k)].  Plane k = nz-1 is the surface (z = Lz).
 *   - A context owns all device memory and one CUDA stream; calls on one
 *     context are not thread-safe and block until their work is done.
 *   - The caller owns host arrays; they are copied, never retained.
 *   - Environment, read at context creation, to select among equivalent
 *     kernels for performance comparisons (results agree to rounding):
 *     SSG_B200_TMA=0/1 forces the plain-load or the persistent TMA-pipelined
 *     FP64 Monge-Ampere y-pass (default: TMA for nx >= 512);
 *     SSG_B200_MP_PLAIN=1 selects the plain-load FP32 y-pass instead of the
 *     TMA-pipelined ones; SSG_B200_MP_WARP=0 selects the team-transform FP32
 *     y-pass at nx = 1024 instead of the one-warp-per-transform kernel, and
 *     SSG_B200_MP_WARP=2, 4 or 8 that kernel's warps per block (default 4);
 *     SSG_B200_MP_XWARP=1 selects FP32 row passes at nx = 1024 with one warp
 *     per row instead of team transforms;
 *     SSG_B200_THOMAS_STAGED=1 selects the shared-memory staged vertical
 *     solve at every depth instead of the register-resident one used for
 *     nz in {8, 12, 16, 24, 32} (bit-identical results);
 *     SSG_B200_GRAPHS=0 runs steps from the host loop instead of CUDA graphs.
 *
 * Each entry point names the SSG.jl function it replaces (file:line in
 * SSG.jl's source tree).
 */
#ifndef SSG_B200_H
#define SSG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SSG_ABI_VERSION 1

typedef enum ssg_status {
    SSG_OK = 0,
    SSG_ERR_ARG = -1,            /* bad argument or size */
    SSG_ERR_CUDA = -2,           /* a CUDA call failed */
    SSG_ERR_NOT_CONVERGED = -3,  /* Monge-Ampere solve hit ma_maxiter */
    SSG_ERR_NONFINITE = -4,      /* NaN/Inf in the solution */
    SSG_ERR_OOM = -5,            /* device allocation failed */
    SSG_ERR_UNSUPPORTED = -6     /* configuration outside what the kernels cover */
} ssg_status;

/* TimeScheme (src/timestep.jl:10-14) */
enum { SSG_SCHEME_AB2 = 0, SSG_SCHEME_RK3 = 1 };

/* Monge-Ampere right-hand side.  SURFACE: interior RHS 0 and dPhi/dz = b_s at
 * the top (the problem documented at src/poisson.jl:1-12).  VOLUME: b_s
 * replicated over z as a volume RHS with homogeneous Neumann rows (what
 * solve_monge_ampere_fields! passes, src/poisson.jl:1077,1096-1113). */
enum { SSG_MA_RHS_SURFACE = 0, SSG_MA_RHS_VOLUME = 1 };

/* Filter types (src/filter.jl:119-169), applied every filter_freq steps:
 *   EXPONENTIAL     exp(-strength ((k_norm - cutoff)/(1 - cutoff))^order) above cutoff
 *   HYPERVISCOSITY  exp(-strength |k|^(2 order) dt)   (strength = nu_p)
 *   CUTOFF          1 for k_norm <= cutoff, else 0
 *   CESARO          (1 - (k_norm - cutoff)/(1 - cutoff))^order between cutoff and 1
 *   CUSTOM          a table set with ssg_set_filter_table (CustomFilter)
 * with k_norm = |k| / sqrt((pi/dx)^2 + (pi/dy)^2). */
enum { SSG_FILTER_EXPONENTIAL = 0, SSG_FILTER_HYPERVISCOSITY = 1, SSG_FILTER_CUTOFF = 2, SSG_FILTER_CESARO = 3,
       SSG_FILTER_CUSTOM = 4 };

/* Field ids for ssg_get_field / ssg_set_field (Fields, src/fields.jl:28-60) */
enum {
    SSG_FIELD_B_S = 0,       /* surface buoyancy b_s (nx*ny) */
    SSG_FIELD_PHI_S = 1,     /* surface streamfunction phi_s = Phi[:,:,nz] (nx*ny), read-only */
    SSG_FIELD_PHI = 2,       /* 3-D potential Phi (nx*ny*nz), read-only */
    SSG_FIELD_DBDT_OLD = 3,  /* AB2 history db_dt_old (nx*ny) */
    SSG_FIELD_U_S = 4,       /* surface u = -d(phi_s)/dy (nx*ny), read-only */
    SSG_FIELD_V_S = 5        /* surface v =  d(phi_s)/dx (nx*ny), read-only */
};

/* Run configuration: Domain (src/domain.jl:103-108), TimeParams
 * (src/timestep.jl:19-40) and the solve_ssg_equation keywords
 * (src/poisson.jl:869-877) in one POD.  Fill with ssg_config_init(). */
typedef struct ssg_config {
    int32_t abi_version;      /* must equal SSG_ABI_VERSION */
    int32_t nx, ny, nz;       /* grid; nx == ny, power of two in [32, 1024]; nz in [4, 64] */
    double lx, ly, lz;        /* domain size (2pi, 2pi, 1) */
    double eps;               /* Monge-Ampere epsilon */
    double dt;                /* time step */
    int32_t scheme;           /* SSG_SCHEME_AB2 / SSG_SCHEME_RK3 */
    int32_t filter_freq;      /* filter every filter_freq steps (0 = never) */
    int32_t filter_order;     /* exponential filter order p */
    int32_t ma_maxiter;       /* Monge-Ampere iteration cap */
    double filter_strength;   /* alpha */
    double filter_cutoff;     /* normalised cutoff c */
    double ma_tol;            /* stop when ||dPhi||/||Phi|| <= ma_tol */
    int32_t ma_per_stage;     /* 1: re-solve Phi before every tendency; 0: phi_s frozen after set_b */
    int32_t ma_rhs_mode;      /* SSG_MA_RHS_SURFACE / SSG_MA_RHS_VOLUME */
    int32_t precision;        /* 0 = FP64 throughout; 1 = mixed: the Monge-Ampere
                                 transforms and products in FP32, the tridiagonal
                                 solve, Phi, norms and b_s in FP64.  In mixed mode
                                 a solve has converged once its relative update
                                 is within 12 FP32 ulps (12 * 2^-24, about 7.2e-7),
                                 and it also stops when the update stops
                                 contracting (the FP32 round-off floor), converged
                                 if that floor is <= 1e-5 */
    int32_t ma_predictor;     /* initial guess of a solve: 0 = previous solution,
                                 1 = linear extrapolation of the last two solutions,
                                 2 = quadratic extrapolation of the last three,
                                 3 = cubic extrapolation of the last four */
    int32_t filter_type;      /* SSG_FILTER_* (src/filter.jl:45-100) */
    int32_t ab2_literal_alias;/* 1: AB2 computes the tendency SSG.jl's timestep_ab2_ls!
                                 computes as written, -P[2 d/dy(b_s d(phi_s)/dx)]:
                                 it passes fields.tmp2 to compute_tendency! as the
                                 output, which jacobian_2d! also uses as scratch
                                 (src/timestep.jl:159, src/nonlinear.jl:48-50,
                                 src/transforms.jl:446,459-462), so the x-flux term
                                 is overwritten and the y-flux term doubled.
                                 0 (default): the conservative Jacobian, as RK3 */
    int32_t ma_bc_guess;      /* 1 (default): the predictor's guess is corrected for
                                 the current surface buoyancy -- the solution's
                                 response to the top Neumann row is linear, so the
                                 mismatch between the extrapolated potential's top
                                 row and b_s is removed by one exact per-mode
                                 vertical solve with that mismatch as the only
                                 right-hand side (surface right-hand side only).
                                 The converged solution is the same; solves start
                                 closer to it.  0: plain extrapolation */
    int32_t nmembers;         /* ensemble members held by the context (0 or 1: one;
                                 at most 1024): independent problems on the same grid
                                 and parameters whose every kernel pass covers all
                                 members in one launch, members one after another in
                                 device memory.  Field arrays of ssg_set_b,
                                 ssg_set_field and ssg_get_field hold the members one
                                 after another (nmembers times the one-member size);
                                 a Monge-Ampere solve iterates until every member's
                                 stop rule has fired, leaving a stopped member as it
                                 is, so each member's fields equal those of a
                                 one-member context bit for bit.  Surface right-hand
                                 side only; the adjoint and ssg_get_diagnostics need
                                 one member */
} ssg_config;

/* Outcome of one Monge-Ampere solve (the diagnostics tuple of
 * solve_ssg_equation, src/poisson.jl:927-958). */
typedef struct ssg_ma_stats {
    int32_t iterations;
    int32_t converged;
    double update;            /* final ||dPhi|| / ||Phi|| */
} ssg_ma_stats;

/* Outcome of ssg_step. */
typedef struct ssg_step_stats {
    int32_t steps;
    int32_t ma_solves;
    int32_t ma_iterations;    /* summed over the solves */
    int32_t ma_iterations_max;
    int32_t ma_unconverged;   /* solves that hit ma_maxiter */
    int32_t pad0;
    double ma_update_max;
    double t;                 /* clock after the call */
    int64_t step;
} ssg_step_stats;

/* update_diagnostics! (src/timestep.jl:304-329) with true integrals over the
 * surface (the reference feeds physical arrays to parsevalsum2, which scales
 * them; these are the energies it means). */
typedef struct ssg_diagnostics {
    double t;
    int64_t step;
    double kinetic_energy;     /* 1/2 integral (u_s^2 + v_s^2) dx dy */
    double buoyancy_variance;  /* integral b_s^2 dx dy */
    double total_buoyancy;     /* integral b_s dx dy */
    int32_t ma_last_iterations;
    int32_t pad0;
} ssg_diagnostics;

typedef struct ssg_ctx ssg_ctx;

/* ABI version of the loaded library. */
int ssg_abi_version(void);

/* Defaults: 2pi x 2pi x 1 domain, eps 0.01, AB2, dt 1e-3, filter every 10
 * steps (order 4, cutoff 0.65, strength 0.1: the legacy filter of
 * src/filter.jl:508-532), ma_tol 1e-10, ma_maxiter 50,
 * per-stage solves, surface right-hand side, FP64, cubic predictor (for
 * precision 1, the quadratic predictor takes fewer iterations: set 2) with
 * the boundary-corrected guess.  Grid left at 0. */
void ssg_config_init(ssg_config* cfg);

/* Domain + allocate_fields + SemiGeostrophicProblem on one device
 * (src/domain.jl:217-230, src/fields.jl:72-116, src/timestep.jl:363-399).
 * Allocates every device buffer of the context; clock t = 0, step = 0. */
int ssg_ctx_create(const ssg_config* cfg, int device, ssg_ctx** out);
int ssg_ctx_destroy(ssg_ctx* ctx);

/* set_b! (src/setICs.jl:21-88): copy b (nx*ny), remove the mean mode,
 * 2/3-dealias, then solve Monge-Ampere from a zero initial guess.  Returns
 * SSG_ERR_NOT_CONVERGED if the solve hit ma_maxiter (state still set). */
int ssg_set_b(ssg_ctx* ctx, const double* b, int64_t n, ssg_ma_stats* stats);

/* solve_monge_ampere_fields! (src/poisson.jl:1068-1090) for the current b_s,
 * warm-started from the current Phi. */
int ssg_solve_ma(ssg_ctx* ctx, ssg_ma_stats* stats);

/* nsteps calls of timestep! (src/timestep.jl:267-285); dt <= 0 uses cfg.dt.
 * With ma_per_stage, Phi is re-solved after every stage update, so phi_s always
 * matches the current b_s.  Returns SSG_ERR_NONFINITE if the buoyancy became
 * non-finite; non-converged solves are counted in stats, not errors. */
int ssg_step(ssg_ctx* ctx, int32_t nsteps, double dt, ssg_step_stats* stats);

/* apply_spectral_filter! (src/timestep.jl:247-260, src/filter.jl:181-272):
 * multiply the surface buoyancy's spectrum by the configured transfer
 * function once, now. */
int ssg_apply_filter(ssg_ctx* ctx);

/* CustomFilter (src/filter.jl:100-109, 169-177): install a transfer table
 * given on the full spectral grid, nx*(ny/2+1) values, kx index fastest
 * (the reference's (Nx, Nyc) layout); the context's filter becomes CUSTOM. */
int ssg_set_filter_table(ssg_ctx* ctx, const double* sigma, int64_t n);

/* Surface diagnostics computed on the device from the spectra (Parseval). */
int ssg_get_diagnostics(ssg_ctx* ctx, ssg_diagnostics* out);

/* save_simulation_state_full / load_simulation_state_full (src/output.jl:318,
 * 1011): the complete state -- clock, surface buoyancy, AB2 history and RK3
 * stage, the potential and the predictor history -- as one opaque blob, so a
 * restored context continues bit for bit.  The blob embeds nx, ny, nz and
 * precision; ssg_restore rejects a blob of another shape. */
int ssg_checkpoint_size(const ssg_ctx* ctx, int64_t* bytes);
int ssg_checkpoint(ssg_ctx* ctx, void* blob, int64_t bytes);
int ssg_restore(ssg_ctx* ctx, const void* blob, int64_t bytes);

/* Vertical grid of make_vertical_grid (src/domain.jl:238-280): the spacing
 * vector Domain.dz (nz values, as the reference computes it for its uniform,
 * stretched and custom grids) from which the d2dz2! rows and the Neumann rows
 * of the Monge-Ampere operator are built, with the reference's indexing of dz.
 * The default is the uniform grid dz = Lz/(nz-1).  Spacings must be finite and
 * non-zero (the reference's surface-concentrated grids run from z = Lz down to
 * 0, so their spacings are negative). */
int ssg_set_vertical_grid(ssg_ctx* ctx, const double* dz, int32_t n);

/* Copy a field to / from host memory (n = element count). */
int ssg_get_field(ssg_ctx* ctx, int32_t field, double* host, int64_t n);
int ssg_set_field(ssg_ctx* ctx, int32_t field, const double* host, int64_t n);

/* TimeState clock (src/timestep.jl:45-86). */
int ssg_get_time(const ssg_ctx* ctx, double* t, int64_t* step);
int ssg_set_time(ssg_ctx* ctx, double t, int64_t step);

/* Device time (ms) of the last ssg_step / ssg_solve_ma call, from CUDA events
 * on the context's stream, and the number of kernels it launched. */
int ssg_last_timing(const ssg_ctx* ctx, double* ms, int64_t* kernel_launches);

/* Per-kernel-class device timing.  While enabled, every launch on the
 * context's stream is bracketed by CUDA events; ssg_kernel_times returns, per
 * class, the summed device milliseconds and launch counts since the last
 * reset (classes: 0 MA x-inverse, 1 MA y-pass, 2 MA x-forward, 3 MA
 * tridiagonal solve, 4 tendency x-inverse, 5 tendency y-pass, 6 tendency
 * x-forward + stage update, 7 field transfer transforms; adjoint: 8 MA
 * x-inverse, 9 MA y-pass, 10 MA x-forward, 11 MA transposed tridiagonal solve,
 * 12 transposed tendency and stage combinations). */
#define SSG_KERNEL_CLASSES 13
int ssg_profile_kernels(ssg_ctx* ctx, int enable);
int ssg_kernel_times(ssg_ctx* ctx, double* ms, int64_t* launches, int32_t nclass);

/* Size of the static device array ssg_tendency_noalloc works in. */
#define SSG_NOALLOC_SCRATCH_BYTES (10u * 1024u * 1024u)

/* ssg_tendency_noalloc has no counterpart in SSG.jl.  It computes what
 * compute_tendency! computes, -P J(phi_s, b_s) with the 2/3 mask P, for
 * callers that cannot allocate device memory: code whose device memory is
 * owned by someone else (a caching allocator or framework pool that must see
 * every byte) and code in time-critical loops, where cudaMalloc may
 * synchronize the device and stall.  phi_s, b_s and dbdt are device arrays of
 * nx*ny doubles (x fastest) on the current device; the fields are taken on the
 * 2/3-dealiased modes, which is where the time step's fields live.  Grids up to
 * 512 x 512 (nx == ny, power of two >= 32); larger grids return SSG_ERR_ARG.
 * The call is asynchronous on `stream` (a cudaStream_t; NULL = legacy default
 * stream) and allocates nothing: its working storage is one static device
 * array of SSG_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
 * until the process exits.  The first call on a device looks up that array's
 * device address; make it before any stream capture on the device.  All calls
 * on a device share the array and leave their data in it, so calls that
 * overlap on the GPU race: serialise them.  Each call writes the tables it
 * needs into the array itself, so it does not depend on an earlier call's
 * grid.  NaN or Inf in the inputs are not reported: they propagate to dbdt. */
int ssg_tendency_noalloc(int32_t nx, int32_t ny, double lx, double ly, const double* phi_s, const double* b_s,
                         double* dbdt, void* stream);

/* ---- Discrete adjoint of the time step (no counterpart in SSG.jl) --------
 * Gradient of a functional of the final surface buoyancy b_T with respect to
 * the initial buoyancy b0 handed to set_b!.  The adjoint is the exact transpose
 * of the discrete step: transposed spectral transforms and Jacobian, the
 * transposed linearised Monge-Ampere solve at the converged potential
 * (implicit-function adjoint: one linear fixed-point solve per forward solve,
 * no unrolling of the iterations), reversed AB2 / RK3 stages and filter.
 * Memory: a device checkpoint every ckpt_every steps; the reverse sweep
 * recomputes each segment from its checkpoint, keeping the segment's stage
 * buoyancies and potentials on the device (a tape), then runs it backwards.
 * The recording tapes the last segment itself, so ckpt_every >= nsteps keeps
 * the whole run on the tape and recomputes nothing.  FP64 only
 * (precision 0), with the potential re-solved every stage (ma_per_stage 1). */
typedef struct ssg_adjoint_stats {
    int32_t steps;                  /* steps recorded (or reversed) */
    int32_t checkpoints;            /* device checkpoints held */
    int32_t forward_solves;         /* Monge-Ampere solves (recording or recomputation) */
    int32_t forward_iterations;
    int32_t adjoint_solves;         /* transposed linearised solves */
    int32_t adjoint_iterations;
    int32_t adjoint_iterations_max;
    int32_t adjoint_unconverged;
    double adjoint_update_max;      /* largest final relative update of an adjoint solve */
    double ms;                      /* device time of the call (CUDA events) */
    int64_t device_bytes;           /* checkpoint, tape and adjoint workspace memory */
} ssg_adjoint_stats;
/* Forward run that the adjoint differentiates: set_b!(b0) (n = nx*ny values,
 * mean removed, dealiased, potential solved), then nsteps steps of the
 * configured scheme with the configured dt, keeping a device checkpoint every
 * ckpt_every steps.  The run starts at the context's clock (ssg_set_time): the
 * filter cadence follows its step count, and an AB2 run that does not start
 * at step 0 uses the context's AB2 history db_dt_old, held constant.  The
 * context ends at the final state, as after ssg_step. */
int ssg_adjoint_record(ssg_ctx* ctx, const double* b0, int64_t n, int32_t nsteps, int32_t ckpt_every,
                       ssg_adjoint_stats* stats);
/* Reverse sweep of the last recorded run: dL_db0 = (d b_T / d b0)^T dL_dbT,
 * both nx*ny host arrays (x fastest).  The context is left at the final state
 * of the recording; the recording can be reversed again with another dL_dbT. */
int ssg_adjoint(ssg_ctx* ctx, const double* dL_dbT, double* dL_db0, int64_t n, ssg_adjoint_stats* stats);

/* ---- Block shapes of the transform passes (no counterpart in SSG.jl) -------
 * The row (x) and column-pair (y) transform passes of a step group their
 * length-N transforms into blocks; the block shape, in threads per block,
 * changes how many transforms share a block and an SM, not the operations of
 * a transform.  Each shape is its own compiled kernel, which may contract a
 * multiply-add differently, so results agree to rounding (measured within
 * 5e-16 relative in FP64, same iteration counts); a pinned shape reproduces
 * bit for bit.  Shapes are tunable for
 * 64 <= nx <= 512: x_threads in {64, 128, 256}, y_threads in {128, 256, 512},
 * 0 meaning the built-in default.  Changing a shape drops the context's cached
 * step graphs.
 * ssg_autotune times each candidate on the context's own grid and precision
 * (reps rounds of one Monge-Ampere iteration and one tendency pass, CUDA
 * events per kernel class), keeps the fastest row shape and then the fastest
 * column-pair shape, returns them, and restores the state the context had.
 * For other nx the shapes stay as they are.  It then tunes the kernel
 * variants below. */
int ssg_autotune(ssg_ctx* ctx, int32_t reps, int32_t* x_threads, int32_t* y_threads);
int ssg_set_tiles(ssg_ctx* ctx, int32_t x_threads, int32_t y_threads);
int ssg_get_tiles(const ssg_ctx* ctx, int32_t* x_threads, int32_t* y_threads);

/* ---- Kernel variants (no counterpart in SSG.jl) ----------------------------
 * The Monge-Ampere y-pass exists as a plain-load kernel, a persistent
 * TMA-pipelined team-transform kernel, and (FP32 at nx = 1024) a kernel with
 * one warp per transform in blocks of 2, 4 or 8 warps; the vertical solve holds
 * each column in registers (nz in {8, 12, 16, 24, 32}) or stages it through
 * shared memory.  ssg_autotune also times these choices (after the block
 * shapes, at every nx) and keeps the fastest; ssg_set_variants pins them
 * (SSG_ERR_UNSUPPORTED for a kernel that does not exist for the context's grid
 * and precision).  Results agree to rounding across y-pass kernels (bit for bit
 * across warps per block) and bit for bit across vertical-solve forms.
 * Changing a variant drops the context's cached step graphs. */
enum { SSG_YPASS_PLAIN = 0, SSG_YPASS_TMA = 1, SSG_YPASS_WARP2 = 2, SSG_YPASS_WARP4 = 4, SSG_YPASS_WARP8 = 8 };
int ssg_set_variants(ssg_ctx* ctx, int32_t y_pass, int32_t thomas_staged);
int ssg_get_variants(const ssg_ctx* ctx, int32_t* y_pass, int32_t* thomas_staged);

/* ---- Batched ensemble on one GPU (no counterpart in SSG.jl) ---------------
 * Contexts on one device advanced together.  ssg_ensemble_step advances every
 * member by nsteps of its own configured dt, in one of two modes:
 *   SSG_ENSEMBLE_THREADS    every member steps as in ssg_step (cached CUDA
 *                           graphs of whole steps on its own stream); worker
 *                           threads issue the members' launches in parallel.
 *   SSG_ENSEMBLE_ONE_GRAPH  once every member's predictor history is full, one
 *                           CUDA graph launch per chunk of steps advances all
 *                           members (each member's steps, Monge-Ampere loops
 *                           included, an independent branch of the graph).
 * stats (n entries, or NULL) receives each member's ssg_step statistics.
 * Members stay ordinary contexts (set, get, step, checkpoint) between calls; a
 * context in an ensemble must not be used from another thread during
 * ssg_ensemble_step.  Many members on one device overlap best with more
 * hardware work queues than the default 8 (CUDA_DEVICE_MAX_CONNECTIONS=32,
 * set before the process first uses CUDA). */
enum { SSG_ENSEMBLE_THREADS = 0, SSG_ENSEMBLE_ONE_GRAPH = 1 };
typedef struct ssg_ensemble ssg_ensemble;
int ssg_ensemble_create(ssg_ctx* const* members, int32_t n, int32_t mode, ssg_ensemble** out);
int ssg_ensemble_step(ssg_ensemble* e, int32_t nsteps, ssg_step_stats* stats);
int ssg_ensemble_destroy(ssg_ensemble* e);
const char* ssg_ensemble_last_error(const ssg_ensemble* e);

/* State transfer between n one-member contexts solo[0..n) and the n members
 * of `batch` (ssg_config.nmembers = n; every configuration field equal apart
 * from nmembers; one device).  ssg_members_gather copies member i's state
 * from solo[i] -- the buoyancy, the AB2 history / RK3 stage buffers, the
 * potential and its predictor history -- with solo[0]'s clock, filter table
 * and vertical grid; every solo context must be at the same time and step,
 * with the same predictor history length, filter table and vertical grid
 * (else SSG_ERR_ARG, nothing copied).  Stepping `batch` then advances each
 * member exactly as its one-member context would have.  ssg_members_scatter
 * copies the members' state and the clock back.  Device-to-device copies;
 * both synchronise. */
int ssg_members_gather(ssg_ctx* batch, ssg_ctx* const* solo, int32_t n);
int ssg_members_scatter(ssg_ctx* batch, ssg_ctx* const* solo, int32_t n);

/* ---- The reference's own multigrid (solve_ssg_equation and its parts) ----
 * An ssg_mg is SSGMultigridSolver's hierarchy of SSGLevels
 * (src/poisson.jl:33-127): physical 3-D fields Phi, b (right-hand side), r
 * and the 2-D bs_surface on n_levels grids, each the previous one coarsened
 * by create_coarse_domain (src/coarse_domain.jl:26-32: halve, at least 5,
 * even; nz kept).  The functions reproduce the reference's as written -- the
 * spectral smoother diverges and the SOR smoother ignores the right-hand side
 * (SSG.jl behaviour, not the documented problem; the time step's solver is
 * ssg_solve_ma).  Fields use the layout of the context API (x fastest). */
enum { SSG_MG_PHI = 0, SSG_MG_RHS = 1, SSG_MG_RESIDUAL = 2, SSG_MG_BS_SURFACE = 3 };
/* smoother ids: :spectral, :sor, :enhanced (with metrics), :adaptive (picks
 * :sor or :enhanced from the largest spacing ratio of dz; :sor on a uniform
 * grid) */
enum { SSG_SMOOTHER_SPECTRAL = 0, SSG_SMOOTHER_SOR = 1, SSG_SMOOTHER_ENHANCED = 2, SSG_SMOOTHER_ADAPTIVE = 3 };
typedef struct ssg_mg ssg_mg;
int ssg_mg_create(int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz, int32_t n_levels, int device,
                  ssg_mg** out);
int ssg_mg_destroy(ssg_mg* mg);
int ssg_mg_level_shape(const ssg_mg* mg, int32_t level, int32_t* nx, int32_t* ny, int32_t* nz);
int ssg_mg_set(ssg_mg* mg, int32_t level, int32_t field, const double* host, int64_t n);
/* Vertical spacing Domain.dz (nz values) of every level, replacing the uniform
 * default: coarse levels keep nz and z (src/coarse_domain.jl:55-65).  Same
 * rules as ssg_set_vertical_grid. */
int ssg_mg_set_vertical_grid(ssg_mg* mg, const double* dz, int32_t n);
int ssg_mg_get(ssg_mg* mg, int32_t level, int32_t field, double* host, int64_t n);
/* compute_ssg_residual! (src/poisson.jl:228-253), including its boundary side
 * effect on Phi */
int ssg_mg_residual(ssg_mg* mg, int32_t level, double eps);
/* apply_ssg_boundary_conditions! (src/poisson.jl:262-364) */
int ssg_mg_boundary(ssg_mg* mg, int32_t level);
/* ssg_spectral_smoother! / ssg_sor_smoother! / _enhanced! / _adaptive!
 * (src/poisson.jl:402-697) */
int ssg_mg_smooth(ssg_mg* mg, int32_t level, int32_t smoother, int32_t iters, double omega, double eps);
/* restrict_ssg_3d! / prolongate_ssg_3d! (src/poisson.jl:706-732): injection
 * between coarse_level and coarse_level - 1 */
int ssg_mg_restrict(ssg_mg* mg, int32_t coarse_level);
int ssg_mg_prolongate(ssg_mg* mg, int32_t coarse_level);
/* ssg_v_cycle! (src/poisson.jl:802-860) from level 0 */
int ssg_mg_v_cycle(ssg_mg* mg, int32_t smoother, double omega, double eps);
/* norm_field (src/poisson.jl:986-995) */
int ssg_mg_norm(ssg_mg* mg, int32_t level, int32_t field, double* out);
/* solve_ssg_equation's iteration loop (src/poisson.jl:900-959): V-cycles until
 * norm_field(r) < tol; SSG_ERR_NOT_CONVERGED after maxiter */
int ssg_mg_solve(ssg_mg* mg, double eps, double tol, int32_t maxiter, int32_t smoother, double omega,
                 int32_t* iterations, double* residual, int32_t* converged);
const char* ssg_mg_last_error(const ssg_mg* mg);

/* Text of the last error on this context (or of the last failed create when
 * ctx is NULL). */
const char* ssg_last_error(const ssg_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* SSG_B200_H */
