# SSGB200.jl -- Julia binding of libssg_b200.so (C ABI: include/ssg_b200.h),
# the B200 implementation of SSG.jl's time step.  It sits beside SSG.jl: an
# SSG.jl script keeps make_domain and swaps the problem constructor and the
# drivers for the ones below, which keep SSG.jl's names and arguments.
#
# Not run in this repository (no Julia runtime on its machines).  The struct
# layouts are checked against the C header by tests/test_julia_binding.py,
# which parses this file.
module SSGB200

using Libdl
using ChainRulesCore

export SemiGeostrophicProblem, set_b!, solve_monge_ampere_fields!, timestep!, stepforward!, step_until!,
       apply_spectral_filter!, set_filter_table!, set_vertical_grid!, read_field, write_field!, diagnostics,
       save_simulation_state_full, load_simulation_state_full!, record!, adjoint, run_ssg,
       members_gather!, members_scatter!

# the library: ENV["SSG_B200_LIB"], else the in-tree build next to this package
const lib = get(ENV, "SSG_B200_LIB",
                normpath(joinpath(@__DIR__, "..", "..", "..", "ssg.jl_b200", "ssg_b200", "libssg_b200.so")))

const ABI_VERSION = 1

# struct ssg_config (field order and types as in include/ssg_b200.h)
mutable struct SsgConfig
    abi_version::Int32
    nx::Int32
    ny::Int32
    nz::Int32
    lx::Float64
    ly::Float64
    lz::Float64
    eps::Float64
    dt::Float64
    scheme::Int32
    filter_freq::Int32
    filter_order::Int32
    ma_maxiter::Int32
    filter_strength::Float64
    filter_cutoff::Float64
    ma_tol::Float64
    ma_per_stage::Int32
    ma_rhs_mode::Int32
    precision::Int32
    ma_predictor::Int32
    filter_type::Int32
    ab2_literal_alias::Int32
    ma_bc_guess::Int32
    nmembers::Int32
end

function SsgConfig()
    c = SsgConfig(0, 0, 0, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 0, 0, 0, 0, 0.0, 0.0, 0.0, 0, 0, 0, 0, 0, 0, 0, (0,))
    ccall((:ssg_config_init, lib), Cvoid, (Ref{SsgConfig},), c)
    return c
end

# struct ssg_ma_stats
struct MaStats
    iterations::Int32
    converged::Int32
    update::Float64
end

# struct ssg_step_stats
struct StepStats
    steps::Int32
    ma_solves::Int32
    ma_iterations::Int32
    ma_iterations_max::Int32
    ma_unconverged::Int32
    pad0::Int32
    ma_update_max::Float64
    t::Float64
    step::Int64
end

# struct ssg_diagnostics
struct Diagnostics
    t::Float64
    step::Int64
    kinetic_energy::Float64
    buoyancy_variance::Float64
    total_buoyancy::Float64
    ma_last_iterations::Int32
    pad0::Int32
end

# struct ssg_adjoint_stats
struct AdjointStats
    steps::Int32
    checkpoints::Int32
    forward_solves::Int32
    forward_iterations::Int32
    adjoint_solves::Int32
    adjoint_iterations::Int32
    adjoint_iterations_max::Int32
    adjoint_unconverged::Int32
    adjoint_update_max::Float64
    ms::Float64
    device_bytes::Int64
end

# status codes and ids (enums of include/ssg_b200.h)
const SSG_OK, SSG_ERR_ARG, SSG_ERR_CUDA, SSG_ERR_NOT_CONVERGED, SSG_ERR_NONFINITE, SSG_ERR_OOM,
      SSG_ERR_UNSUPPORTED = 0, -1, -2, -3, -4, -5, -6
const B_S, PHI_S, PHI, DBDT_OLD, U_S, V_S = 0, 1, 2, 3, 4, 5
const FILTERS = Dict(:exponential => 0, :hyperviscosity => 1, :cutoff => 2, :cesaro => 3, :custom => 4)
const PREDICTORS = Dict(:previous => 0, :extrapolate => 1, :quadratic => 2, :cubic => 3)

struct SsgError <: Exception
    status::Int
    msg::String
end
Base.showerror(io::IO, e::SsgError) = print(io, "ssg_b200 (", e.status, "): ", e.msg)

last_error(ctx) = unsafe_string(ccall((:ssg_last_error, lib), Cstring, (Ptr{Cvoid},), ctx))
check(rc, ctx; allow=()) = (rc == SSG_OK || rc in allow) ? rc : throw(SsgError(rc, last_error(ctx)))

# stands in for SemiGeostrophicProblem: the context owns every device buffer
mutable struct GPUProblem
    ctx::Ptr{Cvoid}
    nx::Int
    ny::Int
    nz::Int
    dt::Float64
    scheme::Symbol
    cfg::SsgConfig
    nmembers::Int
end

"""
    SemiGeostrophicProblem(domain; scheme=:RK3, dt=0.01, initial_time=0.0, filter_freq=10,
                           filter_strength=0.1, filter_order=4, filter_cutoff=0.65, filter=:exponential,
                           eps=0.01, ma_tol=1e-10, ma_maxiter=50, ma_per_stage=true, ma_rhs=:surface,
                           ma_predictor=:auto, precision=:fp64, ab2_literal_alias=false,
                           ma_bc_guess=true, nmembers=1, device=0)

SSG.jl's `SemiGeostrophicProblem(domain; scheme, dt, initial_time, filter_freq,
filter_strength, ...)` (src/timestep.jl:363) on one GPU.  `domain` is SSG.jl's
`Domain`: `Nx, Ny, Nz, Lx, Ly, Lz`, and `z_grid`/`dz` for stretched and custom
vertical grids, are read from it.  `scheme` is `:AB2` (`AB2_LowStorage`) or
`:RK3`.  `ma_predictor=:auto` is `:cubic` in FP64 and `:quadratic` in mixed
precision.  `filter` is one of `:exponential, :hyperviscosity, :cutoff, :cesaro`
(a table for any other transfer function: `set_filter_table!`).  `nmembers > 1`
holds that many independent ensemble members of this grid in one context: fields
gain a last dimension of length `nmembers` (`set_b!` takes (Nx, Ny, nmembers)).
"""
function SemiGeostrophicProblem(domain; scheme=:RK3, dt=0.01, initial_time=0.0, filter_freq=10,
                                filter_strength=0.1, filter_order=4, filter_cutoff=0.65, filter=:exponential,
                                eps=0.01, ma_tol=1e-10, ma_maxiter=50, ma_per_stage=true, ma_rhs=:surface,
                                ma_predictor=:auto, precision=:fp64, ab2_literal_alias=false, ma_bc_guess=true,
                                nmembers=1, device=0)
    c = SsgConfig()
    c.nx, c.ny, c.nz = domain.Nx, domain.Ny, domain.Nz
    c.lx, c.ly, c.lz = domain.Lx, domain.Ly, domain.Lz
    c.eps, c.dt = eps, dt
    sch = scheme in (:AB2, :AB2_LowStorage) ? :AB2 : scheme in (:RK3, :RK3_LowStorage) ? :RK3 :
          throw(ArgumentError("Time integration scheme $scheme not implemented yet"))
    c.scheme = sch == :AB2 ? 0 : 1
    c.filter_freq, c.filter_order = filter_freq, filter_order
    c.filter_strength, c.filter_cutoff = filter_strength, filter_cutoff
    c.filter_type = FILTERS[filter]
    c.ma_tol, c.ma_maxiter = ma_tol, ma_maxiter
    c.ma_per_stage = ma_per_stage ? 1 : 0
    c.ma_rhs_mode = ma_rhs == :surface ? 0 : 1
    c.precision = precision == :mixed ? 1 : 0
    c.ma_predictor = PREDICTORS[ma_predictor == :auto ? (precision == :mixed ? :quadratic : :cubic) : ma_predictor]
    c.ab2_literal_alias = ab2_literal_alias ? 1 : 0
    c.ma_bc_guess = ma_bc_guess ? 1 : 0
    c.nmembers = nmembers
    out = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:ssg_ctx_create, lib), Cint, (Ref{SsgConfig}, Cint, Ref{Ptr{Cvoid}}), c, device, out), C_NULL)
    p = GPUProblem(out[], domain.Nx, domain.Ny, domain.Nz, dt, sch, c, max(nmembers, 1))
    finalizer(q -> q.ctx == C_NULL || ccall((:ssg_ctx_destroy, lib), Cint, (Ptr{Cvoid},), q.ctx), p)
    if hasproperty(domain, :z_grid) && Symbol(domain.z_grid) != :uniform
        set_vertical_grid!(p, Vector{Float64}(domain.dz))
    end
    initial_time == 0 || set_time!(p, initial_time, 0)
    return p
end

function set_vertical_grid!(p::GPUProblem, dz::Vector{Float64})
    check(ccall((:ssg_set_vertical_grid, lib), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int32), p.ctx, dz, length(dz)), p.ctx)
end

function get_time(p::GPUProblem)
    t = Ref{Float64}(0.0)
    s = Ref{Int64}(0)
    check(ccall((:ssg_get_time, lib), Cint, (Ptr{Cvoid}, Ref{Float64}, Ref{Int64}), p.ctx, t, s), p.ctx)
    return t[], s[]
end

set_time!(p::GPUProblem, t, step) =
    check(ccall((:ssg_set_time, lib), Cint, (Ptr{Cvoid}, Float64, Int64), p.ctx, t, step), p.ctx)

"set_b! (src/setICs.jl:21): zero mean, dealias, Monge-Ampere solve; returns the solve's MaStats."
function set_b!(p::GPUProblem, b::AbstractArray{Float64}, domain=nothing)
    want = p.nmembers > 1 ? (p.nx, p.ny, p.nmembers) : (p.nx, p.ny)
    size(b) == want || throw(DimensionMismatch("b must be of size $want"))
    bc = Array{Float64}(b)
    st = Ref{MaStats}()
    GC.@preserve bc begin
        rc = ccall((:ssg_set_b, lib), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64, Ref{MaStats}),
                   p.ctx, bc, length(bc), st)
    end
    check(rc, p.ctx; allow=(SSG_ERR_NOT_CONVERGED,))  # not converged: the state is still set
    return st[]
end

"solve_monge_ampere_fields! (src/poisson.jl:1068): returns converged."
function solve_monge_ampere_fields!(p::GPUProblem, domain=nothing; verbose=false)
    st = Ref{MaStats}()
    rc = ccall((:ssg_solve_ma, lib), Cint, (Ptr{Cvoid}, Ref{MaStats}), p.ctx, st)
    check(rc, p.ctx; allow=(SSG_ERR_NOT_CONVERGED,))
    verbose && println("[SSG] ", st[].iterations, " iterations, update ", st[].update)
    return st[].converged != 0
end

"stepforward! (src/timestep.jl:449): nsteps steps of the problem's dt."
function stepforward!(p::GPUProblem, nsteps::Integer=1)
    st = Ref{StepStats}()
    check(ccall((:ssg_step, lib), Cint, (Ptr{Cvoid}, Int32, Float64, Ref{StepStats}), p.ctx, nsteps, p.dt, st),
          p.ctx)
    return st[]
end

"timestep! (src/timestep.jl:267): one step; returns dt."
timestep!(p::GPUProblem, args...) = (stepforward!(p, 1); p.dt)

"step_until! (src/timestep.jl:404-444): steps of dt, the last one shortened to land on stop_time."
function step_until!(p::GPUProblem, stop_time::Real)
    t, _ = get_time(p)
    stop_time > t || throw(ArgumentError("stop_time ($stop_time) must be greater than current time ($t)"))
    st = Ref{StepStats}()
    while t < stop_time
        check(ccall((:ssg_step, lib), Cint, (Ptr{Cvoid}, Int32, Float64, Ref{StepStats}),
                    p.ctx, 1, min(p.dt, stop_time - t), st), p.ctx)
        t = st[].t
    end
    _, step = get_time(p)
    set_time!(p, stop_time, step)
    return p
end

"apply_spectral_filter! (src/timestep.jl:247): filter b_s once with the problem's filter."
apply_spectral_filter!(p::GPUProblem, args...) = check(ccall((:ssg_apply_filter, lib), Cint, (Ptr{Cvoid},), p.ctx), p.ctx)

"CustomFilter (src/filter.jl:100): the transfer function on the (Nx, Ny/2+1) spectral grid."
function set_filter_table!(p::GPUProblem, sigma::AbstractMatrix{Float64})
    size(sigma) == (p.nx, p.ny ÷ 2 + 1) || throw(DimensionMismatch("sigma must be $(p.nx) x $(p.ny ÷ 2 + 1)"))
    s = Matrix{Float64}(sigma)
    GC.@preserve s check(ccall((:ssg_set_filter_table, lib), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64),
                               p.ctx, s, length(s)), p.ctx)
end

"A field as a Julia array (ids B_S, PHI_S, PHI (3-D), DBDT_OLD, U_S, V_S)."
function read_field(p::GPUProblem, id::Integer)
    mem = p.nmembers > 1 ? (p.nmembers,) : ()
    out = id == PHI ? Array{Float64}(undef, p.nx, p.ny, p.nz, mem...) : Array{Float64}(undef, p.nx, p.ny, mem...)
    GC.@preserve out check(ccall((:ssg_get_field, lib), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Int64),
                                 p.ctx, id, out, length(out)), p.ctx)
    return out
end

"Write b_s (B_S) or the AB2 history (DBDT_OLD)."
function write_field!(p::GPUProblem, id::Integer, a::AbstractArray{Float64})
    m = Array{Float64}(a)
    GC.@preserve m check(ccall((:ssg_set_field, lib), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Int64),
                               p.ctx, id, m, length(m)), p.ctx)
end

"""
    members_gather!(batch, solos)

Copy the state of the one-member problems `solos` into the members of `batch`
(a problem built with `nmembers = length(solos)` and otherwise the same
parameters): device to device, with the clock of `solos[1]`.  Stepping `batch`
then advances every member exactly as its own problem would.
`members_scatter!(batch, solos)` copies the members' state back.
"""
function members_gather!(batch::GPUProblem, solos::AbstractVector{GPUProblem})
    ptrs = Ptr{Cvoid}[q.ctx for q in solos]
    check(ccall((:ssg_members_gather, lib), Cint, (Ptr{Cvoid}, Ptr{Ptr{Cvoid}}, Int32), batch.ctx, ptrs,
                length(ptrs)), batch.ctx)
    return batch
end

function members_scatter!(batch::GPUProblem, solos::AbstractVector{GPUProblem})
    ptrs = Ptr{Cvoid}[q.ctx for q in solos]
    check(ccall((:ssg_members_scatter, lib), Cint, (Ptr{Cvoid}, Ptr{Ptr{Cvoid}}, Int32), batch.ctx, ptrs,
                length(ptrs)), batch.ctx)
    return solos
end

"update_diagnostics! (src/timestep.jl:304) as device reductions."
function diagnostics(p::GPUProblem)
    d = Ref{Diagnostics}()
    check(ccall((:ssg_get_diagnostics, lib), Cint, (Ptr{Cvoid}, Ref{Diagnostics}), p.ctx, d), p.ctx)
    return d[]
end

"""
    save_simulation_state_full(filename, p)

The complete device state (clock, b_s, AB2 history, RK3 stage, potential and
predictor history) as the library's checkpoint blob; `load_simulation_state_full!`
continues the run bit for bit.  (SSG.jl writes JLD2 datasets; a maintainer
would write the blob and the fields from `read_field` into the same file.)
"""
function save_simulation_state_full(filename::AbstractString, p::GPUProblem)
    n = Ref{Int64}(0)
    check(ccall((:ssg_checkpoint_size, lib), Cint, (Ptr{Cvoid}, Ref{Int64}), p.ctx, n), p.ctx)
    blob = Vector{UInt8}(undef, n[])
    GC.@preserve blob check(ccall((:ssg_checkpoint, lib), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Int64), p.ctx, blob, n[]),
                            p.ctx)
    write(filename, blob)
    return filename
end

function load_simulation_state_full!(p::GPUProblem, filename::AbstractString)
    blob = read(filename)
    GC.@preserve blob check(ccall((:ssg_restore, lib), Cint, (Ptr{Cvoid}, Ptr{UInt8}, Int64),
                                  p.ctx, blob, length(blob)), p.ctx)
    return p
end

# ---- discrete adjoint ---------------------------------------------------------

"set_b!(p, b0) and nsteps steps with a device checkpoint every ckpt_every steps (clock restarted at 0)."
function record!(p::GPUProblem, b0::AbstractMatrix{Float64}, nsteps::Integer; ckpt_every::Integer=20)
    set_time!(p, 0.0, 0)
    b = Matrix{Float64}(b0)
    st = Ref{AdjointStats}()
    GC.@preserve b check(ccall((:ssg_adjoint_record, lib), Cint,
                               (Ptr{Cvoid}, Ptr{Float64}, Int64, Int32, Int32, Ref{AdjointStats}),
                               p.ctx, b, length(b), nsteps, ckpt_every, st), p.ctx)
    return st[]
end

"(d b_T / d b0)^T dL_dbT for the run last recorded by record!."
function adjoint(p::GPUProblem, dL_dbT::AbstractMatrix{Float64})
    lam = Matrix{Float64}(dL_dbT)
    g = similar(lam)
    st = Ref{AdjointStats}()
    GC.@preserve lam g check(ccall((:ssg_adjoint, lib), Cint,
                                   (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int64, Ref{AdjointStats}),
                                   p.ctx, lam, g, length(g), st), p.ctx)
    return g
end

"b_T after nsteps steps from set_b!(p, b0): the differentiable run."
function run_ssg(p::GPUProblem, b0::AbstractMatrix{Float64}, nsteps::Integer; ckpt_every::Integer=20)
    record!(p, b0, nsteps; ckpt_every=ckpt_every)
    return read_field(p, B_S)
end

function ChainRulesCore.rrule(::typeof(run_ssg), p::GPUProblem, b0::AbstractMatrix{Float64}, nsteps::Integer;
                              ckpt_every::Integer=20)
    bT = run_ssg(p, b0, nsteps; ckpt_every=ckpt_every)
    pullback(ΔbT) = (NoTangent(), NoTangent(), adjoint(p, Matrix{Float64}(unthunk(ΔbT))), NoTangent())
    return bT, pullback
end

end # module
