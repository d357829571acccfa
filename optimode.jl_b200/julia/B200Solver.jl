# B200Solver: the libomb200 backend for MaxwellEigenmodes' solve_ω² / solve_k.
#
# Drop this file into lib/MaxwellEigenmodes/src/solvers/ (include it after gpu.jl) and set
# OMB200_LIB to the path of libomb200.so.  It adds one concrete AbstractEigensolver with the
# same method set and keyword contract as GPUSolver (src/solvers/gpu.jl:37-49, 201-242);
# every device step runs in the C library (include/omb200.h) through `ccall`.

export B200Solver, solve_k_batch

const OMB200_LIB = get(ENV, "OMB200_LIB", "libomb200.so")

# ---- C structs (layouts match include/omb200.h) ------------------------------------
struct OmbGrid
    Nx::Int32
    Ny::Int32
    Dx::Float64
    Dy::Float64
end

struct OmbOptions
    k_tol::Float64
    eig_tol::Float64
    max_eigsolves::Int32
    maxiter::Int32
    precision::Int32
    preconditioner::Int32
    newton::Int32
    canonicalize::Int32
    seed::UInt64
    guard_bands::Int32
    warm_start::Int32
end

struct OmbInstance
    grid::OmbGrid
    omega::Float64
    epsinv::Ptr{Float64}
    nev::Int32
    kguess::Float64
    Hguess::Ptr{Float64}
    nguess::Int32
    kguess_bands::Ptr{Float64}
end

struct OmbResult
    kmags::Ptr{Float64}
    evecs::Ptr{Float64}
    residuals::Ptr{Float64}
    dw2dk::Ptr{Float64}
    status::Ptr{Int32}
    iterations::Ptr{Int32}
    newton_steps::Ptr{Int32}
end

const _PREC = Dict(:fp32 => Int32(0), :fp64 => Int32(1), :mixed => Int32(2))
const _PRECOND = Dict(:mpb => Int32(1), :diag => Int32(2))
const _NEWTON = Dict(:inner => Int32(0), :outer => Int32(1))
const _WARM = Dict(:none => Int32(0), :sweep => Int32(1), :cells => Int32(2), :learned => Int32(3),
                   :sweep_learned => Int32(4))

"""
    B200Solver(; precision=:mixed, preconditioner=:diag, newton=:inner, device=0,
               maxiter=1000, guard_bands=1, warm_start=:none, logger=NullLogger())

NVIDIA B200 (sm_100a) backend: batched device LOBPCG with Newton steps on k inside the
iteration, FP32 iterations polished in FP64 to the requested tolerance.  `warm_start=:sweep`
makes `solve_k_batch` start the instances that share one ε⁻¹ array from the solved instance
nearest their mean ω (a frequency sweep); `warm_start=:cells` starts instances that share ω
from the middle one (the cells of an eigenmode expansion, `eme(...; warmstart=true)`);
`warm_start=:learned` starts instances on 128², 256² or 512² grids from the learned network
attached with `b200_attach_warmstart` (fields and n_eff of bands 0..3; same tolerances);
`warm_start=:sweep_learned` is `:sweep` with the first-solved instances started from the network.
"""
struct B200Solver{L<:AbstractLogger} <: AbstractEigensolver{L}
    logger::L
    device::Int
    precision::Symbol
    preconditioner::Symbol
    newton::Symbol
    maxiter::Int
    guard_bands::Int
    warm_start::Symbol
end

B200Solver(; precision=:mixed, preconditioner=:diag, newton=:inner, device=0, maxiter=1000,
    guard_bands=1, warm_start=:none, logger=NullLogger()) =
    B200Solver(logger, device, precision, preconditioner, newton, maxiter, guard_bands, warm_start)

const _OMB_CTX = Dict{Int,Ptr{Cvoid}}()

function _omb_check(rc)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:omb_last_error, OMB200_LIB), Cstring, ()))
    error("libomb200 (B200Solver) failed with status $rc: $msg")
end

function _omb_ctx(s::B200Solver)
    get!(_OMB_CTX, s.device) do
        h = Ref{Ptr{Cvoid}}(C_NULL)
        _omb_check(ccall((:omb_ctx_create, OMB200_LIB), Cint, (Cint, Ref{Ptr{Cvoid}}), s.device, h))
        h[]
    end
end

function _omb_options(s::B200Solver; k_tol=1e-8, eig_tol=1e-8, max_eigsolves=60, maxiter=s.maxiter)
    OmbOptions(k_tol, eig_tol, max_eigsolves, maxiter, _PREC[s.precision], _PRECOND[s.preconditioner],
        _NEWTON[s.newton], Int32(1), UInt64(0), Int32(s.guard_bands), _WARM[s.warm_start])
end

_omb_grid(g::Grid{2}) = OmbGrid(g.Nx, g.Ny, g.Δx, g.Δy)

"""
    solve_k_batch(ωs, ε⁻¹s, grids, s::B200Solver; nevs, k_tol, eig_tol, ...) -> Vector{(kmags, evecs)}

Solve many independent cross-sections in one device run (new API: the reference callers
loop over `solve_k`).
"""
function solve_k_batch(ωs, ε⁻¹s, grids, s::B200Solver; nevs=fill(1, length(ωs)), max_eigsolves=60,
    maxiter=s.maxiter, k_tol=1e-8, eig_tol=1e-8, kguesses=nothing, Hguesses=nothing)
    n = length(ωs)
    # one converted array per distinct input, so a sweep over ω shares its ε⁻¹ pointer
    conv = IdDict{Any,Array{Float64,4}}()
    eps = [get!(() -> convert(Array{Float64,4}, e), conv, e) for e in ε⁻¹s]
    kmags = [zeros(Float64, nevs[i]) for i in 1:n]
    evecs = [zeros(ComplexF64, 2 * grids[i].Nx * grids[i].Ny, nevs[i]) for i in 1:n]
    status = [zeros(Int32, nevs[i]) for i in 1:n]
    guesses = [Hguesses === nothing ? nothing : reduce(hcat, Hguesses[i]) for i in 1:n]
    GC.@preserve eps kmags evecs status guesses begin
        insts = [OmbInstance(_omb_grid(grids[i]), ωs[i], pointer(eps[i]), nevs[i],
            kguesses === nothing ? 0.0 : Float64(first(kguesses[i])),
            guesses[i] === nothing ? Ptr{Float64}(C_NULL) : Ptr{Float64}(pointer(guesses[i])),
            guesses[i] === nothing ? 0 : size(guesses[i], 2), Ptr{Float64}(C_NULL)) for i in 1:n]
        res = [OmbResult(pointer(kmags[i]), Ptr{Float64}(pointer(evecs[i])), C_NULL, C_NULL,
            pointer(status[i]), C_NULL, C_NULL) for i in 1:n]
        opt = Ref(_omb_options(s; k_tol, eig_tol, max_eigsolves, maxiter))
        rc = ccall((:omb_solve_k, OMB200_LIB), Cint,
            (Ptr{Cvoid}, Ptr{OmbInstance}, Cint, Ref{OmbOptions}, Ptr{OmbResult}),
            _omb_ctx(s), insts, n, opt, res)
        _omb_check(rc)
    end
    return [(kmags[i], [evecs[i][:, j] for j in 1:nevs[i]]) for i in 1:n]
end

# solve_k(ω, ε⁻¹, grid, solver; ...) with the reference's keyword set (src/solve.jl:182-196)
function solve_k(ω::T0, ε⁻¹::AbstractArray{T0,4}, grid::Grid{2,T0}, s::B200Solver; nev=1,
    max_eigsolves=60, maxiter=s.maxiter, k_tol=1e-8, eig_tol=1e-8, log=false, kguess=nothing,
    Hguess=nothing, f_filter=nothing, overwrite=false) where {T0<:Real}
    hg = Hguess === nothing ? nothing : [Hguess isa AbstractMatrix ? collect(eachcol(Hguess)) :
                                         (eltype(Hguess) <: Number ? [Hguess] : collect(Hguess))]
    out = solve_k_batch([Float64(ω)], [ε⁻¹], [grid], s; nevs=[nev], max_eigsolves, maxiter, k_tol,
        eig_tol, kguesses=kguess === nothing ? nothing : [kguess], Hguesses=hg)
    return out[1]
end

# solve_ω²(ms, solver; nev, maxiter, tol): writes ms.H⃗ and ms.ω² like gpu.jl:201-211
function solve_ω²(ms::ModeSolver{2,T}, s::B200Solver; nev=1, maxiter=s.maxiter, tol=1e-8, log=false,
    f_filter=nothing) where {T<:Real}
    n2 = size(ms.H⃗, 1)
    evals = zeros(Float64, nev)
    evecs = zeros(ComplexF64, n2, nev)
    eps = convert(Array{Float64,4}, ms.M̂.ε⁻¹)
    guess = convert(Matrix{ComplexF64}, ms.H⃗)
    opt = Ref(_omb_options(s; eig_tol=tol, maxiter))
    GC.@preserve eps evals evecs guess begin
        rc = ccall((:omb_solve_omega2, OMB200_LIB), Cint,
            (Ptr{Cvoid}, Ref{OmbGrid}, Cdouble, Ptr{Float64}, Cint, Ptr{Float64}, Cint, Ref{OmbOptions},
             Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Int32}),
            _omb_ctx(s), Ref(_omb_grid(ms.grid)), ms.M̂.k⃗[3], eps, nev, Ptr{Float64}(pointer(guess)),
            min(nev, size(guess, 2)), opt, evals, Ptr{Float64}(pointer(evecs)), C_NULL, C_NULL)
        _omb_check(rc)
    end
    evecs_out = [evecs[:, j] for j in 1:nev]
    ms.H⃗[:, 1:nev] .= evecs
    ms.ω²[1:nev] .= complex.(evals)
    return evals, evecs_out
end

# rrule(solve_k, ...) for B200Solver: same contract as src/solve.jl:213-289 — the pullback
# returns (NoTangent(), ω̄, ε̄⁻¹, NoTangent(), NoTangent()); AbstractZero cotangents (whole
# tuple or per band) become NULL / all-zero columns.
function ChainRulesCore.rrule(::typeof(solve_k), ω::T0, ε⁻¹::AbstractArray{T0,4}, grid::Grid{2,T0},
    s::B200Solver; nev=1, max_eigsolves=60, maxiter=s.maxiter, k_tol=1e-8, eig_tol=1e-8, log=false,
    kguess=nothing, Hguess=nothing, f_filter=nothing, overwrite=false) where {T0<:Real}
    kmags, evecs = solve_k(ω, ε⁻¹, grid, s; nev, max_eigsolves, maxiter, k_tol, eig_tol, kguess, Hguess)
    eps = convert(Array{Float64,4}, ε⁻¹)
    function b200_solve_k_pullback(ΔΩ)
        ΔΩ isa AbstractZero && return (NoTangent(), 0.0, zero(eps), NoTangent(), NoTangent())
        k̄mags, ēvecs = ΔΩ
        kbar = k̄mags isa AbstractZero ? nothing : [k isa AbstractZero ? 0.0 : Float64(k) for k in k̄mags]
        n2 = length(first(evecs))
        ebar = ēvecs isa AbstractZero ? nothing :
               reduce(hcat, [e isa AbstractZero ? zeros(ComplexF64, n2) : ComplexF64.(e) for e in ēvecs])
        V = reduce(hcat, evecs)
        ω̄ = Ref(0.0)
        ε̄⁻¹ = zeros(Float64, size(eps))
        opt = Ref(_omb_options(s; k_tol, eig_tol, max_eigsolves, maxiter))
        GC.@preserve eps kmags V kbar ebar ε̄⁻¹ begin
            rc = ccall((:omb_pullback, OMB200_LIB), Cint,
                (Ptr{Cvoid}, Ref{OmbGrid}, Cdouble, Ptr{Float64}, Cint, Ptr{Float64}, Ptr{Float64},
                 Ptr{Float64}, Ptr{Float64}, Ref{OmbOptions}, Ref{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Int32}),
                _omb_ctx(s), Ref(_omb_grid(grid)), Float64(ω), eps, nev, kmags, Ptr{Float64}(pointer(V)),
                kbar === nothing ? Ptr{Float64}(C_NULL) : pointer(kbar),
                ebar === nothing ? Ptr{Float64}(C_NULL) : Ptr{Float64}(pointer(ebar)),
                opt, ω̄, ε̄⁻¹, C_NULL, C_NULL)
            _omb_check(rc)
        end
        return (NoTangent(), ω̄[], ε̄⁻¹, NoTangent(), NoTangent())
    end
    return ((kmags, evecs), b200_solve_k_pullback)
end

# ---- 3D cells periodic along ẑ (src/grads/period.jl) ----------------------------------------
# solve_k_periodic(ω, ε⁻¹, Λ, grid::Grid{3}, ::B200Solver; nev) and its rrule, whose pullback
# returns (NoTangent(), ω̄, ε̄⁻¹, Λ̄, NoTangent(), NoTangent()) like period.jl:227-240.

struct OmbGrid3
    Nx::Int32
    Ny::Int32
    Nz::Int32
    Dx::Float64
    Dy::Float64
    Dz::Float64
end

_omb_grid3(g::Grid{3}, Λ) = OmbGrid3(g.Nx, g.Ny, g.Nz, g.Δx, g.Δy, Float64(Λ))

function solve_k_periodic(ω::T, ε⁻¹::AbstractArray{T,5}, Λ::Real, grid::Grid{3,T}, s::B200Solver; nev=1,
    max_eigsolves=60, maxiter=s.maxiter, k_tol=1e-8, eig_tol=1e-8, kguess=nothing, kwargs...) where {T<:Real}
    eps = convert(Array{Float64,5}, ε⁻¹)
    kmags = zeros(Float64, nev)
    evecs = zeros(ComplexF64, 2 * grid.Nx * grid.Ny * grid.Nz, nev)
    opt = Ref(_omb_options(s; k_tol, eig_tol, max_eigsolves, maxiter))
    GC.@preserve eps kmags evecs begin
        rc = ccall((:omb_solve_k_periodic, OMB200_LIB), Cint,
            (Ptr{Cvoid}, Ref{OmbGrid3}, Cdouble, Ptr{Float64}, Cint, Cdouble, Ref{OmbOptions}, Ptr{Float64},
             Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Int32}, Ptr{Int32}),
            _omb_ctx(s), Ref(_omb_grid3(grid, Λ)), Float64(ω), eps, nev,
            kguess === nothing ? 0.0 : Float64(first(kguess)), opt, kmags, Ptr{Float64}(pointer(evecs)),
            C_NULL, C_NULL, C_NULL, C_NULL)
        _omb_check(rc)
    end
    return kmags, [evecs[:, j] for j in 1:nev]
end

function ChainRulesCore.rrule(::typeof(solve_k_periodic), ω::T, ε⁻¹::AbstractArray{T,5}, Λ::Real,
    grid::Grid{3,T}, s::B200Solver; nev=1, max_eigsolves=60, maxiter=s.maxiter, k_tol=1e-8, eig_tol=1e-8,
    kwargs...) where {T<:Real}
    kmags, evecs = solve_k_periodic(ω, ε⁻¹, Λ, grid, s; nev, max_eigsolves, maxiter, k_tol, eig_tol, kwargs...)
    eps = convert(Array{Float64,5}, ε⁻¹)
    function b200_solve_k_periodic_pullback(ΔΩ)
        ΔΩ isa AbstractZero && return (NoTangent(), 0.0, zero(eps), 0.0, NoTangent(), NoTangent())
        k̄mags, ēvecs = ΔΩ
        kbar = k̄mags isa AbstractZero ? nothing : [k isa AbstractZero ? 0.0 : Float64(k) for k in k̄mags]
        n2 = length(first(evecs))
        ebar = ēvecs isa AbstractZero ? nothing :
               reduce(hcat, [e isa AbstractZero ? zeros(ComplexF64, n2) : ComplexF64.(e) for e in ēvecs])
        V = reduce(hcat, evecs)
        ω̄, Λ̄ = Ref(0.0), Ref(0.0)
        ε̄⁻¹ = zeros(Float64, size(eps))
        opt = Ref(_omb_options(s; k_tol, eig_tol, max_eigsolves, maxiter))
        GC.@preserve eps kmags V kbar ebar ε̄⁻¹ begin
            rc = ccall((:omb_pullback_periodic, OMB200_LIB), Cint,
                (Ptr{Cvoid}, Ref{OmbGrid3}, Cdouble, Ptr{Float64}, Cint, Ptr{Float64}, Ptr{Float64},
                 Ptr{Float64}, Ptr{Float64}, Ref{OmbOptions}, Ref{Float64}, Ptr{Float64}, Ref{Float64}, Ptr{Int32}),
                _omb_ctx(s), Ref(_omb_grid3(grid, Λ)), Float64(ω), eps, nev, kmags, Ptr{Float64}(pointer(V)),
                kbar === nothing ? Ptr{Float64}(C_NULL) : pointer(kbar),
                ebar === nothing ? Ptr{Float64}(C_NULL) : Ptr{Float64}(pointer(ebar)),
                opt, ω̄, ε̄⁻¹, Λ̄, C_NULL)
            _omb_check(rc)
        end
        return (NoTangent(), ω̄[], ε̄⁻¹, Λ̄[], NoTangent(), NoTangent())
    end
    return ((kmags, evecs), b200_solve_k_periodic_pullback)
end

# ---- Kottke smoothing on the device -------------------------------------------------------
# `SmoothingPlan` / `smooth_ε(plan, mat_vals)` of lib/DielectricSmoothing/src/smoothing_plan.jl
# computed by libomb200.  Shapes are passed as convex polygons: one (n, 2) vertex matrix per
# shape in priority order (a GeometryPrimitives Polygon's vertices, or a Cuboid's four
# corners); `minds` are the reference's 1-based material columns, the background last.
# `smooth_ε` gains a method for the device plan (MaxwellEigenmodes already has
# `using DielectricSmoothing`, src/MaxwellEigenmodes.jl:29).

mutable struct B200SmoothingPlan
    h::Ptr{Cvoid}
    grid::Grid{2,Float64}
end

function b200_smoothing_plan(polys::AbstractVector{<:AbstractMatrix}, minds, grid::Grid{2};
                             fill::Symbol=:plane, device::Int=0)
    nv = Int32[size(p, 1) for p in polys]
    verts = Float64[]
    for p in polys, i in axes(p, 1)
        push!(verts, p[i, 1], p[i, 2])
    end
    md = Int32[m - 1 for m in minds]
    h = Ref{Ptr{Cvoid}}(C_NULL)
    _omb_check(ccall((:omb_smoothing_plan_create, OMB200_LIB), Cint,
        (Ptr{Cvoid}, Ref{OmbGrid}, Int32, Ptr{Int32}, Ptr{Float64}, Ptr{Int32}, Int32, Ref{Ptr{Cvoid}}),
        _omb_ctx(B200Solver(; device=device)), _omb_grid(grid), length(polys), nv, verts, md,
        fill === :exact ? Int32(1) : Int32(0), h))
    plan = B200SmoothingPlan(h[], grid)
    finalizer(p -> ccall((:omb_smoothing_plan_destroy, OMB200_LIB), Cint, (Ptr{Cvoid},), p.h), plan)
    return plan
end

"""
    smooth_ε(plan::B200SmoothingPlan, mat_vals) -> Array{Float64,5}

The `(3, 3, 3, Nx, Ny)` smoothed (ε, ∂ωε, ∂²ωε) of `smooth_ε(plan, mat_vals)`, computed on
the device; `sliceinv_3x3` of its ε slice comes from `b200_smooth_epsinv`.
"""
function DielectricSmoothing.smooth_ε(plan::B200SmoothingPlan, mat_vals::AbstractMatrix{<:Real})
    M = Matrix{Float64}(mat_vals)
    out = Array{Float64}(undef, 3, 3, 3, plan.grid.Nx, plan.grid.Ny)
    _omb_check(ccall((:omb_smooth_eps, OMB200_LIB), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Int32, Int32, Ptr{Float64}, Ptr{Float64}),
        plan.h, M, size(M, 2), 1, out, C_NULL))
    return out
end

function b200_smooth_epsinv(plan::B200SmoothingPlan, mat_vals::AbstractMatrix{<:Real})
    M = Matrix{Float64}(mat_vals)
    out = Array{Float64}(undef, 3, 3, plan.grid.Nx, plan.grid.Ny)
    _omb_check(ccall((:omb_smooth_eps, OMB200_LIB), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Int32, Int32, Ptr{Float64}, Ptr{Float64}),
        plan.h, M, size(M, 2), 1, C_NULL, out))
    return out
end


# ---- learned warm start, autotuning and failure-detection controls ----------------------
# (new API of this backend; the reference has no counterpart)

"""
    b200_attach_warmstart(params::Vector{Float32}; device=0, batch_cap=32)

Create the warm-start network on `device`, load its FP32 parameters (the layout of
`omb_warmstart_get_params`: per layer W as [cout × 9·cin] row-major, then the biases; the
committed `omb200/data/warmstart_net.npz` holds them under "params", readable with NPZ.jl)
and attach it to the device's context, so `B200Solver(; warm_start=:learned)` uses it.
"""
function b200_attach_warmstart(params::Vector{Float32}; device::Int=0, batch_cap::Int=32)
    n = ccall((:omb_warmstart_num_params, OMB200_LIB), Int64, ())
    length(params) == n || error("expected $n warm-start parameters, got $(length(params))")
    ctx = _omb_ctx(B200Solver(; device=device))
    h = Ref{Ptr{Cvoid}}(C_NULL)
    _omb_check(ccall((:omb_warmstart_create, OMB200_LIB), Cint, (Ptr{Cvoid}, Int32, UInt64, Ref{Ptr{Cvoid}}),
        ctx, batch_cap, UInt64(0), h))
    _omb_check(ccall((:omb_warmstart_set_params, OMB200_LIB), Cint, (Ptr{Cvoid}, Ptr{Float32}), h[], params))
    _omb_check(ccall((:omb_ctx_set_warmstart, OMB200_LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), ctx, h[]))
    return h[]
end

"""
    b200_autotune(grid::Grid{2}; ncol=4, device=0) -> (row, col, wave)

Tune the FP32 operator tiles of `grid` now (batched solves tune unseen grids by themselves,
like FFTW planning at `ModeSolver` construction, src/maxwell.jl:940-943).
"""
function b200_autotune(grid::Grid{2}; ncol::Int=4, device::Int=0)
    r, c, w = Ref{Int32}(0), Ref{Int32}(0), Ref{Int32}(0)
    _omb_check(ccall((:omb_autotune, OMB200_LIB), Cint,
        (Ptr{Cvoid}, Ref{OmbGrid}, Int32, Ref{Int32}, Ref{Int32}, Ref{Int32}, Ptr{Float64}),
        _omb_ctx(B200Solver(; device=device)), _omb_grid(grid), ncol, r, c, w, C_NULL))
    return (r[], c[], w[])
end

"Limit (seconds) of the device's bounded pipeline waits; a wait that runs out is an error."
b200_set_wait_limit(seconds::Real; device::Int=0) = _omb_check(ccall((:omb_ctx_set_wait_limit, OMB200_LIB), Cint,
    (Ptr{Cvoid}, Float64), _omb_ctx(B200Solver(; device=device)), Float64(seconds)))
