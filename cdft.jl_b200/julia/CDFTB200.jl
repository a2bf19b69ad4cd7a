"""
    CDFTB200

Julia shim that routes cDFT.jl's `converge!` / `δFδρ_res` / `F_res` for PC-SAFT systems to
libcdft_b200 (B200, sm_100a) through `ccall`.  Select it with
`DFTSystem(model, structure, fields, DFTOptions(B200Device()))`.

Struct layouts mirror `include/cdft_b200.h` field by field (plain bits, C alignment).
"""
module CDFTB200

using cDFT
using cDFT: DFTSystem, DFTOptions, DFTProblem, AASol
using Clapeyron: PCSAFTModel
import Clapeyron                 # qualified calls (Clapeyron.assoc_pair_length)
using ChainRulesCore
using CUDA

const LIB = get(ENV, "CDFT_B200_LIB", joinpath(@__DIR__, "..", "cdft_b200", "libcdft_b200.so"))
const MAX_NC = 4
const MAX_ASSOC = 8

"""
    B200Device(; mixed = false)

The device of `DFTOptions` that routes a PC-SAFT system to libcdft_b200.  `mixed = true`
selects the mixed-precision path (FP32 convolutions and Φ; FP64 Anderson, norms and
integrals; an FP64 polish to the FP64 fixed point).  `DFTOptions(B200Device(); precision =
Float64)` is the default; `precision = Float32` (the reference's all-FP32 mode,
devices.jl:29-40) is refused: the library computes no FP32 solver.
"""
struct B200Device
    mixed::Bool
end
B200Device(; mixed::Bool = false) = B200Device(mixed)
export B200Device

struct CDFTAssocPair
    icomp::Cint
    jcomp::Cint
    isite::Cint
    jsite::Cint
    n_ia::Cint
    n_jb::Cint
    eps_ab::Cdouble
    kappa_ab::Cdouble
end

struct CDFTSystemDesc
    nd::Cint
    ngrid::NTuple{3,Cint}
    bounds::NTuple{6,Cdouble}             # [lb, ub] per dimension
    coord::Cint
    nc::Cint
    m::NTuple{MAX_NC,Cdouble}
    hsd::NTuple{MAX_NC,Cdouble}
    sigma::NTuple{MAX_NC * MAX_NC,Cdouble}
    eps::NTuple{MAX_NC * MAX_NC,Cdouble}
    L::Cdouble
    T::Cdouble
    n_assoc::Cint
    assoc::NTuple{MAX_ASSOC,CDFTAssocPair}
    mu_res_plus_ln_rhob::NTuple{MAX_NC,Cdouble}
    vext::Ptr{Cdouble}
    precision::Cint
end

struct CDFTSolverOpts
    m::Cint
    maxit::Cint
    rtol::Cdouble
    atol::Cdouble
    beta::Cdouble
    picard_maxit::Cint
    picard_beta::Cdouble
    picard_rtol::Cdouble
    picard_atol::Cdouble
    time_budget_s::Cdouble
    iters_per_launch::Cint
    engine::Cint
    mixed_switch_rtol::Cdouble
    snapshot_every::Cint
    snapshot::Ptr{Cvoid}            # void (*)(void* user, int system, int evaluations, const double* rho)
    snapshot_user::Ptr{Cvoid}
end

mutable struct CDFTResult
    idid::Cint
    errcode::Cint
    iterations::Cint
    evaluations::Cint
    resnorm::Cdouble
    tol::Cdouble
    history::Ptr{Cdouble}
    history_cap::Cint
    history_len::Cint
    CDFTResult() = new(0, 0, 0, 0, 0.0, 0.0, C_NULL, 0, 0)
end

function check(rc)
    if rc != 0
        buf = Vector{UInt8}(undef, 512)
        ccall((:cdft_last_error, LIB), Cint, (Ptr{UInt8}, Csize_t), buf, length(buf))
        error("cdft_b200 error $rc: " * unsafe_string(pointer(buf)))
    end
    return rc
end

pad(v, n) = ntuple(i -> i <= length(v) ? Float64(v[i]) : 0.0, n)

# Everything DFTSystem carries into the hot path (base.jl:50-73, PCSAFT.jl:65-72,213-285),
# in SI units; the library forms the reduced parameters itself.
function system_desc(system::DFTSystem{<:PCSAFTModel}, vext::Union{Nothing,Array{Float64}})
    model, st, sp = system.model, system.structure, system.species
    nc = length(model)
    nc <= MAX_NC || error("at most $MAX_NC components")
    nd = length(st.ngrid)
    (p, T) = st.conditions
    sig = model.params.sigma.values
    eps = model.params.epsilon.values
    sigma = pad([sig[i, j] for i in 1:nc for j in 1:nc], MAX_NC * MAX_NC)
    epsv = pad([eps[i, j] for i in 1:nc for j in 1:nc], MAX_NC * MAX_NC)
    b = zeros(6)
    for d in 1:nd
        b[2d-1], b[2d] = st.bounds[d]
    end
    ng = ntuple(d -> d <= nd ? Cint(st.ngrid[d]) : Cint(1), 3)
    nassoc = Clapeyron.assoc_pair_length(model)
    nassoc <= MAX_ASSOC || error("at most $MAX_ASSOC association pairs per system")
    empty = CDFTAssocPair(0, 0, 0, 0, 0, 0, 0.0, 0.0)
    pairs = if nassoc >= 1
        (icomp, jcomp, isite, jsite, epsa, kap, _, _, nsflat, nscum, _) =
            cDFT.pack_assoc_params(model, sp.size ./ cDFT.length_scale(model))
        ntuple(MAX_ASSOC) do p
            p > nassoc && return empty
            ia = nscum[icomp[p]] + isite[p]
            jb = nscum[jcomp[p]] + jsite[p]
            CDFTAssocPair(icomp[p] - 1, jcomp[p] - 1, isite[p] - 1, jsite[p] - 1,
                          nsflat[ia], nsflat[jb], epsa[p], kap[p])
        end
    else
        ntuple(_ -> empty, MAX_ASSOC)
    end
    coord = st isa cDFT.DFTStructByCoord{cDFT.Cartesian} ? 0 :
            st isa cDFT.DFTStructByCoord{cDFT.Spherical} ? 1 :
            st isa cDFT.DFTStructByCoord{cDFT.Cylindrical} ? 2 : error("unsupported coordinates")
    cDFT.fptype(system.options) == Float64 ||
        error("B200Device computes in FP64 or mixed precision (B200Device(mixed = true)); precision = Float32 is not offered")
    prec = system.options.device.mixed ? Cint(1) : Cint(0)
    CDFTSystemDesc(nd, ng, Tuple(b), coord, nc, pad(model.params.segment.values, MAX_NC),
                   pad(sp.size, MAX_NC), sigma, epsv, cDFT.length_scale(model), T, nassoc, pairs,
                   pad(sp.chempot_res .+ log.(sp.bulk_density), MAX_NC),
                   vext === nothing ? Ptr{Cdouble}(C_NULL) : pointer(vext), prec)
end

const PLANS = IdDict{Any,Ptr{Cvoid}}()

function plan_for(system)
    get!(PLANS, system) do
        vext = external_potential(system)
        desc = system_desc(system, vext)
        plan = Ref{Ptr{Cvoid}}(C_NULL)
        GC.@preserve vext check(ccall((:cdft_plan_create, LIB), Cint,
                                      (Ref{CDFTSystemDesc}, Ref{Ptr{Cvoid}}), desc, plan))
        finalizer(system) do _
            ccall((:cdft_plan_destroy, LIB), Cint, (Ptr{Cvoid},), plan[])
        end
        plan[]
    end
end

# preallocate_external_potential (devices.jl:71-102): Vext summed over the system's fields
function external_potential(system)
    fields = system.external_field
    fields === nothing && return nothing
    ρ = cDFT.initialize_profiles(system)
    z = cDFT.get_coords(system.structure)
    V = zeros(size(ρ))
    for f in fields
        V .+= cDFT.evaluate_external_field!(system.structure, f, system.model, ρ, ρ, z)
    end
    return V
end

const B200System = DFTSystem{<:PCSAFTModel,<:Any,<:Any,<:Any,<:Any,<:Any,<:DFTOptions{B200Device}}

solver_opts(method::AASol; every = 0, cb = C_NULL, user = C_NULL) =
    CDFTSolverOpts(method.m, method.maxit, method.rtol, method.atol, method.beta, method.picard_maxit,
                   method.picard_beta, method.picard_rtol, method.picard_atol, 0.0, 0, 0, 0.0,
                   every, cb, user)

# DFTProblem's save_callback / log_interval (converge.jl:31-60,256-267): the library hands out the
# profile every gcd(save_interval, log_interval) evaluations; the free energy of the logged
# profiles is computed once converge! returns (the callback runs while the plan is busy)
mutable struct Hooks
    prob::Any
    shape::Tuple
    logged::Vector{Tuple{Int,Array{Float64}}}
end

function snapshot_hook(user::Ptr{Cvoid}, s::Cint, it::Cint, rho::Ptr{Cdouble})
    h = unsafe_pointer_to_objref(user)::Hooks
    ρ = copy(reshape(unsafe_wrap(Array, rho, prod(h.shape)), h.shape))
    p = h.prob
    p.save_interval > 0 && it % p.save_interval == 0 && p.save_callback(Int(it), ρ)
    p.log_interval > 0 && it % p.log_interval == 0 && push!(h.logged, (Int(it), ρ))
    return nothing
end

function report(prob, method, res, hooks)
    if hooks !== nothing
        for (it, ρ) in hooks.logged
            @info "DFT iter $(lpad(it, 5)) | F = $(round(cDFT.free_energy(prob.system, ρ); sigdigits=6))"
        end
    end
    if method.verbose
        msg = res.idid != 0 ? "DFT converged" : "DFT did not converge"
        @info "$msg after $(res.evaluations) evaluations: err = $(round(res.resnorm; sigdigits=3))"
    end
end

function with_hooks(f, prob, method, shape)
    every = prob.log_interval > 0 && prob.save_interval > 0 ? gcd(prob.log_interval, prob.save_interval) :
            max(prob.log_interval, prob.save_interval)
    every == 0 && return f(solver_opts(method), nothing)
    hooks = Hooks(prob, shape, Tuple{Int,Array{Float64}}[])
    cb = @cfunction(snapshot_hook, Cvoid, (Ptr{Cvoid}, Cint, Cint, Ptr{Cdouble}))
    GC.@preserve hooks f(solver_opts(method; every = every, cb = cb, user = pointer_from_objref(hooks)), hooks)
end

# converge!(prob::DFTProblem, method::AASol, ρ), src/methods/converge.jl:220-254
function cDFT.converge!(prob::DFTProblem{<:B200System}, method::AASol, ρ::Array{Float64})
    res = CDFTResult()
    with_hooks(prob, method, size(ρ)) do opts, hooks
        check(ccall((:cdft_converge, LIB), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ref{CDFTSolverOpts}, Ref{CDFTResult}),
                    plan_for(prob.system), ρ, opts, res))
        report(prob, method, res, hooks)
    end
    return nothing
end

# the same for a profile in device memory (CUDA.jl): the plan runs on the task's stream
function cDFT.converge!(prob::DFTProblem{<:B200System}, method::AASol, ρ::CuArray{Float64})
    res = CDFTResult()
    plan = plan_for(prob.system)
    check(ccall((:cdft_plan_set_stream, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), plan, CUDA.stream().handle))
    with_hooks(prob, method, size(ρ)) do opts, hooks
        check(ccall((:cdft_converge_dev, LIB), Cint,
                    (Ptr{Cvoid}, CuPtr{Float64}, Ref{CDFTSolverOpts}, Ref{CDFTResult}),
                    plan, pointer(ρ), opts, res))
        report(prob, method, res, hooks)
    end
    return nothing
end

"""
    converge_batch!(systems, ρs; kwargs...)

Converge many independent B200 systems (state points, pore widths; uneven grids) in one
batch: every kernel launch covers all of them (cdft_batch_converge).  The keywords are
converge!'s (`AASol(system; kwargs...)`, converge.jl:3-13), shared by the batch; the
systems must agree in the number of components, dimension and precision.  `ρs` are
`Array{Float64}` (host) or `CuArray{Float64}` (device) profiles, converged in place.
Returns the per-system (idid, errcode, evaluations).
"""
function converge_batch!(systems::AbstractVector, ρs::AbstractVector; kwargs...)
    n = length(systems)
    n == length(ρs) || error("systems and profiles differ in length")
    method = AASol(first(systems); kwargs...)
    opts = solver_opts(method)
    plans = Ptr{Cvoid}[plan_for(s) for s in systems]
    # cdft_result records are laid out contiguously for the library
    buf = Vector{UInt8}(undef, n * sizeof(CDFTResult))
    if all(r -> r isa CuArray, ρs)
        check(ccall((:cdft_plan_set_stream, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), plans[1], CUDA.stream().handle))
        for p in plans[2:end]
            check(ccall((:cdft_plan_set_stream, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), p, CUDA.stream().handle))
        end
        ptrs = [reinterpret(Ptr{Float64}, pointer(r)) for r in ρs]
        check(ccall((:cdft_batch_converge_dev, LIB), Cint,
                    (Ptr{Ptr{Cvoid}}, Cint, Ptr{Ptr{Float64}}, Ref{CDFTSolverOpts}, Ptr{UInt8}),
                    plans, n, ptrs, opts, buf))
    else
        GC.@preserve ρs begin
            ptrs = [pointer(r) for r in ρs]
            check(ccall((:cdft_batch_converge, LIB), Cint,
                        (Ptr{Ptr{Cvoid}}, Cint, Ptr{Ptr{Float64}}, Ref{CDFTSolverOpts}, Ptr{UInt8}),
                        plans, n, ptrs, opts, buf))
        end
    end
    out = [unsafe_load(Ptr{CDFTResult}(pointer(buf)) + (k - 1) * sizeof(CDFTResult)) for k in 1:n]
    return [(r.idid != 0, Int(r.errcode), Int(r.evaluations)) for r in out]
end
export converge_batch!

# δFδρ_res(system, ρ), src/models/models.jl:194-200
function cDFT.δFδρ_res(system::B200System, ρ::Array{Float64})
    out = similar(ρ)
    check(ccall((:cdft_functional_derivative, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}),
                plan_for(system), ρ, out))
    return out
end

# F_res(system, ρ), src/models/models.jl:86-91
function cDFT.F_res(system::B200System, ρ::Array{Float64})
    F = Ref(0.0)
    check(ccall((:cdft_free_energy_res, LIB), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ref{Cdouble}),
                plan_for(system), ρ, F))
    return F[]
end

# δFδρ_res for a device profile (CuArray): cdft_functional_derivative_dev on the task's stream
function cDFT.δFδρ_res(system::B200System, ρ::CuArray{Float64})
    out = similar(ρ)
    plan = plan_for(system)
    check(ccall((:cdft_plan_set_stream, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}), plan, CUDA.stream().handle))
    check(ccall((:cdft_functional_derivative_dev, LIB), Cint, (Ptr{Cvoid}, CuPtr{Float64}, CuPtr{Float64}),
                plan, pointer(ρ), pointer(out)))
    return out
end

# ---------------------------------------------------------------------------
# dγ/dθ: the interfacial tension of a converged two-interface box as a function of the
# model parameters θ = (σ_k [Å], ε_k/k_B [K], m_k), k = 1..nc, with its reverse rule.
# At the converged profile δΩ/δρ = 0, so the pullback needs no pass through converge!:
# dγ/dθ = [k_B T ∂F_res/∂θ|ρ − Σ_i dμ_i/dθ ∫ρ_i + dp/dθ ∫1] / 2  (cdft_grad_params).
# ---------------------------------------------------------------------------
"""
    interface_tension(θ, system, ρ; dμdθ = nothing, dpdθ = nothing)

γ of the converged TwoPhase1DCart profile `ρ` of `system`, whose model has the parameters
`θ` (checked): surface_tension(system, ρ) / 2, the two interfaces of the periodic box
(interfacial_tension.jl:30, surface_tension.jl:28).  `dμdθ` (nc × 3nc, J/mol per unit of θ)
and `dpdθ` (3nc, Pa) describe how the bulk state follows θ (e.g. along the LLE, from
Clapeyron with ForwardDiff); `nothing` holds it fixed.  Differentiable with ChainRulesCore.
"""
"""
    saturation_b200(model, T) -> (p, ρl, ρv)

Vapour-liquid coexistence of a pure PC-SAFT component at every temperature in `T` (K), in
one device launch (`cdft_saturation_pure`): pressures in Pa, densities in mol/m³.  This is
the state `surface_tension(model, T, x)` takes from `bubble_pressure` for a pure component
(src/methods/surface_tension.jl:13-20).  The association pair (2B self-association) comes
from `pack_assoc_params`; its diameters do not enter the bulk equations.
"""
function saturation_b200(model::PCSAFTModel, T::AbstractVector{<:Real})
    length(model) == 1 || error("saturation_b200 covers pure components")
    Tv = Vector{Float64}(T)
    n = length(Tv)
    σ, ϵ = model.params.sigma.values[1, 1], model.params.epsilon.values[1, 1]
    nassoc = Clapeyron.assoc_pair_length(model)
    empty = CDFTAssocPair(0, 0, 0, 0, 0, 0, 0.0, 0.0)
    pairs = if nassoc >= 1
        (icomp, jcomp, isite, jsite, epsa, kap, _, _, nsflat, nscum, _) = cDFT.pack_assoc_params(model, [1.0])
        ntuple(MAX_ASSOC) do p
            p > nassoc && return empty
            CDFTAssocPair(icomp[p] - 1, jcomp[p] - 1, isite[p] - 1, jsite[p] - 1,
                          nsflat[nscum[icomp[p]] + isite[p]], nsflat[nscum[jcomp[p]] + jsite[p]], epsa[p], kap[p])
        end
    else
        ntuple(_ -> empty, MAX_ASSOC)
    end
    d0 = σ * (1 - 0.12 * exp(-3ϵ / Tv[1]))     # hsd and T of the descriptor are not used
    desc = CDFTSystemDesc(1, (Cint(1), Cint(1), Cint(1)), ntuple(_ -> 0.0, 6), 0, 1,
                          pad([model.params.segment.values[1]], MAX_NC), pad([d0], MAX_NC),
                          pad([σ], MAX_NC * MAX_NC), pad([ϵ], MAX_NC * MAX_NC), cDFT.length_scale(model),
                          Tv[1], nassoc, pairs, pad([0.0], MAX_NC), Ptr{Cdouble}(C_NULL), Cint(0))
    p, ρl, ρv, st = zeros(n), zeros(n), zeros(n), zeros(Cint, n)
    check(ccall((:cdft_saturation_pure, LIB), Cint,
                (Ref{CDFTSystemDesc}, Cint, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cdouble}, Ptr{Cint}),
                desc, n, Tv, p, ρl, ρv, st))
    all(==(0), st) || error("no coexistence at T = $(Tv[st .!= 0]) (status $(st[st .!= 0]))")
    return p, ρl, ρv
end

"""
    surface_tension_b200(model, T; mixed = false)

`surface_tension(model, T, [1.0])` (src/methods/surface_tension.jl:13-29) at every
temperature in `T` on the B200: the coexistence from `saturation_b200`, a
`TwoPhase1DCart` on [-10L, 10L] with 201 points per temperature, the systems converged in one
batch and `surface_tension(system, ρ) / 2`.
"""
function surface_tension_b200(model::PCSAFTModel, T::AbstractVector{<:Real}; mixed = false)
    p, ρl, ρv = saturation_b200(model, T)
    L = cDFT.length_scale(model)
    systems = [DFTSystem(model, cDFT.TwoPhase1DCart((p[k], Float64(T[k])), [ρl[k]], [ρv[k]], [-10L, 10L], (201,)),
                         DFTOptions(B200Device(mixed))) for k in eachindex(p)]
    ρs = [cDFT.initialize_profiles(s) for s in systems]
    converge_batch!(systems, ρs)
    return [cDFT.surface_tension(s, ρ) / 2 for (s, ρ) in zip(systems, ρs)]
end
export saturation_b200, surface_tension_b200

function interface_tension(θ::AbstractVector, system::B200System, ρ::Array{Float64}; dμdθ = nothing, dpdθ = nothing)
    model = system.model
    nc = length(model)
    θm = reduce(vcat, [[model.params.sigma.values[k, k] * 1e10, model.params.epsilon.values[k, k],
                        model.params.segment.values[k]] for k in 1:nc])
    isapprox(θ, θm; rtol = 1e-12) || error("θ differs from the parameters of the system's model")
    return cDFT.surface_tension(system, ρ) / 2
end
export interface_tension

function ChainRulesCore.rrule(::typeof(interface_tension), θ::AbstractVector, system::B200System,
                              ρ::Array{Float64}; dμdθ = nothing, dpdθ = nothing)
    γ = interface_tension(θ, system, ρ; dμdθ, dpdθ)
    nt = 3 * length(system.model)
    dΩ = zeros(nt)
    μ = dμdθ === nothing ? C_NULL : Matrix{Float64}(transpose(dμdθ))   # row-major nc x 3nc for C
    p = dpdθ === nothing ? C_NULL : Vector{Float64}(dpdθ)
    GC.@preserve μ p check(ccall((:cdft_grad_params, LIB), Cint,
                                 (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                                 plan_for(system), ρ, μ === C_NULL ? C_NULL : pointer(μ),
                                 p === C_NULL ? C_NULL : pointer(p), dΩ))
    function interface_tension_pullback(γ̄)
        return (NoTangent(), unthunk(γ̄) .* dΩ ./ 2, NoTangent(), NoTangent())
    end
    return γ, interface_tension_pullback
end

end # module
