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

const LIB = get(ENV, "CDFT_B200_LIB", joinpath(@__DIR__, "..", "cdft_b200", "libcdft_b200.so"))
const MAX_NC = 4
const MAX_ASSOC = 1

struct B200Device end
export B200Device

struct CDFTAssocPair
    icomp::Cint
    jcomp::Cint
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
    nassoc <= MAX_ASSOC || error("one association pair per system is supported")
    pairs = if nassoc == 1
        (icomp, jcomp, isite, jsite, epsa, kap, _, _, nsflat, nscum, _) =
            cDFT.pack_assoc_params(model, sp.size ./ cDFT.length_scale(model))
        ia = nscum[icomp[1]] + isite[1]
        jb = nscum[jcomp[1]] + jsite[1]
        (CDFTAssocPair(icomp[1] - 1, jcomp[1] - 1, nsflat[ia], nsflat[jb], epsa[1], kap[1]),)
    else
        (CDFTAssocPair(0, 0, 0, 0, 0.0, 0.0),)
    end
    coord = st isa cDFT.DFTStructByCoord{cDFT.Cartesian} ? 0 :
            st isa cDFT.DFTStructByCoord{cDFT.Spherical} ? 1 :
            st isa cDFT.DFTStructByCoord{cDFT.Cylindrical} ? 2 : error("unsupported coordinates")
    prec = cDFT.fptype(system.options) == Float64 ? Cint(0) : Cint(1)
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

# converge!(prob::DFTProblem, method::AASol, ρ), src/methods/converge.jl:220-254
function cDFT.converge!(prob::DFTProblem{<:B200System}, method::AASol, ρ::Array{Float64})
    opts = CDFTSolverOpts(method.m, method.maxit, method.rtol, method.atol, method.beta,
                          method.picard_maxit, method.picard_beta, method.picard_rtol,
                          method.picard_atol, 0.0, 0, 0, 0.0)
    res = CDFTResult()
    check(ccall((:cdft_converge, LIB), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ref{CDFTSolverOpts}, Ref{CDFTResult}),
                plan_for(prob.system), ρ, opts, res))
    if method.verbose
        msg = res.idid != 0 ? "DFT converged" : "DFT did not converge"
        @info "$msg after $(res.evaluations) evaluations: err = $(round(res.resnorm; sigdigits=3))"
    end
    return nothing
end

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

end # module
