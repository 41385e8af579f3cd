"""
    HadaMAGB200

B200 backend for HadaMAG.jl: exact SRE, MC_SRE and Mana on an NVIDIA B200 through
libhadamag_b200.so (C ABI declared in include/hadamag_b200.h).

    using HadaMAG, HadaMAGB200
    SRE(ψ, 2; backend = HadaMAGB200.B200())
    SRE(ψ, 2; backend = HadaMAGB200.B200(devices = [0, 1, 2, 3]))   # one call, four GPUs
    MC_SRE(ψ, 2; backend = HadaMAGB200.B200(), Nβ = 13, Nsamples = 1000, seed = 123)
    Mana(ψ3; backend = HadaMAGB200.B200())
    HadaMAGB200.Mana(ρ)                       # DensityMatrix{ComplexF64,3}
    HadaMAGB200.SRE_grad(ψ, 2)                # value and dSRE/dψ (no reference counterpart)
    Zygote.gradient(v -> HadaMAGB200.sre_value(v, 2), data(ψ))   # through the rrule

Passing the backend object works with the unmodified package: `_choose_backend` gets a
method for `B200` and `_apply_backend` routes to the functions below (the dispatch of
src/Backends/Dispatch.jl:12-90).  A `:b200` symbol needs one extra branch in
`_choose_backend` of HadaMAG itself.

The functions mirror the backend signatures of ext/HadaMAGCUDAExt.jl:1381-1410 (SRE),
src/Backends/Threads.jl:161-221 (MC_SRE) and 223-271 (Mana).  MC_SRE draws its proposal
stream with the calls of src/SRE.jl:142-145 and 164-169 (MersenneTwister(seed + i),
rand(rng, Nsamples) twice, rand(rng, 1:L) per flip) and hands it to the device, so a
given seed reproduces the chains of the CPU backends.
"""
module HadaMAGB200

# Explicit imports only: HadaMAG exports SRE, MC_SRE and Mana, and this module defines its
# own functions of those names (the backend entry points _apply_backend routes to), so
# `using HadaMAG` would bind the names to HadaMAG's functions instead.
import HadaMAG
using HadaMAG: StateVec, DensityMatrix, data, qubits, qudits
using Random
using ChainRulesCore

const LIB = Ref{String}(joinpath(@__DIR__, "..", "..", "..", "libhadamag_b200.so"))
const CTX = Dict{Int,Ptr{Cvoid}}()

const HM_FP64 = Cint(0)
const HM_FP32 = Cint(1)
const HM_PLAIN = Cint(2)

"""
    B200(; device = 0, devices = nothing)

The sm_100a backend.  `device` selects the CUDA device; `devices` (a vector of device
indices) runs the exact SRE over several GPUs in one call, each sweeping a contiguous
share of the Gray range from its own host thread (`hm_sre_multi`: the per-node split of
the :mpi_cuda backend, ext/HadaMAGMPICUDAExt.jl:49-95).
"""
struct B200 <: HadaMAG.AbstractBackend
    device::Int
    devices::Vector{Int}
end
B200(; device::Int = 0, devices = nothing) =
    B200(devices === nothing ? device : first(devices), devices === nothing ? Int[] : collect(Int, devices))

const CURRENT = Ref{B200}(B200())

function context(dev::Int = CURRENT[].device)
    h = get(CTX, dev, C_NULL)
    if h == C_NULL
        r = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:hm_create, LIB[]), Cint, (Ref{Ptr{Cvoid}}, Cint), r, dev)
        rc == 0 || error("hm_create(device = $dev) failed with status $rc (no usable CUDA device?)")
        h = CTX[dev] = r[]
        atexit(() -> ccall((:hm_destroy, LIB[]), Cint, (Ptr{Cvoid},), h))
    end
    return h
end

# HM_ERR_ARG, HM_ERR_SIZE, HM_ERR_Q and HM_ERR_ALIGN are caller errors
function check(rc, what)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:hm_last_error, LIB[]), Cstring, (Ptr{Cvoid},), context()))
    rc in (-1, -2, -3, -7) && throw(ArgumentError("$what: $msg"))
    error("$what failed with status $rc: $msg")
end

function check_multi(rc, what)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:hm_multi_last_error, LIB[]), Cstring, ()))
    rc in (-1, -2, -3, -7) && throw(ArgumentError("$what: $msg"))
    error("$what failed with status $rc: $msg")
end

function SRE(ψ, q::Number; progress = false, precision = HM_FP64, kwargs...)
    progress && @warn "Progress bar not implemented for the B200 backend."
    v = collect(ComplexF64, data(ψ))
    out = zeros(Float64, 1)
    lost = Ref{Float64}(0.0)
    devs = CURRENT[].devices
    if length(devs) > 1
        rc = ccall((:hm_sre_multi, LIB[]), Cint,
                   (Ptr{Cint}, Cint, Ptr{Float64}, Cint, Ptr{Float64}, Cint, Cint, Ptr{Float64}, Ref{Float64}),
                   Cint.(devs), length(devs), reinterpret(Float64, v), qubits(ψ), Float64[q], 1, precision, out,
                   lost)
        check_multi(rc, "hm_sre_multi")
    else
        rc = ccall((:hm_sre, LIB[]), Cint,
                   (Ptr{Cvoid}, Ptr{Float64}, Cint, Ptr{Float64}, Cint, Cint, Ptr{Float64}, Ref{Float64}),
                   context(), reinterpret(Float64, v), qubits(ψ), Float64[q], 1, precision, out, lost)
        check(rc, "hm_sre")
    end
    return (out[1], lost[])
end

function MC_SRE(ψ, q, Nβ::Int, Nsamples::Int; seed::Union{Nothing,Int} = nothing, progress = true)
    Nβ % 2 == 1 || error("Simpson needs an odd number of β points.")
    L = qubits(ψ)
    base_seed = seed === nothing ? rand(1:(10^9)) : seed
    pd = Vector{UInt64}(undef, Nβ * Nsamples)
    rs = Vector{Float64}(undef, Nβ * Nsamples)
    MASK = UInt64(1) .<< (0:(L-1))
    for i = 1:Nβ
        rng = MersenneTwister(base_seed + i)
        tries = floor.(Int, rand(rng, Nsamples) .* 9) .+ 1
        r = rand(rng, Nsamples)
        for t = 1:Nsamples
            Δ = zero(UInt64)
            for _ = 1:tries[t]
                Δ ⊻= MASK[rand(rng, 1:L)]
            end
            pd[(i-1)*Nsamples+t] = Δ
            rs[(i-1)*Nsamples+t] = r[t]
        end
    end
    v = collect(ComplexF64, data(ψ))
    m2 = Ref{Float64}(0.0)
    M2, M2ADD, P2 = zeros(Nβ), zeros(Nβ), zeros(Nβ)
    rc = ccall((:hm_mc_sre, LIB[]), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Cint, Cdouble, Cint, Cint, Ptr{UInt64}, Ptr{Float64},
                Ref{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{UInt64}),
               context(), reinterpret(Float64, v), L, Float64(q), Nβ, Nsamples, pd, rs, m2, M2, M2ADD, P2,
               C_NULL)
    check(rc, "hm_mc_sre")
    return m2[]
end

function Mana(ψ::StateVec{T,3}; progress = false) where {T}
    v = collect(ComplexF64, data(ψ))
    out = Ref{Float64}(0.0)
    rc = ccall((:hm_mana_pure, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cint, Ref{Float64}),
               context(), reinterpret(Float64, v), qudits(ψ), out)
    check(rc, "hm_mana_pure")
    return out[]
end

function Mana(ρ::DensityMatrix{T,3}; kwargs...) where {T}
    m = collect(ComplexF64, data(ρ))          # column-major, as Julia stores it
    out = Ref{Float64}(0.0)
    rc = ccall((:hm_mana_mixed, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cint, Ref{Float64}),
               context(), reinterpret(Float64, vec(m)), qudits(ρ), out)
    check(rc, "hm_mana_mixed")
    return out[]
end

"""
    SRE_grad(ψ, q = 2) -> (value, grad)

Value and gradient of SRE_q; `grad[r] = ∂SRE/∂Re ψ[r] + im * ∂SRE/∂Im ψ[r]`.
"""
function SRE_grad(ψ, q = 2)
    v = collect(ComplexF64, data(ψ))
    g = similar(v)
    val = Ref{Float64}(0.0)
    rc = ccall((:hm_sre_grad, LIB[]), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Cint, Cdouble, Ref{Float64}, Ptr{Float64}),
               context(), reinterpret(Float64, v), qubits(ψ), Float64(q), val, reinterpret(Float64, g))
    check(rc, "hm_sre_grad")
    return (val[], g)
end

"""
    sre_value(v::AbstractVector{ComplexF64}, q = 2) -> Float64

SRE_q of the normalised amplitude vector `v` (length 2^n) as a plain differentiable
function: its `ChainRulesCore.rrule` runs the adjoint kernel (`hm_sre_grad`) once and
returns the value with a pullback.  For a real function of complex input the cotangent
is dSRE/dRe v + im dSRE/dIm v, which is what the kernel produces.
"""
function sre_value(v::AbstractVector{ComplexF64}, q = 2)
    out = zeros(Float64, 1)
    lost = Ref{Float64}(0.0)
    w = collect(v)
    rc = ccall((:hm_sre, LIB[]), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Cint, Ptr{Float64}, Cint, Cint, Ptr{Float64}, Ref{Float64}),
               context(), reinterpret(Float64, w), trailing_zeros(length(w)), Float64[q], 1, HM_FP64, out, lost)
    check(rc, "hm_sre")
    return out[1]
end

function ChainRulesCore.rrule(::typeof(sre_value), v::AbstractVector{ComplexF64}, q)
    w = collect(v)
    g = similar(w)
    val = Ref{Float64}(0.0)
    rc = ccall((:hm_sre_grad, LIB[]), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Cint, Cdouble, Ref{Float64}, Ptr{Float64}),
               context(), reinterpret(Float64, w), trailing_zeros(length(w)), Float64(q), val,
               reinterpret(Float64, g))
    check(rc, "hm_sre_grad")
    sre_pullback(ȳ) = (NoTangent(), ȳ .* g, NoTangent())
    return val[], sre_pullback
end

"""
    apply_2gate!(ψ::StateVec{T,q}, gate, s1, s2)

Two-site gate on sites `s1`, `s2` (1-based, site 1 least significant) on the GPU
(`hm_apply_2gate`), as `HadaMAG.apply_2gate!` (src/State.jl:254-345).
"""
function apply_2gate!(ψ::StateVec{T,q}, gate::AbstractMatrix, s1::Int, s2::Int) where {T,q}
    v = collect(ComplexF64, data(ψ))
    g = collect(ComplexF64, gate)              # column-major, as Julia stores it
    rc = ccall((:hm_apply_2gate, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cint, Cint, Ptr{Float64}, Cint, Cint),
               context(), reinterpret(Float64, v), qudits(ψ), q, reinterpret(Float64, vec(g)), s1, s2)
    check(rc, "hm_apply_2gate")
    data(ψ) .= v
    return ψ
end

"""
    apply_brick_wall_haar!(ψ::StateVec{T,q}, depth, rng = Random.GLOBAL_RNG)

Brick wall of Haar-random two-site gates on the GPU (`hm_brick_wall`); the gates are
drawn on the host with `HadaMAG.haar_random_unitary`, in the reference's layer order
(src/State.jl:200-221), so a given `rng` yields the reference's circuit.
"""
function apply_brick_wall_haar!(ψ::StateVec{T,q}, depth::Int, rng::AbstractRNG = Random.GLOBAL_RNG) where {T,q}
    n = qudits(ψ)
    gates = ComplexF64[]
    ngates = 0
    for layer = 1:depth, s = (isodd(layer) ? 1 : 2):2:(n-1)
        append!(gates, vec(ComplexF64.(HadaMAG.haar_random_unitary(q, 2, rng))))
        ngates += 1
    end
    v = collect(ComplexF64, data(ψ))
    rc = ccall((:hm_brick_wall, LIB[]), Cint, (Ptr{Cvoid}, Ptr{Float64}, Cint, Cint, Cint, Ptr{Float64}, Cint),
               context(), reinterpret(Float64, v), n, q, depth, reinterpret(Float64, gates), ngates)
    check(rc, "hm_brick_wall")
    data(ψ) .= v
    return ψ
end

"""
    reduced_density_matrix(ψ::StateVec{T,q}, NA; side = :right) -> DensityMatrix

ρ_A on the GPU (`hm_reduced_density_matrix`), as `HadaMAG.reduced_density_matrix`
(src/DensityMatrix.jl:94-123).
"""
function reduced_density_matrix(ψ::StateVec{T,q}, NA::Int; side::Symbol = :right) where {T,q}
    side in (:left, :right) || throw(ArgumentError("side must be :left or :right (got $side)"))
    v = collect(ComplexF64, data(ψ))
    dimA = q^NA
    ρ = Matrix{ComplexF64}(undef, dimA, dimA)
    rc = ccall((:hm_reduced_density_matrix, LIB[]), Cint,
               (Ptr{Cvoid}, Ptr{Float64}, Cint, Cint, Cint, Cint, Ptr{Float64}),
               context(), reinterpret(Float64, v), qudits(ψ), q, NA, side === :left ? 0 : 1,
               reinterpret(Float64, vec(ρ)))
    check(rc, "hm_reduced_density_matrix")
    return DensityMatrix(ρ; q = q)
end

"""
    load_state(path; q = 2) -> StateVec

As `HadaMAG.load_state` (src/State.jl:388-404) for .npy and text files, read by
`hm_load_state` straight into page-locked host memory and copied into the StateVec's
vector.  .jld2 files go to `HadaMAG.load_state`.
"""
function load_state(path::AbstractString; q::Int = 2)
    endswith(path, ".jld2") && return HadaMAG.load_state(path; q = q)
    p = Ref{Ptr{Float64}}(C_NULL)
    n = Ref{UInt64}(0)
    rc = ccall((:hm_load_state, LIB[]), Cint, (Cstring, Cint, Ref{Ptr{Float64}}, Ref{UInt64}), path, q, p, n)
    if rc != 0
        msg = unsafe_string(ccall((:hm_io_last_error, LIB[]), Cstring, ()))
        throw(ArgumentError(msg))
    end
    v = copy(reinterpret(ComplexF64, unsafe_wrap(Array, p[], 2 * Int(n[]))))
    ccall((:hm_free_state, LIB[]), Cint, (Ptr{Float64},), p[])
    return StateVec(v; q = q)
end

HadaMAG._choose_backend(b::B200) = b
function HadaMAG._apply_backend(b::B200, fsym, args...; kw...)
    CURRENT[] = b
    return getfield(HadaMAGB200, fsym)(args...; kw...)
end

end # module
