"""
    DiscoDJB200

`ccall` bindings of libdjb200.so (include/djb200.h) for DiscoDJNative: a
`PMSolverB200` that implements `pm_acceleration!` on a B200, and `run_nbody_b200`,
the body of `run_nbody` (native/DiscoDJNative/src/nbody/run_nbody.jl:124-172) with
the particle state resident on the GPU. Host arrays (`Array{Float32,4}`) and device
arrays (`CuArray{Float32,4}`, via their pointers) of shape (n,n,n,3) are both
accepted, exactly as laid out by the reference (`pm.jl:15-17`).

Differentiation: `pm_acceleration_b200`, `pm_step_b200`, `run_states_b200` and
`state_power_spectrum_b200` are pure functions with ChainRulesCore `rrule`s over the
library's hand-written adjoints (djb_pm_acceleration_vjp, djb_step_vjp,
djb_state_power_spectrum_vjp), following the pattern of the reference's
`rrule(cic_deposit)` (src/field/sheet_deposit.jl:118-132); `run_states_b200`
checkpoints the state every `checkpoint_every` steps and re-runs each segment once on
the way back. Zygote picks these rules up, so a loss written with them
differentiates through the B200 step.

Force correction: `ForceNetB200` wraps the `djb_nn_*` network and
`attach_nn!(S, net, scales)` adds its correction to every force of a solver.

Load with `include("DiscoDJB200.jl")` after `using DiscoDJNative`; set
`ENV["DJB200_LIB"]` to the library path if it is not next to this file.
"""
module DiscoDJB200

using DiscoDJNative: PMConfig, Cosmology, stepper_coefficients, Fplus
using ChainRulesCore: ChainRulesCore, NoTangent, unthunk

const LIB = get(ENV, "DJB200_LIB", joinpath(@__DIR__, "..", "lib", "libdjb200.so"))

const MEM_HOST = Int32(0)
const MEM_DEVICE = Int32(1)

struct DjbPMConfig            # djb_pm_config, field by field (PMConfig, pm.jl:35-46)
    res_pm::Int32
    n_part::Int32
    boxsize::Float64
    worder::Int32
    deconvolve::Int32
    antialias::Int32
    grad_order::Int32
    lap_order::Int32
    n_resample::Int32
    resampling::Int32
    lean::Int32
    device::Int32
end

function _check(rc::Integer)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:djb_last_error, LIB), Cstring, ()))
    rc == 1 ? throw(ErrorException(msg)) : error("libdjb200 error $rc: $msg")
end

_mem(x::Array) = MEM_HOST
_mem(x) = MEM_DEVICE                       # CuArray and other device arrays
_ptr(x::Array{Float32}) = pointer(x)
_ptr(x) = reinterpret(Ptr{Float32}, UInt(pointer(x)))

"""    PMSolverB200(cfg::PMConfig, like; lean=false, device=0)"""
mutable struct PMSolverB200
    handle::Ptr{Cvoid}
    cfg::PMConfig
    function PMSolverB200(cfg::PMConfig, like=nothing; lean::Bool=false, device::Integer=0)
        c = DjbPMConfig(cfg.res_pm, cfg.n_part, cfg.boxsize, cfg.worder, cfg.deconvolve, cfg.antialias,
                        cfg.grad_order, cfg.lap_order, cfg.n_resample,
                        cfg.resampling == :fourier ? 0 : cfg.resampling == :linear ? 1 :
                            error("resampling must be :fourier or :linear"),
                        lean, device)
        h = Ref{Ptr{Cvoid}}(C_NULL)
        _check(ccall((:djb_solver_create, LIB), Cint, (Ref{DjbPMConfig}, Ref{Ptr{Cvoid}}), c, h))
        s = new(h[], cfg)
        finalizer(x -> ccall((:djb_solver_destroy, LIB), Cint, (Ptr{Cvoid},), x.handle), s)
        return s
    end
end

"""    pm_acceleration!(acc, S::PMSolverB200, psi) -> acc   (pm.jl:507-521)"""
function pm_acceleration!(acc::AbstractArray{Float32,4}, S::PMSolverB200, psi::AbstractArray{Float32,4})
    _mem(acc) == _mem(psi) || error("acc and psi must live in the same memory")
    _check(ccall((:djb_pm_acceleration, LIB), Cint, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int32),
                 S.handle, _ptr(psi), _ptr(acc), _mem(psi)))
    return acc
end
pm_acceleration!(S::PMSolverB200, psi::AbstractArray{Float32,4}) = pm_acceleration!(similar(psi), S, psi)

_stepper_id(s::Symbol) = s === :bullfrog ? 0 : s === :fastpm ? 1 : s === :symplectic ? 2 :
    error("stepper must be :bullfrog, :fastpm or :symplectic")

"""
    run_nbody_b200(c, psi_ini, pi_ini; boxsize, a_ini, a_end, n_steps, res_pm, kwargs...)

`run_nbody` (run_nbody.jl:124-172) with the PM step on the B200: the stepper
coefficients come from DiscoDJNative's own `stepper_coefficients`; the DKD loop,
the force and the output wrap run in libdjb200. Returns (X or Ψ, P, a_end).
"""
function run_nbody_b200(c::Cosmology, psi_ini::AbstractArray{Float32,4}, pi_ini::AbstractArray{Float32,4};
                        boxsize::Real, a_ini::Real, a_end::Real, n_steps::Int, res_pm::Int,
                        time_var=:D, stepper::Symbol=:bullfrog, antialias::Int=0, grad_kernel_order::Int=4,
                        laplace_kernel_order::Int=0, worder::Int=2, deconvolve::Bool=false,
                        n_resample::Int=1, resampling_method::Symbol=:fourier,
                        return_displacement::Bool=false, lean::Bool=false, device::Integer=0)
    n = size(psi_ini, 1)
    co = stepper_coefficients(c, stepper, a_ini, a_end, n_steps; time_var=time_var)
    cfg = PMConfig(res_pm=res_pm, n_part=n, boxsize=Float64(boxsize), worder=worder, deconvolve=deconvolve,
                   antialias=antialias, grad_order=grad_kernel_order, lap_order=laplace_kernel_order,
                   n_resample=n_resample, resampling=resampling_method)
    S = PMSolverB200(cfg; lean=lean, device=device)
    mom_scale = stepper === :symplectic ? Fplus(c, a_ini) : 1.0
    _check(ccall((:djb_set_state, LIB), Cint, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Float64, Int32),
                 S.handle, _ptr(psi_ini), _ptr(pi_ini), mom_scale, _mem(psi_ini)))
    _check(ccall((:djb_run, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
                 S.handle, n_steps, Float64.(co.ddrift1), Float64.(co.alpha), Float64.(co.beta),
                 Float64.(co.ddrift2)))
    X = similar(psi_ini); P = similar(psi_ini)
    F = Fplus(c, a_end)
    pdiv = stepper === :symplectic ? F : 1.0
    _check(ccall((:djb_get_output, LIB), Cint,
                 (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int32, Float64, Float64, Int32),
                 S.handle, _ptr(X), _ptr(P), return_displacement ? 0 : 1, pdiv, F, _mem(X)))
    return X, P, a_end
end

# ── differentiable forms (ChainRulesCore rrules over the library's adjoints) ──────
"""    pm_acceleration_b200(S, psi) -> acc   (pure form of pm_acceleration!, pm.jl:507-521)"""
pm_acceleration_b200(S::PMSolverB200, psi::AbstractArray{Float32,4}) = pm_acceleration!(similar(psi), S, psi)

function ChainRulesCore.rrule(::typeof(pm_acceleration_b200), S::PMSolverB200, psi::AbstractArray{Float32,4})
    acc = pm_acceleration_b200(S, psi)
    function pm_acceleration_pullback(Δ)
        ā = convert(typeof(psi), unthunk(Δ))
        ψ̄ = similar(psi)
        _check(ccall((:djb_pm_acceleration_vjp, LIB), Cint,
                     (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Ptr{Float32}, Int32),
                     S.handle, _ptr(psi), _ptr(ā), _ptr(ψ̄), _mem(psi)))
        return (NoTangent(), NoTangent(), ψ̄)
    end
    return acc, pm_acceleration_pullback
end

"""
    pm_step_b200(S, psi, mom, dd1, alpha, beta, dd2) -> (psi', mom')

One drift-kick-drift step (run_nbody.jl:156-158) on copies of the state.
"""
function pm_step_b200(S::PMSolverB200, psi::AbstractArray{Float32,4}, mom::AbstractArray{Float32,4},
                      dd1::Real, alpha::Real, beta::Real, dd2::Real)
    _check(ccall((:djb_set_state, LIB), Cint, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Float64, Int32),
                 S.handle, _ptr(psi), _ptr(mom), 1.0, _mem(psi)))
    _check(ccall((:djb_step, LIB), Cint, (Ptr{Cvoid}, Float64, Float64, Float64, Float64),
                 S.handle, dd1, alpha, beta, dd2))
    p = similar(psi); m = similar(mom)
    _check(ccall((:djb_get_state, LIB), Cint, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int32),
                 S.handle, _ptr(p), _ptr(m), _mem(p)))
    return p, m
end

# (ψ̄, M̄) of the state before one step from those after it (djb_step_vjp).
function _step_vjp!(S::PMSolverB200, psi0, mom0, ψ̄, M̄, dd1, alpha, beta, dd2)
    _check(ccall((:djb_step_vjp, LIB), Cint,
                 (Ptr{Cvoid}, Float64, Float64, Float64, Float64, Ptr{Float32}, Ptr{Float32}, Ptr{Float32},
                  Ptr{Float32}, Int32),
                 S.handle, dd1, alpha, beta, dd2, _ptr(psi0), _ptr(mom0), _ptr(ψ̄), _ptr(M̄), _mem(psi0)))
    return ψ̄, M̄
end

_tangent_or_zero(Δ, like) = Δ isa ChainRulesCore.AbstractZero ? fill!(similar(like), 0f0) :
                            convert(typeof(like), copy(unthunk(Δ)))

function ChainRulesCore.rrule(::typeof(pm_step_b200), S::PMSolverB200, psi, mom, dd1, alpha, beta, dd2)
    out = pm_step_b200(S, psi, mom, dd1, alpha, beta, dd2)
    function pm_step_pullback(Δ)
        Δp, Δm = unthunk(Δ)
        ψ̄, M̄ = _step_vjp!(S, psi, mom, _tangent_or_zero(Δp, psi), _tangent_or_zero(Δm, mom), dd1, alpha, beta, dd2)
        return (NoTangent(), NoTangent(), ψ̄, M̄, NoTangent(), NoTangent(), NoTangent(), NoTangent())
    end
    return out, pm_step_pullback
end

"""
    run_states_b200(S, psi0, mom0, co; checkpoint_every=5) -> (psi, mom)

The DKD loop of run_nbody.jl:155-163 over the coefficients `co` (a NamedTuple of
`stepper_coefficients`), returning the final state. Its rrule saves the state every
`checkpoint_every` steps and re-runs each segment once while taking its steps back.
"""
function run_states_b200(S::PMSolverB200, psi0::AbstractArray{Float32,4}, mom0::AbstractArray{Float32,4}, co;
                         checkpoint_every::Int=5)
    p, m = psi0, mom0
    for k in eachindex(co.alpha)
        p, m = pm_step_b200(S, p, m, co.ddrift1[k], co.alpha[k], co.beta[k], co.ddrift2[k])
    end
    return p, m
end

function ChainRulesCore.rrule(::typeof(run_states_b200), S::PMSolverB200, psi0, mom0, co; checkpoint_every::Int=5)
    nsteps = length(co.alpha)
    ckpt = Dict(0 => (copy(psi0), copy(mom0)))
    p, m = psi0, mom0
    for k in 1:nsteps
        p, m = pm_step_b200(S, p, m, co.ddrift1[k], co.alpha[k], co.beta[k], co.ddrift2[k])
        k % checkpoint_every == 0 && k < nsteps && (ckpt[k] = (copy(p), copy(m)))
    end
    function run_states_pullback(Δ)
        Δp, Δm = unthunk(Δ)
        ψ̄ = _tangent_or_zero(Δp, psi0); M̄ = _tangent_or_zero(Δm, mom0)
        starts = sort(collect(keys(ckpt)))
        for (i, c0) in Iterators.reverse(enumerate(starts))
            c1 = i < length(starts) ? starts[i + 1] : nsteps
            states = [ckpt[c0]]
            for k in c0 + 1:c1 - 1
                push!(states, pm_step_b200(S, states[end]..., co.ddrift1[k], co.alpha[k], co.beta[k], co.ddrift2[k]))
            end
            for k in c1:-1:c0 + 1
                p_k, m_k = states[k - c0]
                ψ̄, M̄ = _step_vjp!(S, p_k, m_k, ψ̄, M̄, co.ddrift1[k], co.alpha[k], co.beta[k], co.ddrift2[k])
            end
        end
        return (NoTangent(), NoTangent(), ψ̄, M̄, NoTangent())
    end
    return (p, m), run_states_pullback
end

"""    state_power_spectrum_b200(S, psi; bins=32, logarithmic=true) -> P(k) (Vector{Float64})

P(k) of the particles X = q + psi: CIC deposit on the solver's mesh and the float64
shell sums of `evaluate_power_spectrum` (power_spectrum.jl:25-79).
"""
function state_power_spectrum_b200(S::PMSolverB200, psi::AbstractArray{Float32,4}; bins::Int=32,
                                   logarithmic::Bool=true)
    _check(ccall((:djb_set_state, LIB), Cint, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Float64, Int32),
                 S.handle, _ptr(psi), _ptr(psi), 1.0, _mem(psi)))
    k = zeros(Float64, bins); pk = zeros(Float64, bins); nm = zeros(Int64, bins)
    _check(ccall((:djb_state_power_spectrum, LIB), Cint,
                 (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}, Ptr{Float64}, Ptr{Int64}),
                 S.handle, bins, logarithmic, k, pk, nm))
    return pk
end

function ChainRulesCore.rrule(::typeof(state_power_spectrum_b200), S::PMSolverB200, psi; bins::Int=32,
                              logarithmic::Bool=true)
    pk = state_power_spectrum_b200(S, psi; bins=bins, logarithmic=logarithmic)
    function state_power_spectrum_pullback(Δ)
        p̄ = Float64.(collect(unthunk(Δ)))
        ψ̄ = similar(psi)
        _check(ccall((:djb_state_power_spectrum_vjp, LIB), Cint,
                     (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}, Ptr{Float32}, Int32),
                     S.handle, bins, logarithmic, p̄, _ptr(ψ̄), _mem(ψ̄)))
        return (NoTangent(), NoTangent(), ψ̄)
    end
    return pk, state_power_spectrum_pullback
end

# ── force-correction network ──────────────────────────────────────────────────────
"""    ForceNetB200(; layers=4, cin=4, hidden=32, cout=3, seed=0, device=0)"""
mutable struct ForceNetB200
    handle::Ptr{Cvoid}
    function ForceNetB200(; layers::Integer=4, cin::Integer=4, hidden::Integer=32, cout::Integer=3,
                          seed::Integer=0, device::Integer=0)
        h = Ref{Ptr{Cvoid}}(C_NULL)
        _check(ccall((:djb_nn_create, LIB), Cint, (Int32, Int32, Int32, Int32, UInt64, Int32, Ref{Ptr{Cvoid}}),
                     layers, cin, hidden, cout, seed, device, h))
        net = new(h[])
        finalizer(x -> ccall((:djb_nn_destroy, LIB), Cint, (Ptr{Cvoid},), x.handle), net)
        return net
    end
end

"""    load_params!(net, params::Vector{Float32})   (djb_nn_load)"""
load_params!(net::ForceNetB200, params::Vector{Float32}) =
    _check(ccall((:djb_nn_load, LIB), Cint, (Ptr{Cvoid}, Ptr{Float32}), net.handle, params))

"""
    attach_nn!(S, net, (delta_scale, force_scale, out_scale))

Every force of S then adds out_scale·interp(net([delta_scale·δ, force_scale·F])) at the
particles (djb_solver_attach_nn); `attach_nn!(S, nothing)` detaches.
"""
attach_nn!(S::PMSolverB200, net::ForceNetB200, scales) =
    _check(ccall((:djb_solver_attach_nn, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Float64, Float64, Float64),
                 S.handle, net.handle, scales[1], scales[2], scales[3]))
"""    nn_schedule!(S; every=1, start=0)   (djb_solver_nn_schedule)"""
nn_schedule!(S::PMSolverB200; every::Integer=1, start::Integer=0) =
    _check(ccall((:djb_solver_nn_schedule, LIB), Cint, (Ptr{Cvoid}, Int32, Int32), S.handle, every, start))
attach_nn!(S::PMSolverB200, ::Nothing) =
    _check(ccall((:djb_solver_attach_nn, LIB), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Float64, Float64, Float64),
                 S.handle, C_NULL, 1.0, 1.0, 1.0))

"""
    write_snapshot_b200(S, path, D, L; p_div=1.0, p_mul=1.0)

The study driver's snapshot file (scripts/run_jobs.jl:41-48) from the resident state:
HDF5 "Psi", "Pi" = Mom / p_div · p_mul and root attributes "D", "L"
(djb_state_write_snapshot; pass p_div = Fplus(c, a) as runners.jl:155 divides P).
"""
write_snapshot_b200(S::PMSolverB200, path::AbstractString, D::Real, L::Real; p_div::Real=1.0, p_mul::Real=1.0) =
    _check(ccall((:djb_state_write_snapshot, LIB), Cint, (Ptr{Cvoid}, Cstring, Float64, Float64, Float64, Float64),
                 S.handle, path, D, L, p_div, p_mul))

"""
    lpt_ics_b200(white::CuArray{Float32,3}, boxsize, k_tab, p_tab, D; n_order=2, device=0)
        -> (Psi, Pi) as (n,n,n,3) CuArray{Float32}

The GPU path of `nbody_ics_lpt` (src/ics/grf.jl:118-144, src/lpt/nlpt_core.jl:311,
src/nbody/run_nbody.jl:180-208) at n_order 2 or 3: white noise -> phi(k) with P(k) from the
host table (k_tab, p_tab) -> psi_1 .. psi_n_order -> Psi = sum D^m psi_m, Pi = dPsi/dD
(djb_lpt_ics; the work block is allocated by the call).
"""
function lpt_ics_b200(white::AbstractArray{Float32,3}, boxsize::Real, k_tab::Vector{Float64},
                      p_tab::Vector{Float64}, D::Real; n_order::Integer=2, device::Integer=0)
    n = size(white, 1)
    psi = similar(white, n, n, n, 3)
    pi_ = similar(white, n, n, n, 3)
    _check(ccall((:djb_lpt_ics, LIB), Cint,
                 (Ptr{Cvoid}, Int32, Float64, Ptr{Float64}, Ptr{Float64}, Int32, Int32, Float64, Ptr{Cvoid},
                  Ptr{Cvoid}, Ptr{Cvoid}, Int64, Int32, Ptr{Cvoid}),
                 _ptr(white), n, boxsize, k_tab, p_tab, length(k_tab), n_order, D, _ptr(psi), _ptr(pi_),
                 C_NULL, 0, device, C_NULL))
    return psi, pi_
end

end # module
