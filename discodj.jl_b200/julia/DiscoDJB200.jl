"""
    DiscoDJB200

`ccall` bindings of libdjb200.so (include/djb200.h) for DiscoDJNative: a
`PMSolverB200` that implements `pm_acceleration!` on a B200, and `run_nbody_b200`,
the body of `run_nbody` (native/DiscoDJNative/src/nbody/run_nbody.jl:124-172) with
the particle state resident on the GPU. Host arrays (`Array{Float32,4}`) and device
arrays (`CuArray{Float32,4}`, via their pointers) of shape (n,n,n,3) are both
accepted, exactly as laid out by the reference (`pm.jl:15-17`).

Load with `include("DiscoDJB200.jl")` after `using DiscoDJNative`; set
`ENV["DJB200_LIB"]` to the library path if it is not next to this file.
"""
module DiscoDJB200

using DiscoDJNative: PMConfig, Cosmology, stepper_coefficients, Fplus

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

end # module
