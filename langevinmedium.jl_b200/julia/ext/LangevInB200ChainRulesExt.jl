"""
    LangevInB200ChainRulesExt

ChainRulesCore rule for the engine's pathwise gradients: `heavy_quark_observables(θ, run)`
returns (⟨pT⟩, ⟨cos 2φ⟩, smoothed fraction above the cut) of a configured run at
θ = (a, b, s) — 2πT·D_s = a + b(max(T, Tc)/Tc − 1) and the medium temperature scale s —
and its `rrule` runs the engine's checkpointed forward and hand-written reverse sweep
(`lim_adjoint`) once, the pullback contracting the cotangent with the 3×3 Jacobian.
The noise and the RTA indicators of the forward pass are held fixed. A package
extension of LangevInB200 (Project.toml), loaded with ChainRulesCore (which Zygote,
Diffractor and the like use).
"""
module LangevInB200ChainRulesExt

using ChainRulesCore
using LangevInMedium
using LangevInB200: Ctx, check, libpath, set_spline
const LM = LangevInMedium

"""A configured context (parameters, medium, RTA spline, inverse CDF, initial state
already boosted to the lab) and the step range of the gradient run; the initial state
is saved on the device when the run is made."""
struct AdjointRun
    ctx::Ctx
    m::Float64
    Tmin::Float64
    Tmax::Float64
    first_step::Int
    nsteps::Int
    checkpoint_every::Int
    Tc::Float64
    function AdjointRun(ctx, m, Tmin, Tmax, first_step, nsteps; checkpoint_every = 64, Tc = 0.155)
        check(ctx.ptr, ccall((:lim_state_save, libpath[]), Cint, (Ptr{Cvoid},), ctx.ptr))
        new(ctx, m, Tmin, Tmax, first_step, nsteps, checkpoint_every, Tc)
    end
end

# the drag spline of (a, b) and its derivative tables, as transport.jl:165-196 builds the
# drag spline with DsT_linear (slope b/(2π Tc), offset (a − b)/(2π), Tfo = Tc)
function drag_tables(run::AdjointRun, a, b; nT = 1024)
    kw = (Tmin = run.Tmin, Tmax = run.Tmax, nT = nT, DsT_linear = true, DsT_slope = b / (2π * run.Tc),
          DsT_offset = (a - b) / (2π), Tfo = run.Tc)
    t0, invdT, vals = LM.Transport.build_tau_drag_spline(run.m, 1.0; kw...)
    T = [t0 + (k - 1) / invdT for k in 1:length(vals)]
    base = run.m ./ (T .^ 2) ./ LM.fmGeV ./ (2π) .* LM.Transport.LV_TAUN_SCALE[]   # d tau_drag / d(2πT D_s)
    return t0, invdT, vals, base, base .* (max.(T, run.Tc) ./ run.Tc .- 1.0)
end

function run_adjoint(θ::AbstractVector, run::AdjointRun)
    a, b, s = Float64.(θ)
    t0, invdT, vals, dda, ddb = drag_tables(run, a, b)
    set_spline(run.ctx, 0, t0, invdT, vals)
    set_spline(run.ctx, 2, t0, invdT, dda)                 # LIM_SPLINE_DRAG_DA
    set_spline(run.ctx, 3, t0, invdT, ddb)                 # LIM_SPLINE_DRAG_DB
    check(run.ctx.ptr, ccall((:lim_set_medium_scale, libpath[]), Cint, (Ptr{Cvoid}, Float64), run.ctx.ptr, s))
    check(run.ctx.ptr, ccall((:lim_state_restore, libpath[]), Cint, (Ptr{Cvoid},), run.ctx.ptr))
    obs = zeros(3); grad = zeros(9)
    check(run.ctx.ptr, ccall((:lim_adjoint, libpath[]), Cint,
        (Ptr{Cvoid}, Int64, Int64, Int64, Ptr{Float64}, Ptr{Float64}),
        run.ctx.ptr, run.first_step, run.nsteps, run.checkpoint_every, obs, grad))
    return obs, permutedims(reshape(grad, 3, 3))            # J[o, k] = grad[3(o-1) + k]
end

"""(⟨pT⟩, ⟨cos 2φ⟩, smoothed fraction above the cut) at θ = (a, b, s)."""
heavy_quark_observables(θ::AbstractVector, run::AdjointRun) = run_adjoint(θ, run)[1]

function ChainRulesCore.rrule(::typeof(heavy_quark_observables), θ::AbstractVector, run::AdjointRun)
    obs, J = run_adjoint(θ, run)
    pullback(ȳ) = (NoTangent(), J' * unthunk(ȳ), NoTangent())
    return obs, pullback
end

export AdjointRun, heavy_quark_observables

end # module
