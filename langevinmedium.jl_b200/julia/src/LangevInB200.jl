"""
    LangevInB200

B200 backend for LangevInMedium.jl: the per-particle Langevin time loop runs in the
sm_100a CUDA engine `liblangevin_b200.so` (C-ABI in include/langevin_b200.h), reached
through `ccall`.  Loading this module adds methods to the reference's
`simulate_ensemble_bulk` for two new backend markers; the reference stays unmodified:

    using LangevInMedium, LangevInB200
    simulate_ensemble_bulk(B200Backend(), r_grid, p_grid, dens, Tfield, Vfield, (xgrid, tgrid);
                           x_init = x0, p_init = p0, N_particles = N, Δt = 0.01, ...)

The transport tables are still built by the reference's own `Transport` module
(build_tau_drag_spline / build_taun_current_spline / build_juttner_invcdf, with
LV_TAUN_SCALE honoured) and handed to the engine, so a run differs from the
GPUBackend only in the executor.  Additive keywords: `seed`, `precision` (:fp64 |
:fp32), `collision_mode = :langevin_rta` with `eta_over_s`, `device`.
"""
module LangevInB200

using LangevInMedium
const LM = LangevInMedium

export B200Backend, B200_GCBackend

struct B200Backend <: LM.Backends.AbstractBackend end
struct B200_GCBackend <: LM.Backends.AbstractBackend end

# the in-tree library, built by __graft_entry__.build() (langevinmedium.jl_b200/liblangevin_b200.so)
const libpath = Ref{String}(joinpath(@__DIR__, "..", "..", "liblangevin_b200.so"))

# ---- the C-ABI parameter block: 8 Float64 then 16 Int64, as lim_params -------------------
struct LimParams
    dt::Float64; t0::Float64; m::Float64; DsT::Float64; Tfo::Float64; psi2::Float64
    obs_pt_cut::Float64; obs_pt_width::Float64
    dims::Int64; pdim::Int64; coords::Int64; collision::Int64; relativistic::Int64
    bjorken_redshift::Int64; position_diffusion::Int64; reflecting_boundary::Int64
    integrator_mode::Int64; freezeout_capture::Int64; freezeout_interp::Int64
    precision::Int64; seed::Int64; particle_offset::Int64; stop_after_freezeout::Int64
    block_size::Int64
end

const LIM_ERR_NONFINITE = Cint(-4)      # include/langevin_b200.h
const LIM_COLL = Dict(:langevin => 0, :rta => 1, :langevin_rta => 2, :fluid => 3)

mutable struct Ctx
    ptr::Ptr{Cvoid}
end

function check(ctx::Ptr{Cvoid}, rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:lim_last_error, libpath[]), Cstring, (Ptr{Cvoid},), ctx))
    error(msg)                       # the reference's error(...) convention
end

function create(device::Integer = 0)
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:lim_create, libpath[]), Cint, (Cint, Ptr{Cvoid}, Ref{Ptr{Cvoid}}), device, C_NULL, out)
    check(C_NULL, rc)
    c = Ctx(out[])
    finalizer(c -> (c.ptr != C_NULL && ccall((:lim_destroy, libpath[]), Cint, (Ptr{Cvoid},), c.ptr); c.ptr = C_NULL), c)
    return c
end

set_params(c::Ctx, P::LimParams) =
    check(c.ptr, ccall((:lim_set_params, libpath[]), Cint, (Ptr{Cvoid}, Ref{LimParams}), c.ptr, P))

set_medium_rt(c::Ctx, xg, tg, T, V, V2) =
    check(c.ptr, ccall((:lim_set_medium_rt, libpath[]), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}),
        c.ptr, Vector{Float64}(xg), length(xg), Vector{Float64}(tg), length(tg),
        Matrix{Float64}(T), Matrix{Float64}(V), V2 === nothing ? Ptr{Float64}(C_NULL) : Matrix{Float64}(V2)))

set_spline(c::Ctx, which::Integer, Tmin, invdT, vals) =
    check(c.ptr, ccall((:lim_set_spline, libpath[]), Cint, (Ptr{Cvoid}, Cint, Float64, Float64, Ptr{Float64}, Int64),
        c.ptr, which, Tmin, invdT, Vector{Float64}(vals), length(vals)))

set_invcdf(c::Ctx, vals, nU, nT, Tmin, invdT) =
    check(c.ptr, ccall((:lim_set_invcdf, libpath[]), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64, Int64, Float64, Float64),
        c.ptr, Vector{Float64}(vals), nU, nT, Tmin, invdT))

upload_state(c::Ctx, x::Matrix{Float64}, p::Matrix{Float64}) =
    check(c.ptr, ccall((:lim_upload_state, libpath[]), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Int64),
        c.ptr, x, size(x, 1), p, size(p, 1), size(x, 2)))

function download_state!(c::Ctx, x::Matrix{Float64}, p::Matrix{Float64})
    check(c.ptr, ccall((:lim_download_state, libpath[]), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}), c.ptr, x, p))
    return x, p
end

# sample_particles_from_FONLL (utils.jl:33-172) on the device; f is the (Np, Nr) density.
function sample_fonll(c::Ctx, r_grid, p_grid, f, N::Integer; cartesian::Bool, antithetic::Bool, thermal_pz::Bool)
    fm = Matrix{Float64}(size(f) == (length(p_grid), length(r_grid)) ? f : permutedims(f))
    check(c.ptr, ccall((:lim_sample_fonll, libpath[]), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Cint, Cint, Cint),
        c.ptr, Vector{Float64}(r_grid), length(r_grid), Vector{Float64}(p_grid), length(p_grid), fm, N,
        cartesian, antithetic, thermal_pz))
end

initial_lab_boost(c::Ctx) = check(c.ptr, ccall((:lim_initial_lab_boost, libpath[]), Cint, (Ptr{Cvoid},), c.ptr))

run!(c::Ctx, first_step, nsteps, save_every, hx, hp) =
    check(c.ptr, ccall((:lim_run, libpath[]), Cint,
        (Ptr{Cvoid}, Int64, Int64, Int64, Int64, Ptr{Float64}, Ptr{Float64}),
        c.ptr, first_step, nsteps, save_every, 0, hx, hp))

function download_freezeout(c::Ctx, dims, pdim, N)
    pos = zeros(dims, N); mom = zeros(pdim, N); tau = zeros(N); flag = zeros(N)
    check(c.ptr, ccall((:lim_download_freezeout, libpath[]), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), c.ptr, pos, mom, tau, flag))
    return (pos = pos, mom = mom, tau = tau, flag = flag)
end

# ---- simulate_ensemble_bulk(::B200Backend, ...) — mirrors simulate_gpu_wrapper.jl:15-72 ------
function LM.Simulate.simulate_ensemble_bulk(
    backend::B200Backend, r_grid_Langevin, p_grid_Langevin, heavy_quark_density,
    TemperatureEvolutionn, VelocityEvolutionn, SpaceTimeGrid;
    N_particles::Int = 10_000, Δt::Float64 = 0.001, initial_time::Float64 = 0.0, final_time::Float64 = 1.0,
    save_interval::Float64 = 0.1, m::Float64 = 1.0, DsT::Float64 = 0.2, DsT_linear::Bool = false,
    DsT_slope::Float64 = 1.765, DsT_offset::Float64 = -0.159, Tfo::Float64 = 0.156, DsT_quad::Bool = false,
    DsT_Tref::Float64 = 0.0, dimensions::Int = 3, cartesian_spatial_sampling = nothing,
    antithetic_momenta::Bool = false, position_diffusion::Bool = false, momentum_langevin::Bool = true,
    reflecting_boundary::Bool = false, collision_mode::Symbol = :langevin,
    x_init::Union{Nothing, AbstractMatrix} = nothing, p_init::Union{Nothing, AbstractMatrix} = nothing,
    V2Evolutionn::Union{Nothing, AbstractMatrix} = nothing, psi2::Float64 = 0.0,
    freezeout_capture::Bool = false, freezeout_interp::Bool = true, integrator_mode::Int = 0,
    relativistic::Bool = true, momentum_dimensions::Int = 0, bjorken_redshift::Bool = false,
    seed::Integer = 0x4C494D00, precision::Symbol = :fp64, eta_over_s::Float64 = 0.16, device::Integer = 0)

    collision_mode in (:langevin, :rta, :langevin_rta) ||
        error("simulate_ensemble_bulk(::B200Backend): collision_mode=$(collision_mode) is not supported (only :langevin, :rta and :langevin_rta).")
    steps = floor(Int, (final_time - initial_time) / Δt)
    save_every = round(Int, save_interval / Δt)
    num_saves = div(steps, save_every)
    if freezeout_capture
        num_saves = 1
        save_every = max(steps, 1)
    end
    xgrid, tgrid = SpaceTimeGrid
    pdim = momentum_dimensions <= 0 ? dimensions : momentum_dimensions
    device_sampling = x_init === nothing || p_init === nothing
    if device_sampling
        # the FONLL sampler on the device (dimensions 2); other dimensions bring x_init/p_init
        dimensions == 2 ||
            error("B200Backend samples the FONLL initial state on the device for dimensions=2; pass x_init/p_init")
        LM.Utils.check_momentum_dims(dimensions, pdim, false, bjorken_redshift, initial_time)
        N = N_particles
    else
        positions = Matrix{Float64}(x_init); momenta = Matrix{Float64}(p_init)
        radial_mode = dimensions == 1
        LM.Utils.check_momentum_dims(dimensions, pdim, radial_mode, bjorken_redshift, initial_time)
        if size(momenta, 1) < pdim
            momenta = LM.Utils.append_thermal_pz(momenta, positions, m,
                r -> LM.KernelsCPU.interpolate_2d_cpu(xgrid, tgrid, TemperatureEvolutionn, r, initial_time))
        end
        size(momenta, 1) == pdim || error("momentum rows $(size(momenta, 1)) ≠ momentum_dimensions $pdim")
        N = size(positions, 2)
    end

    coll = (!momentum_langevin || DsT == 0.0) ? :fluid : collision_mode
    c = create(device)
    set_params(c, LimParams(Δt, initial_time, m, DsT, Tfo, psi2, 5.0, 0.1, dimensions, pdim, 0, LIM_COLL[coll],
        relativistic, bjorken_redshift, position_diffusion, reflecting_boundary, integrator_mode,
        freezeout_capture, freezeout_interp, precision == :fp32 ? 1 : 0, Int64(seed), 0,
        freezeout_capture ? 1 : 0, 0))
    set_medium_rt(c, xgrid, tgrid, TemperatureEvolutionn, VelocityEvolutionn, V2Evolutionn)
    if momentum_langevin && DsT > 0.0                       # simulate_gpu.jl:96-138
        Tmin = max(float(minimum(TemperatureEvolutionn)), 0.0)
        Tmax = max(float(maximum(TemperatureEvolutionn)), Tmin + eps(Float64))
        kw = (Tmin = Tmin, Tmax = Tmax, nT = 1024, DsT_linear = DsT_linear, DsT_slope = DsT_slope,
              DsT_offset = DsT_offset, Tfo = Tfo, DsT_quad = DsT_quad, DsT_Tref = DsT_Tref)
        t0_, invdT, dvals = LM.Transport.build_tau_drag_spline(m, DsT; kw...)
        set_spline(c, 0, t0_, invdT, dvals)
        if collision_mode == :rta
            _, _, nvals = LM.Transport.build_taun_current_spline(m, DsT; kw...)
            set_spline(c, 1, t0_, invdT, nvals)
        elseif collision_mode == :langevin_rta
            rvals = [5.0 * eta_over_s / (t0_ + (k - 1) / invdT) / LM.fmGeV for k in 1:length(dvals)]
            set_spline(c, 1, t0_, invdT, rvals)
        end
        if collision_mode != :langevin
            inv, nU, nT, Tm, Ti = LM.Transport.build_juttner_invcdf(m, pdim; Tmin = Tmin, Tmax = Tmax)
            set_invcdf(c, inv, nU, nT, Tm, Ti)
        end
    end
    if device_sampling
        sample_fonll(c, r_grid_Langevin, p_grid_Langevin, heavy_quark_density, N;
            cartesian = cartesian_spatial_sampling === nothing ? true : cartesian_spatial_sampling,
            antithetic = antithetic_momenta, thermal_pz = pdim == 3)
    else
        upload_state(c, positions, momenta)
    end
    initial_lab_boost(c)
    if freezeout_capture
        run!(c, 1, steps, 0, C_NULL, C_NULL)
        return download_freezeout(c, dimensions, pdim, N)
    end
    hx = zeros(dimensions, N, num_saves + 1)
    hp = zeros(pdim, N, num_saves + 1)
    x0 = zeros(dimensions, N); p0 = zeros(pdim, N)
    download_state!(c, x0, p0)
    hx[:, :, 1] .= x0; hp[:, :, 1] .= p0
    run!(c, 1, steps, save_every, hx, hp)
    time_points = range(initial_time, final_time, length = num_saves + 1)
    return time_points, [hp[:, :, i] for i in 1:num_saves+1], [hx[:, :, i] for i in 1:num_saves+1]
end

# ---- simulate_ensemble_bulk(::B200Backend, T::Float64; ...) — mirrors simulate.jl:89-109 ----------
# The static-temperature momentum-only path (simulate_cpu.jl:325-404, legacy force
# kernels_cpu.jl:359-404) on the device; the initial momenta come from the reference's
# own sample_initial_particles_at_origin_no_position! (utils.jl:419-465), the |p|
# history starts with their magnitudes.
function LM.Simulate.simulate_ensemble_bulk(
    backend::B200Backend, T::Float64;
    N_particles::Int = 10_000, Δt::Float64 = 0.001, initial_time::Float64 = 0.0, final_time::Float64 = 1.0,
    save_interval::Float64 = 0.1, m::Float64 = 1.0, p0 = 1.0, DsT = 0.2, initial_condition = "delta",
    dimensions::Int = 3, seed::Integer = 0x4C494D00, precision::Symbol = :fp64, device::Integer = 0)

    steps = floor(Int, (final_time - initial_time) / Δt)
    save_every = round(Int, save_interval / Δt)
    num_saves = div(steps, save_every)
    momenta = LM.Utils.sample_initial_particles_at_origin_no_position!(initial_condition, p0, dimensions, N_particles)
    N = size(momenta, 2)
    c = create(device)
    set_params(c, LimParams(Δt, initial_time, m, Float64(DsT), 0.0, 0.0, 5.0, 0.1, dimensions, dimensions, 0,
        LIM_COLL[:langevin], 1, 0, 0, 0, 0, 0, 1, precision == :fp32 ? 1 : 0, Int64(seed), 0, 0, 0))
    check(c.ptr, ccall((:lim_upload_state, libpath[]), Cint, (Ptr{Cvoid}, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Int64),
        c.ptr, zeros(dimensions, N), dimensions, Matrix{Float64}(momenta), dimensions, N))
    hist = zeros(N, num_saves + 1)                  # column k: the |p| snapshot of slot k-1
    hist[:, 1] .= vec(sqrt.(sum(momenta .^ 2, dims = 1)))
    check(c.ptr, ccall((:lim_run_static_T, libpath[]), Cint,
        (Ptr{Cvoid}, Float64, Int64, Int64, Int64, Int64, Int64, Ptr{Float64}),
        c.ptr, T, 1, steps, save_every, 0, num_saves + 1, hist))
    time_points = range(initial_time, final_time, length = num_saves + 1)
    return time_points, [hist[:, k] for k in 1:num_saves+1]
end

# ---- simulate_ensemble_bulk(::B200_GCBackend, ...) — mirrors simulate.jl:117-141 ----------------
# sample_initial_particles_milne! (utils.jl:350-400) runs on the device: the profiles are
# evaluated at the 200 bin centers of (0, maximum(xgrid)), and T(r) for the momentum
# width on a 1601-node table.
function sample_milne(c::Ctx, x_lo, x_hi, Tc, urc, muc, rT, TT, N::Integer)
    check(c.ptr, ccall((:lim_sample_milne, libpath[]), Cint,
        (Ptr{Cvoid}, Float64, Float64, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
         Int64, Int64),
        c.ptr, x_lo, x_hi, length(Tc), Tc, urc, muc, rT, TT, length(rT), N))
end

function LM.Simulate.simulate_ensemble_bulk(
    backend::B200_GCBackend, T_profile_MIS, ur_profile_MIS, mu_profile_MIS,
    TemperatureEvolutionn, VelocityEvolutionn, SpaceTimeGrid;
    N_particles::Int = 10_000, Δt::Float64 = 0.001, initial_time::Float64 = 0.0, final_time::Float64 = 1.0,
    save_interval::Float64 = 0.1, m::Float64 = 1.0, DsT::Float64 = 0.2, dimensions::Int = 2,
    seed::Integer = 0x4C494D00, precision::Symbol = :fp64, device::Integer = 0)

    @assert dimensions == 2 "Milne sampling requires dim = 2 (τ, r)"
    steps = floor(Int, (final_time - initial_time) / Δt)
    save_every = Int(save_interval / Δt)
    num_saves = div(steps, save_every)
    xgrid, tgrid = SpaceTimeGrid
    c = create(device)
    set_params(c, LimParams(Δt, initial_time, m, DsT, 0.0, 0.0, 5.0, 0.1, 2, 2, 1, LIM_COLL[:langevin],
        1, 0, 0, 0, 0, 0, 1, precision == :fp32 ? 1 : 0, Int64(seed), 0, 0, 0))
    set_medium_rt(c, xgrid, tgrid, TemperatureEvolutionn, VelocityEvolutionn, nothing)
    if DsT > 0.0                                           # simulate_cpu_general_coords.jl:72-80
        Tmin = max(float(minimum(TemperatureEvolutionn)), 0.0)
        Tmax = max(float(maximum(TemperatureEvolutionn)), Tmin + eps(Float64))
        t0_, invdT, dvals = LM.Transport.build_tau_drag_spline(m, DsT; Tmin = Tmin, Tmax = Tmax, nT = 1024)
        set_spline(c, 0, t0_, invdT, dvals)
    end
    x_hi = float(maximum(xgrid))
    edges = range(0.0, x_hi, length = 201)
    centers = (edges[1:end-1] .+ edges[2:end]) ./ 2
    rT = collect(range(0.0, x_hi, length = 1601))
    sample_milne(c, 0.0, x_hi, Float64.(T_profile_MIS.(centers, initial_time)),
        Float64.(ur_profile_MIS.(centers, initial_time)), Float64.(mu_profile_MIS.(centers, initial_time)),
        rT, Float64.(T_profile_MIS.(rT, initial_time)), N_particles)
    N = N_particles
    hx = zeros(2, N, num_saves + 1)
    hp = zeros(2, N, num_saves + 1)
    x0 = zeros(2, N); p0 = zeros(2, N)
    download_state!(c, x0, p0)
    hx[:, :, 1] .= x0; hp[:, :, 1] .= p0
    rc = ccall((:lim_run, libpath[]), Cint, (Ptr{Cvoid}, Int64, Int64, Int64, Int64, Ptr{Float64}, Ptr{Float64}),
        c.ptr, 1, steps, save_every, 0, hx, hp)
    rc == 0 || rc == LIM_ERR_NONFINITE || check(c.ptr, rc)   # the Milne CPU driver has no NaN/Inf check
    time_points = range(initial_time, final_time, length = num_saves + 1)
    # simulate_cpu_general_coords.jl:53-55, :120-124: |p^r| first, then |p| over (p^τ, p^r); the r row
    momenta_history = [i == 1 ? abs.(hp[2, :, 1]) : vec(sqrt.(sum(hp[:, :, i] .^ 2, dims = 1))) for i in 1:num_saves+1]
    position_history = [reshape(hx[2, :, i], 1, N) for i in 1:num_saves+1]
    return time_points, momenta_history, position_history
end

end # module
