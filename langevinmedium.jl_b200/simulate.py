"""``simulate_ensemble_bulk`` for the B200 engine — the drop-in for the reference's
CPU and GPU paths.

Mirrors ``Simulate.simulate_ensemble_bulk`` (src/simulate.jl:21-141) and its GPU
twin (src/simulate_gpu_wrapper.jl:15-108, src/simulate_gpu.jl:26-462): the same
positional arguments, keyword arguments (``Δt`` included), defaults, error
messages and return values, dispatched on the backend marker exactly as the
reference dispatches on ``CPUBackend``/``GPUBackend``.  The time loop runs in the
CUDA engine; this module only prepares tables and copies state in and out.

Additive keywords (not in the reference): ``seed`` (Philox key), ``precision``
("fp64" | "fp32"), ``collision_mode=:langevin_rta`` with ``tau_R`` / ``eta_over_s``
(the combined OU + RTA step), ``device``, ``stream``, ``block_size``.
"""
from __future__ import annotations

import math
import threading
from dataclasses import dataclass

import numpy as np

from . import capi
from . import transport as tr
from .backends import B200Backend, B200_GCBackend
from .utils import append_thermal_pz, check_momentum_dims, radial_reduction

DEFAULT_SEED = 0x4C494D00
_local = threading.local()


def _engine(device: int, stream) -> capi.Engine:
    """One engine context per (thread, device, stream), reused across calls."""
    cache = getattr(_local, "engines", None)
    if cache is None:
        cache = _local.engines = {}
    key = (int(device), int(stream or 0))
    eng = cache.get(key)
    if eng is None:
        eng = cache[key] = capi.Engine(device=device, stream=stream)
    return eng


def _sym(x) -> str:
    s = str(x)
    return s[1:] if s.startswith(":") else s


@dataclass
class FreezeOut:
    """The freeze-out NamedTuple of simulate_gpu.jl:396: (pos, mom, tau, flag)."""
    pos: np.ndarray
    mom: np.ndarray
    tau: np.ndarray
    flag: np.ndarray

    def __iter__(self):
        return iter((self.pos, self.mom, self.tau, self.flag))


def _time_points(t0: float, tf: float, n: int) -> np.ndarray:
    return np.linspace(t0, tf, n)


def simulate_ensemble_bulk(backend, *args, **kwargs):
    """Dispatch on the backend marker and the first positional argument (simulate.jl:21,
    :89, :117; simulate_gpu_wrapper.jl:15, :74): a real temperature selects the
    static-temperature momentum-only path."""
    if isinstance(backend, B200Backend):
        if len(args) == 1 and isinstance(args[0], (int, float, np.floating, np.integer)):
            return _simulate_static_T(float(args[0]), **kwargs)
        return _simulate_cartesian(*args, **kwargs)
    if isinstance(backend, B200_GCBackend):
        return _simulate_milne(*args, **kwargs)
    raise TypeError(f"simulate_ensemble_bulk: no method for backend {type(backend).__name__} "
                    "(use B200Backend() or B200_GCBackend())")


def _simulate_static_T(T: float, *, N_particles: int = 10_000, Δt: float = 0.001, initial_time: float = 0.0,
                       final_time: float = 1.0, save_interval: float = 0.1, m: float = 1.0, p0=1.0, DsT=0.2,
                       initial_condition="delta", dimensions: int = 3,
                       # additive
                       seed: int = DEFAULT_SEED, precision: str = "fp64", device: int = 0, stream=None,
                       block_size: int = 0):
    """simulate_ensemble_bulk(::CPUBackend, T::Float64; ...) (simulate.jl:89-109 ->
    simulate_cpu.jl:325-404): momentum-only Langevin at a fixed temperature with the
    legacy force kappa = 2.5 T^3 (kernels_cpu.jl:359-404).  Returns (time_points,
    momenta_history) with one |p| vector per saved step (the initial one first).  DsT
    is accepted and, as in the reference, not used."""
    total_time = final_time - initial_time
    steps = int(math.floor(total_time / Δt))
    save_every = int(round(save_interval / Δt))
    if save_every == 0:
        raise ZeroDivisionError("save_interval/Δt rounds to 0 (DivideError in the reference)")
    num_saves = steps // save_every
    rng = np.random.default_rng(int(seed) & 0xFFFFFFFFFFFFFFFF)
    from .utils import sample_initial_particles_at_origin_no_position
    momenta = sample_initial_particles_at_origin_no_position(initial_condition, p0, dimensions, N_particles, rng)
    N = momenta.shape[1]
    hist = np.zeros((num_saves + 1, N))
    hist[0] = np.sqrt(np.sum(momenta ** 2, axis=0))
    eng = _engine(device, stream)
    eng.set_params(dt=Δt, t0=initial_time, m=m, DsT=float(DsT), dims=int(dimensions), pdim=int(dimensions),
                   precision=capi.LIM_FP32 if precision == "fp32" else capi.LIM_FP64, seed=int(seed),
                   block_size=block_size)
    eng.upload_state(np.zeros((int(dimensions), N)), momenta)
    eng.run_static_T(T, 1, steps, save_every, 0, hist)
    time_points = _time_points(initial_time, final_time, num_saves + 1)
    return time_points, [hist[k].copy() for k in range(num_saves + 1)]


def _simulate_cartesian(r_grid_Langevin, p_grid_Langevin, heavy_quark_density,
                        TemperatureEvolutionn, VelocityEvolutionn, SpaceTimeGrid, *,
                        N_particles: int = 10_000, Δt: float = 0.001, initial_time: float = 0.0,
                        final_time: float = 1.0, save_interval: float = 0.1, m: float = 1.0,
                        DsT: float = 0.2, DsT_linear: bool = False, DsT_slope: float = 1.765,
                        DsT_offset: float = -0.159, Tfo: float = 0.156, DsT_quad: bool = False,
                        DsT_Tref: float = 0.0, dimensions: int = 3, cartesian_spatial_sampling=None,
                        antithetic_momenta: bool = False, position_diffusion: bool = False,
                        momentum_langevin: bool = True, reflecting_boundary: bool = False,
                        collision_mode=":langevin", x_init=None, p_init=None, V2Evolutionn=None,
                        psi2: float = 0.0, freezeout_capture: bool = False, freezeout_interp: bool = True,
                        integrator_mode: int = 0, relativistic: bool = True, momentum_dimensions: int = 0,
                        bjorken_redshift: bool = False,
                        # additive
                        seed: int = DEFAULT_SEED, precision: str = "fp64", eta_over_s: float = 0.16,
                        tau_R_factor: float = 5.0, device: int = 0, stream=None, block_size: int = 0,
                        stop_after_freezeout: bool = True, snapshot_reduce=None, tables: str = "host",
                        pinned_history: bool = False):
    mode = _sym(collision_mode)
    if mode not in ("langevin", "rta", "langevin_rta"):
        raise ValueError(f"simulate_ensemble_bulk(::B200Backend): collision_mode=:{mode} is not supported "
                         "(only :langevin, :rta and :langevin_rta).")
    if integrator_mode not in (0, 1):
        raise ValueError("integrator_mode must be 0 (pre-point exact OU) or 1 (drift-midpoint)")
    # --- derived parameters (simulate_gpu.jl:65-75) ---
    total_time = final_time - initial_time
    steps = int(math.floor(total_time / Δt))
    save_every = int(round(save_interval / Δt))
    if save_every == 0:
        raise ZeroDivisionError("save_interval/Δt rounds to 0 (DivideError in the reference)")
    num_saves = steps // save_every
    if freezeout_capture:
        num_saves = 1
        save_every = max(steps, 1)
    xgrid, tgrid = SpaceTimeGrid
    xgrid = np.asarray(xgrid, dtype=np.float64)
    tgrid = np.asarray(tgrid, dtype=np.float64)
    Tfield = np.asarray(TemperatureEvolutionn, dtype=np.float64)
    Vfield = np.asarray(VelocityEvolutionn, dtype=np.float64)
    rng = np.random.default_rng(int(seed) & 0xFFFFFFFFFFFFFFFF)
    # --- initial state (simulate_cpu.jl:63-94) ---
    pdim = dimensions if momentum_dimensions <= 0 else momentum_dimensions
    device_sampling = x_init is None or p_init is None
    if device_sampling:
        # sample_particles_from_FONLL (utils.jl:33-172) on the device, with the thermal p_z
        # of append_thermal_pz (utils.jl:533-551) from the medium at initial_time
        if dimensions != 2:
            raise NotImplementedError("the B200 backend samples the FONLL initial state on the device for "
                                      "dimensions=2; for dimensions 1 and 3 pass x_init/p_init")
        check_momentum_dims(dimensions, pdim, False, bjorken_redshift, initial_time)
        do_cartesian = True if cartesian_spatial_sampling is None else bool(cartesian_spatial_sampling)
        N = int(N_particles)
    else:
        x_matrix = np.array(x_init, dtype=np.float64, ndmin=2)
        p_matrix = np.array(p_init, dtype=np.float64, ndmin=2)
        radial_mode = dimensions == 1
        if radial_mode:
            if x_matrix.shape[0] >= 2:
                positions, momenta = radial_reduction(x_matrix[:2], p_matrix[:2], r_grid_Langevin, rng)
            else:
                positions, momenta = x_matrix, p_matrix
        else:
            positions, momenta = x_matrix.copy(), p_matrix.copy()
        check_momentum_dims(dimensions, pdim, radial_mode, bjorken_redshift, initial_time)
    if not device_sampling and momenta.shape[0] < pdim:
        from .utils import _rt_interp_host
        momenta = append_thermal_pz(momenta, positions, m,
                                    lambda r: _rt_interp_host(xgrid, tgrid, Tfield, r, initial_time),
                                    antithetic=antithetic_momenta and x_init is None, rng=rng)
    if not device_sampling:
        if momenta.shape[0] != pdim:
            raise ValueError(f"momentum rows {momenta.shape[0]} ≠ momentum_dimensions {pdim}")
        if positions.shape[0] != dimensions:
            raise ValueError(f"position rows {positions.shape[0]} ≠ dimensions {dimensions}")
        N = positions.shape[1]
        if momenta.shape[1] != N:
            raise ValueError("x_init and p_init hold different particle counts")

    # --- engine configuration ---
    if not momentum_langevin or DsT == 0.0:
        coll = capi.LIM_COLL_FLUID
    elif mode == "rta":
        coll = capi.LIM_COLL_RTA
    elif mode == "langevin_rta":
        coll = capi.LIM_COLL_LANGEVIN_RTA
    else:
        coll = capi.LIM_COLL_LANGEVIN
    eng = _engine(device, stream)
    eng.set_params(dt=Δt, t0=initial_time, m=m, DsT=DsT, Tfo=Tfo, psi2=psi2, dims=dimensions, pdim=pdim,
                   coords=capi.LIM_COORDS_CARTESIAN, collision=coll, relativistic=int(bool(relativistic)),
                   bjorken_redshift=int(bool(bjorken_redshift)), position_diffusion=int(bool(position_diffusion)),
                   reflecting_boundary=int(bool(reflecting_boundary)), integrator_mode=integrator_mode,
                   freezeout_capture=int(bool(freezeout_capture)), freezeout_interp=int(bool(freezeout_interp)),
                   precision=capi.LIM_FP32 if precision == "fp32" else capi.LIM_FP64, seed=seed,
                   stop_after_freezeout=int(bool(stop_after_freezeout and freezeout_capture)), block_size=block_size)
    eng.set_medium_rt(xgrid, tgrid, Tfield, Vfield, V2Evolutionn)
    # --- transport tables (simulate_gpu.jl:90-138) ---
    if tables not in ("host", "device"):
        raise ValueError('tables must be "host" (transport.py, as the reference) or "device"')
    if momentum_langevin and DsT > 0.0 and tables == "device":
        Tmin, Tmax = tr.spline_range(Tfield)
        dkw = dict(Tmin=Tmin, Tmax=Tmax, nT=1024, DsT_linear=DsT_linear, DsT_slope=DsT_slope,
                   DsT_offset=DsT_offset, Tfo=Tfo, DsT_quad=DsT_quad, DsT_Tref=DsT_Tref)
        eng.build_time_spline(capi.LIM_SPLINE_DRAG, capi.LIM_TIME_DRAG, m, DsT, **dkw)
        if mode == "rta":
            eng.build_time_spline(capi.LIM_SPLINE_RTA, capi.LIM_TIME_TAUN, m, DsT, **dkw)
        elif mode == "langevin_rta":
            eng.build_time_spline(capi.LIM_SPLINE_RTA, capi.LIM_TIME_TAUR, m, DsT, eta_over_s=eta_over_s,
                                  factor=tau_R_factor, **dkw)
        if mode in ("rta", "langevin_rta"):
            eng.build_juttner_invcdf(m, pdim, Tmin=Tmin, Tmax=Tmax, nT=256, nU=2048, np_=8192)
    elif momentum_langevin and DsT > 0.0:
        Tmin, Tmax = tr.spline_range(Tfield)
        dkw = dict(Tmin=Tmin, Tmax=Tmax, nT=1024, DsT_linear=DsT_linear, DsT_slope=DsT_slope,
                   DsT_offset=DsT_offset, Tfo=Tfo, DsT_quad=DsT_quad, DsT_Tref=DsT_Tref)
        t0_, inv_, vals = tr.build_tau_drag_spline(m, DsT, **dkw)
        eng.set_spline(capi.LIM_SPLINE_DRAG, t0_, inv_, vals)
        if mode == "rta":
            _, _, nvals = tr.build_taun_current_spline(m, DsT, **dkw)
            eng.set_spline(capi.LIM_SPLINE_RTA, t0_, inv_, nvals)
        elif mode == "langevin_rta":
            _, _, rvals = tr.build_tau_R_spline(m, DsT, eta_over_s=eta_over_s, factor=tau_R_factor, **dkw)
            eng.set_spline(capi.LIM_SPLINE_RTA, t0_, inv_, rvals)
        if mode in ("rta", "langevin_rta"):
            inv, nU, nT, Ttmin, Tinv = tr.build_juttner_invcdf(m, pdim, Tmin=Tmin, Tmax=Tmax, nT=256, nU=2048, np_=8192)
            eng.set_invcdf(inv, nU, nT, Ttmin, Tinv)
    elif mode in ("rta", "langevin_rta"):
        eng.set_invcdf(np.zeros(4), 2, 2, 0.0, 1.0)   # reference default table (simulate_gpu.jl:124-128)
    if device_sampling:
        eng.sample_fonll(r_grid_Langevin, p_grid_Langevin, heavy_quark_density, N, cartesian=do_cartesian,
                         antithetic=antithetic_momenta, thermal_pz=pdim == 3)
    else:
        eng.upload_state(positions, momenta)
    eng.initial_lab_boost()

    if freezeout_capture:
        eng.run(1, steps)
        fo = eng.download_freezeout()
        return FreezeOut(fo["pos"], fo["mom"], fo["tau"], fo["flag"])

    nslots = num_saves + 1
    if snapshot_reduce is not None:
        # additive: every snapshot reduced on the device (observable sums, n(r), p_T
        # spectrum, cos 2 phi per p_T bin) instead of the FP64 history
        spec = capi.reduce_spec(*snapshot_reduce)
        first = eng.reduce_state(spec)
        rest = eng.run_reduced(1, steps, save_every, 1, nslots - 1, spec) if nslots > 1 else None
        red = {k: (np.vstack([first[k][None, :], rest[k]]) if rest is not None else first[k][None, :])
               for k in first}
        return _time_points(initial_time, final_time, nslots), red
    # additive: pinned_history puts the history in page-locked memory (faster copies,
    # slower to allocate)
    alloc = capi.pinned_empty if pinned_history else np.empty
    hx = alloc(nslots * N * dimensions)
    hp = alloc(nslots * N * pdim)
    eng.download_state_flat(hx[: N * dimensions], hp[: N * pdim])
    eng.run(1, steps, save_every, 0, hx, hp)
    time_points = _time_points(initial_time, final_time, nslots)
    mom = [hp[k * N * pdim:(k + 1) * N * pdim].reshape(N, pdim).T for k in range(nslots)]
    pos = [hx[k * N * dimensions:(k + 1) * N * dimensions].reshape(N, dimensions).T for k in range(nslots)]
    return time_points, mom, pos


MILNE_BINS = 200          # the reference's radial bins (simulate_cpu_general_coords.jl:41)
MILNE_T_TABLE = 1601      # nodes of the T(r) table that sets the initial momentum width


def _simulate_milne(T_profile_MIS, ur_profile_MIS, mu_profile_MIS, TemperatureEvolutionn, VelocityEvolutionn,
                    SpaceTimeGrid, *, N_particles: int = 10_000, Δt: float = 0.001, initial_time: float = 0.0,
                    final_time: float = 1.0, save_interval: float = 0.1, m: float = 1.0, DsT: float = 0.2,
                    dimensions: int = 2, x_init=None, p_init=None, seed: int = DEFAULT_SEED,
                    precision: str = "fp64", device: int = 0, stream=None, block_size: int = 0):
    """Milne (tau, r) driver (simulate_cpu_general_coords.jl:18-133)."""
    if dimensions != 2:
        raise ValueError("Milne coordinates evolve (τ, r): dimensions must be 2")
    total_time = final_time - initial_time
    steps = int(math.floor(total_time / Δt))
    q = save_interval / Δt
    if q != math.floor(q):
        raise ValueError(f"InexactError: Int64({q})")          # Int(save_interval/Δt)
    save_every = int(q)
    num_saves = steps // save_every
    xgrid, tgrid = SpaceTimeGrid
    Tfield = np.asarray(TemperatureEvolutionn, dtype=np.float64)
    device_sampling = x_init is None or p_init is None
    if device_sampling:
        N = int(N_particles)
    else:
        positions = np.array(x_init, dtype=np.float64, ndmin=2)
        momenta = np.array(p_init, dtype=np.float64, ndmin=2)
        N = positions.shape[1]
    eng = _engine(device, stream)
    eng.set_params(dt=Δt, t0=initial_time, m=m, DsT=DsT, dims=2, pdim=2, coords=capi.LIM_COORDS_MILNE,
                   collision=capi.LIM_COLL_LANGEVIN, precision=capi.LIM_FP32 if precision == "fp32" else capi.LIM_FP64,
                   seed=seed, block_size=block_size)
    eng.set_medium_rt(np.asarray(xgrid, dtype=np.float64), np.asarray(tgrid, dtype=np.float64), Tfield,
                      np.asarray(VelocityEvolutionn, dtype=np.float64))
    if DsT > 0.0:
        Tmin, Tmax = tr.spline_range(Tfield)
        t0_, inv_, vals = tr.build_tau_drag_spline(m, DsT, Tmin=Tmin, Tmax=Tmax, nT=1024)
        eng.set_spline(capi.LIM_SPLINE_DRAG, t0_, inv_, vals)
    if device_sampling:
        # sample_initial_particles_milne!(m, 2, N, τ0, profiles..., (0, maximum(xgrid)), 200)
        # (simulate_cpu_general_coords.jl:40-41) on the device: the profiles are evaluated at
        # the 200 bin centers, and T(r) for the momentum width on MILNE_T_TABLE nodes
        x_hi = float(np.max(np.asarray(xgrid, dtype=np.float64)))
        edges = np.linspace(0.0, x_hi, MILNE_BINS + 1)
        centers = (edges[:-1] + edges[1:]) / 2
        prof = lambda f, rs: np.array([float(f(r, initial_time)) for r in rs])
        r_T = np.linspace(0.0, x_hi, MILNE_T_TABLE)
        eng.sample_milne(0.0, x_hi, prof(T_profile_MIS, centers), prof(ur_profile_MIS, centers),
                         prof(mu_profile_MIS, centers), r_T, prof(T_profile_MIS, r_T), N)
    else:
        eng.upload_state(positions, momenta)
    nslots = num_saves + 1
    hx = np.empty(nslots * N * 2)
    hp = np.empty(nslots * N * 2)
    eng.download_state_flat(hx[: N * 2], hp[: N * 2])
    try:
        eng.run(1, steps, save_every, 0, hx, hp)
    except capi.LimError as e:          # the Milne CPU driver has no NaN/Inf check
        if e.code != capi.LIM_ERR_NONFINITE:
            raise
    time_points = _time_points(initial_time, final_time, nslots)
    momenta_history = []
    position_history = []
    for k in range(nslots):
        P = hp[k * N * 2:(k + 1) * N * 2].reshape(N, 2)
        X = hx[k * N * 2:(k + 1) * N * 2].reshape(N, 2)
        # simulate_cpu_general_coords.jl:53-55 and :120-124: |p| over (p^τ, p^r) and the r row
        momenta_history.append(np.abs(P[:, 1]) if k == 0 else np.sqrt(np.sum(P ** 2, axis=1)))
        position_history.append(X[:, 1].reshape(1, N).copy())
    return time_points, momenta_history, position_history
