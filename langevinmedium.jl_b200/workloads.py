"""Synthetic workloads with the shapes, sizes and value distributions of the
benchmark configurations (the reference ships no dataset; inputs are seeded).

A workload is plain data: engine parameters, a medium description, transport
tables and an initial state (Julia layout (rows, N)).  ``configure(engine, wl)``
loads it into an engine; test and benchmark code build the CPU restatement's
medium from the same description.

  static_box  — uniform T = 0.30 GeV, zero flow, charm, 3-D, |p| ~ U[0,10] GeV
                isotropic, x ~ U[-5,5]^3 fm, 2πT·D_s = 6, Δt = 0.01, 1000 steps, FP64.
  bjorken     — T(τ) = 0.40 (0.6/τ)^(1/3) GeV, τ 0.6 → 10 fm/c, charm, 2πT·D_s = 4,
                Langevin + RTA with τ_R = 5 (η/s)/T, η/s = 0.16, Δτ = 0.005 (1880 steps),
                p_T ∝ (p_T²+4)^-3 per d²p_T, φ uniform, rapidity uniform in [-1,1].
  grid2p1     — 201×201 cells at 0.1 fm, 100 τ slices 0.6 → 10 fm/c, elliptic Gaussian
                T0 = 0.45 GeV (σx 3.0, σy 2.4 fm) × (0.6/τ)^(1/3), radial flow
                u^r = tanh(0.05 r (τ-0.6)) read as the flow velocity (the reference's
                velocity fields are velocities), freeze-out latch at T < 0.155 GeV, Δt = 0.01.
  adjoint_grid — the grid medium for pathwise gradients: 1e6 charm, 2000 steps of
                Δt = 0.0047 (τ 0.6 → 10), no freeze-out, 2πT·D_s = a + b (T/0.155 - 1)
                and a temperature scale s.
  batch       — 256 independent ensembles (counts log-uniform in [1e3, 1e6], charm or
                bottom, 2πT·D_s ~ U[2,8], 500-2000 steps capped to τ ≤ 10), half Bjorken,
                half 2+1D grids with T0 ~ U[0.35,0.55] GeV and σy/σx ~ U[0.7,1.0].
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import capi
from . import transport as tr

TWO_PI = 2.0 * math.pi


@dataclass
class Workload:
    name: str
    params: dict                      # Engine.set_params keywords
    medium: dict                      # {"kind": "rt"|"bjorken"|"grid", ...arrays}
    splines: dict = field(default_factory=dict)   # which -> (Tmin, invdT, vals)
    invcdf: tuple | None = None       # (vals, nU, nT, Tmin, invdT)
    x: np.ndarray | None = None       # (dims, N)
    p: np.ndarray | None = None       # (pdim, N)
    first_step: int = 1
    steps: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.x.shape[1])

    @property
    def particle_steps(self) -> int:
        return self.n * self.steps


def configure(eng: capi.Engine, wl: Workload, *, upload: bool = True):
    """Load a workload into an engine (parameters, medium, tables, state)."""
    eng.set_params(**wl.params)
    med = wl.medium
    if med["kind"] == "rt":
        eng.set_medium_rt(med["xgrid"], med["tgrid"], med["T"], med["V"], med.get("V2"))
    elif med["kind"] == "bjorken":
        eng.set_medium_bjorken(med["T0"], med["tau0"], med["power"], med["r_max"])
    elif med["kind"] == "grid_lazy":
        g = grid2p1_fields(**med["args"])
        eng.set_medium_grid(g["T"], g["ux"], g["uy"], g["x0"], g["dx"], g["y0"], g["dy"], g["tau0"], g["dtau"])
        del g
    else:
        eng.set_medium_grid(med["T"], med["ux"], med["uy"], med["x0"], med["dx"], med["y0"], med["dy"],
                            med["tau0"], med["dtau"])
    for which, (a, b, v) in wl.splines.items():
        eng.set_spline(which, a, b, v)
    if wl.invcdf is not None:
        eng.set_invcdf(*wl.invcdf)
    if wl.meta.get("scale", 1.0) != 1.0:
        eng.set_medium_scale(wl.meta["scale"])
    if upload:
        eng.upload_state(wl.x, wl.p)


# ---------------------------------------------------------------------------------
# initial states
# ---------------------------------------------------------------------------------
def powerlaw_pt(u: np.ndarray) -> np.ndarray:
    """Inverse CDF of dN/d²p_T ∝ (p_T²+4)^-3: in s = p_T² the CDF is 1 - (4/(s+4))², so
    p_T = 2 sqrt((1-u)^(-1/2) - 1)."""
    return 2.0 * np.sqrt((1.0 - u) ** -0.5 - 1.0)


def rapidity_momenta(rng, N, m):
    """p_T power law, φ uniform, rapidity y ~ U[-1,1], p_z = m_T sinh y (η_s = 0 at τ0)."""
    pT = powerlaw_pt(rng.random(N))
    phi = TWO_PI * rng.random(N)
    y = rng.uniform(-1.0, 1.0, N)
    mT = np.sqrt(m * m + pT * pT)
    return np.vstack([pT * np.cos(phi), pT * np.sin(phi), mT * np.sinh(y)])


# ---------------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------------
def static_box(N=100_000, *, steps=1000, precision="fp64", seed=0x4C494D00, rng_seed=1):
    m, T, DsT, dt = 1.5, 0.30, 6.0 / TWO_PI, 0.01
    rng = np.random.default_rng(rng_seed)
    x = rng.uniform(-5.0, 5.0, (3, N))
    pm = rng.uniform(0.0, 10.0, N)
    d = rng.standard_normal((3, N))
    d /= np.linalg.norm(d, axis=0)
    p = pm * d
    xgrid = np.arange(0.0, 20.0 + 1e-9, 0.5)
    tgrid = np.arange(0.0, steps * dt + 2.0 + 1e-9, 1.0)
    Tf = np.full((xgrid.size, tgrid.size), T)
    Vf = np.zeros_like(Tf)
    Tmin, Tmax = tr.spline_range(Tf)
    spl = {capi.LIM_SPLINE_DRAG: tr.build_tau_drag_spline(m, DsT, Tmin=Tmin, Tmax=Tmax, nT=1024)}
    params = dict(dt=dt, t0=0.0, m=m, DsT=DsT, dims=3, pdim=3, collision=capi.LIM_COLL_LANGEVIN,
                  relativistic=1, precision=capi.LIM_FP32 if precision == "fp32" else capi.LIM_FP64, seed=seed)
    return Workload("static_box", params, dict(kind="rt", xgrid=xgrid, tgrid=tgrid, T=Tf, V=Vf), spl, None,
                    x, p, 1, steps, dict(T=T))


def bjorken(N=1_000_000, *, precision="fp32", table=True, steps=None, seed=0x4C494D01, rng_seed=2,
            dt=0.005, eta_over_s=0.16):
    m, T0, tau0, tauf, DsT = 1.5, 0.40, 0.6, 10.0, 4.0 / TWO_PI
    nsteps = int(math.floor((tauf - tau0) / dt))
    if steps is None:
        steps = nsteps
    rng = np.random.default_rng(rng_seed)
    x = rng.normal(0.0, 3.0, (2, N))
    p = rapidity_momenta(rng, N, m)
    Tfun = lambda tau: T0 * (tau0 / np.maximum(tau, tau0)) ** (1.0 / 3.0)
    Tlo, Thi = float(Tfun(tau0 + (nsteps + 2) * dt)), T0
    if table:
        xgrid = np.arange(0.0, 20.0 + 1e-9, 0.5)
        tgrid = tau0 + dt * np.arange(nsteps + 3)
        Tf = np.broadcast_to(Tfun(tgrid)[None, :], (xgrid.size, tgrid.size)).copy()
        med = dict(kind="rt", xgrid=xgrid, tgrid=tgrid, T=Tf, V=np.zeros_like(Tf))
        Tmin, Tmax = tr.spline_range(Tf)
    else:
        med = dict(kind="bjorken", T0=T0, tau0=tau0, power=1.0 / 3.0, r_max=20.0)
        Tmin, Tmax = Tlo, Thi
    spl = {capi.LIM_SPLINE_DRAG: tr.build_tau_drag_spline(m, DsT, Tmin=Tmin, Tmax=Tmax, nT=1024),
           capi.LIM_SPLINE_RTA: tr.build_tau_R_spline(m, DsT, eta_over_s=eta_over_s, Tmin=Tmin, Tmax=Tmax, nT=1024)}
    inv = tr.build_juttner_invcdf(m, 3, Tmin=Tmin, Tmax=Tmax)
    params = dict(dt=dt, t0=tau0, m=m, DsT=DsT, dims=2, pdim=3, collision=capi.LIM_COLL_LANGEVIN_RTA,
                  relativistic=1, bjorken_redshift=1,
                  precision=capi.LIM_FP32 if precision == "fp32" else capi.LIM_FP64, seed=seed)
    return Workload("bjorken", params, med, spl, inv, x, p, 1, steps, dict(T0=T0, tau0=tau0))


def grid2p1_fields(nx=201, ny=201, nt=100, dx=0.1, tau0=0.6, tauf=10.0, T0=0.45, sx=3.0, sy=2.4, flow=0.05):
    xs = (np.arange(nx) - (nx - 1) / 2) * dx
    ys = (np.arange(ny) - (ny - 1) / 2) * dx
    taus = np.linspace(tau0, tauf, nt)
    X, Y = np.meshgrid(xs, ys, indexing="xy")          # (ny, nx)
    prof = np.exp(-X ** 2 / (2 * sx ** 2) - Y ** 2 / (2 * sy ** 2))
    R = np.sqrt(X ** 2 + Y ** 2)
    T = np.empty((nt, ny, nx), np.float32)
    ux = np.empty_like(T)
    uy = np.empty_like(T)
    with np.errstate(invalid="ignore", divide="ignore"):
        cx = np.where(R > 0, X / R, 0.0)
        cy = np.where(R > 0, Y / R, 0.0)
    for k, tau in enumerate(taus):
        T[k] = T0 * prof * (tau0 / tau) ** (1.0 / 3.0)
        ur = np.tanh(flow * R * (tau - tau0))
        ux[k] = ur * cx
        uy[k] = ur * cy
    return dict(kind="grid", T=T, ux=ux, uy=uy, x0=float(xs[0]), dx=dx, y0=float(ys[0]), dy=dx, tau0=tau0,
                dtau=float(taus[1] - taus[0]))


def grid2p1(N=5_000_000, *, m=1.5, precision="fp32", steps=None, seed=0x4C494D02, rng_seed=3, dt=0.01,
            fields=None, Tfo=0.155, freezeout=True, eta_over_s=0.16, DsT=4.0 / TWO_PI, sx=3.0, sy=2.4):
    med = fields or grid2p1_fields(sx=sx, sy=sy)
    tau0 = med["tau0"]
    tauf = tau0 + (med["T"].shape[0] - 1) * med["dtau"]
    nsteps = int(math.floor((tauf - tau0) / dt))
    if steps is None:
        steps = nsteps
    rng = np.random.default_rng(rng_seed)
    # positions ∝ (Gaussian profile)^2: a Gaussian with σ/√2 per axis
    x = np.vstack([rng.normal(0.0, sx / math.sqrt(2), N), rng.normal(0.0, sy / math.sqrt(2), N)])
    p = rapidity_momenta(rng, N, m)
    Tmin, Tmax = tr.spline_range(med["T"])
    spl = {capi.LIM_SPLINE_DRAG: tr.build_tau_drag_spline(m, DsT, Tmin=Tmin, Tmax=Tmax, nT=1024),
           capi.LIM_SPLINE_RTA: tr.build_tau_R_spline(m, DsT, eta_over_s=eta_over_s, Tmin=Tmin, Tmax=Tmax, nT=1024)}
    inv = tr.build_juttner_invcdf(m, 3, Tmin=Tmin, Tmax=Tmax)
    params = dict(dt=dt, t0=tau0, m=m, DsT=DsT, Tfo=Tfo, dims=2, pdim=3, collision=capi.LIM_COLL_LANGEVIN_RTA,
                  relativistic=1, bjorken_redshift=1, freezeout_capture=int(freezeout), freezeout_interp=1,
                  stop_after_freezeout=int(freezeout),
                  precision=capi.LIM_FP32 if precision == "fp32" else capi.LIM_FP64, seed=seed)
    return Workload("grid2p1", params, med, spl, inv, x, p, 1, steps, dict(m=m))


def grid2p1_lazy(**kw):
    """A grid medium described by its generator arguments; ``configure`` builds the
    fields when it loads the engine and drops them afterwards (the batch holds 128
    grids of 64 MB each on the device, not on the host)."""
    return dict(kind="grid_lazy", args=kw)


def batch(E=256, *, precision="fp32", seed=0x4C494D04, rng_seed=4, n_range=(1e3, 1e6), steps_range=(500, 2000),
          grid_shape=(201, 201, 100), offset0=0):
    """E independent ensembles for one batched launch: particle counts log-uniform in
    n_range, masses from {1.5, 4.75} GeV, 2πT·D_s uniform in [2, 8], step counts uniform
    in steps_range and capped to the medium's τ range 0.6 → 10 fm/c (1880 steps of the
    Bjorken ensembles, 940 of the grid ones); half use the Bjorken medium (analytic T(τ),
    Δτ = 0.005), half 2+1D grids with T0 uniform in [0.35, 0.55] GeV and σy/σx uniform in
    [0.7, 1.0] (σx = 3 fm, Δt = 0.01).  Langevin + RTA, no freeze-out.  Particle ids are consecutive across
    ensembles (particle_offset), so every ensemble has its own noise."""
    rng = np.random.default_rng(rng_seed)
    nx, ny, nt = grid_shape
    kinds = np.array(["bjorken"] * (E // 2) + ["grid"] * (E - E // 2))
    rng.shuffle(kinds)
    lo, hi = math.log(n_range[0]), math.log(n_range[1])
    invcdf_cache = {}
    out = []
    offset = int(offset0)
    for e in range(E):
        n = int(round(math.exp(rng.uniform(lo, hi))))
        m = float(rng.choice([1.5, 4.75]))
        DsT = float(rng.uniform(2.0, 8.0)) / TWO_PI
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        prec = capi.LIM_FP32 if precision == "fp32" else capi.LIM_FP64
        if kinds[e] == "bjorken":
            T0, tau0, dt = 0.40, 0.6, 0.005
            steps = min(steps, int(math.floor((10.0 - tau0) / dt)))      # the medium's tau range, 0.6 -> 10
            med = dict(kind="bjorken", T0=T0, tau0=tau0, power=1.0 / 3.0, r_max=20.0)
            Tmin, Tmax = T0 * (tau0 / (tau0 + (steps + 2) * dt)) ** (1.0 / 3.0), T0
            x = rng.normal(0.0, 3.0, (2, n))
            meta = dict(kind="bjorken", m=m)
        else:
            T0 = float(rng.uniform(0.35, 0.55))
            sx = 3.0
            sy = sx * float(rng.uniform(0.7, 1.0))
            tau0, dt = 0.6, 0.01
            steps = min(steps, int(math.floor((10.0 - tau0) / dt)))      # the grid's tau range, 0.6 -> 10
            med = grid2p1_lazy(nx=nx, ny=ny, nt=nt, T0=T0, sx=sx, sy=sy)
            # the field's minimum: the grid corner at the last slice (grid2p1_fields)
            xm, ym = (nx - 1) / 2 * 0.1, (ny - 1) / 2 * 0.1
            Tmin = T0 * math.exp(-xm ** 2 / (2 * sx ** 2) - ym ** 2 / (2 * sy ** 2)) * (tau0 / 10.0) ** (1.0 / 3.0)
            Tmax = T0
            x = np.vstack([rng.normal(0.0, sx / math.sqrt(2), n), rng.normal(0.0, sy / math.sqrt(2), n)])
            meta = dict(kind="grid", m=m, T0=T0, sx=sx, sy=sy)
        p = rapidity_momenta(rng, n, m)
        spl = {capi.LIM_SPLINE_DRAG: tr.build_tau_drag_spline(m, DsT, Tmin=Tmin, Tmax=Tmax, nT=1024),
               capi.LIM_SPLINE_RTA: tr.build_tau_R_spline(m, DsT, eta_over_s=0.16, Tmin=Tmin, Tmax=Tmax, nT=1024)}
        if m not in invcdf_cache:
            invcdf_cache[m] = tr.build_juttner_invcdf(m, 3, Tmin=1e-3, Tmax=0.56)
        params = dict(dt=dt, t0=tau0, m=m, DsT=DsT, dims=2, pdim=3, collision=capi.LIM_COLL_LANGEVIN_RTA,
                      relativistic=1, bjorken_redshift=1, precision=prec, seed=seed, particle_offset=offset)
        meta.update(DsT=DsT)
        out.append(Workload(f"batch[{e}]", params, med, spl, invcdf_cache[m], x, p, 1, steps, meta))
        offset += n
    return out


def adjoint_grid(N=1_000_000, *, a=3.0, b=2.0, scale=1.0, steps=2000, m=1.5, precision="fp32",
                 seed=0x4C494D03, rng_seed=5, dt=0.0047, fields=None, eta_over_s=0.16, pt_cut=5.0, pt_width=0.1):
    """Differentiation workload: the 2+1D grid medium, charm, Langevin + RTA, no freeze-out,
    2πT·D_s = a + b (max(T, 0.155)/0.155 - 1), medium temperature scale s.  The drag
    spline comes with its derivative tables in (a, b) for lim_adjoint.  dt = 0.0047 fm/c:
    2000 steps span the grid's τ range 0.6 → 10 fm/c (with a longer step the run would
    leave the grid's last time slice, where the medium is held constant)."""
    med = fields or grid2p1_fields()
    tau0 = med["tau0"]
    rng = np.random.default_rng(rng_seed)
    sx, sy = 3.0, 2.4
    x = np.vstack([rng.normal(0.0, sx / math.sqrt(2), N), rng.normal(0.0, sy / math.sqrt(2), N)])
    p = rapidity_momenta(rng, N, m)
    Tmin, Tmax = tr.spline_range(med["T"])
    Tm, inv, vals, d_da, d_db = tr.build_drag_spline_ab(m, a, b, Tmin=Tmin, Tmax=Tmax, nT=1024)
    spl = {capi.LIM_SPLINE_DRAG: (Tm, inv, vals), capi.LIM_SPLINE_DRAG_DA: (Tm, inv, d_da),
           capi.LIM_SPLINE_DRAG_DB: (Tm, inv, d_db),
           capi.LIM_SPLINE_RTA: tr.build_tau_R_spline(m, 1.0, eta_over_s=eta_over_s, Tmin=Tmin, Tmax=Tmax, nT=1024)}
    inv_cdf = tr.build_juttner_invcdf(m, 3, Tmin=Tmin, Tmax=Tmax)
    params = dict(dt=dt, t0=tau0, m=m, DsT=a / TWO_PI, dims=2, pdim=3, collision=capi.LIM_COLL_LANGEVIN_RTA,
                  relativistic=1, bjorken_redshift=1, obs_pt_cut=pt_cut, obs_pt_width=pt_width,
                  precision=capi.LIM_FP32 if precision == "fp32" else capi.LIM_FP64, seed=seed)
    return Workload("adjoint_grid", params, med, spl, inv_cdf, x, p, 1, steps, dict(m=m, a=a, b=b, scale=scale))
