"""Parity cases: small seeded workloads covering every branch of the step
(medium kinds, dimensions, collision modes, switches), each small enough for the
CPU restatement to finish in seconds."""
from __future__ import annotations

import math
import zlib

import numpy as np

from conftest import load_pkg

TWO_PI = 2 * math.pi


def _tables(wl, tr, capi, Tf, m, DsT, pdim, rta=None, eta_over_s=0.16, spline_range=None):
    Tmin, Tmax = spline_range or tr.spline_range(Tf)
    wl.splines[capi.LIM_SPLINE_DRAG] = tr.build_tau_drag_spline(m, DsT, Tmin=Tmin, Tmax=Tmax, nT=1024)
    if rta == "current":
        wl.splines[capi.LIM_SPLINE_RTA] = tr.build_taun_current_spline(m, DsT, Tmin=Tmin, Tmax=Tmax, nT=1024)
    elif rta == "tauR":
        wl.splines[capi.LIM_SPLINE_RTA] = tr.build_tau_R_spline(m, DsT, eta_over_s=eta_over_s, Tmin=Tmin,
                                                                Tmax=Tmax, nT=1024)
    if rta:
        wl.invcdf = tr.build_juttner_invcdf(m, pdim, Tmin=Tmin, Tmax=Tmax)


def flow_table(xmax=15.0, dx=0.25, tmax=10.0, dt=0.5, t0=0.0, nonuniform=False):
    if nonuniform:
        xgrid = xmax * (np.linspace(0, 1, 61) ** 1.5)
        tgrid = t0 + tmax * (np.linspace(0, 1, 23) ** 1.3)
    else:
        xgrid = np.arange(0.0, xmax + 1e-9, dx)
        tgrid = np.arange(t0, t0 + tmax + 1e-9, dt)
    R, Tm = np.meshgrid(xgrid, tgrid, indexing="ij")
    T = 0.12 + 0.33 * np.exp(-R ** 2 / 40.0) / (1.0 + 0.15 * (Tm - t0))
    V = 0.7 * np.tanh(0.12 * R) * np.tanh(0.35 * (Tm - t0) + 0.05)
    V2 = 0.05 * np.tanh(0.2 * R)
    return xgrid, tgrid, T, V, V2


def initial(rng, N, dims, pdim, spread=4.0, pmax=4.0):
    x = rng.normal(0.0, spread, (dims, N))
    if dims == 1:
        x = np.abs(x)
    p = rng.normal(0.0, pmax / 2, (pdim, N))
    return x, p


CASES = ["static3d", "flow2d", "flow2d_nonrel", "flow2d_v2", "flow2d_midpoint", "flow2d_nonuniform",
         "flow3d", "rta2d", "lrta_bjorken_table", "fluid_redshift", "radial_diffusion_reflect",
         "cart_diffusion_reflect", "freezeout", "milne", "bjorken_analytic", "grid_lrta_fo", "grid_fine_tau_fo",
         "grid_offset_fo"]


def build_case(name: str, precision: str = "fp64", N: int = 2048, steps: int | None = None, seed: int = 7):
    pkg = load_pkg()
    capi, tr, W = pkg.capi, pkg.transport, pkg.workloads
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    prec = capi.LIM_FP32 if precision == "fp32" else capi.LIM_FP64
    base = dict(precision=prec, seed=seed, relativistic=1)
    m, DsT = 1.5, 0.25
    if name == "static3d":
        wl = W.static_box(N=N, steps=steps or 200, precision=precision, seed=seed)
        return wl
    if name.startswith("flow2d") or name in ("flow3d", "rta2d", "cart_diffusion_reflect", "radial_diffusion_reflect",
                                             "freezeout", "fluid_redshift"):
        dims = 3 if name == "flow3d" else (1 if name == "radial_diffusion_reflect" else 2)
        pdim = 3 if name in ("fluid_redshift", "freezeout", "flow3d") else dims
        t0 = 0.5 if name == "fluid_redshift" else 0.0
        xmax = 6.0 if "reflect" in name else 15.0
        xg, tg, T, V, V2 = flow_table(xmax=xmax, t0=t0, nonuniform=(name == "flow2d_nonuniform"))
        if name == "freezeout":
            T = 0.30 * np.exp(-np.meshgrid(xg, tg, indexing="ij")[0] ** 2 / 60.0) * np.exp(
                -0.25 * np.meshgrid(xg, tg, indexing="ij")[1])
        med = dict(kind="rt", xgrid=xg, tgrid=tg, T=T, V=V)
        if name == "flow2d_v2":
            med["V2"] = V2
        p = dict(base, dt=0.01, t0=t0, m=m, DsT=DsT, dims=dims, pdim=pdim, collision=capi.LIM_COLL_LANGEVIN,
                 psi2=0.3)
        if name == "flow2d_nonrel":
            p["relativistic"] = 0
        if name == "flow2d_midpoint":
            p["integrator_mode"] = 1
        if name == "rta2d":
            p["collision"] = capi.LIM_COLL_RTA
        if name == "fluid_redshift":
            p.update(collision=capi.LIM_COLL_FLUID, bjorken_redshift=1)
        if "diffusion" in name:
            p.update(position_diffusion=1, reflecting_boundary=1)
        if name == "freezeout":
            p.update(freezeout_capture=1, freezeout_interp=1, Tfo=0.16)
        x, pp = initial(rng, N, dims, pdim, spread=2.5 if "reflect" in name else 4.0)
        wl = W.Workload(name, p, med, {}, None, x, pp, 1, steps or 300)
        _tables(wl, tr, capi, T, m, DsT, pdim, rta="current" if name == "rta2d" else None)
        return wl
    if name == "lrta_bjorken_table":
        wl = W.bjorken(N=N, precision=precision, steps=steps or 300, seed=seed)
        return wl
    if name == "bjorken_analytic":
        wl = W.bjorken(N=N, precision=precision, steps=steps or 300, seed=seed, table=False)
        return wl
    if name == "milne":
        xg, tg, T, V, _ = flow_table(xmax=12.0, t0=0.6)
        V = 0.3 * V
        p = dict(base, dt=0.01, t0=0.6, m=m, DsT=DsT, dims=2, pdim=2, coords=capi.LIM_COORDS_MILNE,
                 collision=capi.LIM_COLL_LANGEVIN)
        tau = np.full(N, 0.6)
        r = np.abs(rng.normal(0.0, 3.0, N))
        pr = rng.normal(0.0, 1.5, N)
        ptau = np.sqrt(m * m + pr * pr)
        wl = W.Workload(name, p, dict(kind="rt", xgrid=xg, tgrid=tg, T=T, V=V), {}, None,
                        np.vstack([tau, r]), np.vstack([ptau, pr]), 1, steps or 300)
        _tables(wl, tr, capi, T, m, DsT, 2)
        return wl
    if name == "grid_lrta_fo":
        f = W.grid2p1_fields(nx=81, ny=61, nt=24, dx=0.25, sx=3.0, sy=2.4)
        wl = W.grid2p1(N=N, precision=precision, fields=f, steps=steps or 300, seed=seed, dt=0.02)
        return wl
    if name == "grid_fine_tau_fo":
        # time rows (dtau 0.0151) finer than the step (0.02): every step starts a new
        # time row, so the FP32 kernel's latch screen never reuses the step's lookup
        f = W.grid2p1_fields(nx=41, ny=41, nt=160, dx=0.5, tau0=0.6, tauf=3.0, sx=3.0, sy=2.4)
        wl = W.grid2p1(N=N, precision=precision, fields=f, steps=steps or 110, seed=seed, dt=0.02)
        return wl
    if name == "grid_offset_fo":
        # an even node count, a spacing whose reciprocal FP32 does not hold exactly and a
        # grid shifted off the particles' centre: the FP32 cell location's centre node
        # (index 31 of 64) is not at 0, so its TwoSum and low-word terms are all non-zero
        f = W.grid2p1_fields(nx=64, ny=57, nt=24, dx=0.3, sx=3.0, sy=2.4)
        f["x0"] += 1.37
        f["y0"] -= 0.61
        wl = W.grid2p1(N=N, precision=precision, fields=f, steps=steps or 300, seed=seed, dt=0.02)
        return wl
    raise KeyError(name)
