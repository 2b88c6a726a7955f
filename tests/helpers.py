"""Shared test helpers: reference quantities, samplers, the oracle box driver and
the parity metric."""
from __future__ import annotations

import math

import numpy as np
from scipy import integrate
from scipy.special import kve

from conftest import load_pkg

HBARC_TEST = 0.1973269804        # the tests' hbar*c (test_momentum_dims3.jl:23)


def jmean(g, M, T, d):
    """<g(p)> in the d-dimensional Jüttner at (M, T) by quadrature (test_momentum_dims3.jl:27-32)."""
    w = lambda p: p ** (d - 1) * math.exp(-(math.sqrt(p * p + M * M) - M) / T)
    num = integrate.quad(lambda p: g(p) * w(p), 0, np.inf, epsrel=1e-12, limit=200)[0]
    den = integrate.quad(w, 0, np.inf, epsrel=1e-12, limit=200)[0]
    return num / den


def lam1(M, T, d):
    return jmean(lambda p: (M / math.sqrt(p * p + M * M)) * p * p, M, T, d) / jmean(lambda p: p * p, M, T, d)


def p2eq(M, T, d):
    return jmean(lambda p: p * p, M, T, d)


def K2K3(z):
    return kve(2, z) / kve(3, z)


def juttner_sample(rng, M, T, d, N):
    """Isotropic d-dimensional Jüttner sample by rejection (test_momentum_dims3.jl:38-52), vectorised."""
    pmax = 14 * math.sqrt(M * T + T * T)
    w = lambda p: p ** (d - 1) * np.exp(-(np.sqrt(p * p + M * M) - M) / T)
    wmax = np.max(w(np.linspace(1e-6, pmax, 4000)))
    out = np.empty(N)
    filled = 0
    while filled < N:
        k = 2 * (N - filled) + 1000
        p = pmax * rng.random(k)
        acc = rng.random(k) * wmax <= w(p)
        take = p[acc][: N - filled]
        out[filled:filled + take.size] = take
        filled += take.size
    n = rng.standard_normal((d, N))
    n /= np.linalg.norm(n, axis=0)
    return out * n


def est(mom, M):
    """<p^2>, lambda_1, <p_x>, <(M/E) p_x> on one snapshot (test_momentum_dims3.jl:74-78)."""
    p2 = np.sum(mom ** 2, axis=0)
    E = np.sqrt(M * M + p2)
    return dict(p2=np.mean(p2), lam=np.mean((M / E) * p2) / np.mean(p2), jx=np.mean(mom[0]),
                jxw=np.mean((M / E) * mom[0]))


def box_medium(T, t0, tfinal):
    xgrid = np.arange(0.0, 400.0 + 0.25, 0.5)
    tgrid = np.arange(t0, t0 + tfinal + 2 + 1e-9, 1.0)
    Tf = np.full((xgrid.size, tgrid.size), T)
    Vf = np.zeros_like(Tf)
    return xgrid, tgrid, Tf, Vf


def oracle_drive(orc, *, xgrid, tgrid, Tf, Vf, x0, p0, M, DsT, dt, t0, tfinal, save, dims, pdim,
                 redshift=False, momentum_langevin=True, relativistic=True, seed=1, collision=0,
                 V2=None, psi2=0.0, position_diffusion=False, reflecting_boundary=False, integrator_mode=0,
                 Tfo=0.0, freezeout_capture=False, threads=0, rta_spline="current", eta_over_s=0.16):
    """The driver of simulate_cpu.jl:12-323 around the restatement: splines, step-0
    boost, loop with snapshots.  Returns (times, mom_hist, pos_hist, out)."""
    tr = load_pkg().transport
    steps = int(math.floor((t0 + tfinal - t0) / dt))
    save_every = int(round(save / dt))
    num_saves = steps // save_every
    coll = collision
    if not momentum_langevin or DsT == 0.0:
        coll = 3
    P = orc.make_params(dt=dt, t0=t0, m=M, DsT=DsT, Tfo=Tfo, psi2=psi2, dims=dims, pdim=pdim, collision=coll,
                        relativistic=int(relativistic), bjorken_redshift=int(redshift),
                        position_diffusion=int(position_diffusion), reflecting_boundary=int(reflecting_boundary),
                        integrator_mode=integrator_mode, freezeout_capture=int(freezeout_capture), seed=seed)
    md = orc.Medium().rt(xgrid, tgrid, Tf, Vf, V2)
    if momentum_langevin and DsT > 0:
        Tmin, Tmax = tr.spline_range(Tf)
        a, b, v = tr.build_tau_drag_spline(M, DsT, Tmin=Tmin, Tmax=Tmax, nT=1024)
        md.spline(0, a, b, v)
        if coll in (1, 2):
            if rta_spline == "current":
                _, _, v2 = tr.build_taun_current_spline(M, DsT, Tmin=Tmin, Tmax=Tmax, nT=1024)
            else:
                _, _, v2 = tr.build_tau_R_spline(M, DsT, eta_over_s=eta_over_s, Tmin=Tmin, Tmax=Tmax, nT=1024)
            md.spline(1, a, b, v2)
            inv, nU, nT, Tm, Ti = tr.build_juttner_invcdf(M, pdim, Tmin=Tmin, Tmax=Tmax)
            md.invcdf(inv, nU, nT, Tm, Ti)
    x, p = orc.initial_lab_boost(P, md, x0, p0)
    out = orc.run(P, md, x, p, 1, steps, save_every=save_every, first_slot=0, nslots=num_saves + 1,
                  threads=threads)
    mh = [p] + out["hist_p"][1:]
    xh = [x] + out["hist_x"][1:]
    times = np.linspace(t0, t0 + tfinal, num_saves + 1)
    return times, mh, xh, out


def parity(a, b, scale, floor=1e-3):
    """Per-particle relative error ||a_i - b_i|| / max(||b_i||, floor * scale) over the
    rows of (rows, N) arrays; returns (max, p99).  scale: 0.3 GeV for momenta, 1 fm
    for positions."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.ndim == 1:
        a, b = a[None, :], b[None, :]
    if a.size == 0:
        return 0.0, 0.0
    e = np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), floor * scale)
    return float(np.max(e)), float(np.percentile(e, 99))


def oracle_medium(orc, wl):
    """The restatement's medium/tables from a workload description."""
    med = wl.medium
    md = orc.Medium()
    if med["kind"] == "rt":
        md.rt(med["xgrid"], med["tgrid"], med["T"], med["V"], med.get("V2"))
    elif med["kind"] == "bjorken":
        md.bjorken(med["T0"], med["tau0"], med["power"], med["r_max"])
    else:
        md.grid(med["T"], med["ux"], med["uy"], med["x0"], med["dx"], med["y0"], med["dy"], med["tau0"], med["dtau"])
    for w, (a, b, v) in wl.splines.items():
        md.spline(w, a, b, v)
    if wl.invcdf is not None:
        md.invcdf(*wl.invcdf)
    if wl.meta.get("scale", 1.0) != 1.0:
        md.scale(wl.meta["scale"])
    return md


def oracle_params(orc, wl, **over):
    d = dict(wl.params)
    d.update(over)
    return orc.make_params(**d)
