"""Transport coefficients and their tables — host precompute for the engine.

Restates LangevInMedium.jl's ``src/transport.jl`` (paths relative to the reference
project): the drag time ``tau_drag`` (:132-137), the diffusion-current time
``tau_n_main3`` (:58-104), ``effective_DsT`` (:139-156), the uniform linear time
splines (:165-253) and the Jüttner inverse-CDF table (:277-365).  The tables are
built once per run on the host and uploaded; the step kernels only evaluate them.

``LV_TAUN_SCALE`` is read from the environment at import, as ``Transport.__init__``
does (:9-13), and multiplies both splines (:193).
"""
from __future__ import annotations

import math
import os
import warnings

import numpy as np
from scipy import special as _sp

GevInvTofm = 0.197327            # constants.jl:13 (hbar*c in GeV fm)
fmGeV = 1.0 / GevInvTofm         # constants.jl:23
_TINY = 1e-300
EPS = float(np.finfo(np.float64).eps)

LV_TAUN_SCALE = float(os.environ.get("LV_TAUN_SCALE", "1.0"))
if LV_TAUN_SCALE != 1.0:
    warnings.warn("LangevInMedium: tau_n scaled by LV_TAUN_SCALE — DIAGNOSTIC MODE "
                  "(this also rescales eta_D, kappa and hence D_s)")


def besselkx(nu: float, z: float) -> float:
    """Exponentially scaled modified Bessel K: K_nu(z) e^z (Bessels.besselkx)."""
    return float(_sp.kve(nu, z))


def _isfinite(*xs) -> bool:
    return all(math.isfinite(x) for x in xs)


def tau_n_main3(T: float, m: float, DsT: float) -> float:
    """Diffusion-current relaxation time tau_n = D_s z K3/K2 in fm (transport.jl:58-104)."""
    Tm, Mm, Ds = float(T), float(m), float(DsT)
    if not _isfinite(Tm, Mm, Ds) or Tm <= 0.0 or Mm <= 0.0 or Ds <= 0.0:
        return 0.0
    z = Mm / Tm
    if z <= 0.0:
        return 0.0
    K2x = besselkx(2, z)
    K3x = besselkx(3, z)
    denominator = max(abs(K2x), _TINY)
    sgn = math.copysign(1.0, 1.0 if K2x == 0 else K2x)
    if z > 50.0:
        ratio_K3K2 = K3x / denominator * sgn
        tau = (Ds / Tm) * z * ratio_K3K2
        return min(tau / fmGeV, 1e20)
    K1x = besselkx(1, z)
    K5x = besselkx(5, z)
    numerator = 2 * K1x - 3 * K3x + K5x
    ratio = numerator / denominator * sgn
    z3_over_Tm = z * z * z / Tm
    if not math.isfinite(z3_over_Tm) or z3_over_Tm > 1e50:
        z3_over_Tm = 1e50
    tau = (Ds / 48.0) * z3_over_Tm * ratio
    if not math.isfinite(tau) or abs(tau) > 1e50:
        return 1e50 * math.copysign(1.0, tau)
    return tau / fmGeV


def tau_drag(T: float, m: float, DsT: float) -> float:
    """Drag time 1/eta_D = m DsT / T^2 in fm (transport.jl:132-137)."""
    Tm, Mm, Ds = float(T), float(m), float(DsT)
    if not _isfinite(Tm, Mm, Ds) or Tm <= 0.0 or Mm <= 0.0 or Ds <= 0.0:
        return 0.0
    return Mm * Ds / (Tm * Tm) / fmGeV


def tau_R_eta_s(T: float, m: float, DsT: float, eta_over_s: float = 0.16, factor: float = 5.0) -> float:
    """RTA relaxation time tau_R = factor (eta/s) / T in fm (the RTA prescription of the
    Bjorken workload; ``m`` and ``DsT`` are accepted for the common time-function signature)."""
    Tm = float(T)
    if not math.isfinite(Tm) or Tm <= 0.0:
        return 0.0
    return factor * eta_over_s / Tm / fmGeV


def effective_DsT(T, DsT, *, DsT_linear=False, DsT_slope=1.765, DsT_offset=-0.159, Tfo=0.156,
                  DsT_quad=False, DsT_Tref=0.0) -> float:
    """transport.jl:139-156."""
    if DsT_quad:
        if DsT_linear:
            raise ValueError("effective_DsT: DsT_quad and DsT_linear are mutually exclusive")
        if not DsT_Tref > 0.0:
            raise ValueError("effective_DsT: DsT_quad requires DsT_Tref > 0")
        x = float(T) / float(DsT_Tref)
        return float(DsT) * x * x
    if not DsT_linear:
        return float(DsT)
    Tf = max(float(T), float(Tfo))
    return float(DsT_slope) * Tf + float(DsT_offset)


def _build_time_spline(timefn, m, DsT, *, Tmin, Tmax, nT=400, DsT_linear=False, DsT_slope=1.765,
                       DsT_offset=-0.159, Tfo=0.156, DsT_quad=False, DsT_Tref=0.0):
    """Uniform-grid linear spline of timefn(T, m, DsT_eff) in fm (transport.jl:165-196).
    Returns (Tmin, invdT, vals)."""
    Tmin_f, Tmax_f, n = float(Tmin), float(Tmax), int(nT)
    if n < 2:
        raise ValueError("nT must be >= 2")
    if not Tmin_f > 0.0:
        raise ValueError("Tmin must be > 0")
    if not Tmax_f > Tmin_f:
        raise ValueError("Tmax must be > Tmin")
    dT = (Tmax_f - Tmin_f) / (n - 1)
    invdT = 1.0 / dT
    vals = np.empty(n, dtype=np.float64)
    for i in range(n):
        Ti = Tmin_f + i * dT
        Ds = effective_DsT(Ti, DsT, DsT_linear=DsT_linear, DsT_slope=DsT_slope, DsT_offset=DsT_offset,
                           Tfo=Tfo, DsT_quad=DsT_quad, DsT_Tref=DsT_Tref)
        vals[i] = timefn(Ti, m, Ds) * LV_TAUN_SCALE
    return Tmin_f, invdT, vals


def build_tau_drag_spline(m, DsT, **kw):
    """Spline of the DRAG time tau_drag (transport.jl:208-209)."""
    return _build_time_spline(tau_drag, m, DsT, **kw)


def build_taun_current_spline(m, DsT, **kw):
    """Spline of the diffusion-current time tau_n_main3 (transport.jl:221-222)."""
    return _build_time_spline(tau_n_main3, m, DsT, **kw)


def build_tau_R_spline(m, DsT, *, eta_over_s=0.16, factor=5.0, **kw):
    """Spline of the RTA time tau_R = factor (eta/s)/T used by the combined Langevin+RTA step."""
    fn = lambda T, mm, D: tau_R_eta_s(T, mm, D, eta_over_s=eta_over_s, factor=factor)
    return _build_time_spline(fn, m, DsT, **kw)


def ds_linear_params(a, b, Tc=0.155):
    """2πT·D_s = a + b (max(T, Tc)/Tc - 1): the reference's linear D_s form
    (effective_DsT with DsT_linear, transport.jl:139-156) with Tfo = Tc,
    DsT_slope = b/(2π Tc) and DsT_offset = (a - b)/(2π)."""
    two_pi = 2.0 * math.pi
    return dict(DsT_linear=True, DsT_slope=float(b) / (two_pi * Tc), DsT_offset=(float(a) - float(b)) / two_pi,
                Tfo=float(Tc))


def build_drag_spline_ab(m, a, b, *, Tc=0.155, Tmin, Tmax, nT=1024):
    """Drag-time spline for 2πT·D_s = a + b (max(T, Tc)/Tc - 1) and its exact derivatives
    with respect to a and b on the same grid (tau_drag = m D_s T / T^2, transport.jl:132-137):
    returns (Tmin, invdT, vals, d_da, d_db)."""
    Tm, inv, vals = build_tau_drag_spline(m, 1.0, Tmin=Tmin, Tmax=Tmax, nT=nT, **ds_linear_params(a, b, Tc))
    T = Tm + np.arange(len(vals)) / inv
    base = float(m) / (T * T) / fmGeV / (2.0 * math.pi) * LV_TAUN_SCALE
    d_da = base.copy()
    d_db = base * (np.maximum(T, Tc) / Tc - 1.0)
    return Tm, inv, vals, d_da, d_db


def eval_tau_n_spline(T, Tmin, invdT, tau_vals) -> float:
    """transport.jl:231-253 (scalar)."""
    n = len(tau_vals)
    if n < 2:
        return float(tau_vals[0])
    x = float(T)
    if not math.isfinite(x):
        return 0.0
    u = (x - Tmin) * invdT
    i = int(math.floor(u)) + 1
    i = min(max(i, 1), n - 1)
    t = u - (i - 1)
    return (1.0 - t) * float(tau_vals[i - 1]) + t * float(tau_vals[i])


def build_juttner_invcdf(m, dimensions, *, Tmin, Tmax, nT=256, nU=2048, np_=8192, quantile_cap=1.0e-6):
    """Inverse-CDF table of P(p*) ∝ p*^(d-1) exp(-(E-m)/T) (transport.jl:277-365).

    Returns (invCDF, nU, nT, Ttab_min, Ttab_invdT) with invCDF[jT*nU + iu] = p*(u_iu; T_jT).
    """
    M = float(m)
    d = int(dimensions)
    a = d - 1
    nTi, nUi, npi = int(nT), int(nU), int(np_)
    if nTi < 2:
        raise ValueError("nT must be >= 2")
    if nUi < 2:
        raise ValueError("nU must be >= 2")
    if npi < 2:
        raise ValueError("np must be >= 2")
    Tmin_f = max(float(Tmin), 1e-4)
    Tmax_f = max(float(Tmax), Tmin_f * (1.0 + 1e-6))
    span = Tmax_f - Tmin_f
    Tmin_f = max(Tmin_f - 0.02 * span, 1e-4)
    Tmax_f = Tmax_f + 0.02 * span
    dT = (Tmax_f - Tmin_f) / (nTi - 1)
    invdT = 1.0 / dT
    inv = np.empty(nUi * nTi, dtype=np.float64)
    kk = np.arange(npi, dtype=np.float64)
    u = np.arange(nUi, dtype=np.float64) / (nUi - 1)
    thr = 1.0 - float(quantile_cap)
    for jT in range(nTi):
        T = Tmin_f + jT * dT
        pmax = 16.0 * math.sqrt(M * T) + 16.0 * T
        dp = pmax / (npi - 1)
        p = kk * dp
        E = np.sqrt(M * M + p * p)
        if a == 0:
            w = np.exp(-(E - M) / T)
        else:
            w = (p ** a) * np.exp(-(E - M) / T)
        w[0] = 1.0 if a == 0 else 0.0
        inc = 0.5 * (w[:-1] + w[1:]) * dp
        cdf = np.empty(npi)
        cdf[0] = 0.0
        cdf[1:] = np.cumsum(inc)
        norm = cdf[-1]
        invnorm = 1.0 / norm if norm > 0.0 else 0.0
        cdf *= invnorm
        cdf[-1] = 1.0
        hit = np.nonzero(cdf >= thr)[0]
        p_hi = p[hit[0]] if hit.size else p[-1]
        # monotone sweep: k = 1 + #{j >= 2 : cdf[j] < u} (1-based), i.e. 0-based below
        k = np.searchsorted(cdf[1:], u, side="left")
        k = np.minimum(k, npi - 2)
        c0, c1 = cdf[k], cdf[k + 1]
        p0, p1 = p[k], p[k + 1]
        with np.errstate(divide="ignore", invalid="ignore"):
            frac = np.where(c1 > c0, (u - c0) / (c1 - c0), 0.0)
        frac = np.clip(frac, 0.0, 1.0)
        pval = p0 + frac * (p1 - p0)
        inv[jT * nUi:(jT + 1) * nUi] = np.where(pval < p_hi, pval, p_hi)
    return inv, nUi, nTi, Tmin_f, invdT


def spline_range(Tfield) -> tuple[float, float]:
    """Tmin/Tmax used by the drivers (simulate_cpu.jl:191-192)."""
    Tmin = max(float(np.min(Tfield)), 0.0)
    Tmax = max(float(np.max(Tfield)), Tmin + EPS)
    return Tmin, Tmax
