"""Known-answer tests of the transport layer, ported from the reference's
test/runtests.jl:34-128 (same inputs, same tolerances).  CPU only."""
import math

import numpy as np
import pytest
from scipy.special import kve

M_CHARM = 1.5
DST = 0.11634


def tau_n_reference(tr, T, M, DsT):
    return (DsT / T) * (M / T) * (kve(3, M / T) / kve(2, M / T)) / tr.fmGeV


def test_bessel_identity(lmb):
    """runtests.jl:36-40: 2K1 - 3K3 + K5 = (48/z^2) K3."""
    Kx = lmb.transport.besselkx
    for z in (0.5, 1.0, 2.0, 5.0, 9.6, 20.0, 40.0):
        assert math.isclose(2 * Kx(1, z) - 3 * Kx(3, z) + Kx(5, z), (48 / z ** 2) * Kx(3, z), rel_tol=1e-9)


def test_tau_n_main3_closed_form(lmb):
    """runtests.jl:42-51."""
    tr = lmb.transport
    for T in (0.6, 0.5, 0.4, 0.3, 0.25, 0.2, 0.156, 0.12, 0.1):
        assert math.isclose(tr.tau_n_main3(T, M_CHARM, DST), tau_n_reference(tr, T, M_CHARM, DST), rel_tol=1e-8)
        assert tr.tau_n_main3(T, M_CHARM, DST) > 0
    assert tr.tau_n_main3(-1.0, M_CHARM, DST) == 0.0
    assert tr.tau_n_main3(0.3, M_CHARM, 0.0) == 0.0
    assert tr.tau_n_main3(0.3, M_CHARM, -1.0) == 0.0


def test_tau_n_main3_z50_branch(lmb):
    """runtests.jl:53-59."""
    tr = lmb.transport
    Tb, Ta = M_CHARM / 49.99, M_CHARM / 50.01
    assert math.isclose(tr.tau_n_main3(Tb, M_CHARM, DST), tau_n_reference(tr, Tb, M_CHARM, DST), rel_tol=1e-8)
    assert math.isclose(tr.tau_n_main3(Ta, M_CHARM, DST), tau_n_reference(tr, Ta, M_CHARM, DST), rel_tol=1e-6)
    assert math.isclose(tr.tau_n_main3(Tb, M_CHARM, DST), tr.tau_n_main3(Ta, M_CHARM, DST), rel_tol=1e-3)


def test_tau_n_nonrelativistic_limit(lmb):
    """runtests.jl:61-66."""
    tr = lmb.transport
    ratio = lambda T: tr.tau_n_main3(T, M_CHARM, DST) * T ** 2 * tr.fmGeV / (DST * M_CHARM)
    assert ratio(0.05) > 1.0
    assert ratio(0.05) < ratio(0.20)
    assert abs(ratio(0.02) - 1.0) <= 0.05


def test_effective_DsT(lmb):
    """runtests.jl:68-77."""
    e = lmb.transport.effective_DsT
    assert e(0.3, DST) == DST and e(0.6, DST) == DST
    slope, offset, Tfo = 1.765, -0.159, 0.156
    assert math.isclose(e(0.30, DST, DsT_linear=True), slope * 0.30 + offset, rel_tol=1e-12)
    assert math.isclose(e(0.10, DST, DsT_linear=True), slope * Tfo + offset, rel_tol=1e-12)
    assert math.isclose(e(Tfo, DST, DsT_linear=True), slope * Tfo + offset, rel_tol=1e-12)
    with pytest.raises(ValueError):
        e(0.3, DST, DsT_quad=True, DsT_linear=True, DsT_Tref=0.2)
    with pytest.raises(ValueError):
        e(0.3, DST, DsT_quad=True)
    assert math.isclose(e(0.4, DST, DsT_quad=True, DsT_Tref=0.2), DST * 4.0, rel_tol=1e-15)


def test_drag_vs_current_time(lmb):
    """runtests.jl:79-104: tau_drag is the Einstein drag, tau_n/tau_drag = K3/K2, incl. the splines."""
    tr = lmb.transport
    for T in (0.156, 0.20, 0.30, 0.40):
        for dst in (0.116, 0.371):
            z = M_CHARM / T
            td = tr.tau_drag(T, M_CHARM, dst)
            tn = tr.tau_n_main3(T, M_CHARM, dst)
            assert math.isclose(td, M_CHARM * dst / T ** 2 / tr.fmGeV, rel_tol=1e-12)
            assert math.isclose((T / (M_CHARM * (1 / td))) * T * tr.fmGeV, dst, rel_tol=1e-12)
            assert math.isclose(tn / td, kve(3, z) / kve(2, z), rel_tol=1e-12)
            assert tn > td
    Tmin, Tmax, nT = 0.10, 0.50, 128
    _, _, dvals = tr.build_tau_drag_spline(M_CHARM, DST, Tmin=Tmin, Tmax=Tmax, nT=nT)
    _, _, nvals = tr.build_taun_current_spline(M_CHARM, DST, Tmin=Tmin, Tmax=Tmax, nT=nT)
    dT = (Tmax - Tmin) / (nT - 1)
    for i in range(nT):
        z = M_CHARM / (Tmin + i * dT)
        assert math.isclose(nvals[i] / dvals[i], kve(3, z) / kve(2, z), rel_tol=1e-12)


def test_fdr_closure_ou_variance(lmb):
    """runtests.jl:106-127: kappa/(2 eta_D) = MT and the exact-OU stationary variance -> MT (5%)."""
    tr = lmb.transport
    T = 0.3
    tn = tr.tau_drag(T, M_CHARM, DST)
    eta = 1.0 / tn
    kap = 2 * M_CHARM * T / tn
    assert math.isclose(kap / (2 * eta), M_CHARM * T, rel_tol=1e-12)
    dt = 0.02 * tn
    a = math.exp(-eta * dt)
    noise_pref = math.sqrt(kap) * math.sqrt((1 - a * a) / (2 * eta * dt))
    rng = np.random.default_rng(20260615)
    p = np.zeros(40_000)
    for _ in range(800):
        p = a * p + math.sqrt(dt) * noise_pref * rng.standard_normal(p.size)
    assert math.isclose(np.var(p), M_CHARM * T, rel_tol=0.05)


def test_spline_builder_errors_and_eval(lmb):
    """transport.jl:182-184 errors; eval_tau_n_spline extrapolates linearly and returns 0 on NaN."""
    tr = lmb.transport
    with pytest.raises(ValueError, match="Tmin must be > 0"):
        tr.build_tau_drag_spline(M_CHARM, DST, Tmin=0.0, Tmax=0.5, nT=16)
    with pytest.raises(ValueError, match="Tmax must be > Tmin"):
        tr.build_tau_drag_spline(M_CHARM, DST, Tmin=0.5, Tmax=0.5, nT=16)
    with pytest.raises(ValueError, match="nT must be >= 2"):
        tr.build_tau_drag_spline(M_CHARM, DST, Tmin=0.1, Tmax=0.5, nT=1)
    a, inv, v = tr.build_tau_drag_spline(M_CHARM, DST, Tmin=0.1, Tmax=0.5, nT=5)
    assert tr.eval_tau_n_spline(float("nan"), a, inv, v) == 0.0
    assert tr.eval_tau_n_spline(0.1, a, inv, v) == v[0]
    lo = tr.eval_tau_n_spline(0.0, a, inv, v)
    assert math.isclose(lo, v[0] - (v[1] - v[0]) * (0.1 * inv), rel_tol=1e-12)


def test_juttner_invcdf_table(lmb):
    """transport.jl:277-365: monotone rows, p*(0)=0, capped top quantile, and the mean of p*^2
    of a row against quadrature of p^(d-1) exp(-(E-m)/T)."""
    from helpers import jmean
    tr = lmb.transport
    M = 1.5
    for d in (2, 3):
        inv, nU, nT, Tmin, invdT = tr.build_juttner_invcdf(M, d, Tmin=0.2, Tmax=0.4, nT=16, nU=2048, np_=8192)
        tab = inv.reshape(nT, nU)
        assert np.all(np.diff(tab, axis=1) >= 0)
        assert np.all(tab[:, 0] == 0.0)
        j = 7
        T = Tmin + j / invdT
        # midpoint rule in u of p*(u)^2 = <p^2> of the distribution
        u = (np.arange(nU) + 0.5) / nU
        pu = np.interp(u * (nU - 1), np.arange(nU), tab[j])
        assert math.isclose(np.mean(pu ** 2), jmean(lambda p: p * p, M, T, d), rel_tol=5e-3)
