"""Device initial-state sampling (lim_sample_fonll) against the oracle's restatement on
the same Philox counters: positions and momenta agree to FP64 rounding in both state
precisions, for Cartesian and polar sampling, antithetic pairs, odd counts and the
thermal p_z of each medium kind; the errors of the reference (zero normalisation) and
of an exhausted rejection loop come back as error codes.  Then a run started from the
device sample matches the oracle run started from the oracle's sample."""
import numpy as np
import pytest

from helpers import oracle_drive, parity
from test_sample_oracle import fonll_like, milne_profiles

pytestmark = pytest.mark.gpu

SEED = 0x5EED5A3


def _media(orc):
    xg = np.linspace(0.0, 12.0, 49)
    tg = np.linspace(0.4, 3.0, 27)
    T = 0.45 * np.exp(-xg[:, None] ** 2 / 50.0) * (0.6 / tg[None, :]) ** (1 / 3)
    V = 0.05 * xg[:, None] * np.ones_like(tg)[None, :]
    nx = ny = 41
    nt = 9
    gx = np.linspace(-10, 10, nx)
    X, Y = np.meshgrid(gx, gx)
    Tg = np.stack([0.5 * np.exp(-(X ** 2 + 0.8 * Y ** 2) / 40.0) * (1 - 0.05 * k) for k in range(nt)]).astype(np.float32)
    ux = (0.02 * X * np.ones((nt, 1, 1))).astype(np.float32)
    uy = (0.02 * Y * np.ones((nt, 1, 1))).astype(np.float32)
    grid = dict(T=Tg, ux=ux, uy=uy, x0=-10.0, dx=0.5, y0=-10.0, dy=0.5, tau0=0.4, dtau=0.3)
    return {
        "rt": (lambda e: e.set_medium_rt(xg, tg, T, V), lambda: orc.Medium().rt(xg, tg, T, V)),
        "bjorken": (lambda e: e.set_medium_bjorken(0.42, 0.4), lambda: orc.Medium().bjorken(0.42, 0.4)),
        "grid": (lambda e: e.set_medium_grid(**grid), lambda: orc.Medium().grid(**grid)),
    }


def _engine(lmb, prec, pdim, t0=0.6, m=1.5, seed=SEED, offset=0):
    e = lmb.capi.Engine(0)
    e.set_params(dims=2, pdim=pdim, coords=lmb.capi.LIM_COORDS_CARTESIAN, t0=t0, m=m, dt=0.01,
                 precision=lmb.capi.LIM_FP32 if prec == "fp32" else lmb.capi.LIM_FP64, seed=seed,
                 particle_offset=offset)
    return e


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("cart,anti,n", [(True, False, 4096), (False, False, 4096), (True, True, 4097),
                                         (False, True, 33), (True, False, 1)])
@pytest.mark.parametrize("medium", ["rt", "bjorken", "grid"])
def test_sample_matches_oracle(lmb, orc, prec, cart, anti, n, medium):
    r, p, f = fonll_like()
    dev_set, orc_md = _media(orc)[medium]
    e = _engine(lmb, prec, 3, offset=17)
    dev_set(e)
    e.sample_fonll(r, p, f, n, cartesian=cart, antithetic=anti, thermal_pz=True)
    xd, pd = e.download_state()
    P = orc.make_params(seed=SEED, dims=2, pdim=3, t0=0.6, m=1.5, particle_offset=17)
    xo, po, failed = orc.sample_fonll(P, orc_md(), r, p, f, n, cartesian=cart, antithetic=anti, thermal_pz=True)
    assert failed == 0
    assert xd.shape == (2, n) and pd.shape == (3, n)
    assert np.max(np.abs(xd - xo)) <= 1e-12 * max(1.0, np.max(np.abs(xo)))
    assert np.max(np.abs(pd[:2] - po[:2])) <= 1e-12 * max(1.0, np.max(np.abs(po)))
    # p_z: the FP32 state precision reads the medium from its FP32 tables, so the local
    # temperature (and with it p_z) carries FP32 rounding there
    tol_pz = 1e-12 if prec == "fp64" else 1e-6
    assert np.max(np.abs(pd[2] - po[2])) <= tol_pz * max(1.0, np.max(np.abs(po[2])))
    assert np.any(po[2] != 0.0)


def test_sample_transverse_only_and_transposed_table(lmb, orc):
    r, p, f = fonll_like()
    e = _engine(lmb, "fp64", 2)
    e.sample_fonll(r, p, f.T, 500, cartesian=True)            # Nr x Np is accepted (transposed)
    xd, pd = e.download_state()
    P = orc.make_params(seed=SEED, dims=2, pdim=2, t0=0.6, m=1.5)
    xo, po, _ = orc.sample_fonll(P, None, r, p, f, 500, cartesian=True)
    assert np.max(np.abs(xd - xo)) <= 1e-12 * 10 and np.max(np.abs(pd - po)) <= 1e-12 * 10


def test_sample_errors(lmb):
    r, p, _ = fonll_like(nr=5, np_=5)
    e = _engine(lmb, "fp64", 2)
    with pytest.raises(RuntimeError, match="normalization is zero"):
        e.sample_fonll(r, p, np.zeros((5, 5)), 8, cartesian=False)
    with pytest.raises(RuntimeError, match="no accepted trial"):
        e.sample_fonll(r, p, np.zeros((5, 5)), 8, cartesian=True)
    e.sample_fonll(r, p, np.ones((5, 5)), 0, cartesian=True)  # empty ensemble
    e3 = _engine(lmb, "fp64", 3)
    with pytest.raises(RuntimeError, match="needs the medium"):
        e3.sample_fonll(r, p, np.ones((5, 5)), 8, thermal_pz=True)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_run_from_device_sample(lmb, orc, prec):
    """simulate_ensemble_bulk without x_init/p_init samples on the device; the oracle,
    started from its own sample of the same counters, gives the same final state."""
    r, p, f = fonll_like()
    xg = np.linspace(0.0, 12.0, 49)
    tg = np.linspace(0.0, 2.0, 41)
    T = 0.40 * np.exp(-xg[:, None] ** 2 / 80.0) * np.ones_like(tg)[None, :]
    V = 0.3 * np.tanh(0.1 * xg[:, None]) * np.ones_like(tg)[None, :]
    N, dt, steps = 3000, 0.01, 50
    out = lmb.simulate_ensemble_bulk(
        lmb.B200Backend(), r, p, f, T, V, (xg, tg), N_particles=N, Δt=dt, initial_time=0.0, final_time=steps * dt,
        save_interval=steps * dt, m=1.5, DsT=0.3, dimensions=2, momentum_dimensions=3, antithetic_momenta=True,
        position_diffusion=False, reflecting_boundary=False, Tfo=0.0, seed=SEED, precision=prec)
    _, mom, pos = out
    P = orc.make_params(seed=SEED, dims=2, pdim=3, t0=0.0, m=1.5)
    xo, po, failed = orc.sample_fonll(P, orc.Medium().rt(xg, tg, T, V), r, p, f, N, cartesian=True, antithetic=True,
                                      thermal_pz=True)
    assert failed == 0
    _, mh, xh, _ = oracle_drive(orc, xgrid=xg, tgrid=tg, Tf=T, Vf=V, x0=xo, p0=po, M=1.5, DsT=0.3, dt=dt, t0=0.0,
                                tfinal=steps * dt, save=steps * dt, dims=2, pdim=3, seed=SEED)
    tol = 1e-12 if prec == "fp64" else 1e-5
    for k in (0, -1):
        emax, e99 = parity(mom[k], mh[k], 0.3)
        assert (emax if prec == "fp64" else e99) <= tol, (k, emax, e99)
        emax, e99 = parity(pos[k], xh[k], 1.0)
        assert (emax if prec == "fp64" else e99) <= tol, (k, emax, e99)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [1, 777, 20_000])
def test_milne_sample_matches_oracle(lmb, orc, prec, n):
    c, Tc, urc, muc, Tf = milne_profiles()
    rT = np.linspace(0.0, 10.0, 1601)
    e = lmb.capi.Engine(0)
    e.set_params(dims=2, pdim=2, coords=lmb.capi.LIM_COORDS_MILNE, t0=0.4, m=1.5, dt=0.01, seed=SEED,
                 particle_offset=5, precision=lmb.capi.LIM_FP32 if prec == "fp32" else lmb.capi.LIM_FP64)
    e.sample_milne(0.0, 10.0, Tc, urc, muc, rT, Tf(rT), n)
    xd, pd = e.download_state()
    P = orc.make_params(seed=SEED, dims=2, pdim=2, m=1.5, t0=0.4, particle_offset=5)
    xo, po, failed = orc.sample_milne(P, 0.0, 10.0, Tc, urc, muc, rT, Tf(rT), n)
    assert failed == 0
    assert np.max(np.abs(xd - xo)) <= 1e-12 * 10
    assert np.max(np.abs(pd - po)) <= 1e-12 * max(1.0, np.max(np.abs(po)))


def test_milne_sample_errors(lmb):
    c, Tc, urc, muc, Tf = milne_profiles(nbins=4)
    rT = np.linspace(0.0, 10.0, 5)
    e = lmb.capi.Engine(0)
    e.set_params(dims=2, pdim=2, coords=lmb.capi.LIM_COORDS_MILNE, t0=0.4, m=1.5, dt=0.01)
    with pytest.raises(RuntimeError, match="no positive finite maximum"):
        e.sample_milne(0.0, 10.0, np.zeros(4), urc, muc, rT, Tf(rT), 8)
    ec = _engine(lmb, "fp64", 2)
    with pytest.raises(RuntimeError, match="requires dim = 2"):
        ec.sample_milne(0.0, 10.0, Tc, urc, muc, rT, Tf(rT), 8)


def test_milne_run_from_device_sample(lmb, orc):
    """simulate_ensemble_bulk(B200_GCBackend()) without x_init samples on the device: the
    first snapshot is the oracle's sample (|p^r| and r), and the run stays finite."""
    c, Tc, urc, muc, Tf = milne_profiles()
    xg = np.linspace(0.0, 10.0, 41)
    tg = np.linspace(0.4, 2.4, 21)
    T = (0.42 * np.exp(-xg[:, None] ** 2 / 30.0) + 0.05) * (0.4 / tg[None, :]) ** (1 / 3)
    V = 0.05 * xg[:, None] * np.ones_like(tg)[None, :]
    prof_T = lambda r, tau: 0.42 * np.exp(-r ** 2 / 30.0) + 0.05
    prof_ur = lambda r, tau: 0.04 * r
    prof_mu = lambda r, tau: 0.02 * np.sin(r)
    N = 4000
    t, mom, pos = lmb.simulate_ensemble_bulk(lmb.B200_GCBackend(), prof_T, prof_ur, prof_mu, T, V, (xg, tg),
                                             N_particles=N, Δt=0.01, initial_time=0.4, final_time=0.9,
                                             save_interval=0.25, m=1.5, DsT=0.3, seed=SEED)
    P = orc.make_params(seed=SEED, dims=2, pdim=2, m=1.5, t0=0.4)
    edges = np.linspace(0.0, 10.0, 201)
    cen = (edges[:-1] + edges[1:]) / 2
    rT = np.linspace(0.0, 10.0, 1601)
    xo, po, failed = orc.sample_milne(P, 0.0, 10.0, prof_T(cen, 0.4), prof_ur(cen, 0.4), prof_mu(cen, 0.4), rT,
                                      prof_T(rT, 0.4), N)
    assert failed == 0
    assert np.max(np.abs(pos[0][0] - xo[1])) <= 1e-12 * 10
    assert np.max(np.abs(mom[0] - po[1])) <= 1e-12 * 10
    assert len(mom) == 3 and np.all(np.isfinite(mom[-1])) and np.all(np.isfinite(pos[-1]))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_grid_freezeout_run_from_device_sample(lmb, orc, prec):
    """Device FONLL sample (with thermal p_z from the grid medium at tau0), then the 2+1D
    grid Langevin+RTA run with the freeze-out latch and stopping particles, against the
    oracle started from its own sample: the latched outputs agree and the same particles
    freeze out."""
    from helpers import oracle_medium, oracle_params
    r, p, f = fonll_like()
    fields = lmb.workloads.grid2p1_fields(nx=81, ny=61, nt=24, dx=0.25)
    n, steps = 2048, 300
    wl = lmb.workloads.grid2p1(N=n, precision=prec, fields=fields, steps=steps, dt=0.02)
    e = lmb.capi.Engine(0)
    lmb.workloads.configure(e, wl, upload=False)
    e.sample_fonll(r, p, f, n, cartesian=True, thermal_pz=True)
    e.initial_lab_boost()
    e.run(1, steps)
    fo = e.download_freezeout()
    P = oracle_params(orc, wl)
    md = oracle_medium(orc, wl)
    xo, po, failed = orc.sample_fonll(P, md, r, p, f, n, cartesian=True, thermal_pz=True)
    assert failed == 0
    x0, p0 = orc.initial_lab_boost(P, md, xo, po)
    out = orc.run(P, md, x0, p0, 1, steps)
    assert np.array_equal(fo["flag"], out["fo_flag"])
    assert np.count_nonzero(fo["flag"]) > 0
    for a, b, sc in ((fo["mom"], out["fo_mom"], 0.3), (fo["pos"], out["fo_pos"], 1.0)):
        emax, e99 = parity(a, b, sc, 1e-2 if prec == "fp64" else 1.0)
        if prec == "fp64":
            assert emax <= 1e-12, emax
        else:
            assert e99 <= 1e-5 and emax <= 1e-3, (emax, e99)
