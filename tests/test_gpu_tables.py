"""Transport tables built on the device (lim_build_time_spline, lim_build_juttner_invcdf)
against the host builders that restate transport.jl (transport.py), and a run on
device-built tables against the oracle on host-built ones."""
import numpy as np
import pytest

from helpers import box_medium, oracle_drive, parity

pytestmark = pytest.mark.gpu

FORMS = [dict(), dict(DsT_linear=True, DsT_slope=1.765, DsT_offset=-0.159, Tfo=0.156),
         dict(DsT_quad=True, DsT_Tref=0.2)]


def _engine(lmb):
    e = lmb.capi.Engine(0)
    e.set_params(dims=2, pdim=3, dt=0.01, m=1.5)
    return e


@pytest.mark.parametrize("form", range(len(FORMS)))
@pytest.mark.parametrize("m", [1.5, 4.75])
def test_time_splines_match_host(lmb, form, m):
    tr, capi = lmb.transport, lmb.capi
    e = _engine(lmb)
    kw = dict(Tmin=0.1, Tmax=0.6, nT=1024, **FORMS[form])
    for kind, host, rtol in ((capi.LIM_TIME_DRAG, tr.build_tau_drag_spline, 1e-14),
                             (capi.LIM_TIME_TAUN, tr.build_taun_current_spline, 1e-11),
                             (capi.LIM_TIME_TAUR, tr.build_tau_R_spline, 1e-14)):
        e.build_time_spline(capi.LIM_SPLINE_DRAG, kind, m, 0.2, **kw)
        t0, inv, vals = e.get_spline(capi.LIM_SPLINE_DRAG)
        h0, hinv, hvals = host(m, 0.2, **kw)
        assert t0 == h0 and inv == pytest.approx(hinv, rel=1e-15)
        assert np.allclose(vals, hvals, rtol=rtol, atol=0.0), (kind, np.max(np.abs(vals / hvals - 1)))


def test_time_spline_errors(lmb):
    capi = lmb.capi
    e = _engine(lmb)
    for kw, msg in ((dict(Tmin=0.0, Tmax=0.6), "Tmin must be > 0"), (dict(Tmin=0.3, Tmax=0.2), "Tmax must be > Tmin"),
                    (dict(Tmin=0.1, Tmax=0.6, nT=1), "nT must be >= 2"),
                    (dict(Tmin=0.1, Tmax=0.6, DsT_linear=True, DsT_quad=True, DsT_Tref=0.2), "mutually exclusive"),
                    (dict(Tmin=0.1, Tmax=0.6, DsT_quad=True), "DsT_Tref > 0")):
        with pytest.raises(RuntimeError, match=msg):
            e.build_time_spline(capi.LIM_SPLINE_DRAG, capi.LIM_TIME_DRAG, 1.5, 0.2, **kw)


@pytest.mark.parametrize("dims", [1, 2, 3])
@pytest.mark.parametrize("m", [1.5, 4.75])
def test_juttner_invcdf_matches_host(lmb, dims, m):
    e = _engine(lmb)
    e.build_juttner_invcdf(m, dims, Tmin=0.12, Tmax=0.55)
    vals, nU, nT, t0, inv = e.get_invcdf()
    hv, hnU, hnT, ht0, hinv = lmb.transport.build_juttner_invcdf(m, dims, Tmin=0.12, Tmax=0.55)
    assert (nU, nT) == (hnU, hnT) and t0 == ht0 and inv == pytest.approx(hinv, rel=1e-15)
    # the CDF is summed in another order (a block scan): entries agree to ~1e-15 except
    # where the inverse is steep (the tails), and never by more than one momentum step
    d = np.abs(vals - hv)
    assert np.mean(d <= 1e-12 * np.maximum(hv, 1.0)) > 0.999
    pmax = 16.0 * np.sqrt(m * 0.6) + 16.0 * 0.6
    assert np.max(d) <= pmax / 8191 * 1.0001


def test_run_on_device_tables_matches_oracle(lmb, orc):
    """FP64 RTA in a static box: the engine on device-built tables, the oracle on the
    host's.  The tables differ by the order of the CDF sums only: the runs agree to 1e-12
    for 99 % of the particles and to 1e-9 for those resampled in the steep tails of the
    inverse CDF."""
    capi, tr = lmb.capi, lmb.transport
    xg, tg, Tf, Vf = box_medium(0.3, 0.0, 1.0)
    rng = np.random.default_rng(4)
    n = 4000
    x0, p0 = rng.normal(0, 2, (2, n)), rng.normal(0, 1.5, (3, n))
    e = capi.Engine(0)
    e.set_params(dims=2, pdim=3, dt=0.01, m=1.5, DsT=0.3, Tfo=0.0, collision=capi.LIM_COLL_RTA, seed=1)
    e.set_medium_rt(xg, tg, Tf, Vf)
    Tmin, Tmax = tr.spline_range(Tf)
    e.build_time_spline(capi.LIM_SPLINE_DRAG, capi.LIM_TIME_DRAG, 1.5, 0.3, Tmin=Tmin, Tmax=Tmax, nT=1024)
    e.build_time_spline(capi.LIM_SPLINE_RTA, capi.LIM_TIME_TAUN, 1.5, 0.3, Tmin=Tmin, Tmax=Tmax, nT=1024)
    e.build_juttner_invcdf(1.5, 3, Tmin=Tmin, Tmax=Tmax)
    e.upload_state(x0, p0)
    e.initial_lab_boost()
    e.run(1, 100)
    x, p = e.download_state()
    _, mh, xh, _ = oracle_drive(orc, xgrid=xg, tgrid=tg, Tf=Tf, Vf=Vf, x0=x0, p0=p0, M=1.5, DsT=0.3, dt=0.01, t0=0.0,
                                tfinal=1.0, save=1.0, dims=2, pdim=3, seed=1, collision=1)
    for a, b, sc in ((p, mh[-1], 0.3), (x, xh[-1], 1.0)):
        emax, e99 = parity(a, b, sc)
        assert e99 <= 1e-12 and emax <= 1e-9, (emax, e99)


def test_simulate_with_device_tables(lmb):
    """simulate_ensemble_bulk(..., tables="device") follows the host-table run."""
    xg, tg, Tf, Vf = box_medium(0.3, 0.0, 1.0)
    Tf = Tf * (1.0 + 0.3 * np.exp(-xg[:, None] ** 2 / 20.0))
    rng = np.random.default_rng(8)
    n = 3000
    kw = dict(N_particles=n, Δt=0.01, initial_time=0.0, final_time=0.5, save_interval=0.5, m=1.5, DsT=0.25,
              dimensions=2, momentum_dimensions=3, Tfo=0.0, seed=5, collision_mode=":langevin_rta",
              x_init=rng.normal(0, 3, (2, n)), p_init=rng.normal(0, 1, (3, n)))
    args = (lmb.B200Backend(), xg, np.linspace(0, 10, 10), np.ones((xg.size, 10)), Tf, Vf, (xg, tg))
    _, mh, xh = lmb.simulate_ensemble_bulk(*args, tables="host", **kw)
    _, md, xd = lmb.simulate_ensemble_bulk(*args, tables="device", **kw)
    emax, e99 = parity(md[-1], mh[-1], 0.3)
    assert e99 <= 1e-12 and emax <= 1e-9, (emax, e99)
