"""Snapshot reductions on the device (lim_reduce_state, lim_run_reduced) against a
numpy restatement applied to the engine's own downloaded state and history: counts and
the fixed-point cos 2 phi sums agree exactly, the observable sums to FP64 rounding."""
import numpy as np
import pytest

from helpers import box_medium

pytestmark = pytest.mark.gpu

SPEC = (64, 16.0, 50, 5.0)


def reduce_np(x, p, spec, milne=False):
    """The reduction restated: bins floor(v * (bins / max)), overflow last."""
    r_bins, r_max, pt_bins, pt_max = spec
    x = np.asarray(x, dtype=np.float64)
    p = np.asarray(p, dtype=np.float64)
    if milne:
        r, pt, c2 = x[1], np.abs(p[1]), np.zeros(x.shape[1])
    else:
        r2 = np.zeros(x.shape[1])
        for d in range(x.shape[0]):
            r2 = r2 + x[d] * x[d]
        r = np.sqrt(r2)
        px, py = p[0], (p[1] if p.shape[0] >= 2 else np.zeros_like(p[0]))
        px2, py2 = px * px, py * py
        pt2 = px2 + py2
        pt = np.sqrt(pt2)
        with np.errstate(invalid="ignore", divide="ignore"):
            c2 = np.where(pt2 > 0, (px2 - py2) / pt2, 0.0)

    def bins(v, nb, vmax):
        f = np.floor(v * (nb / vmax))
        return np.where((f >= 0) & (f < nb), f, nb).astype(np.int64)

    kr, kp = bins(r, r_bins, r_max), bins(pt, pt_bins, pt_max)
    rc = np.bincount(kr, minlength=r_bins + 1).astype(np.float64)
    pc = np.bincount(kp, minlength=pt_bins + 1).astype(np.float64)
    fixed = np.rint(c2 * 2.0 ** 32).astype(np.int64)
    cs = np.zeros(pt_bins + 1, dtype=np.int64)
    np.add.at(cs, kp, fixed)
    return rc, pc, cs.astype(np.float64) * 2.0 ** -32


def _engine(lmb, prec, pdim=3, coll=None):
    capi = lmb.capi
    xg, tg, Tf, Vf = box_medium(0.3, 0.0, 2.0)
    Vf = 0.4 * np.tanh(0.05 * xg)[:, None] * np.ones_like(tg)[None, :]
    e = capi.Engine(0)
    e.set_params(dims=2, pdim=pdim, coords=capi.LIM_COORDS_CARTESIAN, dt=0.01, m=1.5, DsT=0.3,
                 collision=capi.LIM_COLL_LANGEVIN if coll is None else coll, Tfo=0.0, seed=77,
                 precision=capi.LIM_FP32 if prec == "fp32" else capi.LIM_FP64)
    e.set_medium_rt(xg, tg, Tf, Vf)
    Tmin, Tmax = lmb.transport.spline_range(Tf)
    t0_, inv_, vals = lmb.transport.build_tau_drag_spline(1.5, 0.3, Tmin=Tmin, Tmax=Tmax, nT=1024)
    e.set_spline(capi.LIM_SPLINE_DRAG, t0_, inv_, vals)
    rng = np.random.default_rng(5)
    n = 30_001
    e.upload_state(rng.normal(0, 4.0, (2, n)), rng.normal(0, 1.5, (pdim, n)))
    e.initial_lab_boost()
    return e, n


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_reduce_state_matches_numpy(lmb, prec):
    e, n = _engine(lmb, prec)
    spec = lmb.capi.reduce_spec(*SPEC)
    red = e.reduce_state(spec)
    x, p = e.download_state()
    rc, pc, cs = reduce_np(x, p, SPEC)
    assert np.array_equal(red["r_counts"], rc) and np.array_equal(red["pt_counts"], pc)
    assert np.array_equal(red["pt_cos2"], cs)
    assert red["r_counts"].sum() == n and red["pt_counts"].sum() == n
    ref = e.observables()
    assert red["obs"][0] == n
    assert np.allclose(red["obs"][1] / n, ref["mean_pt"], rtol=1e-12)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_run_reduced_matches_history(lmb, prec):
    """Snapshots reduced on the device equal the numpy reduction of lim_run's history
    from the same start (the runs are deterministic)."""
    e, n = _engine(lmb, prec)
    e.state_save()
    steps, save, nslots = 60, 20, 3
    hx = np.zeros(nslots * n * 2)
    hp = np.zeros(nslots * n * 3)
    e.run(1, steps, save, 1, hx, hp)
    e.state_restore()
    spec = lmb.capi.reduce_spec(*SPEC)
    red = e.run_reduced(1, steps, save, 1, nslots, spec)
    for k in range(nslots):
        x = hx[k * n * 2:(k + 1) * n * 2].reshape(n, 2).T
        p = hp[k * n * 3:(k + 1) * n * 3].reshape(n, 3).T
        rc, pc, cs = reduce_np(x, p, SPEC)
        assert np.array_equal(red["r_counts"][k], rc), k
        assert np.array_equal(red["pt_counts"][k], pc), k
        assert np.array_equal(red["pt_cos2"][k], cs), k
        pt = np.hypot(p[0], p[1])
        assert red["obs"][k][1] == pytest.approx(pt.sum(), rel=1e-12)


def test_reduce_milne_and_errors(lmb):
    capi = lmb.capi
    e = capi.Engine(0)
    e.set_params(dims=2, pdim=2, coords=capi.LIM_COORDS_MILNE, t0=0.4, m=1.5, dt=0.01, DsT=0.0)
    xg, tg, Tf, Vf = box_medium(0.3, 0.4, 2.0)
    e.set_medium_rt(xg, tg, Tf, Vf)
    rng = np.random.default_rng(9)
    n = 5000
    x = np.vstack([np.full(n, 0.4), rng.uniform(0, 12, n)])
    pr = rng.normal(0, 1, n)
    e.upload_state(x, np.vstack([np.sqrt(1.5 ** 2 + pr ** 2), pr]))
    red = e.reduce_state(capi.reduce_spec(*SPEC))
    rc, pc, cs = reduce_np(x, np.vstack([np.sqrt(1.5 ** 2 + pr ** 2), pr]), SPEC, milne=True)
    assert np.array_equal(red["r_counts"], rc) and np.array_equal(red["pt_counts"], pc)
    assert np.all(red["pt_cos2"] == 0)
    for bad in ((0, 16.0, 50, 5.0), (64, 0.0, 50, 5.0), (64, 16.0, 5000, 5.0), (64, np.inf, 50, 5.0)):
        with pytest.raises(RuntimeError, match="lim_reduce_spec"):
            e.reduce_state(capi.reduce_spec(*bad))


def test_simulate_with_snapshot_reduce(lmb):
    xg, tg, Tf, Vf = box_medium(0.3, 0.0, 2.0)
    rng = np.random.default_rng(3)
    n = 4000
    x0, p0 = rng.normal(0, 3, (2, n)), rng.normal(0, 1, (2, n))
    kw = dict(N_particles=n, Δt=0.01, initial_time=0.0, final_time=0.5, save_interval=0.1, m=1.5, DsT=0.3,
              dimensions=2, Tfo=0.0, seed=11, x_init=x0, p_init=p0)
    t, mom, pos = lmb.simulate_ensemble_bulk(lmb.B200Backend(), xg, np.linspace(0, 10, 10), np.ones((xg.size, 10)),
                                             Tf, Vf, (xg, tg), **kw)
    t2, red = lmb.simulate_ensemble_bulk(lmb.B200Backend(), xg, np.linspace(0, 10, 10), np.ones((xg.size, 10)),
                                         Tf, Vf, (xg, tg), snapshot_reduce=SPEC, **kw)
    assert np.allclose(t, t2) and red["r_counts"].shape == (len(mom), SPEC[0] + 1)
    for k in range(len(mom)):
        rc, pc, cs = reduce_np(pos[k], mom[k], SPEC)
        assert np.array_equal(red["r_counts"][k], rc) and np.array_equal(red["pt_counts"][k], pc)
        assert np.array_equal(red["pt_cos2"][k], cs)


def test_history_in_pinned_memory(lmb):
    """lim_run's snapshot copies into page-locked buffers (lim_host_alloc) give the same
    history as into pageable ones."""
    xg, tg, Tf, Vf = box_medium(0.3, 0.0, 2.0)
    rng = np.random.default_rng(6)
    n = 5000
    kw = dict(N_particles=n, Δt=0.01, initial_time=0.0, final_time=0.6, save_interval=0.1, m=1.5, DsT=0.3,
              dimensions=2, Tfo=0.0, seed=12, x_init=rng.normal(0, 3, (2, n)), p_init=rng.normal(0, 1, (2, n)))
    args = (lmb.B200Backend(), xg, np.linspace(0, 10, 10), np.ones((xg.size, 10)), Tf, Vf, (xg, tg))
    _, m0, x0 = lmb.simulate_ensemble_bulk(*args, **kw)
    _, m1, x1 = lmb.simulate_ensemble_bulk(*args, pinned_history=True, **kw)
    assert len(m0) == 7 and all(np.array_equal(a, b) for a, b in zip(m0, m1))
    assert all(np.array_equal(a, b) for a, b in zip(x0, x1))
    buf = lmb.capi.pinned_empty(10)
    buf[:] = np.arange(10)
    assert buf.sum() == 45 and lmb.capi.pinned_empty(0).size == 0
