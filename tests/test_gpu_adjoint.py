"""Pathwise gradients (lim_adjoint): the hand-written reverse sweep with checkpoints
against central finite differences (h = 1e-3) taken with common random numbers and
the RTA indicators held fixed — on the engine (FP64 runs replaying the adjoint run's
RTA decisions) and on the CPU restatement of the reference's step (fed the recorded
variates).  Observables: <pT>, <cos 2 phi> and the fraction above 5 GeV smoothed with
a 0.1 GeV logistic; parameters: (a, b) of 2 pi T D_s = a + b (T/0.155 - 1) and the
medium temperature scale s."""
import numpy as np
import pytest

from helpers import oracle_medium, oracle_params

pytestmark = pytest.mark.gpu

H = 1e-3
THETA = (3.0, 2.0, 1.0)


def fields(lmb):
    return lmb.workloads.grid2p1_fields(nx=81, ny=61, nt=24, dx=0.25)


def workload(lmb, f, theta, N, steps, prec="fp32"):
    a, b, s = theta
    return lmb.workloads.adjoint_grid(N=N, steps=steps, fields=f, a=a, b=b, scale=s, precision=prec, dt=0.02)


def observables(p, cut=5.0, width=0.1):
    px, py = p[0], p[1]
    pt2 = px * px + py * py
    pt = np.sqrt(pt2)
    c2 = np.where(pt2 > 0, (px * px - py * py) / np.where(pt2 > 0, pt2, 1.0), 0.0)
    return np.array([pt.mean(), c2.mean(), (1.0 / (1.0 + np.exp(-(pt - cut) / width))).mean()])


def engine(lmb, wl):
    e = lmb.capi.Engine(0)
    lmb.workloads.configure(e, wl)
    e.initial_lab_boost()
    return e


def compare(tag, G, FD, FD2, obs):
    """The adjoint against central differences at h and h/2.  The interpolated medium,
    transport spline and inverse CDF are piecewise linear: a difference quotient whose
    interval straddles a node is off by a share of the slope jump, an error that grows
    with h, so the reference value is the Richardson combination 2 FD(h/2) - FD(h) and
    the finite-difference error is estimated by |FD(h) - FD(h/2)|.  Errors relative to
    max(|FD|, 1e-3 |obs|); returns (error vs FD(h), error vs the extrapolation, FD error)."""
    scale = np.maximum(np.abs(FD), 1e-3 * np.abs(obs)[:, None])
    err_h = np.abs(G - FD) / scale
    err = np.abs(G - (2 * FD2 - FD)) / scale
    fd_err = np.abs(FD - FD2) / scale
    print(f"{tag}: adjoint\n{G}\nFD (h = {H})\n{FD}\nFD (h = {H / 2})\n{FD2}\n"
          f"rel err vs FD(h)\n{np.array2string(err_h, precision=2)}\n"
          f"rel err vs 2 FD(h/2) - FD(h)\n{np.array2string(err, precision=2)}\n"
          f"FD error estimate\n{np.array2string(fd_err, precision=2)}")
    return err_h, err, fd_err


def central_differences(run_at, hs=(H, H / 2)):
    """run_at(theta) -> observables; central differences in each parameter at each h."""
    out = []
    for h in hs:
        FD = np.zeros((3, 3))
        for k in range(3):
            vals = []
            for sgn in (1, -1):
                th = list(THETA)
                th[k] += sgn * h
                vals.append(run_at(th))
            FD[:, k] = (vals[0] - vals[1]) / (2 * h)
        out.append(FD)
    return out


def test_adjoint_matches_engine_finite_differences(lmb):
    """The FD runs are FP64 engine runs with their own (FP64) variates, so their paths
    differ from the FP32 adjoint run's by FP32 rounding; a particle ending near p_T = 0
    (where d cos 2 phi / dp ~ 1/p_T) or on the steep part of the smoothed p_T cut turns
    that into a gradient difference of order 1/N, hence the large ensemble.  The
    restatement test below feeds the identical variates and needs no such margin."""
    f = fields(lmb)
    N, steps = 200_000, 240
    base = engine(lmb, workload(lmb, f, THETA, N, steps))
    obs, G = base.adjoint(1, steps, checkpoint_every=64)
    fwd_ms, rev_ms = base.adjoint_stats()
    assert fwd_ms > 0 and rev_ms > 0
    # the adjoint advanced the state exactly like a plain run
    x_adj, p_adj = base.download_state()
    assert np.allclose(observables(p_adj), obs, rtol=1e-12, atol=1e-15)

    def run_at(th):
        e = engine(lmb, workload(lmb, f, th, N, steps, prec="fp64"))
        e.copy_rta_decisions(base)
        e.run(1, steps)
        o = observables(e.download_state()[1])
        e.close()
        return o

    FD, FD2 = central_differences(run_at)
    err_h, err, fd_err = compare("engine FD (fp64, fixed RTA)", G, FD, FD2, obs)
    assert np.all(err <= 1e-3 + 2 * fd_err)


def test_adjoint_checkpoint_interval_does_not_change_gradients(lmb):
    f = fields(lmb)
    res = []
    for K in (1, 16, 64, 1000):
        e = engine(lmb, workload(lmb, f, THETA, 4000, 130))
        res.append(e.adjoint(1, 130, checkpoint_every=K))
        e.close()
    for obs, G in res[1:]:
        assert np.array_equal(obs, res[0][0])
        assert np.allclose(G, res[0][1], rtol=1e-6, atol=1e-9)


def test_adjoint_matches_restatement_finite_differences(lmb, orc):
    """Finite differences of the CPU path (the reference's step restated in FP64), fed
    the variates the engine consumed and its RTA decisions."""
    f = fields(lmb)
    N, steps = 20000, 160
    wl = workload(lmb, f, THETA, N, steps)
    e = engine(lmb, wl)
    x0, p0 = e.download_state()
    e.state_save()
    e.record_noise(1, steps)
    e.run(1, steps)
    rec = e.download_noise()
    e.record_noise(1, 0)
    e.state_restore()
    obs, G = e.adjoint(1, steps, checkpoint_every=32)

    def run_at(th):
        w = workload(lmb, f, th, N, steps, prec="fp64")
        P = oracle_params(orc, w, rta_replay=1)
        md = oracle_medium(orc, w)
        return observables(orc.run(P, md, x0, p0, 1, steps, rec=rec)["p"])

    FD, FD2 = central_differences(run_at)
    err_h, err, fd_err = compare("restatement FD (fixed noise and RTA)", G, FD, FD2, obs)
    assert np.all(err <= 1e-3 + 2 * fd_err)


def test_adjoint_validation(lmb):
    capi = lmb.capi
    wl = lmb.workloads.bjorken(N=256, precision="fp64", steps=10)
    e = capi.Engine(0)
    lmb.workloads.configure(e, wl)
    with pytest.raises(capi.LimError, match="FP32"):
        e.adjoint(1, 10)
    wl = lmb.workloads.bjorken(N=256, precision="fp32", steps=10, table=False)
    lmb.workloads.configure(e, wl)
    with pytest.raises(capi.LimError, match="LIM_SPLINE_DRAG_DA"):
        e.adjoint(1, 10)
