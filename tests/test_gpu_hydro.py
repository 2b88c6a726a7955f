"""Runs on ingested hydro backgrounds: an (r, tau) evolution (non-uniform tau nodes)
through simulate_ensemble_bulk against the oracle, and a 2+1D grid medium built by
HydroXY.grid_medium against the same fields handed to the engine directly."""
import numpy as np
import pytest

from helpers import oracle_drive, parity
from test_hydro import rt_case, xy_case

pytestmark = pytest.mark.gpu


def test_rt_hydro_run_matches_oracle(lmb, orc):
    h = rt_case()
    T, V, grid = h.evolution()
    rng = np.random.default_rng(2)
    n = 3000
    x0, p0 = rng.normal(0, 3, (2, n)), rng.normal(0, 1, (3, n))
    kw = dict(N_particles=n, Δt=0.01, initial_time=0.4, final_time=1.4, save_interval=1.0, m=1.5, DsT=0.3,
              dimensions=2, momentum_dimensions=3, Tfo=0.0, seed=9, x_init=x0, p_init=p0)
    _, mom, pos = lmb.simulate_ensemble_bulk(lmb.B200Backend(), h.r, np.linspace(0, 10, 10), np.ones((h.r.size, 10)),
                                             T, V, grid, **kw)
    _, mh, xh, _ = oracle_drive(orc, xgrid=h.r, tgrid=h.tau, Tf=T, Vf=V, x0=x0, p0=p0, M=1.5, DsT=0.3, dt=0.01,
                                t0=0.4, tfinal=1.0, save=1.0, dims=2, pdim=3, seed=9)
    assert parity(mom[-1], mh[-1], 0.3)[0] <= 1e-12
    assert parity(pos[-1], xh[-1], 1.0)[0] <= 1e-12


def test_xy_hydro_grid_medium_is_the_direct_one(lmb):
    capi, tr = lmb.capi, lmb.transport
    h = xy_case()
    g = h.grid_medium()
    vx, vy = h.velocity()
    rng = np.random.default_rng(3)
    n = 5000
    x0, p0 = rng.uniform(-6, 6, (2, n)), rng.normal(0, 1, (3, n))
    out = []
    for direct in (False, True):
        e = capi.Engine(0)
        e.set_params(dims=2, pdim=3, dt=0.01, t0=0.6, m=1.5, DsT=0.3, Tfo=0.0, seed=4, precision=capi.LIM_FP32)
        if direct:
            e.set_medium_grid(h.T.astype(np.float32), vx.astype(np.float32), vy.astype(np.float32), -8.0, 0.5, -7.0,
                              0.5, 0.6, 0.4)
        else:
            e.set_medium_grid(**g)
        Tmin, Tmax = tr.spline_range(h.T)
        e.set_spline(capi.LIM_SPLINE_DRAG, *tr.build_tau_drag_spline(1.5, 0.3, Tmin=Tmin, Tmax=Tmax, nT=1024))
        e.upload_state(x0, p0)
        e.initial_lab_boost()
        e.run(1, 150)
        out.append(e.download_state())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
