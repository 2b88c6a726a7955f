"""The static-temperature momentum-only path (simulate_ensemble_bulk(::CPUBackend,
T::Float64), simulate.jl:89-109 -> simulate_cpu.jl:325-404, legacy force
kernels_cpu.jl:359-404) against its CPU restatement on identical Philox noise,
per particle (FP64 gate 1e-12, FP32 1e-5, the parity metric of the other tests), with
the |p| history, and through the public entry point."""
import numpy as np
import pytest

from helpers import parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [1, 2, 3])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_static_T_matches_restatement(lmb, orc, dims, prec, tol):
    capi = lmb.capi
    rng = np.random.default_rng(100 + dims)
    n, steps, save, T, m, dt = 4096, 200, 50, 0.3, 1.5, 0.01
    p0 = rng.normal(0.0, 1.5, (dims, n))
    nslots = steps // save + 1
    eng = capi.Engine(0)
    eng.set_params(dt=dt, m=m, dims=dims, pdim=dims, seed=0x4C494D05,
                   precision=capi.LIM_FP32 if prec == "fp32" else capi.LIM_FP64)
    eng.upload_state(np.zeros((dims, n)), p0)
    hist = np.full((nslots, n), -1.0)
    eng.run_static_T(T, 1, steps, save, 0, hist)
    _, p = eng.download_state()
    eng.close()
    P = orc.make_params(dt=dt, m=m, dims=dims, pdim=dims, seed=0x4C494D05)
    po, ho = orc.run_static(P, T, p0, 1, steps, save_every=save, nslots=nslots)
    floor = 1e-2 if prec == "fp64" else 1.0
    ep = parity(p, po, 0.3, floor)
    eh = parity(hist[1:], ho[1:], 0.3, floor)
    print(f"static T dims={dims} {prec}: p max {ep[0]:.3g} p99 {ep[1]:.3g}; |p| history max {eh[0]:.3g}")
    assert ep[0] <= tol and eh[0] <= tol
    assert np.all(hist[0] == -1.0)                  # slot 0 is the caller's (the initial |p|)


def test_static_T_public_entry_point(lmb):
    """simulate_ensemble_bulk(B200Backend(), T; ...): the reference's keywords, defaults
    and return shape; the legacy model relaxes to <p^2> = d m T / (1 - eta dt / 2)."""
    T, m, dims = 0.4, 1.5, 3
    tp, hist = lmb.simulate_ensemble_bulk(lmb.B200Backend(), T, N_particles=40_000, Δt=0.01, final_time=30.0,
                                          save_interval=5.0, m=m, p0=1.0, dimensions=dims)
    assert len(tp) == len(hist) == 7 and tp[0] == 0.0 and tp[-1] == 30.0
    assert np.allclose(hist[0], 1.0)                 # "delta": |p| = p0
    eta = 2.5 * T ** 3 / (2 * T * m)
    p2_eq = dims * (2.5 * T ** 3) / (2 * eta) / (1 - eta * 0.01 / 2)
    p2 = np.mean(hist[-1] ** 2)
    print(f"<p^2> after 30 fm: {p2:.4f}, stationary value of the scheme {p2_eq:.4f}")
    assert abs(p2 / p2_eq - 1) < 0.03
    with pytest.raises(ValueError, match="Unknown initial condition: shell"):
        lmb.simulate_ensemble_bulk(lmb.B200Backend(), T, N_particles=10, initial_condition="shell")
