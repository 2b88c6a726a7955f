"""Host side of the static-temperature path: the momentum-only initial sampler of
utils.jl:419-465, and the CPU restatement of the legacy loop (simulate_cpu.jl:325-404)
relaxing to its stationary <p^2> (the Euler scheme's d m T / (1 - eta dt / 2))."""
import numpy as np
import pytest


def test_initial_momenta_delta_and_bimodal(lmb):
    u = lmb.utils
    rng = np.random.default_rng(3)
    p = u.sample_initial_particles_at_origin_no_position("delta", 2.5, 3, 5000, rng)
    assert p.shape == (3, 5000) and np.allclose(np.linalg.norm(p, axis=0), 2.5)
    assert np.all(np.abs(p.mean(axis=1)) < 0.15)            # isotropic
    q = u.sample_initial_particles_at_origin_no_position("bimodal", 1.0, 2, 20000, rng)
    mags = np.linalg.norm(q, axis=0)
    assert q.shape == (2, 20000) and mags.min() >= 0.1 and mags.max() <= 5.0
    assert abs(np.mean(mags) - 1.5) < 0.02                 # equal mixture of 1 and 2 (sigma 0.2)
    with pytest.raises(ValueError, match="Unknown initial condition: ring"):
        u.sample_initial_particles_at_origin_no_position("ring", 1.0, 3, 10, rng)


def test_restatement_relaxes_to_the_scheme_equilibrium(orc):
    T, m, dt, dims, n = 0.4, 1.5, 0.01, 3, 20000
    P = orc.make_params(dt=dt, m=m, dims=dims, pdim=dims, seed=0x4C494D06)
    p0 = np.zeros((dims, n))
    p0[0] = 1.0
    p, hist = orc.run_static(P, T, p0, 1, 3000, save_every=1000, nslots=4)
    eta = 2.5 * T ** 3 / (2 * T * m)
    p2_eq = dims * m * T / (1 - eta * dt / 2)
    p2 = np.mean(np.sum(p ** 2, axis=0))
    assert abs(p2 / p2_eq - 1) < 0.03, (p2, p2_eq)
    assert np.allclose(hist[3], np.linalg.norm(p, axis=0))
