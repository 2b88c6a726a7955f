"""The reference's dynamical known-answer tests on the CPU restatement (the oracle):
this pins the oracle to the reference's own assertions before it is used to check
the CUDA engine.  CPU only (OpenMP)."""
import math

import numpy as np
import pytest
from scipy import integrate

import kat_cases as K
from helpers import K2K3, box_medium, lam1, oracle_drive


@pytest.fixture(scope="module")
def box_run(orc):
    def run(*, M, T, DsT, N, dt, tfinal, save, x0, p0, pdim, t0=0.0, redshift=False, momentum_langevin=True,
            seed=1, relativistic=True):
        xg, tg, Tf, Vf = box_medium(T, t0, tfinal)
        tt, mh, xh, _ = oracle_drive(orc, xgrid=xg, tgrid=tg, Tf=Tf, Vf=Vf, x0=x0, p0=p0, M=M, DsT=DsT, dt=dt,
                                     t0=t0, tfinal=tfinal, save=save, dims=2, pdim=pdim, redshift=redshift,
                                     momentum_langevin=momentum_langevin, relativistic=relativistic, seed=seed)
        return tt, mh, xh
    return run


def test_lambda1_identity_quadrature():
    """(Q) test_momentum_dims3.jl:87-96."""
    for z in (3.48, 5.0, 7.0, 9.62):
        T = K.M_ / z
        assert math.isclose(lam1(K.M_, T, 3), K2K3(z), rel_tol=1e-9)
        assert 1.04 < lam1(K.M_, T, 2) / lam1(K.M_, T, 3) < 1.13


def test_pz_conditional_sampler(lmb):
    """(S) test_momentum_dims3.jl:98-117."""
    from helpers import juttner_sample
    U = lmb.utils
    rng = np.random.default_rng(7)
    for mT, T in ((1.6, 0.3), (2.5, 0.45), (1.5, 0.156)):
        s = U.sample_pz_conditional_juttner(np.full(200_000, mT), np.full(200_000, T), rng)
        w = lambda pz: math.exp(-(math.sqrt(mT * mT + pz * pz) - mT) / T)
        num = integrate.quad(lambda pz: pz * pz * w(pz), -np.inf, np.inf, epsrel=1e-10)[0]
        den = integrate.quad(w, -np.inf, np.inf, epsrel=1e-10)[0]
        assert math.isclose(np.mean(s ** 2), num / den, rel_tol=0.02)
        assert abs(np.mean(s)) < 4 * np.std(s) / math.sqrt(s.size)
    P3 = juttner_sample(rng, K.M_, K.T_, 3, 200_000)
    x = np.zeros((2, P3.shape[1]))
    P = U.append_thermal_pz(P3[:2], x, K.M_, lambda r: K.T_, rng=rng)
    assert math.isclose(np.mean(P[2] ** 2), np.mean(P3[0] ** 2), rel_tol=0.02)
    assert math.isclose(np.mean(P[2] ** 2), np.mean(P[0] ** 2), rel_tol=0.02)
    Pa = U.append_thermal_pz(P3[:2, :1000], x[:, :1000], K.M_, lambda r: K.T_, antithetic=True, rng=rng)
    assert np.all(Pa[2, 1::2] == -Pa[2, 0:-1:2])


def test_check_momentum_dims(lmb):
    """(R) test_momentum_dims3.jl:185-187: the contract refuses the meaningless combinations."""
    U = lmb.utils
    for args in ((2, 3, False, True, 0.0), (2, 4, False, False, 0.4), (3, 2, False, False, 0.4)):
        with pytest.raises(ValueError):
            U.check_momentum_dims(*args)
    U.check_momentum_dims(2, 3, False, True, 0.4)


def test_equilibria(box_run):
    K.case_equilibria(box_run)


def test_l1_decay(box_run):
    K.case_l1_decay(box_run)


def test_bjorken_redshift_telescopes(box_run):
    K.case_bjorken_redshift(box_run)


def test_msd_diffusion_coefficient(box_run):
    K.case_msd(box_run)


def test_relativistic_switch(box_run):
    K.case_relativistic_switch(box_run)
