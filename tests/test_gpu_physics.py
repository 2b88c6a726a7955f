"""The reference's physics tests run on the B200 engine through the public API
(`simulate_ensemble_bulk(B200Backend(), …)`, the drop-in for GPUBackend), in FP64
and FP32 — the analogue of the reference's GPU gate (test_momentum_dims3.jl:203-231),
which compares the GPU path to the CPU path on the same assertions."""
import math

import numpy as np
import pytest

import kat_cases as K
from helpers import K2K3, box_medium, est, oracle_drive

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["fp64", "fp32"])
def box_run(lmb, request):
    prec = request.param

    def run(*, M, T, DsT, N, dt, tfinal, save, x0, p0, pdim, t0=0.0, redshift=False, momentum_langevin=True,
            seed=1, relativistic=True):
        xg, tg, Tf, Vf = box_medium(T, t0, tfinal)
        dens = np.ones((xg.size, 10))       # unused: x_init/p_init bypass the sampler
        return lmb.simulate_ensemble_bulk(
            lmb.B200Backend(), xg, np.linspace(0, 10, 10), dens, Tf, Vf, (xg, tg), x_init=x0, p_init=p0,
            N_particles=N, Δt=dt, initial_time=t0, final_time=t0 + tfinal, save_interval=save, m=M, DsT=DsT,
            dimensions=2, momentum_dimensions=pdim, bjorken_redshift=redshift, position_diffusion=False,
            momentum_langevin=momentum_langevin, reflecting_boundary=False, Tfo=0.0, relativistic=relativistic,
            seed=seed, precision=prec)
    run.precision = prec
    return run


def test_equilibria(box_run):
    K.case_equilibria(box_run)


def test_l1_decay(box_run):
    K.case_l1_decay(box_run, N_D=400_000)


def test_bjorken_redshift_telescopes(box_run):
    K.case_bjorken_redshift(box_run)


def test_msd_diffusion_coefficient(box_run):
    K.case_msd(box_run)


def test_relativistic_switch(box_run):
    K.case_relativistic_switch(box_run)


def test_gpu_agrees_with_cpu_restatement(box_run, orc):
    """test_momentum_dims3.jl:203-231: the GPU ensemble agrees with the CPU one."""
    N, dt, tf = 150_000, 2e-3, 4.0
    rng = np.random.default_rng(11)
    x0 = np.zeros((2, N))
    p0 = 0.9 * rng.standard_normal((3, N))
    _, mg, _ = box_run(M=K.M_, T=K.T_, DsT=K.DST_, N=N, dt=dt, tfinal=tf, save=0.5, x0=x0, p0=p0, pdim=3)
    xg, tg, Tf, Vf = box_medium(K.T_, 0.0, tf)
    _, mc, _, _ = oracle_drive(orc, xgrid=xg, tgrid=tg, Tf=Tf, Vf=Vf, x0=x0, p0=p0, M=K.M_, DsT=K.DST_, dt=dt,
                               t0=0.0, tfinal=tf, save=0.5, dims=2, pdim=3, seed=1)
    eg, ec = est(mg[-1], K.M_), est(mc[-1], K.M_)
    assert mg[-1].shape[0] == 3
    assert math.isclose(eg["p2"], ec["p2"], rel_tol=0.02)
    assert math.isclose(eg["lam"], K2K3(K.M_ / K.T_), rel_tol=0.005)
    assert math.isclose(np.mean(mg[-1][2] ** 2), np.mean(mg[-1][0] ** 2), rel_tol=0.02)
    if box_run.precision == "fp64":
        # same seed, same noise: FP64 agrees particle by particle, not only in the ensemble
        e = np.linalg.norm(mg[-1] - mc[-1], axis=0) / np.maximum(np.linalg.norm(mc[-1], axis=0), 3e-4)
        assert e.max() <= 1e-12
