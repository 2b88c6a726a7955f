"""The method behind the device-built transport tables, checked on the host: the
trapezoidal rule for e^z K_nu(z) = int_0^inf exp(-z (cosh t - 1)) cosh(nu t) dt with the
step and stopping rule of lim_tables.cu agrees with scipy's kve (the function that
transport.py's tau_n_main3 uses, Bessels.besselkx in transport.jl:58-104) to 1e-15
relative over the temperatures and masses the tables cover and far beyond."""
import math

import numpy as np
import pytest
from scipy import special


def besselkx_trapezoid(nu, z):
    h = min(0.125, 0.5 / math.sqrt(z))
    s = 0.5
    for k in range(1, 100000):
        t = k * h
        sh = math.sinh(0.5 * t)
        c = z * (2.0 * sh * sh)
        e = c - nu * t
        if e > 745.0:
            break
        term = math.exp(-c) * math.cosh(nu * t)
        s += term
        if e > 40.0 and term < 1e-18 * s:
            break
    return s * h


@pytest.mark.parametrize("nu", [1, 2, 3, 5])
def test_trapezoid_besselkx_matches_scipy(nu):
    zs = np.concatenate([np.geomspace(1e-3, 1e6, 80), [1.5 / 0.6, 1.5 / 0.155, 4.75 / 0.1, 50.0]])
    err = max(abs(besselkx_trapezoid(nu, z) / special.kve(nu, z) - 1.0) for z in zs)
    assert err < 2e-15
