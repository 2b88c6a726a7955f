"""The torch.autograd bridge of the pathwise gradients: backward returns the incoming
cotangent contracted with the Jacobian of a direct lim_adjoint call on an identically
configured context, and repeated evaluations are deterministic."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _run(lmb, f, N=20000, steps=120):
    AD = importlib.import_module(lmb.__name__ + ".autodiff")
    wl = lmb.workloads.adjoint_grid(N=N, steps=steps, fields=f, dt=0.02)
    e = lmb.capi.Engine(0)
    lmb.workloads.configure(e, wl)
    e.initial_lab_boost()
    Tmin, Tmax = lmb.transport.spline_range(f["T"])
    return AD, wl, e, AD.AdjointRun(e, m=1.5, Tmin=Tmin, Tmax=Tmax, first_step=1, nsteps=steps)


def test_autograd_backward_is_the_adjoint_jacobian(lmb):
    f = lmb.workloads.grid2p1_fields(nx=81, ny=61, nt=24, dx=0.25)
    AD, wl, e, run = _run(lmb, f)
    theta = torch.tensor([3.0, 2.0, 1.0], dtype=torch.float64, requires_grad=True)
    y = AD.pathwise_observables(theta, run)
    w = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float64)
    (y * w).sum().backward()
    # the same run through the C-ABI directly, on a fresh context
    _, wl2, e2, _ = _run(lmb, f)
    obs, G = e2.adjoint(1, wl2.steps, 64)
    assert np.array_equal(y.detach().numpy(), obs)
    assert np.allclose(theta.grad.numpy(), w.numpy() @ G, rtol=1e-12, atol=0)
    # a second evaluation at the same theta repeats the first exactly
    y2 = AD.pathwise_observables(theta.detach(), run)
    assert np.array_equal(y2.numpy(), obs)
