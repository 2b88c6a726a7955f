"""The engine's pathwise gradients (lim_adjoint) as a torch.autograd.Function.

``pathwise_observables(theta, run)`` returns the three final-state observables of a
configured run — <pT>, <cos 2 phi> and the fraction above ``obs_pt_cut`` smoothed with
a logistic of width ``obs_pt_width`` — as a differentiable function of
theta = (a, b, s): 2 pi T D_s = a + b (max(T, Tc)/Tc - 1) (the reference's linear
``effective_DsT`` form, transport.jl:139-156, with Tfo = Tc) and the medium temperature
scale s.  The forward pass runs the checkpointed forward and the hand-written reverse
sweep once; backward contracts the incoming cotangent with the 3 x 3 Jacobian it
returned.  The noise (counter-based, keyed by seed, particle and step) and the RTA
collision indicators of the forward pass are held fixed, so the gradient is the
pathwise derivative of the sampled ensemble.  The Julia counterpart is the
ChainRulesCore rule in julia/ext/LangevInB200ChainRulesExt.jl.
"""
from __future__ import annotations

import numpy as np
import torch

from . import capi
from . import transport as tr


class AdjointRun:
    """A configured engine context (parameters, medium, RTA spline, inverse CDF and an
    initial state, already boosted to the lab) for repeated gradient evaluations.  The
    initial state is saved on the device at construction; every evaluation installs the
    drag spline of (a, b) with its derivative tables and the scale s, restores that
    state and runs lim_adjoint over steps [first_step, first_step + nsteps)."""

    def __init__(self, engine: capi.Engine, *, m: float, Tmin: float, Tmax: float, first_step: int, nsteps: int,
                 checkpoint_every: int = 64, Tc: float = 0.155, nT: int = 1024):
        self.engine = engine
        self.m, self.Tmin, self.Tmax, self.Tc, self.nT = float(m), float(Tmin), float(Tmax), float(Tc), int(nT)
        self.first_step, self.nsteps, self.K = int(first_step), int(nsteps), int(checkpoint_every)
        engine.state_save()

    def evaluate(self, theta) -> tuple[np.ndarray, np.ndarray]:
        """(obs[3], d obs / d theta [3, 3]) at theta = (a, b, s)."""
        a, b, s = (float(v) for v in np.asarray(theta, dtype=np.float64).reshape(3))
        Tm, inv, vals, d_da, d_db = tr.build_drag_spline_ab(self.m, a, b, Tc=self.Tc, Tmin=self.Tmin, Tmax=self.Tmax,
                                                            nT=self.nT)
        e = self.engine
        e.set_spline(capi.LIM_SPLINE_DRAG, Tm, inv, vals)
        e.set_spline(capi.LIM_SPLINE_DRAG_DA, Tm, inv, d_da)
        e.set_spline(capi.LIM_SPLINE_DRAG_DB, Tm, inv, d_db)
        e.set_medium_scale(s)
        e.state_restore()
        return e.adjoint(self.first_step, self.nsteps, self.K)


class PathwiseObservables(torch.autograd.Function):
    """y = obs(theta); backward: theta_bar = y_bar @ (d obs / d theta)."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, run: AdjointRun) -> torch.Tensor:
        obs, jac = run.evaluate(theta.detach().cpu().numpy())
        ctx.save_for_backward(torch.as_tensor(jac, dtype=theta.dtype, device=theta.device))
        return torch.as_tensor(obs, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, y_bar: torch.Tensor):
        (jac,) = ctx.saved_tensors
        return y_bar @ jac, None


def pathwise_observables(theta: torch.Tensor, run: AdjointRun) -> torch.Tensor:
    """Differentiable (<pT>, <cos 2 phi>, smoothed fraction above the cut) of theta = (a, b, s)."""
    return PathwiseObservables.apply(theta, run)
