"""Hydrodynamic backgrounds for the engine: loaders and the conversions the reference's
drivers expect.

The reference ships its hydro background as ``src/data/Fluidum_MIS_HQ.jld2`` (a
FluiduM / Müller-Israel-Stewart (r, tau) evolution), which is absent from the project
and never loaded by its sources; its drivers take the fields directly:

* Cartesian backends: ``TemperatureEvolution`` and ``VelocityEvolution`` as
  (Nr, Nt) matrices on ``SpaceTimeGrid = (r, t)`` (simulate_cpu.jl:12-40), the velocity
  being the radial flow velocity v^r (kernels_cpu.jl:80,105);
* Milne backends: also the profile functions ``T_profile_MIS(r, tau)``,
  ``ur_profile_MIS(r, tau)`` (the radial four-velocity u^r) and ``mu_profile_MIS(r, tau)``
  (simulate_cpu_general_coords.jl:18-41).

:class:`HydroRT` holds an (r, tau) evolution and produces both forms; :class:`HydroXY`
holds a 2+1D (x, y, tau) evolution and produces the engine's grid medium
(``Engine.set_medium_grid``: T and the flow velocity on a uniform grid).  Both read
``.npz`` archives and raw column-major dumps (what Julia's ``write(io, A)`` produces for
an ``Array{Float64}``/``Array{Float32}``) described by a JSON header, so a JLD2 file can
be exported from Julia without further dependencies.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

EPS = float(np.finfo(np.float64).eps)


def _axis(a, name):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if a.size < 2:
        raise ValueError(f"{name}: need at least 2 nodes")
    if not np.all(np.isfinite(a)) or not np.all(np.diff(a) > 0):
        raise ValueError(f"{name}: nodes must be finite and strictly ascending")
    return a


def velocity_from_four(u):
    """v = u / sqrt(1 + u.u) for a spatial four-velocity u (one component, or stacked)."""
    u = np.asarray(u, dtype=np.float64)
    return u / np.sqrt(1.0 + u * u)


def interp2d_clamped(x, y, vals, xi, yi):
    """Vectorised clamped bilinear interpolation on an (Nx, Ny) table: the query is
    clamped to the grid, the cell is the last node <= the query (capped to the last
    cell), and a zero-width cell gives weight 0 (kernels_cpu.jl:22-51)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    v = np.asarray(vals, dtype=np.float64)
    xi = np.clip(np.asarray(xi, dtype=np.float64), x[0], x[-1])
    yi = np.clip(np.asarray(yi, dtype=np.float64), y[0], y[-1])
    i = np.clip(np.searchsorted(x, xi, side="right") - 1, 0, x.size - 2)
    j = np.clip(np.searchsorted(y, yi, side="right") - 1, 0, y.size - 2)
    dx, dy = x[i + 1] - x[i], y[j + 1] - y[j]
    with np.errstate(invalid="ignore", divide="ignore"):
        xd = np.where(np.abs(dx) < EPS, 0.0, (xi - x[i]) / dx)
        yd = np.where(np.abs(dy) < EPS, 0.0, (yi - y[j]) / dy)
    c0 = v[i, j] * (1 - xd) + v[i + 1, j] * xd
    c1 = v[i, j + 1] * (1 - xd) + v[i + 1, j + 1] * xd
    return c0 * (1 - yd) + c1 * yd


@dataclass
class HydroRT:
    """An (r, tau) evolution: T, the radial four-velocity u^r and mu on (Nr, Nt) nodes."""
    r: np.ndarray
    tau: np.ndarray
    T: np.ndarray
    ur: np.ndarray
    mu: np.ndarray | None = None

    def __post_init__(self):
        self.r = _axis(self.r, "r")
        self.tau = _axis(self.tau, "tau")
        shape = (self.r.size, self.tau.size)
        for name in ("T", "ur", "mu"):
            a = getattr(self, name)
            if a is None:
                continue
            a = np.asarray(a, dtype=np.float64)
            if a.shape != shape:
                raise ValueError(f"{name}: shape {a.shape}, expected (Nr, Nt) = {shape}")
            if not np.all(np.isfinite(a)):
                raise ValueError(f"{name}: non-finite values")
            setattr(self, name, a)
        if np.any(self.T < 0):
            raise ValueError("T: negative temperatures")
        if self.mu is None:
            self.mu = np.zeros(shape)

    # -- what the drivers take ------------------------------------------------------
    def evolution(self):
        """(TemperatureEvolution, VelocityEvolution, SpaceTimeGrid) for
        simulate_ensemble_bulk: T, the radial velocity v^r = u^r / sqrt(1 + u^r^2)."""
        return self.T.copy(), velocity_from_four(self.ur), (self.r.copy(), self.tau.copy())

    def profiles(self):
        """(T_profile, ur_profile, mu_profile): callables of (r, tau), clamped bilinear on
        the nodes, for the Milne backend's initial-state sampler."""
        r, tau = self.r, self.tau

        def make(field):
            def f(rq, tq):
                out = interp2d_clamped(r, tau, field, rq, tq)
                return float(out) if np.ndim(out) == 0 else out
            return f
        return make(self.T), make(self.ur), make(self.mu)

    # -- files ----------------------------------------------------------------------
    def save_npz(self, path):
        np.savez(path, r=self.r, tau=self.tau, T=self.T, ur=self.ur, mu=self.mu)

    @classmethod
    def load_npz(cls, path):
        with np.load(path) as z:
            return cls(z["r"], z["tau"], z["T"], z["ur"], z["mu"] if "mu" in z.files else None)

    @classmethod
    def load_raw(cls, header_path):
        """A JSON header {"kind": "rt", "r": [...] | {"file", "n"}, "tau": ..., "T": {"file",
        "dtype"}, "ur": ..., "mu": ...}: raw column-major (Nr, Nt) arrays beside it."""
        h, base = _read_header(header_path, "rt")
        r = _axis_from(h["r"], base)
        tau = _axis_from(h["tau"], base)
        shape = (r.size, tau.size)
        fields = {k: _raw_array(h[k], base, shape) for k in ("T", "ur", "mu") if k in h}
        return cls(r, tau, fields["T"], fields["ur"], fields.get("mu"))


@dataclass
class HydroXY:
    """A 2+1D evolution on (tau, y, x) nodes: T and the flow (four-velocity u^x, u^y, or
    the velocity v^x, v^y when ``four_velocity`` is False), arrays of shape (Nt, Ny, Nx)."""
    x: np.ndarray
    y: np.ndarray
    tau: np.ndarray
    T: np.ndarray
    ux: np.ndarray
    uy: np.ndarray
    four_velocity: bool = True

    def __post_init__(self):
        self.x = _axis(self.x, "x")
        self.y = _axis(self.y, "y")
        self.tau = _axis(self.tau, "tau")
        shape = (self.tau.size, self.y.size, self.x.size)
        for name in ("T", "ux", "uy"):
            a = np.asarray(getattr(self, name), dtype=np.float64)
            if a.shape != shape:
                raise ValueError(f"{name}: shape {a.shape}, expected (Nt, Ny, Nx) = {shape}")
            if not np.all(np.isfinite(a)):
                raise ValueError(f"{name}: non-finite values")
            setattr(self, name, a)
        if np.any(self.T < 0):
            raise ValueError("T: negative temperatures")
        if not self.four_velocity and np.any(self.ux ** 2 + self.uy ** 2 >= 1.0):
            raise ValueError("velocity: |v| >= 1")

    def velocity(self):
        """(v^x, v^y): the flow velocity (v = u / sqrt(1 + u.u) from a four-velocity)."""
        if not self.four_velocity:
            return self.ux, self.uy
        g = np.sqrt(1.0 + self.ux ** 2 + self.uy ** 2)
        return self.ux / g, self.uy / g

    def grid_medium(self, *, nx=None, ny=None, nt=None):
        """Keyword arguments of Engine.set_medium_grid: FP32 fields (Nt, Ny, Nx) on a
        uniform grid.  Uniform input axes pass through; otherwise (or when nx / ny / nt
        ask for another resolution) the fields are resampled trilinearly onto uniform
        nodes spanning the same ranges."""
        vx, vy = self.velocity()
        axes = [self.tau, self.y, self.x]
        want = [nt or self.tau.size, ny or self.y.size, nx or self.x.size]
        uniform = [np.linspace(a[0], a[-1], n) for a, n in zip(axes, want)]
        same = all(a.size == u.size and np.allclose(a, u, rtol=0, atol=1e-12 * max(1.0, abs(a[-1])))
                   for a, u in zip(axes, uniform))
        fields = [self.T, vx, vy]
        if not same:
            fields = [_resample3(f, axes, uniform) for f in fields]
        t, y, x = uniform
        return dict(T=fields[0].astype(np.float32), ux=fields[1].astype(np.float32), uy=fields[2].astype(np.float32),
                    x0=float(x[0]), dx=float(x[1] - x[0]), y0=float(y[0]), dy=float(y[1] - y[0]),
                    tau0=float(t[0]), dtau=float(t[1] - t[0]))

    def save_npz(self, path):
        np.savez(path, x=self.x, y=self.y, tau=self.tau, T=self.T, ux=self.ux, uy=self.uy,
                 four_velocity=np.array(self.four_velocity))

    @classmethod
    def load_npz(cls, path):
        with np.load(path) as z:
            fv = bool(z["four_velocity"]) if "four_velocity" in z.files else True
            return cls(z["x"], z["y"], z["tau"], z["T"], z["ux"], z["uy"], fv)

    @classmethod
    def load_raw(cls, header_path):
        """A JSON header {"kind": "xy", "x", "y", "tau", "T", "ux", "uy",
        "four_velocity": true}: raw column-major (Nx, Ny, Nt) arrays (Julia's order)."""
        h, base = _read_header(header_path, "xy")
        x, y, tau = (_axis_from(h[k], base) for k in ("x", "y", "tau"))
        shape = (x.size, y.size, tau.size)
        f = {k: _raw_array(h[k], base, shape).transpose(2, 1, 0) for k in ("T", "ux", "uy")}
        return cls(x, y, tau, f["T"], f["ux"], f["uy"], bool(h.get("four_velocity", True)))


def _read_header(path, kind):
    p = Path(path)
    h = json.loads(p.read_text())
    if h.get("kind") != kind:
        raise ValueError(f"{p}: header kind {h.get('kind')!r}, expected {kind!r}")
    return h, p.parent


def _axis_from(spec, base):
    if isinstance(spec, dict):
        a = np.fromfile(base / spec["file"], dtype=spec.get("dtype", "<f8"))
        if "n" in spec and a.size != int(spec["n"]):
            raise ValueError(f"{spec['file']}: {a.size} values, expected {spec['n']}")
        return a
    return np.asarray(spec, dtype=np.float64)


def _raw_array(spec, base, shape):
    a = np.fromfile(base / spec["file"], dtype=spec.get("dtype", "<f8")).astype(np.float64)
    if a.size != math.prod(shape):
        raise ValueError(f"{spec['file']}: {a.size} values, expected {math.prod(shape)} for shape {shape}")
    return a.reshape(shape, order="F")


def _interp_axis(src, dst):
    i = np.clip(np.searchsorted(src, dst, side="right") - 1, 0, src.size - 2)
    w = (dst - src[i]) / (src[i + 1] - src[i])
    return i, np.clip(w, 0.0, 1.0)


def _resample3(f, axes, new_axes):
    out = np.asarray(f, dtype=np.float64)
    for ax, (src, dst) in enumerate(zip(axes, new_axes)):
        i, w = _interp_axis(src, dst)
        a = np.take(out, i, axis=ax)
        b = np.take(out, i + 1, axis=ax)
        shape = [1] * out.ndim
        shape[ax] = -1
        w = w.reshape(shape)
        out = a * (1 - w) + b * w
    return out
