"""Host-side helpers of the simulation drivers (initial-state completion and contracts).

Restates the parts of LangevInMedium.jl's ``src/utils.jl`` that sit between the
user's initial state and the time loop: the momentum-dimension contract
``check_momentum_dims`` (:561-573), the thermal p_z completion
``sample_pz_conditional_juttner`` / ``append_thermal_pz`` (:499-551), and the radial
reduction of the drivers (simulate_cpu.jl:102-136), and the momentum-only initial state
of the static-temperature path ``sample_initial_particles_at_origin_no_position!``
(:419-465).  Randomness comes from a numpy
Generator (the reference uses Julia's global RNG; draws are distributionally, not
bitwise, equivalent).
"""
from __future__ import annotations

import math

import numpy as np


def check_momentum_dims(dimensions: int, pdim: int, radial_mode: bool, bjorken_redshift: bool, initial_time: float):
    """utils.jl:561-573 — raise ValueError on the combinations the engine refuses."""
    if pdim != dimensions:
        if not (dimensions == 2 and pdim == 3 and not radial_mode):
            raise ValueError(f"momentum_dimensions={pdim} with dimensions={dimensions} is not supported: "
                             "only (dimensions=2, momentum_dimensions=3) differs from the coupled default.")
    if bjorken_redshift:
        if not (dimensions == 2 and pdim == 3):
            raise ValueError("bjorken_redshift requires dimensions=2 and momentum_dimensions=3 (p_z is row 3).")
        if not initial_time > 0:
            raise ValueError("bjorken_redshift needs initial_time > 0 (Milne τ; dp_z/dτ = −p_z/τ).")


def sample_pz_conditional_juttner(mT: np.ndarray, T: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """Draws from f(p_z) ∝ exp(−sqrt(m_T² + p_z²)/T), vectorised over particles
    (utils.jl:499-522: Gaussian envelope in rapidity for a = m_T/T > 1.05, Laplace
    envelope in p_z otherwise)."""
    mT = np.asarray(mT, dtype=np.float64)
    T = np.broadcast_to(np.asarray(T, dtype=np.float64), mT.shape)
    out = np.zeros(mT.shape)
    ok = (T > 0.0) & (mT > 0.0)
    a = np.where(ok, mT / np.where(T > 0, T, 1.0), 0.0)
    gauss = ok & (a > 1.05)
    lap = ok & ~gauss
    idx = np.nonzero(gauss)[0]
    tries = 0
    while idx.size and tries < 100_000:
        ai = a[idx]
        c = np.maximum(2.0, ai / (ai - 1.0))
        sig = np.sqrt(c / ai)
        y = sig * rng.standard_normal(idx.size)
        ch = np.cosh(y)
        acc = ch * np.exp(-ai * (ch - 1.0) + ai * y * y / (2.0 * c))
        take = rng.random(idx.size) <= acc
        out[idx[take]] = mT[idx[take]] * np.sinh(y[take])
        idx = idx[~take]
        tries += 1
    idx = np.nonzero(lap)[0]
    tries = 0
    while idx.size and tries < 1_000_000:
        b = math.sqrt(2.0) * T[idx]
        sgn = np.where(rng.random(idx.size) < 0.5, -1.0, 1.0)
        pz = -b * np.log(rng.random(idx.size)) * sgn
        m_ = mT[idx]
        acc = np.exp(-(np.sqrt(m_ * m_ + pz * pz) - (m_ + np.abs(pz)) / math.sqrt(2.0)) / T[idx])
        take = rng.random(idx.size) <= acc
        out[idx[take]] = pz[take]
        idx = idx[~take]
        tries += 1
    return out


def append_thermal_pz(momenta, positions, m, T_of_r, *, antithetic=False, rng=None) -> np.ndarray:
    """utils.jl:533-551 — (2, N) transverse LRF momenta -> (3, N) with a thermal p_z."""
    rng = rng or np.random.default_rng()
    momenta = np.asarray(momenta, dtype=np.float64)
    if momenta.shape[0] != 2:
        raise ValueError(f"append_thermal_pz: expected 2 transverse momentum rows, got {momenta.shape[0]}")
    positions = np.asarray(positions, dtype=np.float64)
    N = momenta.shape[1]
    out = np.zeros((3, N))
    out[:2] = momenta
    r = np.sqrt(np.sum(positions ** 2, axis=0))
    T = np.maximum(np.array([float(T_of_r(ri)) for ri in r]) if callable(T_of_r) else np.asarray(T_of_r), 0.0)
    mT = np.sqrt(float(m) ** 2 + momenta[0] ** 2 + momenta[1] ** 2)
    out[2] = sample_pz_conditional_juttner(mT, T, rng)
    if antithetic:
        ev = np.arange(1, N, 2)       # Julia's even i (1-based) are the odd 0-based indices
        out[2, ev] = -out[2, ev - 1]
    return out


def radial_reduction(x2: np.ndarray, p2: np.ndarray, r_grid, rng: np.random.Generator):
    """simulate_cpu.jl:102-136 — Cartesian (2, N) samples -> radial (r, p_r)."""
    x2 = np.asarray(x2, dtype=np.float64)
    p2 = np.asarray(p2, dtype=np.float64)
    r = np.sqrt(x2[0] ** 2 + x2[1] ** 2)
    r_grid = np.asarray(r_grid, dtype=np.float64)
    dr0 = abs(float(r_grid[1] - r_grid[0])) if r_grid.size >= 2 else 0.0
    r_axis_eps = max(1e-12, 0.5 * dr0)
    ex = np.empty_like(r)
    ey = np.empty_like(r)
    reg = r > r_axis_eps
    ex[reg] = x2[0, reg] / r[reg]
    ey[reg] = x2[1, reg] / r[reg]
    ns = int(np.count_nonzero(~reg))
    if ns:
        rx = rng.standard_normal(ns)
        ry = rng.standard_normal(ns)
        invn = 1.0 / (np.sqrt(rx ** 2 + ry ** 2) + np.finfo(np.float64).eps)
        ex[~reg] = rx * invn
        ey[~reg] = ry * invn
    pr = ex * p2[0] + ey * p2[1]
    return r.reshape(1, -1), pr.reshape(1, -1)


def _rt_interp_host(xgrid, tgrid, values, xi, yi) -> float:
    """Clamped bilinear lookup on the (r, t) table (kernels_cpu.jl:22-51), host side,
    used only to complete initial states before the first step."""
    x = np.asarray(xgrid, dtype=np.float64)
    y = np.asarray(tgrid, dtype=np.float64)
    xi = min(max(float(xi), x[0]), x[-1])
    yi = min(max(float(yi), y[0]), y[-1])
    i = int(np.searchsorted(x, xi, side="right")) - 1
    j = int(np.searchsorted(y, yi, side="right")) - 1
    i = min(max(i, 0), x.size - 2)
    j = min(max(j, 0), y.size - 2)
    dx, dy = x[i + 1] - x[i], y[j + 1] - y[j]
    eps = np.finfo(np.float64).eps
    xd = 0.0 if abs(dx) < eps else (xi - x[i]) / dx
    yd = 0.0 if abs(dy) < eps else (yi - y[j]) / dy
    v = np.asarray(values, dtype=np.float64)
    c0 = v[i, j] * (1 - xd) + v[i + 1, j] * xd
    c1 = v[i, j + 1] * (1 - xd) + v[i + 1, j + 1] * xd
    return float(c0 * (1 - yd) + c1 * yd)


def sample_initial_particles_at_origin_no_position(initial_condition, p0, dimensions: int, N_particles: int,
                                                   rng: np.random.Generator) -> np.ndarray:
    """utils.jl:419-465 — the momenta (dimensions, N) of the static-temperature path:
    "delta": |p| = p0 in a random direction (a normalised Gaussian vector); "bimodal":
    |p| from an equal mixture of Normal(1, 0.2) and Normal(2, 0.2) truncated to
    [0.1, 5], in a random direction; anything else is the reference's error."""
    N, d = int(N_particles), int(dimensions)
    if initial_condition == "delta":
        dirs = rng.standard_normal((d, N))
        return p0 * (dirs / np.sqrt(np.sum(dirs ** 2, axis=0)))
    if initial_condition == "bimodal":
        mu = np.where(rng.random(N) < 0.5, 1.0, 2.0)
        mags = np.empty(N)
        todo = np.arange(N)
        while todo.size:                      # truncation to [pmin, pmax] by rejection
            draw = rng.normal(mu[todo], 0.2)
            ok = (draw >= 0.1) & (draw <= 5.0)
            mags[todo[ok]] = draw[ok]
            todo = todo[~ok]
        dirs = rng.standard_normal((d, N))
        return mags * (dirs / np.linalg.norm(dirs, axis=0))
    raise ValueError(f"Unknown initial condition: {initial_condition}")
