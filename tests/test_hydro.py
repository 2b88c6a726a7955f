"""Hydro background ingestion (hydro.py): the (r, tau) evolution's velocity and profile
functions against the reference's conventions and the oracle's restatement of
interpolate_2d_cpu (kernels_cpu.jl:22-51), file round trips (npz, raw column-major dumps
as Julia writes them), the (x, y, tau) grid medium with resampling, and input checks."""
import json

import numpy as np
import pytest

from conftest import load_pkg

H = load_pkg().hydro


def rt_case(nr=41, nt=23):
    r = np.linspace(0.0, 12.0, nr)
    tau = np.geomspace(0.4, 12.0, nt)                 # non-uniform in tau
    T = 0.45 * np.exp(-r[:, None] ** 2 / 40.0) * (0.4 / tau[None, :]) ** (1 / 3)
    ur = 0.08 * r[:, None] * np.sqrt(tau[None, :])
    mu = 0.01 * np.sin(r)[:, None] * np.ones(nt)[None, :]
    return H.HydroRT(r, tau, T, ur, mu)


def test_rt_evolution_and_profiles(orc):
    h = rt_case()
    T, V, (r, tau) = h.evolution()
    assert np.array_equal(T, h.T) and np.array_equal(r, h.r)
    assert np.allclose(V, h.ur / np.sqrt(1 + h.ur ** 2), rtol=0, atol=0)
    assert np.all(np.abs(V) < 1)
    fT, fu, fm = h.profiles()
    rng = np.random.default_rng(1)
    rq = rng.uniform(-1.0, 14.0, 200)                 # includes clamped queries
    tq = rng.uniform(0.2, 14.0, 200)
    lib = orc.lib()
    import ctypes as C
    for f, field in ((fT, h.T), (fu, h.ur), (fm, h.mu)):
        vals = np.ascontiguousarray(field.ravel(order="F"))
        ref = [lib.orc_interp2d_clamped(h.r.ctypes.data_as(orc._DP), h.r.size, h.tau.ctypes.data_as(orc._DP),
                                        h.tau.size, vals.ctypes.data_as(orc._DP), a, b) for a, b in zip(rq, tq)]
        assert np.array_equal(f(rq, tq), np.array(ref))
        assert f(float(rq[0]), float(tq[0])) == ref[0]


def test_rt_npz_and_raw_round_trip(tmp_path):
    h = rt_case()
    h.save_npz(tmp_path / "h.npz")
    g = H.HydroRT.load_npz(tmp_path / "h.npz")
    assert all(np.array_equal(getattr(g, k), getattr(h, k)) for k in ("r", "tau", "T", "ur", "mu"))
    # raw column-major dumps (Julia: write(io, A) of a Matrix{Float64} / Float32)
    h.T.T.astype("<f4").tofile(tmp_path / "T.bin")
    h.ur.T.tofile(tmp_path / "ur.bin")
    h.tau.tofile(tmp_path / "tau.bin")
    hdr = {"kind": "rt", "r": h.r.tolist(), "tau": {"file": "tau.bin", "n": h.tau.size},
           "T": {"file": "T.bin", "dtype": "<f4"}, "ur": {"file": "ur.bin"}}
    (tmp_path / "h.json").write_text(json.dumps(hdr))
    g = H.HydroRT.load_raw(tmp_path / "h.json")
    assert np.array_equal(g.T, h.T.astype(np.float32).astype(np.float64))
    assert np.array_equal(g.ur, h.ur) and np.array_equal(g.tau, h.tau) and np.all(g.mu == 0)


def test_rt_input_checks():
    h = rt_case()
    with pytest.raises(ValueError, match="shape"):
        H.HydroRT(h.r, h.tau, h.T[:, :-1], h.ur)
    with pytest.raises(ValueError, match="ascending"):
        H.HydroRT(h.r[::-1], h.tau, h.T, h.ur)
    with pytest.raises(ValueError, match="negative"):
        H.HydroRT(h.r, h.tau, -h.T, h.ur)
    bad = h.ur.copy()
    bad[3, 4] = np.nan
    with pytest.raises(ValueError, match="non-finite"):
        H.HydroRT(h.r, h.tau, h.T, bad)


def xy_case(nx=33, ny=29, nt=7, four=True):
    x = np.linspace(-8.0, 8.0, nx)
    y = np.linspace(-7.0, 7.0, ny)
    tau = np.linspace(0.6, 3.0, nt)
    Tt, Y, X = np.meshgrid(tau, y, x, indexing="ij")
    T = 0.4 + 0.01 * X - 0.02 * Y - 0.05 * Tt            # linear: trilinear resampling is exact
    ux = 0.03 * X * Tt
    uy = 0.02 * Y * Tt
    return H.HydroXY(x, y, tau, T, ux, uy, four)


def test_xy_grid_medium_and_resampling():
    h = xy_case()
    g = h.grid_medium()
    vx, vy = h.velocity()
    gam = np.sqrt(1 + h.ux ** 2 + h.uy ** 2)
    assert np.array_equal(g["ux"], (h.ux / gam).astype(np.float32)) and np.array_equal(g["uy"], vy.astype(np.float32))
    assert g["T"].shape == (7, 29, 33) and g["dx"] == pytest.approx(0.5) and g["tau0"] == 0.6
    # resampled onto a finer grid: exact for the linear temperature
    f = h.grid_medium(nx=65, ny=57, nt=13)
    x = np.linspace(-8, 8, 65)
    y = np.linspace(-7, 7, 57)
    t = np.linspace(0.6, 3.0, 13)
    Tt, Y, X = np.meshgrid(t, y, x, indexing="ij")
    assert np.allclose(f["T"], (0.4 + 0.01 * X - 0.02 * Y - 0.05 * Tt).astype(np.float32), atol=1e-6)
    # a non-uniform tau axis is resampled onto uniform nodes over the same range
    n = H.HydroXY(h.x, h.y, np.array([0.6, 0.7, 0.9, 1.3, 1.8, 2.4, 3.0]), h.T, h.ux, h.uy)
    m = n.grid_medium()
    assert m["tau0"] == 0.6 and m["dtau"] == pytest.approx(0.4)


def test_xy_raw_round_trip_and_checks(tmp_path):
    h = xy_case(four=False)
    for k in ("T", "ux", "uy"):
        getattr(h, k).tofile(tmp_path / f"{k}.bin")     # (Nt, Ny, Nx) C order = Julia's (Nx, Ny, Nt)
    hdr = {"kind": "xy", "x": h.x.tolist(), "y": h.y.tolist(), "tau": h.tau.tolist(), "four_velocity": False,
           **{k: {"file": f"{k}.bin"} for k in ("T", "ux", "uy")}}
    (tmp_path / "g.json").write_text(json.dumps(hdr))
    g = H.HydroXY.load_raw(tmp_path / "g.json")
    assert all(np.array_equal(getattr(g, k), getattr(h, k)) for k in ("T", "ux", "uy")) and not g.four_velocity
    h.save_npz(tmp_path / "g.npz")
    g2 = H.HydroXY.load_npz(tmp_path / "g.npz")
    assert np.array_equal(g2.T, h.T) and not g2.four_velocity
    with pytest.raises(ValueError, match=r"\|v\| >= 1"):
        H.HydroXY(h.x, h.y, h.tau, h.T, h.ux * 100, h.uy, False)
    with pytest.raises(ValueError, match="header kind"):
        H.HydroRT.load_raw(tmp_path / "g.json")
