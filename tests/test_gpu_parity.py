"""Per-particle parity of the CUDA engine (through the C-ABI) against the CPU FP64
restatement on identical counter-based noise.

Metric: per particle ||a - b|| / max(||b||, floor * s), s = 0.3 GeV for momenta and
1 fm for positions, max over particles.
  FP64 gate 1e-12 with floor 1e-2 (relative down to 3 MeV / 0.01 fm: a momentum that
  passes through zero, as the signed radial one does, keeps the ~1e-15 GeV absolute
  rounding it gathered at the GeV scale).
  FP32 gate 1e-5 with floor 1e-3 (0.3 MeV, 1 um), the two cases of FP32_FLOOR_CASE at a
  larger floor for the reasons given there.  Freeze-out outputs: the one-step split of
  check_latch_one_step.
RTA accept/reject decisions must be identical: a flipped decision moves a momentum
by O(1) and fails either gate."""
import numpy as np
import pytest

from helpers import oracle_medium, oracle_params, parity
from parity_cases import CASES, build_case

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5}
FP32_FLOOR = 1e-3
# Cases whose FP32 error relative to a 1e-3 floor (0.3 MeV, 1 um) exceeds 1e-5 for a
# stated reason, gated at a larger floor (the 1e-3 figure is printed for them too):
#   radial_diffusion_reflect: the 1-D signed radial momentum passes through zero, so a
#     component of ~0.3 MeV carries the ~1e-9 GeV absolute error of the GeV scale;
#   flow2d_v2: the flow speed is modulated by cos 2(phi - psi2) of the particle's FP32
#     azimuth (atan2f, cosf); the frame change then carries an absolute error of order
#     eps_32 E ~ 1e-7 GeV, which particles slower than ~30 MeV show above 1e-5 relative.
FP32_FLOOR_CASE = {"radial_diffusion_reflect": 1.0, "flow2d_v2": 0.1}


def engine_run(lmb, wl, *, record=False, save_every=0, nslots=0, split=None):
    eng = lmb.capi.Engine(0)
    lmb.workloads.configure(eng, wl)
    cart = wl.params.get("coords", 0) == 0
    if cart:
        eng.initial_lab_boost()
    x0, p0 = eng.download_state()
    if record:
        eng.record_noise(wl.first_step, wl.steps)
    hx = hp = None
    if save_every:
        hx = np.zeros(nslots * wl.n * int(eng.params.dims))
        hp = np.zeros(nslots * wl.n * int(eng.params.pdim))
    if split:
        eng.run(wl.first_step, split, save_every, 0, hx, hp)
        eng.run(wl.first_step + split, wl.steps - split, save_every, 0, hx, hp)
    else:
        eng.run(wl.first_step, wl.steps, save_every, 0, hx, hp)
    x, p = eng.download_state()
    out = dict(x0=x0, p0=p0, x=x, p=p, hx=hx, hp=hp)
    if wl.params.get("freezeout_capture"):
        out["fo"] = eng.download_freezeout()
    if record:
        out["rec"] = eng.download_noise()
    out["obs"] = eng.observables()
    eng.close()
    return out


def oracle_run(orc, wl, x0, p0, *, rec=None, save_every=0, nslots=0, **over):
    P = oracle_params(orc, wl, **over)
    md = oracle_medium(orc, wl)
    return orc.run(P, md, x0, p0, wl.first_step, wl.steps, save_every=save_every, nslots=nslots, rec=rec)


def assert_parity(tag, g, o, tol, T=0.3, floor=1e-2, mask=None):
    gx, ox, gp, op = g["x"], o["x"], g["p"], o["p"]
    if mask is not None:
        gx, ox, gp, op = gx[:, mask], ox[:, mask], gp[:, mask], op[:, mask]
    ex = parity(gx, ox, 1.0, floor)
    ep = parity(gp, op, T, floor)
    sx = parity(gx, ox, 1.0, 1e-3)
    sp = parity(gp, op, T, 1e-3)
    print(f"{tag}: x max {ex[0]:.3g} p99 {ex[1]:.3g} | p max {ep[0]:.3g} p99 {ep[1]:.3g}"
          f" | strict x {sx[0]:.3g} p {sp[0]:.3g}")
    assert ex[0] <= tol and ep[0] <= tol, (tag, ex, ep)


@pytest.mark.parametrize("name", CASES)
def test_fp64_parity(lmb, orc, name):
    wl = build_case(name, "fp64")
    over = {"stop_after_freezeout": 0}
    wl.params.update(over)
    g = engine_run(lmb, wl)
    P = oracle_params(orc, wl)
    md = oracle_medium(orc, wl)
    if wl.params.get("coords", 0) == 0:
        x0, p0 = orc.initial_lab_boost(P, md, wl.x, wl.p)
        assert parity(g["p0"], p0, 0.3)[0] <= TOL["fp64"]
    else:
        x0, p0 = wl.x, wl.p
    o = orc.run(P, md, x0, p0, wl.first_step, wl.steps)
    assert o["first_bad"] == -1
    assert_parity(f"{name} fp64", g, o, TOL["fp64"])
    if "fo" in g:
        assert np.array_equal(g["fo"]["flag"], o["fo_flag"])
        assert parity(g["fo"]["pos"], o["fo_pos"], 1.0)[0] <= TOL["fp64"]
        assert parity(g["fo"]["mom"], o["fo_mom"], 0.3)[0] <= TOL["fp64"]
        assert parity(g["fo"]["tau"], o["fo_tau"], 1.0)[0] <= TOL["fp64"]


@pytest.mark.parametrize("name", CASES)
def test_fp32_parity_recorded_noise(lmb, orc, name):
    """FP32 engine vs FP64 restatement fed the variates the engine consumed."""
    wl = build_case(name, "fp32")
    check_fo_outputs(lmb, orc, wl, name, record=True)


@pytest.mark.parametrize("name", ["static3d", "lrta_bjorken_table", "grid_lrta_fo", "grid_fine_tau_fo", "grid_offset_fo",
                                  "milne"])
def test_fp32_parity_philox(lmb, orc, name):
    """FP32 engine vs FP64 restatement regenerating the FP32 uniforms from Philox
    (the whole FP32 error: arithmetic plus the FP32 noise transform)."""
    wl = build_case(name, "fp32")
    check_fo_outputs(lmb, orc, wl, name, record=False)


def check_fo_outputs(lmb, orc, wl, name, record):
    """FP32 comparison with the production freeze-out semantics: a latched particle
    stops (its outputs are the latch), so the latch outputs of particles latched in
    both runs and the states of never-latched particles are compared."""
    g = engine_run(lmb, wl, record=record)
    o = oracle_run(orc, wl, g["x0"], g["p0"], rec=g.get("rec"), precision=1)
    tag = f"{name} fp32/{'rec' if record else 'philox'}"
    if "fo" not in g:
        assert_parity(tag, g, o, TOL["fp32"], floor=FP32_FLOOR_CASE.get(name, FP32_FLOOR))
        return
    gf, of = g["fo"]["flag"], o["fo_flag"]
    assert np.mean(gf == of) >= 0.999, np.mean(gf == of)
    live = (gf == 0) & (of == 0)
    both = (gf == 1) & (of == 1)
    assert_parity(tag + " live", g, o, TOL["fp32"], floor=FP32_FLOOR, mask=live)
    check_latch_one_step(tag, wl, g, o, both)


def check_latch_one_step(tag, wl, g, o, both):
    """The latch's outputs interpolate between the last-above state a (step s - 1) and
    the crossing state b (step s): out = a + frac (b - a), frac = (T_a - Tfo)/(T_a - T_b).
    frac divides by a one-step temperature change, so an FP32 error of the crossing
    temperature dT moves out by (dT / (T_a - T_b)) |b - a|: one step's change of the
    state times the temperature's error over its one-step change.  The gate splits the
    output error accordingly:
      - the states agree: b (the final state of a particle that stopped at its
        crossing) at the FP32 tolerance, and the engine's output equals the oracle's
        interpolation taken with the engine's frac (read off its latched tau) at the
        FP32 tolerance;
      - the frac difference is that of temperature differences below 2e-6 GeV: with
        frac = (T_a - Tfo)/(T_a - T_b), errors dT in T_a and T_b move frac by at most
        dT / (T_a - T_b), so |frac_e - frac_o| (T_a - T_b) is gated.
    Runs without stop_after_freezeout keep moving after the latch (no crossing state
    to compare): their latch outputs are gated by the frac split alone."""
    if not np.any(both):
        return
    Tfo, dt = float(wl.params["Tfo"]), float(wl.params["dt"])
    stop = bool(wl.params.get("stop_after_freezeout", 0))
    ltau, lT = o["fo_ltau"][both], o["fo_lT"][both]
    has_last = lT > Tfo
    frac_o = np.where(has_last, (o["fo_tau"][both] - ltau) / dt, 1.0)
    frac_e = np.where(has_last, (g["fo"]["tau"][both] - ltau) / dt, 1.0)
    same_step = np.abs(frac_e - 0.5) <= 0.5 + 1e-9          # latched at the same step as the oracle
    assert np.mean(same_step) >= 0.999, np.mean(same_step)
    k = same_step & has_last & (frac_o > 1e-6)
    Tb_o = lT[k] - (lT[k] - Tfo) / frac_o[k]
    dT = np.abs(frac_e[k] - frac_o[k]) * (lT[k] - Tb_o)
    a_x, a_p = o["fo_lpos"][:, both][:, k], o["fo_lmom"][:, both][:, k]
    if stop:
        b_x, b_p = o["x"][:, both][:, k], o["p"][:, both][:, k]
        eb = max(parity(g["x"][:, both][:, k], b_x, 1.0, FP32_FLOOR)[0],
                 parity(g["p"][:, both][:, k], b_p, 0.3, FP32_FLOOR)[0])
        out_x = a_x + frac_e[k] * (b_x - a_x)
        out_p = a_p + frac_e[k] * (b_p - a_p)
        er = max(parity(g["fo"]["pos"][:, both][:, k], out_x, 1.0, FP32_FLOOR)[0],
                 parity(g["fo"]["mom"][:, both][:, k], out_p, 0.3, FP32_FLOOR)[0])
    else:
        eb = er = 0.0
    ep = parity(g["fo"]["mom"][:, both], o["fo_mom"][:, both], 0.3, FP32_FLOOR)
    print(f"{tag} latched ({int(k.sum())}): crossing state {eb:.3g}, output at the engine's frac {er:.3g}, "
          f"temperature-equivalent frac difference max {dT.max() if dT.size else 0:.3g} GeV; raw latched momentum max {ep[0]:.3g} "
          f"p99 {ep[1]:.3g}")
    assert eb <= TOL["fp32"] and er <= TOL["fp32"], (tag, eb, er)
    assert dT.size == 0 or dT.max() <= 2e-6, (tag, dT.max())


def test_fp32_variates_against_fp64(lmb, orc):
    """The FP32 noise transform (Box-Muller with the polynomial sine/cosine, the inverse
    normal CDF on the folded uniform) against the FP64 one of the same Philox words:
    the whole FP32 error of the momentum normals, max |dz| / max(1, |z|) <= 1e-6."""
    wl = build_case("lrta_bjorken_table", "fp32", N=4096, steps=40)
    g = engine_run(lmb, wl, record=True)
    P = oracle_params(orc, wl)
    rec = g["rec"]
    worst = 0.0
    for s in range(wl.steps):
        for i in range(0, 4096, 5):
            v = orc.step_variates(P, i, wl.first_step + s)
            d = np.abs(rec[s, 0:3, i] - v[0:3]) / np.maximum(1.0, np.abs(v[0:3]))
            worst = max(worst, float(d.max()))
    print(f"FP32 momentum normals vs FP64: max relative error {worst:.3g}")
    assert worst <= 1e-6


def test_fp64_recorded_noise_matches_regenerated(lmb, orc):
    """The variates the FP64 kernel consumed are the ones the restatement regenerates
    from the same Philox counters (to libm-vs-device rounding of log/sincos/erfc)."""
    wl = build_case("lrta_bjorken_table", "fp64", N=512, steps=40)
    g = engine_run(lmb, wl, record=True)
    P = oracle_params(orc, wl)
    rec = g["rec"]
    collided = 0
    for s in range(wl.steps):
        for i in range(0, 512, 7):
            v = orc.step_variates(P, i, wl.first_step + s)
            assert np.allclose(rec[s, 0:4, i], v[0:4], rtol=1e-14, atol=1e-15)
            if rec[s, 4, i] != 0.0:               # recorded only when the particle collided
                collided += 1
                assert rec[s, 4, i] == v[4]       # raw uniform: bit-identical
                assert np.allclose(rec[s, 5:8, i], v[5:8], rtol=1e-14, atol=1e-15)
    assert collided > 0
    o = oracle_run(orc, wl, g["x0"], g["p0"], rec=rec)
    assert_parity("fp64/rec", g, o, 1e-13)


def test_history_snapshots(lmb, orc):
    wl = build_case("flow2d", "fp64", N=1024, steps=100)
    g = engine_run(lmb, wl, save_every=25, nslots=5)
    P = oracle_params(orc, wl)
    md = oracle_medium(orc, wl)
    x0, p0 = orc.initial_lab_boost(P, md, wl.x, wl.p)
    o = orc.run(P, md, x0, p0, 1, 100, save_every=25, nslots=5)
    n = wl.n
    for k in range(1, 5):
        gx = g["hx"][k * n * 2:(k + 1) * n * 2].reshape(n, 2).T
        gp = g["hp"][k * n * 2:(k + 1) * n * 2].reshape(n, 2).T
        assert parity(gx, o["hist_x"][k], 1.0)[0] <= 1e-12
        assert parity(gp, o["hist_p"][k], 0.3)[0] <= 1e-12


def test_chunked_run_is_bit_identical(lmb):
    """Counter-based noise: splitting the step range across launches changes nothing."""
    for prec in ("fp64", "fp32"):
        wl = build_case("lrta_bjorken_table", prec, N=4096, steps=120)
        a = engine_run(lmb, wl)
        b = engine_run(lmb, wl, split=47)
        assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["p"], b["p"])


def test_philox_device_matches_host(lmb, orc):
    eng = lmb.capi.Engine(0)
    rng = np.random.default_rng(5)
    for _ in range(64):
        ctr = [int(v) for v in rng.integers(0, 2 ** 32, 4, dtype=np.uint64)]
        key = [int(v) for v in rng.integers(0, 2 ** 32, 2, dtype=np.uint64)]
        assert eng.philox(ctr, key) == orc.philox(ctr, key)
    eng.close()


def test_empty_ensemble(lmb):
    wl = build_case("flow2d", "fp64", N=4, steps=10)
    wl.x = wl.x[:, :0]
    wl.p = wl.p[:, :0]
    eng = lmb.capi.Engine(0)
    lmb.workloads.configure(eng, wl)
    eng.initial_lab_boost()
    eng.run(1, 10)
    x, p = eng.download_state()
    assert x.shape == (2, 0) and p.shape == (2, 0)
    assert eng.observables()["count"] == 0
    eng.close()


@pytest.mark.parametrize("name,prec,comp,rel", [("flow2d", "fp64", 0, 1), ("flow2d", "fp32", 0, 1),
                                               ("freezeout", "fp32", 2, 1), ("freezeout", "fp64", 2, 0)])
def test_nonfinite_state_is_reported(lmb, name, prec, comp, rel):
    """simulate_cpu.jl:293-303: NaN/Inf in the state stops the run with the step.  The
    Cartesian kernels test the positions (a non-finite momentum reaches them through
    E in the same step) and, in Galilean runs, the momenta too (p^z never reaches x
    there)."""
    wl = build_case(name, prec, N=256, steps=10)
    wl.params["relativistic"] = rel
    wl.params["stop_after_freezeout"] = 0
    wl.p[comp, 100] = np.nan
    eng = lmb.capi.Engine(0)
    lmb.workloads.configure(eng, wl)
    with pytest.raises(lmb.capi.LimError, match="NaN/Inf at step 1") as ei:
        eng.run(1, 10)
    assert ei.value.code == lmb.capi.LIM_ERR_NONFINITE
    assert eng.status() == 1
    eng.close()


def test_parameter_validation(lmb):
    capi = lmb.capi
    eng = capi.Engine(0)
    with pytest.raises(capi.LimError, match="momentum_dimensions=4 with dimensions=2"):
        eng.set_params(dims=2, pdim=4)
    with pytest.raises(capi.LimError, match="bjorken_redshift requires dimensions=2"):
        eng.set_params(dims=3, pdim=3, bjorken_redshift=1, t0=1.0)
    with pytest.raises(capi.LimError, match="initial_time > 0"):
        eng.set_params(dims=2, pdim=3, bjorken_redshift=1, t0=0.0)
    with pytest.raises(capi.LimError, match="collision_mode"):
        eng.set_params(collision=9)
    with pytest.raises(capi.LimError) as ei:
        eng.set_medium_rt([0.0, 0.0, 1.0], [0.0, 1.0], np.zeros((3, 2)), np.zeros((3, 2)))
    assert ei.value.code == capi.LIM_ERR_ARG
    eng.set_params(dims=2, pdim=2)
    with pytest.raises(capi.LimError, match="no medium"):
        eng.run(1, 1)
    eng.close()


def test_observables_match_host_reduction(lmb):
    wl = build_case("lrta_bjorken_table", "fp64", N=20000, steps=50)
    g = engine_run(lmb, wl)
    p = g["p"]
    pt = np.hypot(p[0], p[1])
    obs = g["obs"]
    assert obs["count"] == wl.n
    assert np.isclose(obs["mean_pt"], pt.mean(), rtol=1e-12)
    assert np.isclose(obs["mean_cos2phi"], np.mean((p[0] ** 2 - p[1] ** 2) / pt ** 2), rtol=1e-10)
    assert np.isclose(obs["frac_pt_gt"], np.mean(pt > 5.0), rtol=1e-12)
    assert np.isclose(obs["mean_p2"], np.mean(np.sum(p ** 2, axis=0)), rtol=1e-12)


@pytest.mark.parametrize("name,steps", [("grid_lrta_fo", 200), ("grid_fine_tau_fo", 110)])
def test_live_list_run_matches_full_grid_run(lmb, name, steps):
    """Runs that stop particles at freeze-out advance a compacted list of the live
    particles; the result equals the run over every particle (the noise-recording
    instantiation takes that path), latch outputs included, and the run split into two
    calls (the FP32 kernel carries the grid lookup of one step into the next, so a launch
    boundary must not change the bits)."""
    for prec in ("fp32", "fp64"):
        wl = build_case(name, prec, N=20000, steps=steps)
        a = engine_run(lmb, wl)
        assert 0.05 < np.mean(a["fo"]["flag"]) < 0.95
        for tag, b in (("record", engine_run(lmb, wl, record=True)), ("split", engine_run(lmb, wl, split=45))):
            assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["p"], b["p"]), (prec, tag)
            for k in ("pos", "mom", "tau", "flag"):
                assert np.array_equal(a["fo"][k], b["fo"][k]), (prec, tag, k)
