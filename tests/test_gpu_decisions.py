"""One-step decision parity: from the engine's own state at every step, the CPU
restatement takes the same step, and the RTA accept/reject decisions and the
freeze-out latch decisions of the two are compared particle by particle.

Restarting the restatement from the engine's state at each step isolates the
decisions from trajectory drift.  FP64 must flip none.  The FP32 path decides a
collision whose uniform lies within 1e-5 of its FP32 probability again in FP64, so it
flips none either unless the FP64 temperatures differ in their last bits; flips are
counted, printed and bounded.  The engine records its decisions through the
noise-recording instantiation (the collision's sample uniform is recorded only when the
particle collides); the restatement writes a decision record."""
import numpy as np
import pytest

from helpers import oracle_medium, oracle_params
from parity_cases import build_case

pytestmark = pytest.mark.gpu

STEPS = 40
N = 8192
FO_FIELDS = 16


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["rta2d", "lrta_bjorken_table", "grid_lrta_fo", "freezeout"])
def test_one_step_decisions(lmb, orc, name, prec):
    wl = build_case(name, prec, N=N, steps=STEPS)
    fo_cap = bool(wl.params.get("freezeout_capture"))
    rta = wl.params["collision"] in (lmb.capi.LIM_COLL_RTA, lmb.capi.LIM_COLL_LANGEVIN_RTA)
    eng = lmb.capi.Engine(0)
    lmb.workloads.configure(eng, wl)
    eng.initial_lab_boost()
    P = oracle_params(orc, wl, precision=1 if prec == "fp32" else 0)
    md = oracle_medium(orc, wl)
    n = wl.n
    rta_dec = rta_flips = fo_dec = fo_flips = collisions = latched = 0
    for s in range(wl.first_step, wl.first_step + STEPS):
        x, p = eng.download_state()
        flag0 = eng.download_freezeout()["flag"].copy() if fo_cap else None
        eng.record_noise(s, 1)
        eng.run(s, 1)
        rec = eng.download_noise()
        fo0 = None
        if fo_cap:
            fo0 = np.zeros((n, FO_FIELDS))
            fo0[:, 7] = flag0                       # only the flag enters the latch decision
        o = orc.run(P, md, x, p, s, 1, fo=None if fo0 is None else fo0.reshape(-1), decisions=True)
        if rta:
            live = flag0 == 0 if fo_cap else np.ones(n, bool)
            col_e = rec[0, 4, :] != 0.0
            col_o = (o["dec"][0] & 1) != 0
            rta_dec += int(live.sum())
            rta_flips += int(np.sum((col_e != col_o) & live))
            collisions += int(col_o[live].sum())
        if fo_cap:
            flag1 = eng.download_freezeout()["flag"]
            lat_e = (flag0 == 0) & (flag1 != 0)
            lat_o = (o["dec"][0] & 2) != 0
            fo_dec += int((flag0 == 0).sum())
            fo_flips += int(np.sum(lat_e != lat_o))
            latched += int(lat_o.sum())
    eng.close()
    print(f"{name} {prec}: RTA {rta_flips} flips / {rta_dec} decisions ({collisions} collisions); "
          f"freeze-out {fo_flips} flips / {fo_dec} decisions ({latched} latched)")
    if rta:
        assert collisions > 0
    if fo_cap:
        assert latched > 0
    if prec == "fp64":
        assert rta_flips == 0 and fo_flips == 0
    else:
        assert rta_flips <= max(2, 1e-5 * rta_dec), rta_flips
        assert fo_flips <= max(2, 1e-4 * fo_dec), fo_flips
