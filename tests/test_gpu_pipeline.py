"""Ensembles streamed through two slots of contexts (pipeline.EnsembleStream): the
copies of neighbouring passes overlap each run, and every pass must give the
freeze-out outputs and final state of the same ensemble run alone, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def lane_workloads(lmb, npasses, prec):
    """Per pass and lane (charm, bottom) a grid workload with its own initial state."""
    W = lmb.workloads
    fields = W.grid2p1_fields(nx=41, ny=41, nt=24, dx=0.5)
    out = []
    for k in range(npasses):
        row = []
        for lane, m in enumerate((1.5, 4.75)):
            wl = W.grid2p1(N=3000 + 500 * lane, m=m, fields=fields, precision=prec, steps=180,
                           rng_seed=11 + 7 * k + lane)
            wl.params["particle_offset"] = 100_000 * lane
            row.append(wl)
        out.append(row)
    return out


def alone(lmb, wl):
    e = lmb.capi.Engine(0)
    lmb.workloads.configure(e, wl)
    e.initial_lab_boost()
    e.run(wl.first_step, wl.steps)
    res = (e.download_freezeout(), e.download_state())
    e.close()
    return res


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_streamed_passes_match_runs_alone(lmb, prec):
    capi, W = lmb.capi, lmb.workloads
    K = 3
    wls = lane_workloads(lmb, K, prec)
    engines = []
    for slot in range(2):
        row = []
        for lane in range(2):
            e = capi.Engine(0)
            W.configure(e, wls[0][lane], upload=False)
            row.append(e)
        engines.append(row)
    got = {}

    def load(k, lane, eng):
        wl = wls[k][lane]
        dims, pdim = int(wl.params["dims"]), int(wl.params["pdim"])
        eng.upload_state_flat(capi.julia_layout(wl.x, dims), capi.julia_layout(wl.p, pdim), wl.n)
        eng.initial_lab_boost()

    def unload(k, lane, eng):
        assert (k, lane) not in got
        got[(k, lane)] = (eng.download_freezeout(), eng.download_state())

    stream = lmb.pipeline.EnsembleStream(engines)
    stream.run(K, wls[0][0].first_step, wls[0][0].steps, load, unload)
    assert sorted(got) == [(k, l) for k in range(K) for l in range(2)]
    for k in range(K):
        for lane in range(2):
            (f, (x, p)), (fr, (xr, pr)) = got[(k, lane)], alone(lmb, wls[k][lane])
            assert f["flag"].sum() > 0
            for key in ("pos", "mom", "tau", "flag"):
                assert np.array_equal(f[key], fr[key]), (k, lane, key)
            assert np.array_equal(x, xr) and np.array_equal(p, pr), (k, lane)
    for row in engines:
        for e in row:
            e.close()

