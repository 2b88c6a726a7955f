"""The batched persistent launch (lim_batch_*): many ensembles of uneven particle
counts, step ranges, masses, transport tables and media in one launch per chunk of
steps, replayed as a CUDA graph.  A particle's noise depends on (seed, particle id,
step) only, so the batch must reproduce separate lim_run calls bit for bit, for every
launch shape the autotuner may pick."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [dict(), dict(block=128, chunk_steps=16), dict(block=64, chunk_steps=7, reg_cap=1),
          dict(block=256, chunk_steps=1000, blocks_per_sm=1, reg_cap=1)]


def make_engines(lmb, wls):
    engs = []
    for wl in wls:
        e = lmb.capi.Engine(0)
        lmb.workloads.configure(e, wl)
        e.initial_lab_boost()
        e.state_save()
        engs.append(e)
    return engs


def small_batch(lmb, prec, E=8, **kw):
    kw.setdefault("n_range", (300, 5000))
    kw.setdefault("steps_range", (20, 90))
    kw.setdefault("grid_shape", (41, 41, 20))
    return lmb.workloads.batch(E=E, precision=prec, **kw)


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_batch_bit_identical_to_separate_runs(lmb, prec):
    wls = small_batch(lmb, prec)
    assert {w.meta["kind"] for w in wls} == {"bjorken", "grid"}
    engs = make_engines(lmb, wls)
    ref = []
    for e, wl in zip(engs, wls):
        e.run(wl.first_step, wl.steps)
        ref.append(e.download_state())
        e.state_restore()
    b = lmb.capi.Batch(0)
    for e, wl in zip(engs, wls):
        b.add(e, wl.first_step, wl.steps)
    for sh in SHAPES:
        for e in engs:
            e.state_restore()
        b.set_shape(**sh)
        b.run()
        ms, launches, ps = b.stats()
        assert ps == sum(w.n * w.steps for w in wls) and launches >= 1 and ms > 0
        for k, e in enumerate(engs):
            x, p = e.download_state()
            assert np.array_equal(x, ref[k][0]) and np.array_equal(p, ref[k][1]), (sh, k)
    b.close()


def test_batch_rebuilds_after_a_context_changes(lmb):
    """A context re-uploaded with another particle count after the batch was prepared
    is picked up by the next run (the graph is rebuilt, no stale pointers)."""
    wls = small_batch(lmb, "fp32", E=4)
    engs = make_engines(lmb, wls)
    b = lmb.capi.Batch(0)
    for e, wl in zip(engs, wls):
        b.add(e, wl.first_step, wl.steps)
    b.run()
    wl = wls[1]
    keep = slice(0, wl.n // 2)
    wl.x, wl.p = wl.x[:, keep].copy(), wl.p[:, keep].copy()
    engs[1].upload_state(wl.x, wl.p)
    engs[1].initial_lab_boost()
    engs[1].state_save()
    b.run()
    x, p = engs[1].download_state()
    engs[1].state_restore()
    engs[1].run(wl.first_step, wl.steps)
    x2, p2 = engs[1].download_state()
    assert x.shape[1] == wl.n and np.array_equal(x, x2) and np.array_equal(p, p2)


def test_batch_autotuner_restores_state(lmb):
    wls = small_batch(lmb, "fp32", E=6)
    engs = make_engines(lmb, wls)
    before = [e.download_state() for e in engs]
    b = lmb.capi.Batch(0)
    for e, wl in zip(engs, wls):
        b.add(e, wl.first_step, wl.steps)
    shape, ms = b.tune()
    assert shape["block"] in (128, 256) and shape["chunk_steps"] in (64, 256, 1024, 0) and ms > 0
    assert b.shape() == shape
    for e, (x0, p0) in zip(engs, before):
        x, p = e.download_state()
        assert np.array_equal(x, x0) and np.array_equal(p, p0)


def test_batch_validation_and_nonfinite(lmb):
    capi = lmb.capi
    wls = small_batch(lmb, "fp32", E=3)
    engs = make_engines(lmb, wls)
    b = capi.Batch(0)
    b.add(engs[0], 1, wls[0].steps)
    with pytest.raises(capi.LimError, match="already in the batch"):
        b.add(engs[0], 1, 10)
    with pytest.raises(capi.LimError, match="block must be"):
        b.set_shape(block=96)
    odd = small_batch(lmb, "fp64", E=1)[0]
    e64 = capi.Engine(0)
    lmb.workloads.configure(e64, odd)
    b.add(e64, 1, odd.steps)
    with pytest.raises(capi.LimError, match="precision"):
        b.run()
    b.close()
    # NaN in one ensemble: reported with that ensemble and the step
    b = capi.Batch(0)
    for e, wl in zip(engs, wls):
        b.add(e, wl.first_step, wl.steps)
    wl = wls[2]
    wl.p[0, 3] = np.nan
    engs[2].upload_state(wl.x, wl.p)
    with pytest.raises(capi.LimError, match=r"NaN/Inf at step 1 \(ensemble 2\)") as ei:
        b.run()
    assert ei.value.code == capi.LIM_ERR_NONFINITE
