"""The schedule of pipeline.EnsembleStream, on stand-in contexts (no GPU): each pass
is loaded before its run and unloaded after it, in its own slot; the runs of two
passes never overlap; the copies of passes k - 1 and k + 1 happen during run k."""
import threading
import time

import pytest


class FakeEngine:
    def __init__(self, log, slot, lane):
        self.log, self.slot, self.lane = log, slot, lane
        self.lock = threading.Lock()

    def run(self, first_step, nsteps):
        self.log.append(("run+", self.slot, self.lane, time.perf_counter()))
        time.sleep(0.02)
        self.log.append(("run-", self.slot, self.lane, time.perf_counter()))


@pytest.mark.parametrize("npasses", [1, 2, 5])
def test_stream_schedule(lmb, npasses):
    log = []
    E = [[FakeEngine(log, s, l) for l in range(2)] for s in range(2)]
    state = {}                        # (slot, lane) -> pass held

    def load(k, lane, eng):
        assert eng is E[k % 2][lane]
        state[(eng.slot, lane)] = k
        log.append(("load", k, lane, time.perf_counter()))

    def unload(k, lane, eng):
        assert eng is E[k % 2][lane] and state[(eng.slot, lane)] == k
        log.append(("unload", k, lane, time.perf_counter()))

    lmb.pipeline.EnsembleStream(E).run(npasses, 1, 10, load, unload)
    loads = sorted((e[1], e[2]) for e in log if e[0] == "load")
    unloads = sorted((e[1], e[2]) for e in log if e[0] == "unload")
    assert loads == unloads == [(k, l) for k in range(npasses) for l in range(2)]
    # runs: one per (pass, lane), slot k % 2, and pass k + 1 starts after pass k ended
    starts = [e for e in log if e[0] == "run+"]
    ends = [e for e in log if e[0] == "run-"]
    assert len(starts) == len(ends) == 2 * npasses
    for k in range(npasses):
        sk = [e for e in starts[2 * k:2 * k + 2]]
        assert {e[1] for e in sk} == {k % 2}
        if k:
            prev_end = max(e[3] for e in ends[2 * (k - 1):2 * k])
            assert min(e[3] for e in sk) >= prev_end
    t_load = {(e[1], e[2]): e[3] for e in log if e[0] == "load"}
    t_unload = {(e[1], e[2]): e[3] for e in log if e[0] == "unload"}
    for k in range(npasses):
        run_start = min(e[3] for e in starts[2 * k:2 * k + 2])
        run_end = max(e[3] for e in ends[2 * k:2 * k + 2])
        for l in range(2):
            assert t_load[(k, l)] <= run_start and t_unload[(k, l)] >= run_end
            if k + 1 < npasses:       # the next pass is loaded while this one runs
                assert t_load[(k + 1, l)] < run_end


def test_stream_needs_distinct_contexts(lmb):
    log = []
    e = FakeEngine(log, 0, 0)
    with pytest.raises(ValueError):
        lmb.pipeline.EnsembleStream([[e], [e]])
    with pytest.raises(ValueError):
        lmb.pipeline.EnsembleStream([[e], []])
