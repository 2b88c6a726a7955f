"""Many ensembles through the engine with their host <-> device copies hidden.

A host that simulates a sequence of ensembles (events, parameter points, batches of
a large sample) one ``simulate_ensemble_bulk`` call at a time pays, per ensemble, the
upload of its initial state and the download of its results on top of the run: for
the 2+1D grid workload (1e7 particles, FP64 host arrays in the reference's
column-major layout) 400 MB in and 560 MB out, about 16 ms over PCIe against a
92 ms run.  ``EnsembleStream`` keeps two slots of engine contexts, each on its own
CUDA stream: while the ensemble of pass k runs in one slot, the other slot downloads
the outputs of pass k - 1 and uploads (and boosts to the lab frame) the initial state
of pass k + 1, so the copies go through the copy engines under the run.  Runs never
overlap: pass k + 1 starts when pass k has finished.  A slot holds one context per
*lane* (an ensemble shape, e.g. one heavy-quark species); the lanes of a pass run
concurrently, as separate ``simulate_ensemble_bulk`` calls on separate streams would.

Every call goes through the C-ABI (``capi.Engine``); the C calls release the GIL, so
one host thread per (slot, lane) keeps each stream fed.  A pass's results are those
of the same ensemble run alone (the contexts of a lane are configured alike and a
particle's noise depends only on its id and step).
"""
from __future__ import annotations

import threading
from typing import Callable, Sequence

from . import capi


def run_concurrently(fns: Sequence[Callable[[], None]]) -> None:
    """Run the callables on one host thread each and re-raise the first failure."""
    errs: list[BaseException] = []

    def wrap(f):
        try:
            f()
        except BaseException as e:        # noqa: BLE001 - re-raised below
            errs.append(e)

    ts = [threading.Thread(target=wrap, args=(f,)) for f in fns]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]


class EnsembleStream:
    """Two slots of engine contexts, one context per lane in each.

    ``engines[slot][lane]``: configured contexts (parameters, medium, transport
    tables), each on its own stream; the two contexts of a lane must be configured
    alike.  The stream uses them and leaves them open.  ``run`` advances ``npasses``
    ensembles: ``load(k, lane, eng)`` puts pass k's initial state into ``eng``
    (upload and step-0 boost), ``unload(k, lane, eng)`` reads its results after the
    run of ``nsteps`` steps from ``first_step``.
    """

    SLOTS = 2

    def __init__(self, engines: Sequence[Sequence[capi.Engine]]):
        if len(engines) != self.SLOTS or not engines[0] or len(engines[0]) != len(engines[1]):
            raise ValueError("EnsembleStream: two slots with the same number (>= 1) of lanes")
        if len({id(e) for row in engines for e in row}) != 2 * len(engines[0]):
            raise ValueError("EnsembleStream: every (slot, lane) needs its own context")
        self.engines = [list(row) for row in engines]
        self.lanes = len(engines[0])

    def run(self, npasses: int, first_step: int, nsteps: int,
            load: Callable[[int, int, capi.Engine], None],
            unload: Callable[[int, int, capi.Engine], None]) -> None:
        if npasses <= 0:
            return
        E, L = self.engines, range(self.lanes)
        run_concurrently([lambda l=l: load(0, l, E[0][l]) for l in L])
        for k in range(npasses):
            cur, other = E[k % 2], E[(k + 1) % 2]

            def turnover(l, k=k, other=other):
                # the other slot: results of pass k - 1 out, initial state of pass k + 1 in
                if k >= 1:
                    unload(k - 1, l, other[l])
                if k + 1 < npasses:
                    load(k + 1, l, other[l])

            run_concurrently([lambda l=l, cur=cur: cur[l].run(first_step, nsteps) for l in L] +
                             [lambda l=l: turnover(l) for l in L])
        last = E[(npasses - 1) % 2]
        run_concurrently([lambda l=l: unload(npasses - 1, l, last[l]) for l in L])
