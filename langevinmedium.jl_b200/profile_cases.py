"""Small, self-contained cases of each kernel family, sized for an ncu capture (a few
hundred thousand particles, inputs above L2, a few GB on the device at most):

  python langevinmedium.jl_b200/profile_cases.py bjorken --n 262144 --steps 200
  python langevinmedium.jl_b200/profile_cases.py grid    --n 262144 --steps 200 [--fo]
  python langevinmedium.jl_b200/profile_cases.py adjoint --n 262144 --steps 256
  python langevinmedium.jl_b200/profile_cases.py batch   --ensembles 16
  python langevinmedium.jl_b200/profile_cases.py snapshots --n 1000000 --steps 1880 --save 20 [--compare]

Each prints its device time from the engine's own CUDA events.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["bjorken", "grid", "adjoint", "batch", "snapshots"])
    ap.add_argument("--save", type=int, default=20, help="snapshots: steps between saves")
    ap.add_argument("--compare", action="store_true",
                    help="snapshots: also time no snapshots and the host history (pageable and page-locked)")
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--fo", action="store_true", help="grid: freeze-out latch, particles stop")
    ap.add_argument("--ensembles", type=int, default=16)
    ap.add_argument("--precision", default="fp32")
    a = ap.parse_args()
    import __graft_entry__ as ge
    pkg = ge.load_package()
    W, capi = pkg.workloads, pkg.capi
    if a.case == "batch":
        wls = W.batch(E=a.ensembles, n_range=(1e3, 1e5), steps_range=(100, 400), grid_shape=(201, 201, 100))
        engs = []
        b = capi.Batch(0)
        for wl in wls:
            e = capi.Engine(0)
            W.configure(e, wl)
            e.initial_lab_boost()
            engs.append(e)
            b.add(e, wl.first_step, wl.steps)
        b.run()
        ms, nl, ps = b.stats()
        print(f"batch of {len(wls)}: {ms:.3f} ms, {nl} launches, {ps / (ms * 1e-3):.4g} particle-steps/s")
        return
    if a.case == "snapshots":
        # the Bjorken workload with a snapshot every --save steps, reduced on the device
        wl = W.bjorken(N=a.n, precision=a.precision, steps=a.steps)
        e = capi.Engine(0)
        W.configure(e, wl)
        e.initial_lab_boost()
        nslots = wl.steps // a.save + 1
        spec = capi.reduce_spec(100, 20.0, 100, 10.0)
        if not a.compare:
            e.run_reduced(wl.first_step, wl.steps, a.save, 0, nslots, spec)
            ms, nl = e.last_run_stats()
            print(f"snapshots N={a.n} steps={wl.steps} every {a.save}: {ms:.3f} ms, {nl} launches")
            return
        # wall-clock of the whole call (the copies are part of it), median of 3 after a warm-up
        import time
        import numpy as np
        e.state_save()
        size = nslots * a.n
        page = (np.zeros(size * 2), np.zeros(size * 3))
        pinned = (capi.pinned_empty(size * 2), capi.pinned_empty(size * 3))
        cases = {"none": lambda: e.run(wl.first_step, wl.steps),
                 "reduced": lambda: e.run_reduced(wl.first_step, wl.steps, a.save, 0, nslots, spec),
                 "history, page-locked": lambda: e.run(wl.first_step, wl.steps, a.save, 0, *pinned),
                 "history, pageable": lambda: e.run(wl.first_step, wl.steps, a.save, 0, *page)}
        for name, fn in cases.items():
            ts = []
            for r in range(4):
                e.state_restore()
                t = time.perf_counter()
                fn()
                if r:
                    ts.append(1e3 * (time.perf_counter() - t))
            print(f"{name}: {np.median(ts):.1f} ms ({nslots} snapshots, {size * 40 / 1e9:.2f} GB of history)")
        return
    if a.case == "bjorken":
        wl = W.bjorken(N=a.n, precision=a.precision, steps=a.steps)
    elif a.case == "grid":
        wl = W.grid2p1(N=a.n, precision=a.precision, steps=a.steps, freezeout=a.fo)
    else:
        wl = W.adjoint_grid(N=a.n, steps=a.steps)
    e = capi.Engine(0)
    W.configure(e, wl)
    e.initial_lab_boost()
    if a.case == "adjoint":
        e.state_save()
        e.run(1, wl.steps)
        f_ms = e.last_run_stats()[0]
        e.state_restore()
        e.adjoint(1, wl.steps, 64)
        af, ar = e.adjoint_stats()
        print(f"adjoint N={a.n} steps={wl.steps}: forward {f_ms:.3f} ms; checkpointed forward {af:.3f} + "
              f"reverse {ar:.3f} ms = {(af + ar) / f_ms:.2f} x forward")
        return
    e.run(1, wl.steps)
    ms, nl = e.last_run_stats()
    print(f"{a.case} {a.precision} N={a.n} steps={wl.steps}: {ms:.3f} ms, {nl} launches, "
          f"{wl.particle_steps / (ms * 1e-3):.4g} particle-steps/s")


if __name__ == "__main__":
    main()
