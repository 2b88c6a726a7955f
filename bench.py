#!/usr/bin/env python
"""Throughput of the fused heavy-quark Langevin step on B200.

Headline workload (one benchmark "step" = one full simulation pass): the 2+1D
hydro-like grid medium, 201 x 201 cells at 0.1 fm with 100 tau slices (0.6 -> 10
fm/c), T0 = 0.45 GeV elliptic Gaussian (sigma_x 3.0, sigma_y 2.4 fm) decaying as
(tau0/tau)^(1/3), radial flow u^r = tanh(0.05 r (tau - tau0)); 5e6 charm (1.5 GeV) plus
5e6 bottom (4.75 GeV) quarks per GPU, positions from the squared Gaussian profile, p_T
power law, Langevin (2 pi T D_s = 4) plus RTA (tau_R = 5 eta/s / T), Bjorken redshift,
trilinear medium, freeze-out latch at T < 0.155 GeV with particles stopping there,
dt = 0.01 fm/c (940 steps), FP32 arithmetic.  Synthetic seeded inputs.  The two
species are two engine contexts on two CUDA streams, advanced concurrently.

  value : executed particle-steps/s over all GPUs (a particle's steps up to its
          freeze-out), the state resident in HBM (restored from a device checkpoint
          before every pass, outside the timed region); L2 flushed between passes.
  e2e   : the same through the C-ABI from page-locked host buffers: upload, step-0
          boost, run, download of the freeze-out outputs, every pass.
  accuracy / cpu_baseline : the FP64 CPU restatement (oracle/) on a sample of the same
          particles with the same noise: its throughput on the host cores, and the
          engine's FP32 and FP64 error against it.
  sub-legs (one-GPU run): the same workload in FP64, the Bjorken workload, the batched
          persistent launch of 256 ensembles against 256 separate runs, and the
          forward+adjoint cost against the plain forward.

`--impl reference` times the reference's CPU algorithm (the FP64 restatement, all host
threads) on a bounded sample of the same workload.  Multi-GPU (torchrun): every rank
runs its own 1e7 particles (weak scaling, global particle ids from
langevinmedium.jl_b200/sharding.py, no data-path collective); timing is the max over
ranks.  `--case` runs one small kernel case for a profiler capture; `--cpu-table` times
the restatement on configurations 0-2 at one and at every host thread.
"""
from __future__ import annotations

import argparse
import copy
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s on 1 B200 (plain vs batched; fwd+adjoint cost) at ≤1e-5 rel err"
WORKLOAD = "grid2p1_langevin_rta_fo_5e6c_5e6b_fp32"
SPECIES = ((1.5, "charm"), (4.75, "bottom"))
HBM_FALLBACK_GBS = 6650.0
LIVE_SUBCHUNK_STEPS = 32          # steps per launch of a stop-at-freeze-out run (the live list's sub-chunk)


def load_package():
    import __graft_entry__ as ge
    return ge.load_package()


def measured_peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "MEASURED_PEAKS.json (measured on this pool)"
    return {"hbm_gbs": HBM_FALLBACK_GBS}, "fallback (no MEASURED_PEAKS.json)"


# ---------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons, power = [], None, set(), []
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------------
# the headline workload, per rank
# ---------------------------------------------------------------------------------
def headline_workloads(pkg, n_total: int, rank: int, world: int, *, precision: str = "fp32", fields=None):
    """The rank's share of the headline ensemble as one workload per species.  Global
    particle ids come from sharding.shard over all ranks' particles: rank r holds ids
    [first, first + count), the charm quarks first, so a particle's noise does not depend
    on the sharding."""
    W = pkg.workloads
    fields = fields or W.grid2p1_fields()
    first, count = pkg.sharding.shard(n_total, rank, world)
    n_c = count // 2
    out = []
    for k, (m, _) in enumerate(SPECIES):
        n = n_c if k == 0 else count - n_c
        wl = W.grid2p1(N=n, m=m, fields=fields, precision=precision, rng_seed=3 + 10 * k + 100 * rank)
        wl.params["particle_offset"] = first + (0 if k == 0 else n_c)
        out.append(wl)
    return out


def sample_of(wl, n: int):
    """The first n particles of a workload (same particle ids, so the same noise)."""
    s = copy.copy(wl)
    s.params = dict(wl.params)
    s.x = np.ascontiguousarray(wl.x[:, :n])
    s.p = np.ascontiguousarray(wl.p[:, :n])
    return s


def executed_steps(flag, tau, t0: float, dt: float, steps: int) -> float:
    """Steps a stop-at-freeze-out run advances: a particle latched at step s (its tau in
    (t0 + (s-1) dt, t0 + s dt]) ran s steps, one never latched all of them."""
    st = np.where(np.asarray(flag) != 0, np.ceil((np.asarray(tau) - t0) / dt - 1e-9), steps)
    return float(np.clip(st, 0, steps).sum())


def reduce_over_ranks(vals: dict, world: int, device: str) -> dict:
    """The job's figures from every rank's: times (keys ending in _ms) are the max over
    ranks, counts and observable sums the sum.  One all-reduce of each kind, in a fixed
    order on every rank."""
    import torch
    import torch.distributed as dist
    times = sorted(k for k in vals if k.endswith("_ms"))
    sums = sorted(k for k in vals if not k.endswith("_ms"))
    out = dict(vals)
    if world == 1:
        return out
    t = torch.tensor([float(vals[k]) for k in times], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    flat = [np.atleast_1d(np.asarray(vals[k], dtype=np.float64)) for k in sums]
    u = torch.tensor(np.concatenate(flat), dtype=torch.float64, device=device)
    dist.all_reduce(u)
    for k, v in zip(times, t.cpu().numpy()):
        out[k] = float(v)
    off = 0
    for k, a in zip(sums, flat):
        r = u[off:off + a.size].cpu().numpy()
        out[k] = float(r[0]) if np.ndim(vals[k]) == 0 else r
        off += a.size
    return out


def concurrently(fns):
    """Run the callables on one host thread each (the C-ABI calls release the GIL, so
    each context's stream is fed while the others wait on theirs); re-raise failures."""
    errs = []

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


def device_span(streams, body) -> float:
    """ms between an event recorded on streams[0] before body() and one recorded after
    every stream's work of body() (the others wait on the first event and are joined)."""
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e0.record(streams[0])
    for s in streams[1:]:
        s.wait_event(e0)
    body()
    for s in streams[1:]:
        ev = torch.cuda.Event()
        ev.record(s)
        streams[0].wait_event(ev)
    e1 = torch.cuda.Event(enable_timing=True)
    e1.record(streams[0])
    e1.synchronize()
    return e0.elapsed_time(e1)


# ---------------------------------------------------------------------------------
# the CPU restatement: the reference arm, the CPU baseline and the accuracy leg
# ---------------------------------------------------------------------------------
def oracle_run(wl, threads: int):
    """The FP64 restatement on a workload (initial lab boost, then the run); returns
    (seconds of the run, executed particle-steps, output dict)."""
    from oracle import oracle as orc
    P = orc.make_params(**dict(wl.params, precision=0))
    med = wl.medium
    md = orc.Medium()
    if med["kind"] == "rt":
        md.rt(med["xgrid"], med["tgrid"], med["T"], med["V"], med.get("V2"))
    elif med["kind"] == "bjorken":
        md.bjorken(med["T0"], med["tau0"], med["power"], med["r_max"])
    else:
        md.grid(med["T"], med["ux"], med["uy"], med["x0"], med["dx"], med["y0"], med["dy"], med["tau0"], med["dtau"])
    for w, (a, b, v) in wl.splines.items():
        md.spline(w, a, b, v)
    if wl.invcdf is not None:
        md.invcdf(*wl.invcdf)
    x0, p0 = orc.initial_lab_boost(P, md, wl.x, wl.p)
    t = time.perf_counter()
    out = orc.run(P, md, x0, p0, wl.first_step, wl.steps, threads=threads)
    dt = time.perf_counter() - t
    if P.freezeout_capture and P.stop_after_freezeout:
        ex = executed_steps(out["fo_flag"], out["fo_tau"], wl.params["t0"], wl.params["dt"], wl.steps)
    else:
        ex = float(wl.n * wl.steps)
    return dt, ex, out


def cpu_pass(wls, threads: int):
    """One pass of the restatement over the workloads: (seconds, executed
    particle-steps, outputs)."""
    tot_s, tot_ps, outs = 0.0, 0.0, []
    for wl in wls:
        s, ps, out = oracle_run(wl, threads)
        tot_s += s
        tot_ps += ps
        outs.append(out)
    return tot_s, tot_ps, outs


def size_cpu_sample(pkg, target_s: float, threads: int, fields) -> int:
    """Particles per species for ~target_s seconds of one restatement pass."""
    n0 = 1024 * max(1, threads)
    wls = [sample_of(w, n0) for w in headline_workloads(pkg, 2 * n0, 0, 1, precision="fp64", fields=fields)]
    s, _, _ = cpu_pass(wls, threads)
    return max(512, int(n0 * target_s / max(s, 1e-3)))


def per_particle_err(a, b, scale, floor):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.ndim == 1:
        a, b = a[None, :], b[None, :]
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), floor * scale)


def accuracy_against_cpu(pkg, samples, cpu_outs) -> dict:
    """The engine in FP32 and FP64 on the CPU sample's particles (same ids, same noise)
    against the restatement's FP64 result.  Per particle ||a - b|| / max(||b||, f s),
    s = 0.3 GeV for momenta and 1 fm for positions and times, f = 1e-3 (the strict
    floor) and 1: the final state of particles live in both runs, the freeze-out
    outputs (position, momentum, tau) of particles latched in both; a particle's error
    is the largest of its quantities'.  A particle off by more than 1e-2 (floor 1) has
    diverged: a decision (an RTA collision, a freeze-out crossing) fell within the two
    trajectories' difference of its threshold and went the other way, after which the
    trajectories are different draws.  Those are counted, and the maxima are also
    given over the particles that did not diverge."""
    W, capi = pkg.workloads, pkg.capi
    res = {"sample": f"{samples[0].n} charm + {samples[1].n} bottom quarks of the headline workload, 940 steps",
           "metric": "per-particle relative error, max / 99.99th / 99th percentile"}
    for prec in ("fp32", "fp64"):
        errs = {1e-3: {"live": [], "latch": []}, 1.0: {"live": [], "latch": []}}
        flips = 0
        for wl, o in zip(samples, cpu_outs):
            w = sample_of(wl, wl.n)
            w.params["precision"] = capi.LIM_FP32 if prec == "fp32" else capi.LIM_FP64
            e = capi.Engine(0)
            W.configure(e, w)
            e.initial_lab_boost()
            e.run(w.first_step, w.steps)
            x, p = e.download_state()
            f = e.download_freezeout()
            e.close()
            gf, of = f["flag"], o["fo_flag"]
            flips += int(np.sum(gf != of))
            live, both = (gf == 0) & (of == 0), (gf == 1) & (of == 1)
            for fl in errs:
                errs[fl]["live"].append(np.maximum(per_particle_err(p[:, live], o["p"][:, live], 0.3, fl),
                                                   per_particle_err(x[:, live], o["x"][:, live], 1.0, fl)))
                errs[fl]["latch"].append(np.maximum.reduce([
                    per_particle_err(f["mom"][:, both], o["fo_mom"][:, both], 0.3, fl),
                    per_particle_err(f["pos"][:, both], o["fo_pos"][:, both], 1.0, fl),
                    per_particle_err(f["tau"][both], o["fo_tau"][both], 1.0, fl)]))
        out = {"freezeout_flag_mismatches": flips}
        kept = {}
        for k in ("live", "latch"):
            e1 = np.concatenate(errs[1.0][k]) if errs[1.0][k] else np.zeros(0)
            kept[k] = e1 <= 1e-2
            out[f"diverged_{k}"] = int((~kept[k]).sum())
        for fl, d in errs.items():
            for k, parts in d.items():
                e = np.concatenate(parts) if parts else np.zeros(0)
                if e.size == 0:
                    e = np.zeros(1)
                    ok = np.ones(1, bool)
                else:
                    ok = kept[k]
                out[f"{k}_floor{fl:g}"] = [float(e.max()), float(np.percentile(e, 99.99)), float(np.percentile(e, 99))]
                out[f"{k}_floor{fl:g}_max_not_diverged"] = float(e[ok].max()) if ok.any() else 0.0
        res[f"{prec}_vs_fp64_cpu"] = out
    return res


def run_reference(args, rank: int, world: int):
    """The reference arm: the FP64 restatement of the reference's CPU algorithm on a
    bounded sample of the headline workload (both species), all host threads."""
    if rank != 0:
        return
    pkg = load_package()
    from oracle import oracle as orc
    threads = orc.max_threads()
    fields = pkg.workloads.grid2p1_fields()
    n = size_cpu_sample(pkg, 4.0, threads, fields)
    wls = [sample_of(w, n) for w in headline_workloads(pkg, 2 * n, 0, 1, precision="fp64", fields=fields)]
    small = [sample_of(w, max(256, n // 8)) for w in wls]
    for _ in range(args.warmup):
        cpu_pass(small, threads)
    total_s, total_ps = 0.0, 0.0
    for _ in range(args.steps):
        s, ps, _ = cpu_pass(wls, threads)
        total_s += s
        total_ps += ps
    value = total_ps / total_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sample of the headline workload)",
        "config": {"workload": WORKLOAD, "particles_per_step_sample": 2 * n, "steps_per_pass": wls[0].steps,
                   "note": "the reference is Julia, absent from the image and from the GPU box; this arm times its "
                           "CPU algorithm as the C FP64 restatement under oracle/ on all host threads, executed "
                           "particle-steps (particles stop at freeze-out) as in the engine's arm"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{n} charm + {n} bottom quarks x 940 steps (stop at freeze-out) per timed step"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_table(args):
    """The CPU restatement's throughput on the benchmark configurations, at one thread
    and at every host thread: the static box (config 0), the Bjorken table (config 1)
    and the headline 2+1D grid workload (config 2, particles stop at freeze-out);
    samples sized for a few seconds each, median of 3.  One JSON line."""
    pkg = load_package()
    from oracle import oracle as orc
    W = pkg.workloads
    nproc = orc.max_threads()
    fields = W.grid2p1_fields()
    cases = {
        "config0_static_box_fp64": lambda n: [W.static_box(N=n, precision="fp64")],
        "config1_bjorken_langevin_rta_fp64": lambda n: [W.bjorken(N=n, precision="fp64", rng_seed=2)],
        "config2_grid2p1_langevin_rta_fo_fp64": lambda n: [sample_of(w, n) for w in headline_workloads(
            pkg, 2 * n, 0, 1, precision="fp64", fields=fields)],
    }
    out = {"impl": "reference-cpu-table", "unit": "particle-steps/s", "nproc": nproc,
           "note": "the reference is Julia (not on this machine): its CPU algorithm as the C FP64 restatement "
                   "(oracle/), one process; config 2 counts executed particle-steps (stop at freeze-out)"}
    for name, make in cases.items():
        row = {}
        for th in (1, nproc):
            n = 256 * th
            s, _, _ = cpu_pass(make(n), th)
            n = max(256, int(n * args.cpu_seconds / max(s, 1e-3)))
            vals = []
            for _ in range(3):
                s, ps, _ = cpu_pass(make(n), th)
                vals.append(ps / s)
            row[f"threads_{th}"] = {"value": statistics.median(vals), "particles": n * len(make(1)),
                                    "runs": 3, "statistic": "median"}
        out[name] = row
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------------
# roofline
# ---------------------------------------------------------------------------------
def work_counts(pkg, key: str):
    wm = json.loads((Path(pkg.__file__).parent / "work_model.json").read_text())
    w = wm["workloads"][key]
    tot = {}
    for item in w["items"].values():
        for k, c in item.items():
            tot[k] = tot.get(k, 0.0) + c
    return tot, sum(tot.values()), w["hbm_bytes_per_particle_per_launch"]


def per_pipe_roofline(counts, fma_rate, mufu_rate, particle_steps, kernel_s):
    """The work model's per-pipe bound (time per particle-step = count / pipe rate, the
    roofline time the largest of them): FP32 on the FMA pipe and every instruction on
    issue at the measured FMA rate; MUFU and conversions on the XU pipe at the measured
    MUFU rate; integer, FP64 and memory instructions at the B200 SM's nominal lane
    ratios to the FMA pipe (64, 64 and 32 of 128 per clock)."""
    total = sum(counts.values())
    rates = {"issue": (total, fma_rate), "fp32": (counts.get("fp32", 0.0), fma_rate),
             "xu": (counts.get("mufu", 0.0) + counts.get("conv", 0.0), mufu_rate),
             "int": (counts.get("int", 0.0), fma_rate / 2), "fp64": (counts.get("fp64", 0.0), fma_rate / 2),
             "mem": (counts.get("mem", 0.0), fma_rate / 4)}
    t = {k: c / r for k, (c, r) in rates.items()}
    bound = max(t, key=t.get)
    return {"time_per_particle_step_ns": {k: v * 1e9 for k, v in t.items()}, "bound": bound,
            "frac": t[bound] * particle_steps / kernel_s,
            "rates_thread_instr_per_s": {k: r for k, (c, r) in rates.items()},
            "note": "XU count includes the conversions; ALU/FP64/LSU rates nominal ratios of the measured FMA rate"}


def issue_roofline(pkg, key, fma_rate, mufu_rate, particle_steps, seconds, n_particles, launches,
                   live_steps=None):
    """launches: step-kernel launches per particle over the pass; live_steps: for runs on
    a compacted live list, the steps of one sub-chunk launch (each launch reads and
    writes the state of the particles live in it once, so the algorithmic bytes are the
    per-launch figure per live particle times executed particle-steps / live_steps)."""
    counts, i_alg, hbm_pp = work_counts(pkg, key)
    achieved = i_alg * particle_steps / seconds
    peaks, src = measured_peaks()
    if live_steps:
        bytes_total = hbm_pp * particle_steps / live_steps
    else:
        bytes_total = hbm_pp * n_particles * max(1, launches)
    return {
        "bound": "issue", "unit": "Ginst/s", "achieved": achieved / 1e9, "peak": fma_rate / 1e9,
        "frac": achieved / fma_rate, "traffic": None,
        "algorithmic_inst_per_particle_step": i_alg, "inst_mix_per_particle_step": counts,
        "peak_source": "measured in this run: FP32 FMA issue probe (lim_probe_fma_rate), thread-instr/s",
        "per_pipe": per_pipe_roofline(counts, fma_rate, mufu_rate, particle_steps, seconds),
        "hbm": {"algorithmic_bytes": bytes_total, "achieved_gbs": bytes_total / seconds / 1e9,
                "peak_gbs": float(peaks["hbm_gbs"]), "peak_source": src},
    }


# ---------------------------------------------------------------------------------
# sub-legs of the metric (one-GPU run)
# ---------------------------------------------------------------------------------
TUNED = ROOT / "langevinmedium.jl_b200" / "tuned_shapes.json"


def bench_batched(pkg, args, flush):
    """256 ensembles (1e3-1e6 particles, charm/bottom, 2piT Ds in [2, 8], 500-2000 steps
    capped to the media's tau range, half Bjorken, half 2+1D grids): one batched run
    (graph of persistent chunk launches) against the same ensembles as 256 lim_run calls
    back to back."""
    import torch
    W, capi = pkg.workloads, pkg.capi
    wls = W.batch(E=256)
    engs = []
    for wl in wls:
        e = capi.Engine(0)
        W.configure(e, wl)
        e.initial_lab_boost()
        e.state_save()
        engs.append(e)
    ps = sum(w.n * w.steps for w in wls)
    reps = max(1, min(args.steps, 3))

    def restore():
        for e in engs:
            e.state_restore()
        for e in engs:
            e.synchronize()

    sep_wall, sep_dev = [], []
    for r in range(reps + 1):
        restore()
        flush.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        dev = 0.0
        for e, wl in zip(engs, wls):
            e.run(wl.first_step, wl.steps)
            dev += e.last_run_stats()[0]
        wall = time.perf_counter() - t
        if r:                                            # the first pass is the warm-up
            sep_wall.append(wall)
            sep_dev.append(dev)
    b = capi.Batch(0)
    for e, wl in zip(engs, wls):
        b.add(e, wl.first_step, wl.steps)
    props = torch.cuda.get_device_properties(0)
    key = f"{props.name}|sm{props.multi_processor_count}|batch256-rng4-tau10"
    cache = json.loads(TUNED.read_text()) if TUNED.exists() else {}
    tuned_now = key not in cache
    if tuned_now:
        shape, _ = b.tune()
    else:
        shape = cache[key]["shape"]
        b.set_shape(**shape)
    bat_wall, bat_dev = [], []
    launches = 0
    for r in range(reps + 1):
        restore()
        flush.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        b.run()
        wall = time.perf_counter() - t
        ms, nl, _ = b.stats()
        if r:
            bat_wall.append(wall)
            bat_dev.append(ms)
            launches += nl
    b.close()
    for e in engs:
        e.close()
    sep_v, bat_v = ps / statistics.median(sep_wall), ps / statistics.median(bat_wall)
    return {
        "workload": "batch of 256 ensembles: counts log-uniform in [1e3, 1e6], m in {1.5, 4.75} GeV, "
                    "2piT Ds ~ U[2, 8], half Bjorken (dtau 0.005, 500-1880 steps), half 2+1D grids 201x201x100 "
                    "(T0 ~ U[0.35, 0.55] GeV, sy/sx ~ U[0.7, 1], dt 0.01, 500-940 steps: the grid's tau range), "
                    "Langevin+RTA, FP32",
        "particles": sum(w.n for w in wls), "particle_steps": ps, "unit": "particle-steps/s",
        "value": bat_v, "separate_value": sep_v, "speedup": bat_v / sep_v,
        "value_device": ps / (statistics.median(bat_dev) * 1e-3),
        "separate_value_device": ps / (statistics.median(sep_dev) * 1e-3),
        "timing": "wall clock around one lim_batch_run (one CUDA-graph replay) vs around 256 lim_run calls; "
                  "value_device: CUDA events of the graph vs the sum of the runs' event times; median of "
                  f"{reps} after one warm-up, L2 flushed before each",
        "shape": shape, "shape_source": "autotuned in this run (lim_batch_tune)" if tuned_now else
                                         "autotuner result cached in langevinmedium.jl_b200/tuned_shapes.json",
        "shape_key": key, "gpu_launches_per_run": launches // reps, "separate_launches_per_run": 2 * len(wls),
    }


def bench_adjoint(pkg, args):
    """Forward + adjoint cost on the differentiation workload (2+1D grid, 1e6 charm,
    2000 steps of 0.0047 fm/c spanning the grid's tau range, checkpoints every 64 steps)
    against the plain forward."""
    W, capi = pkg.workloads, pkg.capi
    wl = W.adjoint_grid(N=1_000_000, steps=2000)
    e = capi.Engine(0)
    W.configure(e, wl)
    e.initial_lab_boost()
    e.state_save()
    reps = max(1, min(args.steps, 3))
    fwd, adj, fparts, rparts = [], [], [], []
    for r in range(reps + 1):
        e.state_restore()
        e.run(1, wl.steps)
        f_ms = e.last_run_stats()[0]
        e.state_restore()
        obs, G = e.adjoint(1, wl.steps, checkpoint_every=64)
        a_f, a_r = e.adjoint_stats()
        if r:
            fwd.append(f_ms)
            adj.append(a_f + a_r)
            fparts.append(a_f)
            rparts.append(a_r)
    e.close()
    f_ms, a_ms = statistics.median(fwd), statistics.median(adj)
    return {
        "workload": f"2+1D grid medium, 1e6 charm, 2000 steps (dt {wl.params['dt']}), Langevin+RTA, FP32; d/d(a, b, s) "
                    "of <pT>, <cos 2phi>, smoothed fraction pT > 5 GeV; 2piT Ds = a + b (T/0.155 - 1), a=3, b=2, s=1",
        "checkpoint_every": 64, "plain_forward_ms": f_ms, "forward_plus_adjoint_ms": a_ms,
        "checkpointed_forward_ms": statistics.median(fparts), "reverse_sweep_ms": statistics.median(rparts),
        "cost_ratio": a_ms / f_ms, "obs": obs.tolist(), "grad": G.tolist(),
        "timing": f"CUDA events, median of {reps} after one warm-up",
    }


def bench_bjorken(pkg, args, fma_rate, mufu_rate):
    """The Bjorken workload (reference (r, t) table 41 x 1883, 1e6 charm x 1880 steps,
    Langevin+RTA, redshift) in FP32 and FP64: CUDA events, median of 3 after one warm-up."""
    W, capi = pkg.workloads, pkg.capi
    out = {"workload": "Bjorken T(tau) = 0.40 (0.6/tau)^(1/3) GeV as an (r, t) table, 1e6 charm, dtau 0.005 "
                       "(1880 steps), Langevin+RTA, redshift"}
    for prec in ("fp32", "fp64"):
        wl = W.bjorken(N=1_000_000, precision=prec, rng_seed=2)
        e = capi.Engine(0)
        W.configure(e, wl)
        e.initial_lab_boost()
        e.state_save()
        ms = []
        for r in range(4):
            e.state_restore()
            e.run(wl.first_step, wl.steps)
            if r:
                ms.append(e.last_run_stats()[0])
        e.close()
        t = statistics.median(ms)
        leg = {"value": wl.n * wl.steps / (t * 1e-3), "unit": "particle-steps/s", "ms_per_pass": t}
        if prec == "fp32":
            leg["roofline"] = issue_roofline(pkg, "bjorken_langevin_rta_fp32", fma_rate, mufu_rate,
                                             wl.n * wl.steps, t * 1e-3, wl.n, 1)
        out[prec] = leg
    return out


# ---------------------------------------------------------------------------------
# the headline arm
# ---------------------------------------------------------------------------------
class Species:
    """One species of the rank's share: an engine context on its own stream."""

    def __init__(self, pkg, wl, device: int, stream):
        self.wl = wl
        self.stream = stream
        self.eng = pkg.capi.Engine(device=device, stream=stream.cuda_stream)
        pkg.workloads.configure(self.eng, wl)
        self.eng.initial_lab_boost()
        self.eng.state_save()

    def run(self):
        self.eng.run(self.wl.first_step, self.wl.steps)


def measure_headline(pkg, args, rank, world, local_rank, precision="fp32", fields=None, e2e=True, flush=None):
    """Passes of the headline workload on this rank.  Every rank takes the same
    collective steps."""
    import torch
    import torch.distributed as dist
    capi = pkg.capi
    wls = headline_workloads(pkg, world * args.particles, rank, world, precision=precision, fields=fields)
    streams = [torch.cuda.Stream() for _ in wls]
    sp = [Species(pkg, wl, local_rank, s) for wl, s in zip(wls, streams)]
    torch.cuda.synchronize()

    def prepare():
        for s in sp:
            s.eng.state_restore()
        if flush is not None:
            flush.zero_()                                # > L2, between timed passes, not timed
        torch.cuda.synchronize()

    def one_pass():
        concurrently([s.run for s in sp])

    for _ in range(args.warmup):
        prepare()
        one_pass()
    if world > 1:
        dist.barrier()
    pass_ms, launches = [], 0
    for _ in range(args.steps):
        prepare()
        pass_ms.append(device_span(streams, one_pass))
        launches += sum(s.eng.last_run_stats()[1] for s in sp)
    executed = 0.0
    for s in sp:
        f = s.eng.download_freezeout()
        executed += executed_steps(f["flag"], f["tau"], s.wl.params["t0"], s.wl.params["dt"], s.wl.steps)
    sums = np.zeros(capi.LIM_OBS_NUM)
    for s in sp:
        sums += s.eng.observables(from_freezeout=True)["sums"]
    res = {"pass_ms": pass_ms, "launches": launches, "executed": executed,
           "nominal": float(sum(w.n * w.steps for w in wls)), "n": sum(w.n for w in wls), "fo_sums": sums}
    if e2e:
        # the same passes through the C-ABI from page-locked host buffers: upload, step-0
        # boost, run, freeze-out outputs back, every pass.  Streamed (the headline e2e):
        # two slots of contexts (pipeline.EnsembleStream), the copies of the passes before
        # and after overlapping each run; serial: one pass after the other.
        host = []
        for s in sp:
            w = s.wl
            dims, pdim, n = int(w.params["dims"]), int(w.params["pdim"]), w.n
            xb = capi.pinned_empty(n * dims)
            pb = capi.pinned_empty(n * pdim)
            xb[:] = capi.julia_layout(w.x, dims)
            pb[:] = capi.julia_layout(w.p, pdim)
            outs = [[capi.pinned_empty(n * dims), capi.pinned_empty(n * pdim), capi.pinned_empty(n),
                     capi.pinned_empty(n)] for _ in range(2)]
            host.append((xb, pb, outs, n))

        def load(k, lane, eng):
            xb, pb, _, n = host[lane]
            eng.upload_state_flat(xb, pb, n)
            eng.initial_lab_boost()

        def unload(k, lane, eng):
            eng.download_freezeout_flat(*host[lane][2][k % 2])

        def e2e_one(s, lane):
            load(0, lane, s.eng)
            s.run()
            unload(0, lane, s.eng)

        def e2e_pass():
            concurrently([lambda s=s, l=l: e2e_one(s, l) for l, s in enumerate(sp)])

        for _ in range(max(1, args.warmup // 2)):
            e2e_pass()
        if world > 1:
            dist.barrier()
        e2e_ms = []
        for _ in range(args.steps):
            if flush is not None:
                flush.zero_()
            torch.cuda.synchronize()
            e2e_ms.append(device_span(streams, e2e_pass))
        res["e2e_serial_ms"] = e2e_ms
        # the second slot: contexts configured like the first, on streams of their own
        streams2 = [torch.cuda.Stream() for _ in wls]
        sp2 = [Species(pkg, wl, local_rank, st) for wl, st in zip(wls, streams2)]
        ens = pkg.pipeline.EnsembleStream([[s.eng for s in sp], [s.eng for s in sp2]])
        wl0 = wls[0]
        ens.run(2, wl0.first_step, wl0.steps, load, unload)          # warm-up of both slots
        if world > 1:
            dist.barrier()
        if flush is not None:
            flush.zero_()
        torch.cuda.synchronize()
        res["e2e_ms"] = device_span(streams + streams2,
                                    lambda: ens.run(args.steps, wl0.first_step, wl0.steps, load, unload))
        for s in sp2:
            s.eng.close()
        res["h2d"] = int(sum(h[0].nbytes + h[1].nbytes for h in host))
        res["d2h"] = int(sum(sum(o.nbytes for o in h[2][0]) for h in host))
    for s in sp:
        s.eng.close()
    return res


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    pkg = load_package()
    W, capi = pkg.workloads, pkg.capi
    fields = W.grid2p1_fields()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")   # > 126 MB L2
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    h = measure_headline(pkg, args, rank, world, local_rank, "fp32", fields, e2e=True, flush=flush)
    clk = clocks.stop()
    agg = reduce_over_ranks({"pass_ms": float(sum(h["pass_ms"])), "e2e_ms": float(h["e2e_ms"]),
                             "e2e_serial_ms": float(sum(h["e2e_serial_ms"])),
                             "executed": h["executed"], "nominal": h["nominal"], "fo_sums": h["fo_sums"]},
                            world, "cuda")
    total_ms, e2e_total = agg["pass_ms"], agg["e2e_ms"]
    executed, nominal, fo_sums = agg["executed"], agg["nominal"], agg["fo_sums"]
    value = executed * args.steps / (total_ms * 1e-3)
    e2e_value = executed * args.steps / (e2e_total * 1e-3)
    e2e_serial = executed * args.steps / (agg["e2e_serial_ms"] * 1e-3)

    eng0 = capi.Engine(device=local_rank)
    fma_rate, _ = eng0.probe_fma_rate()                 # measured FP32 issue ceiling (thread-instr/s)
    mufu_rate, _ = eng0.probe_mufu_rate()               # measured XU ceiling
    eng0.close()
    pass_s = (total_ms / args.steps) * 1e-3
    roofline = issue_roofline(pkg, "grid2p1_langevin_rta_fo_fp32", fma_rate, mufu_rate, executed / world, pass_s,
                              h["n"], 0, live_steps=LIVE_SUBCHUNK_STEPS)
    roofline["kernel"] = ("k_cart_grid_fo32 (fused Langevin+RTA step with the freeze-out latch, sub-chunks of 32 "
                          "steps over a compacted live list; two species on two streams)")
    roofline["timing"] = ("achieved: algorithmic instructions of the executed particle-steps / the device span of a "
                          "pass (step, step-table and compaction kernels of both species), CUDA events")
    cpu = accuracy = None
    extra = {}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        threads = orc.max_threads()
        ncpu = size_cpu_sample(pkg, 10.0, threads, fields)
        samples = [sample_of(w, ncpu) for w in headline_workloads(pkg, 2 * ncpu, 0, 1, precision="fp64",
                                                                    fields=fields)]
        s, ps, outs = cpu_pass(samples, threads)
        cpu = {"value": ps / s, "unit": "particle-steps/s", "cores": threads, "kind": "port",
               "sample": f"{ncpu} charm + {ncpu} bottom quarks x 940 steps of the headline workload (stop at "
                         f"freeze-out), FP64 restatement (oracle/), {s:.1f} s"}
        accuracy = accuracy_against_cpu(pkg, samples, outs)
    if world == 1 and not args.quick:
        h64 = measure_headline(pkg, argparse.Namespace(**dict(vars(args), steps=min(args.steps, 3), warmup=1)),
                               rank, world, local_rank, "fp64", fields, e2e=True, flush=flush)
        extra["fp64"] = {
            "workload": WORKLOAD.replace("fp32", "fp64"), "unit": "particle-steps/s",
            "value": h64["executed"] * len(h64["pass_ms"]) / (sum(h64["pass_ms"]) * 1e-3),
            "e2e": {"value": h64["executed"] * len(h64["pass_ms"]) / (h64["e2e_ms"] * 1e-3),
                    "unit": "particle-steps/s", "h2d_bytes_per_step": h64["h2d"], "d2h_bytes_per_step": h64["d2h"],
                    "serial": h64["executed"] * len(h64["e2e_serial_ms"]) / (sum(h64["e2e_serial_ms"]) * 1e-3)},
            "ms_per_pass": statistics.median(h64["pass_ms"]),
            "timing": "device span of a pass (both species on two streams), CUDA events, "
                      f"{len(h64['pass_ms'])} passes after one warm-up"}
        extra["bjorken"] = bench_bjorken(pkg, args, fma_rate, mufu_rate)
        extra["batched"] = bench_batched(pkg, args, flush)
        extra["adjoint"] = bench_adjoint(pkg, args)
    elif world > 1:
        extra = {k: {"skipped": "measured in the one-GPU run"} for k in ("fp64", "bjorken", "batched", "adjoint")}
    if rank == 0:
        cnt = max(float(fo_sums[0]), 1.0)
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded 2+1D grid workload)",
            "config": {"workload": WORKLOAD, "particles_per_gpu": args.particles,
                       "species": "5e6 charm (1.5 GeV) + 5e6 bottom (4.75 GeV) per GPU", "steps_per_pass": 940,
                       "medium": "2+1D grid 201x201x100 float4 (T, v^x, v^y), trilinear",
                       "collision": "langevin+rta", "freezeout": "latch at T < 0.155 GeV, particles stop",
                       "executed_particle_steps_per_pass": executed, "nominal_particle_steps_per_pass": nominal,
                       "value_nominal": nominal * args.steps / (total_ms * 1e-3),
                       "precision": "fp32 arithmetic, fp64 momentum accumulation and frame changes",
                       "l2": "flushed between timed passes (256 MB write)", "parallelism": f"dp{world} (particles)"},
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": h["h2d"],
                    "d2h_bytes_per_step": h["d2h"],
                    "method": ("passes streamed through the C-ABI by pipeline.EnsembleStream: two slots of "
                               "contexts, each pass's upload (page-locked FP64 host arrays), step-0 boost, run and "
                               "freeze-out download; the copies of passes k-1 and k+1 overlap the run of pass k, "
                               "runs never overlap; device span of all passes (first upload to last download)"),
                    "serial": e2e_serial,
                    "serial_method": "the same calls one pass after the other, each pass timed alone"},
            "gpu_launches": h["launches"],
            "roofline": roofline,
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            "clocks": clk,
            "observables_at_freezeout": {k: float(v) / cnt for k, v in zip(capi.OBS_NAMES, fo_sums)},
        }
        line["observables_at_freezeout"]["count"] = float(fo_sums[0])
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------
# small cases for a profiler capture (each prints its device time)
# ---------------------------------------------------------------------------------
def run_case(args):
    pkg = load_package()
    W, capi = pkg.workloads, pkg.capi
    a = args
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
        wl = W.bjorken(N=a.n, precision=a.precision, steps=a.case_steps)
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
        wl = W.bjorken(N=a.n, precision=a.precision, steps=a.case_steps)
    elif a.case == "grid":
        wl = W.grid2p1(N=a.n, m=a.mass, precision=a.precision, steps=a.case_steps, freezeout=a.fo)
    else:
        wl = W.adjoint_grid(N=a.n, steps=a.case_steps)
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
          f"{wl.particle_steps / (ms * 1e-3):.4g} nominal particle-steps/s")


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--particles", type=int, default=10_000_000, help="particles per GPU (half charm, half bottom)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="only the headline workload (no sub-legs)")
    ap.add_argument("--cpu-table", action="store_true",
                    help="the CPU restatement's particle-steps/s on configs 0-2 at 1 and all host threads")
    ap.add_argument("--cpu-seconds", type=float, default=3.0, help="--cpu-table: seconds per sample")
    cg = ap.add_argument_group("profiler cases (--case)")
    cg.add_argument("--case", choices=["bjorken", "grid", "adjoint", "batch", "snapshots"])
    cg.add_argument("--n", type=int, default=262144)
    cg.add_argument("--case-steps", type=int, default=200)
    cg.add_argument("--fo", action="store_true", help="grid: freeze-out latch, particles stop")
    cg.add_argument("--mass", type=float, default=1.5)
    cg.add_argument("--precision", default="fp32")
    cg.add_argument("--save", type=int, default=20, help="snapshots: steps between saves")
    cg.add_argument("--compare", action="store_true", help="snapshots: time the snapshot-output options")
    cg.add_argument("--ensembles", type=int, default=16)
    args = ap.parse_args()
    if args.case:
        run_case(args)
        return
    if args.cpu_table:
        cpu_table(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
