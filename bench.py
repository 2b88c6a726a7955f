#!/usr/bin/env python
"""Throughput of the fused heavy-quark Langevin step on B200.

Workload (one benchmark "step" = one full simulation pass): the Bjorken medium
T(tau) = 0.40 (0.6/tau)^(1/3) GeV as a reference (r, t) table, tau 0.6 -> 10 fm/c
with dtau = 0.005 (1880 steps), 1e6 charm quarks per GPU (p_T power law, uniform
phi and rapidity), Langevin (2 pi T D_s = 4) plus RTA (tau_R = 5 eta/s / T), Bjorken
redshift, FP32 arithmetic with FP64 momentum accumulation.  Synthetic seeded inputs.

  value : particle-steps/s over all GPUs, inputs resident in HBM (state restored from a
          device checkpoint before every pass); L2 flushed between passes.
  e2e   : the same through the C-ABI from pinned host buffers: upload, step-0 boost,
          run, download of the final state, every pass.
  batched / adjoint / grid2p1 (one-GPU run): the batched persistent launch of 256
          ensembles against 256 separate runs, the forward+adjoint cost against the
          plain forward, and the 2+1D grid workload with freeze-out and its roofline.

`--impl reference` times the reference's CPU algorithm (the FP64 restatement under
oracle/, all host threads) on a bounded sample of the same workload.
Multi-GPU (torchrun): every rank runs its own 1e6 particles (weak scaling, no
data-path collective); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import re
import math
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
WORKLOAD = "bjorken_langevin_rta_1e6_charm_fp32"


def load_package():
    import __graft_entry__ as ge
    return ge.load_package()


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
# the reference CPU arm and the CPU baseline (FP64 restatement, all host threads)
# ---------------------------------------------------------------------------------
def cpu_sample(pkg, n_particles: int, threads: int = 0, calib_steps: int = 0):
    """Run the restatement on a bounded sample of the workload; returns (particle-steps/s, info)."""
    from oracle import oracle as orc
    W = pkg.workloads
    wl = W.bjorken(N=n_particles, precision="fp64", rng_seed=2)
    steps = calib_steps or wl.steps
    P = orc.make_params(**dict(wl.params, precision=0))
    md = orc.Medium().rt(wl.medium["xgrid"], wl.medium["tgrid"], wl.medium["T"], wl.medium["V"])
    for w, (a, b, v) in wl.splines.items():
        md.spline(w, a, b, v)
    md.invcdf(*wl.invcdf)
    x0, p0 = orc.initial_lab_boost(P, md, wl.x, wl.p)
    t = time.perf_counter()
    out = orc.run(P, md, x0, p0, wl.first_step, steps, threads=threads)
    dt = time.perf_counter() - t
    return n_particles * steps / dt, dict(particles=n_particles, steps=steps, seconds=dt, x=out["x"], p=out["p"])


def accuracy_against_cpu_sample(pkg, n_particles: int, info: dict) -> dict:
    """The engine in FP32 and FP64 on the particles of the timed CPU sample, against
    that sample's FP64 final state (same Philox noise): per particle
    ||a - b|| / max(||b||, floor * scale), scale 0.3 GeV for momenta and 1 fm for
    positions, floor 1e-2 in FP64 and 1 in FP32 (the parity tests' metric)."""
    W, capi = pkg.workloads, pkg.capi
    out = {"sample": f"{n_particles} charm quarks x 1880 steps (the CPU sample's particles)",
           "metric": "per-particle relative error, max and 99.99th percentile"}
    for prec, floor in (("fp64", 1e-2), ("fp32", 1.0)):
        wl = W.bjorken(N=n_particles, precision=prec, rng_seed=2)
        e = capi.Engine(0)
        W.configure(e, wl)
        e.initial_lab_boost()
        e.run(wl.first_step, wl.steps)
        x, p = e.download_state()
        e.close()
        res = {}
        for name, a, b, sc in (("p", p, info["p"], 0.3), ("x", x, info["x"], 1.0)):
            err = np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), floor * sc)
            res[f"{name}_max"] = float(err.max())
            res[f"{name}_p9999"] = float(np.percentile(err, 99.99))
        out[f"{prec}_vs_fp64_cpu"] = res
    return out


def size_cpu_sample(pkg, target_s: float, threads: int) -> int:
    """Particles for ~target_s seconds of the full 1880-step run on `threads` threads."""
    from oracle import oracle as orc
    n0 = 512 * max(1, threads or orc.max_threads())
    rate, _ = cpu_sample(pkg, n0, threads, calib_steps=60)
    return max(256, int(rate * target_s / 1880))


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    pkg = load_package()
    from oracle import oracle as orc
    threads = orc.max_threads()
    n = size_cpu_sample(pkg, 6.0, threads)
    for _ in range(args.warmup):
        cpu_sample(pkg, max(256, n // 8), threads)
    vals = []
    total_ps, total_s = 0, 0.0
    for _ in range(args.steps):
        v, info = cpu_sample(pkg, n, threads)
        vals.append(v)
        total_ps += info["particles"] * info["steps"]
        total_s += info["seconds"]
    value = total_ps / total_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Bjorken workload sample)",
        "config": {"workload": WORKLOAD, "particles_per_step_sample": n, "steps_per_pass": 1880,
                   "note": "the reference is Julia (not installed); this arm times its CPU algorithm as the "
                           "C FP64 restatement under oracle/ on all host threads"},
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{n} charm quarks x 1880 steps per timed step"},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------
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


def work_model(pkg):
    wm = json.loads((Path(pkg.__file__).parent / "work_model.json").read_text())
    w = wm["workloads"]["bjorken_langevin_rta_fp32"]
    tot = {}
    for item in w["items"].values():
        for k, c in item.items():
            tot[k] = tot.get(k, 0.0) + c
    return tot, sum(tot.values()), w["hbm_bytes_per_particle_per_launch"]


def traffic_from_profile():
    """dram__bytes_read + dram__bytes_write of one benchmark launch, from the committed
    ncu summary of the step kernel (its last line)."""
    p = ROOT / "profiles" / "k_cart_bjorken_fp32_traffic.md"
    if p.exists():
        m = re.search(r"^bytes_per_launch_full_size:\s*(\d+)\s*$", p.read_text(), re.M)
        if m:
            return int(m.group(1))
    return None


# ---------------------------------------------------------------------------------
# the other two legs of the metric (measured at N = 1): batched vs separate launches,
# and the forward+adjoint cost; plus the 2+1D grid workload's roofline
# ---------------------------------------------------------------------------------
TUNED = ROOT / "langevinmedium.jl_b200" / "tuned_shapes.json"


def bench_batched(pkg, args, flush):
    """256 ensembles (1e3-1e6 particles, charm/bottom, 2piT Ds in [2, 8], 500-2000 steps,
    half Bjorken, half 2+1D grids): one batched run (graph of persistent chunk launches)
    against the same ensembles as 256 lim_run calls back to back."""
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
    key = f"{props.name}|sm{props.multi_processor_count}|batch256-rng4"
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
                    "2piT Ds ~ U[2, 8], 500-2000 steps, half Bjorken (dtau 0.005), half 2+1D grids 201x201x100 "
                    "(T0 ~ U[0.35, 0.55] GeV, sy/sx ~ U[0.7, 1]), Langevin+RTA, FP32",
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
    2000 steps, checkpoints every 64 steps) against the plain forward."""
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
        "workload": "2+1D grid medium, 1e6 charm, 2000 steps (dt 0.01), Langevin+RTA, FP32; d/d(a, b, s) of "
                    "<pT>, <cos 2phi>, smoothed fraction pT > 5 GeV; 2piT Ds = a + b (T/0.155 - 1), a=3, b=2, s=1",
        "checkpoint_every": 64, "plain_forward_ms": f_ms, "forward_plus_adjoint_ms": a_ms,
        "checkpointed_forward_ms": statistics.median(fparts), "reverse_sweep_ms": statistics.median(rparts),
        "cost_ratio": a_ms / f_ms, "obs": obs.tolist(), "grad": G.tolist(),
        "timing": f"CUDA events, median of {reps} after one warm-up",
    }


def bench_fp64(pkg, args):
    """The headline workload in FP64 (the same 1e6 charm x 1880 steps), for the
    configuration's FP64 run: CUDA events, median of 3 after one warm-up."""
    W, capi = pkg.workloads, pkg.capi
    wl = W.bjorken(N=args.particles, precision="fp64", rng_seed=2)
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
    return {"workload": WORKLOAD.replace("fp32", "fp64"), "unit": "particle-steps/s",
            "value": wl.n * wl.steps / (t * 1e-3), "ms_per_pass": t,
            "timing": "CUDA events of the run (table and step kernels), median of 3 after one warm-up"}


def bench_grid(pkg, args, fma_rate, mufu_rate):
    """The 2+1D grid workload: 5e6 charm + 5e6 bottom, freeze-out at T < 0.155 GeV
    (particles stop when they freeze out), 940 steps of 0.01 fm."""
    W, capi = pkg.workloads, pkg.capi
    wm = json.loads((Path(pkg.__file__).parent / "work_model.json").read_text())
    counts = {}
    for item in wm["workloads"]["grid2p1_langevin_rta_fo_fp32"]["items"].values():
        for k, c in item.items():
            counts[k] = counts.get(k, 0.0) + c
    i_alg = sum(counts.values())
    fields = W.grid2p1_fields()
    tot_ms, executed, nominal = 0.0, 0.0, 0
    reps = max(1, min(args.steps, 3))
    for m, rs in ((1.5, 3), (4.75, 13)):
        wl = W.grid2p1(N=5_000_000, m=m, fields=fields, rng_seed=rs)
        e = capi.Engine(0)
        W.configure(e, wl)
        e.initial_lab_boost()
        e.state_save()
        ms = []
        for r in range(reps + 1):
            e.state_restore()
            e.run(wl.first_step, wl.steps)
            if r:
                ms.append(e.last_run_stats()[0])
        f = e.download_freezeout()
        frozen = f["flag"] != 0
        st = np.where(frozen, np.ceil((f["tau"] - wl.params["t0"]) / wl.params["dt"] - 1e-9), wl.steps)
        executed += float(np.minimum(st, wl.steps).sum())
        nominal += wl.n * wl.steps
        tot_ms += statistics.median(ms)
        e.close()
    rate = executed / (tot_ms * 1e-3)
    return {
        "workload": "2+1D grid 201x201x100 (T0 0.45 GeV, elliptic, radial u^r = tanh(0.05 r (tau - 0.6))), 5e6 charm "
                    "+ 5e6 bottom, Langevin+RTA, freeze-out latch at T < 0.155 GeV, particles stop at freeze-out, "
                    "940 steps, FP32",
        "unit": "particle-steps/s", "value_executed": rate, "value_nominal": nominal / (tot_ms * 1e-3),
        "executed_particle_steps": executed, "nominal_particle_steps": nominal, "kernel_ms": tot_ms,
        "roofline": {"bound": "issue", "unit": "Ginst/s", "algorithmic_inst_per_particle_step": i_alg,
                     "achieved": i_alg * rate / 1e9, "peak": fma_rate / 1e9, "frac": i_alg * rate / fma_rate,
                     "peak_source": "FP32 FMA issue probe (lim_probe_fma_rate), this run",
                     "per_pipe": per_pipe_roofline(counts, fma_rate, mufu_rate, executed, tot_ms * 1e-3)},
        "timing": f"CUDA events of the runs (table, step and compaction kernels), median of {reps} after one warm-up",
    }


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    pkg = load_package()
    W = pkg.workloads
    capi = pkg.capi
    n = args.particles
    stream = torch.cuda.current_stream()
    wl = W.bjorken(N=n, precision="fp32", rng_seed=2 + rank)
    wl.params["particle_offset"] = rank * n              # global particle ids: each rank its own noise streams
    eng = capi.Engine(device=local_rank, stream=stream.cuda_stream)
    W.configure(eng, wl)
    eng.initial_lab_boost()
    eng.state_save()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")   # > 126 MB L2

    def one_pass():
        eng.state_restore()
        eng.run(wl.first_step, wl.steps)

    for _ in range(args.warmup):
        one_pass()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    pass_ms, kern_ms = [], []
    launches = 0
    for _ in range(args.steps):
        flush.zero_()                                    # between timed iterations, not timed
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        one_pass()
        e1.record(stream)
        e1.synchronize()
        pass_ms.append(e0.elapsed_time(e1))
        k, nl = eng.last_run_stats()
        kern_ms.append(k)
        launches += nl
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = float(sum(pass_ms))
    t = torch.tensor([total_ms, float(sum(kern_ms))], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms, total_kern_ms = float(t[0]), float(t[1])
    ps_per_pass = n * wl.steps
    value = world * ps_per_pass * args.steps / (total_ms * 1e-3)

    # physics output of the last pass, reduced over ranks (FP64 observable sums)
    obs = eng.observables()
    sums = torch.tensor(obs["sums"], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(sums)

    # ---- e2e through the C-ABI with pinned host buffers ----
    dims, pdim = 2, 3
    x_host = torch.from_numpy(capi.julia_layout(wl.x, dims).copy()).pin_memory()
    p_host = torch.from_numpy(capi.julia_layout(wl.p, pdim).copy()).pin_memory()
    x_out = torch.empty(n * dims, dtype=torch.float64).pin_memory()
    p_out = torch.empty(n * pdim, dtype=torch.float64).pin_memory()
    xb, pb, xo, po = (a.numpy() for a in (x_host, p_host, x_out, p_out))
    e2e_launches = 0

    def e2e_pass():
        eng.upload_state_flat(xb, pb, n)
        eng.initial_lab_boost()
        eng.run(wl.first_step, wl.steps)
        eng.download_state_flat(xo, po)

    for _ in range(max(1, args.warmup // 2)):
        e2e_pass()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_pass()
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
        e2e_launches += 7          # 2 uploads + boost + table + step + 2 downloads
    te = torch.tensor([float(sum(e2e_ms))], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * ps_per_pass * args.steps / (float(te[0]) * 1e-3)

    # ---- roofline of the step kernel ----
    counts, i_alg, hbm_pp = work_model(pkg)
    fma_rate, _ = eng.probe_fma_rate()                    # measured FP32 issue ceiling (thread-instr/s)
    mufu_rate, _ = eng.probe_mufu_rate()                  # measured XU ceiling
    kern_s = (total_kern_ms / args.steps) * 1e-3
    achieved = i_alg * ps_per_pass / kern_s               # algorithmic thread-instructions per second
    bytes_launch = hbm_pp * n
    roofline = {
        "bound": "issue", "unit": "Ginst/s",
        "achieved": achieved / 1e9, "peak": fma_rate / 1e9, "frac": achieved / fma_rate,
        "traffic": traffic_from_profile(),
        "kernel": "k_cart (fused Langevin+RTA step, 1880 steps per launch)",
        "algorithmic_inst_per_particle_step": i_alg,
        "inst_mix_per_particle_step": counts,
        "peak_source": "measured in this run: FP32 FMA issue probe (lim_probe_fma_rate), thread-instr/s",
        "kernel_ms_per_launch": kern_s * 1e3,
        "per_pipe": per_pipe_roofline(counts, fma_rate, mufu_rate, ps_per_pass, kern_s),
        "hbm": {"algorithmic_bytes_per_launch": bytes_launch, "achieved_gbs": bytes_launch / kern_s / 1e9,
                "peak_gbs": 6544.3, "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
    }
    cpu = accuracy = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        threads = orc.max_threads()
        ncpu = size_cpu_sample(pkg, 12.0, threads)
        rate, info = cpu_sample(pkg, ncpu, threads)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": threads, "kind": "port",
               "sample": f"{ncpu} charm quarks x 1880 steps of the same workload, FP64 restatement (oracle/), "
                         f"{info['seconds']:.1f} s"}
        accuracy = accuracy_against_cpu_sample(pkg, ncpu, info)
    extra = {}
    if world == 1 and not args.quick:
        extra["batched"] = bench_batched(pkg, args, flush)
        extra["adjoint"] = bench_adjoint(pkg, args)
        extra["grid2p1"] = bench_grid(pkg, args, fma_rate, mufu_rate)
        extra["fp64"] = bench_fp64(pkg, args)
    elif world > 1:
        extra["batched"] = extra["adjoint"] = extra["grid2p1"] = extra["fp64"] = {"skipped": "measured in the one-GPU run"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Bjorken workload)",
            "config": {"workload": WORKLOAD, "particles_per_gpu": n, "steps_per_pass": wl.steps,
                       "particle_steps_per_pass_per_gpu": ps_per_pass, "medium": "reference (r,t) table 41x1883",
                       "collision": "langevin+rta", "precision": "fp32 arithmetic, fp64 momentum accumulation",
                       "l2": "flushed between timed passes (256 MB write)", "parallelism": f"dp{world} (particles)"},
            "e2e": {"value": e2e_value, "unit": "particle-steps/s",
                    "h2d_bytes_per_step": int(xb.nbytes + pb.nbytes), "d2h_bytes_per_step": int(xo.nbytes + po.nbytes)},
            "gpu_launches": launches,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            "clocks": clk,
            "observables": {k: float(v) for k, v in zip(capi.OBS_NAMES, (sums.cpu().numpy() /
                                                                       max(float(sums[0]), 1.0)))},
        }
        line["observables"]["count"] = float(sums[0])
        line.update(extra)
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--particles", type=int, default=1_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="only the headline workload (no batched/adjoint/grid legs)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
