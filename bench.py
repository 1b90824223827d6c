#!/usr/bin/env python
"""Benchmark: MC trial moves/s of the GCMC hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload protein|batched]

Workload (one replica per GPU): the synthetic protein system -- 6000 fixed
atoms of a confined random-walk chain in a 64 A periodic box, eight rigid
fragments of 4-12 sites starting at their bulk-concentration counts, confBias
1000, cutoff 12 A, the reference's move schedule and acceptance semantics.
A bench step is CHUNK MC steps (moveArray entries); `value` is MC steps/s with
the state resident on the GPU, `e2e` the same through the runGCMC drop-in
with host arrays (upload, run, download inside the timed region).  The launch
shape comes from the autotuner, run before the timed region (--cells N fixes
the cell-grid resolution instead).

--workload batched: 64 replicas of uneven size (2000-40000 atoms, a muex scan)
advanced together in one context, with the launch shape from the autotuner;
`e2e` through the batched drop-in runGCMC_batch.

--impl reference times the reference's own runGCMC_cuda (built unmodified
from its sources into oracle/_ref) on the same workload (batched: one
replica after another, as the reference has no batched form).
Under torchrun every rank runs an independent replica (its own seed) on its
own GPU; times are the max over ranks ("replicas only", weak scaling).
"""
import argparse
import contextlib
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MC trial moves/sec on 1 B200: batched/force-bias vs plain, ΔE rel err ≤1e-5"
# fixed algorithmic count per atom-site pair: dx, dy, dz 3; r^2 5; 1/r^2 1; sigma^2/r^2 1; s^6 2;
# 4 eps s^6 (s^6 - 1) 3; k q_i q_j / r 1; accumulate 2 (plus one rsqrt)
FLOPS_PER_PAIR = 19
WORKLOAD = ("synthetic protein: 6000-atom random-walk chain in a 24 A sphere, 64 A periodic box, "
            "8 rigid fragments (4-12 sites) at bulk counts, confBias 1000, cutoff 12 A, reference semantics")


def dist_env():
    from pygcmc_b200 import replicas
    return replicas.env()


def replicas_seed(base, rank, stride=1):
    from pygcmc_b200 import replicas
    return replicas.replica_seed(base, rank, stride)


def make_system(seed, mcsteps):
    from pygcmc_b200 import system as S
    return S.protein_system(seed=seed, mcsteps=mcsteps)


WATER_WORKLOAD = ("water box: 800 rigid TIP3P waters in a 30 A periodic box, no fixed atoms, muex -5.8 kcal/mol, "
                  "55 M, confBias 1000, cutoff 12 A, equal move probabilities, translate in a 1 A cube, rotate "
                  "<= 15 degrees about a uniform axis")


def make_water(seed, mcsteps):
    from pygcmc_b200 import system as S
    return S.water_box(n_water=800, box=30.0, seed=seed, mcsteps=mcsteps)


def water_options(**kw):
    from pygcmc_b200._native import default_options
    return default_options(proposal=1, muex_kcal=1, trn_step=1.0, rot_max=float(np.radians(15.0)), **kw)


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(gpu_index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


@contextlib.contextmanager
def quiet_stdout():
    """Silence C-level stdout (the reference prints a newline per call)."""
    sys.stdout.flush()
    saved = os.dup(1)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, 1)
    try:
        yield
    finally:
        os.dup2(saved, 1)
        os.close(null)
        os.close(saved)


def cpu_baseline(seed, budget_s=15.0):
    """The CPU oracle (C restatement, OpenMP over trial poses) on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    s = make_system(seed, 4000)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    oracle.run(s, 20, step0=0, threads=threads, want_energies=False)
    dt = time.perf_counter() - t0
    n = int(min(2000, max(20, budget_s / max(dt / 20, 1e-6))))
    t0 = time.perf_counter()
    oracle.run(s, n, step0=20, threads=threads, want_energies=False)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "moves/s", "cores": threads, "kind": "port",
            "sample": f"MC steps 20..{20 + n} of the same workload on the oracle (FP64, OpenMP over poses)"}


def nominal_fp32_tflops(sm_max_mhz):
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    return sms * 128 * 2 * sm_max_mhz * 1e6 / 1e12, sms


def load_traffic():
    p = os.path.join(ROOT, "profiles", "k_energy_protein6000.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def run_ours(args, ws, rank, local, kind="protein"):
    """One replica per GPU: the protein workload (the headline), or the water box."""
    import torch
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    from pygcmc_b200.gpu import runGCMC
    torch.cuda.set_device(local)
    chunk = args.chunk
    seed = replicas_seed(args.seed, rank)
    prof_steps = 256
    total = (args.warmup + args.steps) * chunk + prof_steps + 64
    water = kind == "water"
    sysm = make_water(seed, total) if water else make_system(seed, total)
    base = water_options() if water else default_options()
    if args.cells > 0:
        base.cells_per_cutoff = args.cells
        opts, t_tune = base, 0.0
    else:  # launch shape from the autotuner (untimed set-up)
        from pygcmc_b200.engine import autotune
        t0 = time.perf_counter()
        opts, _ = autotune(sysm, base, trial_steps=128)
        t_tune = time.perf_counter() - t0
    eng = Engine(sysm.copy(), opts)
    stream = torch.cuda.ExternalStream(eng.stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    for _ in range(args.warmup):
        eng.run(chunk)
    eng.sync()
    c0 = eng.counters()
    kept0 = int(eng.phase_cycles()[6])
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    for a, b in evs:
        with torch.cuda.stream(stream):
            flush.zero_()
        a.record(stream)
        eng.run(chunk)
        b.record(stream)
    eng.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    ms = max_over_ranks(ms, ws)
    barrier(ws)
    c1 = eng.counters()
    kept = int(eng.phase_cycles()[6]) - kept0
    # live per-kernel durations on the same trajectory (kernels launched one by one)
    te, ta, mv = eng.run_profiled(prof_steps)
    c2 = eng.counters()
    eng.sync()
    eng.close()
    # end to end through the drop-in API with host arrays, over the same step range:
    # warm-up calls advance the host state through the first `warmup` chunks
    e2e_state = sysm.pinned()  # host arrays in page-locked memory
    h2d = sum(a.nbytes for a in e2e_state.arrays()[:6]) + 4 * chunk
    d2h = e2e_state.moved_bytes()
    info = e2e_state.SimInfo
    info[0]["mcsteps"] = chunk
    moves = e2e_state.moveArray
    e2e_times = []
    for k in range(args.warmup + args.steps):
        info[0]["seed"] = (seed * 7 + k) & 0xFFFFFFFF
        mv = np.ascontiguousarray(moves[k * chunk:(k + 1) * chunk])
        barrier(ws)
        t0 = time.perf_counter()
        runGCMC(info, e2e_state.fragmentInfo, e2e_state.residueInfo, e2e_state.atomInfo, e2e_state.grid,
                e2e_state.ff, mv, options=opts)
        if k >= args.warmup:
            e2e_times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(sum(e2e_times) * 1e3, ws) / 1e3
    steps_all = args.steps * chunk * ws
    value = steps_all / (ms / 1e3)
    e2e_val = args.steps * chunk * ws / e2e_s
    pairs_prof = c2["pairs"] - c1["pairs"]
    e_ms = float(te.sum())
    a_ms = float(ta.sum())
    sm_max = (clk or {}).get("sm_max_mhz") or 1965.0
    peak, sms = nominal_fp32_tflops(sm_max)
    achieved = pairs_prof * FLOPS_PER_PAIR / (e_ms / 1e3) / 1e12
    traffic = load_traffic()
    # per MC step: pose energies + accept, or (speculating, the default for one
    # replica) re-prepare + completion + accept + speculative prepare + speculative
    # energies; per run call: run-end update + start-step set-up
    speculating = opts.speculate >= 0 and opts.branches <= 1
    launches = args.steps * (2 + (5 if speculating else 2) * 32 * ((chunk + 31) // 32))
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "moves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 pair terms, fp64 sums/acceptance",
        "data": "synthetic (seeded generator; no public dataset)",
        "config": ref_config(WATER_WORKLOAD if water else WORKLOAD, chunk, 1, ws),
        "launch_shape": {"cells_per_cutoff": opts.cells_per_cutoff, "split_items": opts.split_items,
                         "branches": opts.branches, "energy_blocks_per_sm": opts.energy_blocks_per_sm,
                         "energy_variant": opts.energy_variant, "energy_kernel": opts.energy_kernel,
                         "tile_cells": opts.tile_cells,
                         "source": "--cells" if args.cells > 0 else
                         f"autotuned before timing ({t_tune:.1f} s, untimed)"},
        "e2e": {"value": round(e2e_val, 1), "unit": "moves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "mc_steps_per_call": chunk,
                "host_arrays": "page-locked (System.pinned())", "api": "pygcmc_b200.gpu.runGCMC (drop-in for gcmc.gpu.runGCMC)"},
        "roofline": {"bound": "fp32", "kernel": "k_energy (pose energies)",
                     "achieved": round(achieved, 3), "peak": round(peak, 2), "unit": "TFLOP/s",
                     "frac": round(achieved / peak, 5),
                     "peak_source": f"nominal FP32: {sms} SMs x 128 lanes x 2 x {sm_max:.0f} MHz "
                                    "(MEASURED_PEAKS.json has no FP32 figure)",
                     "flops_per_pair": FLOPS_PER_PAIR, "pairs_per_launch": pairs_prof / prof_steps,
                     "avg_launch_us": e_ms / prof_steps * 1e3,
                     "traffic": None if traffic is None else traffic.get("dram_bytes_per_launch"),
                     "share_of_step_time": round(e_ms / (e_ms + a_ms), 3),
                     "timing": "launch by launch, steps in sequence (run_profiled)"},
        "roofline_accept": {"kernel": "k_accept (cluster walk, accept/update; 1 CTA per replica)",
                            "bound": "latency (sequential greedy clustering on one SM)",
                            "avg_launch_us": a_ms / prof_steps * 1e3,
                            "share_of_step_time": round(a_ms / (e_ms + a_ms), 3)},
        "speculation": {"on": speculating, "steps_whose_energies_were_kept": kept,
                        "of_steps": args.steps * chunk},
        "pose_energies_per_s": round((c1["poses"] - c0["poses"]) / (ms / 1e3), 1),
        "pairs_per_s": round((c1["pairs"] - c0["pairs"]) / (ms / 1e3), 1),
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0 and ws == 1 and not args.no_cpu and not water:
        out["cpu_baseline"] = cpu_baseline(seed)
    return out


def summary(out):
    """The figures of a workload's bench line that the default run reports beside its headline."""
    keys = ("value", "unit", "ms_per_step", "steps", "warmup", "config", "e2e", "roofline", "roofline_accept",
            "launch_shape", "autotuned", "speculation", "forcebias", "gradient", "clocks", "gpu_launches",
            "pairs_per_s")
    return {k: out[k] for k in keys if k in out}


BATCH_WORKLOAD = ("64 replicas of uneven size in one context: synthetic proteins of 2000-40000 atoms "
                  "(log-uniform), box 40-100 A at constant protein density, 8 fragments each, muex scan "
                  "-8..0 kcal/mol, own seeds, confBias 1000, cutoff 12 A, reference semantics")


def make_batch(seed, mcsteps, n_rep):
    from pygcmc_b200 import system as S
    return S.replica_batch(n_rep=n_rep, seed=seed, mcsteps=mcsteps)


def run_ours_batched(args, ws, rank, local):
    """All replicas of the batch advance in one context (one pose-energy and one
    accept launch per MC step, replayed from a CUDA graph); the launch shape
    comes from the autotuner, run before the timed region."""
    import torch
    from pygcmc_b200._native import Options, default_options
    from pygcmc_b200.engine import Engine, autotune
    from pygcmc_b200.gpu import runGCMC_batch
    torch.cuda.set_device(local)
    chunk = args.chunk
    seed = replicas_seed(args.seed, rank, 1000)
    prof_steps = 64
    total = (args.warmup + args.steps) * chunk + prof_steps + 256
    t0 = time.perf_counter()
    systems = make_batch(seed, total, args.replicas)
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    best, trials = autotune(systems, default_options(), trial_steps=64)
    t_tune = time.perf_counter() - t0
    nrep = len(systems)
    eng = Engine([x.copy() for x in systems], best)
    stream = torch.cuda.ExternalStream(eng.stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        eng.run(chunk)
    eng.sync()
    c0 = [eng.counters(r) for r in range(nrep)]
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    for a, b in evs:
        with torch.cuda.stream(stream):
            flush.zero_()
        a.record(stream)
        eng.run(chunk)
        b.record(stream)
    eng.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs), ws)
    barrier(ws)
    c1 = [eng.counters(r) for r in range(nrep)]
    te, ta, _ = eng.run_profiled(prof_steps)
    c2 = [eng.counters(r) for r in range(nrep)]
    eng.close()
    # end to end: the batched drop-in with host arrays (upload, run, download per call)
    state = [x.pinned() for x in systems]  # host arrays in page-locked memory
    # the cavity grids travel as voxel bit sets (Options.grid_bits; the same points)
    e2e_opt = Options.from_buffer_copy(best)
    e2e_opt.grid_bits = 1
    h2d = sum(sum(a.nbytes for a in s.arrays_for(e2e_opt)[:6]) + 4 * chunk for s in state)
    d2h = sum(s.moved_bytes() for s in state)
    full_moves = [s.moveArray for s in state]  # page-locked; each call takes a slice of it
    e2e_times = []
    for k in range(args.warmup + args.steps):
        for r, s in enumerate(state):
            s.SimInfo[0]["mcsteps"] = chunk
            s.SimInfo[0]["seed"] = (seed * 7 + 131 * r + k) & 0xFFFFFFFF
            s.moveArray = np.ascontiguousarray(full_moves[r][k * chunk:(k + 1) * chunk])
        barrier(ws)
        t0 = time.perf_counter()
        runGCMC_batch(state, e2e_opt)
        if k >= args.warmup:
            e2e_times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(sum(e2e_times) * 1e3, ws) / 1e3
    moves_all = args.steps * chunk * nrep * ws
    pairs_prof = sum(b["pairs"] - a["pairs"] for a, b in zip(c1, c2))
    e_ms, a_ms = float(te.sum()), float(ta.sum())
    sm_max = (clk or {}).get("sm_max_mhz") or 1965.0
    peak, sms = nominal_fp32_tflops(sm_max)
    achieved = pairs_prof * FLOPS_PER_PAIR / (e_ms / 1e3) / 1e12
    launches = args.steps * (2 + 2 * 32 * best.branches * ((chunk + 31) // 32))
    out = {
        "metric": METRIC, "value": round(moves_all / (ms / 1e3), 1), "unit": "moves/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 pair terms, fp64 sums/acceptance", "data": "synthetic (seeded generator; no public dataset)",
        "config": ref_config(BATCH_WORKLOAD, chunk * nrep, nrep, ws,
                             [int(s.info["totalAtomNum"]) for s in systems][:nrep]),
        "autotuned": {"cells_per_cutoff": best.cells_per_cutoff, "split_items": best.split_items,
                      "branches": best.branches, "energy_blocks_per_sm": best.energy_blocks_per_sm,
                      "trials": len(trials), "tune_s": round(t_tune, 2),
                      "energy_variant": best.energy_variant,
                      "energy_kernel": best.energy_kernel, "tile_cells": best.tile_cells,
                      "persistent": best.persistent,
                      "trial_fields": ["cells_per_cutoff", "split_items", "branches", "energy_blocks_per_sm",
                                       "energy_variant", "energy_kernel", "tile_cells", "persistent", "ms_per_step"],
                      "trial_ms_per_step": [[*t[:5], *t[6:], round(t[5], 4)] for t in trials]},
        "generate_s": round(t_gen, 2),
        "e2e": {"value": round(args.steps * chunk * nrep * ws / e2e_s, 1), "unit": "moves/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "mc_steps_per_call": chunk,
                "host_arrays": "page-locked (System.pinned())", "api": "pygcmc_b200.gpu.runGCMC_batch (all replicas per call)",
                "cavity_grid": "voxel bit sets (Options.grid_bits = 1)"},
        "roofline": {"bound": "fp32", "kernel": "k_energy (pose energies, all replicas)",
                     "achieved": round(achieved, 3), "peak": round(peak, 2), "unit": "TFLOP/s",
                     "frac": round(achieved / peak, 5),
                     "peak_source": f"nominal FP32: {sms} SMs x 128 lanes x 2 x {sm_max:.0f} MHz "
                                    "(MEASURED_PEAKS.json has no FP32 figure)",
                     "flops_per_pair": FLOPS_PER_PAIR, "pairs_per_launch": pairs_prof / prof_steps,
                     "avg_launch_us": e_ms / prof_steps * 1e3, "traffic": None,
                     "share_of_step_time": round(e_ms / (e_ms + a_ms), 3),
                     "timing": "kernels launched one by one (no graph, one branch) over the next 64 steps"},
        "roofline_accept": {"kernel": "k_accept (1 CTA per replica)", "avg_launch_us": a_ms / prof_steps * 1e3,
                            "share_of_step_time": round(a_ms / (e_ms + a_ms), 3)},
        "pairs_per_s": round(sum(b["pairs"] - a["pairs"] for a, b in zip(c0, c1)) / (ms / 1e3), 1),
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0 and ws == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(seed)
        out["cpu_baseline"]["sample"] += " (one 6000-atom replica; replicas are independent, so the CPU rate " \
                                         "for the batch is this rate at the same cores)"
    return out


class RefRunner:
    """The reference's runGCMC_cuda driven over a step range of one system."""

    def __init__(self, L, system, seed):
        self.L, self.s, self.seed = L, system, seed
        self.info = system.SimInfo.copy()
        self.skipped = 0

    def call(self, mv):
        s = self.s
        self.info[0]["mcsteps"] = len(mv)
        with quiet_stdout():
            self.L.runGCMC_cuda(self.info.ctypes.data, s.fragmentInfo.ctypes.data, s.residueInfo.ctypes.data,
                                s.atomInfo.ctypes.data, s.grid.ctypes.data, s.ff.ctypes.data, mv.ctypes.data)

    def run_range(self, a, b):
        """Steps [a, b) in slices; a delete on an empty fragment type (where the
        reference divides by zero, gcmc_move_del.h:113) is skipped.  Returns the
        number of calls made."""
        s, moves = self.s, self.s.moveArray
        calls = 0
        pos = a
        while pos < b:
            tot = s.fragmentInfo["totalNum"].astype(np.int64).copy()
            q = pos
            while q < b:
                f, m = divmod(int(moves[q]), 4)
                if m == 1:
                    if tot[f] <= 0:
                        break
                    tot[f] -= 1
                q += 1
            if q == pos:
                self.skipped += 1
                pos += 1
                continue
            self.info[0]["seed"] = (self.seed * 131 + pos) & 0xFFFFFFFF
            self.call(np.ascontiguousarray(moves[pos:q]))
            calls += 1
            pos = q
        return calls

    def fixed_cost(self):
        """Per-call set-up time (allocation, copies, RNG set-up) from zero-step calls."""
        import torch
        t = []
        for _ in range(3):
            t0 = time.perf_counter()
            self.call(np.zeros(1, np.int32)[:0])
            torch.cuda.synchronize()
            t.append(time.perf_counter() - t0)
        return float(np.median(t))


FB_WORKLOAD = ("force-biased vs plain GCMC on the synthetic protein (6000-atom chain, 64 A box, 8 fragment "
               "types at bulk counts, confBias 1000, cutoff 12 A): REPLICAS replicas of the system (own RNG "
               "streams) in one context; plain = symmetric moves (translate in a cube of half-width h, rotate "
               "about a uniform axis by <= theta); force-biased = each component of the displacement / "
               "rotation vector in [-h, h] / [-theta, theta] with density ~exp(beta f d / 2) from the force / "
               "torque (Pangali-Rao-Berne), Metropolis-Hastings corrected; insert / delete identical; both "
               "scanned over (h, theta) in {(0.5 A, 10 deg), (1 A, 20 deg), (2 A, 40 deg)}; `value` = the "
               "force-biased run at its best step size")
FB_SCAN = ((0.5, 10.0), (1.0, 20.0), (2.0, 40.0))


def time_engine(eng, stream, flush, chunk, warmup, steps):
    """Warm-up chunks, then `steps` timed chunks (CUDA events on the engine's
    stream, L2 flushed before each); returns the summed milliseconds."""
    import torch
    for _ in range(warmup):
        eng.run(chunk)
    eng.sync()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for a, b in evs:
        with torch.cuda.stream(stream):
            flush.zero_()
        a.record(stream)
        eng.run(chunk)
        b.record(stream)
    eng.sync()
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs)


def gradient_throughput(sysm, batches=10, nposes=4096):
    """Forward + backward of the pose energy for `nposes` random rigid poses
    (uniform centre, uniform quaternion) through the autograd wrapper: poses/s."""
    import torch
    from pygcmc_b200 import poses as PZ
    from pygcmc_b200.engine import Engine
    from pygcmc_b200.grad import RigidFragment, lj_table
    dev = torch.device("cuda")
    lt = sysm.meta["lj_types"]
    ffx = int(sysm.SimInfo[0]["ffXNum"])
    with Engine(sysm.copy()) as eng:
        frag = RigidFragment(eng, 0, 0, dtype=torch.float32)
        eps = torch.tensor(lt["eps_kcal"], device=dev, requires_grad=True)
        rmin = torch.tensor(lt["rmin_half"], device=dev, requires_grad=True)
        data = []
        for b in range(batches + 3):
            com, quat = PZ.random_poses(sysm, nposes, seed=100 + b)
            data.append((torch.tensor(com, device=dev, dtype=torch.float32, requires_grad=True),
                         torch.tensor(quat, device=dev, dtype=torch.float32, requires_grad=True)))

        def one(c, q):
            e = frag.energy(c, q, lj_table(eps, rmin, ffx))
            torch.nan_to_num(e, posinf=0.0, neginf=0.0).sum().backward()

        for c, q in data[:3]:
            one(c, q)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for c, q in data[3:]:
            one(c, q)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
    return {"poses_per_s": round(batches * nposes / (ms / 1e3), 1), "batch": nposes, "batches": batches,
            "ms_per_batch": round(ms / batches, 3),
            "gradients": "centre of mass (3), quaternion (4), per-type eps and rmin/2 (24 + 24), site charges"}


def fb_sampling_run(systems, opts, burn, meas, chunk, flush, msd=False):
    """Burn-in, then `meas` timed steps of every replica (CUDA events on the
    engine's stream around each chunk, L2 flushed before it): moves/s and, per
    replica, the integrated autocorrelation times of the total fragment count N
    and the running energy E over the measured steps (Sokal window), the
    decorrelated samples meas / max(tau_N, tau_E), translate / rotate acceptance,
    and with msd=True (fixed-N schedules) the mean square displacement of the
    fragment centres (unwrapped between chunks) over the measured steps."""
    import torch
    from pygcmc_b200 import analysis as A
    from pygcmc_b200.engine import Engine
    nrep = len(systems)
    opts.log_steps = burn + meas
    opts.log_kmax = 1
    eng = Engine([x.copy() for x in systems], opts)
    try:
        stream = torch.cuda.ExternalStream(eng.stream)
        eng.run(burn)
        eng.sync()

        holders = [x.copy() for x in systems] if msd else None

        def centres():
            out = []
            for r in range(nrep):
                st = eng.download(r, into=holders[r])
                idx = np.concatenate([np.arange(int(f["startRes"]), int(f["startRes"]) + int(f["totalNum"]))
                                      for f in st.fragmentInfo])
                out.append(st.residueInfo["position"][idx].astype(np.float64))
            return out

        box = np.array(systems[0].SimInfo[0]["cryst"], dtype=np.float64)
        prev = centres() if msd else None
        disp = [np.zeros_like(c) for c in prev] if msd else None
        ms = 0.0
        for c0 in range(0, meas, chunk):
            n = min(chunk, meas - c0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.zero_()
            a.record(stream)
            eng.run(n)
            b.record(stream)
            eng.sync()
            ms += a.elapsed_time(b)
            if msd:
                cur = centres()
                for r in range(nrep):
                    d = cur[r] - prev[r]
                    disp[r] += d - box * np.round(d / box)
                prev = cur
        rate = nrep * meas / (ms / 1e3)
        per_rep = []
        for r in range(nrep):
            logs, _ = eng.logs(r)
            sm = A.sampling_summary(logs[: burn + meas], systems[r].fragmentInfo["totalNum"].astype(np.int64),
                                    meas / (ms / 1e3), burn=burn)
            if msd:
                sm["msd_A2"] = float((disp[r] ** 2).sum(axis=1).mean())
            per_rep.append(sm)
        out = {"moves_per_s": round(rate, 1), "ms": round(ms, 2), "replicas": nrep, "burn_steps": burn,
               "steps": meas,
               "tau_N_median": float(np.median([x["tau_N"] for x in per_rep])),
               "tau_E_median": float(np.median([x["tau_E"] for x in per_rep])),
               "runs_in_tau": float(np.median([meas / x["tau"] for x in per_rep])),
               "decorrelated_samples_per_s": float(sum(meas / x["tau"] for x in per_rep) / (ms / 1e3)),
               "trn_rot_accept_per_pose": float(np.mean([x["trn_rot_accept_per_pose"] for x in per_rep])),
               "mean_N": float(np.mean([x["mean_N"] for x in per_rep]))}
        if msd:
            out["msd_A2_per_s"] = float(np.mean([x["msd_A2"] for x in per_rep]) / (ms / 1e3))
        return out
    finally:
        eng.close()


def run_ours_forcebias(args, ws, rank, local):
    """Force-biased against plain GCMC on REPLICAS replicas of the synthetic
    protein in one context (the batched force-biased line): each method at each
    step size of FB_SCAN, on the full GCMC schedule (decorrelation of N and E)
    and on a fixed-N translate/rotate schedule (decorrelation of E and the
    fragments' mean square displacement per second), after a burn-in; `value`
    is the force-biased moves/s at the step size with the most decorrelated
    samples/s on the full schedule."""
    import torch
    from pygcmc_b200._native import default_options
    from pygcmc_b200.gpu import runGCMC
    torch.cuda.set_device(local)
    nrep = args.replicas
    seed = replicas_seed(args.seed, rank)
    chunk = 512
    burn, meas = args.warmup * 1024, args.steps * 1024
    total = burn + meas + 64
    base = make_system(seed, total)
    ntype = len(base.fragmentInfo)
    g = np.random.default_rng(seed + 17)
    fixed = base.copy()
    fixed.moveArray = (g.integers(0, ntype, total) * 4 + 2 + g.integers(0, 2, total)).astype(np.int32)
    systems_full = [base.copy() for _ in range(nrep)]
    systems_fixed = [fixed.copy() for _ in range(nrep)]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def opts(method, h, theta):
        th = float(np.radians(theta))
        if method == "plain":
            return default_options(proposal=1, trn_step=2.0 * h, rot_max=th)
        return default_options(proposal=2, fb_trn=h, fb_rot=th)

    scan = {"plain": [], "force_biased": []}
    clk = None
    for method in scan:
        for h, theta in FB_SCAN:
            barrier(ws)
            clocks = ClockSampler(local) if (method == "force_biased" and clk is None) else None
            full = fb_sampling_run(systems_full, opts(method, h, theta), burn, meas, chunk, flush)
            if clocks is not None:
                clk = clocks.stop()
            fix = fb_sampling_run(systems_fixed, opts(method, h, theta), burn, meas, chunk, flush, msd=True)
            scan[method].append({"h_A": h, "theta_deg": theta, "full_gcmc": full, "fixed_N": fix})
    best = {m: max(v, key=lambda e: e["full_gcmc"]["decorrelated_samples_per_s"]) for m, v in scan.items()}
    best_fix = {m: max(v, key=lambda e: e["fixed_N"]["decorrelated_samples_per_s"]) for m, v in scan.items()}
    best_msd = {m: max(v, key=lambda e: e["fixed_N"]["msd_A2_per_s"]) for m, v in scan.items()}
    fbb = best["force_biased"]
    ms_fb = max_over_ranks(fbb["full_gcmc"]["ms"], ws)
    value = nrep * meas * ws / (ms_fb / 1e3)
    # end to end: the runGCMC drop-in with force-biased options (one replica, host arrays per call)
    e2e_state = base.pinned()
    info = e2e_state.SimInfo
    info[0]["mcsteps"] = 8192
    h2d = sum(x.nbytes for x in e2e_state.arrays()[:6]) + 4 * 8192
    d2h = e2e_state.moved_bytes()
    fbopt = opts("force_biased", fbb["h_A"], fbb["theta_deg"])
    times = []
    for k in range(4):
        info[0]["seed"] = (seed * 7 + k) & 0xFFFFFFFF
        mv = np.ascontiguousarray(e2e_state.moveArray[:8192])
        barrier(ws)
        t0 = time.perf_counter()
        runGCMC(info, e2e_state.fragmentInfo, e2e_state.residueInfo, e2e_state.atomInfo, e2e_state.grid,
                e2e_state.ff, mv, options=fbopt)
        if k >= 1:
            times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(sum(times) * 1e3, ws) / 1e3

    def ratio(d, key, sub):
        return round(d["force_biased"][sub][key] / max(d["plain"][sub][key], 1e-30), 3)

    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "moves/s", "n_gpus": ws, "steps": meas // chunk,
        "warmup": burn // chunk, "ms_per_step": round(ms_fb / (meas // chunk), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 pair terms, fp64 sums/acceptance",
        "data": "synthetic (seeded generator; no public dataset)",
        "config": {"workload": FB_WORKLOAD.replace("REPLICAS", str(nrep)),
                   "mc_steps_per_bench_step": chunk * nrep, "replicas_per_gpu": nrep,
                   "parallelism": f"replicas x{ws}", "l2": "flushed (256 MB write) between timed chunks"},
        "e2e": {"value": round(3 * 8192 * ws / e2e_s, 1), "unit": "moves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "mc_steps_per_call": 8192,
                "host_arrays": "page-locked (System.pinned())",
                "api": "pygcmc_b200.gpu.runGCMC(..., options=proposal 2), one replica per call"},
        "forcebias": {
            "scan": scan,
            "best_full_gcmc": {m: [best[m]["h_A"], best[m]["theta_deg"]] for m in best},
            "decorrelated_samples_per_s_ratio": ratio(best, "decorrelated_samples_per_s", "full_gcmc"),
            "fixed_N_decorrelated_samples_per_s_ratio": ratio(best_fix, "decorrelated_samples_per_s", "fixed_N"),
            "fixed_N_msd_per_s_ratio": ratio(best_msd, "msd_A2_per_s", "fixed_N"),
            "moves_per_s_ratio": ratio(best, "moves_per_s", "full_gcmc"),
            "tau": "integrated autocorrelation time (steps) of the total fragment count N and the running "
                   "energy E per replica, Sokal window c=5, over the measured steps after the burn-in; "
                   "decorrelated samples/s = sum over replicas of steps / max(tau_N, tau_E) per second",
        },
        "gradient": gradient_throughput(base),
        "clocks": clk,
        # per 512-step chunk: k_set_run_end, k_prepare, then per step two force-bias
        # pose-energy launches and the accept kernel
        "gpu_launches": (meas // chunk) * (2 + 3 * chunk),
    }
    return out


LARGE_WORKLOAD = ("large periodic slab with Ewald electrostatics and force-biased moves: 150 x 150 x 120 A "
                  "box, 200000 fixed atoms (random-walk chains, 0.09 atoms/A^3, 12 A pore along z), 8 fragment "
                  "types + TIP3P water (15827 waters, 178915 slots), smooth PME 128 x 128 x 96, order 4, alpha "
                  "0.32, FP64 mesh, cutoff 12 A, force-biased translate / rotate (Metropolis-Hastings "
                  "corrected); REPLICAS replicas of the system (own RNG streams) in one context")


def run_ours_large(args, ws, rank, local):
    import torch
    from pygcmc_b200 import system as S
    from pygcmc_b200._native import Options, default_options
    from pygcmc_b200.engine import Engine
    from pygcmc_b200.gpu import runGCMC_batch
    torch.cuda.set_device(local)
    chunk = args.chunk
    nrep = args.replicas
    total = (args.warmup + args.steps) * chunk + 64 + 16
    t0 = time.perf_counter()
    base = S.slab_system(seed=args.seed + rank, mcsteps=total)
    t_gen = time.perf_counter() - t0
    # force-biased translate / rotate under Ewald, as the large configuration asks
    opt = default_options(pme=1, pme_alpha=0.32, branches=min(4, nrep), proposal=2)
    for a, n in enumerate((128, 128, 96)):
        opt.pme_grid[a] = n
    eng = Engine([base.copy() for _ in range(nrep)], opt)
    stream = torch.cuda.ExternalStream(eng.stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    barrier(ws)
    clocks = ClockSampler(local)
    ms = max_over_ranks(time_engine(eng, stream, flush, chunk, args.warmup, args.steps), ws)
    clk = clocks.stop()
    c1 = [eng.counters(r) for r in range(nrep)]
    te, ta, _ = eng.run_profiled(16)
    c2 = [eng.counters(r) for r in range(nrep)]
    eng.close()
    # end to end: the batched drop-in with host arrays (all replicas per call)
    state = [base.pinned() for _ in range(nrep)]  # host arrays in page-locked memory
    e2e_opt = Options.from_buffer_copy(opt)
    e2e_opt.grid_bits = 1  # the cavity grids travel as voxel bit sets (the same points)
    full_moves = [st.moveArray for st in state]
    for r, st in enumerate(state):
        st.SimInfo[0]["mcsteps"] = chunk
    h2d = sum(sum(a.nbytes for a in s_.arrays_for(e2e_opt)[:6]) + 4 * chunk for s_ in state)
    d2h = sum(s_.moved_bytes() for s_ in state)
    times = []
    for k in range(args.warmup + min(args.steps, 3)):
        for r, st in enumerate(state):
            st.SimInfo[0]["seed"] = (args.seed * 7 + 131 * r + k) & 0xFFFFFFFF
            st.moveArray = np.ascontiguousarray(full_moves[r][k * chunk:(k + 1) * chunk])
        barrier(ws)
        t0 = time.perf_counter()
        runGCMC_batch(state, e2e_opt)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(sum(times) * 1e3, ws) / 1e3
    pairs = sum(b["pairs"] - a["pairs"] for a, b in zip(c1, c2))
    e_ms, a_ms = float(te.sum()), float(ta.sum())
    sm_max = (clk or {}).get("sm_max_mhz") or 1965.0
    peak, sms = nominal_fp32_tflops(sm_max)
    achieved = pairs * FLOPS_PER_PAIR / (e_ms / 1e3) / 1e12
    return {
        "metric": METRIC, "value": round(args.steps * chunk * nrep * ws / (ms / 1e3), 1), "unit": "moves/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 pair terms, fp64 sums/acceptance, fp64 PME mesh",
        "data": "synthetic (seeded generator; no public dataset)",
        "config": {"workload": LARGE_WORKLOAD.replace("REPLICAS", str(nrep)), "replicas_per_gpu": nrep,
                   "mc_steps_per_bench_step": chunk, "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (state + meshes of all replicas)", "generate_s": round(t_gen, 2),
                   "proposals": "force-biased translate / rotate (h 0.5 A, 10 deg), uniform SO(3) insertion"},
        "e2e": {"value": round(min(args.steps, 3) * chunk * nrep * ws / e2e_s, 1), "unit": "moves/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "mc_steps_per_call": chunk,
                "host_arrays": "page-locked (System.pinned())", "api": "pygcmc_b200.gpu.runGCMC_batch (all replicas per call)",
                "cavity_grid": "voxel bit sets (Options.grid_bits = 1)"},
        "roofline": {"bound": "fp32", "kernel": "k_energy (pose energies incl. erfc and PME interpolation)",
                     "achieved": round(achieved, 3), "peak": round(peak, 2), "unit": "TFLOP/s",
                     "frac": round(achieved / peak, 5), "flops_per_pair": FLOPS_PER_PAIR,
                     "peak_source": f"nominal FP32: {sms} SMs x 128 lanes x 2 x {sm_max:.0f} MHz",
                     "avg_step_us_pme_and_energy": e_ms / 16 * 1e3, "avg_accept_us": a_ms / 16 * 1e3,
                     "traffic": None},
        # per chunk: k_set_run_end, k_prepare; per graph step: each replica's six mesh-update
        # launches (which return at once when no charge moved), then per branch two force-bias
        # pose-energy launches and the accept kernel
        "gpu_launches": args.steps * (2 + 32 * ((chunk + 31) // 32) * (6 * nrep + 3 * opt.branches)),
        "clocks": clk,
    }


ARRAY_NAMES = ("SimInfo", "fragmentInfo", "residueInfo", "atomInfo", "grid", "ff", "moveArray")


def write_inputs(path, workload, seed, mcsteps, replicas):
    """Build the workload's input arrays and save them to `path` (.npz).  The
    reference arm runs this in a child process, so that the process it times
    loads no code of this repository's library (the generators are in it)."""
    if workload == "batched":
        systems = make_batch(seed, mcsteps, replicas)
    else:
        systems = [make_system(seed, mcsteps)]
    arrs = {f"{r}_{name}": a for r, s in enumerate(systems) for name, a in zip(ARRAY_NAMES, s.arrays())}
    np.savez(path, n=len(systems), **arrs)


def read_inputs(path):
    import types
    z = np.load(path)
    return [types.SimpleNamespace(**{name: np.ascontiguousarray(z[f"{r}_{name}"]) for name in ARRAY_NAMES})
            for r in range(int(z["n"]))]


def run_reference(args, ws, rank, local):
    if rank != 0:
        return None
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libgcmc_ref.so")
    if not os.path.exists(lib_path):
        return {"impl": "reference", "unavailable": "oracle/_ref/libgcmc_ref.so not built (make -C oracle ref)"}
    chunk = args.ref_chunk
    seed = args.seed
    batched = args.workload == "batched"
    mcsteps = (args.warmup + args.steps + 2) * chunk + 16
    with tempfile.TemporaryDirectory() as tmp:  # inputs from a child process (untimed)
        path = os.path.join(tmp, "inputs.npz")
        subprocess.check_call([sys.executable, os.path.abspath(__file__), "--write-inputs", path, "--workload",
                               args.workload, "--seed", str(seed), "--replicas", str(args.replicas),
                               "--mcsteps", str(mcsteps)])
        systems = read_inputs(path)
    import torch
    torch.cuda.set_device(local)
    L = ctypes.CDLL(lib_path)
    L.runGCMC_cuda.restype = None
    L.runGCMC_cuda.argtypes = [ctypes.c_void_p] * 7
    runners = [RefRunner(L, s, seed + 7 * r) for r, s in enumerate(systems)]
    fixed = runners[0].fixed_cost()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    pos = 0
    for _ in range(args.warmup):
        for rr in runners:
            rr.run_range(pos, pos + chunk)
        pos += chunk
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    t_raw, t_adj, n = 0.0, 0.0, 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        calls = 0
        for rr in runners:
            calls += rr.run_range(pos, pos + chunk)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        t_raw += dt
        t_adj += max(dt - calls * fixed, 1e-9)
        pos += chunk
        n += chunk * len(runners)
    clk = clocks.stop()
    value = n / t_adj
    workload = BATCH_WORKLOAD if batched else WORKLOAD
    how = (f"each of the {len(runners)} replicas in turn, {chunk} steps per replica per bench step"
           if batched else f"{chunk} steps per bench step")
    return {
        "metric": METRIC, "value": round(value, 1), "unit": "moves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_adj / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 (reference kernels)", "impl": "reference",
        "data": "synthetic (seeded generator; no public dataset)",
        "config": ref_config(workload, chunk * len(runners) if batched else chunk, len(runners), 1,
                             [int(r.s.SimInfo[0]["totalAtomNum"]) for r in runners] if batched else None),
        "schedule": how,
        "cpu_baseline": {"value": round(value, 1), "unit": "moves/s", "cores": 1, "kind": "reference",
                         "sample": f"reference runGCMC_cuda (unmodified pyGCMC gcmc.cu, sm_100a) on the B200, "
                                   f"{n} MC steps ({how}); the reference has no CPU implementation of this "
                                   f"path; per-call set-up ({fixed * 1e3:.2f} ms) subtracted"},
        "e2e": {"value": round(n / t_raw, 1), "unit": "moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "skipped_deletes_on_empty_types": sum(rr.skipped for rr in runners),
        "clocks": clk,
    }


def ref_config(workload, steps_per_bench_step, replicas, ws, atoms=None):
    """The `config` both arms print for a workload (the same keys and values)."""
    c = {"workload": workload, "mc_steps_per_bench_step": steps_per_bench_step, "replicas_per_gpu": replicas,
         "parallelism": f"replicas x{ws}", "l2": "flushed (256 MB write) between timed chunks"}
    if atoms is not None:
        c["atoms_per_replica"] = atoms
    return c


def run_probe(args):
    """A small fixed run for kernel profiling (ncu) and per-kernel timing: the
    workload's system advanced --probe-warm steps through the graph-captured
    step loop, then --probe-steps steps launched kernel by kernel with CUDA
    events around each launch; prints the per-step kernel times.  Under ncu the
    pose-energy and accept launches after the warm-up are the individually
    launched ones."""
    from pygcmc_b200 import system as S
    from pygcmc_b200._native import default_options
    from pygcmc_b200.engine import Engine
    total = args.probe_warm + args.probe_steps + 64
    if args.workload == "batched":
        s = S.replica_batch(n_rep=args.replicas, seed=args.seed, mcsteps=total)
    elif args.workload == "water":
        s = S.water_box(seed=args.seed, mcsteps=total)
    else:
        s = make_system(args.seed, total)
    if args.workload == "batched":  # the batch's tuned shape
        opt = default_options(cells_per_cutoff=args.cells if args.cells > 0 else 1, split_items=512, energy_variant=1,
                              pair_delta=args.pair_delta)
    else:
        opt = default_options(cells_per_cutoff=args.cells if args.cells > 0 else 2, pair_delta=args.pair_delta)
    if args.probe_fb:  # force-biased translate / rotate (h 2 A, 40 degrees)
        opt.proposal = 2
        opt.fb_trn = 2.0
        opt.fb_rot = float(np.radians(40.0))
    if args.probe_pme > 0:  # Ewald electrostatics on a probe_pme^3 mesh
        opt.pme = 1
        for a in range(3):
            opt.pme_grid[a] = args.probe_pme
    with Engine(s, opt) as eng:
        eng.run(args.probe_warm)
        eng.sync()
        te, ta, mv = eng.run_profiled(args.probe_steps)
        print(json.dumps({"move": (mv % 4).tolist(), "energy_us": [round(float(x) * 1e3, 2) for x in te],
                          "accept_us": [round(float(x) * 1e3, 2) for x in ta], "counters": eng.counters(),
                          "accept_phase_cycles": eng.phase_cycles().tolist()}))


def barrier(ws):
    from pygcmc_b200 import replicas
    replicas.barrier(ws)


def max_over_ranks(x, ws):
    from pygcmc_b200 import replicas
    return replicas.max_over_ranks(x, ws)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["all", "protein", "batched", "forcebias", "large", "water"],
                    default="all",
                    help="all (default): the protein headline and, on one GPU, the batched, water and "
                         "force-bias workloads as sub-results of the same line; protein: one 6000-atom "
                         "replica per GPU; batched: --replicas uneven replicas per GPU; forcebias: force-biased "
                         "vs plain translate/rotate on the protein system; water: the 800-water box; large: "
                         "200000-atom slab with PME, --replicas replicas")
    ap.add_argument("--replicas", type=int, default=0, help="default 64 (batched), 16 (large)")
    ap.add_argument("--chunk", type=int, default=0, help="MC steps per bench step (default 2048; batched 256)")
    ap.add_argument("--ref-chunk", type=int, default=0,
                    help="MC steps per bench step for the reference arm (default: --chunk, same step range)")
    ap.add_argument("--cells", type=int, default=0, help="cells per cutoff (0: autotune the launch shape)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--probe", action="store_true",
                    help="a small fixed run for kernel profiling: --probe-warm graph steps, then --probe-steps "
                         "steps launched kernel by kernel (per-kernel times printed; no bench line)")
    ap.add_argument("--probe-warm", type=int, default=64)
    ap.add_argument("--probe-steps", type=int, default=24)
    ap.add_argument("--probe-pme", type=int, default=0, help="probe: Ewald electrostatics on an N^3 mesh")
    ap.add_argument("--probe-fb", action="store_true", help="probe: force-biased translate / rotate")
    ap.add_argument("--pair-delta", type=int, default=0,
                    help="probe: translate/rotate changes in the pairwise-difference form (0) or as two evaluations (-1)")
    ap.add_argument("--write-inputs", default="", help=argparse.SUPPRESS)  # reference arm's child process
    ap.add_argument("--mcsteps", type=int, default=0, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.probe:
        if args.replicas <= 0:
            args.replicas = 64
        run_probe(args)
        return
    if args.write_inputs:
        write_inputs(args.write_inputs, args.workload, args.seed, args.mcsteps,
                     args.replicas if args.replicas > 0 else 64)
        return
    args.warmup = max(args.warmup, 3)
    if args.chunk <= 0:
        args.chunk = {"batched": 256, "forcebias": 512, "large": 64}.get(args.workload, 2048)
    if args.replicas <= 0:
        args.replicas = 16 if args.workload == "large" else 64
    if args.ref_chunk <= 0:
        args.ref_chunk = 16 if args.workload == "batched" else args.chunk
    ws, rank, local = dist_env()
    if ws > 1:
        import torch
        from pygcmc_b200 import replicas
        torch.cuda.set_device(local)
        replicas.init("nccl", timeout_s=300)
    try:
        if args.impl == "reference":
            out = run_reference(args, ws, rank, local)
        elif args.workload == "batched":
            out = run_ours_batched(args, ws, rank, local)
        elif args.workload == "forcebias":
            out = run_ours_forcebias(args, ws, rank, local)
        elif args.workload == "large":
            out = run_ours_large(args, ws, rank, local)
        elif args.workload == "water":
            out = run_ours(args, ws, rank, local, kind="water")
        else:
            out = run_ours(args, ws, rank, local)
            if args.workload == "all" and ws == 1:
                import copy
                for name, fn, chunk, kw in (("batched", run_ours_batched, 256, {}),
                                            ("water", run_ours, 2048, {"kind": "water"}),
                                            ("forcebias", run_ours_forcebias, 512, {})):
                    sub = copy.copy(args)
                    sub.chunk, sub.no_cpu = chunk, True
                    out[name] = summary(fn(sub, ws, rank, local, **kw))
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if ws > 1:
            from pygcmc_b200 import replicas
            replicas.finalize()


if __name__ == "__main__":
    main()
