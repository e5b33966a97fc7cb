#!/usr/bin/env python
"""Benchmark of the StaRMAP time loop on B200: moment-cell updates/s.

Workload (default): 2D checkerboard lattice, P_39 filtered (820 moments),
350x350 cells on [0,7]^2, bc = 1, sigma_a = 10 / sigma_s0 = 0 on the absorbing
squares and 0 / 1 elsewhere, source q = 1 in the central square, zero initial
condition, dt = 0.5 h, t_final = 3.2 (321 steps), exponential filter of order 4
and strength 10 applied per substep.  Synthetic, deterministic inputs with the
shapes of the reference's lattice example.

One bench step = one full Strang time step (phase A, phase B, phase A) of the
whole problem.  One moment-cell update = one component at one cell advanced
by one step, so a step is n_sys * nx * ny updates.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU runs (torchrun, one process per GPU) run independent replicas of the
workload (the path does not shard); value is the aggregate over all ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# the generated kernels' on-disk cache of this run stays in the tree
os.environ.setdefault("SMG_JIT_CACHE_DIR", os.path.join(ROOT, "_build", "jit_cache"))

WORKLOAD_NAME = ("2D checkerboard lattice P39 filtered (820 moments), 350x350 cells, bc=1, "
                 "substep exp filter p=4 f_eff=10, dt=0.5h, t_final=3.2 (321 steps)")
METRIC = "moment-cell updates/s"
UNIT = "updates/s"


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class Dist:
    """Barrier and max-over-ranks; torch.distributed only when WORLD_SIZE > 1
    (NCCL on the GPUs; gloo on host tensors, which the CPU tests use)."""

    def __init__(self, world, local_rank, backend="nccl"):
        self.world = world
        self.torch = None
        self.cuda = backend == "nccl"
        if world > 1:
            import datetime

            import torch
            import torch.distributed as td
            if self.cuda:
                torch.cuda.set_device(local_rank)
            td.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
            self.torch, self.td = torch, td

    def barrier(self):
        if self.torch is not None:
            self.td.barrier()
            if self.cuda:
                self.torch.cuda.synchronize()

    def max(self, v: float) -> float:
        if self.torch is None:
            return v
        t = self.torch.tensor([float(v)], device="cuda" if self.cuda else "cpu", dtype=self.torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.torch is not None:
            self.td.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.fh.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        load = [s for s in sm if s > 0.5 * mx] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows
                                                        if r[3].replace(".", "").isdigit())}


def aggregate_rate(units_per_step: float, steps: int, world: int, ms_max: float) -> float:
    """Whole-job rate of N replicas (weak scaling): every rank advances its
    own copy of the workload, so the job's units are N times one rank's, over
    the slowest rank's time."""
    return units_per_step * steps * world / (ms_max / 1e3)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(family="jit", name=None):
    """DRAM bytes per step of the phase kernels of `family` from the committed ncu summary (or None)."""
    if name is None:
        name = "phase_kernels_jit_lattice_p39_350_full.txt" if family == "jit" else "phase_kernels_lattice_p39_350.txt"
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_step:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def workload():
    from starmap_b200 import configs, starmap_init
    par = starmap_init(configs.lattice(n=350, n_mom=39, tfinal=3.2, filter_order=4, f_eff=10.0,
                                       f_position="substep"))
    return par


def cpu_sample(par, budget_s: float, nthreads: int, max_steps: int | None = None, warm: int = 0):
    """Time the oracle's C restatement (all given threads) on a bounded prefix of the run."""
    from oracle import c_oracle
    adv = c_oracle.CAdvance(nthreads)

    def stop():
        done = len(adv.step_seconds)
        if max_steps is not None and done >= warm + max_steps:
            return True
        return sum(adv.step_seconds[warm:]) >= budget_s and done > warm

    c_oracle.run(par, nthreads=nthreads, advance=adv, stop=stop)
    secs = adv.step_seconds[warm:]
    return len(secs), sum(secs)


def bench_batch(steps: int = 200):
    """Batched sweep: 256 seeded 2D instances (edge 64..256, N in {3,5,7,11,15},
    8x8-block log-uniform materials, own CFL dt), `steps` steps each.  The
    batch (autotuned over the generated family kernels and the precompiled
    configurations) against a loop of plain per-instance runs with the default
    kernels; the loop's instances are built and their kernels compiled before
    its timing starts (that compile time is reported separately), so the loop
    is timed at its best."""
    from starmap_b200 import configs, starmap_init
    from starmap_b200.batch import _tables, setup_batch
    from starmap_b200.solver import GpuSolver, handle_tables
    pars = [starmap_init(p) for p in configs.batched_sweep()]
    setups, batch = setup_batch(pars)
    mc = sum(S.n_sys * int(np.prod(S.n)) for S, _ in setups)
    U0 = [S.U0 for S, _ in setups]
    batch.set_states(U0)
    batch.set_dt([fs["dt"] for _, fs in setups])
    t0 = time.perf_counter()
    batch.autotune(4)
    tune_s = time.perf_counter() - t0
    batch.set_states(U0)
    batch.run(steps)
    ms, launches = batch.last_run_stats()
    cfg = batch.config()
    used_jit, families = batch.info()
    batch.close()
    solvers = []
    t0 = time.perf_counter()
    for S, fs in setups:
        T = _tables(S, fs)
        sv = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T))
        sv.set_state(S.U0)
        sv.set_dt(fs["dt"])
        sv.run(1)          # builds the instance's kernels
        sv.set_state(S.U0)
        solvers.append(sv)
    sv.sync()
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    dev = 0.0
    per_ms = []
    for sv in solvers:
        sv.run(steps)
        sv.sync()
        per_ms.append(sv.last_run_stats()[0])
        dev += per_ms[-1]
    wall = time.perf_counter() - t0
    for sv in solvers:
        sv.close()
    batched = mc * steps / (ms / 1e3)
    loop = mc * steps / wall
    # the loop's device rate by instance size, and the batch's own HBM fraction
    from starmap_b200.roofline import algorithmic_bytes_per_step
    buckets = {}
    for (S, fs), t in zip(setups, per_ms):
        key = "edge<=128" if int(S.n[1]) <= 128 else "edge>128"
        b = buckets.setdefault(key, {"instances": 0, "moment_cells": 0, "loop_device_ms": 0.0})
        b["instances"] += 1
        b["moment_cells"] += S.n_sys * int(np.prod(S.n))
        b["loop_device_ms"] += t
    for b in buckets.values():
        b["loop_device_value"] = b["moment_cells"] * steps / (b["loop_device_ms"] / 1e3)
        b["share_of_moment_cells"] = b["moment_cells"] / mc
    if len(buckets) == 2:
        sm, lg = buckets["edge<=128"], buckets["edge>128"]
        # if the batch ran the small instances for nothing and the large ones at the loop's rate
        bound = (sm["loop_device_ms"] + lg["loop_device_ms"]) / lg["loop_device_ms"]
    else:
        bound = None
    alg = sum(algorithmic_bytes_per_step(S, _tables(S, fs), fused=True)["step"] for S, fs in setups)
    peak, kind = measured_peak()
    batch_gbs = alg * steps / (ms / 1e3) / 1e9
    return {"value": batched, "unit": UNIT, "instances": len(pars), "moment_cells": mc, "steps": steps,
            "ms": ms, "launches": launches, "config": cfg, "kernels": "generated families" if used_jit else
            "precompiled", "families": families, "autotune_s": tune_s,
            "plain_loop_value": loop, "plain_loop_device_value": mc * steps / (dev / 1e3),
            "plain_loop_setup_s": setup_s,
            "batched_over_plain_loop": batched / loop,
            "batched_over_plain_loop_device": batched / (mc * steps / (dev / 1e3)),
            "loop_by_size": buckets, "loop_speedup_bound_small_free": bound,
            "roofline": {"bound": "hbm", "achieved": batch_gbs, "peak": peak, "unit": "GB/s",
                         "frac": batch_gbs / peak, "peak_kind": kind, "algorithmic_bytes_per_step": alg}}


def bench_adjoint(nsteps: int = 400, n: int = 200, ckpts=(0, 20)):
    """Misfit gradient w.r.t. sigma_a, sigma_s0, q and the initial condition on
    the 2D P15 inverse problem (n x n cells, nsteps steps).  Per checkpoint
    setting (0: as much recorded as memory allows; K: a checkpoint every K
    steps with recompute), one warm-up pass, then the device time of the
    forward and of the backward call against one plain forward (smg_run), and
    a central finite-difference check of the sigma_a gradient along a smooth
    direction."""
    from starmap_b200 import configs, starmap_init
    from starmap_b200.adjoint import MisfitAdjoint
    from starmap_b200.solver import prepare, setup_gpu

    def run_u0(par, steps, reps=1):
        S, fs, sv, T = setup_gpu(par)
        try:
            best = None
            for _ in range(reps):
                sv.set_state(S.U0)
                sv.set_dt(fs["dt"])
                sv.run(steps)
                sv.sync()
                ms = sv.last_run_stats()[0]
                best = ms if best is None else min(best, ms)
            return sv.get_state([0])[0], best
        finally:
            sv.close()

    obs, _ = run_u0(starmap_init(configs.adjoint_problem(n=n, sigma_a_field=configs.true_sigma_a)), nsteps)
    par = starmap_init(configs.adjoint_problem(n=n))
    _, plain_ms = run_u0(par, nsteps, reps=3)
    out = {"nsteps": nsteps, "grid": [n, n], "plain_forward_ms": plain_ms, "modes": []}
    g = None
    for ck in ckpts:
        adj = MisfitAdjoint(par, ckpt_every=ck)
        try:
            adj.forward(obs, nsteps)
            adj.backward()
            t0 = time.perf_counter()
            J = adj.forward(obs, nsteps)
            t1 = time.perf_counter()
            f_ms = adj.last_ms()
            gk = adj.backward()
            t2 = time.perf_counter()
            b_ms = adj.last_ms()
            K = adj.solver.adjoint_segment()
            nbytes = adj.solver.adjoint_bytes()
        finally:
            adj.close()
        g = g if g is not None else gk
        out["modes"].append({
            "ckpt_every": ck, "K": K, "adjoint_bytes": nbytes, "J": J,
            "forward_ms": f_ms, "backward_ms": b_ms,
            "backward_over_plain_forward": b_ms / plain_ms,
            "gradient_over_plain_forward": (f_ms + b_ms) / plain_ms,
            "forward_wall_s": t1 - t0, "backward_wall_s": t2 - t1})
    # directional derivative along a smooth direction, sampled like sigma_a itself
    def bump(x, y):
        return np.sin(1.3 * x + 0.4) * np.cos(0.9 * y - 0.2)
    eps = 1e-6

    def J_of(scale):
        p = starmap_init(configs.adjoint_problem(n=n, sigma_a_field=lambda x, y: 0.1 + scale * bump(x, y)))
        u, _ = run_u0(p, nsteps)
        return 0.5 * float(np.sum((u - obs) ** 2))
    fd = (J_of(eps) - J_of(-eps)) / (2 * eps)
    Sx = prepare(par)
    ad = 0.0
    for grid, gv in g["sigma_a"].items():
        X, Y, Z = Sx.XYZ(grid)
        ad += float(np.sum(gv * bump(Y, Z).reshape(np.shape(gv), order="F")))
    out.update({"n_sys": Sx.n_sys, "fd_directional": fd, "adjoint_directional": ad,
                "fd_rel_err": abs(fd - ad) / abs(fd)})
    # 32 such inverse problems batched (each its own observations), checkpoints every 20 steps
    from starmap_b200.adjoint import batched_gradients
    n_inst, threads = 32, 16
    try:
        grads, tf, tb = batched_gradients([par] * n_inst, [obs * (1.0 + 0.01 * i) for i in range(n_inst)], nsteps,
                                          ckpt_every=20, threads=threads)
        out["batch32"] = {"instances": n_inst, "ckpt_every": 20, "host_threads": threads, "forward_s": tf,
                          "backward_s": tb, "gradients_per_s": n_inst / (tf + tb),
                          "gradient_ms_per_instance": (tf + tb) / n_inst * 1e3,
                          "gradient_over_plain_forward": (tf + tb) / n_inst / (plain_ms / 1e3),
                          "finite": bool(all(np.all(np.isfinite(g["sigma_a"][(1, 1, 1)])) for g in grads))}
    except Exception as e:   # e.g. not enough device memory for 32 recordings
        out["batch32"] = {"instances": n_inst, "error": str(e)[:300]}
    return out


def bench_3d(steps: int = 96, n: int = 128):
    """3D P9 point source (100 moments), n^3 cells, periodic, sigma_sm = 0.5^m,
    substep filter, dt = 0.5h, t_final = 0.75 (96 steps): device throughput and
    the algorithmic HBM fraction of the default kernels."""
    from starmap_b200 import configs, starmap_init
    from starmap_b200.roofline import algorithmic_bytes_per_step
    from starmap_b200.solver import setup_gpu
    par = starmap_init(configs.pointsource3d(n=n))
    S, fs, sv, T = setup_gpu(par)
    try:
        sv.set_state(S.U0)
        sv.set_dt(fs["dt"])
        sv.run(3)
        sv.sync()
        family = {1: "generic", 2: "strip", 3: "staged", 4: "pair", 5: "jit"}[sv.active_variant()[0]]
        sv.set_state(S.U0)
        sv.run(steps)
        sv.sync()
        ms, launches = sv.last_run_stats()
        finite = sv.check_finite() == 0
    finally:
        sv.close()
    alg = algorithmic_bytes_per_step(S, T, fused=True)
    upd = S.n_sys * int(np.prod(S.n)) * steps
    peak, kind = measured_peak()
    achieved = alg["step"] * steps / (ms / 1e3) / 1e9
    return {"workload": f"3D P9 point source, {n}^3 cells, periodic, sigma_sm=0.5^m, substep filter, "
                        f"dt=0.5h, {steps} steps", "n_sys": S.n_sys, "value": upd / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / steps, "kernel_family": family, "launches": int(launches), "finite": finite,
            "state_gb": alg["state_bytes"] / 1e9,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": kind, "algorithmic_bytes_per_step": alg["step"],
                         "traffic": ncu_traffic(name="phase_kernels_jit_pointsource3d_p9.txt") if n == 128 else None}}


def cold_call():
    """--cold-call (run in a fresh process by bench_cold): the whole public
    call a MATLAB user makes -- starmap_init, starmap_solver to t_final with
    host setup, hook sampling, handle creation, kernel compilation (or its
    load from the on-disk cache), upload, all 321 steps and the download of
    the output moment -- timed by the wall clock from before starmap_init."""
    import ctypes
    t0 = time.perf_counter()
    from starmap_b200 import _lib, configs, starmap_init
    from starmap_b200.solver import starmap_solver
    prob = configs.lattice(n=350, n_mom=39, tfinal=3.2, filter_order=4, f_eff=10.0, f_position="substep")
    par = starmap_init(prob)
    out = starmap_solver(par)
    secs = time.perf_counter() - t0
    c, d = ctypes.c_int64(), ctypes.c_int64()
    _lib.lib().smg_jit_stats(ctypes.byref(c), ctypes.byref(d))
    print(json.dumps({"seconds": secs, "programs_compiled": c.value, "programs_from_disk": d.value,
                      "finite": bool(np.all(np.isfinite(out[0]["U"])))}), flush=True)
    return 0


def bench_cold(upd_step: float, nsteps: int = 321):
    """Cold start: the first starmap_solver call of two new processes, the
    first with an empty kernel cache (NVRTC compiles), the second with the
    cache the first one wrote."""
    import shutil
    d = os.path.join(ROOT, "_build", "bench_cold_cache")
    shutil.rmtree(d, ignore_errors=True)
    res = []
    for _ in range(2):
        env = dict(os.environ, SMG_JIT_CACHE_DIR=d)
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cold-call"], env=env,
                           capture_output=True, text=True, timeout=900)
        if r.returncode != 0:
            return {"error": r.stderr[-500:]}
        res.append(json.loads(r.stdout.strip().splitlines()[-1]))
    shutil.rmtree(d, ignore_errors=True)
    mk = lambda r: {"value": upd_step * nsteps / r["seconds"], "unit": UNIT, "seconds": r["seconds"],
                    "programs_compiled": r["programs_compiled"], "programs_from_disk": r["programs_from_disk"]}
    return {"what": "first starmap_solver call of a new process, starmap_init to the returned output, "
                    f"{nsteps} steps, host setup, compilation or cache load, transfers included",
            "empty_cache": mk(res[0]), "warm_cache": mk(res[1])}


def bench_growth(n_mom: int = 39):
    """One growth-factor evaluation of the parabolic time-step search for the
    P39 lattice system (820 moments): on the host (numpy eigenvalues, all
    host threads) and on the GPU (smg_growth_radius), same matrix."""
    from starmap_b200 import configs, starmap_init, timestep
    from starmap_b200.solver import first_step, prepare
    prob = configs.lattice(n=20, n_mom=n_mom)
    prob["timestep"] = 1
    S = prepare(starmap_init(prob))
    fs = first_step(S)
    decay = timestep.decay_vector(S.n_sys, S.gt, S.mom_order, fs["sA"][1, 1, 1], fs["sT"])
    dt = 2 * S.dt_hyp
    out = {"n_sys": S.n_sys}
    for flag, key in ((True, "device"), (False, "host")):
        timestep.use_device_eigenvalues(flag)
        timestep.growth_factor(S.M_sym, S.even, S.odd, decay, dt, 1)      # warm-up (handles, buffers)
        t0 = time.perf_counter()
        la = timestep.growth_factor(S.M_sym, S.even, S.odd, decay, dt, 1)
        out[key + "_ms"] = (time.perf_counter() - t0) * 1e3
        out[key + "_radius"] = la
    timestep.use_device_eigenvalues(None)
    out["host_threads"] = host_threads()
    out["rel_diff"] = abs(out["device_radius"] - out["host_radius"]) / out["host_radius"]
    return out


def host_buffers(S):
    """Initial state and output buffers in pinned host memory: one
    page-locked block each (through torch; pageable numpy if that is
    unavailable), carved into per-component arrays in component order."""
    def alloc(n):
        try:
            import torch
            return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy(), True
        except Exception:
            return np.empty(n, dtype=np.float64), False
    ext = [tuple((int(S.n[d]) + 1) if (int(S.gt[j][d]) == 2 and int(S.bc[d]) == 1) else int(S.n[d])
                 for d in range(3)) for j in range(S.n_sys)]
    total = sum(int(np.prod(e)) for e in ext)
    block_in, p1 = alloc(total)
    block_out, p2 = alloc(total)
    pin_in, pin_out, o = [], {}, 0
    for j, e in enumerate(ext):
        size = int(np.prod(e))
        a = block_in[o:o + size]
        a[:] = np.asarray(np.broadcast_to(S.U0[j], e), dtype=np.float64).ravel(order="F")
        pin_in.append(a.reshape(e, order="F"))
        pin_out[j] = block_out[o:o + size]
        o += size
    return pin_in, pin_out, p1 and p2


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (oracle C port; GNU Octave is not installed)."""
    if rank != 0:
        return 0
    par = workload()
    n_sys = par["Mz"].shape[0]
    cells = int(np.prod(par["n"]))
    threads = host_threads()
    warm = max(0, min(args.warmup, 1))
    steps, secs = cpu_sample(par, budget_s=args.ref_budget, nthreads=threads, max_steps=args.steps, warm=warm)
    value = n_sys * cells * steps / secs
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": secs / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "n_sys": n_sys, "cells": cells, "parallelism": "cpu"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"first {steps} of 321 steps after {warm} warm-up step(s); "
                                   "the oracle's C restatement of starmap_solver.m stands in for the "
                                   "reference, which is MATLAB/GNU Octave code this arm does not run"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=321)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--variant", choices=["auto", "generic", "strip", "staged", "pair", "jit"], default="auto",
                    help="kernel family (all give identical results)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-sweep measurement")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint measurement")
    ap.add_argument("--no-3d", action="store_true", help="skip the 3D P9 measurement")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of CPU-baseline stepping")
    ap.add_argument("--ref-budget", type=float, default=60.0, help="seconds of reference-arm stepping")
    ap.add_argument("--no-cold", action="store_true", help="skip the cold-start measurement")
    ap.add_argument("--no-growth", action="store_true", help="skip the parabolic-step eigenvalue measurement")
    ap.add_argument("--cold-call", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.cold_call:
        return cold_call()
    rank, local_rank, world = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    from starmap_b200 import _lib
    from starmap_b200.roofline import algorithmic_bytes_per_step
    from starmap_b200.solver import GpuSolver, handle_tables, setup_gpu

    _lib.check(_lib.lib().smg_set_device(local_rank))
    dist = Dist(world, local_rank)
    par = workload()
    S, fs, solver, T = setup_gpu(par)
    n_sys = S.n_sys
    cells = int(np.prod(S.n))
    upd_step = n_sys * cells
    variant = {"auto": 0, "generic": 1, "strip": 2, "staged": 3, "pair": 4, "jit": 5}[args.variant]
    solver.set_variant(variant)
    alg = algorithmic_bytes_per_step(S, T, fused=(variant in (0, 3, 4, 5)))
    solver.set_state(S.U0)
    solver.set_dt(fs["dt"])
    solver.run(args.warmup)
    solver.sync()
    family = {1: "generic", 2: "strip", 3: "staged", 4: "pair", 5: "jit"}[solver.active_variant()[0]]

    clocks = ClockSampler(local_rank)
    clocks.start()
    dist.barrier()
    solver.sync()
    solver.run(args.steps)
    solver.sync()
    dist.barrier()
    ms, launches = solver.last_run_stats()
    ms_max = dist.max(ms)
    finite = solver.check_finite() == 0
    solver.close()

    # end to end through the C ABI with host buffers: create (field upload),
    # state upload, the K steps and the state download, every byte included
    e2e = None
    if not args.no_e2e:
        fields_bytes = sum(np.asarray(v).size * 8 for v, _ in T.fields)
        state_bytes = alg["state_bytes"]
        # inputs and outputs in pinned host memory, allocated before the timing
        pin_in, pin_out, pinned = host_buffers(S)
        dist.barrier()
        t0 = time.perf_counter()
        s2 = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T))
        s2.set_variant(variant)
        s2.set_state(pin_in)
        s2.set_dt(fs["dt"])
        s2.run(args.steps)
        Ufin = s2.get_state(out=pin_out)
        t1 = time.perf_counter()
        s2.close()
        el = dist.max(t1 - t0)
        e2e = {"value": upd_step * args.steps * world / el, "unit": UNIT,
               "h2d_bytes_per_step": int((state_bytes + fields_bytes) / args.steps),
               "d2h_bytes_per_step": int(sum(u.size for u in Ufin.values()) * 8 / args.steps),
               "seconds": el, "host_buffers": "one pinned block per direction, carved into component arrays" if pinned
               else "pageable"}
    clk = clocks.stop()

    peak, peak_kind = measured_peak()
    t_step = ms_max / 1e3 / args.steps
    achieved = alg["step"] / t_step / 1e9
    traffic = ncu_traffic(family)
    line = {
        "metric": METRIC, "value": aggregate_rate(upd_step, args.steps, world, ms_max), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD_NAME, "n_sys": n_sys, "cells": cells,
                   "updates_per_step": upd_step, "state_gb": alg["state_bytes"] / 1e9,
                   "l2": "inputs larger than L2 (state %.2f GB > 126 MB), no flush" % (alg["state_bytes"] / 1e9),
                   "parallelism": "replicas" if world > 1 else "single GPU", "variant": args.variant,
                   "kernel_family": family,
                   "launch": "direct launches (a step moves >= 1 GB)" if 24.0 * cells * n_sys >= 1e9
                   else "replayed 64-step CUDA graphs"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_step": alg["step"],
                     "kernel": "phase kernels of the step (A, then B and the fused A-A), "
                               "averaged over the timed steps"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "finite": finite,
    }
    if e2e:
        line["e2e"] = e2e
    if world == 1 and not args.no_cold and e2e:
        line["e2e"]["cold"] = bench_cold(upd_step)
    if world == 1 and not args.no_batch:
        line["batched"] = bench_batch()
    if world == 1 and not args.no_adjoint:
        line["adjoint"] = bench_adjoint()
    if world == 1 and not args.no_3d:
        line["pointsource_3d"] = bench_3d()
    if world == 1 and not args.no_growth:
        try:
            line["parabolic_step_p39"] = bench_growth()
        except Exception as e:
            line["parabolic_step_p39"] = {"error": str(e)[:300]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = host_threads()
        steps, secs = cpu_sample(par, budget_s=args.cpu_budget, nthreads=threads, warm=0)
        line["cpu_baseline"] = {"value": upd_step * steps / secs, "unit": UNIT, "cores": threads,
                                "kind": "port",
                                "sample": f"first {steps} of 321 steps of the same workload, oracle C "
                                          f"restatement (OpenMP, {threads} threads)"}
    dist.barrier()
    dist.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
