"""Benchmark: converged timesteps/s of the SHAKTI head solve + field updates on the 4096^2 seasonal
workload, rel-res 1e-8 linear solves, on 1..N GPUs (one independent replica instance per rank).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form plain|mixed] [--impl ours|reference]

One step is one timestep (update_ieb!, Picard to convergence with every CG solve at
||b - A h||_2 <= 1e-8 ||b||_2, step_b!).  `value` times K device-resident steps with CUDA events
after W warm-up steps; `e2e` re-runs the same K steps from the same state through the public API
with each step's forcing (the ieb field) copied in from pinned host memory and the step's result
(h and b) copied back.  The reference arm (--impl reference) times the CPU restatement of the
reference algorithm on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import __graft_entry__ as entry  # noqa: E402

METRIC = "converged timesteps/s at 4096² (rel-res 1e-8), chosen form vs plain FP64 GPU CG"
UNIT = "timesteps/s"
CG_WORDS = {"plain": 14, "mixed": 14}  # words per cell per CG iteration (A: 7, B: 7)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="plain", choices=["plain", "mixed"])
    ap.add_argument("--precond", default="jacobi", choices=["jacobi", "chebyshev"])
    ap.add_argument("--workload", default="seasonal4096")
    ap.add_argument("--dt", type=float, default=1800.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-sample-s", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--out", default=None, help="also write the JSON line here")
    ap.add_argument("--profile-cg", type=int, default=0,
                    help="profiling case: initialise the workload, assemble once and run exactly this many CG "
                         "iterations (plain, then mixed inner), then exit")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------------------------
def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
        pg = dist
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        load = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------------
def make_sim(shk, w, args, state=None):
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    p = shk.ModelParameters(**w.params)
    sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
    s = state or shk.State(g)
    shk.set_initial_conditions(s, g, p, sl, **w.inputs)
    kw = dict(stop_rule="relres", rtol=1e-8, atol=0.0)
    if args.form == "mixed":
        kw.update(precision="mixed", inner_rtol=1e-2)
    cheb = 4 if args.precond == "chebyshev" else None
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, chebyshev_degree=cheb, **kw)
    ps = shk.PicardSolver(500, 1e-6, ls, g)
    mi = shk.SeasonalBaseMeltInput(**w.melt) if w.melt else shk.ConstantMeltInput()
    sim = shk.Simulation(g, s, 1, args.dt, p, "implicit", [], mi, sl, ps=ps)
    return sim


def run_steps(shk, sim, n, record=None):
    for _ in range(n):
        shk.step(sim)
        sim.total_time += sim.dt
        if record is not None:
            ps = sim.hs.ps
            record.append(dict(picard=ps.last_iter, converged=ps.converged, cg=ps.cg_iters_total))


def measure_cg_iteration(shk, sim, iters=200):
    """Average duration of one CG iteration (kernels A + B) on the current assembled system, by
    CUDA events around exactly `iters` iterations (rtol = 0, itmax = iters)."""
    import torch
    ls = sim.ls
    saved = (ls.rtol, ls.atol, ls.itmax, ls.stop_rule, ls.precision)
    h0 = sim.state.h.clone()
    ls.rtol, ls.atol, ls.itmax, ls.stop_rule, ls.precision = 0.0, 0.0, iters, "relres", "fp64"
    ctx = sim.ctx()
    import ctypes as C
    assert ctx.L.shk_assemble(ctx.h, 0, 0.0) == 0
    o = ls.opts()
    st = shk._lib.shk_cg_stats()
    ctx.L.shk_cg_solve(ctx.h, C.byref(o), C.byref(st))  # warm
    sim.state.h.copy_(h0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ctx.L.shk_cg_solve(ctx.h, C.byref(o), C.byref(st))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    sim.state.h.copy_(h0)
    ls.rtol, ls.atol, ls.itmax, ls.stop_rule, ls.precision = saved
    return ms / max(st.niter, 1), int(st.niter)


def ours(args, world, rank, local, pg):
    import numpy as np
    import torch
    shk = entry.load_package()
    w = shk.configs.WORKLOADS[args.workload]()
    if rank > 0:  # independent replica per rank: same shape, different seed
        w = shk.configs.seasonal_bench(w.nx, w.lx, seed=w.seed + 1000 * rank)
    cells = w.nx * w.ny

    # ---- device-resident pass -------------------------------------------------------------
    sim = make_sim(shk, w, args)
    warm = []
    run_steps(shk, sim, args.warmup, warm)
    torch.cuda.synchronize()
    ctx = sim.ctx()
    launches0 = ctx.launches()
    clocks = ClockSampler(torch.cuda.current_device())
    barrier(pg)
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rec = []
    e0.record()
    run_steps(shk, sim, args.steps, rec)
    e1.record()
    torch.cuda.synchronize()
    barrier(pg)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = ctx.launches() - launches0
    ms_max = max_over_ranks(pg, ms)
    value = world * args.steps / (ms_max / 1e3)
    state_after = sim.state.h.clone()

    # dominant kernel: one CG iteration (k_cg_A + k_cg_B), measured live on the current system
    it_ms, it_n = measure_cg_iteration(shk, sim)
    bytes_per_iter = CG_WORDS["plain"] * 8 * cells
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = bytes_per_iter / (it_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None,
                "kernel": "k_cg_A + k_cg_B (one Jacobi-PCG iteration, Float64)",
                "algorithmic_bytes_per_launch": bytes_per_iter, "us_per_iteration": round(it_ms * 1e3, 2),
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s"}
    traffic_file = ROOT / "profiles" / "cg_traffic_per_cell.json"
    if traffic_file.exists():
        tr = json.loads(traffic_file.read_text())
        roofline["traffic"] = round(tr["bytes_per_cell_per_iteration"] * cells)
        roofline["traffic_source"] = tr.get("source")
    del sim
    torch.cuda.empty_cache()

    # ---- end-to-end pass through the public API with host buffers ---------------------------
    e2e = None
    if not args.no_e2e:
        sim = make_sim(shk, w, args)
        run_steps(shk, sim, args.warmup)
        mi = sim.mi
        host_ieb = torch.empty((w.ny, w.nx), dtype=torch.float64).pin_memory()
        host_h = torch.empty((w.ny, w.nx), dtype=torch.float64).pin_memory()
        host_b = torch.empty((w.ny, w.nx), dtype=torch.float64).pin_memory()
        base_t = torch.from_numpy(np.ascontiguousarray(w.melt["base"].T)) if w.melt else None
        forcings = []
        tt = sim.total_time
        for k in range(args.steps):  # the step's forcing, computed on the host before timing
            v = mi.value(tt) if w.melt else 0.0
            f = torch.empty((w.ny, w.nx), dtype=torch.float64).pin_memory()
            f.copy_(base_t + v if base_t is not None else torch.full((w.ny, w.nx), v))
            forcings.append(f)
            tt += sim.dt
        sim.mi = shk.ConstantMeltInput()  # ieb now arrives from the host each step
        barrier(pg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for k in range(args.steps):
            sim.state.ieb.t().copy_(forcings[k], non_blocking=True)
            shk.step(sim)
            sim.total_time += sim.dt
            host_h.copy_(sim.state.h.t(), non_blocking=True)
            host_b.copy_(sim.state.b.t(), non_blocking=True)
        f1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        barrier(pg)
        e2e_ms = max_over_ranks(pg, f0.elapsed_time(f1))
        same = bool(torch.equal(sim.state.h, state_after))
        e2e = {"value": round(world * args.steps / (e2e_ms / 1e3), 4), "unit": UNIT,
               "h2d_bytes_per_step": cells * 8, "d2h_bytes_per_step": 2 * cells * 8,
               "ms_per_step": round(e2e_ms / args.steps, 3), "wall_s": round(wall, 3),
               "same_trajectory_as_value": same}
        del sim
        torch.cuda.empty_cache()

    # ---- CPU baseline (rank 0, N = 1 only) --------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(shk, w, args, warm, rec)

    total_cg = sum(r["cg"] for r in rec)
    total_pic = sum(r["picard"] for r in rec)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.form == "plain" else "f32+f64",
        "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": f"{w.name}: {w.nx}x{w.ny} cells, {w.lx / 1e3:g} km, seasonal melt + 64 moulins, "
                               f"10% LAND/OTHER_BASIN blobs",
                   "form": f"{args.form}-{args.precond}", "stop": "relres 1e-8 (||b-Ah||/||b||)",
                   "picard": "500 iters, tol 1e-6", "dt_s": args.dt, "sliding": f"RegularizedCoulomb C={w.sliding_C}",
                   "params": w.params, "gap": "implicit", "kface": "arithmetic",
                   "l2": "inputs larger than L2 (about 8 GB resident per GPU)",
                   "parallelism": f"replicas x{world} (independent instances, no data-path collective)"},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(sum_over_ranks(pg, launches)),
        "clocks": clk,
        "timed_steps": {"picard_iters": total_pic, "cg_iters": total_cg,
                        "per_step": rec, "all_converged": all(r["converged"] for r in rec)},
    }
    return line


def cpu_baseline(shk, w, args, warm, rec):
    """The CPU restatement of the reference algorithm on the host cores, on a bounded sample of
    the same workload: the 4096^2 initial state, timing one assembly, one field-update tail, one
    gap step and a run of Jacobi CG iterations; the timestep rate is these costs combined with the
    timed window's Picard and CG iteration counts (identical for the reference algorithm: the
    parity tests match iteration counts to +-1 per solve)."""
    orc = entry.load_oracle()
    orc.build()
    threads = os.cpu_count() or 1
    orc.set_num_threads(threads)
    costs = oracle_costs(orc, w, args.cpu_sample_s)
    steps = len(rec)
    pic = sum(r["picard"] for r in rec)
    cg = sum(r["cg"] for r in rec)
    sec = pic * (costs["assemble_s"] + costs["tail_s"]) + cg * costs["cg_iter_s"] + steps * costs["gap_s"]
    return {"value": round(steps / sec, 6), "unit": UNIT, "cores": orc.num_threads(), "kind": "port",
            "sample": (f"CPU restatement (C, OpenMP {orc.num_threads()} threads) on the {w.nx}^2 initial state: "
                       f"1 assembly ({costs['assemble_s']:.3f} s), 1 tail ({costs['tail_s']:.3f} s), 1 gap step "
                       f"({costs['gap_s']:.3f} s), {costs['cg_iters']} Jacobi CG iterations "
                       f"({costs['cg_iter_s'] * 1e3:.1f} ms each); rate = these costs x the timed window's "
                       f"{pic} Picard and {cg} CG iterations over {steps} steps"),
            "costs": costs}


def oracle_state(orc, w):
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    osl = orc.SlidingSpec(kind=0, C=w.sliding_C)
    orc.set_initial_conditions(st, w.params, osl, w.inputs)
    return st, osl


def oracle_costs(orc, w, budget_s, prepared=None):
    st, osl = prepared or oracle_state(orc, w)
    t0 = time.perf_counter()
    A = orc.assemble(st, w.params)
    t_asm = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc.picard_tail(st, w.params, osl)
    t_tail = time.perf_counter() - t0
    b_saved = st["b"].copy(), st["beta"].copy(), st["b_x"].copy(), st["b_y"].copy()
    t0 = time.perf_counter()
    orc.step_b(st, w.params, 1, 1800.0)
    t_gap = time.perf_counter() - t0
    for arr, v in zip((st["b"], st["beta"], st["b_x"], st["b_y"]), b_saved):
        arr[...] = v
    n = 4
    t0 = time.perf_counter()
    orc.cg(A, st["h"], orc.CgSpec(precond=0, stop_rule=1, rtol=0.0, atol=0.0, itmax=n))
    t_first = time.perf_counter() - t0
    per = t_first / n
    n2 = max(4, min(200, int(max(budget_s - t_first, 1.0) / max(per, 1e-6))))
    t0 = time.perf_counter()
    _, s2 = orc.cg(A, st["h"], orc.CgSpec(precond=0, stop_rule=1, rtol=0.0, atol=0.0, itmax=n2))
    t_cg = time.perf_counter() - t0
    # one CG call = one initial residual matvec + n2 iterations; subtract the setup share
    t_setup = max(t_first - n * (t_cg / n2), 0.0)
    cg_iter = max((t_cg - t_setup) / max(s2["niter"], 1), 1e-9)
    return {"assemble_s": t_asm, "tail_s": t_tail, "gap_s": t_gap, "cg_iter_s": cg_iter, "cg_iters": int(s2["niter"])}


# ---------------------------------------------------------------------------------------------
# reference arm: the CPU restatement of the reference algorithm on the host cores
# ---------------------------------------------------------------------------------------------
def reference(args, world, rank, local, pg):
    if rank != 0:
        return None
    shk = entry.load_package()
    orc = entry.load_oracle()
    orc.build()
    w = shk.configs.WORKLOADS[args.workload]()
    counts_file = ROOT / "profiles" / "step_counts_seasonal4096.json"
    counts = json.loads(counts_file.read_text()) if counts_file.exists() else None
    threads = os.cpu_count() or 1
    orc.set_num_threads(threads)
    per_step = []
    prepared = oracle_state(orc, w)
    for k in range(args.warmup + args.steps):
        c = oracle_costs(orc, w, max(args.cpu_sample_s / 4, 2.0), prepared)
        if k >= args.warmup:
            per_step.append(c)
    mean = {k: statistics.mean(c[k] for c in per_step) for k in ("assemble_s", "tail_s", "gap_s", "cg_iter_s")}
    if counts:
        pic, cg, steps = counts["picard_iters"], counts["cg_iters"], counts["steps"]
    else:
        pic, cg, steps = 1, 0, 1
    sec = pic * (mean["assemble_s"] + mean["tail_s"]) + cg * mean["cg_iter_s"] + steps * mean["gap_s"]
    value = steps / sec
    sample = (f"CPU restatement of the reference algorithm (C, OpenMP {orc.num_threads()} threads; Julia is absent) "
              f"on the {w.nx}^2 workload: each step times 1 assembly, 1 tail, 1 gap step and a run of Jacobi CG "
              f"iterations on the initial state; timesteps/s = these costs x the per-step Picard/CG iteration counts "
              f"of the same workload's timed window ({pic} Picard, {cg} CG over {steps} steps"
              f"{', from ' + counts_file.name if counts else ', counts unavailable: 1 Picard iteration per step'})")
    return {"metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 / value, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": f"{w.name}: {w.nx}x{w.ny} cells", "form": "reference Threads/Float64 CG (Jacobi)"},
            "impl": "reference",
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": orc.num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "costs": mean}


def profile_cg(args):
    """Small, self-ending case for ncu: one assembly and exactly args.profile_cg CG iterations in
    Float64 and in Float32 (mixed inner) on the workload's initial state."""
    import ctypes as C
    import torch
    shk = entry.load_package()
    w = shk.configs.WORKLOADS[args.workload]()
    sim = make_sim(shk, w, args)
    ctx = sim.ctx()
    assert ctx.L.shk_assemble(ctx.h, 0, 0.0) == 0
    out = {}
    for prec in ("fp64", "mixed"):
        ls = sim.ls
        ls.precision, ls.stop_rule, ls.rtol, ls.atol, ls.itmax = prec, "relres", 0.0, 0.0, args.profile_cg
        ls.max_refine = 1
        o = ls.opts()
        if prec == "mixed":
            o.inner_rtol = 1e-30  # inner solve runs exactly itmax iterations
        st = shk._lib.shk_cg_stats()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.L.shk_cg_solve(ctx.h, C.byref(o), C.byref(st))
        torch.cuda.synchronize()
        out[prec] = dict(niter=st.niter, ms=round((time.perf_counter() - t0) * 1e3, 3))
    print(json.dumps({"profile_cg": out, "workload": w.name, "cells": w.nx * w.ny}))


def main():
    args = parse()
    if args.profile_cg:
        return profile_cg(args)
    world, rank, local, pg = dist_setup(args) if args.impl == "ours" else (
        int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0, None)
    try:
        line = ours(args, world, rank, local, pg) if args.impl == "ours" else reference(args, world, rank, local, pg)
        if rank == 0 and line is not None:
            s = json.dumps(line)
            print(s, flush=True)
            if args.out:
                Path(args.out).write_text(s + "\n")
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
