"""Benchmark: converged timesteps/s of the SHAKTI head solve + field updates on the 4096^2 seasonal
workload, rel-res 1e-8 linear solves, on 1..N GPUs (one independent replica instance per rank).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form multigrid|plain|fp32cg]
                    [--impl ours|reference]

One step is one timestep (update_ieb!, Picard to convergence with every CG solve at
||b - A h||_2 <= 1e-8 ||b_G||_2, b_G the GROUNDED rows of b, step_b!).  `value` times K
device-resident steps of the chosen form (default: Float64 CG preconditioned by the Float32
aggregation-multigrid V-cycle) with CUDA events after W warm-up steps; `plain_fp64_gpu` times plain
Float64 Jacobi CG (the reference's algorithm on the GPU) over the window's first --plain-steps
timesteps, from the same state, beside the chosen form's own time for those timesteps; `e2e`
re-runs the chosen form's K steps from the same state through the public API (`HostIO.run`) with
each step's forcing (the ieb field) copied in from pinned host memory and the step's result (h and
b) copied back, the copies overlapping the neighbouring steps' computation.  `cpu_baseline` and
the reference arm (--impl reference) run the CPU restatement of the reference algorithm's real
run loop on the host cores for a bounded time.
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
# Algorithmic bytes per cell of one CG iteration.  Jacobi (Float64): k_cg_A reads aP, aE, aN, r,
# p_old and writes p_new, Ap; k_cg_B reads aP, p_new, Ap, x, r and writes x, r (14 words).  With the
# multigrid preconditioner, k_cg_A reads z instead of r (7 words) and the x/r update is counted
# with the V-cycle's first kernel (mg_vcycle_bytes).
CG_BYTES = {"plain": 14 * 8, "fp32cg": 14 * 4, "multigrid": 7 * 8}
FORMS = {"multigrid": "Float64 CG + Float32 aggregation-multigrid V-cycle preconditioner",
         "plain": "Float64 CG, Jacobi (the reference algorithm)",
         "fp32cg": "Float32 Jacobi CG with Float64 residual replacement"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="multigrid", choices=list(FORMS))
    ap.add_argument("--no-plain", action="store_true", help="skip the plain Float64 comparison pass")
    ap.add_argument("--precond", default="jacobi", choices=["jacobi", "chebyshev"])
    ap.add_argument("--workload", default="seasonal4096")
    ap.add_argument("--dt", type=float, default=1800.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-sample-s", type=float, default=25.0,
                    help="cpu_baseline: wall seconds of the CPU restatement's run loop to time")
    ap.add_argument("--ref-slice-s", type=float, default=5.0,
                    help="reference arm: wall seconds of the CPU run loop per bench step")
    ap.add_argument("--ref-precond", default="chebyshev", choices=["jacobi", "chebyshev"],
                    help="CPU legs: the CPU restatement's preconditioner (Chebyshev(4): the CPU plan)")
    ap.add_argument("--plain-steps", type=int, default=2,
                    help="plain Float64 GPU comparison: timed steps from the chosen form's post-warm-up state")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--out", default=None, help="also write the JSON line here")
    ap.add_argument("--ensemble", type=int, default=0,
                    help="ensemble mode: this many instances of the ragged ensemble workload (sizes 128^2..1024^2); "
                         "prints its own JSON line instead of the 4096^2 one")
    ap.add_argument("--ens-form", default="multigrid", choices=["multigrid", "plain"],
                    help="ensemble mode: Float64 CG with the Float32 multigrid V-cycle (mixed precision) or Jacobi")
    ap.add_argument("--ens-c-range", type=float, nargs=2, default=(5e3, 5e4), metavar=("C_MIN", "C_MAX"),
                    help="ensemble mode: range of the instances' sliding coefficient C (default: the described "
                         "5e3-5e4, with which many instances' Picard loops do not converge)")
    ap.add_argument("--ens-sequential", type=int, default=32,
                    help="ensemble mode: instances also run one after another through the single-instance path")
    ap.add_argument("--warmstart", action="store_true",
                    help="learned-warm-start mode: generate first-Picard-iterate pairs from an ensemble run, train "
                         "the network with the library's kernels, and compare seeded and unseeded timesteps on a "
                         "2048^2 instance; prints its own JSON line")
    ap.add_argument("--ws-instances", type=int, default=96)
    ap.add_argument("--ws-steps", type=int, default=48)
    ap.add_argument("--ws-train", type=int, default=4000)
    ap.add_argument("--nn-infer", type=int, default=0,
                    help="profiling case: this many forward passes of the (untrained) warm-start network on a "
                         "packed 2048^2 state, then exit")
    ap.add_argument("--profile-cg", type=int, default=0,
                    help="profiling case: initialise the workload, assemble once and run exactly this many CG "
                         "iterations of each form, then exit")
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


def _dev(pg):
    return "cpu" if pg.get_backend() == "gloo" else "cuda"


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=_dev(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=_dev(pg))
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def replica_value(pg, world: int, steps: int, ms_local: float):
    """Whole-job timesteps/s of `world` independent replicas, each running `steps` steps: all
    ranks' steps over the slowest rank's device time (the max over ranks)."""
    ms = max_over_ranks(pg, ms_local)
    return world * steps / (ms / 1e3), ms


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
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # the timed region starts once the sampler is producing samples (it takes a moment to start)
            t_end = time.time() + 3.0
            while time.time() < t_end and Path(self.path).stat().st_size == 0:
                time.sleep(0.01)
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
def make_sim(shk, w, args, state=None, form=None):
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    p = shk.ModelParameters(**w.params)
    sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
    s = state or shk.State(g)
    shk.set_initial_conditions(s, g, p, sl, **w.inputs)
    form = form or args.form
    kw = dict(stop_rule="relres", rtol=1e-8, atol=0.0)
    if form == "fp32cg":
        kw.update(precision="mixed", inner_rtol=1e-2)
    cheb = 4 if (args.precond == "chebyshev" and form != "multigrid") else None
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, chebyshev_degree=cheb,
                               multigrid=(form == "multigrid"), **kw)
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


def mg_vcycle_bytes(nx, ny, fused=True):
    """Algorithmic bytes of one V-cycle (all levels, nu = 2 sweeps per side).
    Fused level kernels (the default): level 0 (Float64 residual in, Float64 z out), per fine cell,
    descending half with the CG's r update folded in and its x update once per two iterations --
    62 B on average: r, Ap 16 B, activity flag 1, operator wD dP aE aN 16 in, new r 8, the level's
    iterate 4, coarse rhs 1 out, and every second iteration p, p_prev, x 24 B in and x 8 B out --
    and ascending half 38 B (iterate 4, coarse iterate 1, flag 1, operator 16, r 8 in; z 8 out);
    each coarse level above the bottom, per cell, 26 + 30 B (Float32 rhs).  Per-sweep kernels:
    level 0 17 + 33 + 26 + 34 + 37 B, coarse levels 13 + 29 + 22 + 30 + 29 B.  The levels the
    one-block bottom kernel takes (at most 1400 cells in all, 29 B per cell within 200 KiB) are
    read once (operator 17 B + rhs 4 B per cell) and level lb's result written once (4 B)."""
    dims = [(nx, ny)]
    while dims[-1] != (1, 1):
        a, b = dims[-1]
        dims.append(((a + 1) // 2, (b + 1) // 2))
    cells = [a * b for a, b in dims]
    lb = len(dims) - 1
    rest = 0
    for l in range(len(dims) - 1, 0, -1):
        rest += cells[l]
        if rest * 29 > 200 * 1024 or rest > 1400:
            break
        lb = l
    top, coarse = (100, 56) if fused else (147 + 48, 123)  # per-sweep: plus k_cg_B's 48 B
    total = top * cells[0] if len(dims) > 1 else 37 * cells[0]
    for l in range(1, lb):
        total += coarse * cells[l]
    if len(dims) > 1:
        total += 25 * cells[lb] + sum(17 * cells[l] for l in range(lb + 1, len(dims)))
    return total


def iteration_bytes(form, nx, ny):
    cells = nx * ny
    b = CG_BYTES[form] * cells
    if form == "multigrid":
        b += mg_vcycle_bytes(nx, ny, fused=os.environ.get("SHK_MG_FUSED", "1") != "0")
    return b


# Whole-timestep algorithmic bytes per cell (Float64 words of the reference's data layout): a Picard
# iteration's assembly, field tail and convergence check read 17 and write 24 fields (five
# coefficient arrays, rhs, pw, N, the face gradients, fluxes, Reynolds numbers and stresses, the
# melt terms, K) and write and read back h_prev: 43 words; a gap step reads 7 fields and writes 4.
PICARD_BYTES, GAP_BYTES = 43 * 8, 11 * 8


def step_bytes(form, nx, ny, counts):
    """Algorithmic bytes of the timed window per timestep: every Picard iteration's field work,
    every CG iteration of `form`, every gap step."""
    cells = nx * ny
    total = (counts["picard_iters"] * PICARD_BYTES * cells + counts["cg_iters"] * iteration_bytes(form, nx, ny)
             + counts["steps"] * GAP_BYTES * cells)
    return total / max(counts["steps"], 1)


def step_roofline(form, w, counts, ms_per_step, peaks):
    b = step_bytes(form, w.nx, w.ny, counts)
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = b / (ms_per_step / 1e3) / 1e9
    return {"bound": "hbm", "bytes_per_step": int(b), "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "accounting": (f"per timestep: {counts['picard_iters']}/{counts['steps']} Picard iterations x "
                           f"{PICARD_BYTES} B/cell (assembly, tail, check) + {counts['cg_iters']}/{counts['steps']} "
                           f"CG iterations x {iteration_bytes(form, w.nx, w.ny) / (w.nx * w.ny):.1f} B/cell + "
                           f"{GAP_BYTES} B/cell (gap step)"),
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s (of fallback)"}


def measure_cg_iteration(shk, sim, form, short=20, long=220):
    """Average duration of one CG iteration of `form` (its matvec, update and, for the multigrid
    form, V-cycle kernels) on the current assembled system: CUDA events around a solve of exactly `long`
    iterations minus one of `short` iterations (rtol = 0), so set-up and initial residual cancel."""
    import ctypes as C
    import torch
    ls = sim.ls
    saved = (ls.rtol, ls.atol, ls.itmax, ls.stop_rule, ls.precision, ls.max_refine, ls.inner_rtol)
    h0 = sim.state.h.clone()
    ctx = sim.ctx()
    assert ctx.L.shk_assemble(ctx.h, 0, 0.0) == 0

    def timed(iters):
        ls.rtol, ls.atol, ls.itmax, ls.stop_rule = 0.0, 0.0, iters, "relres"
        if form == "fp32cg":
            ls.precision, ls.max_refine, ls.inner_rtol = "mixed", 1, 1e-30
        o = ls.opts()
        st = shk._lib.shk_cg_stats()
        sim.state.h.copy_(h0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.L.shk_cg_solve(ctx.h, C.byref(o), C.byref(st))
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), int(st.niter)

    timed(short)  # warm (graph capture, caches)
    ms_s, n_s = timed(short)
    ms_l, n_l = timed(long)
    sim.state.h.copy_(h0)
    ls.rtol, ls.atol, ls.itmax, ls.stop_rule, ls.precision, ls.max_refine, ls.inner_rtol = saved
    return (ms_l - ms_s) / max(n_l - n_s, 1), n_l - n_s


def roofline_for(shk, sim, form, w, peaks):
    it_ms, it_n = measure_cg_iteration(shk, sim, form)
    nbytes = iteration_bytes(form, w.nx, w.ny)
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = nbytes / (it_ms / 1e3) / 1e9
    kernel = {"plain": "k_cg_matvec_t<true> + k_cg_B (one Jacobi-PCG iteration, Float64: the p update with "
                       "z = r/aP and the matvec on TMA-staged tiles, then the x/r update)",
              "fp32cg": "k_cg_A + k_cg_B (one Jacobi-PCG iteration, Float32 Laplacian form)",
              "multigrid": "one multigrid-preconditioned CG iteration: the TMA-staged Float64 p update and "
                           "matvec (k_cg_matvec_t), the Float32 V-cycle on TMA-staged tiles (k_mg_down_t, its "
                           "level-0 launch with the CG's x/r update, k_mg_up_t) and the one-block k_mg_bottom"}[form]
    r = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
         "frac": round(achieved / peak, 4), "traffic": None, "kernel": kernel,
         "algorithmic_bytes_per_launch": nbytes, "us_per_iteration": round(it_ms * 1e3, 2),
         "iterations_timed": it_n,
         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s (of fallback)"}
    tf = ROOT / "profiles" / f"traffic_{form}_{w.name}.json"
    if tf.exists():
        tr = json.loads(tf.read_text())
        r["traffic"] = int(tr["dram_bytes_per_iteration"])
        r["traffic_source"] = tr.get("source")
    return r


def timed_pass(shk, w, args, form, pg, clocks=None, steps=None, state=None, keep_snapshot=False):
    """W warm-up steps, then K timed steps of `form` (device-resident), with a CUDA event after
    every step; returns the record.  state: a snapshot (field -> tensor, plus 'total_time') to
    start from instead of the workload's initial state; then no warm-up steps run.
    keep_snapshot: also return the state after the warm-up (before the timed steps)."""
    import torch
    steps = args.steps if steps is None else steps
    sim = make_sim(shk, w, args, form=form)
    warm = []
    if state is not None:
        load_snapshot(sim, state)
    else:
        run_steps(shk, sim, args.warmup, warm)
    snap = snapshot(sim) if keep_snapshot else None
    torch.cuda.synchronize()
    ctx = sim.ctx()
    launches0 = ctx.launches()
    barrier(pg)
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    rec = []
    evs[0].record()
    for k in range(steps):
        run_steps(shk, sim, 1, rec)
        evs[k + 1].record()
    torch.cuda.synchronize()
    barrier(pg)
    clk = clocks.stop() if clocks else None
    ms = evs[0].elapsed_time(evs[-1])
    step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(steps)]
    for r, m in zip(rec, step_ms):
        r["ms"] = round(m, 3)
    return dict(sim=sim, rec=rec, warm=warm, ms=ms, ms_max=max_over_ranks(pg, ms), step_ms=step_ms,
                launches=ctx.launches() - launches0, clocks=clk, h_after=sim.state.h.clone(), snap=snap)


def snapshot(sim) -> dict:
    """Device copies of every State field and the simulation clock."""
    from shakti_b200 import _lib
    snap = {f: getattr(sim.state, f).clone() for f in _lib.STATE_FIELDS}
    snap["total_time"] = sim.total_time
    return snap


def load_snapshot(sim, snap: dict) -> None:
    for f, t in snap.items():
        if f != "total_time":
            getattr(sim.state, f).copy_(t)
    sim.total_time = snap["total_time"]


def counts_of(rec):
    return {"steps": len(rec), "picard_iters": sum(r["picard"] for r in rec), "cg_iters": sum(r["cg"] for r in rec),
            "all_converged": all(r["converged"] for r in rec)}


def bench_config(w, args, world) -> dict:
    """The workload both arms time (the same dict in both JSON lines)."""
    return {"workload": f"{w.name}: {w.nx}x{w.ny} cells, {w.lx / 1e3:g} km, seasonal melt + 64 moulins, "
                        f"10% LAND/OTHER_BASIN blobs",
            "stop": "relres 1e-8: ||b - A h||_2 (every row) <= 1e-8 ||b||_2 over the GROUNDED rows (Float64)",
            "picard": "500 iters, tol 1e-6", "dt_s": args.dt, "sliding": f"RegularizedCoulomb C={w.sliding_C}",
            "params": w.params, "gap": "implicit", "kface": "arithmetic",
            "l2": "inputs larger than L2 (about 8 GB resident per GPU)",
            "parallelism": f"replicas x{world} (independent instances, no data-path collective)"}


def ours(args, world, rank, local, pg):
    import numpy as np
    import torch
    shk = entry.load_package()
    w = shk.configs.WORKLOADS[args.workload]()
    if rank > 0:  # independent replica per rank: same shape, different seed
        w = shk.configs.seasonal_bench(w.nx, w.lx, seed=w.seed + 1000 * rank)
    cells = w.nx * w.ny
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}

    # ---- device-resident pass of the chosen form ---------------------------------------------
    want_plain = not args.no_plain and args.form != "plain" and args.plain_steps > 0
    main = timed_pass(shk, w, args, args.form, pg, ClockSampler(torch.cuda.current_device()),
                      keep_snapshot=want_plain)
    snap = main.pop("snap")
    value, _ = replica_value(pg, world, args.steps, main["ms"])
    roofline = roofline_for(shk, main["sim"], args.form, w, peaks)
    state_after = main.pop("h_after")
    del main["sim"]
    torch.cuda.empty_cache()

    # ---- plain Float64 Jacobi CG on the GPU over the window's first steps --------------------
    # The plain form needs ~100x the chosen form's time per step, so it times the first
    # --plain-steps steps of the window: it starts from the chosen form's state after the warm-up
    # (the same timestep) and is compared with the chosen form's own time for those steps.
    plain = None
    if want_plain:
        ps = min(args.plain_steps, args.steps)
        probe = make_sim(shk, w, args, form="plain")
        load_snapshot(probe, snap)
        plain_roof = roofline_for(shk, probe, "plain", w, peaks)  # also warms the plain form's graphs
        del probe
        pp = timed_pass(shk, w, args, "plain", pg, steps=ps, state=snap)
        del snap
        pv = world * ps / (pp["ms_max"] / 1e3)
        chosen_ms = max_over_ranks(pg, sum(main["step_ms"][:ps]))
        plain = {"value": round(pv, 4), "unit": UNIT, "steps": ps, "ms_per_step": round(pp["ms_max"] / ps, 3),
                 "chosen_ms_per_step_same_steps": round(chosen_ms / ps, 3),
                 "chosen_over_plain": round(pp["ms_max"] / chosen_ms, 3),
                 "window": f"timesteps {args.warmup + 1}..{args.warmup + ps} (the first {ps} of the timed window), "
                           f"from the chosen form's state after the warm-up",
                 "gpu_launches": int(sum_over_ranks(pg, pp["launches"])), "roofline": plain_roof,
                 "timed_steps": dict(counts_of(pp["rec"]), per_step=pp["rec"])}
        del pp
        torch.cuda.empty_cache()

    # ---- end-to-end pass through the public API with host buffers ---------------------------
    e2e = None
    if not args.no_e2e:
        sim = make_sim(shk, w, args)
        run_steps(shk, sim, args.warmup)
        mi = sim.mi
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
        io = shk.HostIO(sim)  # staging buffers and copy streams, allocated before timing
        barrier(pg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        # every step: its forcing host -> device, the solve, its h and b device -> host (the
        # transfers overlap the neighbouring steps' computation)
        io.run(forcings, host_h, host_b)
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

    # ---- CPU baseline (rank 0, N = 1 only): the CPU restatement's real run loop, bounded -----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(shk, w, args)

    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(main["ms_max"] / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": {"plain": "f64", "fp32cg": "f32+f64", "multigrid": "f64+f32"}[args.form],
        "data": "synthetic (seeded generator, no dataset)",
        "config": bench_config(w, args, world),
        "form": FORMS[args.form],
        "roofline": roofline,
        "step_roofline": step_roofline(args.form, w, counts_of(main["rec"]), main["ms_max"] / args.steps, peaks),
        "plain_fp64_gpu": plain,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(sum_over_ranks(pg, main["launches"])),
        "clocks": main["clocks"],
        "timed_steps": dict(counts_of(main["rec"]), per_step=main["rec"]),
    }
    return line


def cpu_rate(pr: dict) -> tuple[float, str]:
    """Timesteps/s of a bounded CPU run: measured over its completed timesteps, or, when it has not
    completed one, the upper bound 1/(seconds spent on the first timestep so far)."""
    if pr["steps_done"] >= 1:
        return pr["steps_done"] / pr["completed_s"], "measured"
    return 1.0 / pr["elapsed"], "upper bound"


def cpu_session(orc, w, args, precond: str):
    st, osl = oracle_state(orc, w)
    spec = orc.CgSpec(precond=1 if precond == "chebyshev" else 0, cheb_degree=4, cheb_nsteps=15, stop_rule=1,
                      rtol=1e-8, atol=0.0)
    melt = orc.seasonal_melt(w.melt) if w.melt else None
    return orc.RunSession(st, w.params, osl, args.dt, kfs=0, gap_scheme=1, cgspec=spec, melt=melt,
                          picard_iters=500, picard_tol=1e-6)


def cpu_sample_text(w, pr, threads, precond, bound, label):
    prog = (f"{pr['steps_done']} timesteps completed" if pr["steps_done"] else
            f"timestep 1 not completed: Picard iteration {pr['pic_iter_now']} in progress")
    return (f"{label}: the CPU restatement's real run loop (update_ieb!, Picard_loop! with CG "
            f"{'Chebyshev(4)' if precond == 'chebyshev' else 'Jacobi'} to the same relres 1e-8, step_b!; C, OpenMP "
            f"{threads} threads) on the {w.nx}^2 workload from its initial state for {pr['elapsed']:.1f} s of wall "
            f"time: {prog}, {pr['picard_iters']} linear solves and {pr['cg_iters']} CG iterations done; value = "
            + ("completed timesteps / their time" if bound == "measured" else
               "1 / elapsed, an upper bound on the CPU's timesteps/s (no timestep finished)"))


def cpu_progress(pr: dict) -> dict:
    return {k: pr[k] for k in ("steps_done", "picard_iters", "cg_iters", "pic_iter_now", "cg_iter_now", "elapsed",
                               "completed_s")}


def cpu_baseline(shk, w, args):
    """The CPU restatement of the reference algorithm on the host cores, on a bounded sample of the
    same workload: its real run loop from the workload's initial state for --cpu-sample-s seconds."""
    orc = entry.load_oracle()
    orc.build()
    threads = os.cpu_count() or 1
    orc.set_num_threads(threads)
    S = cpu_session(orc, w, args, args.ref_precond)
    pr = S.advance(args.cpu_sample_s)
    S.close()
    v, bound = cpu_rate(pr)
    return {"value": round(v, 6), "unit": UNIT, "cores": orc.num_threads(), "kind": "port", "bound": bound,
            "sample": cpu_sample_text(w, pr, orc.num_threads(), args.ref_precond, bound, "bounded sample"),
            "progress": cpu_progress(pr)}


def oracle_state(orc, w):
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    osl = orc.SlidingSpec(kind=0, C=w.sliding_C)
    orc.set_initial_conditions(st, w.params, osl, w.inputs)
    return st, osl


# ---------------------------------------------------------------------------------------------
# reference arm: the CPU restatement of the reference algorithm on the host cores
# ---------------------------------------------------------------------------------------------
def reference(args, world, rank, local, pg):
    """The reference algorithm's CPU implementation (the C restatement; Julia is absent) on all host
    cores: its real run loop on the same workload from the initial state, W + K bench steps of
    --ref-slice-s seconds each (the loop continues across steps; nothing is re-timed or modeled).
    A 4096^2 timestep of the CPU run takes longer than the whole benchmark, so the value is the
    measured rate if any timestep completes and otherwise the upper bound 1/(time spent on the
    first timestep)."""
    if rank != 0:
        return None
    shk = entry.load_package()
    orc = entry.load_oracle()
    orc.build()
    w = shk.configs.WORKLOADS[args.workload]()
    threads = os.cpu_count() or 1
    orc.set_num_threads(threads)
    S = cpu_session(orc, w, args, args.ref_precond)
    for _ in range(args.warmup):
        S.advance(args.ref_slice_s)
    slices = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        pr = S.advance(args.ref_slice_s)
        slices.append(time.perf_counter() - t0)
    S.close()
    value, bound = cpu_rate(pr)
    ms_step = 1e3 * sum(slices) / max(len(slices), 1)
    sample = cpu_sample_text(w, pr, orc.num_threads(), args.ref_precond, bound,
                             f"{args.warmup} + {args.steps} bench steps of {args.ref_slice_s:g} s each")
    cpu = {"value": round(value, 6), "unit": UNIT, "cores": orc.num_threads(), "kind": "port", "bound": bound,
           "sample": sample}
    return {"metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, no dataset)",
            "config": bench_config(w, args, world),
            "form": f"CPU restatement of the reference algorithm (Threads/Float64 CG, "
                    f"{'Chebyshev(4)' if args.ref_precond == 'chebyshev' else 'Jacobi'})",
            "impl": "reference", "cpu_baseline": cpu,
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "progress": cpu_progress(pr),
            "step_note": "each bench step is one slice of the continuing CPU run loop; ms_per_step is the slice"}


def profile_cg(args):
    """Small, self-ending case for ncu: one assembly and exactly args.profile_cg CG iterations of
    the selected form on the workload's initial state."""
    import ctypes as C
    import torch
    shk = entry.load_package()
    w = shk.configs.WORKLOADS[args.workload]()
    sim = make_sim(shk, w, args)
    ctx = sim.ctx()
    assert ctx.L.shk_assemble(ctx.h, 0, 0.0) == 0
    ls = sim.ls
    ls.stop_rule, ls.rtol, ls.atol, ls.itmax = "relres", 0.0, 0.0, args.profile_cg
    if args.form == "fp32cg":
        ls.max_refine = 1
    o = ls.opts()
    if args.form == "fp32cg":
        o.inner_rtol = 1e-30  # the inner solve runs exactly itmax iterations
    st = shk._lib.shk_cg_stats()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.L.shk_cg_solve(ctx.h, C.byref(o), C.byref(st))
    torch.cuda.synchronize()
    out = dict(form=args.form, niter=st.niter, ms=round((time.perf_counter() - t0) * 1e3, 3))
    print(json.dumps({"profile_cg": out, "workload": w.name, "cells": w.nx * w.ny}))


def ensemble_bench(args):
    """Ragged ensemble: converged instance-timesteps/s of `args.ensemble` instances (sizes drawn
    from 128^2..1024^2, per-instance slope, melt, C, b0) advanced together by shk.Ensemble, beside
    the same instances advanced one after another through the single-instance path.  Both arms run
    the same K timesteps from the instances' initial states (graph set-up and the tile autotune
    are outside the timed region)."""
    import torch
    shk = entry.load_package()
    specs = shk.configs.ensemble_specs(args.ensemble, c_range=tuple(args.ens_c_range))
    params = dict(shk.configs.SEASONAL_PARAMS)

    def make(sp):
        w = shk.configs.ensemble_member(**sp)
        g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
        pm = shk.ModelParameters(**params)
        sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
        st = shk.State(g)
        shk.set_initial_conditions(st, g, pm, sl, **w.inputs)
        ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, stop_rule="relres", rtol=1e-8, atol=0.0,
                                   multigrid=args.ens_form == "multigrid")
        ps = shk.PicardSolver(500, 1e-6, ls, g)
        return shk.Simulation(g, st, args.steps, args.dt, pm, "implicit", [], shk.ConstantMeltInput(), sl, ps=ps)

    sims = [make(sp) for sp in specs]
    cells = sum(s.grid.nx * s.grid.ny for s in sims)
    t0 = time.perf_counter()
    ens = shk.Ensemble(sims, autotune_iters=8)
    setup_s = time.perf_counter() - t0
    ens.run(0)  # builds the timestep graph outside the timed region
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    stats = ens.run(args.steps)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    conv = sum(s["steps_converged"] for s in stats)
    by_size = {}
    for sp, th in zip(specs, ens.march_th):
        by_size.setdefault(sp["nx"], th)
    line = {"metric": "converged instance-timesteps/s, ragged ensemble (128^2..1024^2), rel-res 1e-8",
            "instances_all_steps_converged": sum(1 for x in stats if x["steps_converged"] == args.steps),
            "value": round(conv / (ms / 1e3), 3), "unit": "instance-timesteps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": 0, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
            "dtype": "f64+f32" if args.ens_form == "multigrid" else "f64",
            "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": f"ensemble of {len(sims)} instances, sizes "
                                   f"{dict(sorted((k, sum(1 for s in specs if s['nx'] == k)) for k in by_size))}, "
                                   f"{cells / 1e6:.1f} M cells in total",
                       "form": ("batched Float64 CG preconditioned by the Float32 multigrid V-cycle (every level "
                                "kernel one launch over the instances that have the level), "
                                if args.ens_form == "multigrid" else "batched Float64 Jacobi CG, ")
                               + "one launch per kernel over all instances, one CUDA graph per timestep (device-side "
                                 "Picard and CG loops)",
                       "params": params, "sliding_C_range": list(args.ens_c_range),
                       "picard": "500 iters, tol 1e-6", "dt_s": args.dt,
                       "timing": "the same K steps from the initial states in both arms"},
            "march_th_by_size": by_size, "setup_s": round(setup_s, 2),
            "instance_steps": len(sims) * args.steps, "converged_instance_steps": conv,
            "picard_iters": sum(s["picard_iters"] for s in stats), "cg_iters": sum(s["cg_iters"] for s in stats),
            "clocks": clk}
    ens.close()
    del sims, ens
    torch.cuda.empty_cache()
    if args.ens_sequential:
        # the same first M instances both ways: batched, and one after another
        sub = specs[:args.ens_sequential]
        ens_sims = [make(sp) for sp in sub]
        sub_ens = shk.Ensemble(ens_sims, autotune_iters=8)
        sub_ens.run(0)
        torch.cuda.synchronize()
        e0.record()
        st2 = sub_ens.run(args.steps)
        e1.record()
        torch.cuda.synchronize()
        ms_ens = e0.elapsed_time(e1)
        conv_ens = sum(x["steps_converged"] for x in st2)
        sub_ens.close()
        del ens_sims, sub_ens
        seq = [make(sp) for sp in sub]
        torch.cuda.synchronize()
        e0.record()
        done = 0
        for sim in seq:
            for _ in range(args.steps):
                shk.step(sim)
                sim.total_time += sim.dt
                done += int(sim.hs.ps.converged)
        e1.record()
        torch.cuda.synchronize()
        ms_seq = e0.elapsed_time(e1)
        line["same_instances_both_ways"] = {
            "instances": len(sub), "cells": sum(x.grid.nx * x.grid.ny for x in seq),
            "ensemble": {"value": round(conv_ens / (ms_ens / 1e3), 3), "ms": round(ms_ens, 1)},
            "one_after_another": {"value": round(done / (ms_seq / 1e3), 3), "ms": round(ms_seq, 1)},
            "unit": "instance-timesteps/s", "speedup": round(ms_seq / ms_ens, 2),
            "note": "the first instances of the ensemble; one after another = the single-instance path "
                    "(shk_step per instance, device-side CG loop per solve)"}
    return line


def warmstart_bench(args):
    """Learned warm start: training pairs (first Picard iterate increments) from an ensemble run of
    the plain solver on 128^2 instances, training by the library's BF16 tensor-core kernels, then
    the same 2048^2 instance advanced seeded and unseeded with the multigrid-preconditioned Float64
    CG at rel-res 1e-8: CG and Picard iterations per step, device time per step, and the seeded
    head's error against the unseeded one."""
    import numpy as np
    import torch
    shk = entry.load_package()
    from shakti_b200 import warmstart as ws
    t0 = time.perf_counter()
    net = ws.WarmStartNet(seed=0)
    # training instances whose Picard loops converge (the described C of 5e3-5e4 stops most of them
    # converging under the rel-res rule on the GROUNDED rows); only converged instance-steps are kept
    specs = shk.configs.ensemble_specs(args.ws_instances, seed=99, sizes=(128,), c_range=(0.25, 1e3))
    X, T, M = ws.generate_pairs(shk, net, specs, steps=args.ws_steps, crops=8)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    losses = []
    per = max(1, args.ws_train // 4)
    for lr in (1e-3, 5e-4, 2.5e-4, 1e-4):
        losses += net.train(X, T, M, steps=per, batch=64, lr=lr)
    e1.record()
    torch.cuda.synchronize()
    train_ms = e0.elapsed_time(e1)
    # an instance whose Picard loop converges in a few iterations (C = 0.25; the described C of
    # 5e3-5e4, and even 500, take hundreds of Picard iterations per step at this size)
    spec = dict(nx=2048, seed=556, slope=0.018, melt=8e-8, C=0.25, b0=0.007)
    sim = ws.member_sim(shk, spec, multigrid=True)
    Xp = net.pack(sim.state)
    net.forward(Xp)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(5):
        net.forward(Xp)
    e1.record()
    torch.cuda.synchronize()
    infer_ms = e0.elapsed_time(e1) / 5
    del sim
    ev = ws.evaluate(shk, net, spec, steps=args.steps, settle=2, multigrid=True)
    line = {"metric": "learned warm start at 2048^2: CG iterations and time per converged timestep, seeded vs "
                      "unseeded (rel-res 1e-8)",
            "value": round(ev["seeded"]["cg_per_step"], 2), "unit": "CG iterations/step (seeded)",
            "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": 2,
            "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": "ensemble member at 2048x2048 (dx 156 m), multigrid-preconditioned Float64 CG",
                       "network": "4-level conv encoder-decoder, 32 base channels, BF16 weights/activations, "
                                  "Float32 accumulation (tcgen05.mma kind::f16, TMEM accumulator)",
                       "training": f"{X.shape[0]} pairs of 32x32 crops from {len(specs)} 128^2 instances x "
                                   f"{args.ws_steps} steps, {len(losses)} Adam steps of batch 64"},
            "unseeded": {k: ev["unseeded"][k] for k in ("cg_per_step", "picard_per_step", "ms_per_step")},
            "seeded": {k: ev["seeded"][k] for k in ("cg_per_step", "picard_per_step", "ms_per_step")},
            "seed_accepted": ev["seeded"]["seed"]["seeded"],
            "initial_residual_ratio": [round(b / a, 3) for a, b in zip(ev["seeded"]["seed"]["r_prev"],
                                                                        ev["seeded"]["seed"]["r_seed"])],
            "h_relerr_vs_unseeded": ev["h_relerr_vs_unseeded"],
            "training": {"pairs": int(X.shape[0]), "data_s": round(gen_s, 1), "train_ms": round(train_ms, 1),
                         "loss_first": round(float(np.mean(losses[:50])), 4),
                         "loss_last": round(float(np.mean(losses[-200:])), 4)},
            "inference_ms_2048": round(infer_ms, 3)}
    return line


def nn_infer(args):
    """Small, self-ending case for ncu: forward passes of the warm-start network at 2048^2."""
    import torch
    shk = entry.load_package()
    from shakti_b200 import warmstart as ws
    net = ws.WarmStartNet(seed=0)
    sim = ws.member_sim(shk, dict(nx=2048, seed=556, slope=0.018, melt=8e-8, C=4e4, b0=0.007))
    X = net.pack(sim.state)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.nn_infer):
        net.forward(X)
    torch.cuda.synchronize()
    print(json.dumps({"nn_infer": args.nn_infer, "ms": round((time.perf_counter() - t0) * 1e3, 3)}))


def main():
    args = parse()
    if args.nn_infer:
        return nn_infer(args)
    if args.warmstart:
        line = warmstart_bench(args)
        s = json.dumps(line)
        print(s, flush=True)
        if args.out:
            Path(args.out).write_text(s + "\n")
        return
    if args.profile_cg:
        return profile_cg(args)
    if args.ensemble:
        line = ensemble_bench(args)
        s = json.dumps(line)
        print(s, flush=True)
        if args.out:
            Path(args.out).write_text(s + "\n")
        return
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
