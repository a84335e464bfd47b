"""Simulation / run! / step! and set_initial_conditions! mirroring Shakti.jl (src/simulation.jl,
src/run.jl, src/initial_conditions.jl), driving libshakti_b200."""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _lib
from .model import (Arithmetic, Harmonic, ModelParameters, PrescribedSlidingLaw, State, Grid, AbstractMeltInput,
                    AbstractSlidingLaw)
from .observers import FILE_WRITERS, IOObserver
from .solvers import (_Context, AbstractLinearSolver, CGIterativeSolver, PicardSolver, solve_parabolic_linear_system)


# ---------------------------------------------------------------------------------------------
# Schemes (src/simulation.jl:9-56, src/melt_rate.jl:19-33, src/gap_height.jl:22-43)
# ---------------------------------------------------------------------------------------------
class AbstractHeadScheme:
    pass


class EllipticHeadScheme(AbstractHeadScheme):
    def __init__(self, ps: PicardSolver):
        self.ps = ps


class ParabolicHeadScheme(AbstractHeadScheme):
    def __init__(self, ls: AbstractLinearSolver):
        self.ls = ls


class AbstractGapScheme:
    code = -1


class ExplicitGapScheme(AbstractGapScheme):
    code = 0


class ImplicitGapScheme(AbstractGapScheme):
    code = 1


class AbstractSensibleHeatScheme:
    pass


class WithSensibleHeat(AbstractSensibleHeatScheme):
    pass


class NoSensibleHeat(AbstractSensibleHeatScheme):
    pass


class AbstractOpenBySlidingScheme:
    pass


class WithOpenBySliding(AbstractOpenBySlidingScheme):
    pass


class NoOpenBySliding(AbstractOpenBySlidingScheme):
    pass


# ---------------------------------------------------------------------------------------------
# Observers (src/observer.jl): NoObserver and the in-memory LiveObserver here; IOObserver and its
# file writers in observers.py.
# ---------------------------------------------------------------------------------------------
class AbstractObserver:
    def prepare(self, state):
        pass

    def resume(self, state, t):
        """resume! (src/observer.jl): continue an interrupted run's observation after timestep t."""
        pass

    def observe(self, state, t, total_time):
        pass

    def finalize(self, state):
        pass


class NoObserver(AbstractObserver):
    pass


class LiveObserver(AbstractObserver):
    def __init__(self, tracked_obs, tracked_times):
        self.tracked_obs = list(tracked_obs)
        self.tracked_times = set(int(t) for t in tracked_times)
        self.data = {name: [] for name in self.tracked_obs}
        self.times = []

    def observe(self, state, t, total_time):
        if t in self.tracked_times:
            self.times.append(total_time)
            host = state.to_numpy(self.tracked_obs)
            for name in self.tracked_obs:
                self.data[name].append(host[name])


class Simulation:
    """Simulation(grid, state, tsteps, dt, p, gap_scheme_choice, tracked_obs, mi, sl; ps, ls,
    which_observer, which_file_writer, tracked_times, path, k_face_choice, verbose)
    (src/simulation.jl:105-184)."""

    def __init__(self, grid: Grid, state: State, tsteps: int, dt: float, p: ModelParameters, gap_scheme_choice: str,
                 tracked_obs, mi: AbstractMeltInput, sl: AbstractSlidingLaw, *, ps: PicardSolver | None = None,
                 ls: AbstractLinearSolver | None = None, which_observer=None, which_file_writer=None,
                 tracked_times=None, path=None, k_face_choice: str = "arithmetic", verbose: bool = False):
        for name in tracked_obs:
            if not hasattr(state, "lambda_" if name == "lambda" else name):
                raise ValueError(f'Unknown tracked observable: "{name}" is not a field of State')
        if p.e_v == 0:
            if ps is None:
                raise ValueError("ps (a PicardSolver) must be provided when p.e_v == 0 (elliptic head scheme)")
            self.hs = EllipticHeadScheme(ps)
        else:
            if ls is None:
                raise ValueError("ls (an AbstractLinearSolver) must be provided when p.e_v != 0 (parabolic head scheme)")
            self.hs = ParabolicHeadScheme(ls)
        if gap_scheme_choice == "explicit":
            self.gs = ExplicitGapScheme()
        elif gap_scheme_choice == "implicit":
            self.gs = ImplicitGapScheme()
        else:
            raise ValueError(f'Unknown gap_scheme_choice: "{gap_scheme_choice}" (expected "explicit" or "implicit")')
        self.shs = NoSensibleHeat() if (p.ct == 0 or p.cw == 0) else WithSensibleHeat()
        self.oss = NoOpenBySliding() if p.br == 0 else WithOpenBySliding()
        if k_face_choice == "arithmetic":
            self.kfs = Arithmetic()
        elif k_face_choice == "harmonic":
            self.kfs = Harmonic()
        else:
            raise ValueError(f'Unknown k_face_choice: "{k_face_choice}" (expected "arithmetic" or "harmonic")')
        if len(tracked_obs) == 0:
            self.observer = NoObserver()
        elif which_observer is None:
            raise ValueError('which_observer should be specified as "IO" or "Live" when tracked_obs is not empty.')
        elif which_observer == "IO":
            if which_file_writer is None:
                raise ValueError('which_file_writer should be specified as "NetCDF", "HDF5", "JLD2", or "CSV" when '
                                 'which_observer is "IO".')
            if which_file_writer not in FILE_WRITERS:
                raise ValueError(f'Unknown which_file_writer: "{which_file_writer}" (expected "NetCDF", "HDF5", '
                                 f'"JLD2", or "CSV")')
            if tracked_times is None:
                raise ValueError('tracked_times should be specified when which_observer is "IO".')
            if path is None:
                raise ValueError('path should be specified when which_observer is "IO".')
            self.observer = IOObserver(tracked_obs, tracked_times, FILE_WRITERS[which_file_writer](), path)
        elif which_observer == "Live":
            if tracked_times is None:
                raise ValueError('tracked_times should be specified when which_observer is "Live".')
            self.observer = LiveObserver(tracked_obs, tracked_times)
        else:
            raise ValueError(f'Unknown which_observer: "{which_observer}" (expected "IO" or "Live")')
        self.grid, self.state, self.tsteps, self.dt, self.p = grid, state, int(tsteps), float(dt), p
        self.mi, self.sl, self.verbose = mi, sl, bool(verbose)
        self.total_time = 0.0
        self.step_stats = []

    @property
    def ls(self) -> CGIterativeSolver:
        return self.hs.ps.ls if isinstance(self.hs, EllipticHeadScheme) else self.hs.ls

    def ctx(self) -> _Context:
        return self.ls.ctx.bind(self.state, self.p, self.sl, self.kfs, self.gs.code)


def picard_status(hs: AbstractHeadScheme):
    """src/run.jl:64-65"""
    if isinstance(hs, EllipticHeadScheme):
        return hs.ps.converged, hs.ps.last_iter
    return None, None


def update_ieb(sim: Simulation) -> None:
    """update_ieb!(sim.mi, sim.state, sim.total_time) (src/melt_input.jl:30, 86-94)."""
    ctx = sim.ctx()
    mi = sim.mi.struct()
    _lib.check(ctx.h, ctx.L.shk_update_ieb(ctx.h, C.byref(mi), float(sim.total_time)))


def step_h(sim: Simulation) -> None:
    """src/run.jl:96-108"""
    if isinstance(sim.hs, EllipticHeadScheme):
        ps = sim.hs.ps
        ctx = sim.ctx()
        st = _lib.shk_picard_stats()
        po, o = ps.opts(), ps.ls.opts()
        rc = ctx.L.shk_picard_solve(ctx.h, C.byref(po), C.byref(o), C.byref(st))
        _lib.check(ctx.h, rc, allow=(_lib.OK, _lib.NOT_CONVERGED))
        ps._record(st)
    else:
        ls = sim.hs.ls
        ctx = sim.ctx()
        st = _lib.shk_cg_stats()
        o = ls.opts()
        rc = ctx.L.shk_parabolic_step(ctx.h, float(sim.dt), C.byref(o), C.byref(st))
        _lib.check(ctx.h, rc, allow=(_lib.OK, _lib.NOT_CONVERGED, _lib.BREAKDOWN))
        ls._record(st)


def step_b(sim: Simulation) -> None:
    """step_b! (src/run.jl:154-164)"""
    ctx = sim.ctx()
    _lib.check(ctx.h, ctx.L.shk_step_b(ctx.h, float(sim.dt)))


def step(sim: Simulation) -> None:
    """step! (src/run.jl:82-88)"""
    update_ieb(sim)
    step_h(sim)
    step_b(sim)


# ---------------------------------------------------------------------------------------------
# Checkpoint/restart (src/checkpoint.jl:26-64): the full State and total_time, keyed as the
# reference keys them ("t", "total_time", one key per State field); a numpy .npz container (JLD2
# needs Julia).  Written to path + ".tmp" and renamed into place, so a crash mid-write leaves the
# previous checkpoint intact.
# ---------------------------------------------------------------------------------------------
def save_checkpoint(path: str, sim: Simulation, t: int) -> None:
    import os
    host = {("lambda" if k == "lambda_" else k): v for k, v in sim.state.to_numpy().items()}
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        np.savez(f, t=np.int64(t), total_time=np.float64(sim.total_time), **host)
    os.replace(tmp, path)


def load_checkpoint(sim: Simulation, path: str) -> int:
    """Restores sim.state and sim.total_time in place; returns the timestep saved."""
    import torch
    with np.load(path) as f:
        for name in _lib.STATE_FIELDS:
            key = "lambda" if name == "lambda_" else name
            dst = sim.state[name]
            a = np.asarray(f[key], dtype=np.float64)
            if a.shape != tuple(dst.shape):
                raise ValueError(f"checkpoint field {name} has shape {a.shape}, the state {tuple(dst.shape)}")
            dst.copy_(torch.from_numpy(np.ascontiguousarray(a)))
        t, total_time = int(f["t"]), float(f["total_time"])
    sim.total_time = total_time
    return t


def run(sim: Simulation, checkpoint_every: int | None = None, checkpoint_path: str | None = None,
        restart_path: str | None = None) -> None:
    """run!(sim; checkpoint_every, checkpoint_path, restart_path) (src/run.jl:21-63)."""
    if (checkpoint_every is None) != (checkpoint_path is None):
        raise ValueError("checkpoint_every and checkpoint_path must be given together")
    if restart_path is None:
        sim.total_time = 0.0
        sim.observer.prepare(sim.state)
        sim.observer.observe(sim.state, 0, sim.total_time)
        start_t = 0
    else:
        start_t = load_checkpoint(sim, restart_path)
        sim.observer.resume(sim.state, start_t)
    sim.step_stats = []
    for t in range(start_t + 1, sim.tsteps + 1):
        t0 = time.perf_counter()
        step(sim)
        sim.total_time += sim.dt
        sim.observer.observe(sim.state, t, sim.total_time)
        conv, last = picard_status(sim.hs)
        sim.step_stats.append(dict(converged=conv, last_iter=last,
                                   cg_iters=(sim.hs.ps.cg_iters_total if isinstance(sim.hs, EllipticHeadScheme)
                                             else sim.hs.ls.stats.niter)))
        if checkpoint_every is not None and t % checkpoint_every == 0:
            save_checkpoint(checkpoint_path, sim, t)
        if sim.verbose:
            import torch
            torch.cuda.synchronize()
            print(f"{t} / {sim.tsteps} completed in {time.perf_counter() - t0:.4f}s. "
                  f"Picard converged: {conv} in {last} iterations", flush=True)
    sim.observer.finalize(sim.state)


# ---------------------------------------------------------------------------------------------
# Host-fed runs: per-step inputs from and outputs to host memory, the transfers overlapped with the
# computation (no reference counterpart: the reference's run! keeps every field on its device and
# its observers copy to the host between steps).
# ---------------------------------------------------------------------------------------------
class HostIO:
    """Runs `sim` with per-step input from and output to host memory, overlapping the transfers
    with the computation.  The device staging buffers (the basal input twice, h and b twice each:
    about 6 fields) and the two copy streams are allocated here, once; `run` may be called any
    number of times."""

    def __init__(self, sim: Simulation):
        import torch
        self.sim = sim
        st = sim.state
        self.h2d, self.d2h = torch.cuda.Stream(), torch.cuda.Stream()
        self.stage = [torch.empty_like(st.ieb) for _ in range(2)]
        self.snap_h = [torch.empty_like(st.h) for _ in range(2)]
        self.snap_b = [torch.empty_like(st.b) for _ in range(2)]

    def run(self, ieb_host, h_host=None, b_host=None) -> None:
        """Advance the simulation by len(ieb_host) timesteps (step! as in `run`, without observers
        and with the basal input taken from the host instead of sim.mi): step k uses ieb from the
        pinned host tensor ieb_host[k] and returns its head and gap height into h_host / b_host
        (one pinned tensor each, overwritten every step, or a sequence with one tensor per step).
        Host tensors are shaped (ny, nx), row-major: the fields' memory order.

        Step k+1's input is copied host -> device on one copy stream while step k computes, and
        step k's h and b, snapshotted on the device right after the step, are copied device -> host
        on the other while step k+1 computes, so the host link's time hides behind the solve.
        Returns with every copy ordered before the current stream's next work
        (torch.cuda.synchronize() waits for them)."""
        import torch
        sim, st = self.sim, self.sim.state
        steps = len(ieb_host)
        if steps == 0:
            return
        comp, h2d, d2h = torch.cuda.current_stream(), self.h2d, self.d2h
        stage, snap_h, snap_b = self.stage, self.snap_h, self.snap_b
        want_out = h_host is not None or b_host is not None
        ev = torch.cuda.Event
        in_ready, in_free, snap_ready, out_done = [ev(), ev()], [ev(), ev()], [ev(), ev()], [ev(), ev()]
        start = ev()
        start.record(comp)
        h2d.wait_event(start)
        d2h.wait_event(start)

        def pick(x, k):
            return x if isinstance(x, torch.Tensor) else x[k]

        def issue_in(k):
            s = k % 2
            with torch.cuda.stream(h2d):
                if k >= 2:
                    h2d.wait_event(in_free[s])
                stage[s].t().copy_(ieb_host[k], non_blocking=True)
                in_ready[s].record(h2d)

        issue_in(0)
        if steps > 1:
            issue_in(1)
        for k in range(steps):
            s = k % 2
            comp.wait_event(in_ready[s])
            st.ieb.copy_(stage[s])
            in_free[s].record(comp)
            if k + 2 < steps:
                issue_in(k + 2)
            step_h(sim)
            step_b(sim)
            sim.total_time += sim.dt
            if want_out:
                if k >= 2:
                    comp.wait_event(out_done[s])
                snap_h[s].copy_(st.h)
                snap_b[s].copy_(st.b)
                snap_ready[s].record(comp)
                with torch.cuda.stream(d2h):
                    d2h.wait_event(snap_ready[s])
                    if h_host is not None:
                        pick(h_host, k).copy_(snap_h[s].t(), non_blocking=True)
                    if b_host is not None:
                        pick(b_host, k).copy_(snap_b[s].t(), non_blocking=True)
                    out_done[s].record(d2h)
        comp.wait_stream(h2d)
        comp.wait_stream(d2h)


# ---------------------------------------------------------------------------------------------
# set_initial_conditions! (src/initial_conditions.jl:14-125)
# ---------------------------------------------------------------------------------------------
def _copy_in(dst, arr):
    import torch
    a = np.asarray(arr, dtype=np.float64)
    if a.shape != tuple(dst.shape):
        raise ValueError(f"input shape {a.shape} does not match field shape {tuple(dst.shape)}")
    dst.copy_(torch.from_numpy(np.ascontiguousarray(a)))


def set_initial_conditions(s: State, g: Grid, p: ModelParameters, sl: AbstractSlidingLaw, mask, A_visc, zb, zs, b,
                           G, ub_x, ub_y, ieb, taub_x, taub_y, ctx: _Context | None = None) -> State:
    """Copy the raw inputs into the device State, then derive every field on the GPU in the
    reference's order.  The taub inputs are used only by PrescribedSlidingLaw (initialize_taub!)."""
    for name, arr in (("mask", mask), ("A_visc", A_visc), ("zb", zb), ("zs", zs), ("b", b), ("G", G),
                      ("ub_x", ub_x), ("ub_y", ub_y), ("ieb", ieb)):
        _copy_in(s[name], arr)
    if isinstance(sl, PrescribedSlidingLaw):
        _copy_in(s.taub_x, taub_x)
        _copy_in(s.taub_y, taub_y)
    own = ctx is None
    ctx = ctx or _Context(g)
    try:
        ctx.bind(s, p, sl)
        _lib.check(ctx.h, ctx.L.shk_set_initial_conditions(ctx.h))
    finally:
        if own:
            ctx.close()
    return s
