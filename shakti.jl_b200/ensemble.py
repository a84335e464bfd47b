"""Batched ensembles: many independent Simulations advanced together on one GPU.

The reference runs one Simulation per run! call (src/run.jl:21-63); a study with many independent
instances (parameter sweeps, uncertainty ensembles) loops over them.  `Ensemble(sims)` advances
them together: every kernel of a timestep is one launch over all instances, each timestep is one
CUDA graph launch whose Picard and CG loops run on the device, and the CG stencil kernel's tile
height is autotuned per grid size.  Each instance ends with the fields its own `run` would give
(Float64 CG preconditioned by Jacobi or by the Float32 multigrid V-cycle -- the mixed-precision
form, with every level kernel batched over the instances -- elliptic head scheme, constant melt
input, no head relaxation).
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .model import ConstantMeltInput
from .simulation import EllipticHeadScheme, Simulation


class Ensemble:
    def __init__(self, sims: list[Simulation], autotune_iters: int = 8):
        if not sims:
            raise ValueError("an ensemble needs at least one Simulation")
        dt = sims[0].dt
        for k, sim in enumerate(sims):
            if not isinstance(sim.hs, EllipticHeadScheme):
                raise ValueError(f"simulation {k}: the ensemble runs the elliptic head scheme")
            if not isinstance(sim.mi, ConstantMeltInput):
                raise ValueError(f"simulation {k}: the ensemble needs a ConstantMeltInput (ieb stays as set)")
            if sim.dt != dt:
                raise ValueError("every simulation of an ensemble uses the same dt")
            ls, ps = sim.ls, sim.hs.ps
            if ls.precond is not None or ls.precision != "fp64":
                raise ValueError(f"simulation {k}: the ensemble runs Float64 CG, Jacobi- or multigrid-preconditioned")
            if ps.hr.alpha > 0:
                raise ValueError(f"simulation {k}: the ensemble runs without head relaxation")
        self.sims = sims
        self.dt = dt
        self._po = sims[0].hs.ps.opts()
        self._o = sims[0].ls.opts()
        for k, sim in enumerate(sims[1:], 1):
            po, o = sim.hs.ps.opts(), sim.ls.opts()
            if (po.iters, po.tol, po.check_every) != (self._po.iters, self._po.tol, self._po.check_every):
                raise ValueError(f"simulation {k}: every PicardSolver of an ensemble has the same iters/tol")
            if (o.atol, o.rtol, o.stop_rule, o.itmax, o.precond) != (self._o.atol, self._o.rtol, self._o.stop_rule,
                                                                      self._o.itmax, self._o.precond):
                raise ValueError(f"simulation {k}: every CGIterativeSolver of an ensemble has the same tolerances")
        self._ctxs = [sim.ctx() for sim in sims]  # binds each instance's state, parameters and law
        self.L = self._ctxs[0].L
        arr = (C.c_void_p * len(sims))(*[c.h.value for c in self._ctxs])
        h = C.c_void_p()
        rc = self.L.shk_ensemble_create(len(sims), arr, _lib.cuda_stream_handle(), C.byref(h))
        if rc != _lib.OK:
            raise _lib.ShaktiError(rc, "shk_ensemble_create failed")
        self.h = h
        self.march_th = None
        if autotune_iters:
            self.autotune(autotune_iters)

    def _check(self, rc, allow=(_lib.OK,)):
        if rc not in allow:
            raise _lib.ShaktiError(rc, self.L.shk_ensemble_last_error(self.h).decode())
        return rc

    def autotune(self, iters: int = 8) -> list[int]:
        th = (C.c_int * len(self.sims))()
        self._check(self.L.shk_ensemble_autotune(self.h, int(iters), th))
        self.march_th = list(th)
        return self.march_th

    def run(self, tsteps: int) -> list[dict]:
        """tsteps timesteps of every instance; returns each instance's totals since creation."""
        st = (_lib.shk_ensemble_stats * len(self.sims))()
        self._check(self.L.shk_ensemble_run(self.h, self.dt, int(tsteps), C.byref(self._po), C.byref(self._o), st),
                    allow=(_lib.OK, _lib.NOT_CONVERGED))
        out = []
        for sim, s in zip(self.sims, st):
            sim.total_time += self.dt * tsteps
            ps = sim.hs.ps
            ps.converged = bool(s.last_converged)
            ps.last_iter = int(s.last_picard_iters)
            out.append(dict(steps=s.steps, steps_converged=s.steps_converged, picard_iters=s.picard_iters,
                            cg_iters=s.cg_iters, last_picard_iters=s.last_picard_iters,
                            last_converged=bool(s.last_converged), march_th=s.march_th))
        return out

    def set_snapshots(self, bufs):
        """Per-instance tensors (like each state's h, or None) that receive h after each timestep's
        first Picard iteration."""
        arr = (C.c_void_p * len(self.sims))(*[(b.data_ptr() if b is not None else None) for b in bufs])
        self._bufs_snap = list(bufs)
        self._check(self.L.shk_ensemble_set_snapshots(self.h, arr))

    def launch_blocks(self) -> dict:
        v = [C.c_int() for _ in range(4)]
        self._check(self.L.shk_ensemble_launch_counts(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("stencil", "march", "stream", "flat"), (x.value for x in v)))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.shk_ensemble_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
