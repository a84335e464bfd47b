"""Linear solvers and the Picard solver mirroring Shakti.jl's API (src/linear_solver.jl,
src/preconditioner.jl, src/elliptic_solver.jl), backed by libshakti_b200.

Only the GPU-capable representation exists here, as in the reference under a GPU backend:
CGIterativeSolver(g, MatrixFreeLinearSystem) with Jacobi or Chebyshev.  The CPU-only pieces raise
the reference's construction-time errors (src/linear_solver.jl:209, 804, 834).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

from . import _lib
from .model import Grid, ModelParameters, State, AbstractKFaceScheme, AbstractSlidingLaw, Arithmetic

SQRT_EPS = math.sqrt(2.220446049250313e-16)


class _Context:
    """One libshakti_b200 context: grid + solver workspace (MFLS, Krylov vectors, reductions)."""

    def __init__(self, grid: Grid):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA is not available: the B200 library needs a GPU")
        self.L = _lib.load()
        self.grid = grid
        h = C.c_void_p()
        rc = self.L.shk_create(grid.nx, grid.ny, float(grid.lx), float(grid.ly), _lib.cuda_stream_handle(),
                               C.byref(h))
        if rc != _lib.OK:
            raise _lib.ShaktiError(rc, "shk_create failed")
        self.h = h
        self._bound = None

    def bind(self, state: State, p: ModelParameters, sl: AbstractSlidingLaw | None,
             kfs: AbstractKFaceScheme | None = None, gap: int = 1):
        L, h = self.L, self.h
        if (state.grid.nx, state.grid.ny) != (self.grid.nx, self.grid.ny):
            raise ValueError("state grid does not match the solver's grid")
        _lib.check(h, L.shk_set_stream(h, _lib.cuda_stream_handle()))
        ps = p.struct()
        _lib.check(h, L.shk_set_params(h, C.byref(ps)))
        sls = (sl or _DummyLaw()).struct()
        _lib.check(h, L.shk_set_sliding_law(h, C.byref(sls)))
        _lib.check(h, L.shk_set_schemes(h, (kfs or Arithmetic()).code, int(gap)))
        st = state.struct()
        _lib.check(h, L.shk_bind_state(h, C.byref(st)))
        self._bound = (state, sl)  # keep referenced device buffers alive
        return self

    def launches(self) -> int:
        return int(self.L.shk_kernel_launches(self.h))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.shk_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _DummyLaw(AbstractSlidingLaw):
    kind = 0


class AbstractLinearSolver:
    pass


class AbstractDirectSolver(AbstractLinearSolver):
    pass


class AbstractIterativeSolver(AbstractLinearSolver):
    pass


class AbstractLinearSystem:
    pass


class SparseAssembledLinearSystem(AbstractLinearSystem):
    """CPU-only in the reference (src/linear_solver.jl:72-80); not provided on the GPU."""


class MatrixFreeLinearSystem(AbstractLinearSystem):
    """Per-cell stencil coefficients aP/aE/aW/aN/aS + rhs (src/linear_solver.jl:91-121), living in
    the solver context.  `export()` returns the five coefficient arrays and rhs as CUDA tensors."""

    def __init__(self, grid: Grid, ctx: _Context | None = None):
        self.grid = grid
        self._ctx = ctx

    def export(self) -> dict:
        import torch
        g = self.grid
        out = {k: torch.zeros((g.ny, g.nx), dtype=torch.float64, device="cuda").t() for k in
               ("aP", "aE", "aW", "aN", "aS", "rhs")}
        L, h = self._ctx.L, self._ctx.h
        _lib.check(h, L.shk_export_mfls(h, *[out[k].data_ptr() for k in ("aP", "aE", "aW", "aN", "aS", "rhs")]))
        return out

    def matvec(self, x, y=None):
        """mul!(y, StencilOperator(mfls), x) (src/linear_solver.jl:664-669)."""
        import torch
        if y is None:
            y = torch.empty_like(x)
        L, h = self._ctx.L, self._ctx.h
        _lib.check(h, L.shk_matvec(h, x.data_ptr(), y.data_ptr()))
        return y


class CholeskyDirectSolver(AbstractDirectSolver):
    def __init__(self, g: Grid):
        raise RuntimeError("CholeskyDirectSolver is CPU-only (SparseArrays/CHOLMOD has no GPU path); choose an "
                           "iterative solver under the CUDA backend.")


@dataclass
class CgStats:
    niter: int = 0
    status: int = 0
    refinements: int = 0
    rnorm0: float = 0.0
    rnorm: float = 0.0
    lambda_min: float = 1.0
    lambda_max: float = 1.0
    bounds_valid: bool = False

    @property
    def solved(self) -> bool:
        return self.status == _lib.OK


class ChebyshevPreconditioner:
    """Degree-`degree` Chebyshev semi-iteration on D^-1 A with Lanczos-estimated bounds
    (src/preconditioner.jl:160-267).  Bounds live on the device and persist across solves,
    starting at the (1, 1) placeholder."""

    def __init__(self, solver: "CGIterativeSolver", degree: int, nsteps_estimate: int = 15):
        if degree < 1:
            raise ValueError(f"ChebyshevPreconditioner: degree must be >= 1 (got {degree})")
        if nsteps_estimate < 2:
            raise ValueError(f"ChebyshevPreconditioner: nsteps_estimate must be >= 2 (got {nsteps_estimate})")
        if degree > 32 or nsteps_estimate > 64:
            raise ValueError("ChebyshevPreconditioner: degree <= 32 and nsteps_estimate <= 64 on this backend")
        self._solver = solver
        self.degree = int(degree)
        self.nsteps_estimate = int(nsteps_estimate)

    @property
    def lambda_min(self) -> float:
        return self.bounds()[0]

    @property
    def lambda_max(self) -> float:
        return self.bounds()[1]

    def bounds(self) -> tuple[float, float]:
        ctx = self._solver.ctx
        a, b = C.c_double(), C.c_double()
        _lib.check(ctx.h, ctx.L.shk_get_chebyshev_bounds(ctx.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_bounds(self, lmin: float, lmax: float) -> None:
        ctx = self._solver.ctx
        _lib.check(ctx.h, ctx.L.shk_set_chebyshev_bounds(ctx.h, float(lmin), float(lmax)))

    def update_bounds(self, rhs=None) -> tuple[bool, tuple[float, float]]:
        """update_chebyshev_bounds!(P, rhs) on the solver's assembled operator (src/preconditioner.jl:197-233).
        Returns (adopted, raw_estimate)."""
        ctx = self._solver.ctx
        est = (C.c_double * 2)()
        ok = C.c_int()
        _lib.check(ctx.h, ctx.L.shk_update_chebyshev_bounds(ctx.h, self.nsteps_estimate,
                                                            None if rhs is None else rhs.data_ptr(),
                                                            est, C.byref(ok)))
        return bool(ok.value), (est[0], est[1])

    def ldiv(self, x, y=None):
        """ldiv!(y, P, x) (src/preconditioner.jl:239-267)."""
        import torch
        if y is None:
            y = torch.empty_like(x)
        ctx = self._solver.ctx
        _lib.check(ctx.h, ctx.L.shk_chebyshev_apply(ctx.h, self.degree, x.data_ptr(), y.data_ptr()))
        return y


class CGIterativeSolver(AbstractIterativeSolver):
    """CGIterativeSolver(g, MatrixFreeLinearSystem; chebyshev_degree, chebyshev_nsteps_estimate)
    (src/linear_solver.jl:760-843), with Krylov.jl's cg! keywords exposed:
      atol, rtol, itmax -- Krylov defaults sqrt(eps), sqrt(eps), 2n; stop_rule "krylov" is Krylov's
      preconditioned-norm test, "relres" the unpreconditioned ||b - A x|| <= rtol ||b_G|| (residual
      over every row, b over the GROUNDED rows: the fixed-head rows would otherwise dominate ||b||).
      precision "fp64" (plain) or "mixed" (Float32 stencil + CG inside Float64 iterative refinement;
      relres rule; inner_rtol is the inner Float32 solve's relative tolerance)."""

    def __init__(self, g: Grid, lsy=MatrixFreeLinearSystem, *, chebyshev_degree: int | None = None,
                 chebyshev_nsteps_estimate: int = 15, amg: bool = False, precision: str = "fp64",
                 stop_rule: str = "krylov", atol: float | None = None, rtol: float | None = None, itmax: int = 0,
                 inner_rtol: float = 1e-2, max_refine: int = 0, inner_itmax: int = 0, multigrid: bool = False):
        if lsy is SparseAssembledLinearSystem:
            raise RuntimeError("CGIterativeSolver(g, SparseAssembledLinearSystem) is CPU-only; use "
                               "CGIterativeSolver(g, MatrixFreeLinearSystem) under the CUDA backend.")
        if lsy is not MatrixFreeLinearSystem:
            raise TypeError("lsy must be MatrixFreeLinearSystem")
        if amg:
            raise RuntimeError("AMGPreconditioner is CPU/SparseMatrixCSC-only (AlgebraicMultigrid.jl has no GPU array "
                               "support); use CGIterativeSolver(g, SparseAssembledLinearSystem; amg = true) instead, or "
                               "chebyshev_degree here for a GPU-capable accelerated preconditioner.")
        if multigrid and chebyshev_degree is not None:
            raise ValueError("chebyshev_degree and multigrid are mutually exclusive preconditioner choices; pick one.")
        if multigrid and precision != "fp64":
            raise ValueError("the multigrid preconditioner runs inside the Float64 CG (precision='fp64')")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if stop_rule not in ("krylov", "relres"):
            raise ValueError("stop_rule must be 'krylov' or 'relres'")
        if precision == "mixed" and stop_rule != "relres":
            raise ValueError("the mixed-precision form uses stop_rule='relres'")
        self.grid = g
        self.ctx = _Context(g)
        self.lsy = MatrixFreeLinearSystem(g, self.ctx)
        self.precond = None if chebyshev_degree is None else ChebyshevPreconditioner(
            self, chebyshev_degree, chebyshev_nsteps_estimate)
        self.precision = precision
        self.stop_rule = stop_rule
        self.atol = SQRT_EPS if atol is None else float(atol)
        self.rtol = SQRT_EPS if rtol is None else float(rtol)
        self.itmax = int(itmax)
        self.inner_rtol = float(inner_rtol)
        self.max_refine = int(max_refine)
        self.inner_itmax = int(inner_itmax)
        self.multigrid = bool(multigrid)
        self.stats = CgStats()

    def opts(self) -> _lib.shk_cg_opts:
        cheb = self.precond is not None
        return _lib.default_cg_opts(
            precond=2 if self.multigrid else (1 if cheb else 0), cheb_degree=self.precond.degree if cheb else 4,
            cheb_nsteps=self.precond.nsteps_estimate if cheb else 15,
            stop_rule=0 if self.stop_rule == "krylov" else 1, precision=0 if self.precision == "fp64" else 1,
            max_refine=self.max_refine, atol=self.atol, rtol=self.rtol, inner_rtol=self.inner_rtol,
            itmax=self.itmax, inner_itmax=self.inner_itmax)

    def _record(self, s: _lib.shk_cg_stats):
        self.stats = CgStats(niter=s.niter, status=s.status, refinements=s.refinements, rnorm0=s.rnorm0,
                             rnorm=s.rnorm, lambda_min=s.lambda_min, lambda_max=s.lambda_max,
                             bounds_valid=bool(s.bounds_valid))

    def close(self):
        self.ctx.close()


def solve_elliptic_linear_system(ls: CGIterativeSolver, s: State, g: Grid, p: ModelParameters,
                                 kfs: AbstractKFaceScheme, sl: AbstractSlidingLaw | None = None) -> CgStats:
    """src/linear_solver.jl:915-925: update_MFLS!, preconditioner refresh, cg! warm-started from h."""
    ctx = ls.ctx.bind(s, p, sl, kfs)
    st = _lib.shk_cg_stats()
    o = ls.opts()
    rc = ctx.L.shk_solve_elliptic(ctx.h, C.byref(o), C.byref(st))
    _lib.check(ctx.h, rc, allow=(_lib.OK, _lib.NOT_CONVERGED, _lib.BREAKDOWN))
    ls._record(st)
    return ls.stats


def solve_parabolic_linear_system(ls: CGIterativeSolver, s: State, g: Grid, p: ModelParameters,
                                  kfs: AbstractKFaceScheme, dt: float,
                                  sl: AbstractSlidingLaw | None = None) -> CgStats:
    """src/linear_solver.jl:935-945"""
    ctx = ls.ctx.bind(s, p, sl, kfs)
    st = _lib.shk_cg_stats()
    o = ls.opts()
    rc = ctx.L.shk_solve_parabolic(ctx.h, float(dt), C.byref(o), C.byref(st))
    _lib.check(ctx.h, rc, allow=(_lib.OK, _lib.NOT_CONVERGED, _lib.BREAKDOWN))
    ls._record(st)
    return ls.stats


# ---------------------------------------------------------------------------------------------
# Picard (src/elliptic_solver.jl)
# ---------------------------------------------------------------------------------------------
class NoHeadRelaxation:
    alpha = float("nan")


class UnderHeadRelaxation:
    def __init__(self, alpha: float):
        self.alpha = float(alpha)


class PicardSolver:
    """PicardSolver(iters, tol, ls, g; alpha, check_every) (src/elliptic_solver.jl:59-105).
    h_prev lives in the solver context; delta_h is never materialised (its max-norm is reduced on
    the fly)."""

    def __init__(self, iters: int, tol: float, ls: AbstractLinearSolver, g: Grid, alpha: float | None = None,
                 check_every: int = 1):
        if not isinstance(ls, CGIterativeSolver):
            raise TypeError("ls must be a CGIterativeSolver on this backend")
        self.iters = int(iters)
        self.tol = float(tol)
        self.ls = ls
        self.hr = NoHeadRelaxation() if alpha is None else UnderHeadRelaxation(alpha)
        self.check_every = int(check_every)
        self.converged = False
        self.last_iter = 0
        self.cg_iters_total = 0
        self.cg_solves = 0
        self.cg_breakdowns = 0
        self.max_dh = math.nan
        self.max_h = math.nan

    def opts(self) -> _lib.shk_picard_opts:
        return _lib.shk_picard_opts(iters=self.iters, check_every=self.check_every, tol=self.tol,
                                    alpha=self.hr.alpha)

    def _record(self, s: _lib.shk_picard_stats):
        self.converged = bool(s.converged)
        self.last_iter = int(s.last_iter)
        self.cg_iters_total = int(s.cg_iters_total)
        self.cg_solves = int(s.cg_solves)
        self.cg_breakdowns = int(s.cg_breakdowns)
        self.max_dh = s.max_dh
        self.max_h = s.max_h


def Picard_loop(ps: PicardSolver, state: State, grid: Grid, p: ModelParameters, shs, kfs: AbstractKFaceScheme,
                sl: AbstractSlidingLaw) -> None:
    """src/elliptic_solver.jl:138-176 (shs is derived from p, src/simulation.jl:132)."""
    ctx = ps.ls.ctx.bind(state, p, sl, kfs)
    st = _lib.shk_picard_stats()
    po, o = ps.opts(), ps.ls.opts()
    rc = ctx.L.shk_picard_solve(ctx.h, C.byref(po), C.byref(o), C.byref(st))
    _lib.check(ctx.h, rc, allow=(_lib.OK, _lib.NOT_CONVERGED))
    ps._record(st)


elliptic_solver = Picard_loop


def parabolic_solver(ls: CGIterativeSolver, state: State, grid: Grid, p: ModelParameters, shs,
                     kfs: AbstractKFaceScheme, sl: AbstractSlidingLaw, dt: float) -> CgStats:
    """src/parabolic_solver.jl:16-38"""
    ctx = ls.ctx.bind(state, p, sl, kfs)
    st = _lib.shk_cg_stats()
    o = ls.opts()
    rc = ctx.L.shk_parabolic_step(ctx.h, float(dt), C.byref(o), C.byref(st))
    _lib.check(ctx.h, rc, allow=(_lib.OK, _lib.NOT_CONVERGED, _lib.BREAKDOWN))
    ls._record(st)
    return ls.stats


def picard_tail(ls: CGIterativeSolver, state: State, p: ModelParameters, sl: AbstractSlidingLaw) -> None:
    """The compute_* chain of Picard_iteration! (src/elliptic_solver.jl:193-206), fused."""
    ctx = ls.ctx.bind(state, p, sl)
    _lib.check(ctx.h, ctx.L.shk_picard_tail(ctx.h))
