"""ctypes binding of the CPU restatement in oracle/shakti_oracle.c.

TEST INFRASTRUCTURE ONLY: the test oracle of the CUDA library and the reported CPU baseline.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module; the product
path never does.

Parity pinning: the reference (Julia) cannot run here and holds no stored golden vectors; this
restatement is pinned against the fixtures and known-answer properties of the reference's own test
suite (tests/test_oracle_reference_suite.py) and against a SciPy sparse direct solve standing in
for CHOLMOD.  Arrays are numpy Float64 in Fortran order, shape (nx, ny) / (nx+1, ny) / (nx, ny+1),
the reference's State layout (src/state.jl:13-57).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import shutil
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_shakti.so"

CENTER = ["h", "pw", "po", "b", "beta", "abs_ub", "mdot", "shear", "potential", "sensible", "Re", "K", "G",
          "zb", "zs", "H", "ieb", "lambda_", "A_visc", "N", "mask"]
XFACE = ["dhdx", "q_x", "Re_x", "b_x", "ub_x", "taub_x", "dpwdx", "valid_x"]
YFACE = ["dhdy", "q_y", "Re_y", "b_y", "ub_y", "taub_y", "dpwdy", "valid_y"]
ALL_FIELDS = CENTER + XFACE + YFACE
PARAM_NAMES = ["rho_w", "rho_sw", "rho_i", "g", "nu", "n", "omega", "L", "br", "lr", "ct", "cw", "p_atm",
               "b_min", "b_max", "e_v"]
# ModelParameters keyword defaults (src/model_parameters.jl:55-72)
DEFAULT_PARAMS = dict(rho_w=1000.0, rho_sw=1027.0, rho_i=910.0, g=9.81, nu=1.787e-6, n=3.0, omega=1e-4,
                      L=334e3, br=0.05, lr=2.0, ct=7.5e-8, cw=4.22e3, p_atm=0.0, b_min=0.0, b_max=math.inf,
                      e_v=0.0)
DP = C.POINTER(C.c_double)


class _Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in PARAM_NAMES]


class _Sliding(C.Structure):
    _fields_ = [("kind", C.c_int), ("C", C.c_double), ("v0", C.c_double), ("Cx", DP), ("Cy", DP)]


class _State(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double)] + [
        (f, DP) for f in ALL_FIELDS]


class _CgOpts(C.Structure):
    _fields_ = [("precond", C.c_int), ("cheb_degree", C.c_int), ("cheb_nsteps", C.c_int), ("stop_rule", C.c_int),
                ("atol", C.c_double), ("rtol", C.c_double), ("itmax", C.c_long)]


class _CgStats(C.Structure):
    _fields_ = [("niter", C.c_long), ("status", C.c_int), ("rnorm0", C.c_double), ("rnorm", C.c_double)]


class _ChebState(C.Structure):
    _fields_ = [("lambda_min", C.c_double), ("lambda_max", C.c_double), ("last_estimate_valid", C.c_int)]


class _PicardOpts(C.Structure):
    _fields_ = [("iters", C.c_int), ("check_every", C.c_int), ("tol", C.c_double), ("alpha", C.c_double)]


class _PicardStats(C.Structure):
    _fields_ = [("converged", C.c_int), ("last_iter", C.c_int), ("cg_iters_total", C.c_long),
                ("cg_solves", C.c_int), ("cg_breakdowns", C.c_int)]


class _Melt(C.Structure):
    _fields_ = [("kind", C.c_int)] + [(n, C.c_double) for n in
                                      ("t_start", "period", "omega", "amplitude", "offset", "i_min",
                                       "seconds_per_year")] + [("base", DP)]


class _Progress(C.Structure):
    _fields_ = [("steps_done", C.c_int), ("picard_iters", C.c_long), ("cg_iters", C.c_long),
                ("cg_breakdowns", C.c_int), ("pic_iter_now", C.c_int), ("cg_iter_now", C.c_long),
                ("elapsed", C.c_double), ("completed_s", C.c_double), ("step_s_now", C.c_double),
                ("last_step_s", C.c_double), ("last_picard", C.c_int), ("last_cg", C.c_long),
                ("last_converged", C.c_int), ("all_converged", C.c_int), ("total_time", C.c_double)]


class _Sim(C.Structure):
    _fields_ = [("head_scheme", C.c_int), ("gap_scheme", C.c_int), ("kfs", C.c_int), ("dt", C.c_double)]


def build(force: bool = False) -> Path:
    """Compile the restatement with its Makefile (gcc, OpenMP, -ffp-contract=off)."""
    src = HERE / "shakti_oracle.c"
    if not force and LIB_PATH.exists() and LIB_PATH.stat().st_mtime >= max(
            src.stat().st_mtime, (HERE / "shakti_oracle.h").stat().st_mtime):
        return LIB_PATH
    make = shutil.which("make")
    if make is None:
        raise RuntimeError("make not found; cannot build the oracle")
    subprocess.run([make, "-s", "-C", str(HERE), "-B" if force else "all"], check=True)
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        S = C.POINTER(_State)
        L.orc_set_initial_conditions.argtypes = [S, C.POINTER(_Params), C.POINTER(_Sliding)]
        L.orc_assemble_mfls.argtypes = [S, C.POINTER(_Params), C.c_int, C.c_int, C.c_double] + [DP] * 6
        L.orc_assemble_sals.argtypes = [S, C.POINTER(_Params), C.c_int, C.c_int, C.c_double] + [DP] * 6
        L.orc_matvec.argtypes = [C.c_int, C.c_int] + [DP] * 7
        L.orc_update_chebyshev_bounds.argtypes = [C.c_int, C.c_int] + [DP] * 6 + [C.c_int, C.POINTER(_ChebState), DP]
        L.orc_update_chebyshev_bounds.restype = C.c_int
        L.orc_chebyshev_apply.argtypes = [C.c_int, C.c_int] + [DP] * 5 + [C.c_int, C.POINTER(_ChebState), DP, DP]
        L.orc_cg.argtypes = [C.c_int, C.c_int] + [DP] * 7 + [C.POINTER(_CgOpts), C.POINTER(_ChebState),
                                                              C.POINTER(_CgStats)]
        L.orc_cg.restype = C.c_int
        L.orc_cg_masked.argtypes = [C.c_int, C.c_int] + [DP] * 8 + [C.POINTER(_CgOpts), C.POINTER(_ChebState),
                                                                     C.POINTER(_CgStats)]
        L.orc_cg_masked.restype = C.c_int
        L.orc_picard_tail.argtypes = [S, C.POINTER(_Params), C.POINTER(_Sliding)]
        L.orc_picard_iteration.argtypes = [S, C.POINTER(_Params), C.POINTER(_Sliding), C.c_int, C.POINTER(_CgOpts),
                                           C.POINTER(_ChebState), C.c_double, DP, C.POINTER(_CgStats)]
        L.orc_picard_loop.argtypes = [S, C.POINTER(_Params), C.POINTER(_Sliding), C.c_int, C.POINTER(_CgOpts),
                                      C.POINTER(_ChebState), C.POINTER(_PicardOpts), C.POINTER(_PicardStats)]
        L.orc_picard_loop.restype = C.c_int
        L.orc_parabolic_step.argtypes = [S, C.POINTER(_Params), C.POINTER(_Sliding), C.c_int, C.POINTER(_CgOpts),
                                         C.POINTER(_ChebState), C.c_double, C.POINTER(_CgStats)]
        L.orc_step_b.argtypes = [S, C.POINTER(_Params), C.c_int, C.c_double]
        L.orc_update_ieb.argtypes = [S, C.POINTER(_Melt), C.c_double]
        L.orc_run.argtypes = [S, C.POINTER(_Params), C.POINTER(_Sliding), C.POINTER(_Melt), C.POINTER(_Sim),
                              C.POINTER(_CgOpts), C.POINTER(_ChebState), C.POINTER(_PicardOpts), C.c_int,
                              DP, C.POINTER(_PicardStats)]
        L.orc_run.restype = C.c_int
        L.orc_session_create.argtypes = [S, C.POINTER(_Params), C.POINTER(_Sliding), C.POINTER(_Melt),
                                         C.POINTER(_Sim), C.POINTER(_CgOpts), C.POINTER(_ChebState),
                                         C.POINTER(_PicardOpts), C.c_double]
        L.orc_session_create.restype = C.c_void_p
        L.orc_session_advance.argtypes = [C.c_void_p, C.c_double, C.c_int, C.POINTER(_Progress)]
        L.orc_session_advance.restype = C.c_int
        L.orc_session_destroy.argtypes = [C.c_void_p]
        for name in ("orc_compute_face_masks", "orc_apply_mask_to_sliding", "orc_compute_H", "orc_compute_abs_ub",
                     "orc_compute_N", "orc_compute_dhdxy", "orc_compute_dpwdxy", "orc_compute_Re",
                     "orc_compute_b_xy"):
            getattr(L, name).argtypes = [S]
        for name in ("orc_compute_po", "orc_compute_h", "orc_compute_pw", "orc_compute_q_xy_lagged",
                     "orc_compute_Re_xy_lagged", "orc_compute_q_and_Re_xy", "orc_compute_mdot", "orc_compute_K",
                     "orc_compute_beta"):
            getattr(L, name).argtypes = [S, C.POINTER(_Params)]
        L.orc_compute_taub_xy.argtypes = [S, C.POINTER(_Params), C.POINTER(_Sliding)]
        L.orc_num_threads.restype = C.c_int
        L.orc_set_num_threads.argtypes = [C.c_int]
        _LIB = L
    return _LIB


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1)
    return a.ctypes.data_as(DP)


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return lib().orc_num_threads()


@dataclass
class SlidingSpec:
    """kind: 0 RegularizedCoulomb, 1 Field, 2 V0, 3 Linear, 4 Prescribed (face arrays pre-staggered)."""
    kind: int = 0
    C: float = 0.0
    v0: float = 0.0
    Cx: np.ndarray | None = None
    Cy: np.ndarray | None = None


@dataclass
class CgSpec:
    precond: int = 0          # 0 Jacobi, 1 Chebyshev
    cheb_degree: int = 4
    cheb_nsteps: int = 15
    stop_rule: int = 0        # 0 Krylov default, 1 relative residual
    atol: float = math.sqrt(np.finfo(np.float64).eps)
    rtol: float = math.sqrt(np.finfo(np.float64).eps)
    itmax: int = 0


def _cg(spec: CgSpec) -> _CgOpts:
    return _CgOpts(spec.precond, spec.cheb_degree, spec.cheb_nsteps, spec.stop_rule, spec.atol, spec.rtol,
                   spec.itmax)


@dataclass
class OracleState:
    """All State fields as Fortran-ordered numpy arrays plus grid spacing."""
    nx: int
    ny: int
    lx: float
    ly: float
    fields: dict = field(default_factory=dict)
    cheb: _ChebState = field(default_factory=lambda: _ChebState(1.0, 1.0, 0))

    def __post_init__(self):
        self.dx = self.lx / (self.nx - 1)
        self.dy = self.ly / (self.ny - 1)
        for f in CENTER:
            self.fields[f] = np.zeros((self.nx, self.ny), order="F")
        for f in XFACE:
            self.fields[f] = np.zeros((self.nx + 1, self.ny), order="F")
        for f in YFACE:
            self.fields[f] = np.zeros((self.nx, self.ny + 1), order="F")
        self.fields["valid_x"][:] = 1.0
        self.fields["valid_y"][:] = 1.0
        self._keep = []

    def __getitem__(self, k):
        return self.fields["lambda_" if k == "lambda" else k]

    def struct(self) -> _State:
        s = _State(self.nx, self.ny, self.dx, self.dy)
        for f in ALL_FIELDS:
            arr = self.fields[f]
            assert arr.flags.f_contiguous and arr.dtype == np.float64
            setattr(s, f, _ptr(arr))
        return s

    def copy(self) -> "OracleState":
        o = OracleState(self.nx, self.ny, self.lx, self.ly)
        for f in ALL_FIELDS:
            o.fields[f][...] = self.fields[f]
        o.cheb = _ChebState(self.cheb.lambda_min, self.cheb.lambda_max, self.cheb.last_estimate_valid)
        return o


def params_struct(p: dict | None) -> _Params:
    d = dict(DEFAULT_PARAMS)
    if p:
        d.update(p)
    return _Params(*[float(d[n]) for n in PARAM_NAMES])


def sliding_struct(sl: SlidingSpec, keep: list) -> _Sliding:
    s = _Sliding(sl.kind, sl.C, sl.v0, None, None)
    if sl.Cx is not None:
        cx = np.asfortranarray(sl.Cx, dtype=np.float64)
        cy = np.asfortranarray(sl.Cy, dtype=np.float64)
        keep += [cx, cy]
        s.Cx, s.Cy = _ptr(cx), _ptr(cy)
    return s


def set_initial_conditions(st: OracleState, p: dict | None, sl: SlidingSpec, inputs: dict) -> None:
    """set_initial_conditions! (src/initial_conditions.jl:14-125): copy the raw inputs, then derive."""
    for k in ("mask", "A_visc", "zb", "zs", "b", "G", "ub_x", "ub_y", "ieb"):
        st.fields[k][...] = np.asarray(inputs[k], dtype=np.float64)
    if sl.kind == 4:  # PrescribedSlidingLaw: initialize_taub! copies taub (src/sliding_law.jl:103-107)
        st.fields["taub_x"][...] = inputs["taub_x"]
        st.fields["taub_y"][...] = inputs["taub_y"]
    keep = []
    s = st.struct()
    lib().orc_set_initial_conditions(C.byref(s), C.byref(params_struct(p)), C.byref(sliding_struct(sl, keep)))


def assemble(st: OracleState, p: dict | None, kfs: int = 0, parabolic: bool = False, dt: float = 0.0,
             sals: bool = False) -> dict:
    n = (st.nx, st.ny)
    out = {k: np.zeros(n, order="F") for k in ("aP", "aE", "aW", "aN", "aS", "rhs")}
    fn = lib().orc_assemble_sals if sals else lib().orc_assemble_mfls
    s = st.struct()
    fn(C.byref(s), C.byref(params_struct(p)), int(kfs), int(parabolic), float(dt),
       *[_ptr(out[k]) for k in ("aP", "aE", "aW", "aN", "aS", "rhs")])
    return out


def matvec(A: dict, x: np.ndarray) -> np.ndarray:
    nx, ny = A["aP"].shape
    x = np.asfortranarray(x, dtype=np.float64)
    y = np.zeros((nx, ny), order="F")
    lib().orc_matvec(nx, ny, *[_ptr(A[k]) for k in ("aP", "aE", "aW", "aN", "aS")], _ptr(x), _ptr(y))
    return y


def update_chebyshev_bounds(A: dict, rhs: np.ndarray, nsteps: int, cheb: _ChebState):
    nx, ny = A["aP"].shape
    est = np.zeros(2)
    rhs = np.asfortranarray(rhs, dtype=np.float64)
    ok = lib().orc_update_chebyshev_bounds(nx, ny, *[_ptr(A[k]) for k in ("aP", "aE", "aW", "aN", "aS")],
                                           _ptr(rhs), int(nsteps), C.byref(cheb), est.ctypes.data_as(DP))
    return bool(ok), (float(est[0]), float(est[1]))


def chebyshev_apply(A: dict, degree: int, cheb: _ChebState, x: np.ndarray) -> np.ndarray:
    nx, ny = A["aP"].shape
    x = np.asfortranarray(x, dtype=np.float64)
    y = np.zeros((nx, ny), order="F")
    lib().orc_chebyshev_apply(nx, ny, *[_ptr(A[k]) for k in ("aP", "aE", "aW", "aN", "aS")], int(degree),
                              C.byref(cheb), _ptr(x), _ptr(y))
    return y


def cg(A: dict, x0: np.ndarray, spec: CgSpec, cheb: _ChebState | None = None, mask: np.ndarray | None = None):
    """Krylov.jl cg! with warm start x0 on the assembled system; returns (x, stats dict).  With
    `mask` (State.mask), the relative-residual rule divides by the GROUNDED rows' ||rhs|| only."""
    nx, ny = A["aP"].shape
    x = np.array(x0, dtype=np.float64, order="F", copy=True)
    cheb = cheb if cheb is not None else _ChebState(1.0, 1.0, 0)
    st = _CgStats()
    ptrs = [_ptr(A[k]) for k in ("aP", "aE", "aW", "aN", "aS", "rhs")]
    if mask is None:
        lib().orc_cg(nx, ny, *ptrs, _ptr(x), C.byref(_cg(spec)), C.byref(cheb), C.byref(st))
    else:
        m = np.asfortranarray(mask, dtype=np.float64)
        lib().orc_cg_masked(nx, ny, *ptrs, _ptr(m), _ptr(x), C.byref(_cg(spec)), C.byref(cheb), C.byref(st))
    return x, dict(niter=st.niter, status=st.status, rnorm0=st.rnorm0, rnorm=st.rnorm)


def picard_tail(st: OracleState, p: dict | None, sl: SlidingSpec) -> None:
    keep = []
    s = st.struct()
    lib().orc_picard_tail(C.byref(s), C.byref(params_struct(p)), C.byref(sliding_struct(sl, keep)))


def compute(st: OracleState, name: str, p: dict | None = None, sl: SlidingSpec | None = None) -> None:
    """Run one reference kernel by name, e.g. compute(st, 'q_xy_lagged', p)."""
    L = lib()
    s = st.struct()
    fn = getattr(L, "orc_compute_" + name)
    if name == "taub_xy":
        keep = []
        fn(C.byref(s), C.byref(params_struct(p)), C.byref(sliding_struct(sl, keep)))
    elif fn.argtypes and len(fn.argtypes) == 2:
        fn(C.byref(s), C.byref(params_struct(p)))
    else:
        fn(C.byref(s))


def picard_loop(st: OracleState, p: dict | None, sl: SlidingSpec, kfs: int, cgspec: CgSpec, iters: int = 500,
                tol: float = 1e-6, alpha: float = float("nan"), check_every: int = 1) -> dict:
    keep = []
    s = st.struct()
    ps = _PicardStats()
    rc = lib().orc_picard_loop(C.byref(s), C.byref(params_struct(p)), C.byref(sliding_struct(sl, keep)), int(kfs),
                               C.byref(_cg(cgspec)), C.byref(st.cheb),
                               C.byref(_PicardOpts(iters, check_every, tol, alpha)), C.byref(ps))
    return dict(rc=rc, converged=bool(ps.converged), last_iter=ps.last_iter, cg_iters_total=ps.cg_iters_total,
                cg_solves=ps.cg_solves, cg_breakdowns=ps.cg_breakdowns)


def parabolic_step(st: OracleState, p: dict | None, sl: SlidingSpec, kfs: int, cgspec: CgSpec, dt: float) -> dict:
    keep = []
    s = st.struct()
    cs = _CgStats()
    lib().orc_parabolic_step(C.byref(s), C.byref(params_struct(p)), C.byref(sliding_struct(sl, keep)), int(kfs),
                             C.byref(_cg(cgspec)), C.byref(st.cheb), float(dt), C.byref(cs))
    return dict(niter=cs.niter, status=cs.status)


def step_b(st: OracleState, p: dict | None, gap_scheme: int, dt: float) -> None:
    s = st.struct()
    lib().orc_step_b(C.byref(s), C.byref(params_struct(p)), int(gap_scheme), float(dt))


def melt_struct(mi: dict | None, keep: list | None = None) -> _Melt:
    """kind 0 constant, 1 seasonal (uniform), 2 seasonal plus mi['base'] (an (nx, ny) field)."""
    if not mi or mi.get("kind", 0) == 0:
        return _Melt(0, 0, 0, 0, 0, 0, 0, 1, None)
    base = None
    if mi.get("base") is not None:
        b = np.asfortranarray(mi["base"], dtype=np.float64)
        if keep is not None:
            keep.append(b)
        base = _ptr(b)
    return _Melt(2 if base is not None else 1, mi["t_start"], mi["period"], mi["omega"], mi["amplitude"],
                 mi["offset"], mi["i_min"], mi["seconds_per_year"], base)


def seasonal_melt(w_melt: dict) -> dict:
    """The oracle melt spec of a workload's seasonal melt (t_start, t_end, amplitude, offset, i_min,
    seconds_per_year and optional base), with period and omega derived as SeasonalMeltInput does
    (src/melt_input.jl:49-66)."""
    period = w_melt["t_end"] - w_melt["t_start"]
    return dict(kind=1, t_start=w_melt["t_start"], period=period, omega=2 * math.pi / period,
                amplitude=w_melt["amplitude"], offset=w_melt["offset"], i_min=w_melt["i_min"],
                seconds_per_year=w_melt["seconds_per_year"], base=w_melt.get("base"))


def update_ieb(st: OracleState, mi: dict | None, t: float) -> None:
    keep = []
    s = st.struct()
    lib().orc_update_ieb(C.byref(s), C.byref(melt_struct(mi, keep)), float(t))


def run(st: OracleState, p: dict | None, sl: SlidingSpec, tsteps: int, dt: float, *, kfs: int = 0,
        gap_scheme: int = 1, head_scheme: int | None = None, cgspec: CgSpec | None = None, melt: dict | None = None,
        picard_iters: int = 500, picard_tol: float = 1e-6, alpha: float = float("nan"), check_every: int = 1,
        total_time: float = 0.0):
    """run!(sim) time loop (src/run.jl:37-43) for tsteps steps; returns (total_time, per-step stats)."""
    pp = dict(DEFAULT_PARAMS)
    pp.update(p or {})
    if head_scheme is None:
        head_scheme = 0 if pp["e_v"] == 0.0 else 1
    keep = []
    s = st.struct()
    per = (_PicardStats * max(tsteps, 1))()
    tt = C.c_double(total_time)
    rc = lib().orc_run(C.byref(s), C.byref(params_struct(p)), C.byref(sliding_struct(sl, keep)),
                       C.byref(melt_struct(melt, keep)), C.byref(_Sim(head_scheme, gap_scheme, kfs, dt)),
                       C.byref(_cg(cgspec or CgSpec())), C.byref(st.cheb),
                       C.byref(_PicardOpts(picard_iters, check_every, picard_tol, alpha)), int(tsteps),
                       C.byref(tt), per)
    stats = [dict(converged=per[i].converged, last_iter=per[i].last_iter, cg_iters_total=per[i].cg_iters_total,
                  cg_solves=per[i].cg_solves, cg_breakdowns=per[i].cg_breakdowns) for i in range(tsteps)]
    return rc, tt.value, stats


def sparse_matrix(A: dict):
    """The SALS matrix as scipy CSR from MFLS/SALS bands (row = ix + iy*nx)."""
    import scipy.sparse as sp
    nx, ny = A["aP"].shape
    n = nx * ny
    idx = np.arange(n).reshape((nx, ny), order="F")
    rows, cols, vals = [idx.ravel(order="F")], [idx.ravel(order="F")], [A["aP"].ravel(order="F")]
    for key, di, dj in (("aE", 1, 0), ("aW", -1, 0), ("aN", 0, 1), ("aS", 0, -1)):
        a = A[key]
        ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
        ok = (ii + di >= 0) & (ii + di < nx) & (jj + dj >= 0) & (jj + dj < ny)
        rows.append(idx[ok])
        cols.append(idx[(ii + di)[ok], (jj + dj)[ok]])
        vals.append(-a[ok])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


def direct_solve(A: dict) -> np.ndarray:
    """CHOLMOD stand-in: SciPy SuperLU on the assembled (SPD) matrix."""
    import scipy.sparse.linalg as spla
    M = sparse_matrix(A).tocsc()
    x = spla.spsolve(M, A["rhs"].ravel(order="F"))
    return x.reshape(A["aP"].shape, order="F")


class RunSession:
    """The run! loop (src/run.jl:37-43) as a resumable session: advance(seconds) spends about that
    much wall time on it and stops between two CG iterations; nothing is recomputed on the next
    call.  Same arguments and arithmetic as run()."""

    def __init__(self, st: OracleState, p: dict | None, sl: SlidingSpec, dt: float, *, kfs: int = 0,
                 gap_scheme: int = 1, head_scheme: int | None = None, cgspec: CgSpec | None = None,
                 melt: dict | None = None, picard_iters: int = 500, picard_tol: float = 1e-6,
                 alpha: float = float("nan"), check_every: int = 1, total_time: float = 0.0):
        pp = dict(DEFAULT_PARAMS)
        pp.update(p or {})
        if head_scheme is None:
            head_scheme = 0 if pp["e_v"] == 0.0 else 1
        self._keep = [st]
        self._s = st.struct()
        self._h = lib().orc_session_create(
            C.byref(self._s), C.byref(params_struct(p)), C.byref(sliding_struct(sl, self._keep)),
            C.byref(melt_struct(melt, self._keep)), C.byref(_Sim(head_scheme, gap_scheme, kfs, dt)),
            C.byref(_cg(cgspec or CgSpec())), C.byref(st.cheb),
            C.byref(_PicardOpts(picard_iters, check_every, picard_tol, alpha)), float(total_time))

    def advance(self, seconds: float, max_steps: int = 0) -> dict:
        pr = _Progress()
        more = lib().orc_session_advance(self._h, float(seconds), int(max_steps), C.byref(pr))
        d = {name: getattr(pr, name) for name, _ in _Progress._fields_}
        d["more"] = bool(more)
        return d

    def close(self) -> None:
        if self._h:
            lib().orc_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
