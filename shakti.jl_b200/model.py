"""Data model mirroring Shakti.jl: Grid, ModelParameters, State, mask constants, sliding laws,
melt inputs and K-face schemes (src/grid.jl, src/model_parameters.jl, src/state.jl, src/mask.jl,
src/sliding_law.jl, src/melt_input.jl, src/k_face_scheme.jl).

State arrays are torch Float64 CUDA tensors of shape (nx, ny) / (nx+1, ny) / (nx, ny+1) with
column-major strides (1, nx): element (ix, iy) sits at ix + iy*nx, the reference's layout, so the
device pointers go to the C ABI unchanged.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, fields

import numpy as np

from . import _lib

# Mask values (src/mask.jl:21-41)
GROUNDED = 0.0
OCEAN = 1.0
LAND = 2.0
OTHER_BASIN = 3.0

SECONDS_PER_YEAR = 365 * 86400.0


# ---------------------------------------------------------------------------------------------
# Grid (src/grid.jl:8-35)
# ---------------------------------------------------------------------------------------------
@dataclass(frozen=True)
class Grid:
    nx: int
    ny: int
    lx: float
    ly: float

    def __post_init__(self):
        if self.nx < 2 or self.ny < 2:
            raise ValueError("Grid needs nx >= 2 and ny >= 2 (dx = lx/(nx-1))")

    @property
    def dx(self) -> float:
        return float(self.lx) / (self.nx - 1)

    @property
    def dy(self) -> float:
        return float(self.ly) / (self.ny - 1)

    @property
    def dx2(self) -> float:
        return self.dx * self.dx

    @property
    def dy2(self) -> float:
        return self.dy * self.dy

    @property
    def x(self) -> np.ndarray:
        return np.arange(self.nx) * self.dx

    @property
    def y(self) -> np.ndarray:
        return np.arange(self.ny) * self.dy


# ---------------------------------------------------------------------------------------------
# ModelParameters (src/model_parameters.jl:9-84)
# ---------------------------------------------------------------------------------------------
@dataclass(frozen=True)
class ModelParameters:
    rho_w: float = 1000.0
    rho_sw: float = 1027.0
    rho_i: float = 910.0
    g: float = 9.81
    nu: float = 1.787e-6
    n: float = 3.0
    omega: float = 1e-4
    L: float = 334e3
    br: float = 0.05
    lr: float = 2.0
    ct: float = 7.5e-8
    cw: float = 4.22e3
    p_atm: float = 0.0
    b_min: float = 0.0
    b_max: float = math.inf
    e_v: float = 0.0

    def as_dict(self) -> dict:
        return {f.name: float(getattr(self, f.name)) for f in fields(self)}

    def struct(self) -> _lib.shk_params:
        return _lib.shk_params(*[float(getattr(self, n)) for n in _lib.PARAM_NAMES])


def canonical_exponent(n):
    """src/model_parameters.jl:122-123"""
    return int(n) if float(n).is_integer() else n


def pow_(x, n):
    """src/model_parameters.jl:133-134"""
    return x ** n


# ---------------------------------------------------------------------------------------------
# State (src/state.jl:13-137)
# ---------------------------------------------------------------------------------------------
def _colmajor(torch, rows: int, cols: int, device, fill: float = 0.0):
    t = torch.full((cols, rows), fill, dtype=torch.float64, device=device)
    return t.t()  # shape (rows, cols), strides (1, rows)


class State:
    """All State fields as column-major Float64 CUDA tensors (mask defaults to all-GROUNDED,
    valid_x/valid_y to 1.0, every other field to 0).  `lambda` is stored as `lambda_`."""

    def __init__(self, grid: Grid, device: str = "cuda"):
        import torch
        dev = torch.device(device)
        if dev.type != "cuda":
            raise ValueError("State lives in CUDA device memory; the B200 library has no CPU path")
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA is not available: the B200 library needs a GPU")
        self.grid = grid
        nx, ny = grid.nx, grid.ny
        for f in _lib.CENTER_FIELDS:
            setattr(self, f, _colmajor(torch, nx, ny, dev))
        for f in _lib.XFACE_FIELDS:
            setattr(self, f, _colmajor(torch, nx + 1, ny, dev, 1.0 if f == "valid_x" else 0.0))
        for f in _lib.YFACE_FIELDS:
            setattr(self, f, _colmajor(torch, nx, ny + 1, dev, 1.0 if f == "valid_y" else 0.0))

    def __getitem__(self, name: str):
        return getattr(self, "lambda_" if name == "lambda" else name)

    def struct(self) -> _lib.shk_state:
        return _lib.shk_state(*[getattr(self, f).data_ptr() for f in _lib.STATE_FIELDS])

    def to_numpy(self, names=None) -> dict:
        """Host copies (Fortran-ordered numpy) of the requested fields."""
        names = names or _lib.STATE_FIELDS
        out = {}
        for n in names:
            t = self["lambda_" if n == "lambda" else n]
            out[n] = np.asfortranarray(t.detach().cpu().numpy())
        return out


# ---------------------------------------------------------------------------------------------
# K-face schemes (src/k_face_scheme.jl:1-33)
# ---------------------------------------------------------------------------------------------
class AbstractKFaceScheme:
    code = -1


class Arithmetic(AbstractKFaceScheme):
    code = 0


class Harmonic(AbstractKFaceScheme):
    code = 1


def compute_K_face(kfs: AbstractKFaceScheme, K1: float, K2: float) -> float:
    """src/k_face_scheme.jl:32-33 (scalar form)."""
    if isinstance(kfs, Harmonic):
        return (2 * K1 * K2) / (K1 + K2 + np.finfo(np.float64).eps)
    return (K1 + K2) / 2


# ---------------------------------------------------------------------------------------------
# Sliding laws (src/sliding_law.jl)
# ---------------------------------------------------------------------------------------------
def _stagger(grid: Grid, C) -> tuple[np.ndarray, np.ndarray]:
    """Centre -> face staggering of a coefficient (src/sliding_law.jl:73-90): edge faces copy the
    adjacent cell, interior faces average their two cells."""
    nx, ny = grid.nx, grid.ny
    Ccc = np.asarray(C, dtype=np.float64) if np.ndim(C) else np.full((nx, ny), float(C))
    Cx = np.zeros((nx + 1, ny), order="F")
    Cx[0, :] = Ccc[0, :]
    Cx[nx, :] = Ccc[nx - 1, :]
    Cx[1:nx, :] = (Ccc[0:nx - 1, :] + Ccc[1:nx, :]) / 2
    Cy = np.zeros((nx, ny + 1), order="F")
    Cy[:, 0] = Ccc[:, 0]
    Cy[:, ny] = Ccc[:, ny - 1]
    Cy[:, 1:ny] = (Ccc[:, 0:ny - 1] + Ccc[:, 1:ny]) / 2
    return Cx, Cy


class AbstractSlidingLaw:
    kind = -1
    C = 0.0
    v0 = 0.0
    _host = None

    def _device_faces(self):
        import torch
        if getattr(self, "_dev", None) is None:
            cx, cy = self._host
            self._dev = (torch.from_numpy(np.ascontiguousarray(cx.T)).cuda().t(),
                         torch.from_numpy(np.ascontiguousarray(cy.T)).cuda().t())
        return self._dev

    def struct(self) -> _lib.shk_sliding_law:
        s = _lib.shk_sliding_law(kind=self.kind, C=float(self.C), v0=float(self.v0), Cx=None, Cy=None)
        if self._host is not None:
            cx, cy = self._device_faces()
            s.Cx, s.Cy = cx.data_ptr(), cy.data_ptr()
        return s


class RegularizedCoulombSlidingLaw(AbstractSlidingLaw):
    """src/sliding_law.jl:33-35"""
    kind = 0

    def __init__(self, C: float):
        self.C = float(C)


class RegularizedCoulombFieldSlidingLaw(AbstractSlidingLaw):
    """src/sliding_law.jl:270-301"""
    kind = 1

    def __init__(self, grid: Grid, C):
        self._host = _stagger(grid, C)
        self.Cx, self.Cy = self._host


class RegularizedCoulombV0SlidingLaw(AbstractSlidingLaw):
    """src/sliding_law.jl:412-450"""
    kind = 2

    def __init__(self, grid: Grid, C, v0: float):
        self._host = _stagger(grid, C)
        self.Cx, self.Cy = self._host
        self.v0 = float(v0)


class LinearSlidingLaw(AbstractSlidingLaw):
    """src/sliding_law.jl:61-90: C staggered then squared once at construction."""
    kind = 3

    def __init__(self, grid: Grid, C):
        cx, cy = _stagger(grid, C)
        self._host = (cx ** 2, cy ** 2)
        self.Cx2, self.Cy2 = self._host


class PrescribedSlidingLaw(AbstractSlidingLaw):
    """src/sliding_law.jl:45"""
    kind = 4


# ---------------------------------------------------------------------------------------------
# Melt inputs (src/melt_input.jl)
# ---------------------------------------------------------------------------------------------
class AbstractMeltInput:
    def struct(self) -> _lib.shk_melt_input:
        raise NotImplementedError


class ConstantMeltInput(AbstractMeltInput):
    """src/melt_input.jl:22, update_ieb! is a no-op (:30)."""

    def struct(self):
        return _lib.shk_melt_input(kind=0, seconds_per_year=1.0)


class SeasonalMeltInput(AbstractMeltInput):
    """src/melt_input.jl:49-66; uniform cosine window in m/a, applied as m/s."""

    def __init__(self, t_start=0.4, t_end=0.7, amplitude=492.75, offset=493.75, i_min=1.0,
                 seconds_per_year=SECONDS_PER_YEAR):
        self.t_start = float(t_start)
        self.period = float(t_end - t_start)
        self.omega = float(2 * math.pi / self.period)
        self.amplitude = float(amplitude)
        self.offset = float(offset)
        self.i_min = float(i_min)
        self.seconds_per_year = float(seconds_per_year)

    def value(self, t: float) -> float:
        """i_{e->b} in m/s at elapsed time t (src/melt_input.jl:86-94)."""
        yf = math.fmod(t / self.seconds_per_year, 1.0)
        if yf < 0:
            yf += 1.0
        if self.t_start <= yf <= self.t_start + self.period:
            i_ma = self.offset - self.amplitude * math.cos(self.omega * (yf - self.t_start))
        else:
            i_ma = self.i_min
        return i_ma / self.seconds_per_year

    def struct(self):
        return _lib.shk_melt_input(kind=1, t_start=self.t_start, period=self.period, omega=self.omega,
                                   amplitude=self.amplitude, offset=self.offset, i_min=self.i_min,
                                   seconds_per_year=self.seconds_per_year, base=None)


class SeasonalBaseMeltInput(SeasonalMeltInput):
    """Extension (no reference counterpart): ieb = seasonal(t) + base(x, y), e.g. a uniform
    sinusoid plus point moulins.  The reference's SeasonalMeltInput overwrites ieb uniformly
    (src/melt_input.jl:92) and cannot carry a spatial field."""

    def __init__(self, base, **kw):
        super().__init__(**kw)
        self.base_host = np.asfortranarray(np.asarray(base, dtype=np.float64))
        self._dev = None

    def struct(self):
        import torch
        if self._dev is None:
            self._dev = torch.from_numpy(np.ascontiguousarray(self.base_host.T)).cuda().t()
        s = super().struct()
        s.kind = 2
        s.base = self._dev.data_ptr()
        return s
