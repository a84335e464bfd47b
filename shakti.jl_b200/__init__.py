"""shakti_b200 -- B200-native (sm_100a) implementation of Shakti.jl's per-timestep head solve and
field updates, behind the reference's Simulation / run! / PicardSolver / CGIterativeSolver /
MatrixFreeLinearSystem API.

Julia names ending in `!` drop the bang here (run!, step!, set_initial_conditions! -> run, step,
set_initial_conditions).  All compute runs in libshakti_b200.so (CUDA C++ behind a C ABI,
include/shakti_b200.h); this package only binds device buffers and mirrors the API.
"""
from . import _lib
from .model import (GROUNDED, OCEAN, LAND, OTHER_BASIN, SECONDS_PER_YEAR, Grid, ModelParameters, State,
                    canonical_exponent, pow_, AbstractKFaceScheme, Arithmetic, Harmonic, compute_K_face,
                    AbstractSlidingLaw, RegularizedCoulombSlidingLaw, RegularizedCoulombFieldSlidingLaw,
                    RegularizedCoulombV0SlidingLaw, LinearSlidingLaw, PrescribedSlidingLaw, AbstractMeltInput,
                    ConstantMeltInput, SeasonalMeltInput, SeasonalBaseMeltInput)
from .solvers import (AbstractLinearSolver, AbstractDirectSolver, AbstractIterativeSolver, AbstractLinearSystem,
                      SparseAssembledLinearSystem, MatrixFreeLinearSystem, CholeskyDirectSolver, CGIterativeSolver,
                      ChebyshevPreconditioner, CgStats, PicardSolver, NoHeadRelaxation, UnderHeadRelaxation,
                      solve_elliptic_linear_system, solve_parabolic_linear_system, Picard_loop, elliptic_solver,
                      parabolic_solver, picard_tail)
from .simulation import (AbstractHeadScheme, EllipticHeadScheme, ParabolicHeadScheme, AbstractGapScheme,
                         ExplicitGapScheme, ImplicitGapScheme, AbstractSensibleHeatScheme, WithSensibleHeat,
                         NoSensibleHeat, AbstractOpenBySlidingScheme, WithOpenBySliding, NoOpenBySliding,
                         AbstractObserver, NoObserver, LiveObserver, Simulation, run, step, step_h, step_b,
                         update_ieb, picard_status, set_initial_conditions, save_checkpoint, load_checkpoint,
                         HostIO)
from .ensemble import Ensemble
from . import configs

backend = "CUDA"
floattype = "Float64"

__all__ = [n for n in dir() if not n.startswith("_")]
