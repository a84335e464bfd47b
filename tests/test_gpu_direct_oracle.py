"""The GPU direct solve (cuSOLVER sparse Cholesky, tests/gpu_direct.py) as an exact Float64 reference.

It replaces the reference's CholeskyDirectSolver (src/linear_solver.jl:127-221) on the test side:
first checked against the oracle's CPU direct solve (SciPy SuperLU) on the same assembled system,
then used to pin the library's Jacobi and multigrid CG solves at rel-res 1e-12 on the GROUNDED
rows.  Both sides solve the same matrix, so the direct solves agree to Float64 rounding times the
condition number (1e-10 here); the CG solves agree to their solution accuracy (1e-9 for h).
"""
import time

import numpy as np
import pytest

from gpu_direct import cholesky_solve

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


def workload(shk, name):
    if name == "ragged301":
        return shk.configs.seasonal(301, 15e3, seed=4242, C=0.25)
    w = shk.configs.plain(512, 20e3, seed=777, ny=360, ly=20e3 * 359 / 511, C=0.25)
    shk.configs._paint_blobs(w.inputs["mask"], np.random.default_rng(778), 0.1, 2, 6)
    return w


@pytest.mark.parametrize("name", ["ragged301", "tma512x360"])
def test_gpu_direct_solve_pins_cg_solves(shk, orc, cuda, name):
    w = workload(shk, name)
    params = dict(shk.configs.SEASONAL_PARAMS)
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    orc.set_initial_conditions(st, params, orc.SlidingSpec(kind=0, C=w.sliding_C), w.inputs)
    A = orc.assemble(st, params)
    M = orc.sparse_matrix(A)
    t0 = time.perf_counter()
    x_gpu = cholesky_solve(M, A["rhs"].ravel(order="F")).reshape(A["aP"].shape, order="F")
    t1 = time.perf_counter()
    x_cpu = orc.direct_solve(A)
    t2 = time.perf_counter()
    print(f"{name}: GPU Cholesky {t1 - t0:.3f} s, CPU SuperLU {t2 - t1:.3f} s")
    assert relerr(x_gpu, x_cpu) <= 1e-10, relerr(x_gpu, x_cpu)

    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    pm = shk.ModelParameters(**params)
    sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
    for multigrid in (False, True):
        s = shk.State(g)
        shk.set_initial_conditions(s, g, pm, sl, **w.inputs)
        ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, multigrid=multigrid, stop_rule="relres",
                                   rtol=1e-12, atol=0.0)
        stats = shk.solve_elliptic_linear_system(ls, s, g, pm, shk.Arithmetic(), sl)
        assert stats.status == 0
        h = s.h.cpu().numpy()
        assert relerr(h, x_gpu) <= 1e-9, (multigrid, relerr(h, x_gpu))
