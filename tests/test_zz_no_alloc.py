"""The allocation-free solve (shk_cg_solve_static) against the context-based solve.

shk_cg_solve_static serves callers that cannot allocate device memory while they solve (their
device memory belongs to their own pool allocator, they run in a real-time loop where the
device-wide synchronisation of cudaMalloc/cudaFree is unacceptable, or their plugin host forbids
allocation after start-up).  Its scratch is a fixed device array inside the library, shared by all
calls; this test calls it twice in a row on the same inputs and checks both results against
shk_cg_solve on the same assembled system, at the tolerance the other solver tests use.

This file is collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _relerr(a, b):
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


def test_static_solve_matches_context_solve_twice(shk, orc, cuda):
    L = shk._lib.load()
    w = shk.configs.plain64()
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    p = shk.ModelParameters()
    sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
    s = shk.State(g)
    shk.set_initial_conditions(s, g, p, sl, **w.inputs)
    s.h.add_(0.25)  # a warm start that is not already the solution
    # Krylov's rule (the reference's): it reads no mask, and this entry point's operator carries
    # none, so both entry points stop on the same test.
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, rtol=1e-12, atol=0.0, stop_rule="krylov")
    ctx = ls.ctx.bind(s, p, sl)
    assert L.shk_assemble(ctx.h, 0, 0.0) == 0
    A = ls.lsy.export()
    x0 = s.h.clone()
    # the existing entry point
    o = ls.opts()
    st_ref = shk._lib.shk_cg_stats()
    assert L.shk_cg_solve(ctx.h, C.byref(o), C.byref(st_ref)) == 0
    h_ref = s.h.cpu().numpy()
    stream = shk._lib.cuda_stream_handle()
    for call in range(2):
        x = x0.clone()
        st = shk._lib.shk_cg_stats()
        rc = L.shk_cg_solve_static(w.nx, w.ny, A["aP"].data_ptr(), A["aE"].data_ptr(), A["aN"].data_ptr(),
                                   A["rhs"].data_ptr(), x.data_ptr(), C.byref(o), C.byref(st), stream)
        cuda.cuda.synchronize()
        assert rc == 0, (call, rc)
        assert st.status == 0 and abs(st.niter - st_ref.niter) <= 1, (call, st.niter, st_ref.niter)
        assert _relerr(x.cpu().numpy(), h_ref) <= 1e-10, call


def test_static_solve_rejects_oversized_grid(shk, cuda):
    L = shk._lib.load()
    o = shk._lib.default_cg_opts()
    st = shk._lib.shk_cg_stats()
    dummy = cuda.zeros(4, dtype=cuda.float64, device="cuda")
    ptr = dummy.data_ptr()
    rc = L.shk_cg_solve_static(512, 512, ptr, ptr, ptr, ptr, ptr, C.byref(o), C.byref(st), None)
    assert rc == shk._lib.BAD_ARG
