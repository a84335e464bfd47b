"""GPU checks of the multigrid preconditioner's kernel variants and of the CG launch modes.

 - The fused two-sweep level kernels (one kernel per half V-cycle level: 2D tiles with the halo
   staged in shared memory, or warps marching down 32-column strips) against the per-sweep kernels: the same V-cycle, formed with differently contracted
   Float32 multiply-adds, so CG iterates agree to Float32 rounding after 8 iterations (1e-6; an
   indexing error would show at O(1)), and full solves take the same number of iterations (+-1)
   and agree within the rel-res 1e-8 error ball.
 - The TMA-staged tile kernels (levels whose rows have a 16-byte-multiple pitch) against the
   LDG-staged ones: the same V-cycle arithmetic, but the outer CG's dot products are summed over a
   different block count.  After one iteration (h0 + alpha p0, p0 the V-cycle of the same r0) the
   heads agree to Float64 rounding (1e-12); from the second iteration on, last-bit differences of
   r flip Float32 roundings of the V-cycle's input, so after 8 iterations they agree to Float32
   rounding (1e-6).  A staging error would show at O(1).
 - The three ways of issuing CG iterations (direct launches, one CUDA graph per iteration, the whole
   loop as a graph with a device-side WHILE node) run the same kernels in the same order: bit-equal
   solutions and equal iteration counts.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


def ragged_workload(shk):
    # 301 x 301: odd sizes on every level, tiles cut by the domain edge, LAND/OTHER_BASIN blobs
    # (identity rows) and moulins; several levels above the one-block bottom of the V-cycle
    return shk.configs.seasonal(301, 15e3, seed=4242, C=0.25)


def tma_workload(shk, nx, ny):
    # nx a multiple of 16: level 0 (and, for 512, levels 1-2) stage through TMA; ny = 360 leaves
    # ragged tile rows on every level, nx = 400 ragged tile columns; LAND/OTHER_BASIN blobs
    w = shk.configs.plain(nx, 20e3, seed=777, ny=ny, ly=20e3 * (ny - 1) / (nx - 1), C=0.25)
    shk.configs._paint_blobs(w.inputs["mask"], np.random.default_rng(778), 0.1, 2, 6)
    return w


def solve(shk, w, env, monkeypatch, itmax=0, rtol=1e-8, multigrid=True):
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    pm = shk.ModelParameters(**shk.configs.SEASONAL_PARAMS)
    sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
    s = shk.State(g)
    shk.set_initial_conditions(s, g, pm, sl, **w.inputs)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, multigrid=multigrid, stop_rule="relres", rtol=rtol,
                               atol=0.0, itmax=itmax)
    stats = shk.solve_elliptic_linear_system(ls, s, g, pm, shk.Arithmetic(), sl)
    h = s.h.cpu().numpy().copy()
    for k in env:
        monkeypatch.delenv(k)
    return h, stats


@pytest.mark.parametrize("variant", ["1", "2"], ids=["tile", "warp_marching"])
def test_fused_level_kernels_match_per_sweep_kernels(shk, cuda, monkeypatch, variant):
    w = ragged_workload(shk)
    h_f, st_f = solve(shk, w, {"SHK_MG_FUSED": variant}, monkeypatch, itmax=8, rtol=0.0)
    h_u, st_u = solve(shk, w, {"SHK_MG_FUSED": "0"}, monkeypatch, itmax=8, rtol=0.0)
    assert st_f.niter == st_u.niter == 8
    assert relerr(h_f, h_u) <= 1e-6, relerr(h_f, h_u)
    h_f, st_f = solve(shk, w, {"SHK_MG_FUSED": variant}, monkeypatch)
    h_u, st_u = solve(shk, w, {"SHK_MG_FUSED": "0"}, monkeypatch)
    assert st_f.status == st_u.status == 0
    assert abs(st_f.niter - st_u.niter) <= 1, (st_f.niter, st_u.niter)
    assert relerr(h_f, h_u) <= 1e-7


@pytest.mark.parametrize("multigrid", [True, False], ids=["multigrid", "jacobi"])
def test_cg_launch_modes_are_bit_identical(shk, cuda, monkeypatch, multigrid):
    w = ragged_workload(shk)
    out = [solve(shk, w, {"SHK_CG_GRAPHS": m}, monkeypatch, multigrid=multigrid) for m in ("0", "1", "2")]
    (h0, s0), (h1, s1), (h2, s2) = out
    assert s0.status == s1.status == s2.status == 0
    assert s0.niter == s1.niter == s2.niter
    assert np.array_equal(h0, h1) and np.array_equal(h0, h2)


@pytest.mark.parametrize("nx", [512, 400])
def test_tma_tile_kernels_match_ldg_tile_kernels(shk, cuda, monkeypatch, nx):
    w = tma_workload(shk, nx, 360)
    h_t, st_t = solve(shk, w, {"SHK_MG_TMA": "1"}, monkeypatch, itmax=1, rtol=0.0)
    h_l, st_l = solve(shk, w, {"SHK_MG_TMA": "0"}, monkeypatch, itmax=1, rtol=0.0)
    assert st_t.niter == st_l.niter == 1
    assert relerr(h_t, h_l) <= 1e-12, relerr(h_t, h_l)
    h_t, st_t = solve(shk, w, {"SHK_MG_TMA": "1"}, monkeypatch, itmax=8, rtol=0.0)
    h_l, st_l = solve(shk, w, {"SHK_MG_TMA": "0"}, monkeypatch, itmax=8, rtol=0.0)
    assert st_t.niter == st_l.niter == 8
    assert relerr(h_t, h_l) <= 1e-6, relerr(h_t, h_l)
    h_t, st_t = solve(shk, w, {"SHK_MG_TMA": "1"}, monkeypatch)
    h_l, st_l = solve(shk, w, {"SHK_MG_TMA": "0"}, monkeypatch)
    assert st_t.status == st_l.status == 0
    assert abs(st_t.niter - st_l.niter) <= 1, (st_t.niter, st_l.niter)
    assert relerr(h_t, h_l) <= 1e-7


def test_cg_launch_modes_are_bit_identical_tma(shk, cuda, monkeypatch):
    w = tma_workload(shk, 512, 360)
    out = [solve(shk, w, {"SHK_CG_GRAPHS": m}, monkeypatch) for m in ("0", "1", "2")]
    (h0, s0), (h1, s1), (h2, s2) = out
    assert s0.status == s1.status == s2.status == 0
    assert s0.niter == s1.niter == s2.niter
    assert np.array_equal(h0, h1) and np.array_equal(h0, h2)


@pytest.mark.parametrize("which", ["ragged301", "tma512x360"])
def test_cluster_coarse_levels_match_tile_levels_and_bottom(shk, cuda, monkeypatch, which):
    """The coarse levels on one thread-block cluster (slabs of the levels below the tile kernels in
    eight CTAs' shared memory, halo rows read from the neighbouring CTAs, the smallest levels in CTA
    0) against the same V-cycle run by the tile kernels down to the one-block bottom kernel
    (SHK_MG_CLUSTER=0).  The two form the coarse levels' Float32 multiply-adds in a different order,
    so after one CG iteration the heads agree to Float32 rounding of the V-cycle (1e-6), and full
    solves take the same number of iterations (+-1) and agree within the rel-res 1e-8 error ball."""
    w = ragged_workload(shk) if which == "ragged301" else tma_workload(shk, 512, 360)
    h_c, st_c = solve(shk, w, {"SHK_MG_CLUSTER": "1"}, monkeypatch, itmax=1, rtol=0.0)
    h_b, st_b = solve(shk, w, {"SHK_MG_CLUSTER": "0"}, monkeypatch, itmax=1, rtol=0.0)
    assert st_c.niter == st_b.niter == 1
    assert relerr(h_c, h_b) <= 1e-6, relerr(h_c, h_b)
    h_c, st_c = solve(shk, w, {"SHK_MG_CLUSTER": "1"}, monkeypatch)
    h_b, st_b = solve(shk, w, {"SHK_MG_CLUSTER": "0"}, monkeypatch)
    assert st_c.status == st_b.status == 0
    assert abs(st_c.niter - st_b.niter) <= 1, (st_c.niter, st_b.niter)
    assert relerr(h_c, h_b) <= 1e-7, relerr(h_c, h_b)


@pytest.mark.parametrize("itmax", [0, 3, 4])
def test_paired_x_updates_are_bit_identical(shk, cuda, monkeypatch, itmax):
    """The outer CG's x updated once per two iterations (the second of a pair adds both directions'
    terms in the single updates' order; a pending term is added after the last iteration) against x
    updated in every iteration (SHK_MG_PAIR_X=0): the same heads bit for bit and the same iteration
    count -- for a full solve, an odd iteration count (the pending term applied at the end) and an
    even one, and in each CG launch mode."""
    w = tma_workload(shk, 512, 360)
    rtol = 1e-8 if itmax == 0 else 0.0
    for graphs in ("0", "1", "2"):
        h_p, s_p = solve(shk, w, {"SHK_MG_PAIR_X": "1", "SHK_CG_GRAPHS": graphs}, monkeypatch, itmax=itmax, rtol=rtol)
        h_i, s_i = solve(shk, w, {"SHK_MG_PAIR_X": "0", "SHK_CG_GRAPHS": graphs}, monkeypatch, itmax=itmax, rtol=rtol)
        assert s_p.status == s_i.status and s_p.niter == s_i.niter
        if itmax:
            assert s_p.niter == itmax
        assert np.array_equal(h_p, h_i)


def test_tma_multigrid_run_matches_oracle(shk, orc, cuda, monkeypatch):
    """The TMA-staged multigrid form against the oracle (not only against the LDG staging) at
    512 x 360, where levels 0-2 stage through TMA: one linear solve at rel-res 1e-12 on the GROUNDED
    rows against the oracle's Jacobi CG at 1e-13 on the same system, and two timesteps at 1e-13
    against the oracle's run.  The two use different Krylov iterates, so they agree to the solution
    accuracy of the solves (1e-9 for h after one solve), not bit for bit."""
    w = tma_workload(shk, 512, 360)
    params = dict(shk.configs.SEASONAL_PARAMS)
    monkeypatch.setenv("SHK_MG_TMA", "1")
    h_t, st_t = solve(shk, w, {}, monkeypatch, rtol=1e-12)
    assert st_t.status == 0
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    osl = orc.SlidingSpec(kind=0, C=w.sliding_C)
    orc.set_initial_conditions(st, params, osl, w.inputs)
    A = orc.assemble(st, params)
    x, _ = orc.cg(A, st["h"], orc.CgSpec(precond=0, stop_rule=1, rtol=1e-13, atol=0.0), mask=st["mask"])
    assert relerr(h_t, x) <= 1e-9, relerr(h_t, x)

    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    pm = shk.ModelParameters(**params)
    sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
    s = shk.State(g)
    shk.set_initial_conditions(s, g, pm, sl, **w.inputs)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, multigrid=True, stop_rule="relres", rtol=1e-13,
                               atol=0.0)
    sim = shk.Simulation(g, s, 2, 1800.0, pm, "implicit", [], shk.ConstantMeltInput(), sl,
                         ps=shk.PicardSolver(500, 1e-6, ls, g))
    shk.run(sim)
    orc.run(st, params, osl, 2, 1800.0, cgspec=orc.CgSpec(precond=0, stop_rule=1, rtol=1e-13, atol=0.0))
    host = s.to_numpy(["h", "N", "b"])
    # b integrates mdot, which scales with the gradients of h: it carries the solves' differences
    # amplified (3.6e-8 measured with rel-res 1e-12 on the GPU side)
    for f, tol in (("h", 1e-8), ("N", 1e-8), ("b", 1e-7)):
        assert relerr(host[f], st[f]) <= tol, (f, relerr(host[f], st[f]))


def test_tma_wait_give_up_reports_and_recovers(shk, cuda, monkeypatch):
    """The bounded-wait fault path of the TMA-staged kernels, without a fault: a test-only setting
    (SHK_TEST_TMA_FIRST_WAIT=0, read at context creation) gives every launch's first tile wait zero
    polls, so it gives up at once while the copies it issued still arrive.  Each block then waits,
    with the normal bound, for all of its copies before it returns, marks the fault and stops the
    solve; the host reports SHK_CUDA_ERROR "a tile copy did not complete".  A context created
    afterwards with the normal setting solves as usual."""
    w = tma_workload(shk, 512, 360)
    monkeypatch.setenv("SHK_MG_TMA", "1")
    monkeypatch.setenv("SHK_TEST_TMA_FIRST_WAIT", "0")
    with pytest.raises(shk._lib.ShaktiError) as exc:
        solve(shk, w, {}, monkeypatch)
    assert exc.value.status == shk._lib.CUDA_ERROR and "tile copy" in str(exc.value)
    cuda.cuda.synchronize()  # the context is still usable: nothing faulted
    monkeypatch.delenv("SHK_TEST_TMA_FIRST_WAIT")
    h, st = solve(shk, w, {}, monkeypatch)
    assert st.status == 0 and st.niter > 0
    h_l, st_l = solve(shk, w, {"SHK_MG_TMA": "0"}, monkeypatch)
    assert abs(st.niter - st_l.niter) <= 1 and relerr(h, h_l) <= 1e-7
