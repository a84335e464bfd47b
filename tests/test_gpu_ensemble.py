"""GPU tests of the batched ensemble (shk_ensemble_*): instances of uneven sizes advanced together
give each instance the fields and Picard iteration counts of its own single-instance run.

Each instance's batched kernels use the grids of its own context's launches, so every reduction
sums the same partials in the same order: with the context's own CG tile height the ensemble
reproduces the single-instance run (checked at 1e-10 and equal Picard counts).  An autotuned tile
height changes the row-marching kernel's reduction blocks, i.e. the rounding of p'Ap; the fields
then agree to the solves' accuracy (checked on instances whose Picard loop converges fast)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("h", "N", "b", "q_x", "q_y", "mdot", "K")


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)


# (nx, ny, seed, sliding C, melt m/s): ragged sizes, per-instance parameters as in the ensemble
# workload (C in [5e3, 5e4], melt in [1e-9, 1e-7])
SPECS = [(48, 48, 11, 5e3, 1e-9), (64, 40, 12, 2e4, 1e-8), (37, 53, 13, 5e4, 5e-8), (96, 96, 14, 1e4, 1e-7),
         (64, 64, 15, 3e4, 3e-8)]


def make_sim(shk, nx, ny, seed, C, melt, tsteps, rtol=None, multigrid=False):
    w = shk.configs.plain(nx, 10e3 * nx / 64, seed=seed, ny=ny, ly=10e3 * ny / 64, C=C)
    w.inputs["ieb"] = np.full((nx, ny), melt, order="F")
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    pm = shk.ModelParameters()
    sl = shk.RegularizedCoulombSlidingLaw(C)
    s = shk.State(g)
    shk.set_initial_conditions(s, g, pm, sl, **w.inputs)
    if rtol is None:  # Krylov.jl defaults, the reference's configuration
        ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem)
    else:
        ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, stop_rule="relres", rtol=rtol, atol=0.0,
                                   multigrid=multigrid)
    ps = shk.PicardSolver(500, 1e-6, ls, g)
    return shk.Simulation(g, s, tsteps, 3600.0, pm, "implicit", [], shk.ConstantMeltInput(), sl, ps=ps)


def test_ensemble_matches_single_instance_runs(shk, cuda, monkeypatch):
    # the single runs through the row-marching CG kernels, the ones the batched ensemble runs (the
    # TMA-staged tile form sums the dot products over other blocks); read at context creation
    monkeypatch.setenv("SHK_MG_TMA", "0")
    steps = 5
    ens_sims = [make_sim(shk, *sp, steps) for sp in SPECS]
    ref_sims = [make_sim(shk, *sp, steps) for sp in SPECS]
    ens = shk.Ensemble(ens_sims, autotune_iters=0)
    stats = ens.run(steps)
    for sim, st in zip(ref_sims, stats):
        pic = 0
        for _ in range(steps):
            shk.step(sim)
            sim.total_time += sim.dt
            pic += sim.hs.ps.last_iter
            assert sim.hs.ps.converged
        assert st["steps"] == steps and st["steps_converged"] == steps
        assert st["picard_iters"] == pic, (st["picard_iters"], pic)
    for e, r in zip(ens_sims, ref_sims):
        a, b = e.state.to_numpy(list(FIELDS)), r.state.to_numpy(list(FIELDS))
        for f in FIELDS:
            assert relerr(a[f], b[f]) <= 1e-10, (e.grid.nx, e.grid.ny, f, relerr(a[f], b[f]))
    ens.close()


def test_ensemble_autotuned_tiles(shk, cuda):
    specs = [(64, 64, 21, 1e4, 1e-8), (96, 80, 22, 1e4, 1e-8), (128, 128, 23, 1e4, 1e-8)]
    sims = [make_sim(shk, *sp, 3, rtol=1e-12) for sp in specs]
    refs = [make_sim(shk, *sp, 3, rtol=1e-12) for sp in specs]
    ens = shk.Ensemble(sims, autotune_iters=4)
    assert all(th in (4, 8, 16, 32, 64) for th in ens.march_th)
    stats = ens.run(3)
    assert all(s["steps_converged"] == 3 for s in stats)
    for r in refs:
        for _ in range(3):
            shk.step(r)
    for e, r in zip(sims, refs):
        a, b = e.state.to_numpy(list(FIELDS)), r.state.to_numpy(list(FIELDS))
        for f in FIELDS:
            assert relerr(a[f], b[f]) <= 1e-8, (e.grid.nx, f, relerr(a[f], b[f]))
    ens.close()


def test_ensemble_continues_across_runs_and_reports_blocks(shk, cuda):
    sims = [make_sim(shk, *sp, 4) for sp in SPECS[:3]]
    refs = [make_sim(shk, *sp, 4) for sp in SPECS[:3]]
    ens = shk.Ensemble(sims, autotune_iters=0)
    ens.run(2)
    stats = ens.run(2)
    assert all(s["steps"] == 4 for s in stats)
    blocks = ens.launch_blocks()
    assert all(v >= len(sims) for v in blocks.values())
    for r in refs:
        for _ in range(4):
            shk.step(r)
    for e, r in zip(sims, refs):
        assert relerr(e.state.h.cpu().numpy(), r.state.h.cpu().numpy()) <= 1e-10
    ens.close()


# ragged sizes whose V-cycles end at different bottom levels (depths 1 to 3 above the bottom kernel);
# sliding coefficients at which each instance's Picard loop converges at these cell sizes (checked
# on the oracle: 5-15 Picard iterations per step)
MG_SPECS = [(48, 48, 31, 5e3, 1e-9), (200, 150, 32, 2e3, 1e-8), (256, 256, 33, 1e3, 5e-8), (37, 53, 34, 0.25, 1e-7),
            (512, 384, 35, 0.25, 3e-8)]


def test_ensemble_multigrid_form_matches_single_instance_runs(shk, cuda, monkeypatch):
    """The mixed-precision form (Float64 CG, Float32 multigrid V-cycle) batched over instances: every
    level kernel is one launch over the instances that have that level, each instance's bottom
    solve one block of one launch.  Against each instance's own run through the same (LDG-staged)
    level kernels and one-block bottom solve, with the context's own CG tile height (no autotune):
    equal Picard counts, fields within 1e-10."""
    monkeypatch.setenv("SHK_MG_TMA", "0")  # read at context creation: the single runs' staging
    monkeypatch.setenv("SHK_MG_CLUSTER", "0")  # and their coarse levels: the one-block bottom kernel
    steps = 3
    ens_sims = [make_sim(shk, *sp, steps, rtol=1e-10, multigrid=True) for sp in MG_SPECS]
    ref_sims = [make_sim(shk, *sp, steps, rtol=1e-10, multigrid=True) for sp in MG_SPECS]
    ens = shk.Ensemble(ens_sims, autotune_iters=0)
    stats = ens.run(steps)
    for sim, st in zip(ref_sims, stats):
        pic = cg = 0
        for _ in range(steps):
            shk.step(sim)
            sim.total_time += sim.dt
            pic += sim.hs.ps.last_iter
            cg += sim.hs.ps.cg_iters_total
            assert sim.hs.ps.converged
        assert st["steps_converged"] == steps
        assert st["picard_iters"] == pic, (sim.grid.nx, st["picard_iters"], pic)
        assert abs(st["cg_iters"] - cg) <= pic, (sim.grid.nx, st["cg_iters"], cg)
    for e, r in zip(ens_sims, ref_sims):
        a, b = e.state.to_numpy(list(FIELDS)), r.state.to_numpy(list(FIELDS))
        for f in FIELDS:
            assert relerr(a[f], b[f]) <= 1e-10, (e.grid.nx, e.grid.ny, f, relerr(a[f], b[f]))
    # the Jacobi form afterwards on the same ensemble (the timestep graph is rebuilt for the form)
    for sim in ens_sims:
        sim.hs.ps.ls.multigrid = False
    ens._o = ens_sims[0].ls.opts()
    stats = ens.run(1)
    assert all(s["steps"] == steps + 1 for s in stats)
    ens.close()


def test_ensemble_rejects_unsupported_forms(shk, cuda):
    sim = make_sim(shk, *SPECS[0], 1)
    g = sim.grid
    sim.hs.ps.ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, chebyshev_degree=4, stop_rule="relres",
                                         rtol=1e-8, atol=0.0)
    with pytest.raises(ValueError):
        shk.Ensemble([sim])
    other = make_sim(shk, *SPECS[1], 1)
    other.dt = 7200.0
    with pytest.raises(ValueError):
        shk.Ensemble([make_sim(shk, *SPECS[0], 1), other])
