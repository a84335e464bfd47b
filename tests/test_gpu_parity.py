"""GPU parity: libshakti_b200 against the CPU restatement, through the C ABI.

Bars
 - Point-wise and stencil kernels (initial conditions, assembly, matvec, tail, gap): bit-exact,
   except fields that depend on x^(1/n) (taub, shear, mdot), which may differ by a few ulp between
   CUDA's pow and the C library's pow: rtol 4e-15 there.
 - Anything downstream of a reduction (CG, Picard, time stepping): relative max-norm error
   <= 1e-10 in Float64, at tight CG tolerances where stated.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POW_FIELDS = {"taub_x", "taub_y", "shear", "mdot"}
ULP_RTOL = 4e-15


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale


def to_gpu_state(shk, cuda, st, g):
    s = shk.State(g)
    for f in shk._lib.STATE_FIELDS:
        getattr(s, f).copy_(cuda.from_numpy(np.asfortranarray(st.fields[f])))
    return s


def setup_pair(shk, orc, cuda, w, sliding=None, p=None, perturb=False):
    """Initial conditions on both sides; optionally the reference test's h perturbation."""
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    pm = shk.ModelParameters(**(p or {}))
    sl, osl = sliding if sliding else (shk.RegularizedCoulombSlidingLaw(w.sliding_C),
                                       orc.SlidingSpec(kind=0, C=w.sliding_C))
    s = shk.State(g)
    shk.set_initial_conditions(s, g, pm, sl, **w.inputs)
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    orc.set_initial_conditions(st, p, osl, w.inputs)
    if perturb:
        st["h"][...] += 0.01 * np.arange(1, w.nx * w.ny + 1).reshape((w.nx, w.ny), order="F") / max(w.nx * w.ny / 36, 1)
        orc.picard_tail(st, p, osl)
        s = to_gpu_state(shk, cuda, st, g)
    return g, pm, sl, osl, s, st


def compare_state(shk, s, st, fields=None, exact=True, rtol=1e-10):
    host = s.to_numpy()
    bad = []
    for f in fields or shk._lib.STATE_FIELDS:
        a, b = host[f], st.fields[f]
        if exact and f not in POW_FIELDS:
            if not np.array_equal(a, b):
                bad.append((f, relerr(a, b)))
        elif exact:
            if not np.allclose(a, b, rtol=ULP_RTOL, atol=1e-300):
                bad.append((f, relerr(a, b)))
        elif relerr(a, b) > rtol:
            bad.append((f, relerr(a, b)))
    assert not bad, bad


@pytest.mark.parametrize("wname", ["fixture6", "plain64"])
def test_initial_conditions_bitwise(shk, orc, cuda, wname):
    w = shk.configs.WORKLOADS[wname]()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w)
    compare_state(shk, s, st)


@pytest.mark.parametrize("kfs", [0, 1])
@pytest.mark.parametrize("parabolic", [False, True])
def test_assembly_bitwise(shk, orc, cuda, kfs, parabolic):
    w = shk.configs.fixture6()
    p = dict(e_v=1e-3) if parabolic else None
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w, p=p, perturb=True)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem)
    ctx = ls.ctx.bind(s, pm, sl, shk.Harmonic() if kfs else shk.Arithmetic())
    assert ctx.L.shk_assemble(ctx.h, int(parabolic), 60.0) == 0
    gpu = {k: v.cpu().numpy() for k, v in ls.lsy.export().items()}
    ref = orc.assemble(st, p, kfs=kfs, parabolic=parabolic, dt=60.0)
    for k in ("aP", "aE", "aW", "aN", "aS", "rhs"):
        assert np.array_equal(gpu[k], ref[k]), (k, relerr(gpu[k], ref[k]))


def test_matvec_bitwise(shk, orc, cuda):
    w = shk.configs.plain64()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem)
    ctx = ls.ctx.bind(s, pm, sl)
    assert ctx.L.shk_assemble(ctx.h, 0, 0.0) == 0
    x = np.asfortranarray(np.random.default_rng(1).standard_normal((w.nx, w.ny)))
    xt = cuda.from_numpy(np.ascontiguousarray(x.T)).cuda().t()
    y = ls.lsy.matvec(xt).cpu().numpy()
    ref = orc.matvec(orc.assemble(st, None), x)
    assert np.array_equal(y, ref)


@pytest.mark.parametrize("wname", ["fixture6", "plain64"])
def test_picard_tail_bitwise(shk, orc, cuda, wname):
    w = shk.configs.WORKLOADS[wname]()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w, perturb=True)
    st["h"][...] += 0.37  # a fresh head for the tail to consume
    s.h.copy_(cuda.from_numpy(np.asfortranarray(st["h"])))
    orc.picard_tail(st, None, osl)
    shk.picard_tail(shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem), s, pm, sl)
    compare_state(shk, s, st)


@pytest.mark.parametrize("gap", [0, 1])
def test_gap_step_bitwise(shk, orc, cuda, gap):
    w = shk.configs.plain64()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w, perturb=True)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem)
    ctx = ls.ctx.bind(s, pm, sl, shk.Arithmetic(), gap)
    assert ctx.L.shk_step_b(ctx.h, 3600.0) == 0
    orc.step_b(st, None, gap, 3600.0)
    compare_state(shk, s, st, fields=["b", "beta", "b_x", "b_y"])


@pytest.mark.parametrize("precond", [0, 1])
@pytest.mark.parametrize("wname", ["fixture6", "plain64"])
def test_cg_solve_matches_oracle(shk, orc, cuda, precond, wname):
    w = shk.configs.WORKLOADS[wname]()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w, perturb=True)
    A = orc.assemble(st, None)
    for rtol, atol in ((1e-13, 0.0), (math.sqrt(2.2e-16), math.sqrt(2.2e-16))):
        ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, chebyshev_degree=4 if precond else None,
                                   rtol=rtol, atol=atol)
        s2 = to_gpu_state(shk, cuda, st, g)
        stats = shk.solve_elliptic_linear_system(ls, s2, g, pm, shk.Arithmetic(), sl)
        x, ost = orc.cg(A, st["h"], orc.CgSpec(precond=precond, cheb_degree=4, rtol=rtol, atol=atol))
        assert stats.status == 0 and ost["status"] == 0
        assert abs(stats.niter - ost["niter"]) <= 1, (stats.niter, ost["niter"])
        assert relerr(s2.h.cpu().numpy(), x) <= 1e-10


def test_chebyshev_bounds_match_oracle(shk, orc, cuda):
    w = shk.configs.plain64()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w, perturb=True)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, chebyshev_degree=4)
    ctx = ls.ctx.bind(s, pm, sl)
    assert ctx.L.shk_assemble(ctx.h, 0, 0.0) == 0
    assert ls.precond.bounds() == (1.0, 1.0)  # construction-time placeholder
    ok, est = ls.precond.update_bounds()
    cheb = orc._ChebState(1.0, 1.0, 0)
    A = orc.assemble(st, None)
    ook, oest = orc.update_chebyshev_bounds(A, A["rhs"], 15, cheb)
    assert ok == ook
    assert abs(est[0] - oest[0]) <= 1e-10 * abs(oest[0]) and abs(est[1] - oest[1]) <= 1e-10 * abs(oest[1])
    # Chebyshev application: y = M^-1 x
    x = np.asfortranarray(np.random.default_rng(2).standard_normal((w.nx, w.ny)))
    xt = cuda.from_numpy(np.ascontiguousarray(x.T)).cuda().t()
    y = ls.precond.ldiv(xt).cpu().numpy()
    yref = orc.chebyshev_apply(A, 4, cheb, x)
    assert relerr(y, yref) <= 1e-12


def test_chebyshev_zero_rhs_keeps_placeholder(shk, orc, cuda):
    """test/linear_solver_test.jl:218-242 on the device."""
    w = shk.configs.fixture6()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, chebyshev_degree=4)
    ctx = ls.ctx.bind(s, pm, sl)
    assert ctx.L.shk_assemble(ctx.h, 0, 0.0) == 0
    z = cuda.zeros((w.ny, w.nx), dtype=cuda.float64, device="cuda").t()
    ok, est = ls.precond.update_bounds(z)
    assert not ok and math.isnan(est[0]) and math.isnan(est[1])
    assert ls.precond.bounds() == (1.0, 1.0)


def run_pair(shk, orc, cuda, w, tsteps, dt, *, precond=1, kfs="arithmetic", gap="implicit", p=None, rtol=None,
             atol=None, melt=None, sliding=None, alpha=None, check_every=1, stop_rule="krylov"):
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w, sliding=sliding, p=p)
    kw = {}
    if rtol is not None:
        kw.update(rtol=rtol, atol=atol)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, chebyshev_degree=4 if precond else None,
                               stop_rule=stop_rule, **kw)
    mi, omelt = shk.ConstantMeltInput(), None
    if melt is not None:
        mi = shk.SeasonalMeltInput(**melt)
        omelt = dict(kind=1, t_start=mi.t_start, period=mi.period, omega=mi.omega, amplitude=mi.amplitude,
                     offset=mi.offset, i_min=mi.i_min, seconds_per_year=mi.seconds_per_year)
    if pm.e_v == 0:
        ps = shk.PicardSolver(500, 1e-6, ls, g, alpha=alpha, check_every=check_every)
        sim = shk.Simulation(g, s, tsteps, dt, pm, gap, [], mi, sl, ps=ps, k_face_choice=kfs)
    else:
        sim = shk.Simulation(g, s, tsteps, dt, pm, gap, [], mi, sl, ls=ls, k_face_choice=kfs)
    shk.run(sim)
    cg = orc.CgSpec(precond=precond, cheb_degree=4, stop_rule=0 if stop_rule == "krylov" else 1)
    if rtol is not None:
        cg.rtol, cg.atol = rtol, atol
    rc, tt, stats = orc.run(st, p, osl, tsteps, dt, kfs=1 if kfs == "harmonic" else 0,
                            gap_scheme=1 if gap == "implicit" else 0, cgspec=cg, melt=omelt,
                            alpha=float("nan") if alpha is None else alpha, check_every=check_every)
    return sim, s, st, stats


def assert_fields_close(s, st, tol=1e-10, fields=("h", "N", "b", "q_x", "q_y")):
    """Relative max-norm error per field; the two flux components (and the two basal-stress
    components) share one scale, the larger component's max-norm, so a component that is nearly
    zero everywhere is not judged against its own round-off."""
    host = s.to_numpy(list(fields))
    pairs = {"q_x": ("q_x", "q_y"), "q_y": ("q_x", "q_y"), "taub_x": ("taub_x", "taub_y"),
             "taub_y": ("taub_x", "taub_y")}
    errs = {}
    for f in fields:
        scale = max(float(np.max(np.abs(st[k]))) for k in pairs.get(f, (f,)))
        errs[f] = float(np.max(np.abs(host[f] - st[f]))) / max(scale, 1e-300)
    assert all(e <= tol for e in errs.values()), str(errs)


def test_run_fixture_elliptic_tight(shk, orc, cuda):
    sim, s, st, stats = run_pair(shk, orc, cuda, shk.configs.fixture6(), 5, 3600.0, rtol=1e-13, atol=0.0)
    assert sim.hs.ps.converged and sim.hs.ps.last_iter == stats[-1]["last_iter"]
    assert_fields_close(s, st)


def test_run_plain64_default_tolerances(shk, orc, cuda):
    """The 64x64 plain workload: Chebyshev(4), Picard(500, 1e-6), implicit gap, 10 steps of 3600 s,
    Krylov's default CG tolerances on both sides."""
    sim, s, st, stats = run_pair(shk, orc, cuda, shk.configs.plain64(), 10, 3600.0)
    for a, b in zip(sim.step_stats, stats):
        assert a["last_iter"] == b["last_iter"]
    assert_fields_close(s, st)


@pytest.mark.parametrize("kfs,gap,precond", [("harmonic", "explicit", 0), ("harmonic", "implicit", 1),
                                             ("arithmetic", "explicit", 1)])
def test_run_schemes(shk, orc, cuda, kfs, gap, precond):
    sim, s, st, stats = run_pair(shk, orc, cuda, shk.configs.plain64(), 3, 1800.0, precond=precond, kfs=kfs, gap=gap,
                                 rtol=1e-13, atol=0.0)
    assert_fields_close(s, st)


@pytest.mark.parametrize("alpha,check_every", [(0.5, 1), (0.7, 3)])
def test_run_head_relaxation(shk, orc, cuda, alpha, check_every):
    """PicardSolver(500, 1e-6, ls, g; alpha, check_every): relax_h! blends each Picard iterate with
    the previous head, h = alpha h + (1 - alpha) h_prev (src/elliptic_solver.jl:33-46), and the
    convergence test runs every check_every iterations (:162-172).  Same Picard counts step by step
    as the oracle, fields within 1e-10."""
    sim, s, st, stats = run_pair(shk, orc, cuda, shk.configs.plain64(), 4, 3600.0, rtol=1e-12, atol=0.0,
                                 alpha=alpha, check_every=check_every, stop_rule="relres")
    for a, b in zip(sim.step_stats, stats):
        assert a["last_iter"] == b["last_iter"] and a["converged"] == b["converged"]
    assert_fields_close(s, st)


def test_run_parabolic(shk, orc, cuda):
    sim, s, st, stats = run_pair(shk, orc, cuda, shk.configs.plain64(), 5, 1800.0, p=dict(e_v=1e-3), rtol=1e-13,
                                 atol=0.0)
    assert_fields_close(s, st)


def test_run_seasonal_melt(shk, orc, cuda):
    melt = dict(t_start=0.0, t_end=1.0, amplitude=-0.8, offset=0.8, i_min=0.0)
    sim, s, st, stats = run_pair(shk, orc, cuda, shk.configs.fixture6(), 4, 86400.0 * 30, melt=melt, rtol=1e-13,
                                 atol=0.0)
    assert_fields_close(s, st)
    assert np.array_equal(s.ieb.cpu().numpy(), st["ieb"])


@pytest.mark.parametrize("kind", [1, 2, 3, 4])
def test_run_sliding_laws(shk, orc, cuda, kind):
    w = shk.configs.fixture6()
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    C = np.array([[0.2 + 0.01 * i + 0.02 * j for j in range(w.ny)] for i in range(w.nx)])
    if kind == 1:
        sl = shk.RegularizedCoulombFieldSlidingLaw(g, C)
        osl = orc.SlidingSpec(kind=1, Cx=sl.Cx, Cy=sl.Cy)
    elif kind == 2:
        sl = shk.RegularizedCoulombV0SlidingLaw(g, C, 9.51e-6)
        osl = orc.SlidingSpec(kind=2, Cx=sl.Cx, Cy=sl.Cy, v0=9.51e-6)
    elif kind == 3:
        sl = shk.LinearSlidingLaw(g, C)
        osl = orc.SlidingSpec(kind=3, Cx=sl.Cx2, Cy=sl.Cy2)
    else:
        sl = shk.PrescribedSlidingLaw()
        osl = orc.SlidingSpec(kind=4)
        w.inputs["taub_x"] = np.full((w.nx + 1, w.ny), 1e3, order="F")
        w.inputs["taub_y"] = np.full((w.nx, w.ny + 1), -5e2, order="F")
    sim, s, st, stats = run_pair(shk, orc, cuda, w, 3, 3600.0, rtol=1e-13, atol=0.0, sliding=(sl, osl))
    assert_fields_close(s, st, fields=("h", "N", "b", "q_x", "q_y", "taub_x", "taub_y"))


def test_cg_status_codes(shk, orc, cuda):
    """Non-convergence and breakdown are statuses, never hangs: itmax = 1 gives NOT_CONVERGED,
    a NaN in the system gives BREAKDOWN."""
    w = shk.configs.plain64()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w, perturb=True)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, itmax=1, rtol=1e-14, atol=0.0)
    stats = shk.solve_elliptic_linear_system(ls, s, g, pm, shk.Arithmetic(), sl)
    assert stats.status == shk._lib.NOT_CONVERGED and stats.niter == 1
    s2 = to_gpu_state(shk, cuda, st, g)
    s2.ieb[3, 3] = float("nan")
    ls2 = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem)
    stats2 = shk.solve_elliptic_linear_system(ls2, s2, g, pm, shk.Arithmetic(), sl)
    assert stats2.status == shk._lib.BREAKDOWN


@pytest.mark.parametrize("precond", [0, 1])
def test_mixed_precision_single_solve(shk, orc, cuda, precond):
    """Float32 CG with Float64 residual replacement reaches ||b - A h|| <= 1e-8 ||b_G|| (b_G: the
    GROUNDED rows of b) measured with the Float64 operator.  Its distance to a tight solve is judged
    against the plain Float64 CG's distance at the same tolerance."""
    w = shk.configs.plain64()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w, perturb=True)
    A = orc.assemble(st, None)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, chebyshev_degree=4 if precond else None,
                               precision="mixed", stop_rule="relres", rtol=1e-8, atol=0.0)
    stats = shk.solve_elliptic_linear_system(ls, s, g, pm, shk.Arithmetic(), sl)
    assert stats.status == 0, stats
    h = s.h.cpu().numpy()
    res = np.linalg.norm(A["rhs"] - orc.matvec(A, h)) / np.linalg.norm(A["rhs"][st["mask"] == 0])
    assert res <= 1e-8, res
    x_tight, _ = orc.cg(A, st["h"], orc.CgSpec(precond=0, atol=0.0, rtol=1e-14))
    x_plain, _ = orc.cg(A, st["h"], orc.CgSpec(precond=precond, stop_rule=1, atol=0.0, rtol=1e-8), mask=st["mask"])
    e_mixed, e_plain = relerr(h, x_tight), relerr(x_plain, x_tight)
    assert e_mixed <= 10 * e_plain + 1e-12, (e_mixed, e_plain)


def test_mixed_precision_run_field_errors(shk, orc, cuda):
    """Five timesteps of the 64x64 workload, mixed form against the Float64 oracle at the same
    rel-res 1e-8.  Per-field errors (h, N, b, q) are compared with the plain Float64 form's own
    distance from a tight (1e-13) Float64 run, the size of the tolerance ball."""
    w = shk.configs.plain64()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w)
    st_tight = st.copy()
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, precision="mixed", stop_rule="relres", rtol=1e-8,
                               atol=0.0)
    ps = shk.PicardSolver(500, 1e-6, ls, g)
    sim = shk.Simulation(g, s, 5, 3600.0, pm, "implicit", [], shk.ConstantMeltInput(), sl, ps=ps)
    shk.run(sim)
    orc.run(st, None, osl, 5, 3600.0, cgspec=orc.CgSpec(precond=0, stop_rule=1, rtol=1e-8, atol=0.0))
    orc.run(st_tight, None, osl, 5, 3600.0, cgspec=orc.CgSpec(precond=0, stop_rule=1, rtol=1e-13, atol=0.0))
    host = s.to_numpy(["h", "N", "b", "q_x", "q_y"])
    for f in ("h", "N", "b", "q_x", "q_y"):
        e_mixed = relerr(host[f], st_tight[f])
        e_plain = relerr(st[f], st_tight[f])
        assert e_mixed <= 10 * e_plain + 1e-9, (f, e_mixed, e_plain)


@pytest.mark.parametrize("wname", ["fixture6", "plain64"])
def test_multigrid_preconditioned_solve(shk, orc, cuda, wname):
    """Float64 CG preconditioned by the Float32 aggregation-multigrid V-cycle reaches the Float64
    true residual 1e-8 ||b_G|| in far fewer iterations than Jacobi, and lands as close to a tight
    solve as the plain Float64 CG at the same tolerance."""
    w = shk.configs.WORKLOADS[wname]()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w, perturb=True)
    A = orc.assemble(st, None)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, multigrid=True, stop_rule="relres", rtol=1e-8, atol=0.0)
    stats = shk.solve_elliptic_linear_system(ls, s, g, pm, shk.Arithmetic(), sl)
    assert stats.status == 0, stats
    h = s.h.cpu().numpy()
    res = np.linalg.norm(A["rhs"] - orc.matvec(A, h)) / np.linalg.norm(A["rhs"][st["mask"] == 0])
    assert res <= 1e-8, res
    x_tight, _ = orc.cg(A, st["h"], orc.CgSpec(precond=0, atol=0.0, rtol=1e-14))
    x_plain, sp = orc.cg(A, st["h"], orc.CgSpec(precond=0, stop_rule=1, atol=0.0, rtol=1e-8), mask=st["mask"])
    assert relerr(h, x_tight) <= 10 * relerr(x_plain, x_tight) + 1e-12
    assert stats.niter <= max(sp["niter"], 10)


def test_multigrid_run_matches_oracle_tight(shk, orc, cuda):
    """Five timesteps of the 64x64 workload with the multigrid form at a tight tolerance (rel-res
    1e-13) agree with the Float64 oracle run (Jacobi CG, same tolerance) to 1e-8.  The two use
    different Krylov iterates, so they agree to the solution accuracy that rel-res 1e-13 of ||b||
    gives here (~1e-9), not to the 1e-10 that same-algorithm runs reach."""
    w = shk.configs.plain64()
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, multigrid=True, stop_rule="relres", rtol=1e-13,
                               atol=0.0)
    ps = shk.PicardSolver(500, 1e-6, ls, g)
    sim = shk.Simulation(g, s, 5, 3600.0, pm, "implicit", [], shk.ConstantMeltInput(), sl, ps=ps)
    shk.run(sim)
    orc.run(st, None, osl, 5, 3600.0, cgspec=orc.CgSpec(precond=0, stop_rule=1, rtol=1e-13, atol=0.0))
    assert_fields_close(s, st, tol=1e-8)


def test_checkpoint_restart_continues_the_run(shk, orc, cuda, tmp_path):
    """run! with checkpoint_every writes the full State and total_time (keys as the reference's:
    "t", "total_time", one per State field); a fresh Simulation restarted from the step-3 checkpoint
    and run to step 6 ends bit-identical to the uninterrupted six steps (src/run.jl:21-63,
    src/checkpoint.jl:26-64)."""
    w = shk.configs.plain64()

    def make(tsteps):
        g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w)
        ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem)
        ps = shk.PicardSolver(500, 1e-6, ls, g)
        return shk.Simulation(g, s, tsteps, 3600.0, pm, "implicit", [], shk.ConstantMeltInput(), sl, ps=ps)

    with pytest.raises(ValueError):
        shk.run(make(1), checkpoint_every=2)
    full = make(6)
    ck = str(tmp_path / "ck.npz")
    shk.run(full, checkpoint_every=3, checkpoint_path=ck)
    with np.load(ck) as f:
        assert int(f["t"]) == 6 and float(f["total_time"]) == 6 * 3600.0
        assert {("lambda" if n == "lambda_" else n) for n in shk._lib.STATE_FIELDS} <= set(f.files)
    part = make(3)
    ck3 = str(tmp_path / "ck3.npz")
    shk.run(part, checkpoint_every=3, checkpoint_path=ck3)
    resumed = make(6)
    shk.run(resumed, restart_path=ck3)
    assert resumed.total_time == full.total_time
    a, b = resumed.state.to_numpy(), full.state.to_numpy()
    for f in shk._lib.STATE_FIELDS:
        assert np.array_equal(a[f], b[f]), f
