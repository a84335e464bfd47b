"""Per-field error of the chosen form (Float64 CG preconditioned by the Float32 multigrid V-cycle,
rel-res 1e-8 on the GROUNDED rows) against a tight Float64 run of the oracle (the CPU restatement
of the reference algorithm, Jacobi CG to rel-res 1e-13), on the mixed-precision workload's physics
at 1024^2 (seasonal melt, 64 moulins, LAND/OTHER_BASIN blobs; the 4096^2 cell size).

The bar is the tolerance ball: the chosen form's distance from the tight run, per field (h, N, b,
q), is at most ten times the distance of the oracle's own rel-res 1e-8 run from the tight run.
The errors are printed and, when SHK_REPORT_DIR is set, written there as JSON."""
import json
import os

import numpy as np
import pytest

from test_gpu_parity import relerr

pytestmark = pytest.mark.gpu

STEPS = 3
FIELDS = ("h", "N", "b", "q_x", "q_y")


def oracle_run(shk, orc, w, rtol):
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    osl = orc.SlidingSpec(kind=0, C=w.sliding_C)
    orc.set_initial_conditions(st, w.params, osl, w.inputs)
    spec = orc.CgSpec(precond=0, stop_rule=1, rtol=rtol, atol=0.0)
    _, _, stats = orc.run(st, w.params, osl, STEPS, 1800.0, cgspec=spec, melt=orc.seasonal_melt(w.melt))
    assert all(s["converged"] for s in stats), stats
    return st


def field_err(a, b, f):
    if f in ("q_x", "q_y"):  # the two flux components share one scale
        scale = max(float(np.max(np.abs(b["q_x"]))), float(np.max(np.abs(b["q_y"]))))
        return float(np.max(np.abs(a[f] - b[f]))) / scale
    return relerr(a[f], b[f])


def test_chosen_form_field_errors_seasonal1024(shk, orc, cuda):
    w = shk.configs.seasonal1024()
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    p = shk.ModelParameters(**w.params)
    sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
    s = shk.State(g)
    shk.set_initial_conditions(s, g, p, sl, **w.inputs)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, multigrid=True, stop_rule="relres", rtol=1e-8,
                               atol=0.0)
    ps = shk.PicardSolver(500, 1e-6, ls, g)
    sim = shk.Simulation(g, s, STEPS, 1800.0, p, "implicit", [], shk.SeasonalBaseMeltInput(**w.melt), sl, ps=ps)
    shk.run(sim)
    assert all(x["converged"] for x in sim.step_stats), sim.step_stats
    gpu = s.to_numpy(list(FIELDS))
    tight = oracle_run(shk, orc, w, 1e-13)
    ball = oracle_run(shk, orc, w, 1e-8)
    report = {}
    for f in FIELDS:
        e_chosen = field_err(gpu, tight.fields, f)
        e_ball = field_err(ball.fields, tight.fields, f)
        report[f] = {"chosen_vs_tight": e_chosen, "oracle_1e-8_vs_tight": e_ball}
    print("field errors after", STEPS, "steps:", json.dumps(report))
    if os.environ.get("SHK_REPORT_DIR"):
        with open(os.path.join(os.environ["SHK_REPORT_DIR"], "field_errors_seasonal1024.json"), "w") as fh:
            json.dump({"workload": w.name, "steps": STEPS, "picard_per_step": [x["last_iter"] for x in sim.step_stats],
                       "errors": report}, fh, indent=1)
    for f, r in report.items():
        assert r["chosen_vs_tight"] <= 10 * r["oracle_1e-8_vs_tight"] + 1e-12, (f, r)
