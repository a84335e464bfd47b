"""The reference's own test suite, ported onto the CPU restatement (the oracle).

These pin the oracle: every fixture and known-answer property of test/linear_solver_test.jl,
test/parabolic_solver_test.jl and test/sliding_law_test.jl that concerns the head-solve path.
CholeskyDirectSolver is stood in for by a SciPy sparse direct solve.
"""
import math

import numpy as np
import pytest

EPS = np.finfo(np.float64).eps


def isapprox(a, b, rtol=math.sqrt(EPS), atol=0.0):
    """Julia's isapprox for arrays: norm(a-b) <= max(atol, rtol*max(norm(a), norm(b)))."""
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return np.linalg.norm(a - b) <= max(atol, rtol * max(np.linalg.norm(a), np.linalg.norm(b)))


def fresh_state(orc, shk, perturb=True, sl=None, p=None):
    """fixture + the perturb-and-refresh sequence of test/linear_solver_test.jl:38-54."""
    w = shk.configs.fixture6()
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    sl = sl or orc.SlidingSpec(kind=0, C=w.sliding_C)
    orc.set_initial_conditions(st, p, sl, w.inputs)
    if perturb:
        st["h"][...] += 0.01 * np.arange(1, w.nx * w.ny + 1).reshape((w.nx, w.ny), order="F")
        orc.compute(st, "dhdxy")
        orc.compute(st, "pw", p)
        orc.compute(st, "dpwdxy")
        orc.compute(st, "N")
        orc.compute(st, "q_xy_lagged", p)
        orc.compute(st, "Re_xy_lagged", p)
        orc.compute(st, "Re")
        orc.compute(st, "taub_xy", p, sl)
        orc.compute(st, "mdot", p)
        orc.compute(st, "K", p)
    return w, st


def test_fixture_matches_reference_test_block(shk):
    """test/linear_solver_test.jl:8-32: 6x6, 1 km, all four mask kinds, moulin at (3,3)."""
    w = shk.configs.fixture6()
    m = w.inputs["mask"]
    assert (m[-1, 1:] == 1.0).all() and (m[0, 1:] == 2.0).all() and (m[:, 0] == 3.0).all()
    assert (m[1:-1, 1:] == 0.0).all()
    assert w.inputs["ieb"][2, 2] == 3 / (200.0 * 200.0)
    assert np.allclose(w.inputs["zb"][:, 0], -0.02 * np.arange(6) * 200.0)


def test_mfls_agrees_with_sals_and_is_symmetric(orc, shk):
    """test/linear_solver_test.jl:1-83"""
    _, st = fresh_state(orc, shk)
    mf = orc.assemble(st, None, kfs=0)
    sa = orc.assemble(st, None, kfs=0, sals=True)
    assert isapprox(sa["rhs"], mf["rhs"])
    M = orc.sparse_matrix({"aP": sa["aP"], "aE": -sa["aE"], "aW": -sa["aW"], "aN": -sa["aN"], "aS": -sa["aS"],
                           "rhs": sa["rhs"]})
    assert abs(M - M.T).max() == 0.0  # issymmetric(sals.M)
    nx, ny = mf["aP"].shape
    for j in range(ny):
        for i in range(nx):
            assert isapprox(sa["aP"][i, j], mf["aP"][i, j])
            if i < nx - 1:
                assert isapprox(sa["aE"][i, j], -mf["aE"][i, j])
            if i > 0:
                assert isapprox(sa["aW"][i, j], -mf["aW"][i, j])
            if j < ny - 1:
                assert isapprox(sa["aN"][i, j], -mf["aN"][i, j])
            if j > 0:
                assert isapprox(sa["aS"][i, j], -mf["aS"][i, j])


def test_mfls_bitwise_symmetric_couplings(orc, shk):
    """aW(i,j) == aE(i-1,j) and aS(i,j) == aN(i,j-1) exactly, for both k-face schemes: the
    property the CUDA library's 3-array storage relies on."""
    for kfs in (0, 1):
        _, st = fresh_state(orc, shk)
        A = orc.assemble(st, None, kfs=kfs)
        assert (A["aW"][1:, :] == A["aE"][:-1, :]).all() and (A["aW"][0, :] == 0).all()
        assert (A["aS"][:, 1:] == A["aN"][:, :-1]).all() and (A["aS"][:, 0] == 0).all()


@pytest.mark.parametrize("kfs", [0, 1])
def test_cg_matches_direct(orc, shk, kfs):
    """test/linear_solver_test.jl:105-199: MFLS-CG Jacobi and Chebyshev(4) match the direct solve
    (reference tolerance atol 1e-5; here also 1e-10 at a tight CG tolerance), and Chebyshev needs
    no more CG iterations than Jacobi."""
    _, st = fresh_state(orc, shk)
    A = orc.assemble(st, None, kfs=kfs)
    h_direct = orc.direct_solve(A)
    x_j, sj = orc.cg(A, st["h"], orc.CgSpec(precond=0))
    x_c, sc = orc.cg(A, st["h"], orc.CgSpec(precond=1, cheb_degree=4))
    assert np.max(np.abs(x_j - h_direct)) <= 1e-5
    assert np.max(np.abs(x_c - h_direct)) <= 1e-5
    assert sc["niter"] <= sj["niter"]
    x_t, _ = orc.cg(A, st["h"], orc.CgSpec(precond=0, atol=0.0, rtol=1e-14))
    assert np.max(np.abs(x_t - h_direct)) / np.max(np.abs(h_direct)) <= 1e-10


def test_chebyshev_invalid_estimate_keeps_placeholder(orc):
    """test/linear_solver_test.jl:218-242: tridiagonal(4,-1) of size 36 with d = 4 and an all-zero
    rhs; the estimate is NaN and the (1,1) placeholder bounds survive."""
    n = 36
    A = {k: np.zeros((n, 1), order="F") for k in ("aP", "aE", "aW", "aN", "aS", "rhs")}
    A["aP"][:] = 4.0
    A["aE"][:-1] = 1.0  # matvec applies the minus sign
    A["aW"][1:] = 1.0
    cheb = orc._ChebState(1.0, 1.0, 0)
    assert cheb.lambda_min == 1.0 and cheb.lambda_max == 1.0
    ok, est = orc.update_chebyshev_bounds(A, np.zeros((n, 1), order="F"), 15, cheb)
    assert not ok and math.isnan(est[0]) and math.isnan(est[1])
    assert cheb.lambda_min == 1.0 and cheb.lambda_max == 1.0


def test_chebyshev_estimate_brackets_spectrum(orc, shk):
    """The Lanczos-from-CG bounds (shrunk/grown by 0.9/1.1) bracket D^-1 A's extreme eigenvalues
    on a well-conditioned system (src/preconditioner.jl:127-131)."""
    _, st = fresh_state(orc, shk)
    A = orc.assemble(st, None)
    M = orc.sparse_matrix(A).toarray()
    ev = np.linalg.eigvals(np.diag(1 / A["aP"].ravel(order="F")) @ M).real
    cheb = orc._ChebState(1.0, 1.0, 0)
    ok, est = orc.update_chebyshev_bounds(A, A["rhs"], 15, cheb)
    assert ok
    assert est[0] <= ev.min() * (1 + 1e-8) and est[1] >= ev.max() * (1 - 1e-8)


def test_parabolic_step_moves_h_and_stays_finite(orc, shk):
    """test/parabolic_solver_test.jl:37-55"""
    p = dict(e_v=1e-3)
    w, st = fresh_state(orc, shk, perturb=False, p=p)
    h0 = st["h"].copy()
    orc.parabolic_step(st, p, orc.SlidingSpec(kind=0, C=0.25), 0, orc.CgSpec(precond=0, atol=0, rtol=1e-13), 60.0)
    assert not isapprox(st["h"], h0)
    for k in ("h", "N", "Re", "mdot", "K"):
        assert np.isfinite(st[k]).all()


def test_parabolic_steady_state_matches_elliptic(orc, shk):
    """test/parabolic_solver_test.jl:57-87: 1000 steps of dt = 3600 with b_min = 1e-3; steady h and
    b of both head schemes agree to rtol 1e-4 (direct solves stood in for by tight CG)."""
    sl = orc.SlidingSpec(kind=0, C=0.25)
    pe, pp = dict(e_v=0.0, b_min=1e-3), dict(e_v=1e-3, b_min=1e-3)
    _, se = fresh_state(orc, shk, perturb=False, p=pe)
    _, sp = fresh_state(orc, shk, perturb=False, p=pp)
    cg = orc.CgSpec(precond=0, atol=0.0, rtol=1e-13)
    orc.run(se, pe, sl, 1000, 3600.0, cgspec=cg)
    orc.run(sp, pp, sl, 1000, 3600.0, cgspec=cg)
    assert isapprox(se["h"], sp["h"], rtol=1e-4)
    assert isapprox(se["b"], sp["b"], rtol=1e-4)


def test_linear_sliding_law_scalar(orc, shk):
    """test/sliding_law_test.jl:25-44: uniform C staggers to C^2 and taub_x = C^2 N_f ub_x."""
    w = shk.configs.fixture6()
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    C = 0.25
    lin = shk.LinearSlidingLaw(g, C)
    assert np.allclose(lin.Cx2, C ** 2) and np.allclose(lin.Cy2, C ** 2)
    sl = orc.SlidingSpec(kind=3, Cx=lin.Cx2, Cy=lin.Cy2)
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    orc.set_initial_conditions(st, None, sl, w.inputs)
    for j in range(w.ny):
        for i in range(1, w.nx):
            Nf = (st["N"][i, j] + st["N"][i - 1, j]) / 2
            assert np.isclose(st["taub_x"][i, j], C ** 2 * Nf * st["ub_x"][i, j], rtol=math.sqrt(EPS), atol=0)
    assert np.isfinite(st["taub_x"]).all() and np.isfinite(st["taub_y"]).all()


def test_linear_sliding_law_spatial_staggering(shk):
    """test/sliding_law_test.jl:46-63"""
    w = shk.configs.fixture6()
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    nx, ny = w.nx, w.ny
    C = np.array([[0.1 + 0.01 * (i + 1) + 0.02 * (j + 1) for j in range(ny)] for i in range(nx)])
    lin = shk.LinearSlidingLaw(g, C)
    for j in range(ny):
        for i in range(1, nx):
            assert np.isclose(lin.Cx2[i, j], ((C[i - 1, j] + C[i, j]) / 2) ** 2)
    assert np.allclose(lin.Cx2[0, :], C[0, :] ** 2) and np.allclose(lin.Cx2[nx, :], C[nx - 1, :] ** 2)


def test_linear_sliding_law_picard_converges(orc, shk):
    """test/sliding_law_test.jl:65-77"""
    w = shk.configs.fixture6()
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    lin = shk.LinearSlidingLaw(g, 0.25)
    sl = orc.SlidingSpec(kind=3, Cx=lin.Cx2, Cy=lin.Cy2)
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    orc.set_initial_conditions(st, None, sl, w.inputs)
    res = orc.picard_loop(st, None, sl, 0, orc.CgSpec(precond=0, atol=0.0, rtol=1e-13))
    assert res["converged"]
    assert np.isfinite(st["h"]).all() and np.isfinite(st["N"]).all()


def test_initial_conditions_follow_reference_sequence(orc, shk):
    """set_initial_conditions! (src/initial_conditions.jl:14-125) spot checks on the fixture."""
    w = shk.configs.fixture6()
    st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
    orc.set_initial_conditions(st, None, orc.SlidingSpec(kind=0, C=0.25), w.inputs)
    m = st["mask"]
    assert (st["b"][m != 0.0] == 0.0).all() and (st["b"][m == 0.0] == 0.01).all()
    assert np.array_equal(st["lambda"], 1.5 * st["A_visc"])
    # OCEAN pw = p_atm - rho_sw g min(zb, 0); LAND/OTHER pw = p_atm; GROUNDED pw = po/2
    ocean = m == 1.0
    assert np.array_equal(st["pw"][ocean], 0.0 - 1027.0 * 9.81 * np.minimum(st["zb"][ocean], 0.0))
    assert (st["pw"][(m == 2.0) | (m == 3.0)] == 0.0).all()
    assert np.array_equal(st["pw"][m == 0.0], st["po"][m == 0.0] / 2)
    assert (st["N"][m != 0.0] == 0.0).all()
    # valid faces: interior faces touching OTHER_BASIN invalid, edges 1
    assert (st["valid_y"][:, 1] == 0.0).all() and (st["valid_y"][:, 0] == 1.0).all()
    # ub masked on boundary faces and faces not GROUNDED on both sides
    assert (st["ub_x"][0, :] == 0).all() and (st["ub_x"][-1, :] == 0).all()
    assert (st["ub_x"][2:5, 1:] == 1e-6).all() and (st["ub_x"][:, 0] == 0).all()
    # gradient edge faces never written
    assert (st["dhdx"][0, :] == 0).all() and (st["dhdx"][-1, :] == 0).all()
    for k in ("h", "q_x", "q_y", "Re", "taub_x", "taub_y", "mdot", "K"):
        assert np.isfinite(st[k]).all()
