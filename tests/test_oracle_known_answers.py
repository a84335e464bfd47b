"""Known answers for the oracle, computed without it.

Every formula below is written straight from the reference's kernels, cell by cell in plain Python
floats (IEEE Float64, evaluated in Julia's left-to-right order, integer powers as Julia computes
them), and never calls the C restatement.  The C restatement's outputs on the same hand-perturbed
states must agree bit for bit.  This pins the oracle's arithmetic independently of its own code:
the SALS == MFLS and CG == direct-solve properties of the reference's test suite cannot catch a
wrong coefficient that both sides of those comparisons share.

Reference lines restated here:
  src/field_gradients.jl:95-127   dhdx/dhdy, dpwdx/dpwdy
  src/pressure.jl:1-33            pw, N
  src/water_flux.jl:107-119,192-234  Re (centre), q/Re quadratic, K
  src/sliding_law.jl:213-256      regularized-Coulomb basal stress
  src/melt_rate.jl:106-168        shear, potential, sensible heat, mdot
  src/linear_solver.jl:13-27,438-501  dirichlet_head, MFLS assembly
  src/k_face_scheme.jl:32-61      k-face schemes
  src/gap_height.jl:47-135, src/run.jl:154-164  gap update, beta, b faces
"""
import math

import numpy as np
import pytest

GROUNDED, OCEAN, LAND, OTHER_BASIN = 0.0, 1.0, 2.0, 3.0
EPS = np.finfo(np.float64).eps


def powi(x, n):
    """Julia's Float64 ^ Integer for the exponents used here: x^3 = x*x*x, x^2 = fl(x*x)."""
    if n == 3:
        return x * x * x
    if n == 2:
        return x * x
    if n == 1:
        return x
    raise ValueError(n)


def jsign(x):
    return 1.0 if x > 0 else (-1.0 if x < 0 else x)


def boolmul(flag, y):
    """Julia Bool * Float64: true*y = y, false*y = +-0 with y's sign."""
    return y if flag else math.copysign(0.0, y)


def params(**kw):
    p = dict(rho_w=1000.0, rho_sw=1027.0, rho_i=910.0, g=9.81, nu=1.787e-6, n=3.0, omega=1e-4, L=334e3,
             br=0.05, lr=2.0, ct=7.5e-8, cw=4.22e3, p_atm=0.0, b_min=0.0, b_max=math.inf, e_v=0.0)
    p.update(kw)
    return p


# ---------------------------------------------------------------------------------------------
# The field-update tail (Picard_iteration! after the solve)
# ---------------------------------------------------------------------------------------------
def ka_tail(f, p, C, dx, dy):
    """dhdxy, pw, dpwdxy, N, q/Re (faces), Re (centres), taub (regularized Coulomb), mdot, K."""
    nx, ny = f["h"].shape
    h, zb, po, mask = f["h"], f["zb"], f["po"], f["mask"]
    out = {k: f[k].copy() for k in ("dhdx", "dhdy", "dpwdx", "dpwdy", "q_x", "q_y", "Re_x", "Re_y", "taub_x",
                                    "taub_y")}
    pw = np.zeros((nx, ny), order="F")
    N = np.zeros((nx, ny), order="F")
    for j in range(ny):
        for i in range(nx):
            pw[i, j] = p["rho_w"] * p["g"] * (h[i, j] - zb[i, j])
            N[i, j] = boolmul(mask[i, j] == GROUNDED, po[i, j] - pw[i, j])
    # interior faces only (1-based 2..nx for x, 2..ny for y); edge faces keep their values
    for j in range(ny):
        for i in range(1, nx):
            out["dhdx"][i, j] = ((h[i, j] - h[i - 1, j]) / dx) * f["valid_x"][i, j]
            out["dpwdx"][i, j] = ((pw[i, j] - pw[i - 1, j]) / dx) * f["valid_x"][i, j]
    for j in range(1, ny):
        for i in range(nx):
            out["dhdy"][i, j] = ((h[i, j] - h[i, j - 1]) / dy) * f["valid_y"][i, j]
            out["dpwdy"][i, j] = ((pw[i, j] - pw[i, j - 1]) / dy) * f["valid_y"][i, j]

    def q_re(bf, grad):
        G = abs(grad)
        D = (powi(bf, 3) * p["g"] * G) / (12 * powi(p["nu"], 2))
        Re = 2 * D / (1 + math.sqrt(1 + 4 * p["omega"] * D))
        return -jsign(grad) * p["nu"] * Re, Re

    for j in range(ny):
        for i in range(nx + 1):
            out["q_x"][i, j], out["Re_x"][i, j] = q_re(f["b_x"][i, j], out["dhdx"][i, j])
    for j in range(ny + 1):
        for i in range(nx):
            out["q_y"][i, j], out["Re_y"][i, j] = q_re(f["b_y"][i, j], out["dhdy"][i, j])
    Re = np.zeros((nx, ny), order="F")
    for j in range(ny):
        for i in range(nx):
            Re[i, j] = (out["Re_x"][i, j] + out["Re_x"][i + 1, j] + out["Re_y"][i, j] + out["Re_y"][i, j + 1]) / 4

    n_exp, inv_n = int(p["n"]), 1 / p["n"]
    lam, aub = f["lambda_"], f["abs_ub"]

    def taub(Nf, lf, abs_v, ub):
        if not abs_v > 0:
            return 0.0
        return Nf * C * math.pow(abs_v / (abs_v + powi(abs(Nf), n_exp) * lf), inv_n) * (ub / abs_v)

    for j in range(ny):
        for i in range(nx + 1):
            if i == 0:
                out["taub_x"][i, j] = taub(N[0, j], lam[0, j], aub[0, j], f["ub_x"][0, j])
            elif i == nx:
                out["taub_x"][i, j] = taub(N[nx - 1, j], lam[nx - 1, j], aub[nx - 1, j], f["ub_x"][nx, j])
            else:
                out["taub_x"][i, j] = taub((N[i, j] + N[i - 1, j]) / 2, (lam[i, j] + lam[i - 1, j]) / 2,
                                           (aub[i, j] + aub[i - 1, j]) / 2, f["ub_x"][i, j])
    for j in range(ny + 1):
        for i in range(nx):
            if j == 0:
                out["taub_y"][i, j] = taub(N[i, 0], lam[i, 0], aub[i, 0], f["ub_y"][i, 0])
            elif j == ny:
                out["taub_y"][i, j] = taub(N[i, ny - 1], lam[i, ny - 1], aub[i, ny - 1], f["ub_y"][i, ny])
            else:
                out["taub_y"][i, j] = taub((N[i, j] + N[i, j - 1]) / 2, (lam[i, j] + lam[i, j - 1]) / 2,
                                           (aub[i, j] + aub[i, j - 1]) / 2, f["ub_y"][i, j])

    shear, pot, sens, mdot, K = (np.zeros((nx, ny), order="F") for _ in range(5))
    ux, tx, uy, ty = f["ub_x"], out["taub_x"], f["ub_y"], out["taub_y"]
    qx, qy, gx, gy, px, py = out["q_x"], out["q_y"], out["dhdx"], out["dhdy"], out["dpwdx"], out["dpwdy"]
    Linv = 1 / p["L"]
    for j in range(ny):
        for i in range(nx):
            sh = abs((ux[i + 1, j] * tx[i + 1, j] + ux[i, j] * tx[i, j]) / 2 +
                     (uy[i, j + 1] * ty[i, j + 1] + uy[i, j] * ty[i, j]) / 2)
            pt = abs((qx[i + 1, j] * gx[i + 1, j] + qx[i, j] * gx[i, j]) / 2 +
                     (qy[i, j + 1] * gy[i, j + 1] + qy[i, j] * gy[i, j]) / 2)
            se = (qx[i + 1, j] * px[i + 1, j] + qx[i, j] * px[i, j]) / 2 + \
                 (qy[i, j + 1] * py[i, j + 1] + qy[i, j] * py[i, j]) / 2
            shear[i, j], pot[i, j], sens[i, j] = sh, pt, se
            mdot[i, j] = Linv * (f["G"][i, j] + sh + p["rho_w"] * p["g"] * pt + p["ct"] * p["cw"] * p["rho_w"] * se)
            K[i, j] = (powi(f["b"][i, j], 3) * p["g"]) / (12 * p["nu"] * (1 + p["omega"] * Re[i, j]))
    out.update(pw=pw, N=N, Re=Re, shear=shear, potential=pot, sensible=sens, mdot=mdot, K=K)
    return out


# ---------------------------------------------------------------------------------------------
# MFLS assembly (update_MFLS_kernel!)
# ---------------------------------------------------------------------------------------------
def dirichlet_head(m, zb, p):
    if m == OCEAN:
        pw_bc = p["p_atm"] - p["rho_sw"] * p["g"] * min(zb, 0.0)
        return pw_bc / (p["rho_w"] * p["g"]) + zb
    return p["p_atm"] / (p["rho_w"] * p["g"]) + zb


def ka_assemble(f, p, kfs, dx2, dy2):
    nx, ny = f["h"].shape
    A = {k: np.zeros((nx, ny), order="F") for k in ("aP", "aE", "aW", "aN", "aS", "rhs")}
    mask, K = f["mask"], f["K"]

    def kface(i1, j1, i2, j2):
        m2 = mask[i2, j2]
        if m2 == OTHER_BASIN:
            return 0.0
        if m2 in (OCEAN, LAND):
            return K[i1, j1]
        if kfs == 0:
            return (K[i1, j1] + K[i2, j2]) / 2
        return (2 * K[i1, j1] * K[i2, j2]) / (K[i1, j1] + K[i2, j2] + EPS)

    n, nm1 = p["n"], int(p["n"] - 1)
    for j in range(ny):
        for i in range(nx):
            m = mask[i, j]
            if m in (OCEAN, LAND):
                A["aP"][i, j] = 1.0
                A["rhs"][i, j] = dirichlet_head(m, f["zb"][i, j], p)
                continue
            if m == OTHER_BASIN:
                A["aP"][i, j] = 1.0
                A["rhs"][i, j] = f["h"][i, j]
                continue
            aE = kface(i, j, i + 1, j) / dx2 if i < nx - 1 else 0.0
            aW = kface(i, j, i - 1, j) / dx2 if i > 0 else 0.0
            aN = kface(i, j, i, j + 1) / dy2 if j < ny - 1 else 0.0
            aS = kface(i, j, i, j - 1) / dy2 if j > 0 else 0.0
            Aij, Nij, bij = f["A_visc"][i, j], f["N"][i, j], f["b"][i, j]
            A["aP"][i, j] = (aE + aW + aN + aS) + n * p["rho_w"] * p["g"] * Aij * powi(abs(Nij), nm1) * bij
            drhs = 0.0
            for (a, key, ii, jj, ok) in ((aE, "aE", i + 1, j, i < nx - 1), (aW, "aW", i - 1, j, i > 0),
                                         (aN, "aN", i, j + 1, j < ny - 1), (aS, "aS", i, j - 1, j > 0)):
                if not ok:
                    continue
                mn = mask[ii, jj]
                if mn in (OCEAN, LAND):
                    drhs += a * dirichlet_head(mn, f["zb"][ii, jj], p)
                else:
                    A[key][i, j] = a
            A["rhs"][i, j] = (f["mdot"][i, j] * (1 / p["rho_w"] - 1 / p["rho_i"]) -
                              f["beta"][i, j] * f["abs_ub"][i, j] +
                              Aij * powi(abs(Nij), nm1) * Nij * bij +
                              Aij * powi(abs(Nij), nm1) * (n * p["rho_w"] * p["g"] * f["h"][i, j]) * bij +
                              f["ieb"][i, j] + drhs)
    return A


# ---------------------------------------------------------------------------------------------
# step_b!: gap update, beta, b faces
# ---------------------------------------------------------------------------------------------
def ka_step_b(f, p, implicit, dt):
    nx, ny = f["b"].shape
    b = f["b"].copy(order="F")
    nm1 = int(p["n"] - 1)
    for j in range(ny):
        for i in range(nx):
            if f["mask"][i, j] != GROUNDED:
                continue
            A, N = f["A_visc"][i, j], f["N"][i, j]
            if implicit:
                v = (b[i, j] + dt * (f["mdot"][i, j] / p["rho_i"] + f["beta"][i, j] * f["abs_ub"][i, j])) / \
                    (1 + dt * A * powi(abs(N), nm1) * N)
            else:
                v = b[i, j] + dt * (f["mdot"][i, j] / p["rho_i"] + f["beta"][i, j] * f["abs_ub"][i, j] -
                                    A * powi(abs(N), nm1) * N * b[i, j])
            b[i, j] = min(max(v, p["b_min"]), p["b_max"]) if not math.isnan(v) else v
    beta = f["beta"].copy(order="F")
    if p["br"] != 0:
        for j in range(ny):
            for i in range(nx):
                beta[i, j] = max(0.0, (p["br"] - b[i, j]) / p["lr"])
    b_x = np.zeros((nx + 1, ny), order="F")
    b_y = np.zeros((nx, ny + 1), order="F")
    for j in range(ny):
        b_x[0, j], b_x[nx, j] = b[0, j], b[nx - 1, j]
        for i in range(1, nx):
            b_x[i, j] = (b[i, j] + b[i - 1, j]) / 2
    for i in range(nx):
        b_y[i, 0], b_y[i, ny] = b[i, 0], b[i, ny - 1]
        for j in range(1, ny):
            b_y[i, j] = (b[i, j] + b[i, j - 1]) / 2
    return dict(b=b, beta=beta, b_x=b_x, b_y=b_y)


# ---------------------------------------------------------------------------------------------
# States and comparisons
# ---------------------------------------------------------------------------------------------
def perturbed_states(shk, orc):
    """(name, oracle state, params, C): the reference fixture with its head, gap and velocity
    perturbed by hand, and a 9x7 grid whose mask puts OCEAN, LAND and OTHER_BASIN cells on every
    side of some GROUNDED cell, at two parameter sets (default; p_atm, gap clamps)."""
    out = []
    w = shk.configs.fixture6()
    for pname, pkw in (("default", {}), ("patm_clamped", dict(p_atm=101325.0, b_min=0.004, b_max=0.0105))):
        st = orc.OracleState(w.nx, w.ny, w.lx, w.ly)
        osl = orc.SlidingSpec(kind=0, C=w.sliding_C)
        orc.set_initial_conditions(st, pkw, osl, w.inputs)
        ii, jj = np.meshgrid(np.arange(w.nx), np.arange(w.ny), indexing="ij")
        st["h"][...] += 3.0 * np.sin(0.9 * ii + 0.4 * jj) + 0.25 * jj
        st["b"][...] *= 1.0 + 0.3 * np.cos(1.3 * ii - 0.7 * jj)
        st["ub_x"][...] *= 1.0 + 0.5 * np.sin(np.arange(w.nx + 1))[:, None]
        st["ub_y"][...] = 2e-7 * np.cos(np.arange(w.ny + 1))[None, :]
        orc.compute(st, "abs_ub")
        orc.compute(st, "b_xy")
        orc.compute(st, "beta", pkw)
        out.append((f"fixture6/{pname}", st, pkw, w.sliding_C))
    # a ragged grid with boundary cells of every kind next to GROUNDED cells
    nx, ny = 9, 7
    rng = np.random.default_rng(7)
    mask = np.full((nx, ny), GROUNDED, order="F")
    mask[0, :] = OCEAN
    mask[4, 0] = LAND
    mask[6, 3] = OTHER_BASIN
    mask[3, 5] = LAND
    mask[7, 6] = OCEAN
    mask[2, 2] = OTHER_BASIN
    zb = np.asfortranarray(rng.normal(5.0, 40.0, (nx, ny)))
    inputs = dict(mask=mask, A_visc=np.full((nx, ny), 5e-25, order="F"), zb=zb,
                  zs=np.asfortranarray(zb + 300.0 + rng.uniform(0, 200.0, (nx, ny))),
                  b=np.asfortranarray(rng.uniform(0.002, 0.02, (nx, ny))),
                  G=np.asfortranarray(rng.uniform(0.04, 0.07, (nx, ny))),
                  ub_x=np.asfortranarray(rng.uniform(-1e-6, 2e-6, (nx + 1, ny))),
                  ub_y=np.asfortranarray(rng.uniform(-1e-6, 1e-6, (nx, ny + 1))),
                  ieb=np.asfortranarray(rng.uniform(0, 1e-7, (nx, ny))),
                  taub_x=np.zeros((nx + 1, ny), order="F"), taub_y=np.zeros((nx, ny + 1), order="F"))
    for pname, pkw in (("default", {}), ("patm_clamped", dict(p_atm=101325.0, b_min=0.004, b_max=0.015))):
        st = orc.OracleState(nx, ny, 4e3, 3e3)
        osl = orc.SlidingSpec(kind=0, C=0.3)
        orc.set_initial_conditions(st, pkw, osl, inputs)
        st["h"][...] += rng.normal(0.0, 20.0, (nx, ny))
        out.append((f"ragged9x7/{pname}", st, pkw, 0.3))
    return out


def fields_of(st):
    return {k: st[k].copy(order="F") for k in st.fields}


def assert_bitwise(name, got, want, keys):
    bad = [(k, float(np.max(np.abs(got[k] - want[k])))) for k in keys if not np.array_equal(got[k], want[k])]
    assert not bad, f"{name}: {bad}"


def test_tail_known_answers(orc, shk):
    for name, st, pkw, C in perturbed_states(shk, orc):
        want = ka_tail(fields_of(st), params(**pkw), C, st.dx, st.dy)
        orc.picard_tail(st, pkw, orc.SlidingSpec(kind=0, C=C))
        assert_bitwise(name, fields_of(st), want, sorted(want))


@pytest.mark.parametrize("kfs", [0, 1])
def test_assembly_known_answers(orc, shk, kfs):
    for name, st, pkw, C in perturbed_states(shk, orc):
        orc.picard_tail(st, pkw, orc.SlidingSpec(kind=0, C=C))
        want = ka_assemble(fields_of(st), params(**pkw), kfs, st.dx * st.dx, st.dy * st.dy)
        got = orc.assemble(st, pkw, kfs=kfs)
        assert_bitwise(f"{name}/kfs{kfs}", got, want, ("aP", "aE", "aW", "aN", "aS", "rhs"))
        # an OCEAN/LAND neighbour folds its head into rhs and leaves the coupling at zero
        assert np.any(got["rhs"][st["mask"] == GROUNDED] != 0)


@pytest.mark.parametrize("implicit", [True, False])
def test_gap_step_known_answers(orc, shk, implicit):
    for name, st, pkw, C in perturbed_states(shk, orc):
        orc.picard_tail(st, pkw, orc.SlidingSpec(kind=0, C=C))
        want = ka_step_b(fields_of(st), params(**pkw), implicit, 1800.0)
        orc.step_b(st, pkw, 1 if implicit else 0, 1800.0)
        assert_bitwise(f"{name}/{'implicit' if implicit else 'explicit'}", fields_of(st), want, sorted(want))


def test_reynolds_quadratic_solves_the_flux_law():
    """Re = 2D / (1 + sqrt(1 + 4 omega D)) is the positive root of omega Re^2 + Re - D = 0
    (src/water_flux.jl:123-152), so q = -sign(dh) nu Re satisfies the turbulent flux law
    q = -b^3 g dh / (12 nu (1 + omega |q|/nu)) at the fixed point."""
    p = params()
    for b, dh in ((0.01, 2e-3), (0.3, -5e-2), (1e-3, 1e-6)):
        qs, Re = None, None
        G = abs(dh)
        D = (powi(b, 3) * p["g"] * G) / (12 * powi(p["nu"], 2))
        Re = 2 * D / (1 + math.sqrt(1 + 4 * p["omega"] * D))
        qs = -jsign(dh) * p["nu"] * Re
        assert abs(p["omega"] * Re * Re + Re - D) <= 1e-12 * D
        law = -(b ** 3) * p["g"] * dh / (12 * p["nu"] * (1 + p["omega"] * abs(qs) / p["nu"]))
        assert qs == pytest.approx(law, rel=1e-12)
