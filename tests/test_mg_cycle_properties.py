"""Properties of the multigrid preconditioner's cycle under the library's default smoothing weights,
checked on a NumPy restatement of the cycle (2x2 aggregation, Laplacian-form coarse operators,
identity rows not aggregated, two weighted Jacobi sweeps per side, scaled coarse correction, exact
1x1 solve).  CG needs a symmetric positive definite preconditioner: the cycle applied to the unit
vectors of a small random operator gives an explicit matrix that must be symmetric and have only
positive eigenvalues, for damped Jacobi (0.8, scaling 1.6) and for the degree-2 Chebyshev pair
(scalings 1.45 and 1.3).  The pair's weights are the reciprocals of the roots of the degree-2
Chebyshev polynomial on [0.45, 1.8], as the library computes them.
"""
import numpy as np
import pytest


def chebyshev_pair(lo=0.45, hi=1.8):
    mid, half = 0.5 * (hi + lo), 0.5 * (hi - lo) * np.sqrt(0.5)
    return 1.0 / (mid + half), 1.0 / (mid - half)


class Level:
    """Laplacian-form operator (A x)_i = dP_i x_i + sum_j a_ij (x_i - x_j) on an ny x nx grid."""

    def __init__(self, dP, aE, aN, act):
        self.dP, self.act = dP, act
        self.aE, self.aN = aE.copy(), aN.copy()
        self.aE[:, -1] = 0.0
        self.aN[-1, :] = 0.0
        aW = np.zeros_like(aE); aW[:, 1:] = self.aE[:, :-1]
        aS = np.zeros_like(aN); aS[1:, :] = self.aN[:-1, :]
        self.aW, self.aS = aW, aS
        self.diag = dP + self.aE + aW + self.aN + aS

    def A(self, x):
        y = self.dP * x
        y[:, :-1] += self.aE[:, :-1] * (x[:, :-1] - x[:, 1:])
        y[:, 1:] += self.aW[:, 1:] * (x[:, 1:] - x[:, :-1])
        y[:-1, :] += self.aN[:-1, :] * (x[:-1, :] - x[1:, :])
        y[1:, :] += self.aS[1:, :] * (x[1:, :] - x[:-1, :])
        return y

    def coarsen(self):
        ny, nx = self.dP.shape
        nyc, nxc = (ny + 1) // 2, (nx + 1) // 2
        pad = lambda a, v: np.pad(a, ((0, 2 * nyc - ny), (0, 2 * nxc - nx)), constant_values=v)
        act, dP, aE, aN = pad(self.act, False), pad(self.dP, 0.0), pad(self.aE, 0.0), pad(self.aN, 0.0)
        actc = act.reshape(nyc, 2, nxc, 2).any(axis=(1, 3))
        dPc = np.where(act, dP, 0.0).reshape(nyc, 2, nxc, 2).sum(axis=(1, 3))
        eb = np.zeros((2 * nyc, nxc))
        eb[:, :-1] = np.where(act[:, 1::2][:, :-1] & act[:, 2::2], aE[:, 1::2][:, :-1], 0.0)
        nb = np.zeros((nyc, 2 * nxc))
        nb[:-1] = np.where(act[1::2][:-1] & act[2::2], aN[1::2][:-1], 0.0)
        aEc, aNc = eb.reshape(nyc, 2, nxc).sum(axis=1), nb.reshape(nyc, nxc, 2).sum(axis=2)
        return Level(np.where(actc, dPc, 1.0), np.where(actc, aEc, 0.0), np.where(actc, aNc, 0.0), actc)

    def restrict(self, r):
        ny, nx = r.shape
        out = np.zeros((ny + ny % 2, nx + nx % 2))
        out[:ny, :nx] = np.where(self.act, r, 0.0)
        return out.reshape(out.shape[0] // 2, 2, out.shape[1] // 2, 2).sum(axis=(1, 3))

    def prolong(self, xc):
        ny, nx = self.dP.shape
        return np.where(self.act, np.kron(xc, np.ones((2, 2)))[:ny, :nx], 0.0)


def cycle(lv, l, b, tau1, s2, wc):
    L = lv[l]
    if l == len(lv) - 1:
        return np.where(L.act, b / L.dP, b)
    w = np.where(L.act, tau1, 1.0) / L.diag
    x = w * b                                    # first pre-sweep from zero
    x = x + s2 * w * (b - L.A(x))                # the sweep next to the coarse correction
    xc = cycle(lv, l + 1, lv[l].restrict(b - L.A(x)), tau1, s2, wc)
    x = x + wc * L.prolong(xc)
    x = x + s2 * w * (b - L.A(x))                # the first post-sweep takes the same factor
    return x + w * (b - L.A(x))


def random_hierarchy(ny=10, nx=12, seed=7):
    rng = np.random.default_rng(seed)
    act = rng.random((ny, nx)) > 0.15            # identity rows: about 15 %
    aE = np.where(act & np.roll(act, -1, axis=1), rng.uniform(0.1, 10.0, (ny, nx)), 0.0)
    aN = np.where(act & np.roll(act, -1, axis=0), rng.uniform(0.1, 10.0, (ny, nx)), 0.0)
    dP = np.where(act, rng.uniform(0.0, 0.05, (ny, nx)), 1.0)
    lv = [Level(dP, aE, aN, act)]
    while lv[-1].dP.size > 1:
        lv.append(lv[-1].coarsen())
    return lv


@pytest.mark.parametrize("weights", [(0.8, 1.0, 1.6), ("cheb", 1.45), ("cheb", 1.3)],
                         ids=["jacobi-0.8-1.6", "chebyshev-1.45", "chebyshev-1.3"])
def test_cycle_is_a_symmetric_positive_definite_preconditioner(weights):
    if weights[0] == "cheb":
        t1, t2 = chebyshev_pair()
        tau1, s2, wc = t1, t2 / t1, weights[1]
    else:
        tau1, s2, wc = weights
    lv = random_hierarchy()
    ny, nx = lv[0].dP.shape
    n = nx * ny
    B = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n); e[k] = 1.0
        B[:, k] = cycle(lv, 0, e.reshape(ny, nx), tau1, s2, wc).ravel()
    assert np.max(np.abs(B - B.T)) <= 1e-12 * np.max(np.abs(B))
    assert np.linalg.eigvalsh(0.5 * (B + B.T)).min() > 0.0


def test_chebyshev_pair_smoothing_bounds():
    t1, t2 = chebyshev_pair()
    assert abs(t2 / t1 - 2.4738) < 1e-4
    mu = np.linspace(0.45, 1.8, 20001)
    p = (1 - t1 * mu) * (1 - t2 * mu)
    assert abs(np.abs(p).max() - 1.0 / (2 * (1.125 / 0.675) ** 2 - 1)) < 1e-9   # 1 / T2(mid / half)
    assert np.abs((1 - 0.8 * mu) ** 2).max() > 0.4                              # damped Jacobi: 0.41
    mu2 = np.linspace(1e-6, 2.0, 20001)
    assert np.abs((1 - t1 * mu2) * (1 - t2 * mu2)).max() < 1.0                  # no error grows
