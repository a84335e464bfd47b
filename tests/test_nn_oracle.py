"""The learned-warm-start network's CPU restatement (oracle/nn_oracle.py), pinned by finite
differences: with BF16 rounding switched off its analytic gradients of every layer's weights and
biases match central differences of its own loss."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))

import nn_oracle as no  # noqa: E402

# the network's layer table (name, Cin, Cout), as in shakti.jl_b200/warmstart.py
LAYERS = [("enc0a", 16, 32), ("enc0b", 32, 32), ("enc1a", 32, 64), ("enc1b", 64, 64), ("enc2a", 64, 128),
          ("enc2b", 128, 128), ("enc3a", 128, 256), ("enc3b", 256, 256), ("dec2a", 256, 128), ("dec2b", 128, 128),
          ("dec1a", 128, 64), ("dec1b", 64, 64), ("dec0a", 64, 32), ("dec0b", 32, 32), ("head", 32, 16)]


def test_layer_table_matches_the_package(shk):
    from shakti_b200 import warmstart as ws
    assert [(n, a, b) for n, a, b, _ in ws.LAYERS] == LAYERS


@pytest.fixture
def exact():
    no.EXACT = True
    yield
    no.EXACT = False


def test_oracle_gradients_match_finite_differences(exact):
    g = np.random.default_rng(7)
    params = {n: (g.normal(0, np.sqrt(2.0 / (9 * ci)), size=(9, co, ci)), g.normal(0, 0.05, size=co))
              for n, ci, co in LAYERS}
    X = g.normal(0, 1, size=(1, 8, 8, 16))
    T = g.normal(0, 1, size=(1, 8, 8))

    def loss_of(p):
        Y, A = no.forward(p, None, X)
        return no.backward(p, A, Y, T, None)[0]

    Y, A = no.forward(params, None, X)
    _, G = no.backward(params, A, Y, T, None)
    eps = 1e-6
    checked = 0
    for name in ("enc0a", "enc2b", "enc3b", "dec1a", "dec0b", "head"):
        W, b = params[name]
        for idx in [(0, 0, 0), (4, 1, 3), (8, W.shape[1] - 1, W.shape[2] - 1)]:
            Wp, Wm = W.copy(), W.copy()
            Wp[idx] += eps
            Wm[idx] -= eps
            fd = (loss_of({**params, name: (Wp, b)}) - loss_of({**params, name: (Wm, b)})) / (2 * eps)
            an = G[name][0][idx]
            assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)) + 1e-9, (name, idx, fd, an)
            checked += 1
        bp, bm = b.copy(), b.copy()
        bp[0] += eps
        bm[0] -= eps
        fd = (loss_of({**params, name: (W, bp)}) - loss_of({**params, name: (W, bm)})) / (2 * eps)
        assert abs(fd - G[name][1][0]) <= 1e-5 * max(1.0, abs(fd)) + 1e-9, (name, fd, G[name][1][0])
    assert checked == 18


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-40], dtype=np.float32)
    r = no.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0          # halfway between 1 and 1+2^-7: ties to even
    assert r[2] == np.float32(1.0 + 2 ** -7)     # above halfway: rounds up
    assert r[3] == -2.5
