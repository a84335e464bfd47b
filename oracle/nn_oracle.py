"""CPU restatement (numpy) of the learned-warm-start network's forward and backward passes.

TEST INFRASTRUCTURE ONLY: the test oracle of the GPU training kernels (shakti.jl_b200/csrc/shk_nn.cu,
driven by shakti.jl_b200/warmstart.py).  Nothing in the product imports it.

It follows the GPU pass exactly, operation by operation, including where the GPU rounds to BF16
(every stored activation, the pooled and upsampled tensors, the masked output gradients that feed
the tensor cores), with Float64 accumulation in place of the tensor cores' Float32.  The network
has no counterpart in the reference (it seeds cg!'s x0 = vec(h), src/linear_solver.jl:876-881).
"""
from __future__ import annotations

import numpy as np

OFFSETS = [(t // 3 - 1, t % 3 - 1) for t in range(9)]  # (dy, dx) of tap t


EXACT = False  # True: no BF16 rounding anywhere (Float64 throughout), for finite-difference checks


def bf16(a):
    """Round to BF16 (nearest, ties to even) and back to float32 (identity when EXACT)."""
    if EXACT:
        return np.asarray(a, dtype=np.float64)
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def conv3x3(X, W, bias=None, relu=False, flip=False):
    """X [N,H,W,Cin], W [9,Cout,Cin] -> [N,H,W,Cout] (Float64), zero padding."""
    N, H, Wd, _ = X.shape
    Xp = np.zeros((N, H + 2, Wd + 2, X.shape[3]))
    Xp[:, 1:-1, 1:-1] = X
    Y = np.zeros((N, H, Wd, W.shape[1]))
    for t, (dy, dx) in enumerate(OFFSETS):
        if flip:
            dy, dx = -dy, -dx
        Y += np.einsum("nyxc,oc->nyxo", Xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + Wd], W[t].astype(np.float64))
    if bias is not None:
        Y += bias
    if relu:
        Y = np.maximum(Y, 0.0)
    return Y


def conv3x3_wgrad(X, dY):
    """dW[t, co, ci] = sum_p dY[p, co] X[p + off(t), ci]."""
    N, H, Wd, Cin = X.shape
    Xp = np.zeros((N, H + 2, Wd + 2, Cin))
    Xp[:, 1:-1, 1:-1] = X
    dW = np.zeros((9, dY.shape[3], Cin))
    for t, (dy, dx) in enumerate(OFFSETS):
        dW[t] = np.einsum("nyxo,nyxc->oc", dY, Xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + Wd])
    return dW


def pool2(X):
    N, H, W, C = X.shape
    return X.reshape(N, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def pool2_grad(dY):
    return 0.25 * np.repeat(np.repeat(dY, 2, axis=1), 2, axis=2)


def up2(X):
    return np.repeat(np.repeat(X, 2, axis=1), 2, axis=2)


def up2_grad(dY):
    N, H, W, C = dY.shape
    return dY.reshape(N, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def forward(params, layers, X):
    """params: name -> (W [9,Cout,Cin] float32, b [Cout] float32); returns the head output (Float64)
    and the stored activations (BF16-rounded, as the GPU stores them)."""
    def cv(name, x, relu=True):
        W, b = params[name]
        return bf16(conv3x3(x, bf16(W), b, relu=relu))
    A = {"x0": X}
    A["a0"] = cv("enc0a", X); A["s0"] = cv("enc0b", A["a0"])
    A["p1"] = bf16(pool2(A["s0"])); A["a1"] = cv("enc1a", A["p1"]); A["s1"] = cv("enc1b", A["a1"])
    A["p2"] = bf16(pool2(A["s1"])); A["a2"] = cv("enc2a", A["p2"]); A["s2"] = cv("enc2b", A["a2"])
    A["p3"] = bf16(pool2(A["s2"])); A["a3"] = cv("enc3a", A["p3"]); A["s3"] = cv("enc3b", A["a3"])
    A["d2a"] = cv("dec2a", A["s3"]); A["u2"] = bf16(up2(A["d2a"]) + A["s2"]); A["d2"] = cv("dec2b", A["u2"])
    A["d1a"] = cv("dec1a", A["d2"]); A["u1"] = bf16(up2(A["d1a"]) + A["s1"]); A["d1"] = cv("dec1b", A["u1"])
    A["d0a"] = cv("dec0a", A["d1"]); A["u0"] = bf16(up2(A["d0a"]) + A["s0"]); A["d0"] = cv("dec0b", A["u0"])
    W, b = params["head"]
    Y = conv3x3(A["d0"], bf16(W), b, relu=False)
    return Y, A


def backward(params, A, Y, T, wgt):
    """Loss mean((y0 - t)^2 w) over the pixels and its gradients (name -> (dW, db))."""
    P = T.size
    y0 = Y[..., 0] if EXACT else Y[..., 0].astype(np.float32)
    d = (y0 - T) * (1.0 if wgt is None else wgt)
    loss = float(np.sum(d * (y0 - T)) / P)
    dY = np.zeros_like(Y)
    dY[..., 0] = 2.0 * d / P
    G = {}

    def layer(name, x_in, dout, out=None):
        """gradient through conv `name` (ReLU if out is given): returns d(input) (Float64)."""
        W, b = params[name]
        g = dout if out is None else dout * (out > 0)
        gb = bf16(g)
        G[name] = (conv3x3_wgrad(x_in, gb), g.sum(axis=(0, 1, 2)))
        return conv3x3(gb, bf16(W).transpose(0, 2, 1), None, relu=False, flip=True)

    dd0 = layer("head", A["d0"], dY)
    du0 = layer("dec0b", A["u0"], dd0, A["d0"])
    dd1 = layer("dec0a", A["d1"], up2_grad(du0), A["d0a"])
    ds0 = du0.copy()
    du1 = layer("dec1b", A["u1"], dd1, A["d1"])
    dd2 = layer("dec1a", A["d2"], up2_grad(du1), A["d1a"])
    ds1 = du1.copy()
    du2 = layer("dec2b", A["u2"], dd2, A["d2"])
    ds3 = layer("dec2a", A["s3"], up2_grad(du2), A["d2a"])
    ds2 = du2.copy()
    da3 = layer("enc3b", A["a3"], ds3, A["s3"])
    dp3 = layer("enc3a", A["p3"], da3, A["a3"])
    ds2 = ds2 + pool2_grad(dp3)
    da2 = layer("enc2b", A["a2"], ds2, A["s2"])
    dp2 = layer("enc2a", A["p2"], da2, A["a2"])
    ds1 = ds1 + pool2_grad(dp2)
    da1 = layer("enc1b", A["a1"], ds1, A["s1"])
    dp1 = layer("enc1a", A["p1"], da1, A["a1"])
    ds0 = ds0 + pool2_grad(dp1)
    da0 = layer("enc0b", A["a0"], ds0, A["s0"])
    layer("enc0a", A["x0"], da0, A["a0"])
    return loss, G
