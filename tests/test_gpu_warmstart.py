"""GPU tests of the learned warm start (shk_nn_* kernels, shakti.jl_b200/warmstart.py).

 - Each tensor-core kernel against the CPU restatement (oracle/nn_oracle.py) on identical inputs:
   the forward and input-gradient convolutions, the weight gradient, the ReLU/bias gradient, and
   the pooling / upsampling pairs, to Float32 accumulation accuracy.
 - The whole network's loss and every layer's gradients against the oracle, two ways.  Given the
   GPU's own stored activations, the oracle's backward pass agrees with the GPU's for every layer
   within 1 % in norm for the weights (measured <= 0.25 %) and 2 % for the biases.  End to end, the oracle's own
   forward pass sums exactly where the tensor cores accumulate in Float32, so a stored BF16
   activation whose two sums straddle a rounding boundary differs by one BF16 step; the stored
   activations drift apart by 1e-4 .. 3e-3 (relative) over the fifteen layers and the weight
   gradients, which depend on them through the ReLU masks, by up to ~8 %: that bar is direction
   (cosine >= 0.99) and 15 % in norm.
 - Training lowers the loss; the seeding falls back to the current head when its residual is not
   smaller (bit-identical timestep), and an accepted warm start lowers the first solve's CG
   iterations.
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import nn_oracle as no  # noqa: E402


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def ws(shk, cuda):
    from shakti_b200 import warmstart
    return warmstart


@pytest.mark.parametrize("ci,co,N,H,W", [(16, 32, 1, 40, 37), (32, 64, 2, 16, 24), (64, 128, 1, 33, 17),
                                         (128, 256, 1, 20, 20), (32, 8, 1, 13, 11), (256, 128, 2, 35, 70),
                                         (64, 16, 3, 5, 3)])
def test_tensor_core_convolution(ws, cuda, monkeypatch, ci, co, N, H, W):
    """The convolution forms -- tcgen05 on TMA-loaded halo tiles with the layer's weights resident in
    each CTA where they fit (the default) or restaged with every chunk (SHK_NN_HX_STREAM=1), tcgen05
    with per-tap gathered A tiles (SHK_NN_TC_GATHER=1), mma.sync (SHK_NN_MMA_SYNC=1) -- forward with bias
    and ReLU and the flipped input-gradient form, against the oracle and each other: images whose
    sides are not multiples of the 16 x 8 M tile, several images, 16-channel input (Cin = 16), Cout
    padded to the 16-wide N tile (Cout = 8), the 256-wide tile.  All accumulate BF16 products in
    Float32 (1e-5)."""
    torch = cuda
    net = ws.WarmStartNet(seed=3)
    L, s = net.L, net._s()
    g = np.random.default_rng(ci + co)
    X = torch.from_numpy(g.normal(0, 1, size=(N, H, W, ci)).astype(np.float32)).cuda().to(torch.bfloat16)
    Wf = g.normal(0, 0.1, size=(9, co, ci)).astype(np.float32)
    bias = torch.from_numpy(g.normal(0, 0.1, size=co).astype(np.float32)).cuda()
    wb = torch.from_numpy(Wf).cuda().to(torch.bfloat16)
    Xn, Wn = X.float().cpu().numpy(), wb.float().cpu().numpy()
    out = {}
    for form in ("tc", "stream", "gather", "mma_sync"):
        if form == "mma_sync":
            monkeypatch.setenv("SHK_NN_MMA_SYNC", "1")
        if form == "gather":
            monkeypatch.setenv("SHK_NN_TC_GATHER", "1")
        if form == "stream":
            monkeypatch.setenv("SHK_NN_HX_STREAM", "1")
        Yf = torch.empty((N, H, W, co), dtype=torch.float32, device="cuda")
        Yb = torch.empty((N, H, W, co), dtype=torch.bfloat16, device="cuda")
        assert L.shk_nn_conv3x3(ws._p(X), ws._p(wb), ws._fp(bias), ws._p(Yb), ws._fp(Yf), N, H, W, ci, co, 1, 0,
                                s) == 0
        dX = None
        if co % 16 == 0:  # the input gradient needs Cin % 16 == 0 on its own input
            wt = torch.from_numpy(np.ascontiguousarray(Wf.transpose(0, 2, 1))).cuda().to(torch.bfloat16)
            dX = torch.empty((N, H, W, ci), dtype=torch.float32, device="cuda")
            assert L.shk_nn_conv3x3(ws._p(Yb), ws._p(wt), None, None, ws._fp(dX), N, H, W, co, ci, 0, 1, s) == 0
        torch.cuda.synchronize()
        out[form] = (Yf.cpu().numpy(), Yb.float().cpu().numpy(), None if dX is None else dX.cpu().numpy())
        monkeypatch.delenv("SHK_NN_MMA_SYNC", raising=False)
        monkeypatch.delenv("SHK_NN_TC_GATHER", raising=False)
        monkeypatch.delenv("SHK_NN_HX_STREAM", raising=False)
    fault = C.c_int(-1)
    assert L.shk_nn_conv_fault(C.byref(fault)) == 0 and fault.value == 0
    ref = no.conv3x3(Xn, Wn, bias.cpu().numpy(), relu=True)
    assert rel(out["tc"][0], ref) < 1e-5
    assert rel(out["tc"][0], out["mma_sync"][0]) < 1e-5
    assert rel(out["gather"][0], ref) < 1e-5 and rel(out["mma_sync"][0], ref) < 1e-5
    assert np.array_equal(out["stream"][0], out["tc"][0])  # the same MMAs, weights staged differently
    assert np.array_equal(out["tc"][1], no.bf16(out["tc"][0]))  # the BF16 output is the rounded Float32 one
    if out["tc"][2] is not None:
        # each form's input gradient from its own BF16 forward output (the forms' outputs may differ
        # by one BF16 step where their Float32 sums straddle a rounding boundary)
        for form, (_, yb, dx) in out.items():
            ref_dx = no.conv3x3(yb, Wn.transpose(0, 2, 1), None, flip=True)
            assert rel(dx, ref_dx) < 1e-5, form


def test_kernels_match_oracle(ws, cuda):
    torch = cuda
    net = ws.WarmStartNet(seed=3)
    g = np.random.default_rng(5)
    N, H, W, ci, co = 2, 16, 24, 32, 64
    X = torch.from_numpy(g.normal(0, 1, size=(N, H, W, ci)).astype(np.float32)).cuda().to(torch.bfloat16)
    Wf = g.normal(0, 0.1, size=(9, co, ci)).astype(np.float32)
    bias = torch.from_numpy(g.normal(0, 0.1, size=co).astype(np.float32)).cuda()
    wb = torch.from_numpy(Wf).cuda().to(torch.bfloat16)
    wt = torch.from_numpy(np.ascontiguousarray(Wf.transpose(0, 2, 1))).cuda().to(torch.bfloat16)
    L, s = net.L, net._s()
    Xn, Wn = X.float().cpu().numpy(), wb.float().cpu().numpy()
    Yf = torch.empty((N, H, W, co), dtype=torch.float32, device="cuda")
    assert L.shk_nn_conv3x3(ws._p(X), ws._p(wb), ws._fp(bias), None, ws._fp(Yf), N, H, W, ci, co, 1, 0, s) == 0
    ref = no.conv3x3(Xn, Wn, bias.cpu().numpy(), relu=True)
    assert rel(Yf.cpu().numpy(), ref) < 1e-5
    dY = torch.from_numpy(g.normal(0, 1, size=(N, H, W, co)).astype(np.float32)).cuda().to(torch.bfloat16)
    dX = torch.empty((N, H, W, ci), dtype=torch.float32, device="cuda")
    assert L.shk_nn_conv3x3(ws._p(dY), ws._p(wt), None, None, ws._fp(dX), N, H, W, co, ci, 0, 1, s) == 0
    ref = no.conv3x3(dY.float().cpu().numpy(), Wn.transpose(0, 2, 1), None, flip=True)
    assert rel(dX.cpu().numpy(), ref) < 1e-5
    dW = torch.zeros((9, co, ci), dtype=torch.float32, device="cuda")
    assert L.shk_nn_conv3x3_wgrad(ws._p(X), ws._p(dY), ws._fp(dW), N, H, W, ci, co, s) == 0
    assert rel(dW.cpu().numpy(), no.conv3x3_wgrad(Xn, dY.float().cpu().numpy())) < 1e-5
    # ReLU gradient and bias gradient
    Yb = torch.from_numpy(g.normal(0, 1, size=(N, H, W, co)).astype(np.float32)).cuda().to(torch.bfloat16)
    dYf = torch.from_numpy(g.normal(0, 1, size=(N, H, W, co)).astype(np.float32)).cuda()
    dm = torch.empty((N, H, W, co), dtype=torch.bfloat16, device="cuda")
    db = torch.zeros(co, dtype=torch.float32, device="cuda")
    assert L.shk_nn_relu_grad(ws._fp(dYf), ws._p(Yb), ws._p(dm), ws._fp(db), N * H * W, co, 1, s) == 0
    gref = dYf.cpu().numpy() * (Yb.float().cpu().numpy() > 0)
    assert np.array_equal(dm.float().cpu().numpy(), no.bf16(gref))
    assert rel(db.cpu().numpy(), gref.sum(axis=(0, 1, 2))) < 1e-5
    # pooling / upsampling and their gradients
    P = torch.empty((N, H // 2, W // 2, ci), dtype=torch.bfloat16, device="cuda")
    assert L.shk_nn_pool2(ws._p(X), ws._p(P), N, H, W, ci, s) == 0
    assert rel(P.float().cpu().numpy(), no.bf16(no.pool2(Xn))) < 1e-3
    U = torch.empty((N, H, W, ci), dtype=torch.bfloat16, device="cuda")
    assert L.shk_nn_up2_add(ws._p(P), ws._p(X), ws._p(U), N, H, W, ci, s) == 0
    assert rel(U.float().cpu().numpy(), no.bf16(no.up2(P.float().cpu().numpy()) + Xn)) < 1e-3
    gc = torch.from_numpy(g.normal(0, 1, size=(N, H // 2, W // 2, ci)).astype(np.float32)).cuda()
    gf = torch.empty((N, H, W, ci), dtype=torch.float32, device="cuda")
    assert L.shk_nn_pool2_grad(ws._fp(gc), ws._fp(gf), N, H, W, ci, 0, s) == 0
    assert rel(gf.cpu().numpy(), no.pool2_grad(gc.cpu().numpy())) < 1e-6
    gc2 = torch.empty((N, H // 2, W // 2, ci), dtype=torch.float32, device="cuda")
    assert L.shk_nn_up2_grad(ws._fp(gf), ws._fp(gc2), N, H // 2, W // 2, ci, s) == 0
    assert rel(gc2.cpu().numpy(), no.up2_grad(gf.cpu().numpy())) < 1e-6


def test_network_gradients_match_oracle(ws, cuda):
    torch = cuda
    net = ws.WarmStartNet(seed=3)
    g = np.random.default_rng(1)
    N, H, W = 2, 16, 16
    X = torch.from_numpy(g.normal(0, 1, size=(N, H, W, 16)).astype(np.float32)).cuda().to(torch.bfloat16)
    Tn = g.normal(0, 1, size=(N, H, W)).astype(np.float32)
    T = torch.from_numpy(Tn).cuda()
    loss = float(net.loss_and_grad(X, T, torch.ones_like(T)).item())
    params = net.params_numpy()
    Y, A = no.forward(params, None, X.float().cpu().numpy())
    lref, G = no.backward(params, A, Y, Tn, None)
    assert abs(loss - lref) <= 1e-3 * abs(lref)
    # the oracle's backward pass fed the GPU's own stored activations and head output
    Ag = {k: v.float().cpu().numpy() for k, v in net._acts.items()}
    _, Gg = no.backward(params, Ag, net._bufs["y"].cpu().numpy(), Tn, None)
    report = {}
    for name, *_ in ws.LAYERS:
        gw = net.P[name]["gw"].cpu().numpy().ravel()
        gb = net.P[name]["gb"].cpu().numpy()
        rw = G[name][0].ravel()
        cos = float(gw @ rw / (np.linalg.norm(gw) * np.linalg.norm(rw)))
        report[name] = (round(rel(gw, rw), 5), round(rel(gw, Gg[name][0].ravel()), 6))
        assert cos >= 0.99 and rel(gw, rw) <= 0.15, (name, cos, rel(gw, rw))
        assert rel(gb, G[name][1]) <= 0.15, name
        assert rel(gw, Gg[name][0].ravel()) <= 0.01 and rel(gb, Gg[name][1]) <= 0.02, (name, report[name])
    print("weight-gradient rel. error per layer (end to end, given the GPU's activations):", report)
    print("stored activations, rel. error vs the oracle's forward pass:",
          {k: round(rel(Ag[k], A[k]), 6) for k in A})


def test_training_lowers_the_loss(ws, cuda):
    """A learnable target (a fixed random 3x3 stencil of the inputs) on random images."""
    torch = cuda
    net = ws.WarmStartNet(seed=0)
    g = np.random.default_rng(2)
    S, H = 256, 16
    Xn = g.normal(0, 1, size=(S, H, H, 16)).astype(np.float32)
    Xn[..., 7:] = 0.0
    k = g.normal(0, 0.5, size=(3, 3))
    Xp = np.pad(Xn[..., 0], ((0, 0), (1, 1), (1, 1)))
    Tn = sum(k[i, j] * Xp[:, i:i + H, j:j + H] for i in range(3) for j in range(3)).astype(np.float32)
    X = torch.from_numpy(Xn).cuda().to(torch.bfloat16)
    T = torch.from_numpy(Tn).cuda()
    M = torch.ones_like(T)
    losses = net.train(X, T, M, steps=300, batch=32, lr=2e-3)
    assert np.mean(losses[-30:]) < 0.25 * np.mean(losses[:10]), (np.mean(losses[:10]), np.mean(losses[-30:]))


def _settled(shk, ws, spec, steps=2):
    sim = ws.member_sim(shk, spec)
    for _ in range(steps):
        shk.step(sim)
        sim.total_time += sim.dt
    return sim


SPEC = dict(nx=64, seed=555, slope=0.012, melt=5e-8, C=2e4, b0=0.004)


def test_fallback_reproduces_the_unseeded_step(shk, ws, cuda):
    """An untrained network's head is rejected (larger initial residual): the timestep is then
    exactly the unseeded one."""
    net = ws.WarmStartNet(seed=1)
    a, b = _settled(shk, ws, SPEC), _settled(shk, ws, SPEC)
    stats = {}
    used = ws.step_seeded(a, net, stats)
    shk.step(b)
    assert not used and stats["r_seed"][0] > stats["r_prev"][0]
    assert cuda.equal(a.state.h, b.state.h) and cuda.equal(a.state.b, b.state.b)
    assert a.hs.ps.cg_iters_total == b.hs.ps.cg_iters_total


def test_accepted_warm_start_lowers_the_first_solve(shk, ws, cuda):
    """The seeding path itself: the exact first Picard iterate as the guess is accepted and the
    first solve then needs far fewer CG iterations, the solution unchanged to its tolerance."""
    ref = _settled(shk, ws, SPEC)
    base = _settled(shk, ws, SPEC)
    sim = _settled(shk, ws, SPEC)
    ws._one_picard(ref)                        # G(h): the first Picard iterate
    g1 = ref.state.h.clone()
    st_base = ws._one_picard(base)
    ctx = sim.ctx()
    r0, b0, r1, b1 = (C.c_double() for _ in range(4))
    assert ctx.L.shk_initial_residual(ctx.h, C.byref(r0), C.byref(b0)) == 0
    assert ctx.L.shk_residual_of(ctx.h, ws._p(g1), C.byref(r1), C.byref(b1)) == 0
    assert r1.value < 0.1 * r0.value  # G(h) is itself only solved to rel-res 1e-8
    assert ctx.L.shk_set_cg_warm_start(ctx.h, ws._p(g1)) == 0
    st = ws._one_picard(sim)
    assert st.cg_iters_total < 0.5 * st_base.cg_iters_total, (st.cg_iters_total, st_base.cg_iters_total)
    h, hb = sim.state.h.cpu().numpy(), base.state.h.cpu().numpy()
    assert np.max(np.abs(h - hb)) <= 1e-6 * np.max(np.abs(hb))


def test_trained_network_gain_is_measured(shk, ws, cuda):
    """Trains on first-Picard-iterate pairs from a small ensemble run of the plain solver, then runs
    an unseen instance seeded and unseeded.  The seed is used only when it lowers the first solve's
    initial residual, so the seeded run never needs more CG iterations; the measured CG iterations,
    acceptance and residual ratios are the network's gain over the method without it."""
    torch = cuda
    net = ws.WarmStartNet(seed=0)
    specs = shk.configs.ensemble_specs(16, seed=99, sizes=(64,))
    X, T, M = ws.generate_pairs(shk, net, specs, steps=12, crops=4)
    assert X.shape[0] > 100
    losses = net.train(X, T, M, steps=300, batch=32, lr=1e-3)
    assert np.mean(losses[-30:]) < np.mean(losses[:10])
    ev = ws.evaluate(shk, net, SPEC, steps=3, settle=2)
    seeded, unseeded = ev["seeded"], ev["unseeded"]
    print("warm-start gain:", {k: (unseeded[k], seeded[k]) for k in ("cg_per_step", "picard_per_step")},
          "accepted", seeded["seed"]["seeded"], "r_seed/r_prev",
          [round(b / a, 2) for a, b in zip(seeded["seed"]["r_prev"], seeded["seed"]["r_seed"])])
    # the evaluation is only meaningful where Picard converges (this instance: 9-15 iterations a step)
    for r in unseeded["per_step"] + seeded["per_step"]:
        assert r["converged"] and r["picard"] < 500, r
    for u, s_, used in zip(unseeded["per_step"], seeded["per_step"], seeded["seed"]["seeded"]):
        if not used:
            assert s_["cg"] == u["cg"] and s_["picard"] == u["picard"]
    assert ev["h_relerr_vs_unseeded"] <= 1e-4
