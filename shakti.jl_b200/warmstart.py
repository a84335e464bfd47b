"""Learned warm start: a small convolutional encoder-decoder that predicts the head increment of
the coming timestep, trained and run by the library's own BF16 tensor-core kernels (shk_nn_*).

No counterpart in the reference, whose solves start from the current head (cg! x0 = vec(h),
src/linear_solver.jl:876-881).  The network predicts the timestep's first Picard iterate; the
prediction seeds that iteration's CG solve when its initial residual ||b - A x0|| is below the
current head's (else the solve starts from the current head), and every solve still runs to its
tolerance (rel-res 1e-8), Picard to its own.

Network (4 levels, 32 base channels, ReLU; NHWC; BF16 weights and activations, Float32
accumulation and gradients): two 3x3 convolutions per encoder level (32, 64, 128, 256 channels)
with 2x2 average pooling between levels; per decoder level a 3x3 convolution at the coarse level,
nearest 2x upsampling plus the encoder's skip tensor, and a second 3x3 convolution; a 3x3 head to
the (normalised) increment.  Input: h, b, N, zb, zs, ieb and mask, each normalised by the
training set's mean and spread, padded to 16 channels.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib

# name, Cin, Cout, ReLU
LAYERS = [("enc0a", 16, 32, True), ("enc0b", 32, 32, True), ("enc1a", 32, 64, True), ("enc1b", 64, 64, True),
          ("enc2a", 64, 128, True), ("enc2b", 128, 128, True), ("enc3a", 128, 256, True), ("enc3b", 256, 256, True),
          ("dec2a", 256, 128, True), ("dec2b", 128, 128, True), ("dec1a", 128, 64, True), ("dec1b", 64, 64, True),
          ("dec0a", 64, 32, True), ("dec0b", 32, 32, True), ("head", 32, 16, False)]
IN_FIELDS = ("h", "b", "N", "zb", "zs", "ieb", "mask")
HEAD_C = 16


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _fp(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float)) if t is not None else None


class WarmStartNet:
    def __init__(self, seed: int = 0):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA is not available: the B200 library needs a GPU")
        self.L = _lib.load()
        self.torch = torch
        self.dev = torch.device("cuda")
        g = np.random.default_rng(seed)
        self.P = {}
        for name, cin, cout, _ in LAYERS:
            fan_in = 9 * (7 if name == "enc0a" else cin)
            std = math.sqrt(2.0 / fan_in) * (0.1 if name == "head" else 1.0)
            w = g.normal(0.0, std, size=(9, cout, cin)).astype(np.float32)
            if name == "enc0a":
                w[:, :, 7:] = 0.0
            self.P[name] = dict(
                w=torch.from_numpy(w).to(self.dev), b=torch.zeros(cout, dtype=torch.float32, device=self.dev),
                wb=torch.empty((9, cout, cin), dtype=torch.bfloat16, device=self.dev),
                wt=torch.empty((9, cin, cout), dtype=torch.bfloat16, device=self.dev),
                gw=torch.zeros((9, cout, cin), dtype=torch.float32, device=self.dev),
                gb=torch.zeros(cout, dtype=torch.float32, device=self.dev),
                mw=torch.zeros((9, cout, cin), dtype=torch.float32, device=self.dev),
                vw=torch.zeros((9, cout, cin), dtype=torch.float32, device=self.dev),
                mb=torch.zeros(cout, dtype=torch.float32, device=self.dev),
                vb=torch.zeros(cout, dtype=torch.float32, device=self.dev), cin=cin, cout=cout)
        self._refresh()
        self.norm = torch.tensor([0.0, 1.0] * 7, dtype=torch.float32, device=self.dev)
        self.dh_scale = 1.0
        self.step_no = 0
        self.losses = []
        self._bufs = {}

    # ---- plumbing -----------------------------------------------------------------------------
    def _chk(self, rc, what):
        if rc != _lib.OK:
            raise _lib.ShaktiError(rc, what)

    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def _refresh(self):
        for name, cin, cout, _ in LAYERS:
            p = self.P[name]
            self._chk(self.L.shk_nn_wcast(_fp(p["w"]), _p(p["wb"]), _p(p["wt"]), p["w"].numel(), cout, cin, self._s()),
                      "wcast")

    def _buf(self, key, shape, dtype):
        t = self._bufs.get(key)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = self.torch.empty(shape, dtype=dtype, device=self.dev)
            self._bufs[key] = t
        return t

    def params_numpy(self):
        return {n: (self.P[n]["w"].cpu().numpy(), self.P[n]["b"].cpu().numpy()) for n, *_ in LAYERS}

    def set_normalisation(self, means, spreads, dh_scale):
        v = []
        for m, s in zip(means, spreads):
            v += [float(m), 1.0 / float(s)]
        self.norm = self.torch.tensor(v, dtype=self.torch.float32, device=self.dev)
        self.dh_scale = float(dh_scale)

    # ---- forward / backward ------------------------------------------------------------------
    def _conv(self, name, X, N, H, W, relu, out_key, f32=False):
        p = self.P[name]
        bf = self.torch.bfloat16
        Y = None if f32 else self._buf(out_key, (N, H, W, p["cout"]), bf)
        Yf = self._buf(out_key, (N, H, W, p["cout"]), self.torch.float32) if f32 else None
        self._chk(self.L.shk_nn_conv3x3(_p(X), _p(p["wb"]), _fp(p["b"]), _p(Y), _fp(Yf), N, H, W, p["cin"],
                                        p["cout"], int(relu), 0, self._s()), f"conv {name}")
        return Yf if f32 else Y

    def forward(self, X):
        """X: [N, H, W, 16] BF16 (H, W multiples of 8) -> head output [N, H, W, 16] Float32."""
        N, H, W, _ = X.shape
        bf = self.torch.bfloat16
        A = self._acts = {"x0": X}
        A["a0"] = self._conv("enc0a", X, N, H, W, True, "a0")
        A["s0"] = self._conv("enc0b", A["a0"], N, H, W, True, "s0")
        h, w = H, W
        for lvl in (1, 2, 3):
            c = self.P[f"enc{lvl - 1}b"]["cout"]
            pk = self._buf(f"p{lvl}", (N, h // 2, w // 2, c), bf)
            self._chk(self.L.shk_nn_pool2(_p(A[f"s{lvl - 1}"]), _p(pk), N, h, w, c, self._s()), "pool")
            h, w = h // 2, w // 2
            A[f"p{lvl}"] = pk
            A[f"a{lvl}"] = self._conv(f"enc{lvl}a", pk, N, h, w, True, f"a{lvl}")
            A[f"s{lvl}"] = self._conv(f"enc{lvl}b", A[f"a{lvl}"], N, h, w, True, f"s{lvl}")
        prev = A["s3"]
        for lvl in (2, 1, 0):
            A[f"d{lvl}a"] = self._conv(f"dec{lvl}a", prev, N, h, w, True, f"d{lvl}a")
            c = self.P[f"dec{lvl}a"]["cout"]
            h, w = h * 2, w * 2
            u = self._buf(f"u{lvl}", (N, h, w, c), bf)
            self._chk(self.L.shk_nn_up2_add(_p(A[f"d{lvl}a"]), _p(A[f"s{lvl}"]), _p(u), N, h, w, c, self._s()), "up")
            A[f"u{lvl}"] = u
            A[f"d{lvl}"] = self._conv(f"dec{lvl}b", u, N, h, w, True, f"d{lvl}")
            prev = A[f"d{lvl}"]
        return self._conv("head", prev, N, H, W, False, "y", f32=True)

    def _layer_back(self, name, x_in, dout, out, N, H, W, want_dx=True):
        p = self.P[name]
        cout, cin = p["cout"], p["cin"]
        P = N * H * W
        dm = self._buf(f"dm_{name}", (N, H, W, cout), self.torch.bfloat16)
        self._chk(self.L.shk_nn_relu_grad(_fp(dout), _p(out), _p(dm), _fp(p["gb"]), P, cout, int(out is not None),
                                          self._s()), "relu_grad")
        self._chk(self.L.shk_nn_conv3x3_wgrad(_p(x_in), _p(dm), _fp(p["gw"]), N, H, W, cin, cout, self._s()), "wgrad")
        if not want_dx:
            return None
        dx = self._buf(f"dx_{name}", (N, H, W, cin), self.torch.float32)
        self._chk(self.L.shk_nn_conv3x3(_p(dm), _p(p["wt"]), None, None, _fp(dx), N, H, W, cout, cin, 0, 1,
                                        self._s()), "dgrad")
        return dx

    def backward(self, dY):
        A = self._acts
        N, H, W, _ = A["x0"].shape
        f32 = self.torch.float32
        for name, *_ in LAYERS:
            p = self.P[name]
            self._chk(self.L.shk_nn_zero(_fp(p["gw"]), p["gw"].numel(), self._s()), "zero")
            self._chk(self.L.shk_nn_zero(_fp(p["gb"]), p["gb"].numel(), self._s()), "zero")
        d = self._layer_back("head", A["d0"], dY, None, N, H, W)
        hs = [(H, W), (H // 2, W // 2), (H // 4, W // 4), (H // 8, W // 8)]
        ds = {}
        for lvl in (0, 1, 2):
            h, w = hs[lvl]
            du = self._layer_back(f"dec{lvl}b", A[f"u{lvl}"], d, A[f"d{lvl}"], N, h, w)
            c = self.P[f"dec{lvl}a"]["cout"]
            ds[lvl] = self._buf(f"ds{lvl}", (N, h, w, c), f32)
            self._chk(self.L.shk_nn_axpy(_fp(du), _fp(ds[lvl]), du.numel(), 0, self._s()), "axpy")
            hc, wc = hs[lvl + 1]
            dda = self._buf(f"dda{lvl}", (N, hc, wc, c), f32)
            self._chk(self.L.shk_nn_up2_grad(_fp(du), _fp(dda), N, hc, wc, c, self._s()), "up2_grad")
            src = A["s3"] if lvl == 2 else A[f"d{lvl + 1}"]
            d = self._layer_back(f"dec{lvl}a", src, dda, A[f"d{lvl}a"], N, hc, wc)
        # d is now the gradient of s3
        for lvl in (3, 2, 1, 0):
            h, w = hs[lvl]
            if lvl < 3:
                ds_l = ds[lvl]
                c = self.P[f"enc{lvl}b"]["cout"]
                self._chk(self.L.shk_nn_pool2_grad(_fp(d), _fp(ds_l), N, h, w, c, 1, self._s()), "pool2_grad")
                d = ds_l
            da = self._layer_back(f"enc{lvl}b", A[f"a{lvl}"], d, A[f"s{lvl}"], N, h, w)
            src = A["x0"] if lvl == 0 else A[f"p{lvl}"]
            d = self._layer_back(f"enc{lvl}a", src, da, A[f"a{lvl}"], N, h, w, want_dx=lvl > 0)

    def loss_and_grad(self, X, T, M=None):
        """Forward, MSE of output channel 0 against T (weights M), backward; returns the loss."""
        Y = self.forward(X)
        N, H, W, _ = X.shape
        P = N * H * W
        dY = self._buf("dY", tuple(Y.shape), self.torch.float32)
        loss = self._buf("loss", (1,), self.torch.float32)
        self._chk(self.L.shk_nn_zero(_fp(loss), 1, self._s()), "zero")
        self._chk(self.L.shk_nn_mse(_fp(Y), _fp(T), _fp(M), _fp(dY), _fp(loss), P, HEAD_C, 1.0 / P, self._s()), "mse")
        self.backward(dY)
        return loss

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_no += 1
        for name, cin, cout, _ in LAYERS:
            p = self.P[name]
            self._chk(self.L.shk_nn_adam(_fp(p["w"]), _fp(p["gw"]), _fp(p["mw"]), _fp(p["vw"]), _p(p["wb"]),
                                         _p(p["wt"]), p["w"].numel(), cout, cin, lr, b1, b2, eps, self.step_no,
                                         self._s()), "adam")
            self._chk(self.L.shk_nn_adam(_fp(p["b"]), _fp(p["gb"]), _fp(p["mb"]), _fp(p["vb"]), None, None,
                                         p["b"].numel(), cout, 1, lr, b1, b2, eps, self.step_no, self._s()), "adam")

    def train(self, X, T, M, steps: int, batch: int = 32, lr: float = 1e-3, seed: int = 0):
        """Adam on random mini-batches of the pairs (X [S,H,W,16] BF16, T/M [S,H,W] Float32)."""
        g = np.random.default_rng(seed)
        S = X.shape[0]
        out = []
        for k in range(steps):
            idx = self.torch.from_numpy(g.choice(S, size=min(batch, S), replace=False)).to(self.dev)
            xb, tb, mb = X.index_select(0, idx), T.index_select(0, idx), M.index_select(0, idx)
            loss = self.loss_and_grad(xb, tb, mb)
            self.adam_step(lr)
            out.append(loss.clone())
        vals = [float(v.item()) for v in out]
        self.losses += vals
        return vals

    # ---- use on a State -------------------------------------------------------------------------
    def pack(self, state, Hp=None, Wp=None):
        g = state.grid
        Hp = Hp or (g.ny + 7) // 8 * 8
        Wp = Wp or (g.nx + 7) // 8 * 8
        X = self._buf("pack", (1, Hp, Wp, 16), self.torch.bfloat16)
        st = state.struct()
        self._chk(self.L.shk_nn_pack_state(C.byref(st), g.nx, g.ny, Hp, Wp, _fp(self.norm), _p(X), self._s()), "pack")
        return X

    def predict_into(self, state, out):
        """out (Float64 like state.h) = h + predicted increment on GROUNDED cells."""
        g = state.grid
        X = self.pack(state)
        Y = self.forward(X)
        Wp = X.shape[2]
        self._chk(self.L.shk_nn_apply_increment(_fp(Y), HEAD_C, g.nx, g.ny, Wp, self.dh_scale, _p(state.h),
                                                _p(state.mask), _p(out), self._s()), "apply")
        return out


def _one_picard(sim):
    """One Picard iteration of the simulation's solver (update_ieb! first); returns its stats."""
    from .simulation import update_ieb
    update_ieb(sim)
    ctx = sim.ctx()
    ps = sim.hs.ps
    po, o = ps.opts(), ps.ls.opts()
    po.iters = 1
    st = _lib.shk_picard_stats()
    rc = ctx.L.shk_picard_solve(ctx.h, C.byref(po), C.byref(o), C.byref(st))
    _lib.check(ctx.h, rc, allow=(_lib.OK, _lib.NOT_CONVERGED))
    return st


def step_seeded(sim, net: WarmStartNet, stats: dict | None = None, smooth: int = 8, omega: float = 0.8):
    """step! with the learned warm start.

    The first Picard iteration's system is assembled at the current head as usual; the network
    predicts that iteration's solution (the first Picard iterate), `smooth` damped Jacobi sweeps of
    that system remove the prediction's rough error, and the result becomes the initial guess of
    that iteration's CG solve only when its initial residual ||b - A x0|| in this system is below
    the current head's -- otherwise the solve starts from the current head
    (the fallback, i.e. the unseeded method).  Every solve still runs to its tolerance and Picard
    to its own, so the timestep's result is the unseeded method's up to those tolerances."""
    from .simulation import update_ieb, step_h, step_b
    update_ieb(sim)
    ctx = sim.ctx()
    L = ctx.L
    r0, b0, r1, b1 = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    _lib.check(ctx.h, L.shk_initial_residual(ctx.h, C.byref(r0), C.byref(b0)))
    seed = net._buf("seed", tuple(sim.state.h.shape), net.torch.float64)
    net.predict_into(sim.state, seed)
    if smooth:  # the network's rough error components cost residual out of proportion: damp them
        tmp = net._buf("seed_tmp", tuple(sim.state.h.shape), net.torch.float64)
        _lib.check(ctx.h, L.shk_smooth_guess(ctx.h, _p(seed), _p(tmp), int(smooth), float(omega)))
    _lib.check(ctx.h, L.shk_residual_of(ctx.h, _p(seed), C.byref(r1), C.byref(b1)))
    used = r1.value < r0.value
    if used:
        _lib.check(ctx.h, L.shk_set_cg_warm_start(ctx.h, _p(seed)))
    step_h(sim)
    _lib.check(ctx.h, L.shk_set_cg_warm_start(ctx.h, None))
    step_b(sim)
    if stats is not None:
        stats.setdefault("seeded", []).append(bool(used))
        stats.setdefault("r_prev", []).append(r0.value / max(b0.value, 1e-300))
        stats.setdefault("r_seed", []).append(r1.value / max(b1.value, 1e-300))
    return used


# ---------------------------------------------------------------------------------------------
# Training data from ensemble runs of the plain solver, training, and evaluation
# ---------------------------------------------------------------------------------------------
def member_sim(shk, spec: dict, rtol: float = 1e-8, params: dict | None = None, picard_iters: int = 500,
               multigrid: bool = False):
    """A Simulation of one ensemble member (configs.ensemble_member) with the plain Float64 Jacobi
    CG (or the multigrid-preconditioned one) at rel-res `rtol` and Picard(picard_iters, 1e-6)."""
    w = shk.configs.ensemble_member(**spec)
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    pm = shk.ModelParameters(**(params if params is not None else shk.configs.SEASONAL_PARAMS))
    sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
    st = shk.State(g)
    shk.set_initial_conditions(st, g, pm, sl, **w.inputs)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, stop_rule="relres", rtol=rtol, atol=0.0,
                               multigrid=multigrid)
    ps = shk.PicardSolver(picard_iters, 1e-6, ls, g)
    return shk.Simulation(g, st, 1, 1800.0, pm, "implicit", [], shk.ConstantMeltInput(), sl, ps=ps)


def field_stats(sims):
    """Means and spreads of the input fields over the GROUNDED cells of the given states (host)."""
    vals = {f: [] for f in IN_FIELDS}
    for s in sims:
        a = s.state.to_numpy(list(IN_FIELDS))
        for f in IN_FIELDS:
            vals[f].append(a[f].ravel())
    means, spreads = [], []
    for f in IN_FIELDS:
        v = np.concatenate(vals[f])
        m, sd = float(v.mean()), float(v.std())
        means.append(m)
        spreads.append(sd if sd > 0 else 1.0)
    return means, spreads


def generate_pairs(shk, net: WarmStartNet, specs, steps: int, crops: int = 4, crop: int = 32, seed: int = 0,
                   settle: int = 3, picard_iters: int = 100):
    """(input, increment) pairs from an ensemble run of the plain solver: before each of `steps`
    timesteps every instance's state is packed (the network's input), and the increment of the
    timestep's first Picard iterate over the head, G(h(t)) - h(t), is the target; `crops` random crop x crop windows per instance-step whose Picard loop
    converged.  The first `settle` steps (the start-up transient) are run but not recorded, and the
    network's normalisation is set from the states after them; increments are scaled by their
    95th-percentile magnitude.  Returns X [S,crop,crop,16] BF16, T [S,crop,crop] Float32
    (normalised increments), M [S,crop,crop] (1 on GROUNDED)."""
    import torch
    from .ensemble import Ensemble
    sims = [member_sim(shk, sp, picard_iters=picard_iters) for sp in specs]
    ens = Ensemble(sims, autotune_iters=0)
    if settle:
        ens.run(settle)
    means, spreads = field_stats(sims)
    g = np.random.default_rng(seed)
    Xs, Ts, Ms, dhs = [], [], [], []
    net.set_normalisation(means, spreads, 1.0)
    snaps = [torch.empty_like(s.state.h) for s in sims]
    ens.set_snapshots(snaps)
    for k in range(steps):
        packs = [net.pack(s.state).clone() for s in sims]
        h0 = [s.state.h.clone() for s in sims]
        st = ens.run(1)
        for s, X, hb, si, h1 in zip(sims, packs, h0, st, snaps):
            if not si["last_converged"]:
                continue
            gx, gy = s.grid.nx, s.grid.ny
            dh = (h1 - hb).t()                 # (ny, nx)
            msk = (s.state.mask.t() == 0).float()
            for _ in range(crops):
                y0 = int(g.integers(0, max(1, gy - crop + 1)))
                x0 = int(g.integers(0, max(1, gx - crop + 1)))
                Xs.append(X[0, y0:y0 + crop, x0:x0 + crop])
                Ts.append(dh[y0:y0 + crop, x0:x0 + crop].float())
                Ms.append(msk[y0:y0 + crop, x0:x0 + crop])
                dhs.append(dh[y0:y0 + crop, x0:x0 + crop][msk[y0:y0 + crop, x0:x0 + crop] > 0])
    ens.close()
    allv = torch.cat([d.flatten() for d in dhs]).abs()
    dh_scale = float(torch.quantile(allv[:1 << 24].float(), 0.95).item()) if allv.numel() > 1 else 1.0
    dh_scale = dh_scale if dh_scale > 0 else 1.0
    net.dh_scale = dh_scale
    X = torch.stack(Xs).contiguous()
    T = (torch.stack(Ts) / dh_scale).contiguous()
    M = torch.stack(Ms).contiguous()
    return X, T, M


def evaluate(shk, net: WarmStartNet, spec: dict, steps: int, settle: int = 1, multigrid: bool = False):
    """The same instance advanced `steps` timesteps unseeded and with the learned seed (after
    `settle` common steps); per-step CG and Picard iterations, device time, and the seeded head's
    error against the unseeded one."""
    import torch
    out = {}
    runs = {}
    for mode in ("unseeded", "seeded"):
        sim = member_sim(shk, spec, multigrid=multigrid)
        for _ in range(settle):
            shk.step(sim)
            sim.total_time += sim.dt
        rec = []
        stats = {}
        for _ in range(steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if mode == "seeded":
                step_seeded(sim, net, stats)
            else:
                shk.step(sim)
            e1.record()
            torch.cuda.synchronize()
            sim.total_time += sim.dt
            ps = sim.hs.ps
            rec.append(dict(picard=ps.last_iter, cg=ps.cg_iters_total, converged=ps.converged,
                            ms=round(e0.elapsed_time(e1), 3)))
        runs[mode] = sim
        out[mode] = dict(per_step=rec, cg_per_step=float(np.mean([r["cg"] for r in rec])),
                         picard_per_step=float(np.mean([r["picard"] for r in rec])),
                         ms_per_step=float(np.mean([r["ms"] for r in rec])), **({"seed": stats} if stats else {}))
    hu = runs["unseeded"].state.h.cpu().numpy()
    hs = runs["seeded"].state.h.cpu().numpy()
    out["h_relerr_vs_unseeded"] = float(np.max(np.abs(hs - hu)) / np.max(np.abs(hu)))
    return out
