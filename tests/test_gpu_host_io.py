"""HostIO: runs fed from and returned to pinned host memory, with the transfers on two copy streams
overlapping the solve, follow the device-resident run bit for bit."""
import numpy as np
import pytest
import torch

from test_gpu_parity import setup_pair

pytestmark = pytest.mark.gpu


def make_sim(shk, orc, cuda, w, tsteps):
    g, pm, sl, osl, s, st = setup_pair(shk, orc, cuda, w)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem)
    ps = shk.PicardSolver(500, 1e-6, ls, g)
    return shk.Simulation(g, s, tsteps, 3600.0, pm, "implicit", [], shk.ConstantMeltInput(), sl, ps=ps)


def test_host_io_run_matches_device_run(shk, orc, cuda):
    steps = 5
    w = shk.configs.plain64()
    ref = make_sim(shk, orc, cuda, w, steps)
    base = ref.state.ieb.t().cpu().clone()
    forcings = [(base * (1.0 + 0.25 * k)).pin_memory() for k in range(steps)]
    ref_h, ref_b = [], []
    for k in range(steps):  # the same steps with the input set on the device
        ref.state.ieb.t().copy_(forcings[k].cuda())
        shk.step_h(ref)
        shk.step_b(ref)
        ref.total_time += ref.dt
        ref_h.append(ref.state.h.t().cpu().clone())
        ref_b.append(ref.state.b.t().cpu().clone())
    assert not torch.equal(ref_h[1], ref_h[0])

    sim = make_sim(shk, orc, cuda, w, steps)
    io = shk.HostIO(sim)
    hs = [torch.empty_like(x).pin_memory() for x in ref_h]
    bs = [torch.empty_like(x).pin_memory() for x in ref_b]
    io.run(forcings, hs, bs)
    torch.cuda.synchronize()
    for k in range(steps):
        assert torch.equal(hs[k], ref_h[k]) and torch.equal(bs[k], ref_b[k]), k
    assert torch.equal(sim.state.h, ref.state.h) and torch.equal(sim.state.b, ref.state.b)
    assert sim.total_time == ref.total_time

    # one reused output tensor ends holding the last step; a second call continues the run
    sim2 = make_sim(shk, orc, cuda, w, steps)
    io2 = shk.HostIO(sim2)
    h1 = torch.empty_like(ref_h[0]).pin_memory()
    io2.run(forcings[:2], h1, None)
    io2.run(forcings[2:], h1, None)
    torch.cuda.synchronize()
    assert torch.equal(h1, ref_h[-1])
    assert np.array_equal(sim2.state.b.cpu().numpy(), ref.state.b.cpu().numpy())
