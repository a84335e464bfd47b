"""IOObserver (src/observer.jl) through run(): the NetCDF, CSV and JLD2-layout files hold exactly
what an in-memory LiveObserver records for the same run, and a run restarted from a checkpoint
continues writing into the same file (resume!)."""
import csv

import numpy as np
import pytest
import scipy.io

pytestmark = pytest.mark.gpu

OBS = ["h", "N", "b", "q_x"]
TIMES = [0, 2, 3, 5]


def make(shk, w, which, writer=None, path=None, tsteps=5):
    g = shk.Grid(w.nx, w.ny, w.lx, w.ly)
    p = shk.ModelParameters()
    sl = shk.RegularizedCoulombSlidingLaw(w.sliding_C)
    s = shk.State(g)
    shk.set_initial_conditions(s, g, p, sl, **w.inputs)
    ls = shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem, chebyshev_degree=4)
    return shk.Simulation(g, s, tsteps, 3600.0, p, "implicit", OBS, shk.ConstantMeltInput(), sl,
                          ps=shk.PicardSolver(500, 1e-6, ls, g), which_observer=which, which_file_writer=writer,
                          tracked_times=TIMES, path=path)


def live(shk, w):
    sim = make(shk, w, "Live")
    shk.run(sim)
    return sim.observer


def test_netcdf_observer_matches_live(shk, cuda, tmp_path):
    w = shk.configs.plain64()
    ref = live(shk, w)
    path = str(tmp_path / "run.nc")
    shk.run(make(shk, w, "IO", "NetCDF", path))
    with scipy.io.netcdf_file(path, "r", mmap=False) as nc:
        assert np.array_equal(nc.variables["time"][:], ref.times)
        for n in OBS:
            for k in range(len(TIMES)):
                assert np.array_equal(nc.variables[n][k].T, ref.data[n][k]), (n, k)


def test_netcdf_observer_resumes_after_restart(shk, cuda, tmp_path):
    w = shk.configs.plain64()
    ref = live(shk, w)
    path, ck = str(tmp_path / "run.nc"), str(tmp_path / "ck.npz")
    shk.run(make(shk, w, "IO", "NetCDF", path, tsteps=3), checkpoint_every=3, checkpoint_path=ck)
    shk.run(make(shk, w, "IO", "NetCDF", path, tsteps=5), restart_path=ck)
    with scipy.io.netcdf_file(path, "r", mmap=False) as nc:
        for n in OBS:
            for k in range(len(TIMES)):
                assert np.array_equal(nc.variables[n][k].T, ref.data[n][k]), (n, k)


def test_csv_and_jld2_layout_observers(shk, cuda, tmp_path):
    from shakti_b200 import observers
    w = shk.configs.plain64()
    ref = live(shk, w)
    pcsv, pj = str(tmp_path / "run.csv"), str(tmp_path / "run.jld2.npz")
    shk.run(make(shk, w, "IO", "CSV", pcsv))
    shk.run(make(shk, w, "IO", "JLD2", pj))
    with open(pcsv, newline="") as fh:
        rows = list(csv.reader(fh))
    assert rows[0] == ["t", "total_time"] + [f"{n}{s}" for n in OBS for s in ("_min", "_max", "_mean")]
    assert [int(r[0]) for r in rows[1:]] == TIMES
    for k, r in enumerate(rows[1:]):
        assert float(r[1]) == ref.times[k]
        for j, n in enumerate(OBS):
            a = ref.data[n][k]
            mn, mx, mean = (float(v) for v in r[2 + 3 * j:5 + 3 * j])
            assert mn == a.min() and mx == a.max() and mean == pytest.approx(a.mean(), rel=1e-12)
    d = observers.load_jld2_standin(pj)
    assert list(d["tracked_obs"]) == OBS and list(d["tracked_times"]) == TIMES
    for k in range(len(TIMES)):
        assert float(d[f"total_time/{k + 1}"]) == ref.times[k]
        for n in OBS:
            assert np.array_equal(d[f"{n}/{k + 1}"], ref.data[n][k])


def test_io_observer_validation(shk, cuda, tmp_path):
    w = shk.configs.fixture6()
    with pytest.raises(ValueError, match="which_file_writer"):
        make(shk, w, "IO")
    with pytest.raises(ValueError, match="Unknown which_file_writer"):
        make(shk, w, "IO", "XLS", str(tmp_path / "x"))
    with pytest.raises(RuntimeError, match="HDF5"):
        make(shk, w, "IO", "HDF5", str(tmp_path / "x.h5"))
