"""The NetCDF classic writer of IOObserver (no GPU): files it writes are read back by SciPy's
independent NetCDF reader with the reference's layout -- dimension "time" and "<name>_x",
"<name>_y" per field, variable file shape (time, <name>_y, <name>_x), i.e. the Julia
(x, y, time) array -- and variables above 4 GiB switch the header to CDF-5."""
import numpy as np
import scipy.io


def test_netcdf_file_reads_back(shk, tmp_path):
    from shakti_b200 import observers
    rng = np.random.default_rng(3)
    shapes = {"h": (7, 5), "q_x": (8, 5)}
    path = str(tmp_path / "out.nc")
    f = observers._NetCDFFile(path, shapes, ntimes=3, resume=False)
    data = {k: [np.asfortranarray(rng.normal(size=s)) for _ in range(3)] for k, s in shapes.items()}
    for idx in (2, 0, 1):  # any order, like a resumed run
        f.write(idx, 1800.0 * idx, {k: data[k][idx] for k in shapes})
    f.close()
    with scipy.io.netcdf_file(path, "r", mmap=False) as nc:
        assert nc.version_byte == 2
        assert nc.dimensions["time"] == 3 and nc.dimensions["h_x"] == 7 and nc.dimensions["h_y"] == 5
        assert nc.variables["h"].dimensions == ("time", "h_y", "h_x")
        assert np.array_equal(nc.variables["time"][:], [0.0, 1800.0, 3600.0])
        for k in shapes:
            for idx in range(3):
                assert np.array_equal(nc.variables[k][idx].T, data[k][idx])


def test_netcdf_large_variables_use_cdf5(shk):
    from shakti_b200 import observers
    L = observers._NcLayout([("time", 40), ("h_x", 4096), ("h_y", 4096)], [("time", [0]), ("h", [0, 2, 1])])
    assert L.version == 5 and L.header[:4] == b"CDF\x05"
    assert L.size["h"] == 40 * 4096 * 4096 * 8
    L2 = observers._NcLayout([("time", 2), ("h_x", 64), ("h_y", 64)], [("time", [0]), ("h", [0, 2, 1])])
    assert L2.version == 2 and L2.header[:4] == b"CDF\x02"
