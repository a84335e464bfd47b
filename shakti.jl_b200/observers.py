"""File observers: IOObserver and its writers (src/observer.jl:59-72,139-335).

The reference records the tracked State fields at the tracked timesteps into a file:
  NetCDFFileWriter  one variable per field, shape (field shape..., ntimes) plus "time"
  HDF5FileWriter    the same layout in HDF5
  JLD2FileWriter    one key per field and tracked time ("name/idx", "total_time/idx")
  CSVFileWriter     one row per tracked time: t, total_time, name_min, name_max, name_mean

Here the NetCDF file is written in the NetCDF classic format by this module (CDF-2, the 64-bit
offset variant, or CDF-5 when a variable exceeds 4 GiB), with the reference's names: a dimension
"time" of length len(tracked_times), dimensions "<name>_x" and "<name>_y" per field, and variables
of file shape (time, <name>_y, <name>_x) -- the Julia (x, y, time) column-major array, so the
time slice of a field is its device array byte for byte.  JLD2 is a Julia format: its writer keeps
the reference's key layout in an npz (zip) archive.  HDF5 needs a library this environment lacks
and raises.  CSV statistics are reduced on the device.

Overlap: at a tracked step the fields are copied on the device into a staging slot (a
device-to-device copy on the solve's stream), copied to pinned host memory on a separate copy
stream, and written to the file by a worker thread, while the following timesteps run.  Two
staging slots: a third tracked step waits only for the first slot's write.
"""
from __future__ import annotations

import concurrent.futures as cf
import csv
import os
import struct
import zipfile
from io import BytesIO

import numpy as np

_NC_DIMENSION, _NC_VARIABLE, _NC_DOUBLE = 10, 11, 6


class AbstractFileWriter:
    ext = ""


class NetCDFFileWriter(AbstractFileWriter):
    """NetCDF classic (src/observer.jl:17, openfile!/write2file! :129-140, :240-248)."""


class HDF5FileWriter(AbstractFileWriter):
    """src/observer.jl:24; needs an HDF5 library, which this environment does not have."""


class JLD2FileWriter(AbstractFileWriter):
    """src/observer.jl:32; the key layout ("tracked_obs", "tracked_times", "name/idx",
    "total_time/idx") in an npz archive: JLD2 is a Julia format."""


class CSVFileWriter(AbstractFileWriter):
    """src/observer.jl:40; one row of min/max/mean per tracked time."""


FILE_WRITERS = {"NetCDF": NetCDFFileWriter, "HDF5": HDF5FileWriter, "JLD2": JLD2FileWriter, "CSV": CSVFileWriter}


# ---------------------------------------------------------------------------------------------
# NetCDF classic: header and fixed-size variables (big-endian)
# ---------------------------------------------------------------------------------------------
def _pad4(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 4)


class _NcLayout:
    """Header bytes and each variable's data offset for fixed-size Float64 variables."""

    def __init__(self, dims: list[tuple[str, int]], vars_: list[tuple[str, list[int]]]):
        sizes = {}
        for v, dimids in vars_:
            n = 8
            for d in dimids:
                n *= dims[d][1]
            sizes[v] = n
        # CDF-2 stores vsize in 32 bits: every variable but the last must stay below 4 GiB
        self.version = 5 if any(s >= (1 << 32) - 4 for s in sizes.values()) else 2
        big = self.version == 5
        cnt = (lambda v: struct.pack(">q", v)) if big else (lambda v: struct.pack(">i", v))
        off = lambda v: struct.pack(">q", v)  # noqa: E731 (CDF-2 and CDF-5 offsets are 64-bit)

        def name(s: str) -> bytes:
            b = s.encode()
            return cnt(len(b)) + _pad4(b)

        def header(begins):
            h = b"CDF" + bytes([self.version]) + cnt(0)
            h += struct.pack(">i", _NC_DIMENSION) + cnt(len(dims))
            for nm, ln in dims:
                h += name(nm) + cnt(ln)
            h += struct.pack(">i", 0) + cnt(0)  # no global attributes (ABSENT)
            h += struct.pack(">i", _NC_VARIABLE) + cnt(len(vars_))
            for (nm, dimids), b in zip(vars_, begins):
                h += name(nm) + cnt(len(dimids))
                for d in dimids:
                    h += cnt(d)
                h += struct.pack(">i", 0) + cnt(0)  # no variable attributes
                vs = sizes[nm]
                h += struct.pack(">i", _NC_DOUBLE) + (cnt(vs) if big else struct.pack(">I", min(vs, (1 << 32) - 1)))
                h += off(b)
            return h

        hlen = len(header([0] * len(vars_)))
        begins, pos = [], hlen
        for nm, _ in vars_:
            begins.append(pos)
            pos += sizes[nm]
        self.header = header(begins)
        self.begin = {nm: b for (nm, _), b in zip(vars_, begins)}
        self.size = sizes
        self.total = pos


class _NetCDFFile:
    def __init__(self, path: str, fields: dict, ntimes: int, resume: bool):
        dims = [("time", ntimes)]
        vars_ = [("time", [0])]
        for nm, shape in fields.items():
            dims += [(f"{nm}_x", shape[0]), (f"{nm}_y", shape[1])]
            vars_.append((nm, [0, len(dims) - 1, len(dims) - 2]))  # (time, y, x): Julia (x, y, time)
        self.L = _NcLayout(dims, vars_)
        self.shapes = fields
        if resume and os.path.exists(path):
            self.fh = open(path, "r+b")
        else:
            self.fh = open(path, "w+b")
            self.fh.write(self.L.header)
            self.fh.truncate(self.L.total)

    def write(self, idx: int, total_time: float, host: dict) -> None:
        fh, L = self.fh, self.L
        fh.seek(L.begin["time"] + 8 * idx)
        fh.write(struct.pack(">d", total_time))
        for nm, a in host.items():
            nx, ny = self.shapes[nm]
            fh.seek(L.begin[nm] + idx * nx * ny * 8)
            # the column-major (nx, ny) slice is the C-ordered (y, x) record; stored big-endian
            fh.write(np.asarray(a, dtype=">f8").tobytes(order="F"))
        fh.flush()

    def close(self) -> None:
        self.fh.close()


# ---------------------------------------------------------------------------------------------
# IOObserver
# ---------------------------------------------------------------------------------------------
def _csv_columns(tracked_obs):
    return ["t", "total_time"] + [f"{n}{s}" for n in tracked_obs for s in ("_min", "_max", "_mean")]


class IOObserver:
    """IOObserver(tracked_obs, tracked_times, fr, path) (src/observer.jl:66-79)."""

    def __init__(self, tracked_obs, tracked_times, fr: AbstractFileWriter, path: str):
        if isinstance(fr, type):
            fr = fr()
        if isinstance(fr, HDF5FileWriter):
            raise RuntimeError("HDF5FileWriter needs an HDF5 library (HDF5.jl in the reference); none is available "
                               "here -- use NetCDFFileWriter, JLD2FileWriter or CSVFileWriter")
        self.tracked_obs = list(tracked_obs)
        self.tracked_times = [int(t) for t in tracked_times]
        self.fr = fr
        self.path = str(path)
        self.handle = None
        self._pool = None
        self._slots = []
        self._pending = []

    # -- staging: device snapshot, pinned host copy on a copy stream, file write on a thread -----
    def _start(self, state):
        import torch
        self._pool = cf.ThreadPoolExecutor(max_workers=1)
        self._stream = torch.cuda.Stream()
        if isinstance(self.fr, CSVFileWriter):
            return
        self._slots = []
        for _ in range(2):
            dev = {n: torch.empty_like(state[n]) for n in self.tracked_obs}
            host = {n: torch.empty(tuple(reversed(state[n].shape)), dtype=state[n].dtype).pin_memory().t()
                    for n in self.tracked_obs}
            self._slots.append(dict(dev=dev, host=host, future=None, event=torch.cuda.Event()))
        self._next = 0

    def _shapes(self, state):
        return {n: tuple(state[n].shape) for n in self.tracked_obs}

    def prepare(self, state):
        """prepare! / openfile! (src/observer.jl:112-176)."""
        self._start(state)
        if isinstance(self.fr, NetCDFFileWriter):
            self.handle = _NetCDFFile(self.path, self._shapes(state), len(self.tracked_times), resume=False)
        elif isinstance(self.fr, JLD2FileWriter):
            with zipfile.ZipFile(self.path, "w") as z:
                _npz_put(z, "tracked_obs", np.array(self.tracked_obs))
                _npz_put(z, "tracked_times", np.array(self.tracked_times))
            self.handle = self.path
        else:
            with open(self.path, "w", newline="") as fh:
                csv.writer(fh).writerow(_csv_columns(self.tracked_obs))
            self.handle = self.path

    def resume(self, state, resume_t: int):
        """resume! / reopenfile! (src/observer.jl:178-234): continue writing into the same file."""
        self._start(state)
        if isinstance(self.fr, NetCDFFileWriter):
            self.handle = _NetCDFFile(self.path, self._shapes(state), len(self.tracked_times), resume=True)
        elif isinstance(self.fr, JLD2FileWriter):
            self.handle = self.path
        else:  # drop rows a crashed run wrote after the checkpoint
            with open(self.path, newline="") as fh:
                rows = list(csv.reader(fh))
            keep = [rows[0]] + [r for r in rows[1:] if int(r[0]) <= resume_t]
            with open(self.path, "w", newline="") as fh:
                csv.writer(fh).writerows(keep)
            self.handle = self.path

    def observe(self, state, t, total_time):
        """observe! / write2file! (src/observer.jl:236-300)."""
        if t not in self.tracked_times:
            return
        idx = self.tracked_times.index(t)
        import torch
        if isinstance(self.fr, CSVFileWriter):
            stats = []
            for n in self.tracked_obs:
                f = state[n]
                mn, mx = torch.aminmax(f)
                stats.append(torch.stack([mn, mx, f.mean()]))
            vals = torch.cat(stats).cpu().tolist()
            row = [t, repr(float(total_time))] + [repr(v) for v in vals]
            self._pending.append(self._pool.submit(_csv_append, self.path, row))
            return
        slot = self._slots[self._next]
        self._next ^= 1
        if slot["future"] is not None:  # this slot's previous write
            slot["future"].result()
        main = torch.cuda.current_stream()
        for n in self.tracked_obs:
            slot["dev"][n].copy_(state[n])
        done_dev = torch.cuda.Event()
        done_dev.record(main)
        with torch.cuda.stream(self._stream):
            self._stream.wait_event(done_dev)
            for n in self.tracked_obs:
                slot["host"][n].copy_(slot["dev"][n], non_blocking=True)
            slot["event"].record(self._stream)
        # the staging slot is free for the solve once its device copy is done; the file write waits
        # for the host copy on the worker thread
        ev, host = slot["event"], slot["host"]
        slot["future"] = self._pool.submit(self._write, idx, float(total_time), ev, host)

    def _write(self, idx, total_time, ev, host):
        ev.synchronize()
        arrays = {n: host[n].numpy() for n in self.tracked_obs}
        if isinstance(self.fr, NetCDFFileWriter):
            self.handle.write(idx, total_time, arrays)
        else:
            with zipfile.ZipFile(self.path, "a") as z:
                _npz_put(z, f"total_time/{idx + 1}", np.array(total_time))
                for n, a in arrays.items():
                    _npz_put(z, f"{n}/{idx + 1}", np.asfortranarray(a))

    def finalize(self, state):
        """finalize! / close_handle! (src/observer.jl:302-335): waits for every pending write."""
        for s in self._slots:
            if s["future"] is not None:
                s["future"].result()
        for f in self._pending:
            f.result()
        if isinstance(self.fr, NetCDFFileWriter) and self.handle is not None:
            self.handle.close()
        if self._pool is not None:
            self._pool.shutdown(wait=True)


def _csv_append(path, row):
    with open(path, "a", newline="") as fh:
        csv.writer(fh).writerow(row)


def _npz_put(z: zipfile.ZipFile, key: str, a: np.ndarray) -> None:
    """Adds (or, on a resumed run, replaces) key.npy in the archive, as np.savez names members."""
    buf = BytesIO()
    np.save(buf, a, allow_pickle=False)
    # a zip member cannot be replaced in place: a resumed run appends the key again, and the later
    # member wins on load (load_jld2_standin)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", UserWarning)  # zipfile's "Duplicate name"
        z.writestr(key + ".npy", buf.getvalue())


def load_jld2_standin(path: str) -> dict:
    """The JLD2 stand-in's keys -> arrays (the last written member of each key)."""
    out = {}
    with zipfile.ZipFile(path) as z:
        for info in z.infolist():
            with z.open(info) as fh:
                out[info.filename[:-4]] = np.load(BytesIO(fh.read()), allow_pickle=False)
    return out
