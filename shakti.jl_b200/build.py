"""Builds libshakti_b200.so (sm_100a) in-tree with nvcc.

The library is plain CUDA C++ behind a C ABI (include/shakti_b200.h); it links only the CUDA
runtime.  --fmad=false keeps every a*b+c as two rounded operations so the field kernels and the
Float64 CG reproduce the reference's unfused Float64 arithmetic bit for bit.  The multigrid
preconditioner and the warm-start network carry no such parity requirement and are compiled with
fused multiply-adds.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libshakti_b200.so"
SOURCES = ["shk_api.cu", "shk_fields.cu", "shk_krylov.cu", "shk_mg.cu", "shk_ensemble.cu", "shk_nn.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FMAD = {"shk_mg.cu", "shk_nn.cu"}  # sources compiled with --fmad=true


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list[str]:
    # /usr/bin/g++ is the system compiler nvcc supports; an exported CXX may be a wrapper.
    return ["-ccbin", "/usr/bin/g++"] if Path("/usr/bin/g++").exists() else []


def sources() -> list[Path]:
    return [CSRC / s for s in SOURCES]


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "shakti_b200.h", Path(__file__)]
    return all(d.stat().st_mtime <= t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    if not force and up_to_date():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    common = [nvcc(), *host_compiler(), *ARCH, "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", str(ROOT / "include"),
              "--expt-relaxed-constexpr", "--extended-lambda"]
    if verbose:
        common += ["-Xptxas", "-v"]
    common += list(extra or [])
    for src in sources():
        obj = objdir / (src.stem + ".o")
        fmad = "--fmad=true" if src.name in FMAD else "--fmad=false"
        cmd = [*common, fmad, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *host_compiler(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
