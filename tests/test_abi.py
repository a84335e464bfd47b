"""The C ABI library loads and exports every symbol include/shakti_b200.h declares; the Python
binding's signature table matches the header.  No compute calls (runs without a GPU)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "shakti_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"SHK_API\s+[^;(]*?\b(shk_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in ("shk_create", "shk_picard_solve", "shk_cg_solve", "shk_run", "shk_destroy"):
        assert s in syms


def test_library_exports_every_declared_symbol(shk):
    from shakti_b200 import _lib
    L = _lib.load()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_binding_table_covers_header(shk):
    from shakti_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared_symbols()


def test_version_and_status_strings(shk):
    from shakti_b200 import _lib
    L = _lib.load()
    assert L.shk_version() >= 1
    assert L.shk_status_string(0) == b"ok"
    assert L.shk_status_string(2) == b"breakdown"


def test_struct_layouts_match_header(shk, tmp_path):
    """ctypes mirrors of the C structs have the sizes and field offsets gcc gives the header."""
    import shutil
    import subprocess
    from shakti_b200 import _lib
    cc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else shutil.which("gcc")
    structs = {"shk_params": _lib.shk_params, "shk_state": _lib.shk_state, "shk_cg_opts": _lib.shk_cg_opts,
               "shk_cg_stats": _lib.shk_cg_stats, "shk_picard_opts": _lib.shk_picard_opts,
               "shk_picard_stats": _lib.shk_picard_stats, "shk_melt_input": _lib.shk_melt_input,
               "shk_sliding_law": _lib.shk_sliding_law, "shk_ensemble_stats": _lib.shk_ensemble_stats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            cname = "lambda" if fname == "lambda_" else fname
            lines.append(f'  printf("{name}.{fname} %zu\\n", offsetof({name}, {cname}));')
    lines.append("  return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                           check=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(out[name]) == ctypes.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(out[f"{name}.{fname}"]) == getattr(cls, fname).offset, (name, fname)


def test_package_fails_loudly_without_gpu(shk):
    """No CPU fallback: constructing device state without CUDA raises."""
    import pytest
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    g = shk.Grid(6, 6, 1e3, 1e3)
    with pytest.raises(RuntimeError):
        shk.State(g)
    with pytest.raises(RuntimeError):
        shk.CGIterativeSolver(g, shk.MatrixFreeLinearSystem)
