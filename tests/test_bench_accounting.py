"""bench.py's algorithmic byte counts (the roofline numerator), on CPU: per-cell figures of one CG
iteration for each form, and the multigrid V-cycle's sum over the levels of a 4096^2 hierarchy
(levels 1-6 on tile kernels, levels 7-12 -- at most 1400 cells -- in the one-block bottom kernel)."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_plain_iteration_bytes():
    n = 4096 * 4096
    assert bench.iteration_bytes("plain", 4096, 4096) == 112 * n   # 14 Float64 words per cell
    assert bench.iteration_bytes("fp32cg", 4096, 4096) == 56 * n    # the same words in Float32


def test_multigrid_iteration_bytes(monkeypatch):
    monkeypatch.delenv("SHK_MG_FUSED", raising=False)
    n0 = 4096 * 4096
    # matvec 56 B + level 0 (100 B: descending half with the CG's r update and, every second
    # iteration, its x update -- 62 B on average -- ascending half 38 B) + levels 1-6 at 56 B per
    # level cell + the bottom (25 B at level 7, 17 B below)
    coarse = sum((4096 >> l) ** 2 for l in range(1, 7))
    bottom = 25 * 32 * 32 + 17 * sum((32 >> k) ** 2 for k in range(1, 6))
    expect = 56 * n0 + 100 * n0 + 56 * coarse + bottom
    assert bench.iteration_bytes("multigrid", 4096, 4096) == expect
    assert abs(expect / n0 - 174.66) < 0.01


def test_step_bytes():
    n = 4096 * 4096
    counts = {"picard_iters": 46, "cg_iters": 160, "steps": 16}
    expect = (46 * 43 * 8 * n + 160 * bench.iteration_bytes("multigrid", 4096, 4096) + 16 * 11 * 8 * n) / 16
    assert bench.step_bytes("multigrid", 4096, 4096, counts) == expect

    class W:
        nx = ny = 4096

    r = bench.step_roofline("multigrid", W, counts, 14.56, {"hbm_gbs": 6539.0})
    assert r["peak"] == 6539.0 and abs(r["achieved"] - expect / 14.56e-3 / 1e9) < 0.1
    assert r["peak_source"].endswith("(of measured)")
