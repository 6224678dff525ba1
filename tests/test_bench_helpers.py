"""bench.py's accounting on CPU: face-site counts per launch, and the
per-kernel table's GB/s, fraction of peak and GFLOP/s (1872 flops per site
of a D application)."""
import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
import bench  # noqa: E402


def test_face_sites_per_launch():
    # one colour of the reference partition at 32^3x64: one 16x32x32x64 block,
    # all but its 14x30x30x62 interior
    assert bench.sites_per_launch("dslash_face_f32", (32, 32, 32, 64), (2, 1, 1, 1), 1) == \
        16 * 32 * 32 * 64 - 14 * 30 * 30 * 62
    # 16 blocks of 4^4 per colour at 8^4 with NB (2,2,2,2), 2 RHS
    assert bench.sites_per_launch("dslash_face_f16", (8, 8, 8, 8), (2, 2, 2, 2), 2) == \
        8 * (256 - 16) * 2
    assert bench.sites_per_launch("dslash_full_f64", (8, 8, 8, 8), (2, 2, 2, 2), 1) == 4096
    assert bench.sites_per_launch("jinv_step_f32", (8, 8, 8, 8), (2, 2, 2, 2), 4) == 2048 * 4


def test_kernel_table():
    L, NB = (32, 32, 32, 64), (2, 1, 1, 1)
    Vh = 32 * 32 * 32 * 64 // 2
    # 10 launches of 1 ms each moving 768 B per site on Vh sites
    t = bench.kernel_table({"jinv_step_f32": (10, 10.0, 10 * 768.0 * Vh)}, 6546.2, L, NB)
    row = t["jinv_step_f32"]
    assert row["share"] == 1.0
    assert row["GBps"] == pytest.approx(768.0 * Vh / 1e-3 / 1e9, rel=1e-3)
    assert row["frac_of_peak"] == pytest.approx(row["GBps"] / 6546.2, rel=1e-3)
    assert row["GFLOPs"] == pytest.approx(1872 * Vh / 1e-3 / 1e9, rel=1e-3)
    # without the geometry the table has no GFLOP/s
    assert "GFLOPs" not in bench.kernel_table({"jinv_step_f32": (1, 1.0, 1.0)}, 1.0)["jinv_step_f32"]
