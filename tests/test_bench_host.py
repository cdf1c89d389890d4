"""bench.py's host-side arithmetic, no GPU: the setup roofline's compulsory bytes and the
batch statistics on one rank."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "parallax-world_b200")]

import bench  # noqa: E402


def test_setup_roofline_counts_compulsory_bytes():
    # levels 1..3 hold 100, 10 and 1 blocks; level 0 is matrix-free (its count unused)
    info = {"levels": 4, "blocks": [999, 100, 10, 1] + [0] * 12}
    cells, setup_ms, peak = 1000, 2.0, 6000.0
    r = bench.setup_roofline(info, cells, setup_ms, peak)
    # the piece once (5 B a cell); every coarse level written in FP64 and FP32; each
    # coarse level but the top read once more in FP64
    want = 5 * cells + (100 + 10 + 1) * (288 + 144) + (100 + 10) * 288
    assert r["bytes_per_setup"] == want
    assert r["achieved"] == pytest.approx(want / (setup_ms / 1000.0) / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / peak)
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["traffic"] is None


def test_batch_stats_one_rank():
    infos = [{"status": 0, "residual": 5e-9, "refinements": 0, "iterations": 40},
             {"status": 0, "residual": 2e-8, "residual_floor": 3e-8, "refinements": 2, "iterations": 60},
             {"status": 0, "residual": 2e-8, "residual_floor": 1e-9, "refinements": 1, "iterations": 50},
             {"status": 3, "residual": 1.0, "refinements": 0, "iterations": 20000}]
    st = bench.batch_stats(infos, 1e-8, 1)
    assert st["pieces"] == 4
    assert st["failed"] == 1
    assert st["above_tol"] == 1      # the third: above tol and above its floor
    assert st["at_fp64_floor"] == 1  # the second: above tol, within its floor
    assert st["replaced"] == 2
