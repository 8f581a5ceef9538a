"""The pair kernel's tile order checked on the host: the index arithmetic
that k_tile_segments runs on the GPU (loquat_b200/csrc/lq_tile.h) is
compiled with g++ into tests/tile_order_check.cpp, which asserts over
random cell-start tables that the segments partition the material slots
into a permutation of the targets, one column's tz cells per segment."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_tile_order_is_a_permutation_of_compact_column_runs(tmp_path):
    gxx = shutil.which("g++") or "g++"
    exe = tmp_path / "tile_order_check"
    cmd = [gxx, "-std=c++17", "-O1", "-Wall", "-Werror", f"-I{ROOT / 'loquat_b200' / 'csrc'}",
           str(ROOT / "tests" / "tile_order_check.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
