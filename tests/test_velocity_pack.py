"""The mixed form's packed neighbour velocity checked on the host: the
shared-exponent encoding that k_pack_neighbors writes and the pair kernel
decodes on the GPU (loquat_b200/csrc/lq_pack.h) is compiled with g++ into
tests/velocity_pack_check.cpp, which asserts over random and edge-case
velocities that the decode equals the rounding rule stated independently
in doubles, with every error at most half the shared quantum."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_packed_velocity_rounds_to_the_shared_quantum(tmp_path):
    gxx = shutil.which("g++") or "g++"
    exe = tmp_path / "velocity_pack_check"
    cmd = [gxx, "-std=c++17", "-O1", "-ffp-contract=off", "-Wall", "-Werror",
           f"-I{ROOT / 'loquat_b200' / 'csrc'}", str(ROOT / "tests" / "velocity_pack_check.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
