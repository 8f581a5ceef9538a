"""The reference arm of bench.py on the CPU: `--impl reference` times the
FP64 oracle on the workload itself (all host threads, then one thread) and
prints one JSON line with the keys the bench contract asks for, with the
same `config` as the GPU arm; it loads no library of the product.  Under
torchrun only rank 0 runs and prints it, the other ranks exit 0 without
work."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run_bench(args, **env):
    e = dict(os.environ, PYTHONPATH=str(ROOT), **env)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True, env=e,
                       cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_prints_one_contract_line():
    lines = run_bench(["--impl", "reference", "--config", "column", "--steps", "1", "--warmup", "0"])
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"].startswith("column collapse")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["single_thread"]["cores"] == 1 and d["single_thread"]["value"] > 0
    # the workload itself, not a sample: the column's 50,000 soil particles
    assert d["config"]["npm"] == 50000 and set(d["config"]) == {"workload", "np", "npm", "npb", "ncell"}


def test_reference_arm_loads_no_product_library():
    """The CPU arm derives the case's Parameters with the oracle, so the
    CUDA library of the product is never mapped into its process."""
    code = ("import sys, bench; rc = bench.main(['--impl', 'reference', '--config', 'column', '--steps', '1', "
            "'--warmup', '0']); maps = open('/proc/self/maps').read(); "
            "assert 'liblqb200' not in maps, 'product library loaded'; "
            "assert 'liblq_oracle' in maps; sys.exit(rc)")
    e = dict(os.environ, PYTHONPATH=str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=e, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def test_reference_arm_other_ranks_exit_quietly():
    lines = run_bench(["--impl", "reference", "--config", "column", "--steps", "1", "--warmup", "0"],
                      RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    assert lines == []


def test_clock_sampler_reads_clocks_and_throttle_reasons(tmp_path, monkeypatch):
    """The clock record beside each bench line: median SM clock under load,
    the maximum, and every throttle reason seen active (a fake nvidia-smi
    prints the sampled rows)."""
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/bin/sh\n"
                    "echo '0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active'\n"
                    "echo '0, 1800, 1965, 990.5, 0x4, Not Active, Not Active, Not Active, Active'\n"
                    "echo '0, 1950, 1965, 950.0, 0x0, Not Active, Not Active, Not Active, Not Active'\n"
                    "exec sleep 30\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    sys.path.insert(0, str(ROOT))
    try:
        import bench
    finally:
        sys.path.pop(0)
    import time

    s = bench.ClockSampler(None)
    time.sleep(0.5)
    c = s.stop()
    assert c == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
