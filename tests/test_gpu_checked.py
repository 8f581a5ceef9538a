"""The bounds-checked build (-D LQ_CHECKED, loquat_b200/liblqb200_checked.so)
stands in for a device memory checker: its list and grid kernels check every
index they gather or scatter through.  Runs of the native driver (both
precision forms, Shepard passes and list rebuilds, two-level lists with
their renewals, a batched ensemble with frames, the von Wolffersdorff
model) must
count no violation.  Each run is a child process that loads the checked
library in place of the product one.  The checked build's Adami walks its
lists in pairs (the product build's path from 4 M boundary particles on),
the product build's in groups of four at these sizes: the same run through
both must give the same state."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
CHECKED = ROOT / "loquat_b200" / "liblqb200_checked.so"

SCRIPT = r"""
import numpy as np
import loquat_b200 as lq
from loquat_b200 import cases
c = cases.small_column(velocity_noise=0.3, shepard=7, seed=61)
for mixed, shape in ((False, 0), (True, 0), (True, 9), (False, 10)):
    s = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
    s.set_pair_shape(shape)          # 9, 10: targets in tile order
    s.step(60)
    assert s.rebuilds() >= 2
    assert not s.health().any()
comb, _ = cases.ensemble(n=4, count_range=(1.5e3, 4.0e3), seed=13, shepard=7)
for shape in (0, 8):
    s = lq.Simulation(comb.par, *comb.arrays())
    s.set_materials(comb.meta["materials"])
    s.set_frames(comb.meta["frames"])
    s.set_pair_shape(shape)
    s.step(30)
for mixed, shape in ((False, 0), (True, 9)):
    s = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
    s.set_pair_shape(shape)
    s.set_skin(0.02)
    s.set_wide_skin(0.15)            # two-level lists: renewals from the wide lists
    s.step(60)
    assert s.renewals() >= 3 and s.rebuilds() >= 2
    assert not s.health().any()
v = cases.small_column(model=3, velocity_noise=0.05, shepard=7, seed=62)
s = lq.Simulation(v.par, *v.arrays(), mixed=True)
s.set_hypoplastic(v.meta["hypoplastic"])
s.set_pair_shape(7)
s.step(20)
print("VIOLATIONS", lq.bounds_violations())
"""


def run_child(lib):
    env = dict(os.environ, LOQUAT_B200_LIB=str(lib), PYTHONPATH=str(ROOT))
    r = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True, env=env, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    line = [l for l in r.stdout.splitlines() if l.startswith("VIOLATIONS")][-1]
    n = int(line.split()[1])
    if n > 0:
        print("\n".join(l for l in r.stdout.splitlines() if "LQ_CHECKED" in l))
    return n


def test_checked_build_counts_no_bounds_violation(cuda):
    from loquat_b200 import build

    srcs = list((ROOT / "loquat_b200" / "csrc").iterdir()) + list((ROOT / "include").iterdir())
    if not CHECKED.exists() or CHECKED.stat().st_mtime < max(p.stat().st_mtime for p in srcs):
        build.build_checked()      # a checked library older than the sources tests other code
    assert run_child(CHECKED) == 0


def test_product_build_reports_no_checks(cuda):
    assert run_child(ROOT / "loquat_b200" / "liblqb200.so") == -1


STATE_SCRIPT = r"""
import sys
import numpy as np
import loquat_b200 as lq
from loquat_b200 import cases
c = cases.small_column(velocity_noise=0.3, shepard=7, seed=63).with_ids()
out = {}
for mixed in (False, True):
    s = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
    s.set_skin(0.02)
    s.set_wide_skin(0.15)
    s.step(40)
    for k, a in enumerate(s.download()):
        out[f"{int(mixed)}_{k}"] = a
np.savez(sys.argv[1], **out)
"""


def test_checked_and_product_builds_compute_the_same_state(cuda, tmp_path):
    """Adami in pairs (checked build) against groups of four (product
    build), with everything else equal: two-level lists, renewals, sorts,
    Shepard passes, both precision forms."""
    import numpy as np

    from loquat_b200 import build
    from helpers import by_id, rel_l2

    srcs = list((ROOT / "loquat_b200" / "csrc").iterdir()) + list((ROOT / "include").iterdir())
    if not CHECKED.exists() or CHECKED.stat().st_mtime < max(p.stat().st_mtime for p in srcs):
        build.build_checked()
    states = {}
    for name, lib in (("checked", CHECKED), ("product", ROOT / "loquat_b200" / "liblqb200.so")):
        path = tmp_path / f"{name}.npz"
        env = dict(os.environ, LOQUAT_B200_LIB=str(lib), PYTHONPATH=str(ROOT))
        r = subprocess.run([sys.executable, "-c", STATE_SCRIPT, str(path)], capture_output=True, text=True, env=env,
                           timeout=600, cwd=ROOT)
        assert r.returncode == 0, r.stdout + r.stderr
        states[name] = np.load(path)
    for mixed in (0, 1):
        a = by_id([states["checked"][f"{mixed}_{k}"] for k in range(5)])
        b = by_id([states["product"][f"{mixed}_{k}"] for k in range(5)])
        errs = [rel_l2(x, y) for x, y in zip(a, b)]
        print("mixed" if mixed else "plain", [f"{e:.1e}" for e in errs])
        assert max(errs) < 1e-5, (mixed, errs)
