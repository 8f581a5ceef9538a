"""Long run: the 50k-particle column collapse (0.2 x 0.1 x 0.02 m soil at
dr = 2 mm, Drucker-Prager phi = 19.8 deg, Shepard every 30 steps) for 2000
steps on the GPU, against the FP64 oracle's run stored in
tests/golden/column_runout.npz (made by tests/golden/make_column_runout.py).
The runout distance (advance of the soil front) and the free-surface
profile must agree within 1 %."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from loquat_b200 import cases

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))


@pytest.mark.parametrize("mixed", [False, True])
def test_column_collapse_runout_and_surface_vs_oracle(lq, cuda, mixed):
    from make_column_runout import front_and_profile

    z = np.load(GOLDEN / "column_runout.npz")
    c = cases.column_collapse()
    dr, x0, nbins = float(z["dr"]), float(z["x0"]), z["profiles"].shape[1]
    sim = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
    done = 0
    report = []
    for k, n in enumerate(z["steps"]):
        sim.step(int(n) - done)
        done = int(n)
        pos, vel, idep, s, e = sim.download()
        front, prof = front_and_profile(pos, idep, dr, x0, nbins)
        run_gpu = front - float(z["front0"])
        run_ref = float(z["fronts"][k]) - float(z["front0"])
        occupied = z["profiles"][k] > 0
        surf = np.linalg.norm(prof[occupied] - z["profiles"][k][occupied]) / np.linalg.norm(z["profiles"][k][occupied])
        report.append((int(n), run_gpu, run_ref, surf))
    print("mixed" if mixed else "plain", [(n, f"{a * 1e3:.4f} mm", f"{b * 1e3:.4f} mm", f"{c:.2e}")
                                          for n, a, b, c in report])
    assert not sim.health().any()
    n, run_gpu, run_ref, surf = report[-1]
    assert run_ref > 1.5 * dr                     # the front has moved (3.9 mm after 2000 steps)
    assert abs(run_gpu - run_ref) <= 0.01 * run_ref, report
    assert surf < 0.01, report
