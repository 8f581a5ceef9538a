"""Long-run golden data: the FP64 oracle on the 50k-particle column collapse.

    python tests/golden/make_column_runout.py [--steps 2000] [--out DIR]

Runs the oracle (CPU, all threads) on the column-collapse case (0.2 x 0.1 x
0.02 m soil at dr = 2 mm, Drucker-Prager phi = 19.8 deg, 3-layer Adami floor
and walls, Shepard every 30 steps) and stores the runout front and the
free-surface profile after every 500 steps in column_runout.npz, for
tests/test_gpu_runout.py.
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

BIN_CELLS = 4   # surface-profile bin width in particle spacings


def front_and_profile(pos, idep, dr, x0, nbins):
    """Runout front (largest soil x) and surface profile (highest soil z in
    x bins of BIN_CELLS * dr starting at the back wall x0)."""
    soil = np.asarray(idep)[:, 0] == 1
    x = np.asarray(pos)[soil, 0]
    z = np.asarray(pos)[soil, 2]
    width = BIN_CELLS * dr
    b = np.clip(((x - x0) / width).astype(int), 0, nbins - 1)
    prof = np.zeros(nbins)
    np.maximum.at(prof, b, z)
    return float(np.max(x)), prof


def main(argv=None):
    import oracle
    from loquat_b200 import cases

    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=500)
    ap.add_argument("--out", type=Path, default=HERE)
    a = ap.parse_args(argv)
    c = cases.column_collapse()
    dr = c.meta["dr"]
    x0 = 3 * dr
    nbins = int(round(0.6 / (BIN_CELLS * dr)))
    oracle.set_threads(0)
    sim = oracle.OracleSim(c.par, *c.arrays())
    marks, fronts, profiles = [], [], []
    t0 = time.time()
    done = 0
    while done < a.steps:
        sim.step(a.every)
        done += a.every
        pos, vel, idep, s, e = sim.get()
        f, p = front_and_profile(pos, idep, dr, x0, nbins)
        marks.append(done)
        fronts.append(f)
        profiles.append(p)
        print(done, f, time.time() - t0, flush=True)
    f0, p0 = front_and_profile(c.pospres, c.idep, dr, x0, nbins)
    a.out.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(a.out / "column_runout.npz", steps=np.array(marks), fronts=np.array(fronts),
                        profiles=np.array(profiles), front0=f0, profile0=p0, dr=dr, x0=x0, bin_cells=BIN_CELLS)


if __name__ == "__main__":
    main()
