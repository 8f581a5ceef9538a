"""Golden data of the von Wolffersdorff workloads at their stated sizes, from
the FP64 oracle.

    python tests/golden/make_stated.py slope    [--out DIR]
    python tests/golden/make_stated.py inclined [--out DIR]

slope:    the sand slope failure, 2.0 x 0.6 x 0.35 m at 45 deg, dr = 5 mm
          (2,852,360 soil + 642,780 boundary particles), seed 1 as the bench
          generates it; a seeded 0.5 % sample of the soil particles.
inclined: the block on the 30 deg plane, 1.0 x 1.0 x 0.25 m at dr = 2.5 mm
          (16.0 M soil + 1.63 M boundary particles), seed 1; a seeded 0.1 %
          sample of the soil particles.

The sampled particles carry their rank in the sample in idep.w (exact as a
float, whatever the particle count) and every other particle -1, so they
can be found after any re-sorting; no kernel reads idep.w.

After 1, 10 and 100 steps the velocity and density, stress and void ratio
of the sample (by original index) go to <what>_stated.npz for
tests/test_gpu_stated.py.  The oracle runs on every host thread; the case's
Parameters are derived by the oracle.
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

MARKS = (1, 10, 100)
SAMPLE = {"slope": (0.005, 31), "inclined": (0.001, 32)}     # fraction, seed


def sample_ids(case, what: str):
    """Original indices of the seeded soil sample."""
    frac, seed = SAMPLE[what]
    n = int(round(frac * (case.par.np - case.par.npb)))
    return np.sort(np.random.default_rng(seed).choice(np.arange(case.par.npb, case.par.np), n, replace=False))


def stated_case(what: str):
    """The workload with the sample tagged in idep.w; returns (case, ids)."""
    from loquat_b200 import cases

    c = cases.slope_failure(seed=1) if what == "slope" else cases.inclined_block(seed=1)
    ids = sample_ids(c, what)
    c.idep[:, 3] = -1.0
    c.idep[ids, 3] = np.arange(ids.size, dtype=np.float32)
    return c, ids


def pick(arrays, n: int):
    """Rows of (pos, vel, idep, str, stn) of the n tagged particles, in
    sample order."""
    tag = np.asarray(arrays[2])[:, 3]
    rows = np.nonzero(tag >= 0)[0]
    assert rows.size == n
    rows = rows[np.argsort(tag[rows], kind="stable")]
    assert (np.asarray(arrays[2])[rows, 3] == np.arange(n)).all()
    return [np.asarray(a)[rows] for a in arrays]


def main(argv=None):
    import oracle
    from loquat_b200 import cases

    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["slope", "inclined"])
    ap.add_argument("--out", type=Path, default=HERE)
    a = ap.parse_args(argv)
    cases.use_parameter_initializer(oracle.initialize_parameters)
    c, ids = stated_case(a.what)
    oracle.set_threads(0)
    sim = oracle.OracleSim(c.par, *c.arrays())
    sim.set_vw(c.meta["hypoplastic"])
    t0 = time.time()
    done = 0
    data = {}
    for m in MARKS:
        sim.step(m - done)
        done = m
        pos, vel, idep, s, e = pick(sim.get(), ids.size)
        data[f"vel_{m}"] = vel.astype(np.float32)
        data[f"str_{m}"] = s.astype(np.float32)
        data[f"void_{m}"] = idep[:, 2].astype(np.float32)
        print(m, time.time() - t0, flush=True)
    sim.close()
    a.out.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(a.out / f"{a.what}_stated.npz", ids=ids, marks=np.array(MARKS), np=c.par.np,
                        npm=c.par.npm, **data)


if __name__ == "__main__":
    main()
