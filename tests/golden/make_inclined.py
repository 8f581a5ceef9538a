"""Golden data of the inclined-plane workload's long run, for drift checks:
the FP64 oracle advanced continuously from the initial state.

    python tests/golden/make_inclined.py [--out DIR]

The von Wolffersdorff block on a 30 deg plane (the inclined-plane workload's
geometry and sand, e0 = 0.65) at dr = 12.5 mm with 0.5 m of plane below it
(128 k soil particles), seed 3, particle indices in idep.w.  Every 1000
steps up to 3000 the density, velocity, stress, void ratio and position of
a seeded 1 % sample of the soil particles go to inclined_drift.npz for
tests/test_gpu_checkpoints.py.  Runs on every host thread; the case's
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

MARKS = (1000, 2000, 3000)
SAMPLE_SEED = 2024


def drift_case():
    from loquat_b200 import cases

    return cases.inclined_block(dr=0.0125, runout=0.5, seed=3).with_ids()


def sample_ids(case):
    nb, n = case.par.npb, case.par.np
    return np.sort(np.random.default_rng(SAMPLE_SEED).choice(np.arange(nb, n), size=max(1, (n - nb) // 100),
                                                           replace=False))


def pick(arrays, ids):
    """Rows whose idep.w index is in ids, in ids order."""
    idx = np.asarray(arrays[2])[:, 3].astype(np.int64)
    where = np.empty(int(idx.max()) + 1, np.int64)
    where[idx] = np.arange(idx.size)
    return [np.asarray(a)[where[ids]] for a in arrays]


def main(argv=None):
    import oracle
    from loquat_b200 import cases

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=HERE)
    a = ap.parse_args(argv)
    cases.use_parameter_initializer(oracle.initialize_parameters)
    c = drift_case()
    ids = sample_ids(c)
    oracle.set_threads(0)
    sim = oracle.OracleSim(c.par, *c.arrays())
    sim.set_vw(c.meta["hypoplastic"])
    data, done, t0 = {}, 0, time.time()
    for m in MARKS:
        sim.step(m - done)
        done = m
        pos, vel, idep, s, e = pick(sim.get(), ids)
        data[f"pos_{m}"] = pos[:, :3].astype(np.float32)
        data[f"vel_{m}"] = vel.astype(np.float32)
        data[f"str_{m}"] = s.astype(np.float32)
        data[f"void_{m}"] = idep[:, 2].astype(np.float32)
        print(m, time.time() - t0, flush=True)
    sim.close()
    a.out.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(a.out / "inclined_drift.npz", ids=ids, marks=np.array(MARKS), np=c.par.np, npm=c.par.npm,
                        **data)


if __name__ == "__main__":
    main()
