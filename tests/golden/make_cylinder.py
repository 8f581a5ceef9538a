"""Golden data of the cylinder collapse (Drucker-Prager phi = 30 deg,
E = 5 MPa, rho = 2000 kg/m^3, h = 1.3 dr, dr = 2.949 mm) from the FP64 oracle.

    python tests/golden/make_cylinder.py full   [--out DIR]
    python tests/golden/make_cylinder.py runout [--out DIR]

full:   the workload at its stated size (R = 0.2 m, H = 0.4 m: 1,967,104 soil
        + 344,763 boundary particles).  After 1, 10 and 100 steps the
        velocity, density and stress of a seeded 1 % sample of the soil
        particles (by original index) go to cylinder_full.npz for
        tests/test_gpu_scale.py.
runout: the same material and spacing on a cylinder scaled by 1/4
        (R = 0.05 m, H = 0.1 m), run for the workload's 5000 steps and on to
        20000; the runout radius (largest radial distance of a soil particle
        from the axis) and the free-surface profile (highest soil particle
        per radial bin) every 1000 steps go to cylinder_runout.npz.

Both run the oracle on every host thread; the case is generated exactly as
the GPU tests generate it (cases.cylinder_collapse, seed 1, particle indices
in idep.w), with Parameters derived by the oracle.
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

FULL_MARKS = (1, 10, 100)
SAMPLE_FRACTION = 0.01
SAMPLE_SEED = 20
RUNOUT_SCALE = 0.25
RUNOUT_EVERY = 1000
RUNOUT_STEPS = 20000
BIN_CELLS = 4          # radial bin width of the surface profile, in particle spacings


def full_case():
    from loquat_b200 import cases

    return cases.cylinder_collapse(seed=1).with_ids()


def runout_case():
    from loquat_b200 import cases

    return cases.cylinder_collapse(radius=0.2 * RUNOUT_SCALE, height=0.4 * RUNOUT_SCALE, seed=1)


def sample_ids(case):
    """Original indices of the seeded soil sample."""
    rng = np.random.default_rng(SAMPLE_SEED)
    n = int(round(SAMPLE_FRACTION * case.par.npm))
    return np.sort(rng.choice(np.arange(case.par.npb, case.par.np), n, replace=False))


def pick(arrays, ids):
    """Rows of (pos, vel, idep, str, stn) whose idep.w index is in ids, in ids order."""
    idx = np.asarray(arrays[2])[:, 3].astype(np.int64)
    where = np.empty(int(idx.max()) + 1, np.int64)
    where[idx] = np.arange(idx.size)
    rows = where[ids]
    return [np.asarray(a)[rows] for a in arrays]


def axis_of(case):
    side = case.par.domain_size_x
    return side / 2.0, side / 2.0


def radius_and_profile(pos, idep, dr, axis, nbins):
    """Runout radius (largest soil distance from the axis) and surface
    profile (highest soil z per radial bin of BIN_CELLS * dr)."""
    soil = np.asarray(idep)[:, 0] == 1
    p = np.asarray(pos)[soil]
    r = np.hypot(p[:, 0] - axis[0], p[:, 1] - axis[1])
    b = np.clip((r / (BIN_CELLS * dr)).astype(int), 0, nbins - 1)
    prof = np.zeros(nbins)
    np.maximum.at(prof, b, p[:, 2])
    return float(r.max()), prof


def make_full(out: Path):
    import oracle
    from loquat_b200 import cases

    cases.use_parameter_initializer(oracle.initialize_parameters)
    c = full_case()
    ids = sample_ids(c)
    oracle.set_threads(0)
    sim = oracle.OracleSim(c.par, *c.arrays())
    t0 = time.time()
    done = 0
    data = {}
    for m in FULL_MARKS:
        sim.step(m - done)
        done = m
        pos, vel, idep, s, e = pick(sim.get(), ids)
        data[f"vel_{m}"] = vel.astype(np.float32)
        data[f"str_{m}"] = s.astype(np.float32)
        print(m, time.time() - t0, flush=True)
    sim.close()
    np.savez_compressed(out / "cylinder_full.npz", ids=ids, marks=np.array(FULL_MARKS), np=c.par.np,
                        npm=c.par.npm, **data)


def make_runout(out: Path):
    import oracle
    from loquat_b200 import cases

    cases.use_parameter_initializer(oracle.initialize_parameters)
    c = runout_case()
    dr = c.meta["dr"]
    axis = axis_of(c)
    nbins = int(np.ceil(0.5 * c.par.domain_size_x / (BIN_CELLS * dr)))
    r0, p0 = radius_and_profile(c.pospres, c.idep, dr, axis, nbins)
    oracle.set_threads(0)
    sim = oracle.OracleSim(c.par, *c.arrays())
    marks, radii, profiles = [], [], []
    t0 = time.time()
    done = 0
    while done < RUNOUT_STEPS:
        sim.step(RUNOUT_EVERY)
        done += RUNOUT_EVERY
        pos, vel, idep, s, e = sim.get()
        r, p = radius_and_profile(pos, idep, dr, axis, nbins)
        marks.append(done)
        radii.append(r)
        profiles.append(p)
        print(done, r, time.time() - t0, flush=True)
    sim.close()
    np.savez_compressed(out / "cylinder_runout.npz", steps=np.array(marks), radii=np.array(radii),
                        profiles=np.array(profiles), radius0=r0, profile0=p0, dr=dr, axis=np.array(axis),
                        bin_cells=BIN_CELLS, np=c.par.np, npm=c.par.npm)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["full", "runout"])
    ap.add_argument("--out", type=Path, default=HERE)
    a = ap.parse_args(argv)
    a.out.mkdir(parents=True, exist_ok=True)
    (make_full if a.what == "full" else make_runout)(a.out)


if __name__ == "__main__":
    main()
