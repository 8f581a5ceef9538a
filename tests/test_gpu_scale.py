"""Whole-step parity where the bench measures, and of batched scenarios.

* The cylinder collapse at its stated size (1,967,104 soil + 344,763
  boundary particles, dr = 2.949 mm, the bench's default workload) after
  1, 10 and 100 steps, in both precision forms, against the FP64 oracle's
  run of the same case on a seeded 1 % sample of the soil particles
  (tests/golden/cylinder_full.npz, made by tests/golden/make_cylinder.py).
  Velocity, stress and the density change must agree within 1e-3 relative
  L2 in the mixed-precision form (the density itself is compared too).
  Plain FP32 is held to 3e-3: at 0.5 m from the origin a float position
  cannot take a step's displacement of ~1e-7 m whole, and a float density
  of ~2000 kg/m^3 resolves its change only to ~1e-4 kg/m^3.
* The same material and spacing on a cylinder scaled by 1/4 for the
  workload's 5000 steps and on to 20000: the runout radius and the
  free-surface profile against the oracle's within 1 %
  (tests/golden/cylinder_runout.npz).
* A batched ensemble of Drucker-Prager columns with their own friction
  angle and cohesion (per-object material rows and frames): each scenario
  of the batch against the oracle run on that scenario alone with its own
  Parameters, after 1, 10 and 100 steps.
Reference step sequence: src/loquat.cu:322-409.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

from loquat_b200 import cases
from helpers import rel_l2

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))

TOL = 1e-3          # the mixed-precision form (the contract)
TOL_PLAIN = 3e-3    # plain FP32

@pytest.mark.parametrize("mixed", [False, True])
def test_cylinder_at_stated_size_vs_oracle_1_10_100_steps(lq, cuda, mixed):
    from make_cylinder import full_case, pick

    z = np.load(GOLDEN / "cylinder_full.npz")
    c = full_case()
    assert c.par.np == int(z["np"]) and c.par.npm == int(z["npm"]) == 1967104
    ids = z["ids"]
    rho0 = c.velrhop[ids, 3].astype(np.float64)
    sim = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
    done = 0
    report = []
    for m in z["marks"]:
        sim.step(int(m) - done)
        done = int(m)
        pos, vel, idep, s, e = pick(sim.download(), ids)
        wv, ws = z[f"vel_{m}"].astype(np.float64), z[f"str_{m}"].astype(np.float64)
        err = {"velocity": rel_l2(vel[:, :3], wv[:, :3]), "stress": rel_l2(s, ws),
               "density change": rel_l2(vel[:, 3] - rho0, wv[:, 3] - rho0), "density": rel_l2(vel[:, 3], wv[:, 3])}
        report.append((int(m), err))
    print("mixed" if mixed else "plain", [(m, {k: f"{v:.2e}" for k, v in e.items()}) for m, e in report])
    assert not sim.health().any()
    sim.close()
    tol = TOL if mixed else TOL_PLAIN
    for m, err in report:
        for k, v in err.items():
            assert v <= tol, (m, k, v)


def _tag(comb, parts):
    for k, p in enumerate(parts):
        p.idep[:, 3] = np.arange(p.par.np, dtype=np.float32)
        (b0, b1), (m0, m1) = comb.meta["slices"][k]
        comb.idep[b0:b1, 3] = p.idep[: p.par.npb, 3]
        comb.idep[m0:m1, 3] = p.idep[p.par.npb:, 3]


def _scenario(arrays, k):
    sel = np.asarray(arrays[2])[:, 0] == k + 1
    a = [np.asarray(x)[sel] for x in arrays]
    o = np.argsort(a[2][:, 3], kind="stable")
    return [x[o] for x in a]


@pytest.mark.parametrize("mixed", [False, True])
def test_batched_scenarios_with_own_materials_vs_oracle(lq, orc, cuda, mixed):
    comb, parts = cases.ensemble(n=4, count_range=(2.0e3, 6.0e3), seed=11, shepard=7)
    _tag(comb, parts)
    mats = comb.meta["materials"]
    assert len({round(float(r[2]), 4) for r in mats[1:]}) == len(parts)     # distinct friction angles
    assert max(float(r[4]) for r in mats[1:]) > 1.0e3                         # cohesion in play
    sim = lq.Simulation(comb.par, *comb.arrays(), mixed=mixed)
    sim.set_materials(mats)
    sim.set_frames(comb.meta["frames"])
    osims = [orc.OracleSim(p.par, *p.arrays()) for p in parts]
    done = 0
    worst = {}
    for m in (1, 10, 100):
        sim.step(m - done)
        batch = sim.download()
        for k, (p, o) in enumerate(zip(parts, osims)):
            o.step(m - done)
            want = o.get()
            ow = np.argsort(want[2][:, 3], kind="stable")
            want = [x[ow] for x in want]
            got = _scenario(batch, k)
            assert got[0].shape[0] == want[0].shape[0]
            mat = want[2][:, 3] >= p.par.npb
            for name, a, b in (("velocity", got[1][mat, :3], want[1][mat, :3]), ("stress", got[3][mat], want[3][mat]),
                               ("density", got[1][mat, 3], want[1][mat, 3])):
                e = rel_l2(a, b)
                worst[(m, name)] = max(worst.get((m, name), 0.0), e)
        done = m
    print("mixed" if mixed else "plain", {f"{m}:{n}": f"{v:.2e}" for (m, n), v in worst.items()})
    assert not sim.health().any()
    sim.close()
    for o in osims:
        o.close()
    for key, v in worst.items():
        assert v <= TOL, (key, v)


@pytest.mark.parametrize("mixed", [False, True])
def test_scaled_cylinder_runout_and_surface_vs_oracle(lq, cuda, mixed):
    """The cylinder's material and spacing on a cylinder scaled by 1/4
    (R = 0.05 m, H = 0.1 m) for the workload's 5000 steps and on to 20000,
    against the oracle's run (tests/golden/cylinder_runout.npz): the runout
    radius (advance of the largest radial distance of a soil particle from
    the axis) and the free-surface profile (highest soil particle per
    radial bin) within 1 %."""
    from make_cylinder import radius_and_profile, runout_case

    z = np.load(GOLDEN / "cylinder_runout.npz")
    c = runout_case()
    assert c.par.np == int(z["np"])
    dr, axis, nbins = float(z["dr"]), tuple(z["axis"]), z["profiles"].shape[1]
    sim = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
    done = 0
    report = []
    for k, n in enumerate(z["steps"]):
        sim.step(int(n) - done)
        done = int(n)
        pos, vel, idep, s, e = sim.download()
        r, prof = radius_and_profile(pos, idep, dr, axis, nbins)
        run_gpu = r - float(z["radius0"])
        run_ref = float(z["radii"][k]) - float(z["radius0"])
        occ = z["profiles"][k] > 0
        surf = np.linalg.norm(prof[occ] - z["profiles"][k][occ]) / np.linalg.norm(z["profiles"][k][occ])
        report.append((int(n), run_gpu, run_ref, surf))
    print("mixed" if mixed else "plain", [(n, f"{a * 1e3:.3f} mm", f"{b * 1e3:.3f} mm", f"{s_:.2e}")
                                          for n, a, b, s_ in report])
    assert not sim.health().any()
    sim.close()
    for n, run_gpu, run_ref, surf in report:
        if n in (5000, int(z["steps"][-1])):
            assert run_ref > dr, (n, run_ref)           # the front has moved
            assert abs(run_gpu - run_ref) <= 0.01 * run_ref, (n, run_gpu, run_ref)
            assert surf < 0.01, (n, surf)
