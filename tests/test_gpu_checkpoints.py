"""Long runs checked against the FP64 oracle on a seeded 1 % subsample of
the soil particles every 1000 steps: at each check the oracle restarts from
the GPU's state (same step number and time, so the Shepard cadence agrees),
both advance one step, and the subsample is compared particle by particle.
This is the inclined-plane workload's checking scheme, at a spacing the
oracle steps in about a second; the full-size workload runs through
`bench.py --config inclined`.  A second test runs the same block for 3000
steps against the oracle advanced continuously from the initial state (a
stored fixture), which measures the accumulated drift."""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases
from helpers import by_id, rel_l2

pytestmark = pytest.mark.gpu


def subsample_errors(got, want, ids):
    g = by_id(got)
    w = by_id(want)
    return dict(rho=rel_l2(g[1][ids, 3], w[1][ids, 3]), vel=rel_l2(g[1][ids, :3], w[1][ids, :3]),
                str=rel_l2(g[3][ids], w[3][ids]), e=rel_l2(g[2][ids, 2], w[2][ids, 2]),
                pos=rel_l2(g[0][ids, :3], w[0][ids, :3]))


def test_inclined_block_subsample_vs_oracle_every_1000_steps(lq, orc, cuda):
    c = cases.inclined_block(dr=0.0125, runout=0.5, seed=3).with_ids()
    nb, n = c.par.npb, c.par.np
    rows = c.meta["hypoplastic"]
    sim = lq.Simulation(c.par, *c.arrays(), mixed=True)
    sim.set_hypoplastic(rows)
    # particles are matched by the original index carried in idep.w; soil
    # particles hold indices [npb, np)
    ids = np.sort(np.random.default_rng(2024).choice(np.arange(nb, n), size=max(1, (n - nb) // 100),
                                                     replace=False))
    report = []
    for check in range(3):
        if check:
            sim.step(999)
        state = sim.download()
        step, time = sim.clock()
        osim = orc.OracleSim(c.par, *state, step0=step, time0=time)
        osim.set_vw(rows)
        sim.step(1)
        osim.step(1)
        e = subsample_errors(sim.download(), osim.get(), ids)
        report.append((step + 1, e))
        assert e["rho"] < 1e-6 and e["vel"] < 1e-4 and e["str"] < 1e-4 and e["e"] < 1e-6, report
        osim.close()
    print("inclined block", n - nb, "soil,", len(ids), "checked:",
          [(s, {k: f"{v:.1e}" for k, v in e.items()}) for s, e in report])
    assert not sim.health().any()
    # the block moved down the plane between the checks
    pos = by_id(sim.download())[0]
    assert np.abs(pos[ids, 0] - c.pospres[ids, 0]).max() > 1e-4


def test_inclined_block_drift_vs_continuous_oracle_run(lq, cuda):
    """The same block run from its initial state for 3000 steps (mixed
    form) against the oracle advanced continuously from the same state
    (tests/golden/inclined_drift.npz, made by tests/golden/make_inclined.py):
    at every 1000 steps the seeded 1 % sample's density, velocity, stress,
    void ratio and displacement must agree, so the errors here are the
    accumulated drift, not one step's."""
    import sys
    from pathlib import Path

    golden = Path(__file__).resolve().parent / "golden"
    sys.path.insert(0, str(golden))
    from make_inclined import drift_case, pick

    z = np.load(golden / "inclined_drift.npz")
    c = drift_case()
    assert c.par.np == int(z["np"])
    ids = z["ids"]
    x0 = c.pospres[ids, :3].astype(np.float64)
    sim = lq.Simulation(c.par, *c.arrays(), mixed=True)
    sim.set_hypoplastic(c.meta["hypoplastic"])
    done, report = 0, []
    for m in z["marks"]:
        sim.step(int(m) - done)
        done = int(m)
        pos, vel, idep, s, e = pick(sim.download(), ids)
        w = {k: z[f"{k}_{m}"].astype(np.float64) for k in ("pos", "vel", "str", "void")}
        err = dict(rho=rel_l2(vel[:, 3], w["vel"][:, 3]), vel=rel_l2(vel[:, :3], w["vel"][:, :3]),
                   str=rel_l2(s, w["str"]), e=rel_l2(idep[:, 2], w["void"]),
                   disp=rel_l2(pos[:, :3] - x0, w["pos"] - x0))
        report.append((int(m), err))
    print("inclined drift", [(m, {k: f"{v:.1e}" for k, v in e.items()}) for m, e in report])
    assert not sim.health().any()
    sim.close()
    for m, e in report:
        assert e["rho"] < 1e-5 and e["e"] < 1e-5, (m, e)
        assert e["vel"] < 1e-3 and e["str"] < 1e-3 and e["disp"] < 1e-3, (m, e)
    assert np.abs(w["pos"][:, 0] - x0[:, 0]).max() > 1e-3      # the block moved down the plane
