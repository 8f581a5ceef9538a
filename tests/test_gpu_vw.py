"""Constitutive model 3 (von Wolffersdorff hypoplasticity with FP64 adaptive
sub-stepping) on the GPU against the FP64 oracle.  The model is not in the
reference; the oracle is written from the published equations and pinned by
the model's own properties (tests/test_oracle_vw.py).

* Whole steps of a small hypoplastic column, plain and mixed forms, after
  1, 10 and 100 steps: density, velocity, stress and the void ratio carried
  in idep.z, per particle.
* The slope and inclined-plane workloads at coarse spacing against the
  oracle over a few steps.
* Error paths: a model-3 simulation without its table, malformed rows, the
  drop-in predictor (which has no table) given model 3."""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases
from helpers import by_id, rel_l2

pytestmark = pytest.mark.gpu

# FP32 state with FP64 sub-stepping vs the FP64 oracle, relative L2 over the
# soil.  The void ratio is stored in float (idep.z) in both forms.
TOL_VW = {1: dict(rho=2e-6, vel=5e-5, str=5e-5, e=1e-6),
          10: dict(rho=5e-6, vel=1e-4, str=1e-4, e=2e-6),
          100: dict(rho=2e-5, vel=5e-4, str=5e-4, e=1e-5)}


def vw_errors(got, want, nb):
    g = by_id(got)
    w = by_id(want)
    mat = np.asarray(w[2])[:, 0] == 1
    return dict(rho=rel_l2(g[1][mat, 3], w[1][mat, 3]), vel=rel_l2(g[1][mat, :3], w[1][mat, :3]),
                str=rel_l2(g[3][mat], w[3][mat]), e=rel_l2(g[2][mat, 2], w[2][mat, 2]),
                pos=rel_l2(g[0][mat, :3], w[0][mat, :3]))


def pair(lq, orc, c, mixed):
    sim = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
    sim.set_hypoplastic(c.meta["hypoplastic"])
    osim = orc.OracleSim(c.par, *c.arrays())
    osim.set_vw(c.meta["hypoplastic"])
    return sim, osim


@pytest.mark.parametrize("mixed", [False, True])
def test_von_wolffersdorff_column_vs_oracle_1_10_100_steps(lq, orc, cuda, mixed):
    c = cases.small_column(model=3, velocity_noise=0.02, shepard=30, seed=21).with_ids()
    sim, osim = pair(lq, orc, c, mixed)
    done = 0
    report = {}
    for n in (1, 10, 100):
        sim.step(n - done)
        osim.step(n - done)
        done = n
        e = vw_errors(sim.download(), osim.get(), c.par.npb)
        report[n] = e
        for k, tol in TOL_VW[n].items():
            assert e[k] < tol, (mixed, n, k, report)
    print("vW", "mixed" if mixed else "plain",
          {n: {k: f"{v:.2e}" for k, v in e.items()} for n, e in report.items()})
    assert not sim.health().any()
    # the void ratio moved (the model is active) and stayed physical
    ev = sim.download()[2][c.par.npb:, 2]
    assert np.abs(ev - 0.70).max() > 1e-4
    assert 0.5 < ev.min() and ev.max() < 1.1


@pytest.mark.parametrize("make", [lambda: cases.slope_failure(dr=0.025, seed=5),
                                  lambda: cases.inclined_block(dr=0.025, runout=0.3, seed=6)],
                         ids=["slope", "inclined"])
def test_workload_geometries_at_coarse_spacing_vs_oracle(lq, orc, cuda, make):
    c = make().with_ids()
    sim, osim = pair(lq, orc, c, True)
    sim.step(20)
    osim.step(20)
    e = vw_errors(sim.download(), osim.get(), c.par.npb)
    print(c.name, c.par.npm, {k: f"{v:.2e}" for k, v in e.items()})
    assert e["rho"] < 1e-5 and e["vel"] < 5e-4 and e["str"] < 5e-4 and e["e"] < 1e-5, e
    assert not sim.health().any()


def test_model_3_needs_its_table_and_checks_rows(lq, cuda):
    c = cases.small_column(model=3, seed=2)
    sim = lq.Simulation(c.par, *c.arrays())
    with pytest.raises(RuntimeError, match="hypoplastic"):
        sim.step(1)
    bad = cases.vw_row().copy()
    bad[3], bad[4] = 0.9, 0.8            # e_d0 > e_c0
    with pytest.raises(RuntimeError, match="row 0"):
        sim.set_hypoplastic(bad)
    sim.set_hypoplastic(c.meta["hypoplastic"])
    sim.step(2)
    assert not sim.health().any()


def test_drop_in_predictor_rejects_model_3(lq, cuda):
    """The reference's Predictor has no von Wolffersdorff table to read."""
    from helpers import dev, par_dev, zeros

    c = cases.small_column(model=3, seed=2)
    n = c.par.np
    pd = par_dev(c.par)
    state = [dev(c.pospres), dev(c.velrhop), dev(c.idep), dev(c.str_), dev(c.stn)]
    ini = [zeros((n, 4)), zeros((n, 4)), zeros((n, 4)), zeros((n, 6)), zeros((n, 6))]
    rates = [zeros((n, 4)), zeros((n, 4)), zeros((n, 6))]
    with pytest.raises(lq.LoquatError, match="model 3"):
        lq.predictor(c.par, pd, state, ini, rates)
    with pytest.raises(lq.LoquatError, match="model 3"):
        lq.corrector(c.par, pd, state, ini, rates)
