"""Batched ensemble: many independent scenarios in one simulation.

Scenarios keep local coordinates, own blocks of grid rows (frames) and own
materials (per-object table); the batch must reproduce each scenario run on
its own, up to float summation order (the batch rebuilds its neighbour
lists when any scenario needs it, which can re-sort a scenario's particles
at different steps)."""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def tag(comb, parts):
    """Write each particle's index within its scenario into idep.w of both
    the combined case and the parts."""
    for k, p in enumerate(parts):
        p.idep[:, 3] = np.arange(p.par.np, dtype=np.float32)
        (b0, b1), (m0, m1) = comb.meta["slices"][k]
        comb.idep[b0:b1, 3] = p.idep[: p.par.npb, 3]
        comb.idep[m0:m1, 3] = p.idep[p.par.npb:, 3]


def scenario(arrays, k):
    sel = np.asarray(arrays[2])[:, 0] == k + 1
    a = [np.asarray(x)[sel] for x in arrays]
    o = np.argsort(a[2][:, 3], kind="stable")
    return [x[o] for x in a]


def test_batched_ensemble_matches_scenarios_run_alone(lq, cuda):
    comb, parts = cases.ensemble(n=6, count_range=(2.0e3, 5.0e3), seed=11, shepard=7)
    tag(comb, parts)
    sim = lq.Simulation(comb.par, *comb.arrays())
    sim.set_materials(comb.meta["materials"])
    sim.set_frames(comb.meta["frames"])
    nsteps = 25
    sim.step(nsteps)
    batch = sim.download()
    assert not sim.health().any()
    for k, p in enumerate(parts):
        alone = lq.Simulation(p.par, *p.arrays())
        alone.step(nsteps)
        want = scenario(alone.download(), k)
        got = scenario(batch, k)
        assert got[0].shape == want[0].shape
        mat = want[2][:, 3] >= p.par.npb
        assert rel_l2(got[0][mat, :3], want[0][mat, :3]) < 1e-6, k
        assert rel_l2(got[1][mat, 3], want[1][mat, 3]) < 1e-6, k
        assert rel_l2(got[1][mat, :3], want[1][mat, :3]) < 1e-4, k
        assert rel_l2(got[3][mat], want[3][mat]) < 1e-4, k


def test_frames_keep_scenarios_apart(lq, cuda):
    """Two copies of one scenario in one batch, one of them with its stress
    scaled: if any pair crossed scenarios the unscaled copy would change."""
    comb, parts = cases.ensemble(n=2, count_range=(3.0e3, 3.0e3), aspect_range=(1.0, 1.0), seed=5)
    # make scenario 1 an exact copy of scenario 0 in local coordinates ...
    (b0, b1), (m0, m1) = comb.meta["slices"][0]
    (c0, c1), (n0, n1) = comb.meta["slices"][1]
    if (b1 - b0, m1 - m0) != (c1 - c0, n1 - n0):
        pytest.skip("scenario sizes differ for this seed")
    for a in comb.arrays():
        a[c0:c1] = a[b0:b1]
        a[n0:n1] = a[m0:m1]
    comb.idep[c0:c1, 0] = 2
    comb.idep[n0:n1, 0] = 2
    comb.meta["materials"][2] = comb.meta["materials"][1]
    base = [a.copy() for a in comb.arrays()]
    comb.str_[n0:n1] *= 3.0         # ... except for its stress
    sim = lq.Simulation(comb.par, *comb.arrays())
    sim.set_materials(comb.meta["materials"])
    sim.set_frames(comb.meta["frames"])
    ref = lq.Simulation(comb.par, *base)
    ref.set_materials(comb.meta["materials"])
    ref.set_frames(comb.meta["frames"])
    for s_ in (sim, ref):
        s_.set_skin(0.5)            # no list rebuild in 10 steps: identical sort order in both
    sim.step(10)
    ref.step(10)
    a, b = sim.download(), ref.download()
    sa, sb = scenario(a, 0), scenario(b, 0)
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)
