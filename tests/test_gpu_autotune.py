"""The autotuner (lq_sim_autotune) and the pair kernel's launch shapes:
every shape gives bit-identical results (each target's sums run in one
thread in the same order), tuning leaves the simulation's state, step and
time as they were, and a tuned simulation steps exactly like a fresh one
configured with the chosen shape and skin."""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases

pytestmark = pytest.mark.gpu


def test_all_pair_kernel_shapes_agree_bit_for_bit(lq, cuda):
    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=81)
    out = []
    for shape in range(5):
        s = lq.Simulation(c.par, *c.arrays(), mixed=True)
        s.set_pair_shape(shape)
        s.step(25)
        out.append(s.download())
    for other in out[1:]:
        for x, y in zip(out[0], other):
            assert np.array_equal(x, y)
    with pytest.raises(lq.LoquatError):
        s.set_pair_shape(7)


@pytest.mark.parametrize("mixed", [False, True])
def test_warp_cooperative_shapes_agree_to_rounding(lq, orc, cuda, mixed):
    """Shapes 5 and 6 (8 and 32 lanes per target, shuffle reductions) sum
    in another order: they match the thread-per-target kernel to float
    rounding and the oracle within the usual tolerances."""
    from helpers import by_id, rel_l2

    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=83).with_ids()
    runs = {}
    for shape in (0, 5, 6):
        s = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
        s.set_pair_shape(shape)
        s.step(30)
        runs[shape] = by_id(s.download())
        assert not s.health().any()
    nb = c.par.npb
    for shape in (5, 6):
        for k, tol in ((1, 1e-5), (3, 1e-4)):
            assert rel_l2(runs[shape][k][nb:], runs[0][k][nb:]) < tol, (shape, k)
    osim = orc.OracleSim(c.par, *c.arrays())
    osim.step(30)
    want = by_id(osim.get())
    assert rel_l2(runs[5][1][nb:, :3], want[1][nb:, :3]) < 1e-4


def test_autotune_leaves_the_state_and_matches_a_fresh_run(lq, cuda):
    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=82)
    a = lq.Simulation(c.par, *c.arrays())
    a.step(11)
    before, clock = a.download(), a.clock()
    shape, skin = a.autotune(steps=8)
    assert 0 <= shape < 7
    assert min(abs(skin - f) for f in (0.02, 0.05, 0.1, 0.2)) < 1e-6
    for x, y in zip(before, a.download()):
        assert np.array_equal(x, y)
    assert a.clock() == clock
    assert not a.health().any()
    a.step(20)
    b = lq.Simulation(c.par, *c.arrays())
    b.step(11)
    b.set_pair_shape(shape)
    b.set_skin(skin)
    b.step(20)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
