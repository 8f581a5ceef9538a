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


THREAD_PER_TARGET = (0, 1, 2, 3, 4, 7, 8, 9, 10)   # 7-10 take their targets in tile order


def test_all_pair_kernel_shapes_agree_bit_for_bit(lq, cuda):
    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=81)
    out = []
    for shape in THREAD_PER_TARGET:
        s = lq.Simulation(c.par, *c.arrays(), mixed=True)
        s.set_pair_shape(shape)
        s.step(25)
        out.append(s.download())
    for other in out[1:]:
        for x, y in zip(out[0], other):
            assert np.array_equal(x, y)
    with pytest.raises(lq.LoquatError):
        s.set_pair_shape(11)


@pytest.mark.parametrize("shape", [7, 8, 9, 10])
def test_tile_order_switched_on_mid_run(lq, cuda, shape):
    """A tiled shape chosen between steps orders the current lists at once
    (no search is pending); the run goes on bit-identically, through later
    searches, with any of them -- also with a particle outside the lattice,
    whose slot sits in the out-of-lattice cell after every material cell."""
    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=84)
    a = lq.Simulation(c.par, *c.arrays())
    b = lq.Simulation(c.par, *c.arrays())
    a.set_pair_shape(0)
    a.step(9)
    b.step(9)
    pos, vel, idep, st, stn = a.download()
    pos[c.par.npb + 5, 0] = -1.0
    a.upload(pos, vel, idep, st, stn)
    b.upload(pos, vel, idep, st, stn)
    a.step(2)
    b.step(2)
    b.set_pair_shape(shape)
    a.step(40)
    b.step(40)
    assert b.rebuilds() > 2
    assert a.health()[1] >= 1
    # the escaped particle is in no material cell, so the Shepard filter's
    # sum over its cell neighbourhood is empty and gives 0/0, as the
    # reference's filter does (no zero guard): compare NaN as equal
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y, equal_nan=True)


def test_default_shape_is_tiled_for_large_cases(lq, cuda):
    """A new simulation starts with the tiled 640 x 1 shape when its targets
    fill four waves of 640-thread blocks on every SM, with shape 0 below
    that, and steps like one given that shape explicitly."""
    import torch

    sms = torch.cuda.get_device_properties(0).multi_processor_count
    small = cases.small_column(velocity_noise=0.3, seed=85)
    assert lq.Simulation(small.par, *small.arrays()).pair_shape() == 0
    n = int(np.ceil((4 * sms * 640 * 1.05) ** (1.0 / 3.0)))
    c = cases.small_column(nsx=n, nsy=n, nsz=n, velocity_noise=0.3, seed=86)
    assert c.par.npm >= 4 * sms * 640
    a = lq.Simulation(c.par, *c.arrays())
    assert a.pair_shape() == 9
    b = lq.Simulation(c.par, *c.arrays())
    b.set_pair_shape(0)
    a.step(12)
    b.step(12)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)


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
    assert 0 <= shape < 11
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


def test_tile_order_with_frames_materials_and_model_3(lq, cuda):
    """Tile order on a batched ensemble (per-object grid rows and materials)
    and on the von Wolffersdorff model in the mixed form: bit-identical to
    slot order."""
    comb, _ = cases.ensemble(n=5, count_range=(2.0e3, 4.0e3), seed=14, shepard=7)
    out = []
    for shape in (0, 8, 9):
        s = lq.Simulation(comb.par, *comb.arrays())
        s.set_materials(comb.meta["materials"])
        s.set_frames(comb.meta["frames"])
        s.set_pair_shape(shape)
        s.step(35)
        assert not s.health().any()
        out.append(s.download())
    for other in out[1:]:
        for x, y in zip(out[0], other):
            assert np.array_equal(x, y)
    v = cases.small_column(model=3, velocity_noise=0.05, shepard=7, seed=63)
    out = []
    for shape in (0, 10):
        s = lq.Simulation(v.par, *v.arrays(), mixed=True)
        s.set_hypoplastic(v.meta["hypoplastic"])
        s.set_pair_shape(shape)
        s.step(25)
        out.append(s.download())
    for x, y in zip(*out):
        assert np.array_equal(x, y)
