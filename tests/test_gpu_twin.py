"""Twin launch shapes of the pair kernel (11-14): a thread owns two
consecutive targets of one tile column and walks the union of their
neighbour lists, gathering each neighbour once for both.

* A target's sums run over its own pairs in the order of its
  thread-per-target list (entries out of its reach add exact zeros), but
  the twin kernel's instruction schedule rounds differently (and the
  compensated sums of the mixed form group the union's entries), so a twin
  shape agrees with the thread-per-target shapes to float rounding.
* The union lists also drive the Shepard and density filters, the batched
  ensemble (frames, per-object materials), model 3, a particle outside the
  lattice (its twin walks its stencil), and switching shapes mid-run.
"""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases
from helpers import by_id, rel_l2

pytestmark = pytest.mark.gpu

TWINS = (11, 12, 13, 14)


def assert_close(a_arrays, b_arrays, tol):
    """Same NaN pattern, and each state array within tol relative L2."""
    for k, (x, y) in enumerate(zip(a_arrays, b_arrays)):
        x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
        assert np.array_equal(np.isnan(x), np.isnan(y)), k
        ok = ~np.isnan(x)
        assert rel_l2(x[ok], y[ok]) <= tol, (k, rel_l2(x[ok], y[ok]))


@pytest.mark.parametrize("shape", TWINS)
def test_twin_shapes_step_like_thread_per_target_plain(lq, cuda, shape):
    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=91).with_ids()
    runs = []
    for sh in (0, shape):
        s = lq.Simulation(c.par, *c.arrays())
        s.set_pair_shape(sh)
        s.step(30)
        assert not s.health().any()
        runs.append(by_id(s.download()))
    assert_close(runs[1], runs[0], 1e-5)


@pytest.mark.parametrize("shape", (11, 12))
def test_twin_shapes_mixed_form_agree_to_rounding(lq, orc, cuda, shape):
    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=92).with_ids()
    runs = {}
    for sh in (0, shape):
        s = lq.Simulation(c.par, *c.arrays(), mixed=True)
        s.set_pair_shape(sh)
        s.step(30)
        assert not s.health().any()
        runs[sh] = by_id(s.download())
    nb = c.par.npb
    for k, tol in ((1, 1e-6), (3, 1e-6)):
        assert rel_l2(runs[shape][k][nb:], runs[0][k][nb:]) < tol, k
    o = orc.OracleSim(c.par, *c.arrays())
    o.step(30)
    want = by_id(o.get())
    assert rel_l2(runs[shape][1][nb:, :3], want[1][nb:, :3]) < 1e-4
    assert rel_l2(runs[shape][3][nb:], want[3][nb:]) < 1e-4


def test_twin_lists_with_frames_materials_filters_and_model_3(lq, cuda):
    comb, _ = cases.ensemble(n=5, count_range=(2.0e3, 4.0e3), seed=14, shepard=7)
    comb.idep[:, 3] = np.arange(comb.par.np, dtype=np.float32)
    comb.par.density_shepard_filter = 5
    out = []
    for shape in (0, 11):
        s = lq.Simulation(comb.par, *comb.arrays(), density_filter=True)
        s.set_materials(comb.meta["materials"])
        s.set_frames(comb.meta["frames"])
        s.set_pair_shape(shape)
        s.step(35)
        assert not s.health().any()
        out.append(by_id(s.download()))
    assert_close(out[1], out[0], 1e-5)
    v = cases.small_column(model=3, velocity_noise=0.05, shepard=7, seed=63).with_ids()
    out = []
    for shape in (0, 12):
        s = lq.Simulation(v.par, *v.arrays())
        s.set_hypoplastic(v.meta["hypoplastic"])
        s.set_pair_shape(shape)
        s.step(25)
        out.append(by_id(s.download()))
    assert_close(out[1], out[0], 1e-5)


@pytest.mark.parametrize("shape", (11, 13))
def test_twin_shape_switched_on_and_off_mid_run_with_escaped_particles(lq, cuda, shape):
    """Into a twin shape and back out between steps (each switch rebuilds
    the lists in the new kind), with particles outside the lattice: their
    slots sit in the out-of-lattice cell, whose twins are split and walk
    their stencils."""
    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=84).with_ids()
    a = lq.Simulation(c.par, *c.arrays())
    b = lq.Simulation(c.par, *c.arrays())
    a.set_pair_shape(0)
    b.set_pair_shape(0)
    a.step(9)
    b.step(9)
    pos, vel, idep, st, stn = a.download()
    pos[c.par.npb + 5, 0] = -1.0
    pos[c.par.npb + 9, 0] = -2.0
    a.upload(pos, vel, idep, st, stn)
    b.upload(pos, vel, idep, st, stn)
    a.step(2)
    b.step(2)
    b.set_pair_shape(shape)
    a.step(20)
    b.step(20)
    b.set_pair_shape(9)
    a.step(20)
    b.step(20)
    assert a.health()[1] >= 2
    assert_close(by_id(b.download()), by_id(a.download()), 1e-5)


def test_twin_neighbour_entries_count_each_targets_own_pairs(lq, cuda):
    c = cases.small_column(velocity_noise=0.1, seed=93)
    a = lq.Simulation(c.par, *c.arrays())
    a.set_pair_shape(0)
    a.step(1)
    b = lq.Simulation(c.par, *c.arrays())
    b.set_pair_shape(11)
    b.step(1)
    assert a.neighbor_entries() == b.neighbor_entries()
