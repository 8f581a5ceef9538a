"""Binary checkpoints of the native driver (lq_sim_save_checkpoint /
lq_sim_load_checkpoint): a simulation restored from the file and the
simulation that continued after saving take bit-identical steps, in both
precision forms, with the model-3 table, with per-object materials and
frames, across Shepard passes and list rebuilds, and from a graph-driven
run into an eagerly launched one."""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases

pytestmark = pytest.mark.gpu


def setup(sim, c):
    if "hypoplastic" in c.meta:
        sim.set_hypoplastic(c.meta["hypoplastic"])
    if "materials" in c.meta:
        sim.set_materials(c.meta["materials"])
        sim.set_frames(c.meta["frames"])
    return sim


def continued_vs_restored(lq, tmp_path, c, mixed, before=23, after=30, graph_after=True):
    a = setup(lq.Simulation(c.par, *c.arrays(), mixed=mixed), c)
    a.step(before)
    path = tmp_path / "state.lqck"
    a.save_checkpoint(path)
    a.step(after)
    b = lq.Simulation.load_checkpoint(path, graph=graph_after, mixed=mixed)
    assert b.clock() == (before, pytest.approx(before * c.par.dt, rel=1e-12))
    b.step(after)
    assert a.clock() == b.clock()
    for k, (x, y) in enumerate(zip(a.download(), b.download())):
        assert np.array_equal(x, y), k
    assert not a.health().any() and not b.health().any()
    return a, b


@pytest.mark.parametrize("mixed", [False, True])
def test_restart_is_bit_identical_drucker_prager(lq, cuda, tmp_path, mixed):
    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=51)
    a, b = continued_vs_restored(lq, tmp_path, c, mixed)
    assert a.rebuilds() >= 1                 # lists were rebuilt in the window


def test_restart_is_bit_identical_von_wolffersdorff_mixed(lq, cuda, tmp_path):
    c = cases.small_column(model=3, velocity_noise=0.05, shepard=7, seed=52)
    continued_vs_restored(lq, tmp_path, c, True)


def test_restart_of_a_batched_ensemble_into_eager_launches(lq, cuda, tmp_path):
    comb, _ = cases.ensemble(n=4, count_range=(1.5e3, 4.0e3), seed=12, shepard=7)
    continued_vs_restored(lq, tmp_path, comb, False, graph_after=False)


def test_checkpoint_of_the_other_form_is_refused(lq, cuda, tmp_path):
    c = cases.small_column(seed=53)
    a = lq.Simulation(c.par, *c.arrays(), mixed=True)
    a.step(2)
    a.save_checkpoint(tmp_path / "m.lqck")
    with pytest.raises(lq.LoquatError, match="LQ_SIM_MIXED"):
        lq.Simulation.load_checkpoint(tmp_path / "m.lqck", mixed=False)
