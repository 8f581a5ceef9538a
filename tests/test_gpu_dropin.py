"""The reference's time step through the drop-in entry points
(loquat_b200.dropin.ReferenceStep: src/loquat.cu:322-409 with a search and
re-sort before each stage) against the FP64 oracle; the neighbour lists the
drop-in interaction carries across calls (its grid tracks particle
identities) against lists built afresh at every call; and the interaction's
working arrays: once reserved at set-up (lq_interaction_reserve, as
LoquatGrid::GridConfig does), its calls allocate no device memory."""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases
from helpers import by_id, rel_l2

pytestmark = pytest.mark.gpu


def test_reference_step_sequence_through_drop_in_entry_points_vs_oracle(lq, orc, cuda):
    from loquat_b200 import dropin

    c = cases.small_column(velocity_noise=0.05, shepard=4, seed=15).with_ids()
    r0, u0 = lq.interaction_stats()
    seq = dropin.ReferenceStep(c.par, *c.arrays())
    seq.step(10)
    got = by_id(seq.download())
    seq.close()
    r1, u1 = lq.interaction_stats()
    assert u1 - u0 > 0 and r1 - r0 >= 1       # the lists were carried over
    o = orc.OracleSim(c.par, *c.arrays())
    o.step(10)
    want = by_id(o.get())
    o.close()
    nb = c.par.npb
    assert rel_l2(got[1][nb:, :3], want[1][nb:, :3]) < 1e-4
    assert rel_l2(got[1][nb:, 3], want[1][nb:, 3]) < 1e-6
    assert rel_l2(got[3][nb:], want[3][nb:]) < 1e-4
    assert rel_l2(got[0][nb:, :3], want[0][nb:, :3]) < 1e-6


def test_carried_lists_match_fresh_lists(lq, cuda):
    """Fast particles (0.3 m/s noise) force several rebuilds in 30 steps;
    between them the carried lists (mapped to the re-sorted slots) give the
    fresh lists' results to float rounding: the same pairs, summed in the
    build's order."""
    from loquat_b200 import dropin

    c = cases.small_column(velocity_noise=0.3, shepard=7, seed=16).with_ids()
    runs = []
    for carry in (True, False):
        r0, u0 = lq.interaction_stats()
        seq = dropin.ReferenceStep(c.par, *c.arrays(), carry=carry)
        seq.step(30)
        runs.append(by_id(seq.download()))
        seq.close()
        r1, u1 = lq.interaction_stats()
        if carry:
            assert r1 - r0 >= 2 and u1 - u0 >= 10, (r1 - r0, u1 - u0)
        else:
            assert (r1, u1) == (r0, u0)
    nb = c.par.npb
    for k, tol in ((0, 1e-7), (1, 1e-5), (3, 1e-5)):
        assert rel_l2(runs[0][k][nb:], runs[1][k][nb:]) < tol, k


def test_reserved_interaction_allocates_nothing_per_call(lq, cuda):
    import torch

    from helpers import copy_from_ptr, dev, par_dev, sync

    c = cases.column_collapse()
    par = c.par
    g = lq.Grid(par.np, par.ncell)
    pd = par_dev(par)
    g.neighbor_search(par, pd, dev(c.pospres))
    a = g.arrays()
    # the state in the grid's order, as the reference's sort leaves it
    perm = torch.from_numpy(copy_from_ptr(a["part_idx"], par.np).astype(np.int64)).cuda()
    st = [dev(x)[perm].contiguous() for x in c.arrays()]
    rates = [torch.zeros((par.np, 4), device="cuda"), torch.zeros((par.np, 4), device="cuda"),
             torch.zeros((par.np, 6), device="cuda")]
    lq.interaction_reserve(par)
    lq.particle_interaction(par, pd, *st, *rates, a["cell_beg"], a["cell_end"])
    sync()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        lq.particle_interaction(par, pd, *st, *rates, a["cell_beg"], a["cell_end"])
    sync()
    free1, _ = torch.cuda.mem_get_info()
    g.close()
    assert free1 == free0
    assert torch.isfinite(rates[0][par.npb:]).all()
