"""The neighbour search that allocates nothing (lq_grid_neighbor_search_noalloc).

Callers that cannot allocate device memory themselves (a host code whose own
pool already holds the GPU's memory, a time-step loop that cannot take
cudaMalloc's device-wide synchronisation) use this entry point: they pass
only inputs and outputs, and the working arrays live in a fixed array inside
the library.  Its results must equal those of lq_grid_neighbor_search, call
after call: the shared array keeps the previous call's contents, so two
calls in a row with different inputs check that nothing stale leaks through.

This file is collected last on purpose, so a run that stops at the first
failure has already run every other test."""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases
from helpers import copy_from_ptr, dev, host, par_dev, sync

pytestmark = pytest.mark.gpu


def reference_search(lq, par, pos_d, pd):
    g = lq.Grid(par.np, par.ncell)
    g.neighbor_search(par, pd, pos_d)
    sync()
    a = g.arrays()
    out = [copy_from_ptr(a[k], n) for k, n in (("part_cel", par.np), ("part_idx", par.np),
                                               ("cell_beg", par.ncell), ("cell_end", par.ncell))]
    g.close()
    return out


def noalloc_search(lq, cuda, par, pos_d, pd):
    outs = [cuda.full((n,), -7, dtype=cuda.int32, device="cuda") for n in (par.np, par.np, par.ncell, par.ncell)]
    lq.grid_neighbor_search_noalloc(par, pd, pos_d, *outs)
    sync()
    return [host(o) for o in outs]


def scrambled(case, seed):
    rng = np.random.default_rng(seed)
    pos = case.pospres.copy()
    k = rng.choice(pos.shape[0], 20, replace=False)
    pos[k[:10], 2] = -1.0                      # outside the lattice
    return pos[rng.permutation(pos.shape[0])]


def test_noalloc_search_matches_allocating_search_two_calls_in_a_row(lq, cuda):
    first = cases.column_collapse()            # 50 k soil + boundary, ~0.16 M particles
    second = cases.small_column(seed=4)        # a different, smaller problem on the same scratch
    for case, seed in ((first, 1), (second, 2)):
        par = case.par
        assert par.np <= lq.LQ_NOALLOC_MAX_PARTICLES and par.ncell <= lq.LQ_NOALLOC_MAX_CELLS
        pos = scrambled(case, seed)
        pos_d, pd = dev(pos), par_dev(par)
        want = reference_search(lq, par, pos_d, pd)
        got = noalloc_search(lq, cuda, par, pos_d, pd)
        for name, a, b in zip(("part_cel", "part_idx", "cell_beg", "cell_end"), got, want):
            assert np.array_equal(a, b), name


def test_noalloc_search_allocates_no_device_memory(lq, cuda):
    """The entry point's promise: after a first call of each problem (which
    loads its kernels), further calls of different sizes leave the device's
    free memory exactly where it was."""
    probs = []
    for case, seed in ((cases.column_collapse(), 3), (cases.small_column(seed=5), 4)):
        par = case.par
        pos_d, pd = dev(scrambled(case, seed)), par_dev(par)
        outs = [cuda.empty((n,), dtype=cuda.int32, device="cuda") for n in (par.np, par.np, par.ncell, par.ncell)]
        probs.append((par, pos_d, pd, outs))
    for par, pos_d, pd, outs in probs:
        lq.grid_neighbor_search_noalloc(par, pd, pos_d, *outs)
    sync()
    free0, _ = cuda.cuda.mem_get_info()
    for _ in range(3):
        for par, pos_d, pd, outs in probs:
            lq.grid_neighbor_search_noalloc(par, pd, pos_d, *outs)
    sync()
    free1, _ = cuda.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"


def test_noalloc_search_rejects_sizes_beyond_its_limits(lq, cuda):
    c = cases.small_column()
    par = c.par.copy()
    par.np = lq.LQ_NOALLOC_MAX_PARTICLES + 1
    par.npm = par.np - par.npb
    with pytest.raises(lq.LoquatError) as e:
        lq.grid_neighbor_search_noalloc(par, 1, 1, 1, 1, 1, 1)   # rejected before any device access
    assert e.value.status == lq.LQ_ERR_ARG and "exceed" in str(e.value)
