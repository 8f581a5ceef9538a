"""Neighbour grid on the GPU: hash, stable sort and bounds are bit-exact
against the oracle's float-key stable sort, including out-of-lattice and
non-finite positions, empty layers and degenerate sizes; the gathers are
exact permutations."""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases
from helpers import copy_from_ptr, dev, par_dev, sync

pytestmark = pytest.mark.gpu


def run_grid(lq, par, pos):
    n = pos.shape[0]
    g = lq.Grid(n, par.ncell)
    pd = par_dev(par)
    pos_d = dev(pos)
    g.neighbor_search(par, pd, pos_d)
    sync()
    a = g.arrays()
    out = dict(part_cel=copy_from_ptr(a["part_cel"], n), part_idx=copy_from_ptr(a["part_idx"], n),
               cell_beg=copy_from_ptr(a["cell_beg"], par.ncell), cell_end=copy_from_ptr(a["cell_end"], par.ncell),
               cell_start=copy_from_ptr(a["cell_start"], par.ncell + 1))
    return g, out


def assert_same_grid(got, want):
    for k in ("part_idx", "part_cel", "cell_beg", "cell_end", "cell_start"):
        assert np.array_equal(got[k], want[k]), k


def perturbed(case, seed, n_out=40):
    rng = np.random.default_rng(seed)
    pos = case.pospres.copy()
    k = rng.choice(pos.shape[0], n_out, replace=False)
    pos[k[: n_out // 4], 0] = -0.05
    pos[k[n_out // 4: n_out // 2], 2] = 1e3
    pos[k[n_out // 2: n_out // 2 + 5], 1] = np.nan
    pos[k[-3:], 0] = np.inf
    return pos[rng.permutation(pos.shape[0])]


@pytest.mark.parametrize("seed", [0, 1])
def test_grid_small_scrambled_with_outliers(lq, orc, cuda, seed):
    c = cases.small_column(seed=seed)
    pos = perturbed(c, seed)
    _, got = run_grid(lq, c.par, pos)
    assert_same_grid(got, orc.grid_float(c.par, pos, c.par.npb))


def test_grid_column_collapse_full_size(lq, orc, cuda):
    c = cases.column_collapse()
    assert c.par.npm == 50_000
    pos = perturbed(c, 7, n_out=200)
    _, got = run_grid(lq, c.par, pos)
    assert_same_grid(got, orc.grid_float(c.par, pos, c.par.npb))


def test_grid_degenerate_sizes(lq, orc, cuda):
    c = cases.small_column()
    par = c.par.copy()
    # all material (no boundary layer), all in one cell, and a single particle
    for npb, pos in [(0, c.pospres[c.par.npb:].copy()),
                     (0, np.tile(np.array([[0.011, 0.011, 0.011, 0.0]], np.float32), (3000, 1))),
                     (1, c.pospres[:1].copy())]:
        par.np, par.npb, par.npm = pos.shape[0], npb, pos.shape[0] - npb
        _, got = run_grid(lq, par, pos)
        assert_same_grid(got, orc.grid_float(par, pos, npb))


def test_grid_repeated_search_reuses_buffers(lq, orc, cuda):
    c = cases.small_column(seed=5)
    g = lq.Grid(c.par.np, c.par.ncell)
    pd = par_dev(c.par)
    for s in range(3):
        pos = perturbed(c, 10 + s)
        g.neighbor_search(c.par, pd, dev(pos))
        sync()
        a = g.arrays()
        assert np.array_equal(copy_from_ptr(a["part_idx"], c.par.np),
                              orc.grid_float(c.par, pos, c.par.npb)["part_idx"])


def test_sort_arrays_are_exact_permutations(lq, orc, cuda):
    t = cuda
    c = cases.small_column(seed=2)
    pos = perturbed(c, 3)
    g, got = run_grid(lq, c.par, pos)
    idx = got["part_idx"]
    rng = np.random.default_rng(0)
    f4 = rng.standard_normal((c.par.np, 4)).astype(np.float32)
    t2 = rng.standard_normal((c.par.np, 6)).astype(np.float32)
    d4, d6 = dev(f4), dev(t2)
    c4, c6 = t.empty_like(d4), t.empty_like(d6)
    g.sort_float4(c.par.np, d4, c4)
    g.sort_tensor2d(c.par.np, d6, c6)
    sync()
    assert np.array_equal(d4.cpu().numpy(), f4[idx])
    assert np.array_equal(d6.cpu().numpy(), t2[idx])
