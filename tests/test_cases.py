"""The case generators at the benchmark configurations' stated sizes, on the
CPU: particle counts, boundary-first order, coordinates inside the grid
that the reference hashes from raw coordinates (src/adami_boundary.cu:80-82),
seeding, and the batched ensemble's frames and material rows.  The GPU tests
and the bench build these cases, and the stated-size fixtures under
tests/golden/ sample them by index, so a generator that changed its counts
or its particle order would invalidate them.  Parameters are derived with
the oracle's restatement of src/loquat.cu:111-139, so no CUDA library is
loaded."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

import oracle
from loquat_b200 import cases

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(autouse=True, scope="module")
def oracle_parameters():
    prev = cases.use_parameter_initializer(oracle.initialize_parameters)
    yield
    cases.use_parameter_initializer(prev)


def check_layout(c):
    """Boundary particles first (object id 0), soil after (id 1), every
    coordinate in [0, cells x 2h) of its axis."""
    par = c.par
    assert c.pospres.shape == (par.np, 4) and c.str_.shape == (par.np, 6)
    assert par.np == par.npb + par.npm
    assert np.all(c.idep[:par.npb, 0] == 0.0) and np.all(c.idep[par.npb:, 0] == 1.0)
    xyz = c.pospres[:, :3].astype(np.float64)
    extent = 2.0 * par.h * np.array([par.cell_num_x, par.cell_num_y, par.cell_num_z], np.float64)
    assert np.all(xyz >= 0.0) and np.all(xyz < extent)


@pytest.mark.parametrize("make,npm,npb", [
    (lambda: cases.column_collapse(), 50_000, 116_184),
    (lambda: cases.cylinder_collapse(seed=1), 1_967_104, 344_763),
    (lambda: cases.slope_failure(seed=1), 2_852_360, 642_780),
    (lambda: cases.inclined_block(seed=1), 16_000_000, 1_627_920),
], ids=["column-50k", "cylinder-1.97M", "slope-2.85M", "inclined-16.0M"])
def test_generators_make_the_stated_sizes(make, npm, npb):
    c = make()
    assert (c.par.npm, c.par.npb) == (npm, npb)
    if c.par.np < 4_000_000:
        check_layout(c)


def test_generators_are_seeded():
    a, b = cases.column_collapse(seed=7), cases.column_collapse(seed=7)
    for x, y in zip(a.arrays(), b.arrays()):
        assert np.array_equal(x, y)
    c = cases.column_collapse(seed=8)
    assert not np.array_equal(a.pospres, c.pospres)
    assert a.par.to_bytes() == c.par.to_bytes()


def test_stated_fixture_sample_matches_the_generator():
    """The slope fixture's sampled particles are the ones the generator and
    the fixture script's sampling give today."""
    sys.path.insert(0, str(GOLDEN))
    from make_stated import stated_case

    z = np.load(GOLDEN / "slope_stated.npz")
    c, ids = stated_case("slope")
    assert (c.par.np, c.par.npm) == (int(z["np"]), int(z["npm"]))
    assert np.array_equal(ids, z["ids"])
    assert np.array_equal(c.idep[ids, 3], np.arange(ids.size, dtype=np.float32))


def test_ensemble_frames_and_materials():
    comb, parts = cases.ensemble()
    assert len(parts) == 256
    assert comb.par.npm == sum(p.par.npm for p in parts) == 14_049_150
    assert comb.par.npb == sum(p.par.npb for p in parts) == 16_163_838
    assert 4_000 < min(p.par.npm for p in parts) and max(p.par.npm for p in parts) < 220_000
    # boundary particles of every scenario first, then soil; object id k + 1
    # for scenario k in both layers
    ids = comb.idep[:, 0]
    assert np.array_equal(np.unique(ids), np.arange(1, 257, dtype=np.float32))
    nb = comb.par.npb
    b_ids = np.concatenate([np.full(p.par.npb, k + 1, np.float32) for k, p in enumerate(parts)])
    m_ids = np.concatenate([np.full(p.par.npm, k + 1, np.float32) for k, p in enumerate(parts)])
    assert np.array_equal(ids[:nb], b_ids) and np.array_equal(ids[nb:], m_ids)
    # each object its own block of grid rows, an empty row between blocks,
    # all inside the grid
    frames = np.asarray(comb.meta["frames"])
    assert frames.shape == (257, 2)
    for k in range(2, 257):
        assert frames[k, 0] >= frames[k - 1, 0] + frames[k - 1, 1] + 1
    assert frames[256, 0] + frames[256, 1] <= comb.par.cell_num_y
    # row k of the material table is scenario k - 1's (K, G, k_phi, k_psi, k_c)
    table = np.asarray(comb.meta["materials"])
    for k, p in enumerate(parts):
        assert np.allclose(table[k + 1], p.meta["material"], rtol=1e-6)
