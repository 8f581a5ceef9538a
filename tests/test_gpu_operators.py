"""Per-operator parity on the GPU, through the C ABI, on identical sorted
inputs:
  * interaction, Adami, Shepard, predictor, corrector against the FP64 oracle
    (relative L2 tolerances stated per test);
  * Adami, Shepard, predictor and corrector also against the reference's
    own kernels compiled from its sources (oracle/_ref), which they match to
    a few float ulps."""
from __future__ import annotations

import numpy as np
import pytest

from loquat_b200 import cases
from helpers import dev, host, par_dev, rel_l2, sorted_state, sync, ulp_diff, zeros

pytestmark = pytest.mark.gpu

# FP32 kernel vs FP64 oracle on one pass, same inputs.  The momentum sum
# cancels terms ~|sigma|/(rho dr) down to ~g, so its relative error is the
# float rounding of those terms; the other outputs do not cancel as much.
TOL_INTERACTION = {"accad_xyz": 5e-4, "drho": 1e-4, "spin": 1e-4, "acestn": 1e-4}
TOL_ADAMI = 1e-5
TOL_SHEPARD = 1e-5
TOL_INTEGRATOR = 1e-6
MAX_ULP_VS_REFERENCE = 64


def interaction_case(**kw):
    return cases.small_column(velocity_noise=0.05, **kw)


@pytest.mark.parametrize("kw", [dict(), dict(hdr=1.3, seed=4), dict(hdr=1.5, seed=5, nsx=12)])
def test_interaction_vs_oracle(lq, orc, cuda, kw):
    c = interaction_case(**kw)
    par = c.par
    g, st = sorted_state(orc, c)
    # Adami first so boundary neighbours carry realistic stress
    st[3] = orc.adami(par, st[0], st[1], st[3], g["cell_beg"], g["cell_end"]).astype(np.float32)
    n = par.np
    d = [dev(a) for a in st]
    accad, spin, acestn = zeros((n, 4)), zeros((n, 4)), zeros((n, 6))
    pd, beg, end = par_dev(par), dev(g["cell_beg"]), dev(g["cell_end"])
    lq.particle_interaction(par, pd, *d, accad, spin, acestn, beg, end)
    sync()
    oa, os_, oe = orc.interaction(par, st[0], st[1], st[3], g["cell_beg"], g["cell_end"])
    m = slice(par.npb, n)
    ga, gs, ge = host(accad)[m], host(spin)[m], host(acestn)[m]
    errs = {"accad_xyz": rel_l2(ga[:, :3], oa[m, :3]), "drho": rel_l2(ga[:, 3], oa[m, 3]),
            "spin": rel_l2(gs, os_[m]), "acestn": rel_l2(ge, oe[m])}
    for k, tol in TOL_INTERACTION.items():
        assert errs[k] < tol, (k, errs)
    assert np.all(host(accad)[: par.npb] == 0.0)  # boundary slots untouched


def test_interaction_artificial_stress_and_no_viscosity(lq, orc, cuda):
    c = interaction_case(seed=9)
    par = c.par
    par.artificial_pressure = 1
    par.artificial_pressure_coefficient = 0.3
    par.viscosity_type = 0
    lq.initialize_parameters(par)
    par.dt = par.cfl * par.h / par.cs
    c.str_[par.npb::7, 0] = 2.0e3     # some tensile components
    g, st = sorted_state(orc, c)
    n = par.np
    d = [dev(a) for a in st]
    accad, spin, acestn = zeros((n, 4)), zeros((n, 4)), zeros((n, 6))
    pd, beg, end = par_dev(par), dev(g["cell_beg"]), dev(g["cell_end"])
    lq.particle_interaction(par, pd, *d, accad, spin, acestn, beg, end)
    sync()
    oa, _, _ = orc.interaction(par, st[0], st[1], st[3], g["cell_beg"], g["cell_end"])
    m = slice(par.npb, n)
    assert rel_l2(host(accad)[m, :3], oa[m, :3]) < TOL_INTERACTION["accad_xyz"]


def adami_inputs(orc, seed=0):
    c = cases.small_column(seed=seed, velocity_noise=0.02)
    g, st = sorted_state(orc, c)
    rng = np.random.default_rng(seed)
    st[1][:, 3] *= (1.0 + 0.02 * rng.standard_normal(c.par.np)).astype(np.float32)  # varied density
    st[3][c.par.npb:] += (1e2 * rng.standard_normal((c.par.npm, 6))).astype(np.float32)
    return c, g, st


def test_adami_vs_oracle_and_reference_kernel(lq, orc, cuda):
    c, g, st = adami_inputs(orc)
    par = c.par
    want = orc.adami(par, st[0], st[1], st[3], g["cell_beg"], g["cell_end"])
    pd, x, v, s_d = par_dev(par), dev(st[0]), dev(st[1]), dev(st[3])
    beg, end = dev(g["cell_beg"]), dev(g["cell_end"])
    lq.adami_boundary(par, pd, x, v, s_d, beg, end)
    sync()
    got = host(s_d)
    b = slice(0, par.npb)
    assert rel_l2(got[b], want[b]) < TOL_ADAMI
    assert np.array_equal(got[par.npb:], st[3][par.npb:])      # material stress untouched
    if orc.ref_available():
        # every buffer is bound to a name until the call returns
        ph, pd = par.copy(), par_dev(par)
        x, v, s_r, beg, end = dev(st[0]), dev(st[1]), dev(st[3]), dev(g["cell_beg"]), dev(g["cell_end"])
        rc = orc.ref_lib().ref_adami(lq.ptr(ph), pd.data_ptr(), x.data_ptr(), v.data_ptr(), s_r.data_ptr(),
                                     beg.data_ptr(), end.data_ptr())
        assert rc == 0
        assert ulp_diff(got, host(s_r)) <= MAX_ULP_VS_REFERENCE


def test_shepard_vs_oracle_and_reference_kernel(lq, orc, cuda):
    c, g, st = adami_inputs(orc, seed=3)
    par = c.par
    want = orc.shepard(par, st[0], st[1], st[3], g["cell_beg"], g["cell_end"])
    pd, x, v, s_d, cache = par_dev(par), dev(st[0]), dev(st[1]), dev(st[3]), zeros((par.np, 6))
    beg, end = dev(g["cell_beg"]), dev(g["cell_end"])
    lq.stress_regularization(par, pd, x, v, s_d, cache, beg, end)
    sync()
    got = host(s_d)
    m = slice(par.npb, par.np)
    assert rel_l2(got[m], want[m]) < TOL_SHEPARD
    assert np.array_equal(got[: par.npb], st[3][: par.npb])
    if orc.ref_available():
        ph, pd = par.copy(), par_dev(par)
        x, v, s_r, cache_r = dev(st[0]), dev(st[1]), dev(st[3]), zeros((par.np, 6))
        beg, end = dev(g["cell_beg"]), dev(g["cell_end"])
        rc = orc.ref_lib().ref_shepard(lq.ptr(ph), pd.data_ptr(), x.data_ptr(), v.data_ptr(), s_r.data_ptr(),
                                       cache_r.data_ptr(), beg.data_ptr(), end.data_ptr())
        assert rc == 0
        assert ulp_diff(got, host(s_r)) <= MAX_ULP_VS_REFERENCE


def integrator_inputs(model, seed):
    c = cases.small_column(model=model, seed=seed, velocity_noise=0.05)
    par = c.par
    rng = np.random.default_rng(seed)
    n = par.np
    st = [a.copy() for a in c.arrays()]
    st[3][par.npb:] += (2e3 * rng.standard_normal((par.npm, 6))).astype(np.float32)
    st[4][:] = (1e-3 * rng.standard_normal((n, 6))).astype(np.float32)
    st[2][:, 1] = np.abs(1e-3 * rng.standard_normal(n)).astype(np.float32)
    accad = np.zeros((n, 4), np.float32)
    accad[:, :3] = rng.standard_normal((n, 3)) * 20.0
    accad[:, 3] = rng.standard_normal(n) * 500.0
    spin = np.zeros((n, 4), np.float32)
    spin[:, :3] = rng.standard_normal((n, 3)) * 5.0
    acestn = (rng.standard_normal((n, 6)) * 20.0).astype(np.float32)
    # a slice of particles pushed far past the yield surface / tension cut-off
    acestn[par.npb::5, 3] *= 200.0
    acestn[par.npb + 1::7, :3] = 500.0
    # the hypoplastic near-zero reset path
    st[3][par.npb + 2::11] = np.float32(0.1)
    return par, st, [accad, spin, acestn]


def _run_ours(lq, par, st, ini, rates, which):
    d = [dev(a) for a in st]
    di = [dev(a) for a in ini]
    dr = [dev(a) for a in rates]
    fn = lq.predictor if which == "predictor" else lq.corrector
    pd = par_dev(par)
    fn(par, pd, d, di, dr)
    sync()
    return [host(a) for a in d], [host(a) for a in di]


def _run_ref(orc, lq, par, st, ini, rates, which):
    d = [dev(a) for a in st]
    di = [dev(a) for a in ini]
    dr = [dev(a) for a in rates]
    f = orc.ref_lib().ref_predictor if which == "predictor" else orc.ref_lib().ref_corrector
    ph, pd = par.copy(), par_dev(par)
    rc = f(lq.ptr(ph), pd.data_ptr(), *[a.data_ptr() for a in d + di + dr])
    assert rc == 0
    return [host(a) for a in d], [host(a) for a in di]


@pytest.mark.parametrize("model", [1, 2])
@pytest.mark.parametrize("which", ["predictor", "corrector"])
def test_integrator_vs_oracle_and_reference_kernel(lq, orc, cuda, model, which):
    par, st, rates = integrator_inputs(model, seed=11 + model)
    rng = np.random.default_rng(5)
    if which == "predictor":
        ini = [np.zeros_like(a) for a in st]
        want = orc.predictor(par, st, rates)
    else:
        ini = [a.copy() for a in st]
        ini[1][:, :3] += (0.01 * rng.standard_normal((par.np, 3))).astype(np.float32)
        want = orc.corrector(par, st, ini, rates)
    got, snap = _run_ours(lq, par, st, ini, rates, which)
    m = slice(par.npb, par.np)
    names = ["pospres", "velrhop", "idep", "str", "stn"]
    for k, name in enumerate(names):
        assert rel_l2(got[k][m], want[k][m]) < TOL_INTEGRATOR, name
        assert np.array_equal(got[k][: par.npb], st[k][: par.npb]), name   # boundary untouched
    if which == "predictor":
        for k in range(5):
            assert np.array_equal(snap[k], st[k])                           # snapshot of every slot
    if orc.ref_available():
        ref, ref_snap = _run_ref(orc, lq, par, st, ini, rates, which)
        for k, name in enumerate(names):
            assert ulp_diff(got[k], ref[k]) <= MAX_ULP_VS_REFERENCE, name
        if which == "predictor":
            for k in range(5):
                assert np.array_equal(snap[k], ref_snap[k])


def test_zero_material_particles_is_a_no_op(lq, cuda):
    c = cases.small_column()
    par = c.par.copy()
    par.np, par.npb, par.npm = par.npb, par.npb, 0
    n = par.np
    accad = zeros((n, 4))
    st = [dev(a[:n]) for a in c.arrays()]
    pd, spin, acestn = par_dev(par), zeros((n, 4)), zeros((n, 6))
    beg = dev(np.full(par.ncell, -1, np.int32))
    ini = [zeros(a.shape) for a in st]
    lq.particle_interaction(par, pd, *st, accad, spin, acestn, beg, beg)
    lq.predictor(par, pd, st, ini, [accad, spin, acestn])
    sync()
    assert float(accad.abs().sum()) == 0.0
