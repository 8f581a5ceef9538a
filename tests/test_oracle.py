"""The FP64 oracle against analytic results and independent restatements.

These pin the oracle before it is trusted as the parity reference:
grid = numpy stable argsort of float keys; Wendland C2 normalisation;
exact SPH responses to linear fields on a lattice; the spin/Jaumann sign
convention through a rigid rotation; Drucker-Prager and hypoplastic cases
worked by hand (reference src/predictor_corrector.cu:30-165)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from loquat_b200 import cases


def numpy_grid(par, pos, npb):
    pos = np.asarray(pos, np.float32)
    ih = np.float32(par.i_h)
    n = pos.shape[0]
    s = np.floor(np.float32(0.5) * pos[:, :3] * ih)      # float32 arithmetic, as the device
    dims = np.array([par.cell_num_x, par.cell_num_y, par.cell_num_z], np.float32)
    ok = np.all((s >= 0) & (s < dims), axis=1)            # NaN compares false
    c = np.where(ok[:, None], s, 0).astype(np.int64)
    key = par.ncell_one_layer * (np.arange(n) >= npb) + (c[:, 0] * par.cell_num_y + c[:, 1]) * par.cell_num_z + c[:, 2]
    key = np.where(ok, key, par.ncell_delete).astype(np.int32)
    idx = np.argsort(key, kind="stable").astype(np.int32)
    start = np.searchsorted(key[idx], np.arange(par.ncell + 1), side="left").astype(np.int32)
    return key[idx], idx, start


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_grid_is_stable_sort_of_float_keys(orc, seed):
    c = cases.small_column(seed=seed)
    rng = np.random.default_rng(seed)
    pos = c.pospres.copy()
    k = rng.choice(pos.shape[0], 40, replace=False)
    pos[k[:10], 0] = -0.01                     # outside, low side
    pos[k[10:20], 2] = 10.0                    # outside, high side
    pos[k[20:25], 1] = np.nan                  # non-finite
    pos = pos[rng.permutation(pos.shape[0])]   # scramble: exercises stability
    g = orc.grid_float(c.par, pos, c.par.npb)
    cel, idx, start = numpy_grid(c.par, pos, c.par.npb)
    assert np.array_equal(g["part_idx"], idx)
    assert np.array_equal(g["part_cel"], cel)
    assert np.array_equal(g["cell_start"], start)
    ne = start[1:] > start[:-1]
    assert np.array_equal(g["cell_beg"], np.where(ne, start[:-1], -1))
    assert np.array_equal(g["cell_end"], np.where(ne, start[1:], -1))
    assert g["part_cel"][-1] == c.par.ncell_delete


def test_wendland_constants_normalise(lq):
    p = lq.Parameters()
    p.dr, p.hdr = 0.002, 1.3
    p.domain_size_x = p.domain_size_y = p.domain_size_z = 0.1
    lq.initialize_parameters(p)
    h, C, Cg = float(p.h), float(p.kernel_normalization_par), float(p.kernel_gradient_normalization_par)
    r = np.linspace(0.0, 2 * h, 200001)
    q = r / h
    W = C * (2 - q) ** 4 * (q + 0.5)
    assert abs(np.trapezoid(W * 4 * np.pi * r * r, r) - 1.0) < 1e-5
    # grad W = C' (2 - q)^3 r_vec  <=>  dW/dr = C' (2 - q)^3 r
    dWdr = np.gradient(W, r)
    mid = slice(1000, 199000)
    assert np.allclose(dWdr[mid], Cg * (2 - q[mid]) ** 3 * r[mid], rtol=1e-4, atol=1e-6 * abs(Cg) * h)


def lattice_block(n=14, dr=0.002, hdr=1.2, rho0=2000.0):
    """Material-only cube (npb = 0) on a regular lattice, away from the origin."""
    from loquat_b200.params import Parameters
    from loquat_b200 import initialize_parameters

    g = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    xyz = (g + 0.5) * dr + 0.01
    p = Parameters()
    p.dr, p.hdr, p.rho0 = dr, hdr, rho0
    p.domain_size_x = p.domain_size_y = p.domain_size_z = 0.02 + n * dr
    p.cs, p.cfl = 30.0, 0.1
    p.constitutive_model = 1
    p.viscosity_type = 0
    p.np, p.npb, p.npm = xyz.shape[0], 0, xyz.shape[0]
    initialize_parameters(p)
    pos = np.zeros((xyz.shape[0], 4))
    pos[:, :3] = xyz
    vel = np.zeros((xyz.shape[0], 4))
    vel[:, 3] = rho0
    interior = np.all((g >= 4) & (g < n - 4), axis=1)
    return p, pos.astype(np.float32).astype(np.float64), vel, interior


def run_interaction(orc, p, pos, vel, s):
    g = orc.grid_float(p, pos.astype(np.float32), p.npb)
    idx = g["part_idx"]
    inv = np.empty_like(idx)
    inv[idx] = np.arange(idx.size)
    accad, spin, acestn = orc.interaction(p, pos[idx], vel[idx], s[idx], g["cell_beg"], g["cell_end"])
    return accad[inv], spin[inv], acestn[inv]


def test_interaction_linear_velocity_field(orc):
    p, pos, vel, interior = lattice_block()
    A = np.array([[0.3, -1.1, 0.4], [0.7, -0.2, 0.5], [-0.6, 0.9, 0.1]])
    vel[:, :3] = (pos[:, :3] - pos[:, :3].mean(0)) @ A.T
    accad, spin, acestn = run_interaction(orc, p, pos, vel, np.zeros((pos.shape[0], 6)))
    D = 0.5 * (A + A.T)
    W = 0.5 * (A - A.T)
    e, w = acestn[interior], spin[interior]
    # on a regular lattice the discrete gradient is the exact one times a
    # normalisation close to 1
    scale = np.median(e[:, 0] / D[0, 0])
    assert 0.9 < scale < 1.1
    for k, (a, b) in enumerate([(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]):
        assert np.allclose(e[:, k], scale * D[a, b], rtol=1e-5, atol=1e-9), k
    assert np.allclose(w[:, 0], scale * W[1, 0], rtol=1e-5)   # W_yx
    assert np.allclose(w[:, 1], scale * W[2, 0], rtol=1e-5)   # W_zx
    assert np.allclose(w[:, 2], scale * W[2, 1], rtol=1e-5)   # W_zy
    # continuity: drho/dt = -rho div v
    assert np.allclose(accad[interior, 3], -p.rho0 * scale * np.trace(A), rtol=1e-5)


def test_interaction_uniform_and_linear_stress(orc):
    p, pos, vel, interior = lattice_block()
    p.acc_z = -9.81
    s = np.tile(np.array([-3.0e4, -2.0e4, -5.0e4, 1.0e3, -2.0e3, 4.0e3]), (pos.shape[0], 1))
    accad, _, _ = run_interaction(orc, p, pos, vel, s)
    # the stress terms (|sigma| / (rho dr) ~ 1e4 m/s^2 each) cancel to the
    # float rounding of the lattice positions
    scale = 5.0e4 / (p.rho0 * p.dr)
    assert np.allclose(accad[interior, :3], [0.0, 0.0, -9.81], atol=1e-5 * scale)
    # geostatic column: sigma_zz = rho g (z - H) balances gravity
    H = pos[:, 2].max()
    s = np.zeros((pos.shape[0], 6))
    s[:, 2] = p.rho0 * 9.81 * (pos[:, 2] - H)
    accad, _, _ = run_interaction(orc, p, pos, vel, s)
    resid = accad[interior, 2]
    assert np.all(np.abs(resid) < 0.1 * 9.81), np.abs(resid).max()


def test_jaumann_spin_convention_rotates_stress_with_material(orc):
    """A rigid rotation v = Omega x r about z: the interaction pass gives the
    spin, the DP update (elastic: huge cohesion, no friction) then must rotate
    the stress exactly as the material rotates, sigma(t) = R sigma0 R^T."""
    p, pos, vel, interior = lattice_block()
    om = 2.0
    c = pos[:, :3].mean(0)
    vel[:, 0] = -om * (pos[:, 1] - c[1])
    vel[:, 1] = om * (pos[:, 0] - c[0])
    _, spin, acestn = run_interaction(orc, p, pos, vel, np.zeros((pos.shape[0], 6)))
    k = np.flatnonzero(interior)[0]
    w = spin[k, :3] / np.median(spin[interior, 0]) * om    # remove the lattice normalisation
    assert abs(w[0] - om) < 1e-5 * om and abs(w[1]) < 1e-5 * om and abs(w[2]) < 1e-5 * om
    assert np.abs(acestn[interior]).max() < 1e-5 * om
    p.model_par_1, p.model_par_2 = 1e6, 1e6
    p.model_par_3, p.model_par_4, p.model_par_5 = 0.0, 0.0, 1e12
    s0 = np.array([-5.0, -1.0, -2.0, 0.0, 0.0, 0.0])
    s = s0.copy()
    pp, ep = 0.0, 0.0
    n, T = 2000, 0.3
    for _ in range(n):
        pp, ep, s = orc.dp_update(p, T / n, w, np.zeros(6), pp, ep, s)
    th = om * T
    R = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    S0 = np.diag(s0[:3])
    St = R @ S0 @ R.T
    got = np.array([[s[0], s[3], s[4]], [s[3], s[1], s[5]], [s[4], s[5], s[2]]])
    assert np.allclose(got, St, atol=2e-3)


def dp_par(K=5e6, G=2e6, phi=30.0, psi=0.0, c=0.0):
    from loquat_b200.params import Parameters, dp_cone

    p = Parameters()
    kphi, kpsi, kc = dp_cone(phi, psi, c)
    p.model_par_1, p.model_par_2, p.model_par_3, p.model_par_4, p.model_par_5 = K, G, kphi, kpsi, kc
    p.constitutive_model = 1
    return p


def test_dp_elastic_inside_cone(orc):
    p = dp_par()
    s0 = np.array([-1e5, -1e5, -1e5, 0.0, 0.0, 0.0])
    d = np.array([1e-3, -2e-3, 0.5e-3, 1e-4, 0.0, -2e-4])
    dt = 1e-3
    pp, ep, s = orc.dp_update(p, dt, np.zeros(3), d, 0.0, 0.0, s0)
    K, G = float(p.model_par_1), float(p.model_par_2)
    lam = K - 2.0 / 3.0 * G
    want = s0 + dt * (2 * G * d + lam * d[:3].sum() * np.r_[1, 1, 1, 0, 0, 0])
    assert np.allclose(s, want, rtol=1e-12)
    assert ep == 0.0 and abs(pp + want[:3].mean()) < 1e-6


def test_dp_return_to_cone_and_tension_cut(orc):
    p = dp_par(psi=10.0, c=2e3)
    kphi, kpsi, kc = float(p.model_par_3), float(p.model_par_4), float(p.model_par_5)
    s0 = np.array([-1e4, -1e4, -1e4, 0.0, 0.0, 0.0])
    d = np.array([0.0, 0.0, 0.0, 5e-1, 0.0, 0.0])            # shear well past the cone
    pp, ep, s = orc.dp_update(p, 1e-2, np.zeros(3), d, 0.0, 0.0, s0)
    sm = s[:3].mean()
    dev = s.copy()
    dev[:3] -= sm
    tau = math.sqrt(0.5 * (dev[:3] @ dev[:3] + 2 * dev[3:] @ dev[3:]))
    assert abs(tau + kphi * sm - kc) < 1e-6 * abs(kc + 1e4)
    assert ep > 0 and abs(pp + sm) < 1e-9
    # isotropic extension beyond the tension cut-off lands on sm = tenf
    pp, ep, s = orc.dp_update(p, 1.0, np.zeros(3), np.array([1e-2, 1e-2, 1e-2, 0, 0, 0]), 0.0, 0.0,
                              np.zeros(6))
    tenf = kc / kphi
    assert abs(s[:3].mean() - tenf) < 1e-9 * tenf and ep > 0


def test_hypo_reset_keeps_xz(orc):
    """|tr T| < 4 resets T to diag(-1,-1,-2) but the reference clears xy twice
    and never xz (src/predictor_corrector.cu:140-141); the xz term survives."""
    from loquat_b200.params import Parameters

    p = Parameters()
    c1, c2, c3, c4 = -106.5, -801.5, -797.1, 1077.7
    p.model_par_1, p.model_par_2, p.model_par_3, p.model_par_4, p.model_par_5 = c1, c2, c3, c4, 0.0
    p.constitutive_model = 2
    c1, c2, c3, c4 = (float(p.model_par_1), float(p.model_par_2), float(p.model_par_3),
                      float(p.model_par_4))                    # the record holds floats
    s0 = np.array([-0.1, -0.2, 0.1, 0.05, 0.7, -0.3])        # |tr| < 4
    d = np.array([1e-3, 0.0, -1e-3, 0.0, 2e-3, 0.0])
    dt = 1e-3
    s = orc.hypo_update(p, dt, d, np.zeros(3), s0)
    T = np.array([-1.0, -1.0, -2.0, 0.0, 0.7, 0.0])          # xz kept
    t1 = -4.0
    Ts = T.copy()
    Ts[:3] -= t1 / 3.0
    contract = lambda a, b: a[:3] @ b[:3] + 2 * a[3:] @ b[3:]  # noqa: E731
    rate = d * (c1 * t1) + T * (c2 * d[:3].sum() + c3 * contract(T, d) / t1) + (T + Ts) * c4 * math.sqrt(
        contract(d, d))
    want = s0 + rate * dt
    pres = want[:3].mean()
    if pres > 0:
        want[:3] -= pres
    assert np.allclose(s, want, rtol=1e-12, atol=1e-15)


def test_oracle_sim_confined_block_stays_geostatic(orc):
    """A soil block in a closed box of Adami walls settles only slightly:
    velocities stay small and the vertical stress stays near rho g depth."""
    c = cases.small_column(nsx=10, nsy=6, nsz=10, shepard=0, front_wall=True)
    sim = orc.OracleSim(c.par, *c.arrays())
    sim.step(40)
    pos, vel, idep, s, stn = sim.get()
    nb = c.par.npb
    vmax = np.abs(vel[nb:, :3]).max()
    assert vmax < 0.05, vmax
    top = c.meta["top"]
    depth = top - pos[nb:, 2]
    deep = depth > 4 * c.par.dr
    want = -c.par.rho0 * 9.81 * depth[deep]
    got = s[nb:, 2][deep]
    assert np.median(np.abs(got - want) / np.abs(want)) < 0.15


def test_oracle_extensions_density_filter_and_dynamic_step(orc):
    """Density filter: a uniform density is a fixed point and noise is
    smoothed; dynamic step: never above cfl h / cs, equal to it at rest."""
    import numpy as np
    from loquat_b200 import cases

    c = cases.small_column(velocity_noise=0.0, shepard=0, seed=5)
    c.par.density_shepard_filter = 1
    o = orc.OracleSim(c.par, *c.arrays())
    o.set_extensions(density_filter=True, dynamic_dt=True)
    o.step(2)
    nb = c.par.npb
    rho = o.get()[1][nb:, 3]
    assert np.allclose(rho, c.par.rho0, rtol=2e-3)
    fixed = c.par.cfl * c.par.h / c.par.cs
    assert o.time() <= 2 * fixed * (1 + 1e-7)
    noisy = c.velrhop.copy()
    rng = np.random.default_rng(3)
    noisy[nb:, 3] *= 1 + rng.uniform(-1e-2, 1e-2, c.par.npm)
    p = orc.OracleSim(c.par, c.pospres, noisy, c.idep, c.str_, c.stn)
    p.set_extensions(density_filter=True)
    p.step(2)
    after = p.get()[1][nb:, 3]
    assert np.std(after) < 0.6 * np.std(noisy[nb:, 3])


def test_gather_rounding_experiment_switch(orc):
    """The oracle's precision experiment rounds only the neighbours'
    gathered velocity / sigma over rho^2: the rates move by about the
    16-bit rounding, and switching it off restores the exact rates."""
    p, pos, vel, interior = lattice_block()
    rng = np.random.default_rng(7)
    vel[:, :3] = rng.normal(0.0, 0.3, size=(pos.shape[0], 3))
    s = np.tile(np.array([-3.0e4, -2.0e4, -5.0e4, 1.0e3, -2.0e3, 4.0e3]), (pos.shape[0], 1))
    s *= 1.0 + 0.1 * rng.random((pos.shape[0], 1))
    exact = run_interaction(orc, p, pos, vel, s)
    err = {}
    try:
        for mode, field in ((orc.GATHER_F16_VELOCITY, 2), (orc.GATHER_BF16_STRESS, 0),
                            (orc.GATHER_FP21_VELOCITY, 2), (orc.GATHER_SHARED_EXP18_VELOCITY, 2)):
            orc.set_gather_rounding(mode)
            got = run_interaction(orc, p, pos, vel, s)
            d = np.linalg.norm(got[field][interior] - exact[field][interior]) / np.linalg.norm(exact[field][interior])
            err[mode] = d
            assert 1e-9 < d < 5e-2, (mode, d)
    finally:
        orc.set_gather_rounding(0)
    # finer packing, smaller error: FP16 (11 bits) > 21-bit floats (13) >
    # a shared exponent with 18-bit mantissas
    assert err[orc.GATHER_F16_VELOCITY] > err[orc.GATHER_FP21_VELOCITY] > err[orc.GATHER_SHARED_EXP18_VELOCITY]
    again = run_interaction(orc, p, pos, vel, s)
    for a, b in zip(again, exact):
        assert np.array_equal(a, b)
