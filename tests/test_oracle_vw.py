"""The oracle's von Wolffersdorff hypoplastic model (constitutive model 3,
not in the reference; written from von Wolffersdorff 1996) against the
model's defining properties.  CPU only."""
from __future__ import annotations

import math

import numpy as np
import pytest

# sand of the slope configurations: phic 30 deg, hs 2.6 GPa, n 0.27,
# ed0 0.61, ec0 0.98, ei0 1.10, alpha 0.18, beta 1.0; tolerance 1e-4
ROW = np.array([30.0, 2.6e9, 0.27, 0.61, 0.98, 1.10, 0.18, 1.0, 1e-4, 2000], np.float32)


def test_rate_is_homogeneous_of_degree_one_in_stretching(orc):
    s = np.array([-2e4, -1.5e4, -3e4, 1e3, -2e3, 5e2])
    d = np.array([1e-3, -2e-3, -4e-3, 5e-4, 1e-4, -3e-4])
    r1, e1 = orc.vw_rate(ROW, s, 0.72, d, np.zeros(3))
    r2, e2 = orc.vw_rate(ROW, s, 0.72, 3.0 * d, np.zeros(3))
    assert np.allclose(r2, 3.0 * r1, rtol=1e-12) and math.isclose(e2, 3.0 * e1, rel_tol=1e-12)


def test_isotropic_compression_stays_isotropic_and_densifies(orc):
    s = np.array([-1e4, -1e4, -1e4, 0, 0, 0.0])
    d = np.array([-1e-2, -1e-2, -1e-2, 0, 0, 0.0])
    e = 0.80
    for _ in range(50):
        s, e, _ = orc.vw_update(ROW, 1e-2, d, np.zeros(3), s, e)
    assert np.allclose(s[:3], s[0], rtol=1e-10) and np.allclose(s[3:], 0.0)
    assert s[0] < -1e4 and e < 0.80
    # e after 0.5 % volumetric compression: (1 + e) shrinks by exp(-0.015)
    assert math.isclose(1 + e, 1.80 * math.exp(-3 * 50 * 1e-2 * 1e-2), rel_tol=1e-3)


def test_substepping_converges(orc):
    s0 = np.array([-1e4, -1e4, -2e4, 0, 0, 0.0])
    d = np.array([2e-3, 2e-3, -1e-2, 0, 3e-3, 0.0])
    w = np.array([0.5, -0.2, 0.1])
    loose = ROW.copy()
    tight = ROW.copy()
    tight[8] = 1e-7
    a, ea, na = orc.vw_update(loose, 0.5, d, w, s0, 0.75)
    b, eb, nb = orc.vw_update(tight, 0.5, d, w, s0, 0.75)
    assert nb > na >= 1
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-3


def test_substep_cap_still_integrates_the_whole_step(orc):
    s0 = np.array([-1e4, -1e4, -2e4, 0, 0, 0.0])
    d = np.array([2e-3, 2e-3, -1e-2, 0, 3e-3, 0.0])
    capped = ROW.copy()
    capped[8], capped[9] = 1e-12, 20            # tolerance out of reach, 20 sub-steps at most
    a, ea, na = orc.vw_update(capped, 0.5, d, np.zeros(3), s0, 0.75)
    b, eb, nb = orc.vw_update(ROW, 0.5, d, np.zeros(3), s0, 0.75)
    assert na <= 20
    # every trial is rejected until the last allowed one, which spans the rest of the
    # interval in one Heun step: same end time, coarser result
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 5e-2


def test_triaxial_compression_reaches_the_critical_state(orc):
    """Drained triaxial compression at constant cell pressure: at large axial
    strain the stress ratio q/p tends to M = 6 sin phic / (3 - sin phic),
    dilatancy dies out and the void ratio tends to the critical one."""
    p0 = 1.0e5
    s = np.array([-p0, -p0, -p0, 0, 0, 0.0])
    e = 0.85
    dt = 1.0
    da = -5e-4                       # axial strain per step (compression)
    dr = -0.5 * da                   # first guess of the lateral rate
    for _ in range(2400):            # 120 % axial strain
        # lateral rate that keeps the cell pressure: secant on sigma_r
        def lateral(x):
            t, _, _ = orc.vw_update(ROW, dt, np.array([x, x, da, 0, 0, 0]), np.zeros(3), s, e)
            return t[0] + p0
        f0, f1 = lateral(dr), lateral(dr * 1.01 + 1e-9)
        dr = dr - f0 * (dr * 0.01 + 1e-9) / (f1 - f0)
        s, e, _ = orc.vw_update(ROW, dt, np.array([dr, dr, da, 0, 0, 0]), np.zeros(3), s, e)
    p = -(s[0] + s[1] + s[2]) / 3.0
    q = abs(s[2] - s[0])
    sphi = math.sin(math.radians(ROW[0]))
    M = 6 * sphi / (3 - sphi)
    assert abs(s[0] + p0) < 1e-3 * p0
    assert abs(q / p - M) < 0.02 * M, (q / p, M)
    ec = ROW[4] * math.exp(-(3 * p / ROW[1]) ** ROW[2])
    assert abs(e - ec) < 0.01 * ec, (e, ec)
    assert abs(2 * dr / da + 1) < 0.02               # volumetric / axial strain rate -> 0


def test_states_outside_the_limit_surface_give_finite_rates(orc):
    """Near-zero and tensile stresses (free surface) must not produce NaN:
    tr T >= -3 Pa is reset, tan psi beyond sqrt2 is scaled back inside."""
    d = np.array([1e-3, -2e-3, -4e-3, 5e-4, 1e-4, -3e-4])
    for s in ([-2.94, -1.95, 1.65, -1.0, -3.09, 0.55],      # tr T = -3.24 Pa, tan psi = 3.1
              [-5e3, 2e3, 1e3, 0, 0, 0],                      # tension in two directions
              [1.0, 1.0, 1.0, 0, 0, 0],                       # all tension
              [-1e4, 0.0, 0.0, 0, 0, 0]):                     # uniaxial: tan psi = sqrt2 exactly
        r, er = orc.vw_rate(ROW, np.array(s, float), 0.7, d, np.array([0.1, 0.0, -0.2]))
        assert np.isfinite(r).all() and math.isfinite(er), s
        t, e, n = orc.vw_update(ROW, 1e-3, d, np.zeros(3), np.array(s, float), 0.7)
        assert np.isfinite(t).all() and math.isfinite(e), s


def test_projection_is_continuous_at_the_limit_surface(orc):
    """Just inside and just outside tan psi = sqrt2 (1 - 1e-3) the rate is the same."""
    d = np.array([-1e-3, 5e-4, 5e-4, 0, 0, 0.0])
    lim = math.sqrt(2.0) * (1 - 1e-3)
    p = 1e4
    # axisymmetric compression state with tan psi = x: That* = diag(2, -1, -1) x / (3 sqrt2)
    def state(x):
        ts = np.array([2, -1, -1]) * x / (3 * math.sqrt(2))
        th = ts + 1.0 / 3.0
        return np.concatenate([-3 * p * th, np.zeros(3)])
    a, _ = orc.vw_rate(ROW, state(lim * (1 - 1e-9)), 0.7, d, np.zeros(3))
    b, _ = orc.vw_rate(ROW, state(lim * (1 + 1e-9)), 0.7, d, np.zeros(3))
    c, _ = orc.vw_rate(ROW, state(lim * 1.5), 0.7, d, np.zeros(3))
    assert np.allclose(a, b, rtol=1e-6)
    assert np.allclose(b, c, rtol=1e-6)    # the scaled-back state is the same
