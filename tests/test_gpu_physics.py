"""Physics regression on the GPU (the reference has no tests; these are the
checks a geomechanics user expects of the scheme):

* a soil block at rest in a closed box of Adami walls keeps v ~ 0 and the
  geostatic sigma_zz ~ -rho g depth;
* a small spherical pulse in a cube of fluid-like elastic material (G = 0,
  no yield) spreads at the sound speed sqrt(K / rho) -- the reference's cs
  convention -- in both precision forms."""
from __future__ import annotations

import math

import numpy as np
import pytest

from loquat_b200 import cases
from loquat_b200.params import elastic_moduli
from helpers import by_id

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mixed", [False, True])
def test_confined_block_stays_geostatic(lq, cuda, mixed):
    c = cases.small_column(nsx=16, nsy=8, nsz=16, shepard=30, front_wall=True, seed=91).with_ids()
    sim = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
    sim.step(400)
    pos, vel, idep, s, stn = by_id(sim.download())
    nb = c.par.npb
    H = c.meta["top"] - 3 * c.par.dr
    vmax = np.abs(vel[nb:, :3]).max()
    assert vmax < 0.02 * math.sqrt(9.81 * H), vmax
    depth = c.meta["top"] - pos[nb:, 2]
    deep = depth > 4 * c.par.dr
    want = -c.par.rho0 * 9.81 * depth[deep]
    got = s[nb:, 2][deep]
    assert np.median(np.abs(got - want) / np.abs(want)) < 0.15
    assert not sim.health().any()


def sphere_pulse(n=56, dr=0.002, hdr=1.2, rho0=2000.0, E=1.0e6, nu=0.3, amp=0.01, width=4.0, alpha=0.05):
    """A cube of soil with free surfaces, no gravity and no initial stress,
    and a smooth spherical pulse of radial velocity at its centre.
    Material: Drucker-Prager with G = 0 and a yield surface out of reach
    (the tension cut k_c / k_phi at 1e9 Pa), so the stress is a pressure
    and waves travel at sqrt(K / rho0).  Without walls, nothing slows the
    front (no-slip walls lower the discrete strain rate of their
    neighbours)."""
    soil = cases._lattice(n, n, n, dr, (0.0, 0.0, 0.0))
    K, G = elastic_moduli(E, nu)
    par = cases._base_parameters(dr, hdr, rho0, (n * dr,) * 3, E, nu, 0.1, 1,
                                 lambda K_, G_: (K_, 0.0, 1e-6, 0.0, 1.0e3), 0, alpha, (0.0, 0.0, 0.0))
    c = cases.assemble("sphere_pulse", par, np.zeros((0, 3)), soil, np.random.default_rng(0), 0.0, rho0, 0.0,
                       0.0, 0.0, 1.0, meta=dict(dr=dr))
    ctr = np.full(3, n * dr / 2)
    d = c.pospres[:, :3].astype(np.float64) - ctr
    r = np.linalg.norm(d, axis=1)
    w = width * dr
    prof = amp * np.exp(-(r / w) ** 2) * (r / w)
    c.velrhop[:, :3] = (prof[:, None] * d / np.maximum(r, 1e-12)[:, None]).astype(np.float32)
    c.meta.update(ctr=ctr, K=K, n=n)
    return c


def front_radius(c, arrays, lo=0.0, hi=None):
    """Radius of the outgoing front: the peak of r v_r (radial velocity in
    shells of one spacing, times r to undo the spherical spreading) between
    radii lo and hi, refined by a parabola through its neighbours.  The
    window keeps the search off the ringing that the pulse leaves behind
    near the centre."""
    pos, vel = by_id(arrays)[:2]
    dr = c.meta["dr"]
    d = pos[:, :3].astype(np.float64) - c.meta["ctr"]
    r = np.linalg.norm(d, axis=1)
    vr = (vel[:, :3].astype(np.float64) * d).sum(1) / np.maximum(r, 1e-12)
    k = np.floor(r / dr).astype(int)
    nb = c.meta["n"] // 2
    ok = k < nb
    prof = np.bincount(k[ok], weights=(r * vr)[ok], minlength=nb) / np.maximum(np.bincount(k[ok], minlength=nb), 1)
    j0 = max(2, int(lo / dr))
    j1 = min(nb - 2, int(hi / dr) if hi is not None else nb - 2)
    j = int(np.argmax(prof[j0:j1])) + j0
    a, b, cc = prof[j - 1], prof[j], prof[j + 1]
    off = 0.5 * (a - cc) / (a - 2 * b + cc) if (a - 2 * b + cc) != 0 else 0.0
    return (j + 0.5 + off) * dr


@pytest.mark.parametrize("mixed", [False, True])
def test_pulse_travels_at_the_sound_speed(lq, cuda, mixed):
    c = sphere_pulse().with_ids()
    sim = lq.Simulation(c.par, *c.arrays(), mixed=mixed)
    dt = float(c.par.dt)
    sim.step(40)
    r1 = front_radius(c, sim.download())
    sim.step(60)
    cs = math.sqrt(c.meta["K"] / float(c.par.rho0))
    travel = 60 * dt * cs
    r2 = front_radius(c, sim.download(), r1 + 0.5 * travel, r1 + 1.5 * travel)
    speed = (r2 - r1) / (60 * dt)
    print("front speed", speed, "sqrt(K/rho)", cs, "front at", r1 / c.meta["dr"], r2 / c.meta["dr"], "dr")
    assert r2 < 0.45 * c.meta["n"] * c.meta["dr"]       # still inside the cube
    assert abs(speed / cs - 1.0) < 0.05, (speed, cs)
    assert not sim.health().any()
