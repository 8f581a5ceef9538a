"""Seeded synthetic cases in LOQUAT's input conventions.

The reference ships one example whose particle file is absent, so every input
is generated here: soil on a jittered cubic lattice, Adami dummy particles in
layers on the floor (and walls), geostatic K0 stress, boundary particles
stored first (reference src/loquat_io.cu:204-237 reads them in file order and
the kernels index material particles from npb).  Coordinates start at 0
because the reference grid hashes raw coordinates (src/adami_boundary.cu:80-82).

Parameter conventions pinned by the reference's example
(examples/sand_collapse_plane.xml:12-28): cs = sqrt(K / rho0), dt = cfl h / cs,
k_phi = 6 sin(phi) / (sqrt(3) (3 + sin(phi))).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .params import Parameters, dp_cone, elastic_moduli


@dataclass
class Case:
    name: str
    par: Parameters
    pospres: np.ndarray   # (np, 4) x, y, z, pressure
    velrhop: np.ndarray   # (np, 4) vx, vy, vz, density
    idep: np.ndarray      # (np, 4) object id, plastic strain, void ratio (model 3), free
    str_: np.ndarray      # (np, 6) stress, tension positive
    stn: np.ndarray       # (np, 6) strain
    meta: dict = field(default_factory=dict)

    @property
    def np_(self) -> int:
        return self.pospres.shape[0]

    def arrays(self):
        return self.pospres, self.velrhop, self.idep, self.str_, self.stn

    def with_ids(self) -> "Case":
        """Copy whose idep.w holds each particle's original index (exact in
        float below 2**24), so particles can be matched after re-sorting;
        no kernel reads idep.w (idep.z is the void ratio of model 3)."""
        idep = self.idep.copy()
        n = idep.shape[0]
        if n >= 1 << 24:
            raise ValueError("with_ids: particle indices from 2**24 on are not exact in idep.w")
        idep[:, 3] = np.arange(n, dtype=np.float64).astype(np.float32)
        return Case(self.name, self.par.copy(), self.pospres.copy(), self.velrhop.copy(), idep,
                    self.str_.copy(), self.stn.copy(), dict(self.meta))


def _lattice(nx, ny, nz, dr, origin):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pts = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    return (pts + 0.5) * dr + np.asarray(origin, np.float64)


def _base_parameters(dr, hdr, rho0, domain, E, nu, cfl, model, model_pars, shepard, alpha, gravity):
    p = Parameters()
    p.domain_size_x, p.domain_size_y, p.domain_size_z = map(float, domain)
    p.domain_min_x = p.domain_min_y = p.domain_min_z = 0.0
    p.dr, p.hdr, p.rho0 = dr, hdr, rho0
    K, G = elastic_moduli(E, nu)
    p.cs = math.sqrt(K / rho0)
    p.cfl = cfl
    p.constitutive_model = model
    (p.model_par_1, p.model_par_2, p.model_par_3, p.model_par_4, p.model_par_5) = model_pars(K, G)
    p.density_shepard_filter = 0
    p.stress_shepard_filter = shepard
    p.dynamic_time_step = 0
    p.integration_method = 1
    p.viscosity_type = 1
    p.artificial_viscosity_alpha = alpha
    p.artificial_pressure = 0
    p.artificial_pressure_coefficient = 0.0
    p.acc_x, p.acc_y, p.acc_z = gravity
    p.time = 0.0
    p.output_frequency = 1.0
    p.output_number = 0
    p.output_format = 1
    return p


_initializer = None


def use_parameter_initializer(fn):
    """Derive the constants of every generated case's Parameters with `fn`
    in place of the library's lq_initialize_parameters; both restate
    reference src/loquat.cu:111-139 in the same float arithmetic, so the
    records are bit-identical.  A caller that must not load the CUDA
    library (a CPU-only timing of the same workload) passes its own; None
    restores the library's.  Returns the previous setting."""
    global _initializer
    prev, _initializer = _initializer, fn
    return prev


def _parameter_initializer():
    if _initializer is not None:
        return _initializer
    from . import initialize_parameters

    return initialize_parameters


def assemble(name, par, boundary_xyz, soil_xyz, rng, jitter, rho0, gravity_z, top_z, floor_z, K0,
             object_ids=(0, 1), meta=None) -> Case:
    """Stacks boundary then soil particles, jitters them, sets geostatic stress.

    Soil stress: sigma_zz = rho0 g (top - z) (negative: compression), sigma_xx =
    sigma_yy = K0 sigma_zz, pressure = -tr(sigma)/3.  Boundary stress starts at
    0 (the Adami pass overwrites it)."""
    initialize_parameters = _parameter_initializer()

    nb, ns = boundary_xyz.shape[0], soil_xyz.shape[0]
    xyz = np.concatenate([boundary_xyz, soil_xyz], axis=0)
    if jitter > 0:
        xyz = xyz + rng.uniform(-jitter, jitter, size=xyz.shape)
    n = nb + ns
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = xyz.astype(np.float32)
    vel = np.zeros((n, 4), np.float32)
    vel[:, 3] = rho0
    idep = np.zeros((n, 4), np.float32)
    idep[:nb, 0] = object_ids[0]
    idep[nb:, 0] = object_ids[1]
    s = np.zeros((n, 6), np.float32)
    z = pos[nb:, 2].astype(np.float64)
    top = top_z(pos[nb:, :3].astype(np.float64)) if callable(top_z) else top_z
    szz = rho0 * gravity_z * (top - z)  # gravity_z < 0 -> compression below the top
    szz = np.minimum(szz, 0.0)
    s[nb:, 2] = szz
    s[nb:, 0] = K0 * szz
    s[nb:, 1] = K0 * szz
    pos[nb:, 3] = (-(s[nb:, 0].astype(np.float64) + s[nb:, 1] + s[nb:, 2]) / 3.0).astype(np.float32)
    stn = np.zeros((n, 6), np.float32)
    par.np, par.npb, par.npm = n, nb, ns
    initialize_parameters(par)
    par.dt = par.cfl * par.h / par.cs
    m = dict(meta or {})
    m.update(np=n, npb=nb, npm=ns)
    return Case(name, par, pos, vel, idep, s, stn, m)


def column_collapse(dr=0.002, length=0.2, height=0.1, thickness=0.02, runout=0.6, layers=3, hdr=1.2,
                    rho0=2650.0, E=0.84e6, nu=0.3, phi=19.8, psi=0.0, cohesion=0.0, cfl=0.1, alpha=0.25,
                    shepard=30, seed=1, jitter_frac=0.01, side_walls=True, name="column_collapse") -> Case:
    """Granular column collapse: the 3D slab of the reference's
    sand_collapse_plane shape class.  Soil block length x height x thickness
    against a back wall at x = 0, on a floor, between two side walls (y),
    all of `layers` Adami layers; the floor and side walls run `runout` in x."""
    b = layers * dr
    nsx, nsy, nsz = round(length / dr), round(thickness / dr), round(height / dr)
    nrx = round(runout / dr)
    nwy = nsy + 2 * layers if side_walls else nsy
    wall_top = height + 0.1 * height
    nwz = round(wall_top / dr)
    y0 = b if side_walls else 0.0
    soil = _lattice(nsx, nsy, nsz, dr, (b, y0, b))
    parts = [_lattice(nrx + layers, nwy, layers, dr, (0.0, 0.0, 0.0))]          # floor
    parts.append(_lattice(layers, nsy, nwz, dr, (0.0, y0, b)))                   # back wall
    if side_walls:
        parts.append(_lattice(nrx + layers, layers, nwz, dr, (0.0, 0.0, b)))     # y = 0 side
        parts.append(_lattice(nrx + layers, layers, nwz, dr, (0.0, y0 + nsy * dr, b)))
    bnd = np.concatenate(parts, axis=0)
    domain = ((nrx + layers) * dr, nwy * dr, b + 1.5 * height)
    kphi, kpsi, kc = dp_cone(phi, psi, cohesion)
    par = _base_parameters(dr, hdr, rho0, domain, E, nu, cfl, 1, lambda K, G: (K, G, kphi, kpsi, kc), shepard,
                           alpha, (0.0, 0.0, -9.81))
    K0 = 1.0 - math.sin(math.radians(phi))
    rng = np.random.default_rng(seed)
    return assemble(name, par, bnd, soil, rng, jitter_frac * dr, rho0, -9.81, b + height, b, K0,
                    meta=dict(config="column", dr=dr, soil_lattice=(nsx, nsy, nsz), phi=phi))


def cylinder_collapse(dr=0.002949, radius=0.2, height=0.4, floor_radius_factor=2.5, layers=3, hdr=1.3,
                      rho0=2000.0, E=5.0e6, nu=0.3, phi=30.0, psi=0.0, cohesion=0.0, cfl=0.1, alpha=0.25,
                      shepard=30, seed=1, jitter_frac=0.01, name="cylinder_collapse") -> Case:
    """Axisymmetric cylinder collapse on a square Adami floor of half-width
    floor_radius_factor * radius.  At dr = 2.949 mm the cylinder holds about
    1.96 M soil particles (at 4 mm it would hold 0.79 M)."""
    b = layers * dr
    half = floor_radius_factor * radius
    nf = round(2 * half / dr)
    side = nf * dr
    cx = cy = side / 2.0
    nr = int(math.ceil(radius / dr)) + 1
    nz = round(height / dr)
    ii = np.arange(-nr, nr)
    gx, gy = np.meshgrid(ii, ii, indexing="ij")
    px = (gx.ravel() + 0.5) * dr
    py = (gy.ravel() + 0.5) * dr
    inside = px * px + py * py <= radius * radius
    px, py = px[inside] + cx, py[inside] + cy
    zs = (np.arange(nz) + 0.5) * dr + b
    soil = np.stack([np.repeat(px[None, :], nz, 0).ravel(), np.repeat(py[None, :], nz, 0).ravel(),
                     np.repeat(zs[:, None], px.size, 1).ravel()], axis=1)
    bnd = _lattice(nf, nf, layers, dr, (0.0, 0.0, 0.0))
    domain = (side, side, b + 1.15 * height)
    kphi, kpsi, kc = dp_cone(phi, psi, cohesion)
    par = _base_parameters(dr, hdr, rho0, domain, E, nu, cfl, 1, lambda K, G: (K, G, kphi, kpsi, kc), shepard,
                           alpha, (0.0, 0.0, -9.81))
    K0 = 1.0 - math.sin(math.radians(phi))
    rng = np.random.default_rng(seed)
    return assemble(name, par, bnd, soil, rng, jitter_frac * dr, rho0, -9.81, b + height, b, K0,
                    meta=dict(config="cylinder", dr=dr, radius=radius, height=height, phi=phi))


def small_column(nsx=16, nsy=6, nsz=12, dr=0.002, layers=3, hdr=1.2, model=1, seed=3, jitter_frac=0.01,
                 velocity_noise=0.0, shepard=5, hypo_pars=(-300.0, -500.0, -300.0, -200.0, 0.0),
                 E=0.84e6, nu=0.3, phi=19.8, cohesion=0.0, rho0=2650.0, alpha=0.25, front_wall=False,
                 e0=0.70, vw=None, name="small_column") -> Case:
    """A few-thousand-particle column for parity tests.  `velocity_noise`
    (m/s) adds a seeded random velocity to the soil so every term of the
    interaction pass is exercised from the first step.  model 2 uses the
    four-parameter hypoplastic law with `hypo_pars` = (c1, c2, c3, c4, cohesion);
    in that form the ||D|| term only dissipates for c4 < 0 (T is compressive),
    and a positive c4 makes the explicit update blow up within tens of steps.
    `front_wall` closes the box at the soil's free face (a confined block).
    model 3 (von Wolffersdorff) uses the row `vw` (vw_row() by default),
    initial void ratio e0 in idep.z and density rho0 as given; the row is
    returned in meta["hypoplastic"] for Simulation.set_hypoplastic."""
    b = layers * dr
    nrx = nsx + (0 if front_wall else 10)
    soil = _lattice(nsx, nsy, nsz, dr, (b, b, b))
    nwy = nsy + 2 * layers
    nwz = nsz + 2
    parts = [
        _lattice(nrx + 2 * layers, nwy, layers, dr, (0.0, 0.0, 0.0)),
        _lattice(layers, nsy, nwz, dr, (0.0, b, b)),
        _lattice(nrx + 2 * layers, layers, nwz, dr, (0.0, 0.0, b)),
        _lattice(nrx + 2 * layers, layers, nwz, dr, (0.0, b + nsy * dr, b)),
    ]
    if front_wall:
        parts.append(_lattice(layers, nsy, nwz, dr, (b + nsx * dr, b, b)))
    bnd = np.concatenate(parts)
    domain = ((nrx + 2 * layers) * dr, nwy * dr, b + 1.6 * nsz * dr)
    if model == 1:
        kphi, kpsi, kc = dp_cone(phi, 0.0, cohesion)
        pars = lambda K, G: (K, G, kphi, kpsi, kc)  # noqa: E731
    elif model == 2:
        pars = lambda K, G: tuple(hypo_pars)  # noqa: E731
    else:
        pars = lambda K, G: (0.0, 0.0, 0.0, 0.0, 0.0)  # noqa: E731
    par = _base_parameters(dr, hdr, rho0, domain, E, nu, 0.1, model, pars, shepard, alpha, (0.0, 0.0, -9.81))
    K0 = 1.0 - math.sin(math.radians(phi))
    rng = np.random.default_rng(seed)
    c = assemble(name, par, bnd, soil, rng, jitter_frac * dr, rho0, -9.81, b + nsz * dr, b, K0,
                 meta=dict(config="small", dr=dr, top=b + nsz * dr))
    if model == 3:
        c.idep[c.par.npb:, 2] = e0
        row = vw_row() if vw is None else np.asarray(vw, np.float32)
        c.meta["hypoplastic"] = np.stack([row, row])
    if velocity_noise > 0:
        nb = c.par.npb
        c.velrhop[nb:, :3] = rng.uniform(-velocity_noise, velocity_noise, size=(c.par.npm, 3)).astype(np.float32)
    return c


# ------------------------------------------------ von Wolffersdorff sand
# Sand of the slope and inclined-plane workloads: phi_c (deg), h_s (Pa), n,
# e_d0, e_c0, e_i0, alpha, beta.
VW_SAND = (30.0, 2.6e9, 0.27, 0.61, 0.98, 1.10, 0.18, 1.0)


def vw_row(sand=VW_SAND, tol=1e-4, max_substeps=64) -> np.ndarray:
    """One row of the model-3 table (Simulation.set_hypoplastic)."""
    return np.array(list(sand) + [tol, max_substeps], np.float32)


def vw_modulus(p, e, sand=VW_SAND) -> float:
    """Isotropic tangent stiffness of the von Wolffersdorff model at mean
    pressure p (Pa, compression positive) and void ratio e: for T = -p I and
    D = eps I the rate is 3 fb fe (1 + a^2/3) eps I, plus the |D| term for
    loading; returns fb fe (1 + a^2 + fd a), an upper bound of the
    constrained modulus used to size the sound speed."""
    phic, hs, n, ed0, ec0, ei0, alpha, beta = sand
    sp = math.sin(math.radians(phic))
    a = math.sqrt(3.0) * (3.0 - sp) / (2.0 * math.sqrt(2.0) * sp)
    pr = 3.0 * max(p, 1.0) / hs
    x = math.exp(-pr ** n)
    ei, ec, ed = ei0 * x, ec0 * x, ed0 * x
    den = 3.0 + a * a - a * math.sqrt(3.0) * ((ei0 - ed0) / (ec0 - ed0)) ** alpha
    fb = (hs / n) * (ei0 / ec0) ** beta * (1.0 + ei) / ei * pr ** (1.0 - n) / den
    fe = (ec / e) ** beta
    fd = max((e - ed) / (ec - ed), 0.0) ** alpha
    return fb * fe * (1.0 + a * a + fd * a)


def _vw_parameters(dr, hdr, rho, domain, p_max, e0, sand, cfl, shepard, alpha, gravity):
    """Parameters of a model-3 case: cs from the tangent stiffness at twice
    the largest initial mean pressure (the explicit step must resolve the
    stiffest soil, at the base)."""
    M = vw_modulus(2.0 * p_max, e0, sand)
    E = 3.0 * M * (1.0 - 2.0 * 0.3)   # K = M at nu = 0.3 in elastic_moduli
    return _base_parameters(dr, hdr, rho, domain, E, 0.3, cfl, 3, lambda K, G: (0.0,) * 5, shepard, alpha,
                            gravity)


def slope_failure(dr=0.005, length=2.0, height=0.6, width=0.35, angle=45.0, runout=1.0, layers=3, hdr=1.2,
                  e0=0.70, rho_s=2650.0, sand=VW_SAND, tol=1e-4, max_substeps=64, cfl=0.1, alpha=0.25,
                  shepard=30, seed=1, jitter_frac=0.01, name="slope_failure") -> Case:
    """Sand slope failure with the von Wolffersdorff model: a trapezoid of
    soil `length` long and `height` high whose free face drops at `angle`
    towards +x, `width` thick between two side walls, against a back wall at
    x = 0, on a floor that runs `runout` beyond the toe.  Density
    rho_s / (1 + e0); geostatic stress from the local surface with
    K0 = 1 - sin(phi_c); void ratio e0 in idep.z.  At the defaults (2.0 x 0.6
    x 0.35 m at dr = 5 mm) the soil holds 2,852,360 particles (642,780 in
    the walls and floor): the stated geometry at that spacing, not a 4.2 M
    count."""
    b = layers * dr
    rho = rho_s / (1.0 + e0)
    nsx, nsy, nsz = round(length / dr), round(width / dr), round(height / dr)
    t = math.tan(math.radians(angle))
    block = _lattice(nsx, nsy, nsz, dr, (0.0, 0.0, 0.0))
    top = np.minimum(height, (length - block[:, 0]) * t)
    soil = block[block[:, 2] < top] + np.array([b, b, b])
    nrx = nsx + round(runout / dr)
    nwy = nsy + 2 * layers
    nwz = round(1.1 * height / dr)
    bnd = np.concatenate([
        _lattice(nrx + layers, nwy, layers, dr, (0.0, 0.0, 0.0)),               # floor
        _lattice(layers, nsy, nwz, dr, (0.0, b, b)),                            # back wall
        _lattice(nrx + layers, layers, nwz, dr, (0.0, 0.0, b)),                 # side walls
        _lattice(nrx + layers, layers, nwz, dr, (0.0, b + nsy * dr, b)),
    ])
    domain = ((nrx + layers) * dr, nwy * dr, b + 1.5 * height)
    p_max = rho * 9.81 * height * (1.0 + 2.0 * (1.0 - math.sin(math.radians(sand[0])))) / 3.0
    par = _vw_parameters(dr, hdr, rho, domain, p_max, e0, sand, cfl, shepard, alpha, (0.0, 0.0, -9.81))
    K0 = 1.0 - math.sin(math.radians(sand[0]))
    surface = lambda x: b + np.minimum(height, (length - (x[:, 0] - b)) * t)  # noqa: E731
    c = assemble(name, par, bnd, soil, np.random.default_rng(seed), jitter_frac * dr, rho, -9.81, surface, b, K0,
                 meta=dict(config="slope", dr=dr, length=length, height=height, angle=angle, e0=e0))
    c.idep[c.par.npb:, 2] = e0
    row = vw_row(sand, tol, max_substeps)
    c.meta["hypoplastic"] = np.stack([row, row])
    return c


def inclined_block(dr=0.0025, length=1.0, width=1.0, height=0.25, angle=30.0, runout=1.0, upslope=0.1, layers=3,
                   hdr=1.2, e0=0.65, rho_s=2650.0, sand=VW_SAND, tol=1e-4, max_substeps=64, cfl=0.1, alpha=0.25,
                   shepard=30, seed=1, jitter_frac=0.01, name="inclined_block") -> Case:
    """Soil block on an inclined plane with the von Wolffersdorff model.  The
    frame is the plane's: z is normal to it and gravity is rotated,
    g = 9.81 (sin angle, 0, -cos angle), so the block runs out towards +x.
    The block (length x width x height) starts `upslope` from the plane's
    upper end, between two side walls, with `runout` of plane below it.
    Initial stress is the infinite-slope state: sigma_zz = rho g_z (top - z),
    sigma_xx = sigma_yy = K0 sigma_zz, sigma_xz = rho g_x (top - z).  At
    dr = 2.5 mm the block holds 16.0 M particles (1.0 x 1.0 x 0.25 m at
    4 mm would hold 3.9 M)."""
    b = layers * dr
    rho = rho_s / (1.0 + e0)
    th = math.radians(angle)
    gx, gz = 9.81 * math.sin(th), -9.81 * math.cos(th)
    nsx, nsy, nsz = round(length / dr), round(width / dr), round(height / dr)
    nup = round(upslope / dr)
    nrx = nup + nsx + round(runout / dr)
    nwy = nsy + 2 * layers
    nwz = round(1.2 * height / dr)
    soil = _lattice(nsx, nsy, nsz, dr, (nup * dr, b, b))
    bnd = np.concatenate([
        _lattice(nrx, nwy, layers, dr, (0.0, 0.0, 0.0)),                        # plane
        _lattice(nrx, layers, nwz, dr, (0.0, 0.0, b)),                          # side walls
        _lattice(nrx, layers, nwz, dr, (0.0, b + nsy * dr, b)),
    ])
    domain = (nrx * dr, nwy * dr, b + 2.0 * height)
    K0 = 1.0 - math.sin(math.radians(sand[0]))
    p_max = rho * abs(gz) * height * (1.0 + 2.0 * K0) / 3.0
    par = _vw_parameters(dr, hdr, rho, domain, p_max, e0, sand, cfl, shepard, alpha, (gx, 0.0, gz))
    c = assemble(name, par, bnd, soil, np.random.default_rng(seed), jitter_frac * dr, rho, gz, b + height, b, K0,
                 meta=dict(config="inclined", dr=dr, angle=angle, e0=e0))
    nb = c.par.npb
    depth = np.maximum(b + height - c.pospres[nb:, 2].astype(np.float64), 0.0)
    c.str_[nb:, 4] = (rho * gx * depth).astype(np.float32)
    c.idep[nb:, 2] = e0
    row = vw_row(sand, tol, max_substeps)
    c.meta["hypoplastic"] = np.stack([row, row])
    return c


def config_case(index: int, **kw) -> Case:
    """Case of one of the benchmark configurations (0-based):
    0 column collapse 50k, 1 cylinder collapse ~1.96M (plain FP32 form),
    2 von Wolffersdorff slope failure 2.85M, 4 von Wolffersdorff block on
    a 30 degree plane 16.0M (3 is the ensemble(), a set of cases)."""
    if index == 0:
        return column_collapse(**kw)
    if index == 1:
        return cylinder_collapse(**kw)
    if index == 2:
        return slope_failure(**kw)
    if index == 4:
        return inclined_block(**kw)
    raise ValueError(f"configuration {index} has no single-case generator")


def _column_parts(nsx, nsy, nsz, dr, layers, runout_cells, wall_top_cells):
    """Soil block and Adami walls (floor, back wall, two side walls) of one
    column-collapse scenario in local coordinates starting at 0."""
    b = layers * dr
    nwy = nsy + 2 * layers
    nrx = nsx + runout_cells
    soil = _lattice(nsx, nsy, nsz, dr, (b, b, b))
    bnd = np.concatenate([
        _lattice(nrx + layers, nwy, layers, dr, (0.0, 0.0, 0.0)),
        _lattice(layers, nsy, wall_top_cells, dr, (0.0, b, b)),
        _lattice(nrx + layers, layers, wall_top_cells, dr, (0.0, 0.0, b)),
        _lattice(nrx + layers, layers, wall_top_cells, dr, (0.0, b + nsy * dr, b)),
    ])
    extent = ((nrx + layers) * dr, nwy * dr, b + nsz * dr)
    return soil, bnd, extent


def ensemble(n=256, seed=4, dr=0.002, hdr=1.2, count_range=(5.0e3, 2.0e5), aspect_range=(0.5, 4.0),
             phi_range=(20.0, 40.0), cohesion_range=(0.0, 5.0e3), thickness_layers=10, layers=3,
             runout_frac=0.5, rho0=2650.0, E=0.84e6, nu=0.3, cfl=0.1, alpha=0.25, shepard=30, jitter_frac=0.01):
    """An ensemble of independent Drucker-Prager column collapses.

    Scenario k has a soil count drawn log-uniform on count_range, aspect
    ratio H/L uniform on aspect_range, friction angle uniform on phi_range
    (degrees) and cohesion uniform on cohesion_range (Pa); all share dr, h,
    density and elasticity, hence one time step.  Returns (combined, parts).
    `parts` are the scenarios as standalone cases.  `combined` holds all of
    them in one particle set for a single simulation: every particle of
    scenario k (boundary and soil) has object id k + 1 and keeps its local
    coordinates; meta["frames"] gives each object its own block of grid
    rows (with an empty row between blocks, so no pair crosses scenarios)
    and meta["materials"] its (K, G, k_phi, k_psi, k_c) -- for
    Simulation.set_frames and Simulation.set_materials."""
    rng = np.random.default_rng(seed)
    K, G = elastic_moduli(E, nu)
    lo, hi = np.log(count_range[0]), np.log(count_range[1])
    parts = []
    for k in range(n):
        count = float(np.exp(rng.uniform(lo, hi)))
        a = float(rng.uniform(*aspect_range))
        phi = float(rng.uniform(*phi_range))
        coh = float(rng.uniform(*cohesion_range))
        nsy = thickness_layers
        nsx = max(2, int(round(np.sqrt(count / (nsy * a)))))
        nsz = max(2, int(round(a * nsx)))
        runout = max(2, int(round(runout_frac * nsx)))
        soil, bnd, extent = _column_parts(nsx, nsy, nsz, dr, layers, runout, int(round(1.1 * nsz)))
        kphi, kpsi, kc = dp_cone(phi, 0.0, coh)
        par_k = _base_parameters(dr, hdr, rho0, (extent[0], extent[1], 1.5 * extent[2]), E, nu, cfl, 1,
                                 lambda K_, G_, a=(K, G, kphi, kpsi, kc): a, shepard, alpha, (0.0, 0.0, -9.81))
        b = layers * dr
        part = assemble(f"ensemble_{k}", par_k, bnd, soil, np.random.default_rng(int(rng.integers(1 << 30))),
                        jitter_frac * dr, rho0, -9.81, b + nsz * dr, b, 1.0 - np.sin(np.radians(phi)),
                        object_ids=(k + 1, k + 1),
                        meta=dict(config="ensemble", scenario=k, phi=phi, cohesion=coh, aspect=nsz / nsx,
                                  extent=extent, material=(K, G, kphi, kpsi, kc)))
        parts.append(part)
    return combine(parts), parts


def combine(parts):
    """One particle set holding the given ensemble scenarios (cases from
    ensemble(), all with the same dr, h and time step): boundary particles
    of every scenario first, then soil; each scenario keeps its local
    coordinates and object id.  meta["frames"] gives object k its own block
    of grid rows with an empty row between blocks, meta["materials"] its
    constitutive parameters, meta["slices"] each part's (boundary, soil)
    slot ranges."""
    if not parts:
        raise ValueError("no scenarios")
    p0 = parts[0].par
    dr, hdr = float(p0.dr), float(p0.hdr)
    n = max(int(p.idep[0, 0]) for p in parts)
    two_h = 2.0 * hdr * dr
    table = np.zeros((n + 1, 5), np.float32)
    frames = np.zeros((n + 1, 2), np.int32)
    row = 0
    for p in parts:
        k = int(p.idep[0, 0])
        table[k] = p.meta["material"]
        rows = int(np.floor(p.meta["extent"][1] / two_h)) + 2
        frames[k] = (row, rows)
        row += rows + 1
    xsize = max(p.meta["extent"][0] for p in parts)
    zsize = max(p.meta["extent"][2] for p in parts)
    K, G = float(p0.model_par_1), float(p0.model_par_2)
    E = 9.0 * K * G / (3.0 * K + G)
    nu = (3.0 * K - 2.0 * G) / (2.0 * (3.0 * K + G))
    par = _base_parameters(dr, hdr, float(p0.rho0), (xsize, row * two_h, 1.5 * zsize), E, nu, float(p0.cfl), 1,
                           lambda K_, G_: tuple(table[int(parts[0].idep[0, 0])]), int(p0.stress_shepard_filter),
                           float(p0.artificial_viscosity_alpha), (float(p0.acc_x), float(p0.acc_y), float(p0.acc_z)))
    par.cs = p0.cs
    nb = sum(p.par.npb for p in parts)
    ns = sum(p.par.npm for p in parts)
    arrays = [np.zeros((nb + ns, 4), np.float32), np.zeros((nb + ns, 4), np.float32),
              np.zeros((nb + ns, 4), np.float32), np.zeros((nb + ns, 6), np.float32),
              np.zeros((nb + ns, 6), np.float32)]
    ob, om = 0, nb
    slices = []
    for p in parts:
        pb, pm = p.par.npb, p.par.npm
        for a_out, a_in in zip(arrays, p.arrays()):
            a_out[ob:ob + pb] = a_in[:pb]
            a_out[om:om + pm] = a_in[pb:]
        slices.append(((ob, ob + pb), (om, om + pm)))
        ob += pb
        om += pm
    initialize_parameters = _parameter_initializer()

    par.np, par.npb, par.npm = nb + ns, nb, ns
    initialize_parameters(par)
    par.dt = par.cfl * par.h / par.cs
    assert par.cell_num_y >= row
    assert abs(par.dt - p0.dt) <= 1e-12 * p0.dt, "scenarios must share one time step"
    return Case("ensemble", par, *arrays,
                meta=dict(config="ensemble", n=len(parts), materials=table, frames=frames, slices=slices,
                          np=nb + ns, npb=nb, npm=ns))
