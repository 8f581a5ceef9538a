"""The `loquat` command-line driver (counterpart of the reference's
executable, src/loquat.cu:216-476): reads <project>.xml/.dat, writes
output_<n>.xml with <n>.dat or per-object .vtu files at the reference's
output cadence, and its final state equals the library's own run."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from loquat_b200 import cases

pytestmark = pytest.mark.gpu
APP = Path(__file__).resolve().parents[1] / "loquat_b200" / "bin" / "loquat"


def project(lq, tmp_path, output_format, nsteps_out=3, every=4):
    c = cases.small_column(velocity_noise=0.02, shepard=5, seed=31)
    par = c.par
    par.output_format = output_format
    par.output_frequency = every * par.dt * 0.999
    par.time_max = nsteps_out * every * par.dt * 0.9999
    proj = tmp_path / "case"
    lq.save_parameters(str(proj) + ".xml", par)
    lq.save_particles(str(proj) + ".dat", *c.arrays())
    return c, proj


def run(proj):
    r = subprocess.run([str(APP), str(proj)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_driver_dat_outputs_and_final_state(lq, cuda, tmp_path):
    if not APP.exists():
        pytest.fail("driver not built: python -m loquat_b200.build")
    c, proj = project(lq, tmp_path, output_format=1)
    out = run(proj)
    assert "Simulation finished" in out and "Average FPS" in out
    d = Path(str(proj))
    xmls = sorted(d.glob("output_*.xml"))
    dats = sorted(d.glob("*.dat"))
    assert len(xmls) == len(dats) >= 3
    # outputs read back as inputs (formats kept, round trip exact)
    last = max(int(p.stem) for p in dats)
    par = lq.load_parameters(d / f"output_{last}.xml")
    assert par.output_number == last and par.np == c.par.np
    arrs = lq.load_particles(d / f"{last}.dat", par.np)
    assert np.all(np.isfinite(arrs[0]))
    # the state saved after step s equals the library's state after s + 1 steps
    import re

    s = [int(m) for m in re.findall(r"Step = (\d+)", out)][-1]
    sim = lq.Simulation(c.par, *c.arrays())
    sim.step(s + 1)
    want = sim.download()
    for k, (a, b) in enumerate(zip(arrs, want)):
        if k == 2:
            a, b = a[:, :2], b[:, :2]      # idep.z/.w are not in the .dat format
        assert np.array_equal(a, b), k
    assert par.time > 0


def test_driver_vtu_outputs(lq, cuda, tmp_path):
    if not APP.exists():
        pytest.fail("driver not built: python -m loquat_b200.build")
    c, proj = project(lq, tmp_path, output_format=2)
    run(proj)
    d = Path(str(proj))
    vtus = sorted(d.glob("*_0.vtu"))
    ids = sorted({int(p.name.split("_")[0]) for p in d.glob("*.vtu")})
    assert ids == [0, 1]                      # boundary object 0, soil object 1
    text = (d / "1_0.vtu").read_text()
    assert f'NumberOfPoints="{c.par.npm}"' in text
    for name in ("Pressure", "Velocity", "Density", "PlasticStrain", "Stress", "Strain", "connectivity"):
        assert f'Name="{name}"' in text


def test_driver_runs_model_3_from_the_parameter_file(lq, cuda, tmp_path):
    """constitutive-model 3 with the vw-* keys: the driver sets the table and
    the initial void ratio, and its final state equals the library's run."""
    if not APP.exists():
        pytest.fail("driver not built: python -m loquat_b200.build")
    c = cases.small_column(model=3, velocity_noise=0.02, shepard=5, seed=33)
    par = c.par
    every = 4
    par.output_format = 1
    par.output_frequency = every * par.dt * 0.999
    par.time_max = 3 * every * par.dt * 0.9999
    row = c.meta["hypoplastic"][1]
    proj = tmp_path / "vw"
    lq.save_parameters(str(proj) + ".xml", par, hypoplastic=(row, 0.70))
    idep = c.idep.copy()
    idep[:, 2] = 0.0                          # the particle file carries no void ratio
    lq.save_particles(str(proj) + ".dat", c.pospres, c.velrhop, idep, c.str_, c.stn)
    out = run(proj)
    d = Path(str(proj))
    last = max(int(p.stem) for p in d.glob("*.dat"))
    got = lq.load_particles(d / f"{last}.dat", par.np)
    assert lq.load_hypoplastic(d / f"output_{last}.xml")[1] == np.float32(0.70)
    import re

    s = [int(m) for m in re.findall(r"Step = (\d+)", out)][-1]
    sim = lq.Simulation(c.par, *c.arrays())
    sim.set_hypoplastic(c.meta["hypoplastic"])
    sim.step(s + 1)
    want = sim.download()
    for k, (a, b) in enumerate(zip(got, want)):
        if k == 2:
            a, b = a[:, :2], b[:, :2]
        assert np.array_equal(a, b), k


def test_driver_with_the_opt_in_extensions(lq, cuda, tmp_path):
    """--density-filter --dynamic-dt: the steps take their length from the
    device, the loop reads the time back, and the last output equals the
    library's run with the same options and the same number of steps."""
    if not APP.exists():
        pytest.fail("driver not built: python -m loquat_b200.build")
    c = cases.small_column(velocity_noise=0.3, shepard=5, seed=35)
    par = c.par
    par.density_shepard_filter = 4
    par.output_format = 1
    par.output_frequency = 5 * par.dt
    par.time_max = 12 * par.dt
    proj = tmp_path / "ext"
    lq.save_parameters(str(proj) + ".xml", par)
    lq.save_particles(str(proj) + ".dat", *c.arrays())
    r = subprocess.run([str(APP), str(proj), "--density-filter", "--dynamic-dt"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    import re

    steps = [int(m) for m in re.findall(r"Step = (\d+)", r.stdout)]
    assert len(steps) >= 2
    d = Path(str(proj))
    last = max(int(p.stem) for p in d.glob("*.dat"))
    got = lq.load_particles(d / f"{last}.dat", par.np)
    t_file = lq.load_parameters(d / f"output_{last}.xml").time
    sim = lq.Simulation(c.par, *c.arrays(), density_filter=True, dynamic_dt=True)
    sim.step(steps[-1] + 1)
    want = sim.download()
    for k, (a, b) in enumerate(zip(got, want)):
        if k == 2:
            a, b = a[:, :2], b[:, :2]
        assert np.array_equal(a, b), k
    assert t_file == np.float32(sim.clock()[1])
    assert sim.clock()[1] >= par.time_max * (1 - 1e-6)
