"""C ABI and drop-in surface: library loads, every declared symbol is
exported, the reference-shaped headers link, and the host-only calls
(parameter derivation, XML/.dat formats, error reporting) behave like the
reference's.  No test here needs a GPU."""
from __future__ import annotations

import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "loquat_b200.h"


def declared_c_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lq_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol(lq):
    names = declared_c_functions()
    assert len(names) >= 30
    L = lq.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(lq.exported_symbols())
    out = subprocess.run(["nm", "-D", "--defined-only", str(lq.lib_path())], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    for n in names:
        assert n in exported, n


def test_drop_in_cxx_symbols_exported(lq):
    out = subprocess.run(["nm", "-DC", "--defined-only", str(lq.lib_path())], capture_output=True, text=True,
                         check=True).stdout
    for sig in [
        "LoquatGrid::LoquatGrid()",
        "LoquatGrid::~LoquatGrid()",
        "LoquatGrid::GridConfig(Parameters*)",
        "LoquatGrid::ResizeArrayLength(int, int)",
        "LoquatGrid::NeighborSearch(Parameters*, Parameters*, float4*, float4*)",
        "LoquatGrid::SortArrayFloat4(int, float4*, float4*)",
        "LoquatGrid::SortArrayTensor2d(int, tensor2d*, tensor2d*)",
        "ParticleInteraction(Parameters*, Parameters*, float4*, float4*, float4*, tensor2d*, tensor2d*, float4*, "
        "float4*, tensor2d*, int const*, int const*)",
        "AdamiBoundary(Parameters*, Parameters*, float4*, float4*, tensor2d*, int const*, int const*)",
        "StressRegularization(Parameters*, Parameters*, float4*, float4*, tensor2d*, tensor2d*, int const*, "
        "int const*)",
        "Predictor(Parameters*, Parameters*, float4*, float4*, float4*, tensor2d*, tensor2d*, float4*, float4*, "
        "float4*, tensor2d*, tensor2d*, float4*, float4*, tensor2d*)",
        "Corrector(Parameters*, Parameters*, float4*, float4*, float4*, tensor2d*, tensor2d*, float4*, float4*, "
        "float4*, tensor2d*, tensor2d*, float4*, float4*, tensor2d*)",
    ]:
        assert sig in out, sig


def test_reference_shaped_caller_links(lq, tmp_path):
    gxx = shutil.which("g++") or "g++"
    exe = tmp_path / "abi_link_check"
    cmd = [gxx, "-std=c++17", f"-I{ROOT / 'include'}", "-I/usr/local/cuda/include",
           str(ROOT / "tests" / "abi_link_check.cpp"), f"-L{lq.lib_path().parent}", "-llqb200",
           f"-Wl,-rpath,{lq.lib_path().parent}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split()[1] == "208"


def test_parameters_layout(lq):
    assert lq.lib().lq_parameters_size() == 208 == ctypes.sizeof(lq.Parameters)
    assert lq.lib().lq_abi_version() == 1
    # field offsets follow the reference order: np first, output_format last
    assert lq.Parameters.np.offset == 0
    assert lq.Parameters.output_format.offset == 204
    assert lq.Parameters.kernel_dr.offset == 200


def test_initialize_parameters_matches_reference_arithmetic(lq, orc):
    """lq_initialize_parameters vs the oracle's restatement of
    reference src/loquat.cu:111-139 on the reference example's numbers."""
    p = lq.Parameters()
    p.dr, p.hdr, p.rho0 = 0.05, 1.5, 1850.0
    p.domain_size_x, p.domain_size_y, p.domain_size_z = 6.3, 2.3, 1.3
    p.artificial_pressure = 1
    q = p.copy()
    lq.initialize_parameters(p)
    orc.initialize_parameters(q)
    assert p.to_bytes() == q.to_bytes()
    assert abs(p.h - 0.075) < 1e-7
    assert p.cell_num_x == int(0.5 / 0.075 * 6.3) + 1
    assert p.ncell == 2 * p.ncell_one_layer + 1 and p.ncell_delete == p.ncell - 1
    # Wendland C2: W(0) = 16 C / 2 = 8 C
    assert abs(p.kernel_zero - 8.0 * p.kernel_normalization_par) < 1e-3 * p.kernel_zero


def test_example_parameter_conventions(lq):
    """The reference example pins cs = sqrt(K / rho0), dt = cfl h / cs and the
    Drucker-Prager cone k_phi(30 deg) = 0.494872
    (examples/sand_collapse_plane.xml:12-28)."""
    K, G = lq.elastic_moduli(6.0e6, 0.3)
    assert abs(K - 5.0e6) < 1 and abs(G - 2.30769e6) < 10
    assert abs(np.sqrt(K / 1850.0) - 51.9875) < 1e-3
    kphi, kpsi, kc = lq.dp_cone(30.0)
    assert abs(kphi - 0.494872) < 1e-6 and kpsi == 0.0 and kc == 0.0
    p = lq.Parameters()
    p.dr, p.hdr, p.cfl, p.cs = 0.05, 1.5, 0.2, 51.9875
    p.domain_size_x = p.domain_size_y = p.domain_size_z = 1.0
    lq.initialize_parameters(p)
    lq.update_time_step(p)
    assert abs(p.dt - 0.000288531) < 1e-9


def _example_xml():
    return """<?xml version="1.0" encoding="utf-8" ?>
<parameters>
  <number-of-particles type="int">3</number-of-particles>
  <number-of-boundary-particles type="int">1</number-of-boundary-particles>
  <number-of-material-particles type="int">2</number-of-material-particles>
  <domain-size-x type="float">6.3</domain-size-x>
  <domain-size-y type="float">2.3</domain-size-y>
  <domain-size-z type="float">1.3</domain-size-z>
  <domain-min-x type="float">0</domain-min-x>
  <domain-min-y type="float">0</domain-min-y>
  <domain-min-z type="float">0</domain-min-z>
  <particle-size type="float">0.05</particle-size>
  <h-over-dr type="float">1.5</h-over-dr>
  <reference-density type="float">1850</reference-density>
  <speed-of-sound type="float">51.9875</speed-of-sound>
  <cfl-number type="float">0.2</cfl-number>
  <constitutive-model type="int">1</constitutive-model>
  <elastic-K type="float">5e+06</elastic-K>
  <elastic-G type="float">2.30769e+06</elastic-G>
  <DP-kphi type="float">0.494872</DP-kphi>
  <DP-kpsi type="float">0</DP-kpsi>
  <DP-kcohesion type="float">0</DP-kcohesion>
  <acceleration-x type="float">0</acceleration-x>
  <acceleration-y type="float">0</acceleration-y>
  <acceleration-z type="float">-9.81</acceleration-z>
  <time-max type="float">4</time-max>
  <time type="float">0</time>
  <time-step type="float">0.000288531</time-step>
  <output-frequency type="float">0.2</output-frequency>
  <output-number type="int">0</output-number>
  <density-shepard-filter type="int">0</density-shepard-filter>
  <stress-shepard-filter type="int">0</stress-shepard-filter>
  <dynamic-time-step type="int">1</dynamic-time-step>
  <integration-method type="int">1</integration-method>
  <viscosity-type type="int">1</viscosity-type>
  <artificial-viscosity-alpha type="float">0.25</artificial-viscosity-alpha>
  <artificial-pressure type="int">0</artificial-pressure>
  <output-format type="int">2</output-format>
</parameters>
"""


def test_xml_reader_on_reference_example_shape(lq, tmp_path):
    f = tmp_path / "case.xml"
    f.write_text(_example_xml())
    p = lq.load_parameters(f)
    assert (p.np, p.npb, p.npm) == (3, 1, 2)
    assert p.model_par_1 == np.float32(5e6) and p.model_par_3 == np.float32(0.494872)
    assert p.acc_z == np.float32(-9.81) and p.output_format == 2 and p.viscosity_type == 1
    assert p.artificial_viscosity_alpha == np.float32(0.25)
    # round trip through the writer (which writes elastic-G, the key the reader expects)
    g = tmp_path / "out.xml"
    lq.save_parameters(g, p)
    assert "elastic-G" in g.read_text() and "poisson-G" not in g.read_text()
    q = lq.load_parameters(g)
    assert q.to_bytes() == p.to_bytes()


def test_xml_reader_errors(lq, tmp_path):
    f = tmp_path / "bad.xml"
    f.write_text(_example_xml().replace('<cfl-number type="float">0.2</cfl-number>\n', ""))
    with pytest.raises(lq.LoquatError) as e:
        lq.load_parameters(f)
    assert e.value.status == lq.LQ_ERR_NOTFOUND and "cfl-number" in str(e.value)
    f.write_text(_example_xml().replace('<cfl-number type="float">', '<cfl-number type="double">'))
    with pytest.raises(lq.LoquatError) as e:
        lq.load_parameters(f)
    assert "wrong data type" in str(e.value)
    f.write_text(_example_xml().replace('type="int">3</number-of-particles>', 'type="int">4</number-of-particles>'))
    with pytest.raises(lq.LoquatError) as e:
        lq.load_parameters(f)
    assert "wrong number of particles" in str(e.value)
    with pytest.raises(lq.LoquatError):
        lq.load_parameters(tmp_path / "missing.xml")
    f.write_text(_example_xml().replace('<DP-kpsi type="float">0</DP-kpsi>', '<DP-kpsi type="int">0</DP-kpsi>'))
    with pytest.raises(lq.LoquatError) as e:
        lq.load_parameters(f)
    assert "DP-kpsi" in str(e.value)


def test_xml_model_3_extension_keys_round_trip(lq, tmp_path):
    from loquat_b200 import cases

    c = cases.small_column(model=3)
    row = cases.vw_row(tol=2e-4, max_substeps=48)
    f = tmp_path / "vw.xml"
    lq.save_parameters(f, c.par, hypoplastic=(row, 0.70))
    text = f.read_text()
    assert '<constitutive-model type="int">3</constitutive-model>' in text
    assert '<vw-max-substeps type="int">48</vw-max-substeps>' in text
    q = lq.load_parameters(f)
    assert q.constitutive_model == 3 and q.np == c.par.np
    f2 = tmp_path / "vw2.xml"
    lq.save_parameters(f2, q, hypoplastic=lq.load_hypoplastic(f))
    assert f2.read_text() == text
    got, e0 = lq.load_hypoplastic(f)
    assert np.array_equal(got, row) and e0 == np.float32(0.70)
    # a model-3 file without the keys names the first missing one
    g = tmp_path / "plain.xml"
    lq.save_parameters(g, c.par)
    with pytest.raises(lq.LoquatError) as e:
        lq.load_hypoplastic(g)
    assert e.value.status == lq.LQ_ERR_NOTFOUND and "vw-phi-c" in str(e.value)


def test_dat_round_trip_and_errors(lq, tmp_path):
    rng = np.random.default_rng(0)
    n = 257
    arrs = [rng.standard_normal((n, 4)).astype(np.float32) for _ in range(3)] + \
           [rng.standard_normal((n, 6)).astype(np.float32) for _ in range(2)]
    arrs[2][:, 2:] = 0.0  # idep.z/.w are not part of the format
    f = tmp_path / "p.dat"
    lq.save_particles(f, *arrs)
    lines = f.read_text().splitlines()
    assert len(lines) == n and all(len(l.split()) == 22 for l in lines)
    back = lq.load_particles(f, n)
    for a, b in zip(arrs, back):
        assert np.array_equal(a, b)
    # truncated file
    f.write_text("\n".join(lines[:-1]) + "\n")
    with pytest.raises(lq.LoquatError) as e:
        lq.load_particles(f, n)
    assert "truncated" in str(e.value)
    f.write_text(lines[0].replace(lines[0].split()[3], "abc", 1) + "\n")
    with pytest.raises(lq.LoquatError):
        lq.load_particles(f, 1)


def test_null_arguments_are_rejected_without_a_gpu(lq):
    L = lq.lib()
    assert L.lq_initialize_parameters(None) == lq.LQ_ERR_ARG
    assert L.lq_particle_interaction(*([None] * 13)) == lq.LQ_ERR_ARG
    assert L.lq_sim_step(None, 1) == lq.LQ_ERR_ARG
    assert b"bad argument" in L.lq_last_error()
    assert L.lq_status_string(lq.LQ_ERR_IO) == b"I/O error"


def test_checkpoint_reader_rejects_foreign_and_truncated_files(lq, tmp_path):
    """Checked before any device work, so this runs without a GPU."""
    import ctypes
    import struct

    from loquat_b200 import cases

    def load(path):
        h = ctypes.c_void_p()
        return lq.lib().lq_sim_load_checkpoint(str(path).encode(), 0, ctypes.byref(h)), h

    f = tmp_path / "x.lqck"
    f.write_bytes(b"not a checkpoint at all")
    st, h = load(f)
    assert st == lq.LQ_ERR_IO and "not a LOQUAT-B200 checkpoint" in lq.lib().lq_last_error().decode()
    assert not h.value
    c = cases.small_column(seed=1)
    par = c.par
    head = b"LQB200CK" + struct.pack("<IIqdfiii", 1, 0, 5, 0.5, 0.0, par.np, par.npb, par.npm) + par.to_bytes()
    f.write_bytes(head + b"\0" * 100)                       # arrays cut short
    st, _ = load(f)
    assert st == lq.LQ_ERR_IO and "truncated" in lq.lib().lq_last_error().decode()
    f.write_bytes(b"LQB200CK" + struct.pack("<I", 7))       # unknown version
    st, _ = load(f)
    assert st == lq.LQ_ERR_IO and "version 7" in lq.lib().lq_last_error().decode()
    st, _ = load(tmp_path / "missing.lqck")
    assert st == lq.LQ_ERR_IO
