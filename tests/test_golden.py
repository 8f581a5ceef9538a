"""The FP64 oracle against golden vectors produced by the reference's own
CUDA kernels (src/predictor_corrector.cu, src/adami_boundary.cu,
src/field_smoothing.cu compiled unchanged; see tests/golden/make_golden.py).

This pins the oracle's predictor, corrector, Drucker-Prager and hypoplastic
updates, Adami extrapolation and Shepard filter to the reference itself:
the only differences allowed are FP32 (reference) vs FP64 (oracle)
rounding.  Runs on the CPU."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from loquat_b200.params import Parameters

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 1e-5   # relative L2, FP32 reference vs FP64 oracle, one update


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a))


def load(name):
    f = GOLDEN / name
    if not f.exists():
        pytest.fail(f"golden fixture {name} missing: run tests/golden/make_golden.py on a GPU")
    z = np.load(f)
    par = Parameters.from_bytes(z["params"].tobytes())
    return par, z


@pytest.mark.parametrize("model", [1, 2])
@pytest.mark.parametrize("which", ["predictor", "corrector"])
def test_oracle_integrator_matches_reference_kernels(orc, model, which):
    par, z = load(f"ref_{which}_model{model}.npz")
    st = [z["pos"], z["vel"], z["idep"], z["str"], z["stn"]]
    rates = [z["accad"], z["spin"], z["acestn"]]
    if which == "predictor":
        got = orc.predictor(par, st, rates)
    else:
        ini = [z["pos0"], z["vel0"], z["idep0"], z["str0"], z["stn0"]]
        got = orc.corrector(par, st, ini, rates)
    want = [z["out_pos"], z["out_vel"], z["out_idep"], z["out_str"], z["out_stn"]]
    m = slice(par.npb, par.np)
    for k, name in enumerate(["pos", "vel", "idep", "str", "stn"]):
        assert rel(got[k][m], want[k][m]) < TOL, (name, rel(got[k][m], want[k][m]))
        # the reference leaves boundary slots alone
        assert np.array_equal(want[k][: par.npb], st[k][: par.npb]), name
    # plastic strain actually changed somewhere (return map exercised)
    assert np.any(want[2][m, 1] != st[2][m, 1])


def test_oracle_adami_and_shepard_match_reference_kernels(orc):
    par, z = load("ref_adami_shepard.npz")
    pos, vel, s = z["pos"], z["vel"], z["str"]
    got = orc.adami(par, pos, vel, s, z["cell_beg"], z["cell_end"])
    b = slice(0, par.npb)
    assert rel(got[b], z["out_adami"][b]) < TOL
    assert np.array_equal(z["out_adami"][par.npb:], s[par.npb:])
    got = orc.shepard(par, pos, vel, s, z["cell_beg"], z["cell_end"])
    m = slice(par.npb, par.np)
    assert rel(got[m], z["out_shepard"][m]) < TOL
    assert np.array_equal(z["out_shepard"][: par.npb], s[: par.npb])
