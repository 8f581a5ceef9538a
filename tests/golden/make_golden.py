"""Generate golden vectors from the reference's own CUDA kernels.

    python tests/golden/make_golden.py [--out DIR]   # on a machine with a CUDA GPU

Runs the reference's Predictor, Corrector (Drucker-Prager and hypoplastic),
AdamiBoundary and StressRegularization -- src/predictor_corrector.cu,
src/adami_boundary.cu, src/field_smoothing.cu compiled unchanged for sm_100a
into oracle/_ref/ by `make -C oracle ref` -- on small seeded inputs and stores
inputs and outputs as .npz files beside this script.  tests/test_golden.py
checks the FP64 oracle against them on the CPU.

The inputs are built from the case generator (a jittered soil column with
Adami walls); cell bounds come from the oracle's float-key grid, which the
GPU tests prove bit-exact with the product's grid.
"""
from __future__ import annotations

import ctypes
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def main(argv=None):
    import argparse

    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", type=Path, default=HERE, help="directory for the .npz files (default: beside this script)")
    out_dir = ap.parse_args(argv).out
    out_dir.mkdir(parents=True, exist_ok=True)

    import oracle
    from loquat_b200 import cases

    assert torch.cuda.is_available(), "needs a CUDA device"
    assert oracle.ref_available(), "build the reference kernels first: make -C oracle ref"
    R = oracle.ref_lib()

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()

    def devi(a):
        return torch.from_numpy(np.ascontiguousarray(a, np.int32)).cuda()

    def par_dev(par):
        return torch.from_numpy(np.frombuffer(par.to_bytes(), np.uint8).copy()).cuda()

    out_files = []

    # ---------------------------------------------------- integrator cases
    for model in (1, 2):
        c = cases.small_column(nsx=8, nsy=4, nsz=8, model=model, seed=40 + model, velocity_noise=0.05)
        par = c.par
        n = par.np
        rng = np.random.default_rng(100 + model)
        st = [a.copy() for a in c.arrays()]
        st[3][par.npb:] += (2e3 * rng.standard_normal((par.npm, 6))).astype(np.float32)
        st[3][par.npb + 2::11] = np.float32(0.1)        # hypoplastic near-zero reset path
        st[4][:] = (1e-3 * rng.standard_normal((n, 6))).astype(np.float32)
        st[2][:, 1] = np.abs(1e-3 * rng.standard_normal(n)).astype(np.float32)
        accad = np.zeros((n, 4), np.float32)
        accad[:, :3] = rng.standard_normal((n, 3)) * 20.0
        accad[:, 3] = rng.standard_normal(n) * 500.0
        spin = np.zeros((n, 4), np.float32)
        spin[:, :3] = rng.standard_normal((n, 3)) * 5.0
        acestn = (rng.standard_normal((n, 6)) * 20.0).astype(np.float32)
        acestn[par.npb::5, 3] *= 200.0                   # far past the yield surface
        acestn[par.npb + 1::7, :3] = 500.0               # past the tension cut-off
        ini = [a.copy() for a in st]
        ini[1][:, :3] += (0.01 * rng.standard_normal((n, 3))).astype(np.float32)
        for which in ("predictor", "corrector"):
            d = [dev(a) for a in st]
            di = [dev(a) for a in (ini if which == "corrector" else [np.zeros_like(a) for a in st])]
            dr = [dev(a) for a in (accad, spin, acestn)]
            ph, pd = par.copy(), par_dev(par)
            f = R.ref_predictor if which == "predictor" else R.ref_corrector
            rc = f(ctypes.addressof(ph), pd.data_ptr(), *[x.data_ptr() for x in d + di + dr])
            assert rc == 0, rc
            outs = [x.cpu().numpy() for x in d]
            name = out_dir / f"ref_{which}_model{model}.npz"
            np.savez_compressed(
                name, params=np.frombuffer(par.to_bytes(), np.uint8),
                pos=st[0], vel=st[1], idep=st[2], str=st[3], stn=st[4],
                pos0=ini[0], vel0=ini[1], idep0=ini[2], str0=ini[3], stn0=ini[4],
                accad=accad, spin=spin, acestn=acestn,
                out_pos=outs[0], out_vel=outs[1], out_idep=outs[2], out_str=outs[3], out_stn=outs[4])
            out_files.append(name)

    # ------------------------------------------------- Adami and Shepard
    c = cases.small_column(nsx=10, nsy=5, nsz=8, seed=44, velocity_noise=0.02)
    par = c.par
    g = oracle.grid_float(par, c.pospres, par.npb)
    idx = g["part_idx"]
    st = [a[idx].copy() for a in c.arrays()]
    rng = np.random.default_rng(7)
    st[1][:, 3] *= (1.0 + 0.02 * rng.standard_normal(par.np)).astype(np.float32)
    st[3][par.npb:] += (1e2 * rng.standard_normal((par.npm, 6))).astype(np.float32)
    ph, pd = par.copy(), par_dev(par)
    x, v, beg, end = dev(st[0]), dev(st[1]), devi(g["cell_beg"]), devi(g["cell_end"])
    s_a = dev(st[3])
    assert R.ref_adami(ctypes.addressof(ph), pd.data_ptr(), x.data_ptr(), v.data_ptr(), s_a.data_ptr(),
                       beg.data_ptr(), end.data_ptr()) == 0
    s_s, cache = dev(st[3]), torch.zeros((par.np, 6), dtype=torch.float32, device="cuda")
    assert R.ref_shepard(ctypes.addressof(ph), pd.data_ptr(), x.data_ptr(), v.data_ptr(), s_s.data_ptr(),
                         cache.data_ptr(), beg.data_ptr(), end.data_ptr()) == 0
    name = out_dir / "ref_adami_shepard.npz"
    np.savez_compressed(name, params=np.frombuffer(par.to_bytes(), np.uint8), pos=st[0], vel=st[1], str=st[3],
                        cell_beg=g["cell_beg"], cell_end=g["cell_end"], out_adami=s_a.cpu().numpy(),
                        out_shepard=s_s.cpu().numpy())
    out_files.append(name)
    for f in out_files:
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
