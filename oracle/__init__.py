"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the FP64 CPU oracle
(``oracle/lq_oracle.cpp``) and of the reference's own open kernels compiled
into ``oracle/_ref/``.  Imported by tests/, __graft_entry__.smoke() (as the
checker) and bench.py's CPU-baseline leg; never by the product package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liblq_oracle.so"
REF_LIB = HERE / "_ref" / "libref_kernels.so"
# Where the reference's sources are read from when its open kernels are
# compiled into _ref/ (LOQUAT_REFERENCE overrides the default location of
# the read-only checkout).
REFERENCE_TREE = Path(os.environ.get("LOQUAT_REFERENCE") or "/root/reference")

_lib = None
_ref = None
_VP, _I, _D, _LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference tree is present, the
    reference-kernel harness)."""
    subprocess.run(["make", "-C", str(HERE), "liblq_oracle.so"], check=True, capture_output=True)
    if ref and (REFERENCE_TREE / "src" / "predictor_corrector.cu").exists():
        subprocess.run(["make", "-C", str(HERE), "ref", f"REF={REFERENCE_TREE}"], check=True, capture_output=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build(ref=False)
        L = ctypes.CDLL(str(LIB))
        L.or_sim_create.restype = _VP
        L.or_sim_create.argtypes = [_VP] * 6 + [_LL, _D]
        L.or_sim_step.argtypes = [_VP, _I]
        L.or_sim_get.argtypes = [_VP] * 6
        L.or_sim_destroy.argtypes = [_VP]
        L.or_sim_steps_done.restype = _LL
        L.or_sim_steps_done.argtypes = [_VP]
        L.or_set_threads.argtypes = [_I]
        L.or_set_gather_rounding.argtypes = [_I]
        L.or_initialize_parameters.argtypes = [_VP]
        L.or_grid_float.argtypes = [_VP, _I, _I] + [_VP] * 6
        L.or_interaction.argtypes = [_VP, _I, _I] + [_VP] * 8
        L.or_adami.argtypes = [_VP, _I, _I] + [_VP] * 5
        L.or_shepard.argtypes = [_VP, _I, _I] + [_VP] * 6
        L.or_predictor.argtypes = [_VP, _I, _I] + [_VP] * 8
        L.or_corrector.argtypes = [_VP, _I, _I] + [_VP] * 13
        L.or_dp_update.argtypes = [_VP, _D] + [_VP] * 5
        L.or_hypo_update.argtypes = [_VP, _D] + [_VP] * 3
        L.or_sim_set_vw.argtypes = [_VP, _I, _VP]
        L.or_sim_set_extensions.argtypes = [_VP, _I, _I]
        L.or_sim_time.restype = ctypes.c_double
        L.or_sim_time.argtypes = [_VP]
        L.or_vw_update.argtypes = [_VP, _D, _VP, _VP, _VP, _VP]
        L.or_vw_rate.argtypes = [_VP, _VP, _D, _VP, _VP, _VP, _VP]
        _lib = L
    return _lib


def ref_available() -> bool:
    return REF_LIB.exists()


def ref_lib():
    """The reference's own predictor/corrector/Adami/Shepard kernels (GPU)."""
    global _ref
    if _ref is None:
        L = ctypes.CDLL(str(REF_LIB))
        for n in ("ref_predictor", "ref_corrector"):
            getattr(L, n).argtypes = [_VP] * 15
        L.ref_adami.argtypes = [_VP] * 7
        L.ref_shepard.argtypes = [_VP] * 8
        _ref = L
    return _ref


def _d(a, cols):
    return np.ascontiguousarray(np.asarray(a, np.float64).reshape(-1, cols))


def _p(a):
    return a.ctypes.data


def set_threads(n: int = 0) -> int:
    return lib().or_set_threads(n)


GATHER_F16_VELOCITY, GATHER_F16_STRESS, GATHER_BF16_VELOCITY, GATHER_BF16_STRESS = 1, 2, 4, 8
GATHER_FP21_VELOCITY, GATHER_SHARED_EXP18_VELOCITY = 16, 32


def set_gather_rounding(mode: int = 0) -> None:
    """Precision experiment: the interaction rounds a neighbour's gathered
    velocity and/or sigma/rho^2 to FP16 or BF16, or the velocity to three
    21-bit floats (GATHER_FP21_VELOCITY) or to one shared exponent with
    three 18-bit mantissas (GATHER_SHARED_EXP18_VELOCITY) (bit mask of the
    GATHER_* constants), as a GPU form with packed gathers would; 0
    restores exact gathers.  Applies to every later interaction of this
    process."""
    lib().or_set_gather_rounding(int(mode))


def initialize_parameters(par) -> None:
    lib().or_initialize_parameters(ctypes.addressof(par))


def grid_float(par, pos, npb):
    """Bit-exact grid of float positions: dict of part_cel, part_idx, cell_beg,
    cell_end, cell_start."""
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 4)
    n = pos.shape[0]
    out = dict(part_cel=np.empty(n, np.int32), part_idx=np.empty(n, np.int32),
               cell_beg=np.empty(par.ncell, np.int32), cell_end=np.empty(par.ncell, np.int32),
               cell_start=np.empty(par.ncell + 1, np.int32))
    lib().or_grid_float(ctypes.addressof(par), n, npb, _p(pos), *[_p(out[k]) for k in
                                                                 ("part_cel", "part_idx", "cell_beg", "cell_end",
                                                                  "cell_start")])
    return out


def interaction(par, pos, vel, str_, beg, end):
    pos, vel, s = _d(pos, 4), _d(vel, 4), _d(str_, 6)
    n = pos.shape[0]
    accad, spin, acestn = np.zeros((n, 4)), np.zeros((n, 4)), np.zeros((n, 6))
    beg = np.ascontiguousarray(beg, np.int32)
    end = np.ascontiguousarray(end, np.int32)
    lib().or_interaction(ctypes.addressof(par), n, par.npb, _p(pos), _p(vel), _p(s), _p(accad), _p(spin),
                         _p(acestn), _p(beg), _p(end))
    return accad, spin, acestn


def adami(par, pos, vel, str_, beg, end):
    pos, vel, s = _d(pos, 4), _d(vel, 4), _d(str_, 6).copy()
    beg = np.ascontiguousarray(beg, np.int32)
    end = np.ascontiguousarray(end, np.int32)
    lib().or_adami(ctypes.addressof(par), pos.shape[0], par.npb, _p(pos), _p(vel), _p(s), _p(beg), _p(end))
    return s


def shepard(par, pos, vel, str_, beg, end):
    pos, vel, s = _d(pos, 4), _d(vel, 4), _d(str_, 6)
    out = s.copy()
    beg = np.ascontiguousarray(beg, np.int32)
    end = np.ascontiguousarray(end, np.int32)
    lib().or_shepard(ctypes.addressof(par), pos.shape[0], par.npb, _p(pos), _p(vel), _p(s), _p(out), _p(beg),
                     _p(end))
    return out


def predictor(par, state, rates):
    st = [_d(state[0], 4).copy(), _d(state[1], 4).copy(), _d(state[2], 4).copy(), _d(state[3], 6).copy(),
          _d(state[4], 6).copy()]
    r = [_d(rates[0], 4), _d(rates[1], 4), _d(rates[2], 6)]
    lib().or_predictor(ctypes.addressof(par), st[0].shape[0], par.npb, *map(_p, st), *map(_p, r))
    return st


def corrector(par, state, ini, rates):
    st = [_d(state[0], 4).copy(), _d(state[1], 4).copy(), _d(state[2], 4).copy(), _d(state[3], 6).copy(),
          _d(state[4], 6).copy()]
    iv = [_d(ini[0], 4), _d(ini[1], 4), _d(ini[2], 4), _d(ini[3], 6), _d(ini[4], 6)]
    r = [_d(rates[0], 4), _d(rates[1], 4), _d(rates[2], 6)]
    lib().or_corrector(ctypes.addressof(par), st[0].shape[0], par.npb, *map(_p, st), *map(_p, iv), *map(_p, r))
    return st


def dp_update(par, dtp, spin3, d6, p, ep, s6):
    spin3, d6, s6 = _d(spin3, 3).ravel().copy(), _d(d6, 6).ravel().copy(), _d(s6, 6).ravel().copy()
    pp, ee = np.array([p], np.float64), np.array([ep], np.float64)
    lib().or_dp_update(ctypes.addressof(par), dtp, _p(spin3), _p(d6), _p(pp), _p(ee), _p(s6))
    return float(pp[0]), float(ee[0]), s6


def hypo_update(par, dtp, d6, spin3, s6):
    spin3, d6, s6 = _d(spin3, 3).ravel().copy(), _d(d6, 6).ravel().copy(), _d(s6, 6).ravel().copy()
    lib().or_hypo_update(ctypes.addressof(par), dtp, _p(d6), _p(spin3), _p(s6))
    return s6


class OracleSim:
    """FP64 whole-step oracle (reference src/loquat.cu:322-409)."""

    def __init__(self, par, pospres, velrhop, idep, str_, stn, step0: int = 0, time0: float = 0.0):
        self.par = par
        arrs = [_d(pospres, 4), _d(velrhop, 4), _d(idep, 4), _d(str_, 6), _d(stn, 6)]
        self.np = arrs[0].shape[0]
        self.h = lib().or_sim_create(ctypes.addressof(par), *map(_p, arrs), step0, time0)

    def set_vw(self, rows):
        """Model-3 (von Wolffersdorff) material rows, n x 10, by object id."""
        self._vw = np.ascontiguousarray(rows, np.float32).reshape(-1, 10)
        lib().or_sim_set_vw(self.h, self._vw.shape[0], _p(self._vw))

    def set_extensions(self, density_filter: bool = False, dynamic_dt: bool = False):
        """Features the reference declares but does not apply: the density
        Shepard filter and the dynamic time step."""
        lib().or_sim_set_extensions(self.h, int(density_filter), int(dynamic_dt))

    def time(self) -> float:
        return lib().or_sim_time(self.h)

    def step(self, n: int = 1):
        if lib().or_sim_step(self.h, n) != 0:
            raise RuntimeError("OracleSim.step: constitutive model 3 needs set_vw first")

    def get(self):
        n = self.np
        out = [np.empty((n, 4)), np.empty((n, 4)), np.empty((n, 4)), np.empty((n, 6)), np.empty((n, 6))]
        lib().or_sim_get(self.h, *map(_p, out))
        return out

    def close(self):
        if self.h:
            lib().or_sim_destroy(self.h)
            self.h = None

    __del__ = close


def vw_update(row, dt, d6, spin3, s6, e):
    row = np.ascontiguousarray(row, np.float32)
    d6, spin3, s6 = _d(d6, 6).ravel().copy(), _d(spin3, 3).ravel().copy(), _d(s6, 6).ravel().copy()
    ee = np.array([e], np.float64)
    n = lib().or_vw_update(_p(row), dt, _p(d6), _p(spin3), _p(s6), _p(ee))
    return s6, float(ee[0]), n


def vw_rate(row, s6, e, d6, spin3):
    row = np.ascontiguousarray(row, np.float32)
    s6, d6, spin3 = _d(s6, 6).ravel().copy(), _d(d6, 6).ravel().copy(), _d(spin3, 3).ravel().copy()
    r, er = np.zeros(6), np.zeros(1)
    lib().or_vw_rate(_p(row), _p(s6), e, _p(d6), _p(spin3), _p(r), _p(er))
    return r, float(er[0])
