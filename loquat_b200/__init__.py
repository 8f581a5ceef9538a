"""LOQUAT-B200: sm_100a kernels for LOQUAT's per-step SPH path.

Python host mirror of the C ABI in ``include/loquat_b200.h``.  Every call goes
through ``liblqb200.so`` (built in-tree by ``python -m loquat_b200.build``); there
is no CPU fallback, and importing a function whose library is missing raises.

Device arrays are passed as integer device addresses or as objects with a
``data_ptr()`` method (torch tensors).  Host arrays are numpy arrays.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from .params import Parameters, PARAMETER_FIELDS, dp_cone, elastic_moduli  # noqa: F401

# LOQUAT_B200_LIB selects another build of the same library (kernel variants
# compared side by side); by default the in-tree build is used.
_LIB_PATH = Path(os.environ.get("LOQUAT_B200_LIB") or Path(__file__).resolve().parent / "liblqb200.so")
_lib = None

LQ_OK, LQ_ERR_ARG, LQ_ERR_CUDA, LQ_ERR_ALLOC, LQ_ERR_IO, LQ_ERR_STATE, LQ_ERR_NOTFOUND = range(7)
LQ_SIM_GRAPH = 1
LQ_SIM_MIXED = 2
LQ_SIM_DENSITY_FILTER = 4
LQ_SIM_DYNAMIC_DT = 8


class LoquatError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


_VP, _I, _F, _D, _LL, _SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_longlong, ctypes.c_size_t

# name -> (restype, argtypes); the declarations of include/loquat_b200.h
_SIGNATURES = {
    "lq_abi_version": (_I, []),
    "lq_parameters_size": (_SZ, []),
    "lq_last_error": (ctypes.c_char_p, []),
    "lq_status_string": (ctypes.c_char_p, [_I]),
    "lq_initialize_parameters": (_I, [_VP]),
    "lq_update_time_step": (_I, [_VP]),
    "lq_grid_create": (_I, [_I, _I, ctypes.POINTER(_VP)]),
    "lq_grid_resize": (_I, [_VP, _I, _I]),
    "lq_grid_destroy": (_I, [_VP]),
    "lq_grid_neighbor_search": (_I, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "lq_grid_arrays": (_I, [_VP] + [ctypes.POINTER(_VP)] * 5),
    "lq_grid_sort_float4": (_I, [_VP, _I, _VP, _VP, _VP]),
    "lq_grid_sort_tensor2d": (_I, [_VP, _I, _VP, _VP, _VP]),
    "lq_grid_neighbor_search_noalloc": (_I, [_VP] * 8),
    "lq_interaction_reserve": (_I, [_VP]),
    "lq_interaction_stats": (_I, [ctypes.POINTER(_LL), ctypes.POINTER(_LL)]),
    "lq_particle_interaction": (_I, [_VP] * 13),
    "lq_adami_boundary": (_I, [_VP] * 8),
    "lq_stress_regularization": (_I, [_VP] * 9),
    "lq_predictor": (_I, [_VP] * 16),
    "lq_corrector": (_I, [_VP] * 16),
    "lq_sim_create": (_I, [_VP] * 6 + [_I, ctypes.POINTER(_VP)]),
    "lq_sim_destroy": (_I, [_VP]),
    "lq_sim_step": (_I, [_VP, _I]),
    "lq_sim_synchronize": (_I, [_VP]),
    "lq_sim_stream": (_I, [_VP, ctypes.POINTER(_VP)]),
    "lq_sim_upload": (_I, [_VP] * 6),
    "lq_sim_download": (_I, [_VP] * 6),
    "lq_sim_state": (_I, [_VP] + [ctypes.POINTER(_VP)] * 5),
    "lq_sim_clock": (_I, [_VP, ctypes.POINTER(_LL), ctypes.POINTER(_D)]),
    "lq_sim_health": (_I, [_VP, _VP]),
    "lq_sim_launches_per_step": (_I, [_VP, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "lq_sim_profile": (_I, [_VP, _I, _VP, _VP]),
    "lq_sim_set_skin": (_I, [_VP, _F]),
    "lq_sim_set_materials": (_I, [_VP, _I, _VP]),
    "lq_sim_set_hypoplastic": (_I, [_VP, _I, _VP]),
    "lq_sim_set_frames": (_I, [_VP, _I, _VP]),
    "lq_sim_rebuilds": (_I, [_VP, ctypes.POINTER(_LL)]),
    "lq_sim_rebuild_launches": (_I, [_VP, ctypes.POINTER(_I)]),
    "lq_sim_set_wide_skin": (_I, [_VP, _F]),
    "lq_sim_wide_skin": (_I, [_VP, ctypes.POINTER(_F)]),
    "lq_sim_renewals": (_I, [_VP, ctypes.POINTER(_LL)]),
    "lq_sim_renewal_launches": (_I, [_VP, ctypes.POINTER(_I)]),
    "lq_sim_set_pair_shape": (_I, [_VP, _I]),
    "lq_sim_pair_shape": (_I, [_VP, ctypes.POINTER(_I)]),
    "lq_sim_autotune": (_I, [_VP, _I, ctypes.POINTER(_I), ctypes.POINTER(_F)]),
    "lq_debug_bounds_violations": (_I, [ctypes.POINTER(_LL)]),
    "lq_sim_save_checkpoint": (_I, [_VP, ctypes.c_char_p]),
    "lq_sim_load_checkpoint": (_I, [ctypes.c_char_p, _I, ctypes.POINTER(_VP)]),
    "lq_sim_neighbor_entries": (_I, [_VP, ctypes.POINTER(_LL), ctypes.POINTER(_LL)]),
    "lq_io_load_parameters": (_I, [ctypes.c_char_p, _VP]),
    "lq_io_save_parameters": (_I, [ctypes.c_char_p, _VP]),
    "lq_io_load_hypoplastic": (_I, [ctypes.c_char_p, _VP, ctypes.POINTER(_F)]),
    "lq_io_save_parameters_vw": (_I, [ctypes.c_char_p, _VP, _VP, _F]),
    "lq_io_load_particles": (_I, [ctypes.c_char_p, _I] + [_VP] * 5),
    "lq_io_save_particles": (_I, [ctypes.c_char_p, _I] + [_VP] * 5),
    "lq_io_save_vtu": (_I, [ctypes.c_char_p, _I, _I] + [_VP] * 5),
}


def lib_path() -> Path:
    return _LIB_PATH


def lib():
    """The loaded C library.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise RuntimeError(
                f"LOQUAT-B200 CUDA library missing at {_LIB_PATH}; build it with "
                "`python -m loquat_b200.build` (there is no CPU fallback)")
        L = ctypes.CDLL(str(_LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGNATURES)


def check(status: int, what: str = "") -> None:
    if status != LQ_OK:
        msg = lib().lq_last_error().decode(errors="replace")
        raise LoquatError(status, f"{what}: {msg}" if what else msg)


def ptr(x) -> int | None:
    """Address of a device tensor / numpy array / raw integer pointer."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if isinstance(x, Parameters):
        return ctypes.addressof(x)
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    raise TypeError(f"cannot take the address of {type(x)}")


def initialize_parameters(par: Parameters) -> Parameters:
    check(lib().lq_initialize_parameters(ctypes.byref(par)), "lq_initialize_parameters")
    return par


def update_time_step(par: Parameters) -> Parameters:
    check(lib().lq_update_time_step(ctypes.byref(par)), "lq_update_time_step")
    return par


LQ_NOALLOC_MAX_PARTICLES = 1048576
LQ_NOALLOC_MAX_CELLS = 1048575


def grid_neighbor_search_noalloc(par_host, par_dev, pospres, part_cel, part_idx, cell_beg, cell_end, stream=None):
    """lq_grid_neighbor_search_noalloc: the neighbour search for callers that
    cannot allocate device memory; outputs are caller-provided device arrays
    and the working arrays are a fixed array inside the library (see
    include/loquat_b200.h for the limits and the sharing rules)."""
    check(lib().lq_grid_neighbor_search_noalloc(ptr(par_host), ptr(par_dev), ptr(pospres), ptr(part_cel),
                                                ptr(part_idx), ptr(cell_beg), ptr(cell_end), stream),
          "lq_grid_neighbor_search_noalloc")


# ------------------------------------------------------------------ operators
def interaction_reserve(par_host) -> None:
    """lq_interaction_reserve: sizes particle_interaction's working arrays
    for par_host's particle and cell counts, once, before a step loop."""
    check(lib().lq_interaction_reserve(ptr(par_host)), "lq_interaction_reserve")


def interaction_stats():
    """lq_interaction_stats: (fresh list builds, calls that carried the
    lists over) of particle_interaction on the current device."""
    a, b = _LL(), _LL()
    check(lib().lq_interaction_stats(ctypes.byref(a), ctypes.byref(b)), "lq_interaction_stats")
    return a.value, b.value


def particle_interaction(par_host, par_dev, pospres, velrhop, idep, str_, stn, accad, spin, acestn,
                         cell_beg, cell_end, stream=None):
    """lq_particle_interaction (reference src/particle_interaction.h:27-40)."""
    check(lib().lq_particle_interaction(ptr(par_host), ptr(par_dev), ptr(pospres), ptr(velrhop), ptr(idep),
                                        ptr(str_), ptr(stn), ptr(accad), ptr(spin), ptr(acestn),
                                        ptr(cell_beg), ptr(cell_end), stream), "lq_particle_interaction")


def adami_boundary(par_host, par_dev, pospres, velrhop, str_, cell_beg, cell_end, stream=None):
    """lq_adami_boundary (reference src/adami_boundary.h:27-34)."""
    check(lib().lq_adami_boundary(ptr(par_host), ptr(par_dev), ptr(pospres), ptr(velrhop), ptr(str_),
                                  ptr(cell_beg), ptr(cell_end), stream), "lq_adami_boundary")


def stress_regularization(par_host, par_dev, pospres, velrhop, str_, cache, cell_beg, cell_end, stream=None):
    """lq_stress_regularization (reference src/field_smoothing.h:27-35)."""
    check(lib().lq_stress_regularization(ptr(par_host), ptr(par_dev), ptr(pospres), ptr(velrhop), ptr(str_),
                                         ptr(cache), ptr(cell_beg), ptr(cell_end), stream),
          "lq_stress_regularization")


def predictor(par_host, par_dev, state, ini, rates, stream=None):
    """lq_predictor; state/ini = (pospres, velrhop, idep, str, stn), rates = (accad, spin, acestn)."""
    check(lib().lq_predictor(ptr(par_host), ptr(par_dev), *map(ptr, state), *map(ptr, ini), *map(ptr, rates),
                             stream), "lq_predictor")


def corrector(par_host, par_dev, state, ini, rates, stream=None):
    """lq_corrector; same argument groups as predictor()."""
    check(lib().lq_corrector(ptr(par_host), ptr(par_dev), *map(ptr, state), *map(ptr, ini), *map(ptr, rates),
                             stream), "lq_corrector")


class Grid:
    """lq_grid_* (the LoquatGrid of reference src/loquat_grid.h:28-66)."""

    def __init__(self, np_: int, ncell: int):
        h = _VP()
        check(lib().lq_grid_create(np_, ncell, ctypes.byref(h)), "lq_grid_create")
        self.handle = h
        # held here so that a collection at interpreter exit, after the
        # module's globals are gone, can still release the grid
        self._destroy = lib().lq_grid_destroy

    def close(self):
        if getattr(self, "handle", None):
            self._destroy(self.handle)
            self.handle = None

    __del__ = close

    def neighbor_search(self, par_host, par_dev, pospres, idep=None, stream=None):
        check(lib().lq_grid_neighbor_search(self.handle, ptr(par_host), ptr(par_dev), ptr(pospres), ptr(idep),
                                            stream), "lq_grid_neighbor_search")

    def arrays(self) -> dict:
        out = [_VP() for _ in range(5)]
        check(lib().lq_grid_arrays(self.handle, *[ctypes.byref(o) for o in out]), "lq_grid_arrays")
        return dict(zip(["part_cel", "part_idx", "cell_beg", "cell_end", "cell_start"], [o.value for o in out]))

    def sort_float4(self, n, data, cache, stream=None):
        check(lib().lq_grid_sort_float4(self.handle, n, ptr(data), ptr(cache), stream), "lq_grid_sort_float4")

    def sort_tensor2d(self, n, data, cache, stream=None):
        check(lib().lq_grid_sort_tensor2d(self.handle, n, ptr(data), ptr(cache), stream), "lq_grid_sort_tensor2d")


def _sim_flags(graph, mixed, density_filter, dynamic_dt) -> int:
    return ((LQ_SIM_GRAPH if graph else 0) | (LQ_SIM_MIXED if mixed else 0)
            | (LQ_SIM_DENSITY_FILTER if density_filter else 0) | (LQ_SIM_DYNAMIC_DT if dynamic_dt else 0))


class Simulation:
    """Whole-step driver (lq_sim_*): the hot loop of reference src/loquat.cu:322-409."""

    def __init__(self, par: Parameters, pospres, velrhop, idep, str_, stn, graph: bool = True, mixed: bool = False,
                 density_filter: bool = False, dynamic_dt: bool = False):
        """density_filter / dynamic_dt switch on the density Shepard filter
        (every par.density_shepard_filter steps) and the dynamic time step,
        which the reference declares but never applies."""
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (pospres, velrhop, idep, str_, stn)]
        h = _VP()
        flags = _sim_flags(graph, mixed, density_filter, dynamic_dt)
        check(lib().lq_sim_create(ctypes.byref(par), *[a.ctypes.data for a in arrs], flags, ctypes.byref(h)),
              "lq_sim_create")
        self.handle = h
        self._destroy = lib().lq_sim_destroy    # usable at interpreter exit too
        self.np = par.np
        self.par = par.copy()

    @classmethod
    def load_checkpoint(cls, path, graph: bool = True, mixed: bool = False, density_filter: bool = False,
                        dynamic_dt: bool = False) -> "Simulation":
        """A simulation restored from lq_sim_save_checkpoint's file (every
        option but `graph` must match the saved run's)."""
        h = _VP()
        flags = _sim_flags(graph, mixed, density_filter, dynamic_dt)
        check(lib().lq_sim_load_checkpoint(os.fsencode(str(path)), flags, ctypes.byref(h)), "lq_sim_load_checkpoint")
        self = cls.__new__(cls)
        self.handle = h
        self._destroy = lib().lq_sim_destroy
        with open(path, "rb") as f:
            f.seek(48)           # magic, version, flags, step, time, skin, three counts
            self.par = Parameters.from_bytes(f.read(ctypes.sizeof(Parameters)))
        self.np = self.par.np
        return self

    def close(self):
        if getattr(self, "handle", None):
            self._destroy(self.handle)
            self.handle = None

    __del__ = close

    def step(self, n: int = 1):
        check(lib().lq_sim_step(self.handle, n), "lq_sim_step")

    def synchronize(self):
        check(lib().lq_sim_synchronize(self.handle), "lq_sim_synchronize")

    def stream(self) -> int:
        s = _VP()
        check(lib().lq_sim_stream(self.handle, ctypes.byref(s)), "lq_sim_stream")
        return s.value or 0

    def download(self, out=None):
        n = self.np
        if out is None:
            out = (np.empty((n, 4), np.float32), np.empty((n, 4), np.float32), np.empty((n, 4), np.float32),
                   np.empty((n, 6), np.float32), np.empty((n, 6), np.float32))
        check(lib().lq_sim_download(self.handle, *[ptr(a) for a in out]), "lq_sim_download")
        return out

    def upload(self, pospres, velrhop, idep, str_, stn):
        check(lib().lq_sim_upload(self.handle, *[ptr(a) for a in (pospres, velrhop, idep, str_, stn)]),
              "lq_sim_upload")

    def state_pointers(self) -> dict:
        out = [_VP() for _ in range(5)]
        check(lib().lq_sim_state(self.handle, *[ctypes.byref(o) for o in out]), "lq_sim_state")
        return dict(zip(["pospres", "velrhop", "idep", "str", "stn"], [o.value for o in out]))

    def clock(self):
        s, t = _LL(), _D()
        check(lib().lq_sim_clock(self.handle, ctypes.byref(s), ctypes.byref(t)), "lq_sim_clock")
        return s.value, t.value

    def health(self) -> np.ndarray:
        h = np.zeros(4, np.int32)
        check(lib().lq_sim_health(self.handle, h.ctypes.data), "lq_sim_health")
        return h

    PHASES = ("search", "gather", "adami", "interaction", "integrate", "shepard", "list", "renew")

    def profile(self, n: int) -> dict:
        """Runs n steps eagerly with CUDA events around each phase; returns
        {phase: (total_ms, launches)}."""
        ms = np.zeros(len(self.PHASES), np.float64)
        cnt = np.zeros(len(self.PHASES), np.int32)
        check(lib().lq_sim_profile(self.handle, n, ms.ctypes.data, cnt.ctypes.data), "lq_sim_profile")
        return {p: (float(ms[k]), int(cnt[k])) for k, p in enumerate(self.PHASES)}

    def set_skin(self, skin_over_h: float):
        check(lib().lq_sim_set_skin(self.handle, skin_over_h), "lq_sim_set_skin")

    def set_materials(self, table):
        """Per-object model parameters: row k (5 floats) applies to material
        particles whose idep.x is k."""
        t = np.ascontiguousarray(table, np.float32).reshape(-1, 5)
        check(lib().lq_sim_set_materials(self.handle, t.shape[0], t.ctypes.data), "lq_sim_set_materials")

    def set_hypoplastic(self, table):
        """Constitutive model 3 rows (10 floats per object id): phi_c (deg),
        h_s, n, e_d0, e_c0, e_i0, alpha, beta, sub-step tolerance, maximum
        sub-steps.  The void ratio is carried in idep.z."""
        t = np.ascontiguousarray(table, np.float32).reshape(-1, 10)
        check(lib().lq_sim_set_hypoplastic(self.handle, t.shape[0], t.ctypes.data), "lq_sim_set_hypoplastic")

    def set_frames(self, rows):
        """Per-object grid rows: rows[k] = (first row, number of rows)."""
        r = np.ascontiguousarray(rows, np.int32).reshape(-1, 2)
        check(lib().lq_sim_set_frames(self.handle, r.shape[0], r.ctypes.data), "lq_sim_set_frames")

    def rebuilds(self) -> int:
        c = _LL()
        check(lib().lq_sim_rebuilds(self.handle, ctypes.byref(c)), "lq_sim_rebuilds")
        return c.value

    def rebuild_launches(self) -> int:
        c = _I()
        check(lib().lq_sim_rebuild_launches(self.handle, ctypes.byref(c)), "lq_sim_rebuild_launches")
        return c.value

    def set_wide_skin(self, wide_over_h: float):
        """Two-level lists: wide lists with cut-off 2h + wide_over_h h from
        each sort, the stages' lists renewed from them without a search; 0
        (or a value not above the skin) gives one-level lists."""
        check(lib().lq_sim_set_wide_skin(self.handle, wide_over_h), "lq_sim_set_wide_skin")

    def wide_skin(self) -> float:
        c = _F()
        check(lib().lq_sim_wide_skin(self.handle, ctypes.byref(c)), "lq_sim_wide_skin")
        return c.value

    def renewals(self) -> int:
        """Lists renewed from the wide lists without a search so far."""
        c = _LL()
        check(lib().lq_sim_renewals(self.handle, ctypes.byref(c)), "lq_sim_renewals")
        return c.value

    def renewal_launches(self) -> int:
        c = _I()
        check(lib().lq_sim_renewal_launches(self.handle, ctypes.byref(c)), "lq_sim_renewal_launches")
        return c.value

    def set_pair_shape(self, shape: int):
        check(lib().lq_sim_set_pair_shape(self.handle, shape), "lq_sim_set_pair_shape")

    def pair_shape(self) -> int:
        v = ctypes.c_int()
        check(lib().lq_sim_pair_shape(self.handle, ctypes.byref(v)), "lq_sim_pair_shape")
        return v.value

    def autotune(self, steps: int = 20):
        """Chooses the pair kernel's launch shape and the list skin by timing
        (state left as it was); returns (shape, skin / h)."""
        sh, sk = _I(), _F()
        check(lib().lq_sim_autotune(self.handle, steps, ctypes.byref(sh), ctypes.byref(sk)), "lq_sim_autotune")
        return sh.value, sk.value

    def save_checkpoint(self, path):
        """Binary checkpoint (state, FP64 copies, step, time, tables); the
        run that continues and a run loaded from the file step identically."""
        check(lib().lq_sim_save_checkpoint(self.handle, os.fsencode(str(path))), "lq_sim_save_checkpoint")

    def neighbor_entries(self):
        """(material, boundary) entries in the current neighbour lists."""
        a, b = _LL(), _LL()
        check(lib().lq_sim_neighbor_entries(self.handle, ctypes.byref(a), ctypes.byref(b)),
              "lq_sim_neighbor_entries")
        return a.value, b.value

    def launches_per_step(self):
        a, b = _I(), _I()
        check(lib().lq_sim_launches_per_step(self.handle, ctypes.byref(a), ctypes.byref(b)),
              "lq_sim_launches_per_step")
        return a.value, b.value


# -------------------------------------------------------------------- formats
def load_parameters(xml_path) -> Parameters:
    p = Parameters()
    check(lib().lq_io_load_parameters(os.fsencode(str(xml_path)), ctypes.byref(p)), "lq_io_load_parameters")
    return p


def save_parameters(xml_path, par: Parameters, hypoplastic=None) -> None:
    """Writes the parameter file; `hypoplastic` = (10-float row, initial void
    ratio) adds the model-3 keys."""
    if hypoplastic is None:
        check(lib().lq_io_save_parameters(os.fsencode(str(xml_path)), ctypes.byref(par)), "lq_io_save_parameters")
        return
    row = np.ascontiguousarray(hypoplastic[0], np.float32).reshape(10)
    check(lib().lq_io_save_parameters_vw(os.fsencode(str(xml_path)), ctypes.byref(par), row.ctypes.data,
                                         float(hypoplastic[1])), "lq_io_save_parameters_vw")


def load_hypoplastic(xml_path):
    """(10-float model-3 row, initial void ratio) from a parameter file."""
    row = np.zeros(10, np.float32)
    e0 = _F()
    check(lib().lq_io_load_hypoplastic(os.fsencode(str(xml_path)), row.ctypes.data, ctypes.byref(e0)),
          "lq_io_load_hypoplastic")
    return row, e0.value


def load_particles(dat_path, np_: int):
    arrs = (np.empty((np_, 4), np.float32), np.empty((np_, 4), np.float32), np.empty((np_, 4), np.float32),
            np.empty((np_, 6), np.float32), np.empty((np_, 6), np.float32))
    check(lib().lq_io_load_particles(os.fsencode(str(dat_path)), np_, *[a.ctypes.data for a in arrs]),
          "lq_io_load_particles")
    return arrs


def save_particles(dat_path, pospres, velrhop, idep, str_, stn) -> None:
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (pospres, velrhop, idep, str_, stn)]
    check(lib().lq_io_save_particles(os.fsencode(str(dat_path)), arrs[0].shape[0], *[a.ctypes.data for a in arrs]),
          "lq_io_save_particles")


def save_vtu(directory, output_number: int, pospres, velrhop, idep, str_, stn) -> None:
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (pospres, velrhop, idep, str_, stn)]
    check(lib().lq_io_save_vtu(os.fsencode(str(directory)), output_number, arrs[0].shape[0],
                               *[a.ctypes.data for a in arrs]), "lq_io_save_vtu")


def bounds_violations() -> int:
    """Index-bounds violations counted by a bounds-checked build of the
    library (loaded through LOQUAT_B200_LIB); -1 for the product build."""
    c = _LL()
    check(lib().lq_debug_bounds_violations(ctypes.byref(c)), "lq_debug_bounds_violations")
    return c.value
