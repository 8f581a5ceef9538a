"""The 208-byte ``Parameters`` record (include/types.h) as a ctypes structure.

Field order and types are the reference's ABI (reference include/types.h:89-155);
``PARAMETER_FIELDS`` is that layout, and ``Parameters`` mirrors it so host code
can fill a record and pass it by pointer to the C ABI.
"""
from __future__ import annotations

import ctypes

I, F = ctypes.c_int, ctypes.c_float

PARAMETER_FIELDS = [
    ("np", I), ("npb", I), ("npm", I), ("np_delete", I),
    ("domain_size_x", F), ("domain_size_y", F), ("domain_size_z", F),
    ("domain_min_x", F), ("domain_min_y", F), ("domain_min_z", F),
    ("cell_num_x", I), ("cell_num_y", I), ("cell_num_z", I),
    ("ncell", I), ("ncell_one_layer", I), ("ncell_delete", I),
    ("h", F), ("i_h", F), ("eta", F), ("dr", F), ("hdr", F),
    ("m", F), ("cs", F), ("cfl", F), ("rho0", F),
    ("constitutive_model", I),
    ("model_par_1", F), ("model_par_2", F), ("model_par_3", F), ("model_par_4", F), ("model_par_5", F),
    ("density_shepard_filter", I), ("stress_shepard_filter", I), ("dynamic_time_step", I),
    ("integration_method", I), ("viscosity_type", I),
    ("artificial_viscosity_alpha", F),
    ("artificial_pressure", I), ("artificial_pressure_coefficient", F),
    ("acc_x", F), ("acc_y", F), ("acc_z", F),
    ("time_max", F), ("time", F), ("dt", F), ("output_frequency", F),
    ("output_number", I),
    ("kernel_normalization_par", F), ("kernel_gradient_normalization_par", F),
    ("kernel_zero", F), ("kernel_dr", F),
    ("output_format", I),
]


class Parameters(ctypes.Structure):
    _fields_ = PARAMETER_FIELDS

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in PARAMETER_FIELDS}

    def copy(self) -> "Parameters":
        p = Parameters()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(self), ctypes.sizeof(Parameters))
        return p

    def to_bytes(self) -> bytes:
        return ctypes.string_at(ctypes.byref(self), ctypes.sizeof(Parameters))

    @classmethod
    def from_bytes(cls, b: bytes) -> "Parameters":
        p = cls()
        ctypes.memmove(ctypes.byref(p), b, ctypes.sizeof(cls))
        return p


assert ctypes.sizeof(Parameters) == 208


def dp_cone(phi_deg: float, psi_deg: float = 0.0, cohesion: float = 0.0):
    """Drucker-Prager constants (k_phi, k_psi, k_c) of the cone inscribed for
    compression, 6 sin(phi) / (sqrt(3) (3 + sin(phi))); the reference's example
    k_phi = 0.494872 is phi = 30 deg on this cone (examples/sand_collapse_plane.xml:18)."""
    import math
    s, sp = math.sin(math.radians(phi_deg)), math.sin(math.radians(psi_deg))
    kphi = 6.0 * s / (math.sqrt(3.0) * (3.0 + s))
    kpsi = 6.0 * sp / (math.sqrt(3.0) * (3.0 + sp))
    kc = 6.0 * cohesion * math.cos(math.radians(phi_deg)) / (math.sqrt(3.0) * (3.0 + s))
    return kphi, kpsi, kc


def elastic_moduli(E: float, nu: float):
    """Bulk and shear modulus from Young's modulus and Poisson's ratio."""
    K = E / (3.0 * (1.0 - 2.0 * nu))
    G = E / (2.0 * (1.0 + nu))
    return K, G
