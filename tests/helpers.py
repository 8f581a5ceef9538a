"""Device-memory helpers for the GPU tests (torch for allocation, cuda-python
for copies out of library-owned device pointers)."""
from __future__ import annotations

import ctypes

import numpy as np


def torch():
    import torch as t
    return t


def dev(a, dtype=None):
    """numpy -> contiguous CUDA tensor (float32 by default for floats)."""
    t = torch()
    a = np.ascontiguousarray(a)
    if dtype is None:
        dtype = np.int32 if a.dtype.kind in "iu" else np.float32
    return t.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def host(x):
    return x.detach().cpu().numpy()


def par_dev(par):
    """The 208-byte Parameters record in device memory."""
    t = torch()
    b = np.frombuffer(par.to_bytes(), np.uint8).copy()
    return t.from_numpy(b).cuda()


def sync():
    torch().cuda.synchronize()


def copy_from_ptr(ptr: int, n: int, dtype=np.int32) -> np.ndarray:
    """Copies n elements from a raw device address into a numpy array."""
    from cuda.bindings import runtime as rt

    out = np.empty(n, dtype)
    if n == 0:
        return out
    err, = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert int(err) == 0, err
    return out


def zeros(shape, dtype=None):
    t = torch()
    return t.zeros(shape, dtype=dtype or t.float32, device="cuda")


def sorted_state(orc, case):
    """Grid of the case's float positions (oracle, bit-exact) and the five
    state arrays gathered into that order."""
    par = case.par
    g = orc.grid_float(par, case.pospres, par.npb)
    idx = g["part_idx"]
    st = [a[idx].copy() for a in case.arrays()]
    return g, st


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)


def ulp_diff(a, b) -> int:
    """Largest distance in float32 units in the last place."""
    a = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.ascontiguousarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return int(np.abs(a - b).max()) if a.size else 0


def by_id(arrays, nb=None):
    """Reorders state arrays by the original index carried in idep.w."""
    ids = np.asarray(arrays[2])[:, 3].astype(np.int64)
    order = np.argsort(ids, kind="stable")
    return [np.asarray(a)[order] for a in arrays]
