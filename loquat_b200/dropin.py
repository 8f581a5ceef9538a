"""The reference's time step through the drop-in entry points.

``ReferenceStep`` runs LoquatSph::RunSimulation's hot loop (reference
src/loquat.cu:322-409) exactly as a caller of the reference's headers does:
the reference's array set (state, ``*_ini`` snapshot, rates and the two sort
caches, src/loquat.cu:142-165), a neighbour search followed by
SortArraysPrimary / SortArraysAll (src/loquat.cu:190-213) before each stage,
AdamiBoundary, ParticleInteraction, Predictor / Corrector, and the Shepard
stress filter every ``stress_shepard_filter`` steps after a fresh search.
Each call goes through the C ABI (``lq_grid_*``, ``lq_adami_boundary``,
``lq_particle_interaction``, ``lq_predictor``, ``lq_corrector``,
``lq_stress_regularization``) on one CUDA stream; device memory comes from
torch.  It measures what a reference caller gets, and lets tests check that
sequence against the oracle.

The grid is this library's (``lq_grid_*``), whose searches track each
particle's identity, so ``lq_particle_interaction`` carries its neighbour
lists from call to call while the particles stay within half a skin of
their positions at the lists' build.  ``carry=False`` hands the
interaction copies of the grid's cell bounds instead, which it cannot
match to a grid: it then builds its lists afresh at every call, as it does
for a caller's own grid.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import (Grid, Parameters, adami_boundary, corrector, interaction_reserve, particle_interaction, predictor,
               stress_regularization)


class ReferenceStep:
    def __init__(self, par: Parameters, pospres, velrhop, idep, str_, stn, device="cuda", stream=None,
                 carry: bool = True):
        import torch

        self.torch = torch
        self.par = par.copy()
        self.par.dt = self.par.cfl * self.par.h / self.par.cs   # src/loquat.cu:329
        n = self.np = par.np
        dev = torch.device(device)
        self.stream = stream if stream is not None else torch.cuda.current_stream(dev)
        self._s = self.stream.cuda_stream

        def f4():
            return torch.zeros((n, 4), dtype=torch.float32, device=dev)

        def t2():
            return torch.zeros((n, 6), dtype=torch.float32, device=dev)

        host = [np.ascontiguousarray(a, np.float32) for a in (pospres, velrhop, idep, str_, stn)]
        self.state = [torch.from_numpy(a).to(dev) for a in host]
        self.ini = [f4(), f4(), f4(), t2(), t2()]
        self.rates = [f4(), f4(), t2()]
        self.f4_cache, self.t2_cache = f4(), t2()
        self.par_dev = torch.empty(ctypes.sizeof(Parameters), dtype=torch.uint8, device=dev)
        self.grid = Grid(n, par.ncell)
        interaction_reserve(self.par)    # set-up allocation, as LoquatGrid::GridConfig makes it
        self.carry = carry
        if not carry:
            self._beg = torch.empty(par.ncell, dtype=torch.int32, device=dev)
            self._end = torch.empty(par.ncell, dtype=torch.int32, device=dev)
        self.step_count = 0
        self.time = 0.0

    def close(self):
        if getattr(self, "grid", None) is not None:
            self.grid.close()
            self.grid = None

    __del__ = close

    def _upload_parameters(self):
        # the host record is copied to the device once per step (src/loquat.cu:337)
        buf = np.frombuffer(self.par.to_bytes(), dtype=np.uint8)
        src = self.torch.from_numpy(buf.copy()).pin_memory()
        with self.torch.cuda.stream(self.stream):
            self.par_dev.copy_(src, non_blocking=True)

    def _search_sort(self, arrays):
        s, g, n = self._s, self.grid, self.np
        g.neighbor_search(self.par, self.par_dev, self.state[0], self.state[2], stream=s)
        for a in arrays:
            if a.shape[1] == 4:
                g.sort_float4(n, a, self.f4_cache, stream=s)
            else:
                g.sort_tensor2d(n, a, self.t2_cache, stream=s)

    def _cells(self):
        a = self.grid.arrays()
        if self.carry:
            return a["cell_beg"], a["cell_end"]
        # copies of the grid's bounds, at addresses the library does not know
        from cuda.bindings import runtime as rt

        nbytes = 4 * self.par.ncell
        kind = rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice
        for dst, src in ((self._beg, a["cell_beg"]), (self._end, a["cell_end"])):
            err, = rt.cudaMemcpyAsync(dst.data_ptr(), src, nbytes, kind, self._s)
            if int(err) != 0:
                raise RuntimeError(f"cell bounds copy failed: {err}")
        return self._beg, self._end

    def step(self, nsteps: int = 1):
        s = self._s
        ph, pd = self.par, self.par_dev
        st, ini, rt = self.state, self.ini, self.rates
        for _ in range(nsteps):
            ph.time = float(np.float32(self.time))
            self._upload_parameters()
            # predictor stage (src/loquat.cu:343-368)
            self._search_sort(st)
            beg, end = self._cells()
            adami_boundary(ph, pd, st[0], st[1], st[3], beg, end, stream=s)
            particle_interaction(ph, pd, *st, *rt, beg, end, stream=s)
            predictor(ph, pd, st, ini, rt, stream=s)
            # corrector stage (src/loquat.cu:371-396)
            self._search_sort(st + ini)
            beg, end = self._cells()
            adami_boundary(ph, pd, st[0], st[1], st[3], beg, end, stream=s)
            particle_interaction(ph, pd, *st, *rt, beg, end, stream=s)
            corrector(ph, pd, st, ini, rt, stream=s)
            # stress regularisation (src/loquat.cu:400-409)
            N = ph.stress_shepard_filter
            if N != 0 and self.step_count % N == 0 and self.step_count != 0:
                self._search_sort(st)
                beg, end = self._cells()
                stress_regularization(ph, pd, st[0], st[1], st[3], self.t2_cache, beg, end, stream=s)
            self.time += float(ph.dt)
            self.step_count += 1

    def download(self):
        self.stream.synchronize()
        return [a.cpu().numpy() for a in self.state]
