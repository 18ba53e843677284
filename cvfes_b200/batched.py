"""Many independent wall meshes advanced together on one GPU.

Each mesh keeps its own ``GPUSolidSolver`` (plan, material, three state buffers,
start-up state), so its sample count, time step and damping are its own.  The
batch packs one descriptor per mesh into a device table and advances all meshes
with one persistent kernel launch per step (``cvfes_batch_step``), captured in CUDA
graphs of ``graph_chunk`` steps.  Two kernels: the fan kernel (``variant`` 1, the
default: slot rows staged by TMA, fan-rotation gathers) and the row-gather kernel
(``variant`` 0).  A mesh advanced in a batch is bitwise identical to the same mesh
advanced alone by the single-mesh kernels.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .solver import GPUSolidSolver, LocalComm


class _Cfg:
    def __init__(self, dt, nSmp, precision, device):
        self.dt = dt
        self.nSmp = nSmp
        self.gpu = type("G", (), dict(precision=precision, use_graph=False, graph_chunk=48,
                                      watchdog=True, device=device))()
        self.pressure_ramp = "linear"


def sm_count(device) -> int:
    return torch.cuda.get_device_properties(device).multi_processor_count


class BatchedSolidSolver:
    """A batch of ``SolidMesh`` ensembles with per-mesh time steps ``dts``."""

    def __init__(self, meshes: Sequence, dts: Sequence[float], precision: int = 32,
                 device="cuda:0", vec: Optional[int] = None, grid: int = 0,
                 graph_chunk: int = 48, max_steps: int = 8192, variant: int = 1):
        if len(meshes) != len(dts) or not meshes:
            raise ValueError("one dt per mesh")
        if graph_chunk % 3:
            raise ValueError("graph_chunk must be a multiple of 3")
        self.device = torch.device(device)
        self.precision = precision
        idx = self.device.index or 0
        self.solvers: List[GPUSolidSolver] = [
            GPUSolidSolver(LocalComm(), m, _Cfg(float(dt), m.nSmp, precision, idx))
            for m, dt in zip(meshes, dts)]
        self.dts = [float(d) for d in dts]
        maxv = 4 if precision == 32 else 2
        if vec is None:
            vec = maxv
            while vec > 1 and any(s.nSmp % vec for s in self.solvers):
                vec //= 2
        self.vec = vec
        self.grid = grid
        self.variant = variant
        self.totals = (_lib.C.c_int64 * 3)()
        self.graph_chunk = graph_chunk
        self.rot = 0
        self.steps = 0
        self.clock = torch.zeros(1, dtype=torch.int64, device=self.device)
        self._p = torch.zeros(max_steps, dtype=torch.float64, device=self.device)
        self._graphs = {}
        self.table = torch.empty(int(_lib.load().cvfes_batch_table_bytes(len(self.solvers))),
                                 dtype=torch.uint8, device=self.device)
        self._pack()

    # ------------------------------------------------------------------ packing
    def _pack(self):
        n = len(self.solvers)
        items = (_lib.BatchItem * n)()
        for i, s in enumerate(self.solvers):
            it = items[i]
            it.mesh = s._desc
            it.coef = ptr(s.plan.coef(self.precision))
            it.invm = ptr(s.plan.invm(self.precision))
            for q in range(3):
                it.buf[q] = ptr(s.bufs[q])
            it.p_sched = ptr(self._p)
            it.dt = self.dts[i]
            it.damp = float(s.damp)
        with torch.cuda.device(self.device):
            call("cvfes_batch_pack", items, n, self.precision, self.vec, ptr(self.table),
                 self.totals)
        if self.variant == 1 and self.totals[2] <= 0:
            self.variant = 0  # a mesh without max_degree: the fan stage cannot be sized
        self.total_items = int(self.totals[self.variant])
        self.n_meshes = n
        self.release_graphs()

    def set_launch(self, vec: Optional[int] = None, grid: Optional[int] = None,
                   variant: Optional[int] = None):
        """Change the tile shape (samples per thread), the persistent grid size or the
        kernel (0 row gather, 1 fan)."""
        if variant is not None and variant != self.variant:
            if variant == 1 and self.totals[2] <= 0:
                raise ValueError("the fan kernel needs every mesh's max_degree")
            self.variant = variant
            self.total_items = int(self.totals[variant])
            self.release_graphs()
        if vec is not None and vec != self.vec:
            self.vec = vec
            self._pack()
        if grid is not None and grid != self.grid:
            self.grid = grid
            self.release_graphs()

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    # ------------------------------------------------------------------ stepping
    def _plain(self, n):
        rot_out = _lib.C.c_int32()
        call("cvfes_batch_advance", ptr(self.table), self.n_meshes, self.totals,
             self.precision, self.vec, self.variant, self.rot, ptr(self.clock), n, self.grid,
             _lib.C.byref(rot_out), self._stream())
        self.rot = rot_out.value

    def Advance(self, pressures, use_graph: bool = True):
        """Advance every mesh by len(pressures) steps with the shared pressure schedule."""
        p = np.ascontiguousarray(pressures, dtype=np.float64).ravel()
        n = p.size
        if n > self._p.numel():
            self._p = torch.zeros(n, dtype=torch.float64, device=self.device)
            self._pack()
        with torch.cuda.device(self.device):
            self._p[:n].copy_(torch.from_numpy(p), non_blocking=False)
            self.clock.zero_()
            done = 0
            chunk = self.graph_chunk
            if use_graph and n >= chunk + 2:
                lead = (3 - self.rot) % 3  # plain steps until the rotation is back at 0
                if lead:
                    self._plain(lead)
                    done += lead
                g = self._graph(chunk)
                while n - done >= chunk:
                    call("cvfes_graph_launch", g, self._stream())
                    done += chunk
            if n - done:
                self._plain(n - done)
        self.steps += n
        cur = (3 - self.rot) % 3
        for s in self.solvers:
            s.cur, s.prev, s.nxt = cur, (cur + 1) % 3, (cur + 2) % 3
            s.step_count = self.steps
        return self

    def _graph(self, chunk):
        key = (chunk, self.vec, self.grid, self.variant)
        g = self._graphs.get(key)
        if g is None:
            h = _lib.C.c_void_p()
            call("cvfes_batch_graph_capture", ptr(self.table), self.n_meshes, self.totals,
                 self.precision, self.vec, self.variant, ptr(self.clock), chunk, self.grid,
                 _lib.C.byref(h))
            g = self._graphs[key] = h.value
        return g

    def release_graphs(self):
        for g in self._graphs.values():
            call("cvfes_graph_destroy", g)
        self._graphs.clear()

    def __del__(self):
        try:
            self.release_graphs()
        except Exception:
            pass

    # ------------------------------------------------------------------ outputs
    def displacement(self, m: int) -> np.ndarray:
        return self.solvers[m].displacement()

    def Norms(self, check_finite: Optional[bool] = None) -> List[np.ndarray]:
        return [s.Norms(check_finite) for s in self.solvers]

    def algorithmic_bytes(self) -> int:
        """Bytes one batched step must move (sum of the per-mesh step formula)."""
        b = 4 if self.precision == 32 else 8
        tot = 0
        for s in self.solvers:
            N, E, S = s.lclNNodes, s.nElms, s.nSmp
            tot += S * b * (10 * N + E) + E * (12 + 45 * b) + 3 * N * b
        return tot

    def sample_count(self) -> int:
        return sum(s.nSmp for s in self.solvers)
