"""Many independent wall meshes advanced together on one GPU.

Each mesh keeps its own ``GPUSolidSolver`` (plan, material, three state buffers,
start-up state), so its sample count, time step and damping are its own.  The
batch packs one descriptor per mesh into a device table and advances the meshes
with persistent kernel launches (``cvfes_batch_step``), captured in CUDA graphs of
``graph_chunk`` steps.  Two kernels: the fan kernel (``variant`` 1, the default:
slot rows staged by TMA, fan-rotation gathers) and the row-gather kernel
(``variant`` 0).  A mesh advanced in a batch is bitwise identical to the same mesh
advanced alone by the single-mesh kernels.

Meshes are packed in groups of one work-item shape (nodes per fan item, which the
sample count sets), one table and one launch per group and step.  The fan kernel's
shared-memory stage is sized for the largest item of its launch, and shared memory
comes out of the same on-chip storage as L1: in one launch over the whole uneven
ensemble the 16-sample tubes' 16-node items set the stage size for everyone, and the
many-sample tubes (most of the bytes) run with little L1 for their neighbour
gathers.  Measured on the 64-tube ensemble (FP32, fan kernel): 14.8 ms/step in one
launch, 11.0 ms as per-shape launches.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .solver import GPUSolidSolver, LocalComm


class _Cfg:
    def __init__(self, dt, nSmp, precision, device, state="auto"):
        self.dt = dt
        self.nSmp = nSmp
        self.gpu = type("G", (), dict(precision=precision, use_graph=False, graph_chunk=48,
                                      watchdog=True, device=device, state=state))()
        self.pressure_ramp = "linear"


def sm_count(device) -> int:
    return torch.cuda.get_device_properties(device).multi_processor_count


def fan_item_nodes(S: int, vec: int) -> int:
    """Nodes per warp of a fan work item (the batch kernel's rule): a warp holds
    32 // min(32, S / vec) nodes of S / vec lanes each."""
    sv = max(1, S // vec)
    return 32 // min(32, sv)


class _Group:
    """Meshes of one fan-item shape: their table, counts, clock and graphs."""

    def __init__(self, idx, device, n_bytes):
        self.idx = list(idx)
        self.totals = (_lib.C.c_int64 * 3)()
        self.clock = torch.zeros(1, dtype=torch.int64, device=device)
        self.table = torch.empty(n_bytes, dtype=torch.uint8, device=device)
        self.graphs = {}


class BatchedSolidSolver:
    """A batch of ``SolidMesh`` ensembles with per-mesh time steps ``dts``.

    ``grouped`` (default) launches each fan-item shape separately; ``False`` puts
    every mesh in one table and one launch per step."""

    def __init__(self, meshes: Sequence, dts: Sequence[float], precision: int = 32,
                 device="cuda:0", vec: Optional[int] = None, grid: int = 0,
                 graph_chunk: int = 48, max_steps: int = 8192, variant: int = 1,
                 grouped: bool = True, state: str = "auto", concurrent: bool = False):
        if len(meshes) != len(dts) or not meshes:
            raise ValueError("one dt per mesh")
        if graph_chunk % 6:
            raise ValueError("graph_chunk must be a multiple of 6")
        self.device = torch.device(device)
        self.precision = precision
        idx = self.device.index or 0
        self.solvers: List[GPUSolidSolver] = [
            GPUSolidSolver(LocalComm(), m, _Cfg(float(dt), m.nSmp, precision, idx, state))
            for m, dt in zip(meshes, dts)]
        self.state_form = self.solvers[0].state_form
        self.dts = [float(d) for d in dts]
        maxv = 4 if precision == 32 else 2
        if vec is None:
            vec = maxv
            while vec > 1 and any(s.nSmp % vec for s in self.solvers):
                vec //= 2
        self.vec = vec
        self.grid = grid
        self.variant = variant
        self.grouped = grouped
        # concurrent: graph chunks of the groups on streams of their own (the meshes are
        # independent).  Off by default: measured 13.6 against 11.2 ms per step of the
        # 64-tube ensemble one group after another, as the groups' persistent launches
        # then share the SMs and L2 for their whole length, not only at their tails.
        self.concurrent = concurrent
        self._group_streams: List[torch.cuda.Stream] = []
        self.totals = (_lib.C.c_int64 * 3)()
        self.graph_chunk = graph_chunk
        self.rot = 0
        self.steps = 0
        self._p = torch.zeros(max_steps, dtype=torch.float64, device=self.device)
        self.groups: List[_Group] = []
        self._pack()

    # ------------------------------------------------------------------ packing
    def _pack(self):
        self.release_graphs()
        keys = [fan_item_nodes(s.nSmp, self.vec) if self.grouped else 0 for s in self.solvers]
        lib = _lib.load()
        self.groups = []
        for k in sorted(set(keys)):
            members = [i for i, kk in enumerate(keys) if kk == k]
            g = _Group(members, self.device, int(lib.cvfes_batch_table_bytes(len(members))))
            items = (_lib.BatchItem * len(members))()
            for j, i in enumerate(members):
                s = self.solvers[i]
                it = items[j]
                it.mesh = s._desc
                it.coef = ptr(s.plan.coef(self.precision))
                it.invm = ptr(s.plan.invm(self.precision))
                for q in range(3):
                    it.buf[q] = ptr(s.bufs[q])
                it.p_sched = ptr(self._p)
                it.dt = self.dts[i]
                it.damp = float(s.damp)
            with torch.cuda.device(self.device):
                call("cvfes_batch_pack", items, len(members), self.precision, self.vec,
                     ptr(g.table), g.totals)
            self.groups.append(g)
        # batch-wide counts: items of either kernel, and the largest fan stage (-1 when
        # some mesh has no max_degree, so the fan kernel cannot be used)
        self.totals[0] = sum(g.totals[0] for g in self.groups)
        self.totals[1] = sum(g.totals[1] for g in self.groups)
        caps = [g.totals[2] for g in self.groups]
        self.totals[2] = -1 if min(caps) <= 0 else max(caps)
        if self.variant == 1 and self.totals[2] <= 0:
            self.variant = 0  # a mesh without max_degree: the fan stage cannot be sized
        self.n_meshes = len(self.solvers)

    def set_launch(self, vec: Optional[int] = None, grid: Optional[int] = None,
                   variant: Optional[int] = None):
        """Change the tile shape (samples per thread), the persistent grid size or the
        kernel (0 row gather, 1 fan)."""
        if variant is not None and variant != self.variant:
            if variant == 1 and self.totals[2] <= 0:
                raise ValueError("the fan kernel needs every mesh's max_degree")
            self.variant = variant
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
        for g in self.groups:
            call("cvfes_batch_advance", ptr(g.table), len(g.idx), g.totals, self.precision,
                 self.vec, self.variant, self.rot, ptr(g.clock), n, self.grid,
                 _lib.C.byref(rot_out), self._stream())
        self.rot = rot_out.value

    def Advance(self, pressures, use_graph: bool = True):
        """Advance every mesh by len(pressures) steps with the shared pressure schedule.

        Each graph chunk (or plain run) takes one group through the same steps, with its
        own device clock indexing the shared schedule.  With ``concurrent`` the groups'
        graph chunks run on streams of their own, joined to the caller's stream before
        the call returns; otherwise one group's chunk after another on the caller's
        stream.  Either way every mesh takes its own steps in order."""
        p = np.ascontiguousarray(pressures, dtype=np.float64).ravel()
        n = p.size
        if n > self._p.numel():
            self._p = torch.zeros(n, dtype=torch.float64, device=self.device)
            self._pack()
        with torch.cuda.device(self.device):
            self._p[:n].copy_(torch.from_numpy(p), non_blocking=False)
            for g in self.groups:
                g.clock.zero_()
            done = 0
            chunk = self.graph_chunk
            if use_graph and n >= chunk + 5:
                lead = (6 - self.rot) % 6  # plain steps until the rotation is back at 0
                if lead:
                    self._plain(lead)
                    done += lead
                graphs = [self._graph(g, chunk) for g in self.groups]
                n_chunks = (n - done) // chunk
                if self.concurrent and len(graphs) > 1:
                    self._launch_concurrent(graphs, n_chunks)
                else:
                    for _ in range(n_chunks):
                        for h in graphs:
                            call("cvfes_graph_launch", h, self._stream())
                done += n_chunks * chunk
            if n - done:
                self._plain(n - done)
        self.steps += n
        self.sync_roles()
        return self

    def _launch_concurrent(self, graphs, n_chunks):
        """n_chunks replays of each group's graph on the group's own stream, after the
        caller's stream's work so far, and the caller's stream waits for all of them."""
        main = torch.cuda.current_stream(self.device)
        while len(self._group_streams) < len(graphs):
            self._group_streams.append(torch.cuda.Stream(device=self.device))
        start = torch.cuda.Event()
        start.record(main)
        for h, st in zip(graphs, self._group_streams):
            st.wait_event(start)
            for _ in range(n_chunks):
                call("cvfes_graph_launch", h, st.cuda_stream)
            end = torch.cuda.Event()
            end.record(st)
            main.wait_event(end)

    def sync_roles(self):
        """Set each mesh solver's buffer roles from the batch's rotation phase
        (``rot`` = steps taken mod 6; the rule of ``cvfes_batch_step``)."""
        for s in self.solvers:
            if s.state_form == "velocity":
                s.cur, s.prev = (2 if self.rot & 1 else 0), 1
                s.nxt = 2 - s.cur
            else:
                cur = (3 - self.rot % 3) % 3
                s.cur, s.prev, s.nxt = cur, (cur + 1) % 3, (cur + 2) % 3
            s.step_count = self.steps

    def _graph(self, g: _Group, chunk):
        key = (chunk, self.vec, self.grid, self.variant)
        h = g.graphs.get(key)
        if h is None:
            out = _lib.C.c_void_p()
            call("cvfes_batch_graph_capture", ptr(g.table), len(g.idx), g.totals,
                 self.precision, self.vec, self.variant, ptr(g.clock), chunk, self.grid,
                 _lib.C.byref(out))
            h = g.graphs[key] = out.value
        return h

    def release_graphs(self):
        for st in getattr(self, "_group_streams", []):
            st.synchronize()  # no graph is destroyed while its replays may still run
        for g in getattr(self, "groups", []):
            for h in g.graphs.values():
                call("cvfes_graph_destroy", h)
            g.graphs.clear()

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
        """Bytes one batched step must move (sum of the per-mesh step formula; the
        velocity-state form reads and writes the increment as well: 13N per sample)."""
        b = 4 if self.precision == 32 else 8
        tot = 0
        for s in self.solvers:
            N, E, S = s.lclNNodes, s.nElms, s.nSmp
            state = 13 * N if s.state_form == "velocity" else 10 * N
            tot += S * b * (state + E) + E * (12 + 45 * b) + 3 * N * b
        return tot

    def sample_count(self) -> int:
        return sum(s.nSmp for s in self.solvers)
