"""Adjoint gradients of a displacement-mismatch objective (inverse wall-stiffness estimation).

For an ensemble of S material samples on one wall mesh, the objective of sample s is

    J_s = sum_{n = k*obs_every <= T} sum_{i in obs} |u_n(i) - uobs_n(i)|^2

over the displacement history of the explicit solid step (zero start, per-step
pressure schedule).  :class:`MismatchProblem` runs the forward pass on the GPU
(the same sm_100a step kernels as the solver, saving the state pair every
``ckpt_every`` steps) and the hand-written discrete adjoint (``cvfes_adjoint_*``:
the reverse recursion fused with the forward step run backwards, restarted from the
saved pairs), and returns dJ_s/dlogE_{e,s} and dJ_s/dlogh_{e,s} per element and
sample.  :func:`wall_mismatch` puts it behind a ``torch.autograd.Function``.

The reference has no differentiation; the forward model is its solid step
(``physicsSolver.py:263-292`` with the material of ``physicsSolver.py:199-202``,
``E*h`` per element and ``h`` at every quadrature point).
"""
from __future__ import annotations

from typing import Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .plan import SolidPlan, lumped_mass_weights


class MismatchProblem:
    """Forward model, objective and adjoint of one mesh with S samples.

    ``obs_nodes`` are node ids of ``mesh`` (global numbering), distinct.  Step
    ``n`` (0-based) uses ``pressures[n]``; observations are taken after steps
    ``obs_every, 2*obs_every, ... <= T``.  ``grad_logh`` also accumulates the
    mass term needed for dJ/dlogh (thickness enters the stiffness and the mass).
    """

    def __init__(self, mesh, dt: float, pressures: Sequence[float], obs_nodes,
                 obs_every: int = 10, ckpt_every: int = 50, precision: int = 64,
                 device="cuda", grad_logh: bool = False, use_graph: bool = True):
        if precision not in (32, 64):
            raise ValueError("precision must be 32 or 64")
        self.device = dev = torch.device(device)
        if dev.type != "cuda":
            raise RuntimeError("MismatchProblem needs a CUDA device; there is no CPU path")
        self.mesh = mesh
        self.precision = precision
        self.dtype = torch.float64 if precision == 64 else torch.float32
        self.dt = float(dt)
        self.damp = float(mesh.damp)
        p = np.ascontiguousarray(pressures, dtype=np.float64).ravel()
        self.T = T = int(p.size)
        self.obs_every = int(obs_every)
        self.ckpt_every = int(ckpt_every)
        if T <= 0 or self.obs_every <= 0 or self.ckpt_every <= 0:
            raise ValueError("need steps > 0 and positive observation / checkpoint intervals")
        self.S = S = int(mesh.nSmp)
        self.N = N = int(mesh.nNodes)
        self.E = E = int(mesh.nElements)
        obs = np.asarray(obs_nodes, dtype=np.int64).ravel()
        if len(np.unique(obs)) != len(obs) or (len(obs) and (obs.min() < 0 or obs.max() >= N)):
            raise ValueError("observation nodes must be distinct node ids of the mesh")
        self.obs_nodes_global = obs
        g2l = np.empty(N, dtype=np.int64)
        g2l[mesh.lclNodeIds] = np.arange(N)
        self.g2l = g2l
        self.grad_logh = bool(grad_logh)
        self.use_graph = use_graph
        lump = getattr(mesh, "mass_lumping", "reference")
        self.mass_weights = np.ascontiguousarray(lumped_mass_weights(mesh.density, lump))
        with torch.cuda.device(dev):
            self.plan = plan = SolidPlan(mesh.nodes[mesh.lclNodeIds], mesh.lclElmNodeIds,
                                         n_clamped=mesh.lclNSpecialHead, clamp_value=mesh.bdyU,
                                         v=mesh.v, density=mesh.density, device=dev,
                                         precisions=(precision,), mass_lumping=lump)
            coefK, gthick = mesh.element_coefficients()
            plan.set_material(coefK, gthick)
            self._mesh_desc = plan.desc(precision)
            dt_ = self.dtype
            z = lambda *shape, dtype=dt_: torch.zeros(shape, dtype=dtype, device=dev)
            self.own = z(3 * E * 28)  # per slot; the owner slot of each element holds its blocks
            call("cvfes_adjoint_owner_blocks", self._mesh_desc, precision, ptr(plan.elems),
                 ptr(plan.elem_slot), ptr(self.own), self._stream())
            self.logE = z(E, S, dtype=torch.float64)
            self.logh = z(E, S, dtype=torch.float64)
            self.thick = z(E, S, dtype=torch.float64)
            self.state = [z(3 * N, S) for _ in range(3)]
            self.adj = [z(3 * N, S) for _ in range(2)]
            n_ck = int(_lib.load().cvfes_adjoint_ckpt_count(T, self.ckpt_every))
            self.ckpt = z(n_ck, 2, 3 * N, S)
            self.p_sched = torch.from_numpy(p).to(dev)
            self.clock = z(1, dtype=torch.int64)
            self.n_obs = len(obs)
            self.n_obs_steps = T // self.obs_every
            self.obs_nodes = torch.from_numpy(g2l[obs].astype(np.int32)).to(dev)
            self.obs = z(max(self.n_obs_steps, 1), max(self.n_obs, 1), 3, S)
            nj = int(_lib.load().cvfes_adjoint_jpart_size(T, self.obs_every, self.n_obs, S))
            self.jpart = z(max(nj, 1), dtype=torch.float64)
            self.J = z(S, dtype=torch.float64)
            self.gamma = z(E, S)
            self.gmass = z(N, S) if self.grad_logh else None
            self.gE = z(E, S, dtype=torch.float64)
            self.gh = z(E, S, dtype=torch.float64) if self.grad_logh else None
        self._desc = self._make_desc(record=0)
        self._desc_rec = self._make_desc(record=1)
        self._graphs = {}
        self._final = None     # (cur, prev) roles after the last forward pass
        self._token = 0        # bumps with every forward pass

    # ------------------------------------------------------------------ plumbing
    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _make_desc(self, record: int) -> _lib.AdjointDesc:
        d = _lib.AdjointDesc()
        d.mesh = self._mesh_desc
        d.precision = self.precision
        d.record = record
        d.coef = ptr(self.plan.coef(self.precision))
        d.invm = ptr(self.plan.invm(self.precision))
        d.owner_blocks = ptr(self.own)
        for q in range(3):
            d.state[q] = ptr(self.state[q])
        for q in range(2):
            d.adj[q] = ptr(self.adj[q])
        d.ckpt = ptr(self.ckpt)
        d.p_sched = ptr(self.p_sched)
        d.clock = ptr(self.clock)
        d.n_steps = self.T
        d.ckpt_every = self.ckpt_every
        d.n_obs = self.n_obs
        d.obs_every = self.obs_every
        d.obs_nodes = ptr(self.obs_nodes)
        d.obs = ptr(self.obs)
        d.jpart = ptr(self.jpart)
        d.J = ptr(self.J)
        d.gamma = ptr(self.gamma)
        d.gmass = ptr(self.gmass)
        d.dt = self.dt
        d.damp = self.damp
        return d

    def set_material(self, logE: torch.Tensor, logh: torch.Tensor) -> None:
        """Per-element, per-sample log E and log h, (E, S) FP64 (copied to the device)."""
        plan = self.plan
        with torch.cuda.device(self.device):
            self.logE.copy_(torch.as_tensor(logE, dtype=torch.float64).reshape(self.E, self.S))
            self.logh.copy_(torch.as_tensor(logh, dtype=torch.float64).reshape(self.E, self.S))
            call("cvfes_adjoint_material", self.E, self.S, ptr(self.logE), ptr(self.logh),
                 ptr(plan.coef64), ptr(plan.coef32), ptr(self.thick), self._stream())
            call("cvfes_solid_mass_load_f64", plan.N, plan.E, self.S, ptr(plan.node_ptr),
                 ptr(plan.slot_rec), ptr(plan.area), ptr(plan.normal), ptr(self.thick), 1,
                 ptr(self.mass_weights), ptr(plan.lm), ptr(plan.invm64), ptr(plan.invm32),
                 ptr(plan.fhat64), ptr(plan.fhat32), self._stream())

    def _run(self, which: int):
        """Forward (0) or reverse (1) pass, replaying a captured graph when enabled."""
        d = self._desc
        st = self._stream()
        if which == 1 and self._final is None:
            raise RuntimeError("run the forward pass (objective) before the gradient")
        if not self.use_graph:
            if which == 0:
                cur, prev = _lib.C.c_int32(), _lib.C.c_int32()
                call("cvfes_adjoint_forward", _lib.C.byref(d), _lib.C.byref(cur),
                     _lib.C.byref(prev), st)
                self._final = (cur.value, prev.value)
            else:
                call("cvfes_adjoint_reverse", _lib.C.byref(d), self._final[0], self._final[1], st)
            return
        key = (which,) + ((self._final,) if which == 1 else ())
        g = self._graphs.get(key)
        if g is None:
            cur, prev = _lib.C.c_int32(), _lib.C.c_int32()
            h = _lib.C.c_void_p()
            fc, fp = self._final if which == 1 else (0, 0)
            call("cvfes_adjoint_capture", _lib.C.byref(d), which, fc, fp, _lib.C.byref(cur),
                 _lib.C.byref(prev), _lib.C.byref(h))
            g = self._graphs[key] = (h.value, (cur.value, prev.value))
        call("cvfes_graph_launch", g[0], st)
        if which == 0:
            self._final = g[1]

    # ------------------------------------------------------------------ public API
    def record_observations(self, logE, logh) -> torch.Tensor:
        """Run the forward model and return u at the observation nodes and steps,
        ``(T // obs_every, n_obs, 3, S)`` at the problem's precision."""
        self.set_material(logE, logh)
        cur, prev = _lib.C.c_int32(), _lib.C.c_int32()
        with torch.cuda.device(self.device):
            call("cvfes_adjoint_forward", _lib.C.byref(self._desc_rec), _lib.C.byref(cur),
                 _lib.C.byref(prev), self._stream())
        self._final = None
        return self.obs[: self.n_obs_steps, : self.n_obs].clone()

    def set_observations(self, obs) -> None:
        o = torch.as_tensor(obs).to(self.device, self.dtype)
        if tuple(o.shape) != (self.n_obs_steps, self.n_obs, 3, self.S):
            raise ValueError(f"observations must be {(self.n_obs_steps, self.n_obs, 3, self.S)}")
        self.obs[: self.n_obs_steps, : self.n_obs].copy_(o)

    def objective(self, logE, logh) -> torch.Tensor:
        """J per sample (S,) FP64 for this material; keeps the checkpoints for `gradient`."""
        self.set_material(logE, logh)
        with torch.cuda.device(self.device):
            self._run(0)
            self._token += 1
            self.plan.check_status()
            return self.J.clone()

    def gradient(self) -> Tuple[torch.Tensor, Optional[torch.Tensor]]:
        """(dJ/dlogE, dJ/dlogh or None), each (E, S) FP64, for the last `objective` call."""
        plan = self.plan
        with torch.cuda.device(self.device):
            self._run(1)
            call("cvfes_adjoint_gradients", _lib.C.byref(self._desc), ptr(plan.elems),
                 ptr(plan.area), ptr(self.mass_weights), ptr(plan.lm), ptr(self.logE),
                 ptr(self.logh), ptr(self.gE), ptr(self.gh), self._stream())
            return self.gE.clone(), (self.gh.clone() if self.gh is not None else None)

    def final_displacement(self) -> torch.Tensor:
        """u_T after the last forward pass, (3N, S) in local node order."""
        if self._final is None:
            raise RuntimeError("no forward pass yet")
        return self.state[self._final[0]]

    def release_graphs(self):
        for g in self._graphs.values():
            call("cvfes_graph_destroy", g[0])
        self._graphs.clear()

    def __del__(self):
        try:
            self.release_graphs()
        except Exception:
            pass


class _WallMismatch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, logE, logh, problem):
        J = problem.objective(logE.detach(), logh.detach())
        ctx.problem = problem
        ctx.token = problem._token
        ctx.save_for_backward(logE, logh)
        return J

    @staticmethod
    def backward(ctx, gJ):
        problem = ctx.problem
        logE, logh = ctx.saved_tensors
        if problem._token != ctx.token:  # another forward ran since: redo this one
            problem.objective(logE.detach(), logh.detach())
        if ctx.needs_input_grad[1] and not problem.grad_logh:
            raise RuntimeError("build the MismatchProblem with grad_logh=True for dJ/dlogh")
        gE, gh = problem.gradient()
        w = gJ.to(torch.float64).reshape(1, -1)
        # gradients in the inputs' own shape and dtype (set_material accepts any shape
        # that reshapes to (E, S), and autograd wants each gradient like its input)
        outE = (gE * w).reshape(logE.shape).to(logE.dtype) if ctx.needs_input_grad[0] else None
        outh = ((gh * w).reshape(logh.shape).to(logh.dtype)
                if (gh is not None and ctx.needs_input_grad[1]) else None)
        return outE, outh, None


def wall_mismatch(logE: torch.Tensor, logh: torch.Tensor, problem: MismatchProblem) -> torch.Tensor:
    """Per-sample mismatch J (S,) with adjoint gradients for logE and logh (E, S)."""
    return _WallMismatch.apply(logE, logh, problem)
