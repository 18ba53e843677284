"""Drop-in GPU solid solver with the reference's class interface.

``GPUSolidSolver(comm, mesh, config)`` keeps the constructor and methods of the
reference class (``physicsSolverSDampGPUs.py:45-496``; identical API in
``physicsSolverGPUs.py:45-490``): ``RefreshContext(physicSolver)``,
``Solve(t, dt)``, ``Save(filename, counter)``, ``ApplyBoundaryCondition``,
``SyncCommNodes`` and ``UnionDisplacement``.  It is constructed the same way by
``TransientSolverGPU`` (``solver.py:148-158``).

Differences by design:
* device memory is owned by torch tensors; every kernel is a libcvfes_b200
  entry point (no OpenCL, no CPU fallback: without a CUDA device the
  constructor raises);
* the Dirichlet rows, the damping and the optional nodal traction are applied
  on the device inside the step kernel, so a step makes no host round trip
  (the reference copies the boundary rows to the host and back every step,
  ``physicsSolverSDampGPUs.py:363-390``);
* the stiffness is the linear template form ``K_s = sum_e (E h)_{e,s} Kt_e``
  assembled once on the undeformed wall (stiffness update interval 0, the
  default), or, with ``stiffness_update_interval`` n >= 1, rebuilt matrix-free with
  the follower pressure on ``x + u`` every n steps (n = 1: ``assemble_K_P``);
* FP64 (default) or FP32 state, chosen by ``[gpu] precision``;
* the second state buffer holds u_{n-1} as in the reference, or (``[gpu] state``
  velocity, the default for the FP32 state) the increment v_n = u_n - u_{n-1},
  updated in place, so the FP32 rounding of u is not fed back into the velocity;
* the numerics are those of the reference's CPU SolidSolver (``[gpu] semantics`` cpu,
  the default) or of the OpenCL class this one replaces (opencl): stiffness
  coefficient mean(E h) over the element's nodes, its lumping of nodal thickness,
  damping force -damp (u - u_prev)/dt per dof with LM on the left-hand side, no
  damping in the start-up acceleration, stiffness and follower pressure rebuilt on
  x + u every step (``physicsSolverSDampGPUs.py:160-175, 325-399``,
  ``physicsSolverSDampGPUs.cl:174-223, 398-429``).
"""
from __future__ import annotations

import math
import os
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .plan import SolidPlan


class LocalComm:
    """Single-rank stand-in for an MPI communicator (mpi4py is not a dependency)."""

    def Get_size(self):
        return 1

    def Get_rank(self):
        return 0

    def Barrier(self):
        return None


class PhysicsSolver:
    """Protocol base of the physics step (``physicsSolver.py:53-84``)."""

    Dof = 3

    def __init__(self, comm, mesh, config):
        self.comm = comm
        self.size = comm.Get_size()
        self.rank = comm.Get_rank()
        self.mesh = mesh
        self.Dof = mesh.dof if mesh is not None else 3
        self.dt = config.dt

    def RefreshContext(self, physicSolver):
        pass

    def Solve(self, t, dt):
        pass

    def Save(self, filename, counter):
        pass

    def Steady(self):
        return False


class FluidSolver(PhysicsSolver):
    """Time source for the solid (``physicsSolver.py:87-99``): records ``t``."""

    def __init__(self, comm, mesh, config):
        PhysicsSolver.__init__(self, comm, mesh, config)
        self.t = 0.0

    def Solve(self, t, dt):
        self.t = t


def pressure_at(t: float, P: float, T: float, ramp: str) -> float:
    """Load schedule of ``RefreshContext`` (physicsSolverSDampGPUs.py:317-322) or a linear ramp."""
    if t > T:
        return P
    if ramp == "linear":
        return P * t / T
    return P / 2.0 - P / 2.0 * math.cos(math.pi / T * t)


class GPUSolidSolver(PhysicsSolver):
    """Ensemble membrane solid on one B200 (see module docstring)."""

    def __init__(self, comm, mesh, config):
        PhysicsSolver.__init__(self, comm, mesh, config)
        gpu = getattr(config, "gpu", None)
        self.precision = getattr(gpu, "precision", 64)
        self.use_graph = getattr(gpu, "use_graph", True)
        self.graph_chunk = getattr(gpu, "graph_chunk", 48)
        self.watchdog = getattr(gpu, "watchdog", True)
        # norms_every = k > 0: every k-th template step computes the FP64 per-sample norms
        # of its new state in the same kernel pass (Norms() then returns them)
        self.norms_every = int(getattr(gpu, "norms_every", 0) or 0)
        # stiffness_update_interval (cvconfig.py:154): 0 keeps the undeformed stiffness and
        # load (linear templates); n >= 1 rebuilds both on x + u every n steps
        self.update_interval = int(getattr(config, "update_interval", 0) or 0)
        # semantics: cpu (SolidSolver's numerics) or opencl (the numerics of the OpenCL class
        # physicsSolverSDampGPUs.py, which rebuilds the stiffness and the follower pressure
        # on x + u every step, so its stiffness update interval is 1)
        self.semantics = str(getattr(gpu, "semantics", "cpu") or "cpu").lower()
        if self.semantics not in ("cpu", "opencl"):
            raise ValueError("semantics must be cpu or opencl")
        if self.semantics == "opencl":
            self.update_interval = 1
        self.state_form = resolve_state_form(getattr(gpu, "state", "auto"), self.precision,
                                             self.update_interval)
        self.InitializeSync()
        if self.InitializeGPU(getattr(gpu, "device", -1)) < 0:
            raise RuntimeError("GPUSolidSolver: no usable CUDA device")

        self.dt_f = getattr(config, "dt_f", 0.01)
        self.stressFilename = getattr(config, "exportBdyStressFilename", None)
        self.useConstantStress = getattr(config, "useConstantStress", False)
        self.constant_T = getattr(config, "constant_T", 1.0)
        self.constantPressure = getattr(config, "constant_pressure", 0.0)
        self.pressure_ramp = getattr(config, "pressure_ramp", "cosine")
        self.nt = 0
        if self.stressFilename is not None:
            if self.useConstantStress:
                self.etrac = np.load("{}.npy".format(self.stressFilename))
            else:
                self.strac = np.load("{}{}.npy".format(self.stressFilename, self.nt))
                self.etrac = np.load("{}{}.npy".format(self.stressFilename, self.nt + 1))
        else:
            self.etrac = None
        self.pressure = 0.0

        self.nSmp = config.nSmp
        self.ndof = mesh.ndof
        self.nNodes = mesh.nNodes
        self.nElms = mesh.nElements
        self.lclNNodes = mesh.lclNNodes
        self.lclNodeIds = mesh.lclNodeIds
        self.lclElmNodeIds = mesh.lclElmNodeIds
        self.lclNDof = self.lclNNodes * mesh.dof
        self.lclNCommNodes = mesh.lclNCommNodes
        self.lclNCommDof = self.lclNCommNodes * mesh.dof
        self.lclNSpecialHeadDof = mesh.lclNSpecialHead * mesh.dof
        self.lclBoundary = mesh.lclBoundary
        self.damp = mesh.damp
        self.dofs = (3 * self.lclNodeIds[:, None] + np.arange(3)[None, :]).ravel()
        self.du = np.asarray(mesh.iniDu)[self.dofs]
        self.u = np.asarray(mesh.iniU)[self.dofs]
        self.InitializeSolver()

    # ------------------------------------------------------------------ set-up
    def InitializeGPU(self, device: int = -1) -> int:
        """Pick the CUDA device of this rank (``physicsSolverSDampGPUs.py:107-131``)."""
        if not torch.cuda.is_available():
            return -1
        n = torch.cuda.device_count()
        if n < self.size:
            print("GPUs is not enough! Actual size: {}, need: {}".format(n, self.size))
            return -1
        idx = device if device >= 0 else int(os.environ.get("LOCAL_RANK", self.rank)) % n
        self.device = torch.device("cuda", idx)
        _lib.load()
        return 0

    def InitializeSync(self):
        self.bdyDofs = (3 * np.asarray(self.mesh.lclBoundary)[:, None] + np.arange(3)).ravel()
        if self.size > 1:
            raise NotImplementedError("GPUSolidSolver runs one mesh on one GPU; mesh partitioning "
                                      "over ranks is outside this package")

    def InitializeSolver(self):
        """Templates, lumped mass, load and the Taylor start ``u_{-1}``
        (``physicsSolverSDampGPUs.py:143-277``, ``physicsSolver.py:209-230``)."""
        m = self.mesh
        dev = self.device
        with torch.cuda.device(dev):
            opencl = self.semantics == "opencl"
            lumping = "opencl" if opencl else getattr(m, "mass_lumping", "reference")
            self.plan = SolidPlan(m.nodes[self.lclNodeIds], self.lclElmNodeIds,
                                  n_clamped=m.lclNSpecialHead, clamp_value=m.bdyU, v=m.v,
                                  density=m.density, device=dev, precisions=(self.precision,),
                                  mass_lumping=lumping)
            coefK, gthick = m.opencl_coefficients() if opencl else m.element_coefficients()
            self.plan.set_material(coefK, gthick)
            self.refresh_desc()
            dtype = torch.float64 if self.precision == 64 else torch.float32
            S, ndof = self.nSmp, self.lclNDof
            self.bufs = [torch.zeros((ndof, S), dtype=dtype, device=dev) for _ in range(3)]
            self.cur, self.prev, self.nxt = 0, 1, 2
            u0 = torch.from_numpy(np.repeat(self.u[:, None], S, axis=1)).to(dev, dtype)
            du0 = torch.from_numpy(np.repeat(self.du[:, None], S, axis=1)).to(dev, dtype)
            self.bufs[self.cur].copy_(u0)
            work = torch.empty_like(u0)
            fn = "cvfes_solid_init_f64" if self.precision == 64 else "cvfes_solid_init_f32"
            call(fn, C_desc(self._desc), ptr(self.plan.coef(self.precision)),
                 ptr(self.plan.invm(self.precision)), ptr(u0), ptr(du0),
                 ptr(self.bufs[self.prev]), ptr(work), float(self.pressure), float(self.dt),
                 float(self.damp), self._stream())
            del work, u0, du0
            self.trac_dev = None
            self.clock = torch.zeros(1, dtype=torch.int64, device=dev)
            self.norm_work = torch.empty(
                int(_lib.load().cvfes_norms_work_size(self.lclNNodes, S)), dtype=torch.float64,
                device=dev)
            self._graphs = {}
            self._p_buf = None
            self._norm_out = None
            self._norm_host = None  # pinned copy of the fused norms, read with the step
            self._norms_step = -1  # step_count at which the norms were fused into a step
            self.step_count = 0
            self.geo_counter = 0
            self.geo_live = False
            self.slot_geo = self.ugeo = None
            if self.update_interval > 0:
                gdt = torch.float64 if self.precision == 64 else torch.float32
                self.slot_geo = torch.empty(8 * 3 * self.plan.E, dtype=gdt, device=dev)
                g64 = self.slot_geo if self.precision == 64 else None
                g32 = self.slot_geo if self.precision == 32 else None
                call("cvfes_solid_slot_geometry_f64", self.plan.E, ptr(self.plan.nodes),
                     ptr(self.plan.elems), ptr(self.plan.slot_rec), ptr(g64), ptr(g32),
                     self._stream())
                self.ugeo = torch.zeros((ndof, S), dtype=dtype, device=dev)

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def refresh_desc(self):
        """Rebuild the C mesh descriptor from the plan (after the plan's tiling or set-up
        arrays change), with this solver's state form."""
        self._desc = self.plan.desc(self.precision)
        self._desc.state_form = 1 if self.state_form == "velocity" else 0
        self._desc.damping_form = 1 if self.semantics == "opencl" else 0
        return self._desc

    # ------------------------------------------------------------------ per step
    def RefreshContext(self, physicSolver):
        """Load at time ``physicSolver.t`` (``physicsSolverSDampGPUs.py:280-322``)."""
        t = physicSolver.t
        ramp_T = self.constant_T
        if self.stressFilename is not None:
            if self.useConstantStress:
                if t > ramp_T:
                    appTrac = self.etrac
                else:
                    appTrac = self.etrac / 2.0 - self.etrac / 2.0 * math.cos(math.pi / ramp_T * t)
            else:
                if t > ramp_T:
                    if int((t - ramp_T) / self.dt_f) > self.nt:
                        self.nt += 1
                        self.strac = self.etrac
                        self.etrac = np.load("{}{}.npy".format(self.stressFilename, self.nt + 1))
                    appTrac = self.strac + (t - ramp_T - self.nt * self.dt_f) * \
                        (self.etrac - self.strac) / self.dt_f
                else:
                    appTrac = self.strac / 2.0 - self.strac / 2.0 * math.cos(math.pi / ramp_T * t)
            self.set_traction(appTrac)
        self.pressure = pressure_at(t, self.constantPressure, self.constant_T, self.pressure_ramp)

    def set_traction(self, appTrac):
        """Nodal traction (N,3) in global node order; boundary rows are zeroed."""
        tr = np.zeros((self.lclNNodes, 4))
        tr[:, :3] = np.asarray(appTrac, dtype=np.float64).reshape(-1, 3)[self.lclNodeIds]
        tr[self.lclBoundary, :] = 0.0
        dtype = torch.float64 if self.precision == 64 else torch.float32
        self.trac_dev = torch.from_numpy(tr).to(self.device, dtype)

    def _solve_geo(self, dt):
        """One step on the deformed geometry with the reference's update counter
        (``physicsSolver.py:296-324``; every step for interval 1, as assemble_K_P), with
        the nodal traction when a traction series drives the wall (calc_u_appTrac)."""
        if self.geo_counter >= self.update_interval:
            if self.update_interval == 1:
                self.geo_live = True
            else:
                self.ugeo.copy_(self.bufs[self.cur])
            self.geo_counter = 1
        else:
            self.geo_counter += 1
        ug = self.bufs[self.cur] if self.geo_live else self.ugeo
        fn = "cvfes_solid_step_geo_f64" if self.precision == 64 else "cvfes_solid_step_geo_f32"
        call(fn, C_desc(self._desc), ptr(self.plan.coef(self.precision)),
             ptr(self.plan.invm(self.precision)), ptr(self.slot_geo), ptr(self.bufs[self.cur]),
             ptr(self.bufs[self.prev]), ptr(self.bufs[self.nxt]), ptr(ug), None, None, 0,
             float(self.pressure), ptr(self.trac_dev), float(self.mesh.v), float(dt),
             float(self.damp), self._stream())

    def Solve(self, t, dt):
        """One explicit step for all samples (``physicsSolverSDampGPUs.py:325-399``)."""
        if self.update_interval > 0:
            with torch.cuda.device(self.device):
                self._solve_geo(dt)
            self.prev, self.cur, self.nxt = self.cur, self.nxt, self.prev
            self.step_count += 1
            return
        fn = "cvfes_solid_step_f64" if self.precision == 64 else "cvfes_solid_step_f32"
        fused = self.norms_every > 0 and (self.step_count + 1) % self.norms_every == 0
        args = [C_desc(self._desc), ptr(self.plan.coef(self.precision)),
                ptr(self.plan.invm(self.precision)), ptr(self.bufs[self.cur]),
                ptr(self.bufs[self.prev]), ptr(self.bufs[self.nxt]), None, None, 0,
                float(self.pressure), ptr(self.trac_dev), float(dt), float(self.damp)]
        with torch.cuda.device(self.device):
            if fused:
                if self._norm_out is None:
                    self._norm_out = torch.empty((self.nSmp, 4), dtype=torch.float64,
                                                 device=self.device)
                if self._norm_host is None:
                    self._norm_host = torch.empty((self.nSmp, 4), dtype=torch.float64,
                                                  pin_memory=True)
                # the call returns with the norms in _norm_host and the status word of
                # the bounded waits read and cleared (one stream synchronisation)
                call(fn.replace("step_", "step_norms_"), *args, ptr(self.norm_work),
                     ptr(self._norm_out), ptr(self._norm_host), 0, self._stream())
            else:
                call(fn, *args, self._stream())
        self._rotate()
        self.step_count += 1
        if fused:
            self._norms_step = self.step_count

    def _rotate(self):
        """Buffer roles after one template step: (u_n, u_{n-1}, free) <- (u_{n+1}, u_n,
        u_{n-1}); in the velocity-state form the increment stays where it is and the two
        displacement buffers swap."""
        if self.state_form == "velocity":
            self.cur, self.nxt = self.nxt, self.cur
        else:
            self.prev, self.cur, self.nxt = self.cur, self.nxt, self.prev

    def Advance(self, pressures, dt: Optional[float] = None, use_graph: Optional[bool] = None):
        """Many steps with a per-step pressure schedule, no host work between steps.

        With ``use_graph`` the steps run as replays of one captured CUDA graph of
        ``graph_chunk`` steps (a multiple of 3; in the velocity-state form the least
        common multiple of it and 2); the remainder runs as plain launches.

        With a nodal traction set (``RefreshContext`` of a traction series), the
        traction is held for the whole call: the steps run as single launches with the
        schedule's pressures, and ``RefreshContext`` is not re-run between them.
        """
        dt = self.dt if dt is None else dt
        use_graph = self.use_graph if use_graph is None else use_graph
        p = self._schedule(pressures)
        n = int(p.numel())
        prec = self.precision
        if self.update_interval > 0:
            if self.trac_dev is not None:  # per-step launches with the held traction
                ph = p.cpu().numpy()
                for j in range(n):
                    self.pressure = float(ph[j])
                    self.Solve(None, dt)
                return self
            return self._advance_geo(p, n, dt)
        with torch.cuda.device(self.device):
            self.clock.zero_()
            done = 0
            chunk = self.graph_chunk
            if self.state_form == "velocity" and chunk % 2:
                chunk *= 2
            if use_graph and self.trac_dev is None and n >= chunk:
                key = (chunk, float(dt), self.cur, self.prev, self.nxt, p.data_ptr())
                g = self._graphs.get(key)
                if g is None:
                    h = _lib.C.c_void_p()
                    b = self.bufs
                    call("cvfes_graph_capture_advance", C_desc(self._desc), prec,
                         ptr(self.plan.coef(prec)), ptr(self.plan.invm(prec)),
                         ptr(b[self.cur]), ptr(b[self.prev]), ptr(b[self.nxt]), ptr(p),
                         ptr(self.clock), chunk, float(dt), float(self.damp), self._stream(),
                         _lib.C.byref(h))
                    g = h.value
                    self._graphs[key] = (g,)
                else:
                    g = g[0]
                while n - done >= chunk:
                    call("cvfes_graph_launch", g, self._stream())
                    done += chunk
            self.step_count += done
            if n - done > 0:
                cur_idx = _lib.C.c_int32()
                prev_idx = _lib.C.c_int32()
                if self.trac_dev is not None:  # Solve counts its own steps
                    ph = p.cpu().numpy()
                    for j in range(done, n):
                        self.pressure = float(ph[j])
                        self.Solve(None, dt)
                else:
                    fn = "cvfes_solid_advance_f64" if prec == 64 else "cvfes_solid_advance_f32"
                    b = self.bufs
                    order = [self.cur, self.prev, self.nxt]
                    call(fn, C_desc(self._desc), ptr(self.plan.coef(prec)),
                         ptr(self.plan.invm(prec)), ptr(b[order[0]]), ptr(b[order[1]]),
                         ptr(b[order[2]]), ptr(p), ptr(self.clock), n - done, float(dt),
                         float(self.damp), _lib.C.byref(cur_idx), _lib.C.byref(prev_idx),
                         self._stream())
                    self.cur, self.prev = order[cur_idx.value], order[prev_idx.value]
                    self.nxt = 3 - self.cur - self.prev
                    self.step_count += n - done
        return self

    def _advance_geo(self, p, n, dt):
        """Geometric steps as plain launches (the geometry update counter is host state)."""
        fn = "cvfes_solid_advance_geo_f64" if self.precision == 64 else \
            "cvfes_solid_advance_geo_f32"
        b = self.bufs
        order = [self.cur, self.prev, self.nxt]
        cur_idx, prev_idx, live = _lib.C.c_int32(), _lib.C.c_int32(), _lib.C.c_int32()
        counter = _lib.C.c_int64(self.geo_counter)
        with torch.cuda.device(self.device):
            self.clock.zero_()
            call(fn, C_desc(self._desc), ptr(self.plan.coef(self.precision)),
                 ptr(self.plan.invm(self.precision)), ptr(self.slot_geo), ptr(b[order[0]]),
                 ptr(b[order[1]]), ptr(b[order[2]]), ptr(self.ugeo), ptr(p), ptr(self.clock), n,
                 self.update_interval, _lib.C.byref(counter), int(self.geo_live),
                 float(self.mesh.v), float(dt), float(self.damp), _lib.C.byref(cur_idx),
                 _lib.C.byref(prev_idx), _lib.C.byref(live), self._stream())
        self.cur, self.prev = order[cur_idx.value], order[prev_idx.value]
        self.nxt = 3 - self.cur - self.prev
        self.geo_counter = counter.value
        self.geo_live = bool(live.value)
        self.step_count += n
        return self

    def _schedule(self, pressures) -> torch.Tensor:
        """Pressure schedule copied into a persistent device buffer: its address never
        changes, so a captured graph (which reads ``p[clock + j]``) stays valid."""
        if isinstance(pressures, torch.Tensor):
            src = pressures.to(self.device, torch.float64).reshape(-1)
        else:
            src = torch.from_numpy(np.ascontiguousarray(pressures, dtype=np.float64).ravel())
        n = int(src.numel())
        if self._p_buf is None or self._p_buf.numel() < n:
            self.release_graphs()
            self._p_buf = torch.empty(max(n, 4096), dtype=torch.float64, device=self.device)
        view = self._p_buf[:n]
        view.copy_(src, non_blocking=True)
        return view

    def release_graphs(self):
        for g in self._graphs.values():
            call("cvfes_graph_destroy", g[0])
        self._graphs.clear()

    def __del__(self):
        try:
            self.release_graphs()
        except Exception:
            pass

    # ------------------------------------------------------------------ outputs
    def Norms(self, check_finite: Optional[bool] = None,
              out: Optional[torch.Tensor] = None) -> np.ndarray:
        """FP64 per-sample (sum u^2, sum du^2, sum m du^2, #non-finite), shape (S, 4).

        ``out``: an (S, 4) FP64 host tensor (pinned, for an asynchronous copy) that
        receives the result; the call returns once it has arrived."""
        chk = self.watchdog if check_finite is None else check_finite
        fresh = self._norms_step == self.step_count  # fused into the last step
        if fresh:  # already on the host, status checked by the step call
            if out is None:
                res = self._norm_host.clone()
            else:
                out.copy_(self._norm_host)
                res = out
        else:
            if self._norm_out is None:
                self._norm_out = torch.empty((self.nSmp, 4), dtype=torch.float64,
                                             device=self.device)
            dev_out = self._norm_out
            fn = "cvfes_solid_norms_f64" if self.precision == 64 else "cvfes_solid_norms_f32"
            if self.state_form == "velocity":
                fn = fn.replace("norms_", "norms_vel_")
            with torch.cuda.device(self.device):
                call(fn, self.lclNNodes, self.nSmp, ptr(self.bufs[self.cur]),
                     ptr(self.bufs[self.prev]), ptr(self.plan.invm(self.precision)),
                     ptr(self.norm_work), ptr(dev_out), int(bool(chk)), self._stream())
                if out is None:
                    res = dev_out.cpu()
                else:
                    out.copy_(dev_out, non_blocking=True)
                    res = out
                self.plan.check_status()
        res = res.numpy()
        if fresh and chk and np.any(res[:, 3] != 0):
            raise _lib.NonFiniteError(_lib.CVFES_ERR_NONFINITE,
                                      "watchdog: %.0f non-finite state values" % res[:, 3].sum())
        return res

    def LambdaMax(self, iters: int = 200, seed: int = 0) -> np.ndarray:
        """Largest eigenvalue of M⁻¹K per sample on the free dofs (FP64 power iteration
        with the template K*u kernel); the central-difference step is stable for
        ``dt < 2/sqrt(lambda_max)``."""
        dev = self.device
        plan = self.plan
        if plan.slot_k64 is None or plan.coef64 is None:
            raise RuntimeError("LambdaMax needs the FP64 templates (precision = fp64)")
        desc = plan.desc(64)
        g = torch.Generator(device=dev)
        g.manual_seed(seed)
        with torch.cuda.device(dev):
            x = torch.randn((self.lclNDof, self.nSmp), dtype=torch.float64, device=dev,
                            generator=g)
            nc = 3 * plan.n_clamped
            x[:nc] = 0
            y = torch.empty_like(x)
            invm3 = plan.invm64.repeat_interleave(3, dim=0)
            lam = torch.zeros(self.nSmp, dtype=torch.float64, device=dev)
            for _ in range(iters):
                x /= torch.linalg.vector_norm(x, dim=0, keepdim=True)
                call("cvfes_solid_kmul_f64", C_desc(desc), ptr(plan.coef64), ptr(x), ptr(y), 0,
                     self._stream())
                y *= invm3
                y[:nc] = 0
                lam = torch.linalg.vector_norm(y, dim=0)
                x, y = y, x
        return lam.cpu().numpy()

    def local_displacement(self) -> torch.Tensor:
        """Current displacement (lclNDof, S) on the device, local node order."""
        return self.bufs[self.cur]

    def displacement(self) -> np.ndarray:
        """Current displacement (ndof, S) as FP64 numpy in global node order."""
        return self.UnionDisplacement(self.bufs[self.cur].double().cpu().numpy())

    def ApplyBoundaryCondition(self, quant):
        """Host-side Dirichlet rows (``physicsSolver.py:327-328``); the step kernel
        applies the same rows on the device."""
        quant[self.bdyDofs, :] = self.mesh.bdyU

    def SyncCommNodes(self, quant):
        """Shared-node sum over ranks; a single GPU owns every node, so nothing to do."""
        return None

    def UnionDisplacement(self, quant):
        resU = np.empty((self.ndof, self.nSmp))
        resU[self.dofs, :] = quant
        return resU

    def Stress(self) -> torch.Tensor:
        """Element stresses (E, S, 5: xx, yy, xy, xz, yz) of the current state on the
        geometry of the last stiffness update (``physicsSolver.py:416-424``)."""
        dev = self.device
        with torch.cuda.device(dev):
            if getattr(self, "_young", None) is None:
                self._young = torch.from_numpy(self.mesh.element_moduli()).to(dev)
            dtype = torch.float64 if self.precision == 64 else torch.float32
            out = torch.empty((self.nElms, self.nSmp, 5), dtype=dtype, device=dev)
            ug = None
            if self.update_interval > 0 and self.geo_counter > 0:
                # the geometry of the last update: u at the start of the last step when it
                # is refreshed every step, else the copy taken at the update
                ug = self.bufs[self.prev] if self.geo_live else self.ugeo
            fn = "cvfes_solid_stress_f64" if self.precision == 64 else "cvfes_solid_stress_f32"
            call(fn, self.nElms, self.nSmp, ptr(self.plan.nodes), ptr(self.plan.elems),
                 ptr(self._young), ptr(self.bufs[self.cur]), ptr(ug), float(self.mesh.v),
                 ptr(out), self._stream())
        return out

    def Save(self, filename, counter):
        """Displacement and element stresses of every sample at this step
        (``physicsSolver.py:383-397``; ``physicsSolverSDampGPUs.py:452-464``)."""
        resU = self.displacement()
        stress = self.Stress().double().cpu().numpy()
        if self.rank == 0:
            from .io import save_displacement
            save_displacement(filename, counter, self.mesh,
                              resU.T.reshape(self.nSmp, self.mesh.nNodes, self.Dof),
                              stress=stress)
        self.comm.Barrier()


def resolve_state_form(state: str, precision: int, update_interval: int) -> str:
    """``[gpu] state``: ``auto`` is the velocity-state form for the FP32 state of the
    template step and the previous-displacement form otherwise (FP64 state, or the
    geometric mode, whose kernels keep the reference's pair of displacements)."""
    state = (state or "auto").lower()
    if state not in ("auto", "previous", "velocity"):
        raise ValueError("state must be auto, previous or velocity")
    if state == "velocity" and update_interval > 0:
        raise ValueError("the velocity-state form is for the template step "
                         "(stiffness_update_interval 0)")
    if state == "auto":
        return "velocity" if precision == 32 and update_interval == 0 else "previous"
    return state


def C_desc(desc):
    return _lib.C.byref(desc)
