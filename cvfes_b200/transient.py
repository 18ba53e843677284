"""Time loop and orchestration mirroring ``solver.py``, ``cvfes.py`` and ``main.py``.

``TransientSolverGPU`` keeps the reference loop (``solver.py:99-158``): the time
grid ``t = arange(0, endtime, dt) ∪ {endtime}``, a fluid stand-in that only
records ``t`` (rounded to ``time_rounding`` decimals, 4 in the reference,
``solver.py:117``), ``RefreshContext`` then ``Solve`` per step, and
``saveResNum`` evenly spaced saves.  When no traction file drives the wall, the
steps between two saves run through ``GPUSolidSolver.Advance`` (one CUDA-graph
replay per chunk of steps, no host work in between) with the same per-step
pressures the per-step path would compute.
"""
from __future__ import annotations

import time
from typing import Optional

import numpy as np

from . import cases as _cases
from . import config as _config
from .mesh import SolidMesh
from .solver import FluidSolver, GPUSolidSolver, LocalComm, pressure_at


class TransientSolverGPU:
    def __init__(self, comm, meshes, config, log=print):
        self.comm = comm
        self.rank = comm.Get_rank()
        self.meshes = meshes
        self.saveResNum = config.saveResNum
        self.saveStressFilename = config.saveStressFilename
        self.dt = config.dt
        self.endtime = config.endtime
        self.restartTimestep = config.restartTimestep
        self.time_rounding = getattr(config, "time_rounding", 4)
        self.t = np.append(np.arange(self.endtime, step=self.dt), self.endtime)
        self.nTimeSteps = len(self.t) - 1
        self.config = config
        self.log = log
        self.fluidSolver = FluidSolver(comm, None, config)
        self.solidSolver = GPUSolidSolver(comm, meshes["wall"], config)

    def _fluid_t(self, k):
        t = self.t[k]
        return round(t, self.time_rounding) if self.time_rounding >= 0 else t

    def Solve(self):
        solid = self.solidSolver
        cfg = self.config
        saveSteps = np.linspace(0, self.nTimeSteps, self.saveResNum + 1, dtype=int) \
            if self.saveResNum else np.array([], dtype=int)
        norms_every = getattr(getattr(cfg, "gpu", None), "norms_every", 0)
        start = time.perf_counter()
        k = self.restartTimestep
        fast = solid.stressFilename is None
        while k < self.nTimeSteps:
            stops = [s for s in saveSteps if s > k]
            if norms_every:
                stops.append((k // norms_every + 1) * norms_every)
            end = min([self.nTimeSteps] + stops)
            if fast:
                pres = np.array([pressure_at(self._fluid_t(j), solid.constantPressure,
                                             solid.constant_T, solid.pressure_ramp)
                                 for j in range(k, end)])
                dts = np.diff(self.t[k:end + 1])
                if np.allclose(dts, dts[0], rtol=1e-9, atol=0):
                    solid.Advance(pres, dt=float(dts[0]))
                    solid.pressure = float(pres[-1])
                else:
                    for j in range(k, end):
                        solid.pressure = float(pres[j - k])
                        solid.Solve(self.t[j], self.t[j + 1] - self.t[j])
            else:
                for j in range(k, end):
                    self.fluidSolver.Solve(self._fluid_t(j), self.t[j + 1] - self.t[j])
                    solid.RefreshContext(self.fluidSolver)
                    solid.Solve(self.t[j], self.t[j + 1] - self.t[j])
            k = end
            if norms_every and k % norms_every == 0:
                nrm = solid.Norms()
                if self.rank == 0:
                    self.log("step {:6d}  t={:.5e}  max|u|^2 sum={:.6e}".format(
                        k, self.t[k], float(nrm[:, 0].max())))
            if k in saveSteps and self.saveStressFilename:
                solid.Save(self.saveStressFilename, k)
        solid.comm.Barrier()
        self.wall_ms = (time.perf_counter() - start) * 1e3
        if self.rank == 0:
            self.log("Rank: {}\t{:10.1f} ms".format(self.rank, self.wall_ms))
        return solid


class CVFES:
    """``cvfes.py:26-117`` for the solid wall: read cfg, build the wall, solve."""

    def __init__(self, comm=None, log=print):
        self.comm = comm if comm is not None else LocalComm()
        self.size = self.comm.Get_size()
        self.rank = self.comm.Get_rank()
        self.log = log

    def ReadInputFile(self, filename, nSmp: Optional[int] = None):
        self.cvConfig = _config.load(filename, nSmp)
        cfg = self.cvConfig
        solid = cfg.equations["solid"]
        wall_cfg = cfg.meshes.get("wall")
        path = wall_cfg.file_path if wall_cfg is not None else "synthetic"
        if path == "synthetic" or cfg.synthetic is not None:
            syn = cfg.synthetic
            case = _cases.CASES[syn["case"]] if syn is not None and "case" in syn \
                else _cases.TubeCase("custom", syn.get_int("nc", 64), syn.get_int("na", 128),
                                     syn.get_float("length", 3.0))
            mesh = _cases.build_mesh(case, n_samples=cfg.nSmp)
        else:
            mesh = SolidMesh.from_npz(path, nSmp=cfg.nSmp)
        mesh.density, mesh.v, mesh.damp = solid.density, solid.v, solid.damp
        mesh.bdyU = float(solid.bdyDisplacement)
        self.meshes = {"wall": mesh}
        if self.rank == 0:
            self.log("Model name: {}".format(cfg.name))
            self.log("Structure mesh size: {} elements, {} nodes".format(mesh.nElements, mesh.nNodes))
            self.log("Solver method: {}".format(cfg.solver.method))
            self.log("Number of samples: {}".format(cfg.solver.nSmp))

    def Distribute(self):
        # single rank: the boundary-first renumbering is done by SolidMesh
        return 0 if self.size == 1 else -1

    def Coloring(self):
        return 0

    def Solve(self):
        if self.cvConfig.solver.method not in ("transient GPU", "transient"):
            self.log("Unknown method: {}".format(self.cvConfig.solver.method))
            return None
        self.solver = TransientSolverGPU(self.comm, self.meshes, self.cvConfig.solver, self.log)
        return self.solver.Solve()


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="ensemble membrane wall solver on one B200")
    ap.add_argument("-s", "--samples", type=int, help="Number of samples.")
    ap.add_argument("-f", "--file", default="cfg/tube64x128.cfg", help="Configuration file.")
    a = ap.parse_args(argv)
    cv = CVFES()
    cv.ReadInputFile(a.file, nSmp=a.samples)
    if cv.Distribute() < 0:
        raise SystemExit(-1)
    if cv.Coloring() < 0:
        raise SystemExit(-1)
    start = time.perf_counter()
    cv.Solve()
    print("OK, rank: {} \t\t\t time: {:10.1f} ms".format(cv.rank, (time.perf_counter() - start) * 1e3))
    return 0


if __name__ == "__main__":
    main()
