"""Synthetic wall workloads: structured tubes with seeded GMRF material.

No public dataset exists for this path; every workload is generated.  The
tube sizes, material law and load follow the workload definitions:

``tube64x128``   straight tube r=0.3 cm, L=3 cm, 64 x 128 nodes, 8 samples, dt 2e-6, 400 steps, FP64
``tube256x1024`` same tube refined to 256 x 1024 nodes, 512 samples, dt 5e-7, 2000 steps
``batched64``    64 tubes, r in [0.15,0.6], L in [1,6], nc in {32..256}, na in [64,1024],
                 S in {16..256}, per-tube CFL dt, 1000 steps
``adjoint64``    tube64x128 mesh, 64 samples, 500 steps, 512 observation nodes
``stenosed512x2048`` stenosed tube L=5 cm, 512 x 2048 nodes, 128 samples, 1000 steps
``stenosed256x512``  the same tube at 256 x 512 nodes, 128 samples, 100 steps (profiles)

Material: ``E = 7e6*exp(0.2 z)``, ``h = 0.04*exp(0.1 z')`` with z, z' independent
per-element GMRF samples (:mod:`cvfes_b200.gmrf`); nu = 0.49, rho = 1,
mass-proportional damping 100 1/s; internal pressure ramped linearly to
1.33e5 dyn/cm^2 over the first 100 steps; both end rings clamped.
"""
from __future__ import annotations

import hashlib
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import gmrf as _gmrf
from .mesh import SolidMesh, TubeGeometry, stenosis_radius, tube_mesh, cfl_dt

P_MAX = 1.33e5
RAMP_STEPS = 100


@dataclass
class TubeCase:
    name: str
    nc: int
    na: int
    length: float
    radius: float = 0.3
    stenosed: bool = False
    n_samples: int = 8
    dt: Optional[float] = 2e-6
    n_steps: int = 400
    seed_E: int = 23
    seed_h: int = 24
    E0: float = 7.0e6
    sigma_logE: float = 0.2
    h0: float = 0.04
    sigma_logh: float = 0.1
    nu: float = 0.49
    density: float = 1.0
    damp: float = 100.0
    tau: float = 0.1
    marginal: str = "exact"
    mass_lumping: str = "reference"
    extra: dict = field(default_factory=dict)

    def geometry(self) -> TubeGeometry:
        rfn = (lambda x: stenosis_radius(x, r0=self.radius)) if self.stenosed else None
        return TubeGeometry(self.nc, self.na, self.length, self.radius, rfn)

    def pressures(self, n_steps: Optional[int] = None) -> np.ndarray:
        n = self.n_steps if n_steps is None else n_steps
        return P_MAX * np.minimum(np.arange(n, dtype=np.float64) / RAMP_STEPS, 1.0)


CASES = {
    "tube64x128": TubeCase("tube64x128", 64, 128, 3.0, n_samples=8, dt=2e-6, n_steps=400),
    # dt = 5e-7 exceeds the stability limit of the reference's lumped mass on this mesh
    # (power iteration: dt_crit 3.8e-7 .. 4.3e-7 over the 512 samples); with row-sum
    # lumping (3x that mass) dt_crit is 6.6e-7 .. 7.4e-7 and the step is stable.
    "tube256x1024": TubeCase("tube256x1024", 256, 1024, 3.0, n_samples=512, dt=5e-7,
                             n_steps=2000, mass_lumping="rowsum"),
    # half-length refinement used for kernel profiles: 1.2 GB of state, still 10x L2
    "tube256x512": TubeCase("tube256x512", 256, 512, 1.5, n_samples=256, dt=5e-7, n_steps=1000,
                            mass_lumping="rowsum"),
    "adjoint64": TubeCase("adjoint64", 64, 128, 3.0, n_samples=64, dt=2e-6, n_steps=500,
                          extra=dict(n_obs=512, obs_every=10, ckpt_every=50)),
    # the stenosed adjoint at half the resolution each way and a tenth of the steps, for
    # kernel profiles of the reverse step: 0.2 GB per state (1.6x L2), 2 checkpoint pairs
    "stenosed256x512": TubeCase("stenosed256x512", 256, 512, 5.0, stenosed=True,
                                n_samples=128, dt=None, n_steps=100,
                                extra=dict(n_obs=1024, obs_every=10, ckpt_every=50,
                                           grad_logh=True)),
    "stenosed512x2048": TubeCase("stenosed512x2048", 512, 2048, 5.0, stenosed=True,
                                 n_samples=128, dt=None, n_steps=1000,
                                 extra=dict(n_obs=4096, obs_every=10, ckpt_every=100,
                                            grad_logh=True)),
}


def _cache_dir() -> str:
    d = os.environ.get("CVFES_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cvfes_b200"))
    os.makedirs(d, exist_ok=True)
    return d


def build_mesh(case: TubeCase, n_samples: Optional[int] = None, cache: bool = True) -> SolidMesh:
    """Generate the tube, its boundary rings and GMRF material (cached on disk)."""
    S = case.n_samples if n_samples is None else n_samples
    nodes, elems, inlet, outlet = tube_mesh(case.geometry())
    key = hashlib.sha1(repr((case.nc, case.na, case.length, case.radius, case.stenosed, S,
                             case.seed_E, case.seed_h, case.E0, case.sigma_logE, case.h0,
                             case.sigma_logh, case.tau, case.marginal)).encode()).hexdigest()[:16]
    path = os.path.join(_cache_dir(), f"{case.name}_{S}_{key}.npz")
    if cache and os.path.exists(path):
        d = np.load(path)
        elmE, elmH = d["elmE"], d["elmThick"]
    else:
        elmE, elmH, _ = _gmrf.material_fields(elems, len(nodes), S, case.seed_E, case.seed_h,
                                              case.E0, case.sigma_logE, case.h0, case.sigma_logh,
                                              case.tau, case.marginal)
        if cache:
            np.savez(path, elmE=elmE, elmThick=elmH)
    return SolidMesh(nodes=nodes, elementNodeIds=elems, boundary=np.concatenate([inlet, outlet]),
                     nSmp=S, density=case.density, v=case.nu, damp=case.damp, bdyU=0.0,
                     elmE=elmE, elmThick=elmH, name=case.name, mass_lumping=case.mass_lumping)


def case_dt(case: TubeCase, mesh: SolidMesh) -> float:
    """The case's dt, or the CFL rule 0.5*h_min/sqrt(E_max/rho) when it has none."""
    if case.dt is not None:
        return case.dt
    return cfl_dt(mesh.nodes, mesh.elementNodeIds, float(np.max(mesh.elmE)), case.density)


def _build_material(args):
    """Worker of :func:`build_meshes`: the GMRF material of one case (cached on disk)."""
    import dataclasses
    case_dict, threads = args
    os.environ["OMP_NUM_THREADS"] = str(threads)
    m = build_mesh(TubeCase(**case_dict))
    return m.elmE, m.elmThick


def build_meshes(cases, processes: Optional[int] = None):
    """Build many tube meshes, generating their GMRF material in parallel processes.

    The pool uses the ``spawn`` start method, so it is safe to call after CUDA has
    been initialised in the parent process.
    """
    import dataclasses
    import multiprocessing as mp
    n = len(cases)
    cores = os.cpu_count() or 1
    procs = max(1, min(n, processes or min(16, cores)))
    threads = max(1, cores // procs)
    todo = [(dataclasses.asdict(c), threads) for c in cases]
    if procs == 1:
        mats = [_build_material(t) for t in todo]
    else:
        with mp.get_context("spawn").Pool(procs) as pool:
            mats = pool.map(_build_material, todo, chunksize=1)
    out = []
    for case, (elmE, elmH) in zip(cases, mats):
        nodes, elems, inlet, outlet = tube_mesh(case.geometry())
        out.append(SolidMesh(nodes=nodes, elementNodeIds=elems,
                             boundary=np.concatenate([inlet, outlet]), nSmp=case.n_samples,
                             density=case.density, v=case.nu, damp=case.damp, bdyU=0.0,
                             elmE=elmE, elmThick=elmH, name=case.name,
                             mass_lumping=case.mass_lumping))
    return out


def batched_cases(n_tubes: int = 64, seed: int = 7):
    """The 64-tube uneven ensemble: random radius, length, resolution and sample count."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_tubes):
        nc = int(rng.choice([32, 64, 128, 256]))
        na = int(rng.integers(64, 1025))
        S = int(rng.choice([16, 32, 64, 128, 256]))
        out.append(TubeCase(f"batch{i:02d}", nc, na, float(rng.uniform(1.0, 6.0)),
                            radius=float(rng.uniform(0.15, 0.6)), n_samples=S, dt=None,
                            n_steps=1000, seed_E=1000 + i, seed_h=2000 + i))
    return out


def adjoint_setup(case: TubeCase, precision: int = 64, device="cuda", n_samples=None,
                  n_steps=None, grad_logh=None, use_graph=True, obs_seed: int = 99,
                  true_seed_offset: int = 500):
    """The mismatch workload of an adjoint case.

    Returns ``(problem, logE, logh, logE_true)``: the :class:`MismatchProblem` with
    observations recorded from a forward run whose log E field comes from a GMRF of a
    different seed (``seed_E + true_seed_offset``), and the (E, S) FP64 starting
    material (the case's own GMRF sample) at which gradients are taken.  Observation
    nodes are a seeded choice of distinct free nodes.
    """
    import dataclasses

    import torch

    from .adjoint import MismatchProblem
    S = case.n_samples if n_samples is None else n_samples
    T = case.n_steps if n_steps is None else n_steps
    mesh = build_mesh(case, n_samples=S)
    true = build_mesh(dataclasses.replace(case, seed_E=case.seed_E + true_seed_offset),
                      n_samples=S)
    dt = case_dt(case, mesh)
    ex = case.extra
    free = np.setdiff1d(np.arange(mesh.nNodes), mesh.boundary)
    rng = np.random.default_rng(obs_seed)
    obs = np.sort(rng.choice(free, size=min(int(ex.get("n_obs", 512)), len(free)), replace=False))
    if grad_logh is None:
        grad_logh = bool(ex.get("grad_logh", False))
    problem = MismatchProblem(mesh, dt, case.pressures(T), obs, obs_every=int(ex.get("obs_every", 10)),
                              ckpt_every=int(ex.get("ckpt_every", 50)), precision=precision,
                              device=device, grad_logh=grad_logh, use_graph=use_graph)
    logE = torch.from_numpy(np.log(mesh.elmE))
    logh = torch.from_numpy(np.log(mesh.elmThick))
    logE_true = torch.from_numpy(np.log(true.elmE))
    problem.set_observations(problem.record_observations(logE_true, logh))
    return problem, logE, logh, logE_true
