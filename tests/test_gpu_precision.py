"""FP32-state forms against the FP64 form at the workloads' full sizes.

The FP64 form matches the oracle to 1e-12 (parity tests, and the full-length fixtures
of ``test_gpu_fixtures.py``); here the FP32 forms, which keep state and element
arithmetic in FP32 (FP64 only in the GMRF, the mass inversion and the norms), are
measured against it at the final step: relative L2 of the displacement.

Two FP32 forms: ``previous`` keeps the reference's pair (u_n, u_{n-1}), whose
difference carries the FP32 rounding of u into the velocity every step; ``velocity``
keeps the increment v_n = u_n - u_{n-1} in its own buffer (the default FP32 form).
The gate, 1e-5, is asserted for the velocity form on every workload; the previous
form's error is printed beside it (run with -s to see the values).
"""
import dataclasses

import pytest
import torch

from cvfes_b200.batched import BatchedSolidSolver
from cvfes_b200.cases import CASES, batched_cases, build_mesh, build_meshes, case_dt
from cvfes_b200.solver import GPUSolidSolver, LocalComm

pytestmark = pytest.mark.gpu
TOL = 1e-5


class Cfg:
    def __init__(self, dt, S, precision, state="auto"):
        self.dt = dt
        self.nSmp = S
        self.gpu = type("G", (), dict(precision=precision, use_graph=True, graph_chunk=48,
                                      watchdog=True, device=0, state=state))()
        self.pressure_ramp = "linear"


def final_state(mesh, dt, pres, precision, state="auto"):
    s = GPUSolidSolver(LocalComm(), mesh, Cfg(dt, mesh.nSmp, precision, state))
    s.Advance(pres)
    out = s.local_displacement().double().clone()
    s.release_graphs()
    return out


def rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def forms_vs_fp64(mesh, dt, pres, label):
    u64 = final_state(mesh, dt, pres, 64)
    assert torch.isfinite(u64).all()
    errs = {st: rel(final_state(mesh, dt, pres, 32, st), u64) for st in ("previous", "velocity")}
    print(f"\n{label}: FP32 vs FP64 rel-L2  previous {errs['previous']:.3e}  "
          f"velocity {errs['velocity']:.3e}")
    return errs


def test_tube256x1024_512_samples_2000_steps(lib, cuda):
    case = CASES["tube256x1024"]
    mesh = build_mesh(case)
    errs = forms_vs_fp64(mesh, case.dt, case.pressures(2000), "tube256x1024, 512 samples, 2000 steps")
    assert errs["velocity"] <= TOL


def test_stenosed_tube_1000_steps(lib, cuda):
    """The stenosed 512x2048 tube (16 of its 128 samples), CFL time step, 1000 steps.

    Its throat elements are the smallest of all workloads (1.5e-3 cm), so neighbour
    displacement differences are the smallest relative to the displacement itself."""
    case = dataclasses.replace(CASES["stenosed512x2048"], n_samples=16)
    mesh = build_mesh(case)
    errs = forms_vs_fp64(mesh, case_dt(case, mesh), case.pressures(1000),
                         "stenosed512x2048, 16 samples, 1000 steps")
    assert errs["velocity"] <= TOL


def test_batched_tubes_1000_steps(lib, cuda):
    """All 64 tubes of the uneven ensemble, each with its own CFL time step."""
    cases = batched_cases(64, seed=7)
    meshes = build_meshes(cases)
    dts = [case_dt(c, m) for c, m in zip(cases, meshes)]
    pres = cases[0].pressures(1000)
    ref, errs = None, {}
    for precision, state in ((64, "previous"), (32, "previous"), (32, "velocity")):
        b = BatchedSolidSolver(meshes, dts, precision=precision, device=cuda, state=state)
        b.Advance(pres)
        if ref is None:
            ref = [s.local_displacement().clone() for s in b.solvers]
            assert all(bool(torch.isfinite(u).all()) for u in ref)
        else:
            errs[state] = [rel(s.local_displacement().double(), r)
                           for s, r in zip(b.solvers, ref)]
        b.release_graphs()
        del b
        torch.cuda.empty_cache()
    for st in ("previous", "velocity"):
        e = errs[st]
        worst = max(range(len(e)), key=lambda i: e[i])
        print(f"\nbatched, 64 tubes, 1000 steps, FP32 {st}: max rel-L2 {e[worst]:.3e} "
              f"(tube {worst}: nc {cases[worst].nc}, na {cases[worst].na}, "
              f"S {cases[worst].n_samples}), median {sorted(e)[len(e) // 2]:.3e}")
    assert max(errs["velocity"]) <= TOL
