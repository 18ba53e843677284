"""Batched multi-mesh step and the autotuners on the GPU."""
import numpy as np
import pytest
import torch

from cvfes_b200 import _lib
from cvfes_b200.batched import BatchedSolidSolver, fan_item_nodes
from cvfes_b200.cases import TubeCase, build_mesh, case_dt
from cvfes_b200.solver import GPUSolidSolver, LocalComm
from oracle import solid_oracle as so

pytestmark = pytest.mark.gpu


def small_batch():
    """Four uneven tubes: different resolution, radius, length and sample count."""
    cases = [TubeCase("b0", 16, 10, 1.0, radius=0.2, n_samples=16, dt=None, seed_E=1, seed_h=2),
             TubeCase("b1", 32, 24, 2.5, radius=0.45, n_samples=32, dt=None, seed_E=3, seed_h=4),
             TubeCase("b2", 12, 40, 4.0, radius=0.3, n_samples=64, dt=None, seed_E=5, seed_h=6),
             TubeCase("b3", 24, 8, 1.5, radius=0.6, n_samples=128, dt=None, seed_E=7, seed_h=8)]
    meshes = [build_mesh(c) for c in cases]
    dts = [case_dt(c, m) for c, m in zip(cases, meshes)]
    return cases, meshes, dts


class _Cfg:
    def __init__(self, dt, S, precision):
        self.dt = dt
        self.nSmp = S
        self.gpu = type("G", (), dict(precision=precision, use_graph=False, graph_chunk=48,
                                      watchdog=True, device=0))()
        self.pressure_ramp = "linear"


@pytest.mark.parametrize("precision", [32, 64])
@pytest.mark.parametrize("variant,grouped,concurrent", [(0, True, True), (1, True, True),
                                                        (1, True, False), (1, False, True)])
def test_batch_equals_meshes_advanced_alone(lib, cuda, precision, variant, grouped, concurrent):
    """Row-gather (0) and fan (1) batch kernels, meshes of 16..128 samples (several nodes
    per warp in the fan layout), one launch per item shape or one for all, the groups'
    graph chunks on streams of their own or one after another: the bits of each mesh
    advanced alone."""
    cases, meshes, dts = small_batch()
    pres = 1.33e5 * np.minimum(np.arange(100) / 100.0, 1.0)
    batch = BatchedSolidSolver(meshes, dts, precision=precision, device=cuda, graph_chunk=24,
                               variant=variant, grouped=grouped, concurrent=concurrent)
    assert batch.variant == variant
    shapes = {fan_item_nodes(m.nSmp, batch.vec) for m in meshes}
    assert len(batch.groups) == (len(shapes) if grouped else 1)
    batch.Advance(pres[:37], use_graph=True)     # graph chunks + plain remainder
    batch.Advance(pres[37:100], use_graph=True)  # starts at a non-zero rotation
    saved = _lib.get_step_tuning(precision)
    try:
        _lib.set_step_tuning(precision, 4 if precision == 32 else 2, 8, 0, 1)  # L1 kernel
        for m, (mesh, dt) in enumerate(zip(meshes, dts)):
            s = GPUSolidSolver(LocalComm(), mesh, _Cfg(dt, mesh.nSmp, precision))
            for p in pres:
                s.pressure = float(p)
                s.Solve(None, dt)
            assert torch.equal(s.local_displacement(), batch.solvers[m].local_displacement()), m
    finally:
        _lib.set_step_tuning(precision, **saved)
    for nrm in batch.Norms():
        assert np.all(nrm[:, 3] == 0)


def test_batch_fp64_against_oracle(lib, cuda):
    cases, meshes, dts = small_batch()
    pres = 1.33e5 * np.minimum(np.arange(60) / 100.0, 1.0)
    batch = BatchedSolidSolver(meshes, dts, precision=64, device=cuda, graph_chunk=12)
    batch.Advance(pres)
    for m, (mesh, dt) in enumerate(zip(meshes, dts)):
        coefK, gthick = mesh.element_coefficients()
        o = so.OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick,
                                 mesh.density, mesh.v, mesh.damp, dt, backend="numpy")
        o.run(pres)
        assert so.rel_l2(batch.displacement(m), o.u) < 1e-12


def test_batch_tuner_restores_state_and_keeps_results(lib, cuda, tmp_path, monkeypatch):
    from cvfes_b200.tune import tune_batch
    monkeypatch.setenv("CVFES_CACHE", str(tmp_path))
    cases, meshes, dts = small_batch()
    pres = 1.33e5 * np.minimum(np.arange(90) / 100.0, 1.0)
    ref = BatchedSolidSolver(meshes, dts, precision=32, device=cuda, graph_chunk=12)
    ref.Advance(pres)
    tuned = BatchedSolidSolver(meshes, dts, precision=32, device=cuda, graph_chunk=12)
    best = tune_batch(tuned, steps=12)
    assert not best["cached"] and len(best["tried"]) >= 2
    tuned.Advance(pres)
    for m in range(len(meshes)):
        assert torch.equal(ref.solvers[m].local_displacement(),
                           tuned.solvers[m].local_displacement())
    again = tune_batch(BatchedSolidSolver(meshes, dts, precision=32, device=cuda), steps=12)
    assert again["cached"] and again["vec"] == best["vec"] and again["grid"] == best["grid"]


def test_step_tuner_picks_a_variant(lib, cuda, tmp_path, monkeypatch):
    from cvfes_b200.cases import CASES
    from cvfes_b200.tune import tune_step
    monkeypatch.setenv("CVFES_CACHE", str(tmp_path))
    case = CASES["tube64x128"]
    mesh = build_mesh(case, n_samples=128)
    s = GPUSolidSolver(LocalComm(), mesh, _Cfg(case.dt, 128, 32))
    saved, saved_pf = _lib.get_step_tuning(32), _lib.get_step_prefetch(32)
    try:
        before = s.local_displacement().clone()
        best = tune_step(s, steps=24)
        assert torch.equal(before, s.local_displacement())
        assert best["ms_per_step"] > 0 and _lib.get_step_tuning(32)["staged"] == best["staged"]
        assert _lib.get_step_prefetch(32) == best["prefetch"]
    finally:
        _lib.set_step_tuning(32, **saved)
        _lib.set_step_prefetch(32, **saved_pf)
