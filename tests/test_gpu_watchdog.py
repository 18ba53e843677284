"""Failure paths on the GPU without a fault: a bounded device wait that runs out.

Every mbarrier wait in the step kernels is bounded; when one gives up, the kernel sets
bit 0 of the mesh's status word and returns, and ``cvfes_status_read`` turns that into
``CVFES_ERR_TIMEOUT``.  ``cvfes_set_wait_probe`` makes the fan kernel's stage barrier
wait for an arrival that never comes (no copy is issued, so nothing is in flight when
the wait gives up after a few polls).  The tests check the status, that the probe step
wrote nothing, and that the context still computes the next step exactly; the second
runs the probe through ``Solve`` with the norms fused into the step, whose one call
reads the norms and the status word back together and raises there.
"""
import numpy as np
import pytest
import torch

from cvfes_b200 import _lib
from cvfes_b200._lib import call, ptr
from cvfes_b200.cases import CASES, build_mesh
from cvfes_b200.solver import GPUSolidSolver, LocalComm

pytestmark = pytest.mark.gpu


class Cfg:
    def __init__(self, dt, S, precision, norms_every=0):
        self.dt = dt
        self.nSmp = S
        self.gpu = type("G", (), dict(precision=precision, use_graph=False, graph_chunk=6,
                                      watchdog=True, device=0, norms_every=norms_every))()
        self.pressure_ramp = "linear"


@pytest.mark.parametrize("precision", [32, 64])
def test_bounded_wait_gives_up_and_context_survives(lib, cuda, precision):
    case = CASES["tube64x128"]
    mesh = build_mesh(case, n_samples=128)
    pres = case.pressures(12)
    s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 128, precision))
    ref = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 128, precision))
    s.Advance(pres[:10])
    ref.Advance(pres[:11])
    u0 = s.bufs[s.cur].clone()
    v0 = s.bufs[s.prev].clone()
    scratch = torch.full_like(u0, float("nan"))
    fn = "cvfes_solid_step_f32" if precision == 32 else "cvfes_solid_step_f64"
    st = torch.cuda.current_stream().cuda_stream
    call("cvfes_set_wait_probe", 64)
    try:
        call(fn, _lib.C.byref(s._desc), ptr(s.plan.coef(precision)), ptr(s.plan.invm(precision)),
             ptr(s.bufs[s.cur]), ptr(s.bufs[s.prev]), ptr(scratch), None, None, 0,
             float(pres[10]), None, float(case.dt), float(mesh.damp), st)
        with pytest.raises(_lib.CvfesError) as err:
            s.plan.check_status()
        assert err.value.code == _lib.CVFES_ERR_TIMEOUT
    finally:
        call("cvfes_set_wait_probe", 0)
    # the probe step wrote nothing
    assert torch.isnan(scratch).all()
    assert torch.equal(s.bufs[s.cur], u0) and torch.equal(s.bufs[s.prev], v0)
    # the status word was cleared by the read, and the next normal step is exact
    s.plan.check_status()
    s.pressure = float(pres[10])
    s.Solve(None, case.dt)
    s.plan.check_status()
    assert torch.equal(s.local_displacement(), ref.local_displacement())


@pytest.mark.parametrize("precision", [32, 64])
def test_fused_step_with_read_back_reports_the_wait(lib, cuda, precision):
    case = CASES["tube64x128"]
    mesh = build_mesh(case, n_samples=128)
    pres = case.pressures(12)
    s = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 128, precision, norms_every=1))
    ref = GPUSolidSolver(LocalComm(), mesh, Cfg(case.dt, 128, precision, norms_every=1))
    for n in range(10):
        for x in (s, ref):
            x.pressure = float(pres[n])
            x.Solve(None, case.dt)
    u0 = s.local_displacement().clone()
    count = s.step_count
    s.pressure = float(pres[10])
    call("cvfes_set_wait_probe", 64)
    try:
        with pytest.raises(_lib.CvfesError) as err:
            s.Solve(None, case.dt)
        assert err.value.code == _lib.CVFES_ERR_TIMEOUT
    finally:
        call("cvfes_set_wait_probe", 0)
    # nothing advanced: the step count, the roles and the state are those before the call
    assert s.step_count == count
    assert torch.equal(s.local_displacement(), u0)
    s.plan.check_status()  # cleared by the step call's read
    for x in (s, ref):
        x.pressure = float(pres[10])
        x.Solve(None, case.dt)
    assert torch.equal(s.local_displacement(), ref.local_displacement())
    ns, nr = s.Norms(), ref.Norms()
    assert s._norms_step == s.step_count
    assert np.array_equal(ns, nr)
