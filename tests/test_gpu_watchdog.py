"""Failure paths on the GPU without a fault: a bounded device wait that runs out.

Every mbarrier wait in the step kernels is bounded; when one gives up, the kernel sets
bit 0 of the mesh's status word and returns, and ``cvfes_status_read`` turns that into
``CVFES_ERR_TIMEOUT``.  ``cvfes_set_wait_probe`` makes the fan kernel's stage barrier
wait for an arrival that never comes (no copy is issued, so nothing is in flight when
the wait gives up after a few polls).  The test checks the status, that the probe step
wrote nothing, and that the context still computes the next step exactly.
"""
import pytest
import torch

from cvfes_b200 import _lib
from cvfes_b200._lib import call, ptr
from cvfes_b200.cases import CASES, build_mesh
from cvfes_b200.solver import GPUSolidSolver, LocalComm

pytestmark = pytest.mark.gpu


class Cfg:
    def __init__(self, dt, S, precision):
        self.dt = dt
        self.nSmp = S
        self.gpu = type("G", (), dict(precision=precision, use_graph=False, graph_chunk=6,
                                      watchdog=True, device=0))()
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
