"""Adjoint gradients of the mismatch objective on the GPU.

Checked against FP64 torch autograd of the reference's step (``oracle/adjoint_oracle``)
and against central finite differences of the FP64 forward model.
"""
import dataclasses

import numpy as np
import pytest
import torch

from cvfes_b200.adjoint import MismatchProblem, wall_mismatch
from cvfes_b200.cases import CASES, TubeCase, adjoint_setup
from oracle import adjoint_oracle as ao

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = torch.as_tensor(a, dtype=torch.float64).cpu()
    b = torch.as_tensor(b, dtype=torch.float64).cpu()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


SMALL = TubeCase("adjsmall", 16, 12, 1.5, radius=0.3, n_samples=8, dt=None, n_steps=70,
                 seed_E=11, seed_h=12, extra=dict(n_obs=24, obs_every=10, ckpt_every=25))


def torch_reference(problem, logE, logh, device, segment_len=0):
    m = problem.mesh
    tw = ao.TorchWall(m.nodes, m.elementNodeIds, m.boundary, m.density, m.v, m.damp, problem.dt,
                      mass_lumping=getattr(m, "mass_lumping", "reference"), device=device)
    obs = problem.obs[: problem.n_obs_steps, : problem.n_obs].to(torch.float64)
    return ao.autograd_gradients(tw, logE.to(device), logh.to(device),
                                 problem.p_sched.cpu().numpy(), problem.obs_nodes_global, obs,
                                 problem.obs_every, segment_len=segment_len)


@pytest.mark.parametrize("precision,tol_J,tol_g", [(64, 1e-12, 1e-9), (32, 1e-5, 1e-4)])
def test_small_tube_against_torch_autograd(lib, cuda, precision, tol_J, tol_g):
    problem, logE, logh, _ = adjoint_setup(SMALL, precision=precision, device=cuda,
                                           grad_logh=True)
    J = problem.objective(logE, logh)
    gE, gh = problem.gradient()
    Jr, gEr, ghr = torch_reference(problem, logE, logh, cuda)
    assert rel(J, Jr) < tol_J
    assert rel(gE, gEr) < tol_g, rel(gE, gEr)
    assert rel(gh, ghr) < tol_g, rel(gh, ghr)


def test_graph_and_plain_passes_agree_bitwise(lib, cuda):
    pg, logE, logh, _ = adjoint_setup(SMALL, precision=32, device=cuda, grad_logh=True)
    pp, _, _, _ = adjoint_setup(SMALL, precision=32, device=cuda, grad_logh=True,
                                use_graph=False)
    for _ in range(2):  # the second round replays the cached graphs
        Jg, Jp = pg.objective(logE, logh), pp.objective(logE, logh)
        (gEg, ghg), (gEp, ghp) = pg.gradient(), pp.gradient()
        assert torch.equal(Jg, Jp) and torch.equal(gEg, gEp) and torch.equal(ghg, ghp)


def test_autograd_function(lib, cuda):
    problem, logE, logh, _ = adjoint_setup(SMALL, precision=64, device=cuda, grad_logh=True)
    lE = logE.clone().to(cuda).requires_grad_(True)
    lh = logh.clone().to(cuda).requires_grad_(True)
    w = torch.linspace(0.5, 1.5, problem.S, dtype=torch.float64, device=cuda)
    J = wall_mismatch(lE, lh, problem)
    problem.objective(logE + 0.01, logh)  # another forward in between: backward redoes its own
    (J * w).sum().backward()
    J2 = problem.objective(logE, logh)
    gE, gh = problem.gradient()
    assert torch.equal(J.detach(), J2)
    assert torch.allclose(lE.grad, gE * w[None, :], rtol=1e-14, atol=0)
    assert torch.allclose(lh.grad, gh * w[None, :], rtol=1e-14, atol=0)


def test_partial_last_segment_and_unobserved_end(lib, cuda):
    """T not a multiple of the checkpoint or observation interval."""
    case = dataclasses.replace(SMALL, n_steps=67, extra=dict(n_obs=24, obs_every=10,
                                                              ckpt_every=20))
    for precision, tol in ((64, 1e-9), (32, 1e-4)):
        problem, logE, logh, _ = adjoint_setup(case, precision=precision, device=cuda,
                                               grad_logh=True)
        problem.objective(logE, logh)
        gE, gh = problem.gradient()
        _, gEr, ghr = torch_reference(problem, logE, logh, cuda)
        assert rel(gE, gEr) < tol and rel(gh, ghr) < tol


def c3_problem(precision, cuda, **kw):
    return adjoint_setup(CASES["adjoint64"], precision=precision, device=cuda, **kw)


def test_c3_against_central_differences(lib, cuda):
    """64x128 tube, 64 samples, 500 steps, 512 observation nodes every 10th step, checkpoints
    every 50: adjoint dJ/dlogE against central differences (step 1e-6) of the FP64 forward on
    32 random elements (all samples at once), FP64 and FP32 adjoints."""
    p64, logE, logh, _ = c3_problem(64, cuda)
    p32, _, _, _ = c3_problem(32, cuda)
    p32.set_observations(p64.obs[: p64.n_obs_steps, : p64.n_obs].to(torch.float32))
    p64.objective(logE, logh)
    g64, _ = p64.gradient()
    p32.objective(logE, logh)
    g32, _ = p32.gradient()
    rng = np.random.default_rng(5)
    elems = rng.choice(p64.E, size=32, replace=False)
    eps = 1e-6
    fd = torch.empty((32, p64.S), dtype=torch.float64)
    for k, e in enumerate(elems):
        d = torch.zeros_like(logE)
        d[e] = eps
        Jp = p64.objective(logE + d, logh)
        Jm = p64.objective(logE - d, logh)
        fd[k] = ((Jp - Jm) / (2 * eps)).cpu()
    # central differences at step 1e-6 carry ~1e-6 relative rounding error themselves
    assert rel(g64[elems].cpu(), fd) < 1e-5, rel(g64[elems].cpu(), fd)
    assert rel(g32[elems].cpu(), fd) < 1e-4, rel(g32[elems].cpu(), fd)


def test_c3_against_torch_autograd(lib, cuda):
    p64, logE, logh, _ = c3_problem(64, cuda, grad_logh=True)
    J = p64.objective(logE, logh)
    gE, gh = p64.gradient()
    Jr, gEr, ghr = torch_reference(p64, logE, logh, cuda, segment_len=50)
    assert rel(J, Jr) < 1e-12
    assert rel(gE, gEr) < 1e-9, rel(gE, gEr)
    assert rel(gh, ghr) < 1e-9, rel(gh, ghr)


def test_problem_rejects_bad_observation_nodes(lib, cuda):
    from cvfes_b200.cases import build_mesh, case_dt
    mesh = build_mesh(SMALL)
    with pytest.raises(ValueError):
        MismatchProblem(mesh, case_dt(SMALL, mesh), np.zeros(20), [3, 3], device=cuda)
    with pytest.raises(ValueError):
        MismatchProblem(mesh, case_dt(SMALL, mesh), np.zeros(20), [mesh.nNodes], device=cuda)


REV_VARIANTS = {
    32: [(4, 8, 0, 1), (2, 8, 0, 1), (1, 2, 1, 2), (2, 2, 1, 2), (4, 2, 1, 1), (2, 4, 1, 2),
         (2, 2, 2, 2), (4, 2, 2, 1), (2, 4, 2, 2)],
    64: [(2, 8, 0, 1), (1, 8, 0, 1), (1, 2, 1, 2), (2, 2, 1, 1), (2, 4, 1, 2), (2, 2, 2, 1),
         (1, 2, 2, 2)],
}


@pytest.mark.parametrize("precision", [32, 64])
def test_reverse_kernel_variants_are_bitwise_identical(lib, cuda, precision):
    """L1-gather, fan-rotation and persistent fan reverse kernels, every tile shape:
    same bits."""
    from cvfes_b200 import _lib
    case = dataclasses.replace(SMALL, n_samples=128 if precision == 32 else 64)
    p, logE, logh, _ = adjoint_setup(case, precision=precision, device=cuda, grad_logh=True)
    saved = _lib.get_adjoint_tuning(precision)
    outs = []
    try:
        for tune in REV_VARIANTS[precision]:
            _lib.set_adjoint_tuning(precision, *tune)
            p.release_graphs()
            p.objective(logE, logh)
            outs.append(p.gradient())
    finally:
        _lib.set_adjoint_tuning(precision, **saved)
    for tune, (gE, gh) in zip(REV_VARIANTS[precision][1:], outs[1:]):
        assert torch.equal(gE, outs[0][0]) and torch.equal(gh, outs[0][1]), tune


def test_autograd_function_flat_fp32_inputs(lib, cuda):
    """Flat FP32 log E / log h (any shape that reshapes to (E, S)) get gradients of their
    own shape and dtype."""
    problem, logE, logh, _ = adjoint_setup(SMALL, precision=64, device=cuda, grad_logh=True)
    lE = logE.reshape(-1).to(cuda, torch.float32).requires_grad_(True)
    lh = logh.reshape(-1).to(cuda, torch.float32).requires_grad_(True)
    J = wall_mismatch(lE, lh, problem)
    J.sum().backward()
    assert lE.grad.shape == lE.shape and lE.grad.dtype == torch.float32
    assert lh.grad.shape == lh.shape and lh.grad.dtype == torch.float32
    problem.objective(lE.detach().double().reshape(logE.shape),
                      lh.detach().double().reshape(logh.shape))
    gE, gh = problem.gradient()
    assert torch.allclose(lE.grad, gE.reshape(-1).float(), rtol=1e-6, atol=0)
    assert torch.allclose(lh.grad, gh.reshape(-1).float(), rtol=1e-6, atol=0)
