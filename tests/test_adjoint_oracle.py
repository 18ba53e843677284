"""The FP64 torch-autograd reference of the mismatch objective, on the CPU.

It is pinned to the NumPy oracle (same displacement history) and its autograd
gradients to central finite differences of itself.
"""
import numpy as np
import pytest
import torch

from cvfes_b200.cases import TubeCase, build_mesh, case_dt
from oracle import adjoint_oracle as ao
from oracle import solid_oracle as so


def tiny(S=2, lumping="reference"):
    case = TubeCase("adjtiny", 8, 6, 1.0, radius=0.3, n_samples=S, dt=None, seed_E=3, seed_h=4,
                    mass_lumping=lumping)
    mesh = build_mesh(case)
    return case, mesh, case_dt(case, mesh)


@pytest.mark.parametrize("lumping", ["reference", "rowsum"])
def test_torch_forward_matches_numpy_oracle(lumping):
    case, mesh, dt = tiny(lumping=lumping)
    pres = 1.33e5 * np.minimum(np.arange(40) / 10.0, 1.0)
    coefK, gthick = mesh.element_coefficients()
    o = so.OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick,
                             mesh.density * (3.0 if lumping == "rowsum" else 1.0), mesh.v,
                             mesh.damp, dt, backend="numpy")
    o.run(pres)
    tw = ao.TorchWall(mesh.nodes, mesh.elementNodeIds, mesh.boundary, mesh.density, mesh.v,
                      mesh.damp, dt, mass_lumping=lumping)
    S = mesh.nSmp
    h = torch.from_numpy(mesh.elmThick)
    coef = torch.from_numpy(mesh.elmE) * h
    LM = tw.lumped_mass(h)
    LC = tw.damp * LM
    u = torch.zeros((3 * tw.N, S), dtype=torch.float64)
    u, up, _ = tw.segment(u, torch.zeros_like(u), coef, LM, LC, LM + 0.5 * dt * LC, pres, 0,
                          torch.zeros(0, dtype=torch.int64), None, 10 ** 9)
    assert so.rel_l2(u.numpy(), o.u) < 1e-13


def test_torch_autograd_matches_central_differences():
    case, mesh, dt = tiny(S=2)
    T, every = 36, 6
    pres = 1.33e5 * np.minimum(np.arange(T) / 10.0, 1.0)
    tw = ao.TorchWall(mesh.nodes, mesh.elementNodeIds, mesh.boundary, mesh.density, mesh.v,
                      mesh.damp, dt)
    free = np.setdiff1d(np.arange(mesh.nNodes), mesh.boundary)
    obs_nodes = free[::3]
    logE = torch.from_numpy(np.log(mesh.elmE))
    logh = torch.from_numpy(np.log(mesh.elmThick))
    with torch.no_grad():
        # observations from a perturbed stiffness field
        rng = np.random.default_rng(0)
        lE_true = logE + torch.from_numpy(0.1 * rng.standard_normal(logE.shape))
        u = torch.zeros((3 * tw.N, mesh.nSmp), dtype=torch.float64)
        h = torch.exp(logh)
        coef = torch.exp(lE_true) * h
        LM = tw.lumped_mass(h)
        LC = tw.damp * LM
        rows = (3 * torch.from_numpy(obs_nodes)[:, None] + torch.arange(3)).reshape(-1)
        obs = []
        up = torch.zeros_like(u)
        for n, p in enumerate(pres):
            u, up, _ = tw.segment(u, up, coef, LM, LC, LM + 0.5 * dt * LC, [p], n,
                                  torch.zeros(0, dtype=torch.int64), None, 10 ** 9)
            if (n + 1) % every == 0:
                obs.append(u[rows].reshape(len(obs_nodes), 3, -1))
        obs = torch.stack(obs)
    J, gE, gh = ao.autograd_gradients(tw, logE, logh, pres, obs_nodes, obs, every,
                                      segment_len=10)
    J2, gE2, gh2 = ao.autograd_gradients(tw, logE, logh, pres, obs_nodes, obs, every)
    assert torch.allclose(gE, gE2, rtol=1e-12, atol=0) and torch.allclose(gh, gh2, rtol=1e-12)
    eps = 1e-6
    for e in (0, 7, 20, 41):
        for which, g in (("E", gE), ("h", gh)):
            d = torch.zeros_like(logE)
            d[e] = eps
            with torch.no_grad():
                a = (logE + d, logh) if which == "E" else (logE, logh + d)
                b = (logE - d, logh) if which == "E" else (logE, logh - d)
                Jp = tw.mismatch(*a, pres, obs_nodes, obs, every)
                Jm = tw.mismatch(*b, pres, obs_nodes, obs, every)
            fd = (Jp - Jm) / (2 * eps)
            assert torch.allclose(fd, g[e], rtol=1e-5, atol=1e-9 * float(J.abs().max())), \
                (which, e, fd, g[e])
