"""FP64 torch-autograd reference of the displacement-mismatch objective.  TEST INFRASTRUCTURE ONLY.

Only ``tests/`` may import this module.  It restates the reference's solid step in
torch so that autograd gives the exact FP64 gradient of

    J_s = sum_{n = k*obs_every <= T} sum_{i in obs} |u_n(i) - uobs_n(i)|^2

with respect to per-element, per-sample log E and log h:

* unit stiffness ``Kt_e`` per element                 -- ``solid_oracle.element_templates``
  (``optimizedSolidAssemble.pyx:530-583``), scaled by ``coefK = E*h``
  (``physicsSolver.py:199-202`` with per-element fields)
* lumped mass ``rho * area * h * sum_g w_g^2 N_g(a)`` -- ``physicsSolver.py:190-197``,
  ``optimizedSolidAssemble.pyx:564-566`` (``rowsum``: weights ``w_g`` instead of ``w_g^2``)
* unit-pressure load ``area/3 * normal``              -- ``optimizedSolidAssemble.pyx:585-590``
* damped central-difference update and Dirichlet rows -- ``physicsSolver.py:263-292``

The run starts from rest (``u_0 = u_{-1} = 0``; ``physicsSolver.py:209-230`` with zero
initial displacement, velocity and pressure).
"""
from __future__ import annotations

import numpy as np
import torch

from . import solid_oracle as so


class TorchWall:
    """Differentiable FP64 forward model on one mesh (global node numbering)."""

    def __init__(self, nodes, elements, boundary, density, v, damp, dt, mass_lumping="reference",
                 bdyU=0.0, device="cpu"):
        self.device = torch.device(device)
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        elements = np.ascontiguousarray(elements, dtype=np.int64)
        self.N = nodes.shape[0]
        self.E = elements.shape[0]
        Kt, T, area = so.element_templates(nodes, elements, v)
        f = np.zeros(3 * self.N)
        np.add.at(f, (3 * elements[:, :, None] + np.arange(3)).ravel(),
                  np.repeat((area / 3.0)[:, None] * T[:, 2], 3, axis=0).ravel())
        w = so.XW[:, 3:4] ** 2 if mass_lumping == "reference" else so.XW[:, 3:4]
        mw = density * (so.XW[:, :3] * w)             # (g, a)
        self.alpha = area[:, None] * mw.sum(axis=0)[None, :]  # (E, 3): mass per unit thickness
        dev = self.device
        self.Kt = torch.from_numpy(Kt).to(dev)
        self.f = torch.from_numpy(f).to(dev)
        self.alpha_t = torch.from_numpy(self.alpha).to(dev)
        self.elements = torch.from_numpy(elements).to(dev)
        self.dofs = (3 * self.elements[:, :, None] + torch.arange(3, device=dev)).reshape(-1, 9)
        bdy = np.asarray(boundary, dtype=np.int64)
        self.bdy_dofs = torch.from_numpy((3 * bdy[:, None] + np.arange(3)).ravel()).to(dev)
        self.damp = float(damp)
        self.dt = float(dt)
        self.bdyU = float(bdyU)

    def kmul(self, coef, u):
        """K(coef) u for u (3N, S)."""
        ue = u[self.dofs]                                   # (E, 9, S)
        y = torch.einsum("eij,ejs->eis", self.Kt, ue) * coef[:, None, :]
        out = torch.zeros_like(u)
        return out.index_add(0, self.dofs.reshape(-1), y.reshape(-1, u.shape[1]))

    def lumped_mass(self, h):
        """(3N, S) lumped mass for per-element thickness h (E, S)."""
        S = h.shape[1]
        m = torch.zeros((self.N, S), dtype=h.dtype, device=h.device)
        for a in range(3):
            m = m.index_add(0, self.elements[:, a], self.alpha_t[:, a:a + 1] * h)
        return m.repeat_interleave(3, dim=0)

    def segment(self, u, up, coef, LM, LC, LHS, pressures, n0, obs_nodes, obs, obs_every):
        """Steps n0 .. n0+len(pressures)-1 from (u, up); returns (u, up, J increment)."""
        dt = self.dt
        J = torch.zeros(u.shape[1], dtype=u.dtype, device=u.device)
        rows = (3 * obs_nodes[:, None] + torch.arange(3, device=u.device)).reshape(-1)
        for k, p in enumerate(pressures):
            n = n0 + k
            RHS = (dt * dt * float(p)) * self.f[:, None] + 2.0 * LM * u \
                - (dt * dt) * self.kmul(coef, u) + (0.5 * dt * LC - LM) * up
            un = RHS / LHS
            un = un.index_fill(0, self.bdy_dofs, self.bdyU)
            up, u = u, un
            if (n + 1) % obs_every == 0:
                d = u[rows] - obs[(n + 1) // obs_every - 1].reshape(-1, u.shape[1])
                J = J + (d * d).sum(dim=0)
        return u, up, J

    def mismatch(self, logE, logh, pressures, obs_nodes, obs, obs_every, segment_len=0):
        """J (S,) for logE, logh (E, S); obs (T//obs_every, n_obs, 3, S).  With
        ``segment_len`` the steps run in recomputed segments (torch checkpointing)."""
        h = torch.exp(logh)
        coef = torch.exp(logE) * h
        LM = self.lumped_mass(h)
        LC = self.damp * LM
        LHS = LM + 0.5 * self.dt * LC
        S = logE.shape[1]
        u = torch.zeros((3 * self.N, S), dtype=torch.float64, device=logE.device)
        up = torch.zeros_like(u)
        obs_nodes = torch.as_tensor(obs_nodes, dtype=torch.int64, device=logE.device)
        J = torch.zeros(S, dtype=torch.float64, device=logE.device)
        p = np.asarray(pressures, dtype=np.float64)
        L = segment_len or len(p)
        for n0 in range(0, len(p), L):
            seg = p[n0:n0 + L]
            if segment_len:
                u, up, dJ = torch.utils.checkpoint.checkpoint(
                    self.segment, u, up, coef, LM, LC, LHS, seg, n0, obs_nodes, obs, obs_every,
                    use_reentrant=False)
            else:
                u, up, dJ = self.segment(u, up, coef, LM, LC, LHS, seg, n0, obs_nodes, obs,
                                         obs_every)
            J = J + dJ
        return J


def autograd_gradients(model: TorchWall, logE, logh, pressures, obs_nodes, obs, obs_every,
                       segment_len=0):
    """(J, dJ/dlogE, dJ/dlogh) by torch autograd (per-sample J, so grad of sum J)."""
    lE = torch.as_tensor(logE, dtype=torch.float64, device=model.device).clone().requires_grad_(True)
    lh = torch.as_tensor(logh, dtype=torch.float64, device=model.device).clone().requires_grad_(True)
    J = model.mismatch(lE, lh, pressures, obs_nodes, obs, obs_every, segment_len)
    gE, gh = torch.autograd.grad(J.sum(), (lE, lh))
    return J.detach(), gE, gh
