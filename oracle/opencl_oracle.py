"""CPU restatement of the reference's OpenCL solid class.  TEST INFRASTRUCTURE ONLY.

Only ``tests/`` use this module.  The reference's GPU solver class
(``physicsSolverSDampGPUs.py``) runs OpenCL kernels (``physicsSolverSDampGPUs.cl``)
that cannot run here (no OpenCL runtime).  This module restates, in NumPy and FP64,
what those kernels compute for the solid step, vectorised over elements and samples:

* ``elmTE`` = the mean of E*h over the element's nodes    -- ``.py:166-175``
* ``assemble_K_M_P`` at start-up: K u0 on the undeformed geometry, the lumped mass
  from nodal thickness, the pressure load                  -- ``.cl:28-223``
* ``calc_ddu`` and the Taylor start ``u_{-1}``             -- ``.cl:398-409``, ``.py:226-276``
* ``assemble_K_P`` every step: the element frame, area, B and stiffness on the
  deformed geometry x + u of each sample, K u and the follower pressure -- ``.cl:232-393``
* ``calc_u``: the damped update with LHS = LM             -- ``.cl:416-429``
* Dirichlet rows, then ``calc_u_appTrac``                 -- ``.py:359-387``, ``.cl:436-446``

Element arithmetic follows the kernels' own formulas (local frame from nodes 1->2 and
the Gram-Schmidt of 2->0, the 3x3 local blocks with the v, (1-v)/2 and k(1-v)/2 terms
over 4 A (1-v^2), the rotation T^T K T); the kernel's mass weights are applied as the
per-node sums of its ab terms (row 2 with its ab = 22 weights).

Pinned against the reference's compiled CPU kernels where the two classes agree (one
thickness and modulus per sample, no damping, stiffness rebuilt every step):
``tests/test_opencl_oracle.py``.
"""
from __future__ import annotations

import numpy as np

SHEAR_K = 5.0 / 6.0
# per-node sums of assemble_K_M_P's mass terms (physicsSolverSDampGPUs.cl:174-223), x rho A/3
MASS_W = np.array([[0.5, 0.25, 0.25], [0.25, 0.5, 0.25], [0.25, 0.375, 0.375]])


def _frames(x):
    """Frame rows T (..., 3, 3), area (...) and the local B terms b, c (..., 3) of
    triangles with node coordinates x (..., 3 nodes, 3)."""
    e = x[..., 2, :] - x[..., 1, :]
    t0 = e / np.sqrt(np.sum(e * e, axis=-1))[..., None]
    f = x[..., 0, :] - x[..., 2, :]
    f = f - np.sum(t0 * f, axis=-1)[..., None] * t0
    t1 = f / np.sqrt(np.sum(f * f, axis=-1))[..., None]
    t2 = np.stack([t0[..., 1] * t1[..., 2] - t0[..., 2] * t1[..., 1],
                   t0[..., 2] * t1[..., 0] - t0[..., 0] * t1[..., 2],
                   t0[..., 0] * t1[..., 1] - t0[..., 1] * t1[..., 0]], axis=-1)
    T = np.stack([t0, t1, t2], axis=-2)
    lx = np.sum(x * t0[..., None, :], axis=-1)   # (..., 3 nodes)
    ly = np.sum(x * t1[..., None, :], axis=-1)
    area = 0.5 * (lx[..., 0] * (ly[..., 1] - ly[..., 2]) - lx[..., 1] * (ly[..., 0] - ly[..., 2])
                  + lx[..., 2] * (ly[..., 0] - ly[..., 1]))
    b = np.stack([ly[..., 1] - ly[..., 2], ly[..., 2] - ly[..., 0], ly[..., 0] - ly[..., 1]], -1)
    c = np.stack([lx[..., 2] - lx[..., 1], lx[..., 0] - lx[..., 2], lx[..., 1] - lx[..., 0]], -1)
    return T, area, b, c


def _element_ku(x, ue, te, v, pressure):
    """K_e u_e and the pressure load of every element and sample.

    x (E,S,3,3) coordinates, ue (E,S,3,3) displacements (node, xyz), te (E,S) the
    coefficient E*h.  Returns (ku (E,S,3,3), p (E,S,3,3), area (E,S))."""
    T, area, b, c = _frames(x)
    pe1, pe2 = 0.5 * (1.0 - v), 0.5 * SHEAR_K * (1.0 - v)
    scale = te / (4.0 * area * (1.0 - v * v))
    ku = np.zeros_like(ue)
    for i in range(3):
        for j in range(i, 3):
            bb, bc, cb, cc = b[..., i] * b[..., j], b[..., i] * c[..., j], c[..., i] * b[..., j], \
                c[..., i] * c[..., j]
            llk = np.zeros(bb.shape + (3, 3))
            llk[..., 0, 0] = bb + cc * pe1
            llk[..., 0, 1] = bc * v + cb * pe1
            llk[..., 1, 0] = cb * v + bc * pe1
            llk[..., 1, 1] = cc + bb * pe1
            llk[..., 2, 2] = (bb + cc) * pe2
            glk = np.einsum("...mi,...mn,...nj->...ij", T, llk, T)       # T^T llK T
            ku[..., i, :] += np.einsum("...ij,...j->...i", glk, ue[..., j, :]) * scale[..., None]
            if j > i:
                ku[..., j, :] += np.einsum("...ji,...j->...i", glk, ue[..., i, :]) * \
                    scale[..., None]
    load = T[..., 2, :] * (pressure * area / 3.0)[..., None]             # (E,S,3)
    p = np.repeat(load[..., None, :], 3, axis=-2)
    return ku, p, area


class OpenCLSolidOracle:
    """FP64 restatement of the OpenCL solid class for small meshes.

    ``vE``, ``vthickness``: nodal fields (N, S); ``u0``, ``du0``: (3N,) as the class's
    ``iniU``/``iniDu``.  ``step(p, trac)`` advances all samples by one ``Solve``."""

    def __init__(self, nodes, elements, boundary, vE, vthickness, density, v, damp, dt,
                 u0=None, du0=None, bdyU=0.0, p0=0.0):
        self.nodes = np.asarray(nodes, dtype=np.float64)
        self.elements = np.asarray(elements, dtype=np.int64)
        self.N = self.nodes.shape[0]
        vE = np.asarray(vE, dtype=np.float64)
        vh = np.asarray(vthickness, dtype=np.float64)
        self.S = vE.shape[1]
        self.v, self.damp, self.dt, self.bdyU = float(v), float(damp), float(dt), bdyU
        bdy = np.asarray(boundary, dtype=np.int64)
        self.bdyDofs = (3 * bdy[:, None] + np.arange(3)[None, :]).ravel()
        self.bdyNodes = bdy
        el = self.elements
        # elmTE: mean of E*h over the element's nodes (physicsSolverSDampGPUs.py:166-175)
        self.te = (vE[el] * vh[el]).mean(axis=1)                          # (E,S)
        u0 = np.zeros(3 * self.N) if u0 is None else np.asarray(u0, dtype=np.float64)
        du0 = np.zeros(3 * self.N) if du0 is None else np.asarray(du0, dtype=np.float64)
        # assemble_K_M_P: undeformed geometry, the same u0 for every sample
        x = np.broadcast_to(self.nodes[el][:, None], (len(el), self.S, 3, 3))
        ue = np.broadcast_to(u0.reshape(-1, 3)[el][:, None], (len(el), self.S, 3, 3))
        ku_e, p_e, area = _element_ku(x, ue, self.te, self.v, p0)
        ku0, p0v = self._gather(ku_e), self._gather(p_e)
        hn = vh[el].swapaxes(1, 2)                                        # (E,S,3 nodes)
        m_e = (float(density) * area / 3.0)[..., None] * np.einsum("ak,esk->esa", MASS_W, hn)
        lm = np.zeros((self.N, self.S))
        np.add.at(lm, el.ravel(), m_e.transpose(0, 2, 1).reshape(-1, self.S))
        self.LM = np.repeat(lm, 3, axis=0)                                # (3N,S)
        self.LHS = self.LM.copy()
        # calc_ddu and the Taylor start (physicsSolverSDampGPUs.py:226-276)
        ddu = (p0v - ku0) / self.LHS
        self.u = np.repeat(u0[:, None], self.S, axis=1)
        self.up = self.u - dt * du0[:, None] + dt ** 2 * ddu / 2.0

    def _gather(self, per_elem):
        """Sum element-node contributions (E,S,3,3) into (3N,S)."""
        out = np.zeros((self.N, 3, self.S))
        np.add.at(out, self.elements.ravel(), per_elem.transpose(0, 2, 3, 1).reshape(-1, 3, self.S))
        return out.reshape(3 * self.N, self.S)

    def step(self, p, trac=None):
        el = self.elements
        us = self.u.reshape(self.N, 3, self.S)[el].transpose(0, 3, 1, 2)    # (E,S,3,3)
        x = self.nodes[el][:, None] + us
        ku_e, p_e, _ = _element_ku(x, us, self.te, self.v, float(p))
        Ku, P = self._gather(ku_e), self._gather(p_e)
        dt = self.dt
        ures = (dt * dt * ((P - self.damp * (self.u - self.up) / dt) - Ku)
                + self.LM * (2.0 * self.u - self.up)) / self.LHS
        ures[self.bdyDofs, :] = self.bdyU
        if trac is not None:
            tr = np.array(trac, dtype=np.float64).reshape(self.N, 3)
            tr[self.bdyNodes] = 0.0
            ures += dt * dt * tr.reshape(-1)[:, None] / self.LHS
        self.up, self.u = self.u, ures
        return ures
