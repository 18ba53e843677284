"""The discrete adjoint that the reverse kernels implement, restated in NumPy on the CPU.

The reverse kernels (``csrc/solid_adjoint.cu``) do not store the forward states: they
run the step backwards from checkpoint pairs ``(u_m, u_{m+1})`` and advance the scaled
adjoint ``chi_n = W lambda_n`` (``W = dt^2 / ((1 + dt c/2) m)``), accumulating

    dJ/dlogE_e = -c_e sum_n chi_{n+1,e}^T Khat_e u_{n,e}
    dJ/dlogh_e = dJ/dlogE_e - h_e sum_{a in e} alpha_{e,a} m_a^-1 sum_n chi_{n+1,a} . r_{n,a}

with ``r_n = p_n fhat - K u_n``.  This file restates that algorithm (increment-form
step, chi recursion, backward reconstruction per checkpoint segment, the two gradient
sums) in NumPy and checks it against FP64 torch autograd of the reference's step
(``oracle/adjoint_oracle.py``), so the recursion is pinned without a GPU.
"""
import numpy as np
import pytest
import torch

from cvfes_b200.cases import TubeCase, build_mesh, case_dt
from oracle import adjoint_oracle as ao


def problem(S=2, T=36, every=6, lumping="reference"):
    case = TubeCase("adjrec", 8, 6, 1.0, radius=0.3, n_samples=S, dt=None, seed_E=3,
                    seed_h=4, mass_lumping=lumping)
    mesh = build_mesh(case)
    dt = case_dt(case, mesh)
    tw = ao.TorchWall(mesh.nodes, mesh.elementNodeIds, mesh.boundary, mesh.density, mesh.v,
                      mesh.damp, dt, mass_lumping=lumping)
    free = np.setdiff1d(np.arange(mesh.nNodes), mesh.boundary)
    obs_nodes = free[::3]
    pres = 1.33e5 * np.minimum(np.arange(T) / 10.0, 1.0)
    logE = np.log(mesh.elmE)
    logh = np.log(mesh.elmThick)
    rng = np.random.default_rng(0)
    obs = 1e-4 * rng.standard_normal((T // every, len(obs_nodes), 3, S))
    return tw, logE, logh, pres, obs_nodes, obs, every


class Emulation:
    """The forward step in increment form and its discrete adjoint, in NumPy."""

    def __init__(self, tw, logE, logh):
        self.Kt = tw.Kt.numpy()                      # (E, 9, 9) unit-coefficient templates
        self.dofs = tw.dofs.numpy()                  # (E, 9)
        self.f = tw.f.numpy()                        # (3N,) unit pressure load
        self.N = tw.N
        self.elements = tw.elements.numpy()
        self.alpha = tw.alpha                        # (E, 3) mass per unit thickness
        self.h = np.exp(logh)
        self.c = np.exp(logE) * self.h               # (E, S)
        S = self.c.shape[1]
        m = np.zeros((self.N, S))
        for a in range(3):
            np.add.at(m, self.elements[:, a], self.alpha[:, a:a + 1] * self.h)
        self.m = m                                   # (N, S) lumped mass per node
        dt, damp = tw.dt, tw.damp
        g = 0.5 * dt * damp
        self.eta = dt * damp / (1.0 + g)
        live = np.ones(3 * self.N, dtype=bool)
        live[tw.bdy_dofs.numpy()] = False
        self.live = live
        self.W = np.where(live[:, None], (dt * dt / (1.0 + g)) / np.repeat(m, 3, axis=0), 0.0)

    def kmul(self, u, c=None):
        c = self.c if c is None else c
        ue = u[self.dofs]                                        # (E, 9, S)
        y = np.einsum("eij,ejs->eis", self.Kt, ue) * c[:, None, :]
        out = np.zeros_like(u)
        np.add.at(out, self.dofs.reshape(-1), y.reshape(-1, u.shape[1]))
        return out

    def residual(self, u, p):
        return p * self.f[:, None] - self.kmul(u)

    def step(self, u, up, p):
        v = (u - up) * (1.0 - self.eta) + self.W * self.residual(u, p)
        return np.where(self.live[:, None], u + v, 0.0)

    def back(self, u, un, p):
        """u_{n-1} from (u_n, u_{n+1}): the step solved for its previous state."""
        dv = ((un - u) - self.W * self.residual(u, p)) / (1.0 - self.eta)
        return np.where(self.live[:, None], u - dv, 0.0)

    def forward(self, pres):
        S = self.c.shape[1]
        hist = [np.zeros((3 * self.N, S))]
        up = np.zeros_like(hist[0])
        for p in pres:
            un = self.step(hist[-1], up, p)
            up = hist[-1]
            hist.append(un)
        return hist                                              # u_0 .. u_T

    def mismatch(self, hist, obs_nodes, obs, every):
        rows = (3 * np.asarray(obs_nodes)[:, None] + np.arange(3)).reshape(-1)
        J = np.zeros(self.c.shape[1])
        g = {}
        for k in range(every, len(hist), every):
            d = hist[k][rows] - obs[k // every - 1].reshape(-1, hist[k].shape[1])
            J += (d * d).sum(axis=0)
            gk = np.zeros_like(hist[k])
            gk[rows] = 2.0 * d
            g[k] = gk
        return J, g

    def gradients(self, states, pres, g, log_h=True):
        """Reverse pass: ``states(n)`` returns u_n; chi recursion and gradient sums."""
        T = len(pres)
        S = self.c.shape[1]
        zero = np.zeros((3 * self.N, S))
        chi1, chi2 = zero, zero                                  # chi_{n+1}, chi_{n+2}
        gam = np.zeros_like(self.c)                              # sum_n chi^T Khat u per element
        gm = np.zeros((self.N, S))                               # sum_n chi . r per node
        for n in range(T, -1, -1):
            # chi_n = W g_n + chi_{n+1} + (1-eta)(chi_{n+1} - chi_{n+2}) - W K chi_{n+1}
            chi = chi1 + (1.0 - self.eta) * (chi1 - chi2) - self.W * self.kmul(chi1)
            if n in g:
                chi = chi + self.W * g[n]
            chi = np.where(self.live[:, None], chi, 0.0)
            if n < T:                                            # terms of step n -> n+1
                u = states(n)
                ue = u[self.dofs]
                xe = chi1[self.dofs]
                gam += np.einsum("eis,eij,ejs->es", xe, self.Kt, ue)
                r = self.residual(u, pres[n])
                gm += (chi1 * r).reshape(self.N, 3, S).sum(axis=1)
            chi1, chi2 = chi, chi1
        gE = -self.c * gam
        if not log_h:
            return gE, None
        mass_term = np.zeros_like(self.c)
        for a in range(3):
            node = self.elements[:, a]
            mass_term += self.alpha[:, a:a + 1] * gm[node] / self.m[node]
        return gE, gE - self.h * mass_term


@pytest.mark.parametrize("lumping", ["reference", "rowsum"])
def test_recursion_matches_torch_autograd(lumping):
    tw, logE, logh, pres, obs_nodes, obs, every = problem(lumping=lumping)
    em = Emulation(tw, logE, logh)
    hist = em.forward(pres)
    J, g = em.mismatch(hist, obs_nodes, obs, every)
    gE, gh = em.gradients(lambda n: hist[n], pres, g)
    Jr, gEr, ghr = ao.autograd_gradients(tw, torch.from_numpy(logE), torch.from_numpy(logh),
                                         pres, obs_nodes, torch.from_numpy(obs), every)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel(J, Jr.numpy()) < 1e-12
    assert rel(gE, gEr.numpy()) < 1e-10
    assert rel(gh, ghr.numpy()) < 1e-10


def test_backward_reconstruction_from_checkpoint_pairs():
    """The reverse pass's states: from the forward pass's final pair (u_{T-1}, u_T) the
    step runs backwards, and at every checkpoint m the saved pair (u_m, u_{m+1}) replaces
    the reconstructed one; the drift stays at rounding level, and the gradients from the
    reconstructed states equal those from the stored history."""
    tw, logE, logh, pres, obs_nodes, obs, every = problem(T=40)
    em = Emulation(tw, logE, logh)
    hist = em.forward(pres)
    T, L = len(pres), 15
    pairs = {m: (hist[m], hist[m + 1]) for m in range(0, T, L)}
    recon = {T: hist[T]}
    u, un = hist[T - 1], hist[T]
    for n in range(T - 1, -1, -1):
        if n in pairs:
            u, un = pairs[n]
        recon[n] = u
        if n > 0:
            u, un = em.back(u, un, pres[n]), u
    scale = max(np.abs(h).max() for h in hist)
    drift = max(np.abs(recon[n] - hist[n]).max() for n in recon) / scale
    assert drift < 1e-10
    J, g = em.mismatch(hist, obs_nodes, obs, every)
    ref = em.gradients(lambda n: hist[n], pres, g)
    got = em.gradients(lambda n: recon[n], pres, g)
    for a, b in zip(got, ref):
        assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(b)
