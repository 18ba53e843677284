"""CPU oracle for the ensemble membrane solid time step.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module; the product path never does.

It restates, in NumPy and FP64, the reference's CPU solid path in
linear-template mode (stiffness assembled once, never updated):

* material coefficients and quadrature tables  -- ``physicsSolver.py:146-202``
* local frame ``T``/``TT``                       -- ``optimizedSolidAssemble.pyx:82-127``
* element B, BᵀDB, stiffness/mass/damping       -- ``optimizedSolidAssemble.pyx:530-583``
* unit-pressure traction ``f``                   -- ``optimizedSolidAssemble.pyx:585-590``
* block-CSR scatter and lumping                 -- ``optimizedSolidAssemble.pyx:365-454``
* node-graph CSR pattern                        -- ``sparse.py:36-64``
* block SpMV ``MultiplyByVector``               -- ``optimizedSolidAssemble.pyx:1250-1274``
* start-up ``u_{-1}`` and ``LHS``               -- ``physicsSolver.py:209-230``
* explicit damped update + Dirichlet            -- ``physicsSolver.py:263-292, 327-328``

Pressure enters by linearity: the traction is assembled once with unit
pressure (``coefs = [1.0, damp]``) and step ``n`` uses ``p_n * f``.

Parity of this restatement is pinned against the reference's own compiled
kernels (``oracle/_ref``, built by ``oracle/Makefile``) and against the golden
fixtures those kernels produced (``tests/golden``).
"""
from __future__ import annotations

import builtins
import glob
import importlib.util
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
SHEAR_K = 5.0 / 6.0

# Quadrature table of physicsSolver.py:146-148: three mid-edge points, weight 1/3.
XW = np.array([[0.5, 0.5, 0.0, 1.0 / 3.0],
               [0.5, 0.0, 0.5, 1.0 / 3.0],
               [0.0, 0.5, 0.5, 1.0 / 3.0]])


# --------------------------------------------------------------------------------------
# The reference's own compiled kernels
# --------------------------------------------------------------------------------------
def load_reference_module():
    """Import ``oracle/_ref/optimizedSolidAssemble`` or return ``None`` if not built.

    The module uses two Python-2 names at call time (``np.float``, ``long``);
    they are restored as aliases of the builtins before import.
    """
    paths = glob.glob(os.path.join(_HERE, "_ref", "optimizedSolidAssemble*.so"))
    if not paths:
        return None
    if not hasattr(np, "float"):
        np.float = float  # type: ignore[attr-defined]
    if not hasattr(builtins, "long"):
        builtins.long = int  # type: ignore[attr-defined]
    spec = importlib.util.spec_from_file_location("optimizedSolidAssemble", paths[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# --------------------------------------------------------------------------------------
# Tables (physicsSolver.py:175-197)
# --------------------------------------------------------------------------------------
def d_matrix(v: float, k: float = SHEAR_K) -> np.ndarray:
    """Membrane + transverse-shear constitutive matrix without E (physicsSolver.py:184-188)."""
    return np.array([[1.0, v, 0.0, 0.0, 0.0],
                     [v, 1.0, 0.0, 0.0, 0.0],
                     [0.0, 0.0, 0.5 * (1 - v), 0.0, 0.0],
                     [0.0, 0.0, 0.0, 0.5 * k * (1 - v), 0.0],
                     [0.0, 0.0, 0.0, 0.0, 0.5 * k * (1 - v)]]) / (1 - v * v)


def local_mass_table(density: float) -> np.ndarray:
    """``tM[g] = N_gᵀ N_g * w_g * rho`` (physicsSolver.py:190-197)."""
    tM = np.zeros((3, 9, 9))
    for g in range(3):
        N = np.zeros((3, 9))
        for a in range(3):
            for d in range(3):
                N[d, 3 * a + d] = XW[g, a]
        tM[g] = N.T @ N * XW[g, 3] * density
    return tM


# --------------------------------------------------------------------------------------
# Element geometry (optimizedSolidAssemble.pyx:82-127, 530-560), vectorised over elements
# --------------------------------------------------------------------------------------
def element_frames(nodes: np.ndarray, elements: np.ndarray):
    """Return ``T (E,3,3)``, ``area (E,)`` and ``B (E,5,9)`` on the given coordinates."""
    p = nodes[elements]                       # (E,3,3): node, xyz
    e0 = p[:, 2] - p[:, 1]
    e1 = p[:, 0] - p[:, 2]
    T = np.empty((len(elements), 3, 3))
    T[:, 0] = e0 / np.sqrt(np.sum(e0 * e0, axis=1))[:, None]
    proj = np.sum(e1 * T[:, 0], axis=1)
    t1 = e1 - proj[:, None] * T[:, 0]
    T[:, 1] = t1 / np.sqrt(np.sum(t1 * t1, axis=1))[:, None]
    T[:, 2, 0] = T[:, 0, 1] * T[:, 1, 2] - T[:, 0, 2] * T[:, 1, 1]
    T[:, 2, 1] = T[:, 0, 2] * T[:, 1, 0] - T[:, 0, 0] * T[:, 1, 2]
    T[:, 2, 2] = T[:, 0, 0] * T[:, 1, 1] - T[:, 0, 1] * T[:, 1, 0]
    lx = np.einsum("enk,ek->en", p, T[:, 0])
    ly = np.einsum("enk,ek->en", p, T[:, 1])
    area = ((lx[:, 1] * ly[:, 2] - lx[:, 2] * ly[:, 1])
            - (lx[:, 0] * ly[:, 2] - lx[:, 2] * ly[:, 0])
            + (lx[:, 0] * ly[:, 1] - lx[:, 1] * ly[:, 0])) * 0.5
    y23, y31, y12 = ly[:, 1] - ly[:, 2], ly[:, 2] - ly[:, 0], ly[:, 0] - ly[:, 1]
    x32, x13, x21 = lx[:, 2] - lx[:, 1], lx[:, 0] - lx[:, 2], lx[:, 1] - lx[:, 0]
    c1 = 2.0 * area
    B = np.zeros((len(elements), 5, 9))
    for (r, c), val in {(0, 0): y23, (2, 1): y23, (3, 2): y23,
                        (0, 3): y31, (2, 4): y31, (3, 5): y31,
                        (0, 6): y12, (2, 7): y12, (3, 8): y12,
                        (1, 1): x32, (2, 0): x32, (4, 2): x32,
                        (1, 4): x13, (2, 3): x13, (4, 5): x13,
                        (1, 7): x21, (2, 6): x21, (4, 8): x21}.items():
        B[:, r, c] = val / c1
    return T, area, B


def block_rotation(T: np.ndarray) -> np.ndarray:
    """9x9 block-diagonal ``TT`` (pyx:116-127)."""
    TT = np.zeros((T.shape[0], 9, 9))
    for a in range(3):
        TT[:, 3 * a:3 * a + 3, 3 * a:3 * a + 3] = T
    return TT


def element_templates(nodes, elements, v):
    """Unit stiffness per element, ``Kt_e = TTᵀ (BᵀDB * area) TT`` (E,9,9).

    The reference forms ``lK = BᵀDB * coefK * area`` per sample and rotates it;
    by linearity ``gK_{e,s} = coefK[e,s] * Kt_e``.
    """
    T, area, B = element_frames(nodes, elements)
    D = d_matrix(v)
    btdb = np.einsum("eki,kl,elj->eij", B, D, B)
    TT = block_rotation(T)
    return np.einsum("eki,ekl,elj->eij", TT, btdb * area[:, None, None], TT), T, area


# --------------------------------------------------------------------------------------
# Block-CSR assembly with damping (pyx:457-599) and SpMV (pyx:1250-1299)
# --------------------------------------------------------------------------------------
def block_positions(indptr, indices, elements):
    """CSR slot of every element block ``(a,b)``: (E,3,3) int64 (the pyx binary search)."""
    rows = elements[:, :, None].repeat(3, axis=2)
    cols = elements[:, None, :].repeat(3, axis=1)
    n = len(indptr) - 1
    key_csr = np.repeat(np.arange(n, dtype=np.int64), np.diff(indptr)) * n + indices
    pos = np.searchsorted(key_csr, (rows * n + cols).ravel())
    return pos.reshape(elements.shape[0], 3, 3)


def assemble_with_damping(nodes, elements, coefK, elmGThick, density, v, damp,
                          indptr, indices, trac=1.0):
    """Restatement of ``OptimizedSolidAssembleWithDamping`` (pyx:457-599).

    Returns ``M, C, K`` (nnzb,S,3,3), ``f`` (3N,), ``LM, LC`` (3N,S).
    """
    E = elements.shape[0]
    S = coefK.shape[1]
    N = nodes.shape[0]
    T, area, B = element_frames(nodes, elements)
    D = d_matrix(v)
    TT = block_rotation(T)
    btdb = np.einsum("eki,kl,elj->eij", B, D, B)
    tM = local_mass_table(density)
    wt = XW[:, 3]
    # lM[e,s] = sum_g tM[g] * h[e,s,g] * wt[g] * area[e]
    lM = np.einsum("gij,esg,g->esij", tM, elmGThick, wt) * area[:, None, None, None]
    lK = btdb[:, None] * (coefK * area[:, None])[:, :, None, None]
    rot = lambda X: np.einsum("eki,eskl,elj->esij", TT, X, TT)
    gM = rot(lM)
    gC = rot(lM * damp)
    gK = rot(lK)
    lf = np.zeros((E, 9))
    lf[:, [2, 5, 8]] = (trac / 3.0) * area[:, None]
    gf = np.einsum("eji,ej->ei", TT, lf)

    pos = block_positions(indptr, indices, elements)
    nnzb = len(indices)

    def scatter(gX):
        out = np.zeros((nnzb, S, 3, 3))
        blocks = gX.reshape(E, S, 3, 3, 3, 3).transpose(0, 2, 4, 1, 3, 5)  # e,a,b,s,i,j
        np.add.at(out, pos.ravel(), blocks.reshape(E * 9, S, 3, 3))
        return out

    M, C, K = scatter(gM), scatter(gC), scatter(gK)
    f = np.zeros(3 * N)
    np.add.at(f, (3 * elements[:, :, None] + np.arange(3)[None, None, :]).ravel(), gf.ravel())
    row_of_slot = np.repeat(np.arange(N), np.diff(indptr))
    LM = np.zeros((N, 3, S))
    LC = np.zeros((N, 3, S))
    np.add.at(LM, row_of_slot, M.sum(axis=3).transpose(0, 2, 1))
    np.add.at(LC, row_of_slot, C.sum(axis=3).transpose(0, 2, 1))
    return M, C, K, f, LM.transpose(0, 1, 2).reshape(3 * N, S), LC.reshape(3 * N, S)


def multiply_by_vector(indptr, indices, K, v, res=None):
    """``res += K v`` for block-CSR ``K (nnzb,S,3,3)`` and ``v (3N,S)`` (pyx:1250-1274)."""
    N = len(indptr) - 1
    S = K.shape[1]
    if res is None:
        res = np.zeros((3 * N, S))
    vb = np.asarray(v).reshape(N, 3, S)[indices]              # (nnzb,3,S)
    prod = np.einsum("nsij,njs->nis", K, vb)                   # (nnzb,3,S)
    rows = np.zeros((N, 3, S))
    nz = np.diff(indptr) > 0
    rows[nz] = np.add.reduceat(prod, indptr[:-1][nz], axis=0)
    res += rows.reshape(3 * N, S)
    return res


def template_multiply(elements, Kt, coefK, u):
    """``K_s u_s`` without the assembled matrix: sum_e coefK[e,s] Kt_e u_e."""
    N3, S = u.shape
    ue = u.reshape(-1, 3, S)[elements].reshape(elements.shape[0], 9, S)
    ye = np.einsum("eij,ejs->eis", Kt, ue) * coefK[:, None, :]
    out = np.zeros((N3 // 3, 3, S))
    np.add.at(out, elements.ravel(), ye.reshape(-1, 3, 3, S).reshape(-1, 3, S))
    return out.reshape(N3, S)


def batched_frames(p):
    """``element_frames`` for coordinates ``p`` (S,E,3,3) of every sample: T (S,E,3,3),
    area (S,E) and B (S,E,5,9) (pyx:82-127, 530-560)."""
    S, E = p.shape[:2]
    e0 = p[:, :, 2] - p[:, :, 1]
    e1 = p[:, :, 0] - p[:, :, 2]
    T = np.empty((S, E, 3, 3))
    T[:, :, 0] = e0 / np.sqrt(np.sum(e0 * e0, axis=-1))[..., None]
    proj = np.sum(e1 * T[:, :, 0], axis=-1)
    t1 = e1 - proj[..., None] * T[:, :, 0]
    T[:, :, 1] = t1 / np.sqrt(np.sum(t1 * t1, axis=-1))[..., None]
    T[:, :, 2, 0] = T[:, :, 0, 1] * T[:, :, 1, 2] - T[:, :, 0, 2] * T[:, :, 1, 1]
    T[:, :, 2, 1] = T[:, :, 0, 2] * T[:, :, 1, 0] - T[:, :, 0, 0] * T[:, :, 1, 2]
    T[:, :, 2, 2] = T[:, :, 0, 0] * T[:, :, 1, 1] - T[:, :, 0, 1] * T[:, :, 1, 0]
    lx = np.einsum("senk,sek->sen", p, T[:, :, 0])
    ly = np.einsum("senk,sek->sen", p, T[:, :, 1])
    area = ((lx[..., 1] * ly[..., 2] - lx[..., 2] * ly[..., 1])
            - (lx[..., 0] * ly[..., 2] - lx[..., 2] * ly[..., 0])
            + (lx[..., 0] * ly[..., 1] - lx[..., 1] * ly[..., 0])) * 0.5
    y23, y31, y12 = ly[..., 1] - ly[..., 2], ly[..., 2] - ly[..., 0], ly[..., 0] - ly[..., 1]
    x32, x13, x21 = lx[..., 2] - lx[..., 1], lx[..., 0] - lx[..., 2], lx[..., 1] - lx[..., 0]
    c1 = 2.0 * area
    B = np.zeros((S, E, 5, 9))
    for (r, c), val in {(0, 0): y23, (2, 1): y23, (3, 2): y23,
                        (0, 3): y31, (2, 4): y31, (3, 5): y31,
                        (0, 6): y12, (2, 7): y12, (3, 8): y12,
                        (1, 1): x32, (2, 0): x32, (4, 2): x32,
                        (1, 4): x13, (2, 3): x13, (4, 5): x13,
                        (1, 7): x21, (2, 6): x21, (4, 8): x21}.items():
        B[:, :, r, c] = val / c1
    return T, area, B


def _block_rot(T):
    S, E = T.shape[:2]
    TT = np.zeros((S, E, 9, 9))
    for a in range(3):
        TT[:, :, 3 * a:3 * a + 3, 3 * a:3 * a + 3] = T
    return TT


def geometric_update(nodes, elements, v, u):
    """Restatement of ``OptimizedSolidAssembleUpdate`` (pyx:710-819) with unit traction, per
    sample on the coordinates ``x + u_s`` (``mesh.py:678-680``): the unit stiffness of every
    element per sample (S,E,9,9) and the unit follower load (3N, S)."""
    N = nodes.shape[0]
    S = u.shape[1]
    xs = nodes[None] + u.T.reshape(S, N, 3)
    T, area, B = batched_frames(xs[:, elements])
    Bt = np.swapaxes(B, -1, -2)
    btdb = (Bt @ d_matrix(v)) @ B * area[..., None, None]
    TT = _block_rot(T)
    Kt = np.swapaxes(TT, -1, -2) @ btdb @ TT
    f = np.zeros((N, 3, S))
    load = (area / 3.0)[..., None] * T[:, :, 2]           # (S,E,3)
    for a in range(3):
        np.add.at(f, elements[:, a], load.transpose(1, 2, 0))
    return Kt, f.reshape(3 * N, S)


def calculate_stress(nodes_s, elements, v, young, u):
    """Restatement of ``OptimizedCalculateStress`` (pyx:1116-1223): on the per-sample
    coordinates ``nodes_s`` (S,N,3), the global (xx, yy, xy, xz, yz) entries of
    ``T^T (E D B TT u_e) T`` per element and sample, (E,S,5)."""
    S, N = nodes_s.shape[:2]
    T, area, B = batched_frames(nodes_s[:, elements])
    TT = _block_rot(T)
    ue = u.reshape(N, 3, S)[elements].reshape(elements.shape[0], 9, S).transpose(2, 0, 1)
    lU = np.einsum("seij,sej->sei", TT, ue)
    ls = np.einsum("kl,selj,sej->sek", d_matrix(v), B, lU) * young.T[..., None]
    L = np.zeros(T.shape)
    L[..., 0, 0] = ls[..., 0]
    L[..., 0, 1] = L[..., 1, 0] = ls[..., 2]
    L[..., 0, 2] = L[..., 2, 0] = ls[..., 3]
    L[..., 1, 1] = ls[..., 1]
    L[..., 1, 2] = L[..., 2, 1] = ls[..., 4]
    G = np.swapaxes(T, -1, -2) @ L @ T
    out = np.stack([G[..., 0, 0], G[..., 1, 1], G[..., 0, 1], G[..., 0, 2], G[..., 1, 2]],
                   axis=-1)
    return out.transpose(1, 0, 2).copy()


# --------------------------------------------------------------------------------------
# Load schedules (RefreshContext semantics)
# --------------------------------------------------------------------------------------
def pressure_cosine(t, P, T):
    """``physicsSolverSDampGPUs.py:317-322``: P/2 - P/2 cos(pi t/T) up to T, then P."""
    return P if t > T else P / 2.0 - P / 2.0 * math.cos(math.pi / T * t)


def pressure_linear_steps(n_steps, P, ramp_steps):
    """``p_n = P * min(n / ramp_steps, 1)`` for n = 0..n_steps-1."""
    n = np.arange(n_steps, dtype=np.float64)
    return P * np.minimum(n / float(ramp_steps), 1.0)


# --------------------------------------------------------------------------------------
# The solid solver in linear-template mode (physicsSolver.py:102-292)
# --------------------------------------------------------------------------------------
class OracleSolidSolver:
    """FP64 CPU solid solver with damping and a per-step pressure.

    ``backend='reference'`` runs the reference's compiled assembly and SpMV;
    ``backend='numpy'`` runs the restatement above;  ``backend='template'``
    never forms the block-CSR matrix (for large meshes; same arithmetic up to
    summation order).
    """

    def __init__(self, nodes, elements, boundary, coefK, elmGThick, density, v, damp, dt,
                 u0=None, du0=None, bdyU=0.0, p0=0.0, backend="numpy", update_interval=0):
        self.nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.elements = np.ascontiguousarray(elements, dtype=np.int64)
        self.N = self.nodes.shape[0]
        self.S = coefK.shape[1]
        self.dt = float(dt)
        self.bdyU = bdyU
        self.backend = backend
        self.v = float(v)
        self.coefK_s = np.ascontiguousarray(coefK, dtype=np.float64)
        # stiffness_update_interval (physicsSolver.py:143-144, 296-324); 0: never
        self.update_interval = int(update_interval)
        self.update_counter = 0
        self.geo = None  # (per-sample stiffness, unit follower load) after an update
        self.update_nodes = None  # x + u at the last update, (S, N, 3)
        bdy = np.asarray(boundary, dtype=np.int64)
        self.bdyDofs = (3 * bdy[:, None] + np.arange(3)[None, :]).ravel()
        coefK = np.ascontiguousarray(coefK, dtype=np.float64)
        elmGThick = np.ascontiguousarray(elmGThick, dtype=np.float64)
        from_mesh_pattern = None
        if backend in ("numpy", "reference"):
            from_mesh_pattern = _pattern(self.elements, self.N)
            self.indptr, self.indices = from_mesh_pattern
        if backend == "reference":
            ref = load_reference_module()
            if ref is None:
                raise RuntimeError("oracle/_ref is not built (make -C oracle)")
            self.ref = ref
            nnzb = len(self.indices)
            self.M = np.zeros((nnzb, self.S, 3, 3))
            self.C = np.zeros((nnzb, self.S, 3, 3))
            self.K = np.zeros((nnzb, self.S, 3, 3))
            f = np.zeros(3 * self.N)
            self.LM = np.zeros((3 * self.N, self.S))
            self.LC = np.zeros((3 * self.N, self.S))
            ref.OptimizedSolidAssembleWithDamping(
                self.nodes, self.elements, np.array([1.0, damp]), np.ascontiguousarray(XW[:, 3]),
                local_mass_table(density), d_matrix(v), coefK, elmGThick,
                self.indptr, self.indices, self.M, self.C, self.K, f, self.LM, self.LC)
            self.f = f
        elif backend == "numpy":
            self.M, self.C, self.K, self.f, self.LM, self.LC = assemble_with_damping(
                self.nodes, self.elements, coefK, elmGThick, density, v, damp,
                self.indptr, self.indices)
        elif backend == "template":
            Kt, _, area = element_templates(self.nodes, self.elements, v)
            self.Kt, self.coefK = Kt, coefK
            T, _, _ = element_frames(self.nodes, self.elements)
            self.f = np.zeros(3 * self.N)
            np.add.at(self.f, (3 * self.elements[:, :, None] + np.arange(3)).ravel(),
                      np.repeat((area / 3.0)[:, None] * T[:, 2], 3, axis=0).ravel())
            # lumped mass row sum of node a: rho * area * sum_g w_g^2 N_g(a) h_g
            mw = density * (XW[:, :3] * XW[:, 3:4] ** 2)          # (g, a)
            m = np.zeros((self.N, self.S))
            for a in range(3):
                ha = np.einsum("esg,g->es", elmGThick, mw[:, a])
                np.add.at(m, self.elements[:, a], ha * area[:, None])
            self.LM = np.repeat(m, 3, axis=0)
            self.LC = damp * self.LM
        else:
            raise ValueError(backend)
        self.f = self.f.reshape(-1)
        # --- LocalInitialize (physicsSolver.py:209-230) ---
        u0 = np.zeros(3 * self.N) if u0 is None else np.asarray(u0, dtype=np.float64)
        du0 = np.zeros(3 * self.N) if du0 is None else np.asarray(du0, dtype=np.float64)
        Ku = self._kmul(np.tile(u0[:, None], (1, self.S)), scale=1.0)
        du = np.tile(du0[:, None], (1, self.S))
        self.u = np.tile(u0[:, None], (1, self.S))
        RHS = p0 * self.f[:, None] - self.LC * du - Ku
        LHS = np.copy(self.LM)
        ddu = np.divide(RHS, LHS, out=np.zeros_like(RHS), where=LHS != 0)
        dt = self.dt
        self.up = self.u - dt * du + 0.5 * (dt ** 2) * ddu
        self.LHS = self.LM + 0.5 * dt * self.LC

    def _geo_update(self):
        """Stiffness and unit follower load on x + u_n (the reference's update step)."""
        self.update_nodes = (self.nodes[None] + self.u.T.reshape(self.S, self.N, 3)).copy()
        if self.backend == "reference":
            S = self.S
            upd = (self.nodes[None] + self.u.T.reshape(S, self.N, 3)).copy()
            nnzb = len(self.indices)
            K = np.zeros((nnzb, S, 3, 3))
            f = np.zeros((3 * self.N, S))
            self.ref.OptimizedSolidAssembleUpdate(upd, self.elements, np.array([1.0]),
                                                  d_matrix(self.v), self.coefK_s, self.indptr,
                                                  self.indices, K, f)
            self.geo = ("bsr", K, f)
        else:
            Kts, f = geometric_update(self.nodes, self.elements, self.v, self.u)
            self.geo = ("templates", Kts, f)

    def _kmul_geo(self, u, scale):
        kind, K, _ = self.geo
        if kind == "bsr":
            res = np.zeros_like(u)
            self.ref.MultiplyByVector(self.indptr, self.indices, scale * K, np.ascontiguousarray(u),
                                      res)
            return res
        N3, S = u.shape
        ue = u.reshape(-1, 3, S)[self.elements].reshape(self.elements.shape[0], 9, S)
        ye = np.einsum("seij,ejs->eis", K, ue) * (scale * self.coefK_s)[:, None, :]
        out = np.zeros((N3 // 3, 3, S))
        np.add.at(out, self.elements.ravel(), ye.reshape(-1, 3, S))
        return out.reshape(N3, S)

    def _kmul(self, u, scale):
        if self.geo is not None:
            return self._kmul_geo(u, scale)
        if self.backend == "reference":
            res = np.zeros_like(u)
            self.ref.MultiplyByVector(self.indptr, self.indices, scale * self.K,
                                      np.ascontiguousarray(u), res)
            return res
        if self.backend == "numpy":
            return multiply_by_vector(self.indptr, self.indices, scale * self.K, u)
        return template_multiply(self.elements, self.Kt, scale * self.coefK, u)

    def step(self, p, trac=None):
        """One ``SolidSolver.Solve`` step (physicsSolver.py:263-292) with pressure ``p``.

        With an update interval, the stiffness and the (unit) follower load are rebuilt on
        x + u_n when the counter reaches the interval (physicsSolver.py:296-324); the load
        of the step is then ``p`` times the follower load of the last update."""
        dt = self.dt
        if self.update_interval:
            if self.update_counter >= self.update_interval:
                self._geo_update()
                self.update_counter = 1
            else:
                self.update_counter += 1
        if self.geo is not None:
            A1 = (dt ** 2) * p * self.geo[2]
        else:
            A1 = (dt ** 2) * (p * self.f)[:, None]
        if trac is not None:
            # nodal traction of the GPU path (calc_u_appTrac, physicsSolverSDampGPUs.cl:436-446)
            A1 = A1 + (dt ** 2) * np.asarray(trac, dtype=np.float64).reshape(-1)[:, None]
        Ku = self._kmul(self.u, scale=dt ** 2)
        A2 = 2.0 * self.LM * self.u - Ku
        A3 = (0.5 * dt * self.LC - self.LM) * self.up
        RHS = A1 + A2 + A3
        u = np.divide(RHS, self.LHS, out=np.zeros_like(RHS), where=self.LHS != 0)
        u[self.bdyDofs, :] = self.bdyU
        self.up = self.u
        self.u = u
        return u

    def stress(self, young):
        """Element stresses (E,S,5) of the current state on the geometry of the last update
        (``physicsSolver.py:416-424``); ``young`` (E,S) is the mean E of each element."""
        nodes_s = self.update_nodes if self.update_nodes is not None else \
            np.repeat(self.nodes[None], self.S, axis=0)
        if self.backend == "reference":
            out = np.empty((self.elements.shape[0], self.S, 5))
            self.ref.OptimizedCalculateStress(np.ascontiguousarray(nodes_s), self.elements,
                                              d_matrix(self.v), np.ascontiguousarray(young),
                                              np.ascontiguousarray(self.u), out)
            return out
        return calculate_stress(nodes_s, self.elements, self.v, young, self.u)

    def run(self, pressures, history_every=0):
        hist = []
        for n, p in enumerate(pressures):
            self.step(float(p))
            if history_every and (n + 1) % history_every == 0:
                hist.append(self.u.copy())
        return hist


def _pattern(elements, n_nodes):
    """``SparseInfo`` (sparse.py:36-64): per node, sorted unique neighbours incl. itself."""
    e = np.asarray(elements, dtype=np.int64)
    rows = np.repeat(e, 3, axis=1).ravel()
    cols = np.tile(e, (1, 3)).ravel()
    key = np.unique(rows * n_nodes + cols)
    r = key // n_nodes
    indptr = np.zeros(n_nodes + 1, dtype=np.int64)
    np.add.at(indptr, r + 1, 1)
    return np.cumsum(indptr), (key % n_nodes).astype(np.int64)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / d) if d > 0 else float(np.linalg.norm(a - b))
