"""Per-element Gaussian Markov random fields for the wall material samples.

The reference samples a nodal Matérn GMRF with CHOLMOD (``GMRF.py:245-354``):
``X = L⁻ᵀ Z`` from the Cholesky factor of the precision, un-permuted, then each
node rescaled to std sigma across samples.  Here the field lives on elements
with precision ``Q = tau*I + L_adj`` (``L_adj`` the graph Laplacian of
edge-adjacent triangles):

* ``Q`` is factored as ``P Q Pᵀ = L D Lᵀ`` by SuperLU with a minimum-degree
  ordering and no pivoting (the role CHOLMOD's AMD-ordered factor plays in
  ``GMRF.py:288``), so ``L_c = L D^{1/2}`` is a Cholesky factor;
* ``z = L_c⁻ᵀ w`` with ``w ~ N(0, I)`` from ``numpy.random.default_rng(seed)``,
  then un-permuted (``GMRF.py:310-311``), so ``cov(z) = Q⁻¹``;
* ``z`` is rescaled to unit marginal std, exactly (``diag(Q⁻¹)`` by selected
  inversion of the factor) or, as the reference does, by the empirical std across
  samples (``GMRF.py:326-328``).

All of this is FP64 and runs once, on the host.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

from . import mesh as _mesh
from ._lib import call, ptr


def element_precision(elements: np.ndarray, n_nodes: int, tau: float = 0.1) -> sp.csc_matrix:
    """``Q = tau*I + (Deg - Adj)`` over edge-adjacent triangles."""
    E = int(elements.shape[0])
    r, c = _mesh.element_adjacency(elements, n_nodes)
    adj = sp.coo_matrix((np.ones(len(r)), (r, c)), shape=(E, E)).tocsr()
    adj.data[:] = 1.0
    deg = np.asarray(adj.sum(axis=1)).ravel()
    return (sp.diags(deg + tau) - adj).tocsc()


class ElementGMRF:
    """Factorised precision of one mesh; draws seeded unit-marginal samples."""

    def __init__(self, elements, n_nodes, tau: float = 0.1, marginal: str = "exact"):
        self.Q = element_precision(elements, n_nodes, tau)
        self.n = self.Q.shape[0]
        lu = sla.splu(self.Q, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0,
                      options=dict(SymmetricMode=True, Equil=False))
        if not np.array_equal(lu.perm_r, lu.perm_c):
            raise RuntimeError("GMRF factorisation pivoted; the precision is not SPD")
        # SuperLU: Pr A Pc = L U with Pr[perm_r[i], i] = 1, i.e. row i of A -> row perm_r[i].
        self.perm = lu.perm_r.copy()                  # A[i] -> position perm[i]
        self.order = np.argsort(self.perm)            # position p holds A index order[p]
        L = lu.L.tocsc()
        U = lu.U.tocsc()
        self.d = U.diagonal().copy()
        if np.any(self.d <= 0):
            raise RuntimeError("GMRF factorisation has a non-positive pivot")
        self.L = L
        self.U = U
        self.marginal = marginal
        self._var = None

    def _csc(self):
        if getattr(self, "_csc_arrays", None) is None:
            L = self.L.copy()
            L.sort_indices()
            self._csc_arrays = (np.ascontiguousarray(L.indptr, dtype=np.int64),
                                np.ascontiguousarray(L.indices, dtype=np.int64),
                                np.ascontiguousarray(L.data, dtype=np.float64))
        return self._csc_arrays

    def variance(self) -> np.ndarray:
        """``diag(Q⁻¹)`` in the original element order (exact, selected inversion)."""
        if self._var is None:
            out = np.empty(self.n)
            colptr, rowind, lval = self._csc()
            d = np.ascontiguousarray(self.d)
            call("cvfes_gmrf_selected_inverse_diag", self.n, ptr(colptr), ptr(rowind),
                 ptr(lval), ptr(d), ptr(out))
            self._var = out[self.perm]
        return self._var

    def sample(self, n_samples: int, seed: int) -> np.ndarray:
        """(E, S) samples with unit marginal standard deviation."""
        rng = np.random.default_rng(seed)
        w = rng.standard_normal((self.n, n_samples))
        # L_cᵀ z_p = w with L_c = L D^{1/2}  =>  Lᵀ z_p = D^{-1/2} w
        zp = np.ascontiguousarray(w / np.sqrt(self.d)[:, None])
        colptr, rowind, lval = self._csc()
        call("cvfes_gmrf_solve_lt", self.n, ptr(colptr), ptr(rowind), ptr(lval), n_samples,
             ptr(zp))
        z = zp[self.perm]
        if self.marginal == "exact":
            z /= np.sqrt(self.variance())[:, None]
        elif self.marginal == "empirical":
            z /= np.std(z, axis=1, keepdims=True)
        else:
            raise ValueError(self.marginal)
        return z


def material_fields(elements, n_nodes, n_samples, seed_E=23, seed_h=24, E0=7.0e6, sigma_logE=0.2,
                    h0=0.04, sigma_logh=0.1, tau=0.1, marginal="exact", gmrf=None):
    """Per-element ``E = E0*exp(sE*z)`` and ``h = h0*exp(sh*z')`` with independent z, z'."""
    g = gmrf if gmrf is not None else ElementGMRF(elements, n_nodes, tau, marginal)
    z = g.sample(n_samples, seed_E)
    zh = g.sample(n_samples, seed_h)
    return E0 * np.exp(sigma_logE * z), h0 * np.exp(sigma_logh * zh), g
