"""CPU restatement of the element GMRF material sampler.  TEST INFRASTRUCTURE ONLY.

Only ``tests/`` and ``bench.py``'s reference arm use this module: it synthesises the
reference arm's inputs without loading the product library.

The reference's sampler (``GMRF.py:245-354``): a Cholesky factor of the precision
``Q`` (CHOLMOD, with a fill-reducing permutation), ``X = L⁻ᵀ Z`` with ``Z ~ N(0, I)``,
un-permuted, then each field rescaled to the wanted standard deviation.  Restated for
the per-element field of the synthetic workloads:

* ``Q = tau I + L_adj`` over edge-adjacent triangles;
* the factor ``P Q Pᵀ = L D Lᵀ`` from SciPy's SuperLU (minimum-degree ordering on
  ``QᵀQ + ...`` no pivoting), the role CHOLMOD's factor plays (``GMRF.py:288``);
* ``z = P⁻¹ L⁻ᵀ D^{-1/2} w`` for the requested columns of ``w ~ N(0, I)`` drawn as one
  ``(E, S)`` array from ``numpy.random.default_rng(seed)``;
* unit marginal standard deviation from ``diag(Q⁻¹)`` (Takahashi recurrences), the
  exact form of the reference's empirical rescale (``GMRF.py:326-328``).

The two sparse kernels are C (``oracle/gmrf_oracle.c``, built into ``oracle/_ref`` by
``oracle/Makefile``).
"""
from __future__ import annotations

import ctypes as C
import glob
import os

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def load_library():
    """``oracle/_ref/libgmrf_oracle.so`` or ``None`` when it is not built."""
    global _lib
    if _lib is None:
        paths = glob.glob(os.path.join(_HERE, "_ref", "libgmrf_oracle.so"))
        if not paths:
            return None
        lib = C.CDLL(paths[0])
        P, I64 = C.c_void_p, C.c_int64
        lib.oracle_solve_lt.argtypes = [I64, P, P, P, I64, I64, P]
        lib.oracle_marginals.argtypes = [I64, P, P, P, P, P]
        lib.oracle_solve_lt.restype = C.c_int
        lib.oracle_marginals.restype = C.c_int
        _lib = lib
    return _lib


def element_adjacency(elements: np.ndarray, n_nodes: int):
    """(rows, cols) of every ordered pair of triangles sharing an edge."""
    e = np.asarray(elements, dtype=np.int64)
    E = e.shape[0]
    a = np.concatenate([e[:, 0], e[:, 1], e[:, 2]])
    b = np.concatenate([e[:, 1], e[:, 2], e[:, 0]])
    key = np.minimum(a, b) * n_nodes + np.maximum(a, b)
    eid = np.tile(np.arange(E, dtype=np.int64), 3)
    order = np.argsort(key, kind="stable")
    key, eid = key[order], eid[order]
    same = key[1:] == key[:-1]
    r, c = eid[:-1][same], eid[1:][same]
    return np.concatenate([r, c]), np.concatenate([c, r])


def precision_matrix(elements, n_nodes, tau=0.1) -> sp.csc_matrix:
    E = int(np.asarray(elements).shape[0])
    r, c = element_adjacency(elements, n_nodes)
    adj = sp.coo_matrix((np.ones(len(r)), (r, c)), shape=(E, E)).tocsr()
    adj.data[:] = 1.0
    deg = np.asarray(adj.sum(axis=1)).ravel()
    return (sp.diags(deg + tau) - adj).tocsc()


class GMRFOracle:
    def __init__(self, elements, n_nodes, tau=0.1):
        lib = load_library()
        if lib is None:
            raise RuntimeError("oracle/_ref/libgmrf_oracle.so is not built (make -C oracle)")
        self.lib = lib
        Q = precision_matrix(elements, n_nodes, tau)
        self.n = Q.shape[0]
        lu = sla.splu(Q, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0,
                      options=dict(SymmetricMode=True, Equil=False))
        if not np.array_equal(lu.perm_r, lu.perm_c):
            raise RuntimeError("the factorisation pivoted")
        self.perm = lu.perm_r.copy()
        self.d = lu.U.diagonal().copy()
        L = lu.L.tocsc()
        L.sort_indices()
        self.colptr = np.ascontiguousarray(L.indptr, dtype=np.int64)
        self.rowind = np.ascontiguousarray(L.indices, dtype=np.int64)
        self.lval = np.ascontiguousarray(L.data, dtype=np.float64)
        self._var = None

    def marginal_variance(self) -> np.ndarray:
        if self._var is None:
            out = np.empty(self.n)
            rc = self.lib.oracle_marginals(self.n, self.colptr.ctypes.data,
                                           self.rowind.ctypes.data, self.lval.ctypes.data,
                                           self.d.ctypes.data, out.ctypes.data)
            if rc != 0:
                raise RuntimeError("oracle_marginals: malformed factor")
            self._var = out[self.perm]
        return self._var

    def sample(self, n_samples: int, seed: int, columns=None) -> np.ndarray:
        """Columns ``columns`` (default all) of the (E, n_samples) unit-marginal field."""
        w = np.random.default_rng(seed).standard_normal((self.n, n_samples))
        cols = np.arange(n_samples) if columns is None else np.asarray(columns)
        zp = np.ascontiguousarray(w[:, cols] / np.sqrt(self.d)[:, None])
        del w
        rc = self.lib.oracle_solve_lt(self.n, self.colptr.ctypes.data, self.rowind.ctypes.data,
                                      self.lval.ctypes.data, zp.shape[1], zp.shape[1],
                                      zp.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle_solve_lt: bad argument")
        return zp[self.perm] / np.sqrt(self.marginal_variance())[:, None]


def material(elements, n_nodes, n_samples, columns, seed_E=23, seed_h=24, E0=7.0e6,
             sigma_logE=0.2, h0=0.04, sigma_logh=0.1, tau=0.1):
    """Per-element ``E = E0 exp(sE z)``, ``h = h0 exp(sh z')`` for the chosen columns of an
    ensemble of ``n_samples``."""
    g = GMRFOracle(elements, n_nodes, tau)
    z = g.sample(n_samples, seed_E, columns)
    zh = g.sample(n_samples, seed_h, columns)
    return E0 * np.exp(sigma_logE * z), h0 * np.exp(sigma_logh * zh)
