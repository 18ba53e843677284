"""Solid wall meshes for the ensemble membrane time step.

The reference reads a VTP wall surface (``mesh.py:130-173``) and builds a
``SolidMesh`` (``mesh.py:591-746``).  VTK is not part of this package: wall
meshes come from a structured tube generator (straight or stenosed) or from
plain arrays / ``.npz`` files.  The attribute names follow the reference's
``SolidMesh`` so that the solver class can consume either.

Node numbering of a generated tube is ring-major: node ``j*nc + i`` sits on
axial ring ``j`` at angle ``2*pi*i/nc``.  Every quad is split along the same
diagonal and wound so that the element normal (third row of the local frame,
``optimizedSolidAssemble.pyx:103-106``) points out of the tube.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

__all__ = [
    "TubeGeometry", "tube_mesh", "stenosis_radius", "SolidMesh",
    "special_assignment", "sparse_pattern", "element_adjacency",
]


def stenosis_radius(x: np.ndarray, r0: float = 0.3, depth: float = 0.5,
                    center: float = 2.5, width: float = 0.3) -> np.ndarray:
    """Radius of the stenosed tube: r0 * (1 - depth * exp(-((x - center)/width)^2))."""
    return r0 * (1.0 - depth * np.exp(-((x - center) / width) ** 2))


@dataclass
class TubeGeometry:
    """Structured tube: ``nc`` nodes around, ``na`` rings along ``length``."""
    nc: int
    na: int
    length: float
    radius: float = 0.3
    radius_fn: Optional[Callable[[np.ndarray], np.ndarray]] = None

    @property
    def n_nodes(self) -> int:
        return self.nc * self.na

    @property
    def n_elements(self) -> int:
        return 2 * self.nc * (self.na - 1)


def tube_mesh(geom: TubeGeometry):
    """Return ``(nodes (N,3) f64, elements (E,3) int64, inlet ring, outlet ring)``.

    Quad ``(j, i)`` has corners n00=(j,i), n01=(j,i+1), n10=(j+1,i), n11=(j+1,i+1)
    (``i`` wraps).  It splits into (n00, n01, n11) and (n00, n11, n10); both have
    (n1-n0)x(n2-n0) along +e_r, i.e. outward.
    """
    nc, na = int(geom.nc), int(geom.na)
    if nc < 3 or na < 2:
        raise ValueError("a tube needs nc >= 3 and na >= 2")
    x = np.linspace(0.0, float(geom.length), na)
    r = geom.radius_fn(x) if geom.radius_fn is not None else np.full(na, float(geom.radius))
    th = 2.0 * np.pi * np.arange(nc) / nc
    nodes = np.empty((na, nc, 3))
    nodes[:, :, 0] = r[:, None] * np.cos(th)[None, :]
    nodes[:, :, 1] = r[:, None] * np.sin(th)[None, :]
    nodes[:, :, 2] = x[:, None]
    nodes = nodes.reshape(-1, 3)

    j = np.arange(na - 1)[:, None]
    i = np.arange(nc)[None, :]
    n00 = j * nc + i
    n01 = j * nc + (i + 1) % nc
    n10 = (j + 1) * nc + i
    n11 = (j + 1) * nc + (i + 1) % nc
    elems = np.empty((na - 1, nc, 2, 3), dtype=np.int64)
    elems[:, :, 0] = np.stack([n00, n01, n11], axis=-1)
    elems[:, :, 1] = np.stack([n00, n11, n10], axis=-1)
    elems = elems.reshape(-1, 3)
    inlet = np.arange(nc, dtype=np.int64)
    outlet = (na - 1) * nc + np.arange(nc, dtype=np.int64)
    return nodes, elems, inlet, outlet


def element_adjacency(elements: np.ndarray, n_nodes: int):
    """Edge-adjacency of triangles: (rows, cols) of every ordered pair sharing an edge."""
    e = np.asarray(elements, dtype=np.int64)
    E = e.shape[0]
    a = np.concatenate([e[:, 0], e[:, 1], e[:, 2]])
    b = np.concatenate([e[:, 1], e[:, 2], e[:, 0]])
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = lo * n_nodes + hi
    eid = np.tile(np.arange(E, dtype=np.int64), 3)
    order = np.argsort(key, kind="stable")
    key, eid = key[order], eid[order]
    same = key[1:] == key[:-1]
    r = eid[:-1][same]
    c = eid[1:][same]
    return np.concatenate([r, c]), np.concatenate([c, r])


def sparse_pattern(elements: np.ndarray, n_nodes: int):
    """Node-graph CSR including the diagonal, sorted columns (``sparse.py:36-64``)."""
    e = np.asarray(elements, dtype=np.int64)
    rows = np.repeat(e, 3, axis=1).ravel()
    cols = np.tile(e, (1, 3)).ravel()
    key = np.unique(rows * n_nodes + cols)
    r = key // n_nodes
    c = key % n_nodes
    indptr = np.zeros(n_nodes + 1, dtype=np.int64)
    np.add.at(indptr, r + 1, 1)
    indptr = np.cumsum(indptr)
    return indptr, c.astype(np.int64)


def special_assignment(elements: np.ndarray, n_nodes: int, boundary: np.ndarray):
    """Single-rank renumbering with boundary nodes first (``meshPartition.py:240-254``).

    Returns ``(lclNodeIds, lclElmNodeIds, lclBoundary, lclNSpecialHead)``:
    local node ``k`` is global node ``lclNodeIds[k]``; the clamped rows are the
    first ``lclNSpecialHead`` local nodes.
    """
    boundary = np.asarray(boundary, dtype=np.int64)
    lcl = np.empty(n_nodes, dtype=np.int64)
    nb = len(boundary)
    lcl[:nb] = boundary
    allids = np.arange(n_nodes, dtype=np.int64)
    lcl[nb:] = allids[~np.isin(allids, boundary)]
    sorter = np.argsort(lcl)
    lcl_elm = sorter[np.searchsorted(lcl, elements, sorter=sorter)]
    lcl_bdy = np.where(np.isin(lcl, boundary))[0]
    return lcl, lcl_elm.astype(np.int64), lcl_bdy.astype(np.int64), nb


@dataclass
class SolidMesh:
    """Wall mesh plus per-sample material fields.

    Mirrors the attributes the reference ``SolidMesh`` exposes to the solid
    solvers (``mesh.py:591-680``, ``meshPartition.py:240-254``).  Material is
    given per element and sample (``elmE``, ``elmThick``, shape (E, S)); nodal
    fields ``vE``/``vthickness`` (N, S) are accepted too and are then
    interpolated to the quadrature points as ``physicsSolver.py:146-165`` does.
    """
    nodes: np.ndarray
    elementNodeIds: np.ndarray
    boundary: np.ndarray
    nSmp: int
    density: float = 1.0
    v: float = 0.49
    damp: float = 0.0
    bdyU: float = 0.0
    elmE: Optional[np.ndarray] = None
    elmThick: Optional[np.ndarray] = None
    vE: Optional[np.ndarray] = None
    vthickness: Optional[np.ndarray] = None
    coefK: Optional[np.ndarray] = None
    gthick: Optional[np.ndarray] = None
    iniU: Optional[np.ndarray] = None
    iniDu: Optional[np.ndarray] = None
    name: str = "wall"
    mass_lumping: str = "reference"
    dof: int = 3
    colorGroups: Optional[list] = field(default=None, repr=False)

    def __post_init__(self):
        self.nodes = np.ascontiguousarray(self.nodes, dtype=np.float64)
        self.elementNodeIds = np.ascontiguousarray(self.elementNodeIds, dtype=np.int64)
        self.boundary = np.ascontiguousarray(self.boundary, dtype=np.int64)
        self.nNodes = int(self.nodes.shape[0])
        self.nElements = int(self.elementNodeIds.shape[0])
        self.gnElements = self.nElements
        self.ndof = self.dof * self.nNodes
        if self.iniU is None:
            self.iniU = np.zeros(self.ndof)
        if self.iniDu is None:
            self.iniDu = np.zeros(self.ndof)
        if self.elmE is None and self.vE is None and self.coefK is None:
            raise ValueError("SolidMesh needs elmE/elmThick, vE/vthickness or coefK/gthick")
        # Single-rank partition: boundary first (reference SpecialAssignment).
        (self.lclNodeIds, self.lclElmNodeIds, self.lclBoundary,
         self.lclNSpecialHead) = special_assignment(self.elementNodeIds, self.nNodes, self.boundary)
        self.lclNNodes = self.nNodes
        self.lclNBoundary = self.lclNSpecialHead
        self.lclNCommNodes = 0

    # -- quadrature-point material, as physicsSolver.py:146-165 and :199-202 --
    def element_coefficients(self):
        """Return ``(coefK (E,S), elmGThick (E,S,3))`` in the reference's meaning.

        Per-element fields give ``coefK = E*h`` and ``elmGThick[:,:,g] = h``.
        Nodal fields are interpolated at the 3 mid-edge points with weight 1/3.
        Explicit ``coefK``/``gthick`` (the reference's own arrays) take precedence.
        """
        if self.coefK is not None:
            return (np.ascontiguousarray(self.coefK, dtype=np.float64),
                    np.ascontiguousarray(self.gthick, dtype=np.float64))
        if self.elmE is not None:
            E = np.asarray(self.elmE, dtype=np.float64)
            h = np.asarray(self.elmThick, dtype=np.float64)
            coefK = np.ascontiguousarray(E * h)
            gthick = np.ascontiguousarray(np.repeat(h[:, :, None], 3, axis=2))
            return coefK, gthick
        gps = np.array([[0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
        wt = np.full(3, 1.0 / 3.0)
        ve = np.asarray(self.vE)[self.elementNodeIds, :].swapaxes(1, 2)
        vh = np.asarray(self.vthickness)[self.elementNodeIds, :].swapaxes(1, 2)
        gE = ve @ gps.T
        gH = np.ascontiguousarray(vh @ gps.T)
        coefK = np.ascontiguousarray((gH * gE) @ wt)
        return coefK, gH

    # -- the OpenCL class's material, physicsSolverSDampGPUs.py:160-175 --
    def opencl_coefficients(self):
        """Return ``(elmTE (E,S), nodal thickness at the element's nodes (E,S,3))`` as the
        OpenCL solver class builds them: the stiffness coefficient is the mean over the
        element's three nodes of ``E * h`` (``physicsSolverSDampGPUs.py:166-175``) and the
        mass uses the thickness of each node (``assemble_K_M_P``,
        ``physicsSolverSDampGPUs.cl:174-223``).  Per-element fields are constant over the
        element's nodes."""
        if self.vE is not None and self.coefK is None and self.elmE is None:
            ve = np.asarray(self.vE, dtype=np.float64)[self.elementNodeIds, :]       # (E,3,S)
            vh = np.asarray(self.vthickness, dtype=np.float64)[self.elementNodeIds, :]
            elm_te = np.ascontiguousarray((ve * vh).mean(axis=1))
            return elm_te, np.ascontiguousarray(vh.swapaxes(1, 2))
        coefK, gthick = self.element_coefficients()
        h = gthick.mean(axis=2) if gthick.ndim == 3 else gthick
        return coefK, np.ascontiguousarray(np.repeat(h[:, :, None], 3, axis=2))

    def element_moduli(self):
        """Young's modulus per element and sample (E,S): the mean over the three quadrature
        points, as the stress recovery uses it (``physicsSolver.py:416-424``).  With only
        explicit ``coefK``/``gthick`` arrays it is ``coefK`` over the mean thickness."""
        if self.elmE is not None and self.coefK is None:
            return np.ascontiguousarray(self.elmE, dtype=np.float64)
        if self.vE is not None and self.coefK is None:
            gps = np.array([[0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
            ve = np.asarray(self.vE)[self.elementNodeIds, :].swapaxes(1, 2)
            return np.ascontiguousarray((ve @ gps.T).mean(axis=2))
        coefK, gthick = self.element_coefficients()
        h = gthick.mean(axis=2) if gthick.ndim == 3 else gthick
        return np.ascontiguousarray(coefK / h)

    def UpdateCoordinates(self, u):
        """Deformed coordinates per sample (``mesh.py:678-680``): (S, N, 3)."""
        return (np.tile(self.nodes, (self.nSmp, 1, 1)).reshape(self.nSmp, self.ndof)
                + np.asarray(u).T).reshape(self.nSmp, self.nNodes, self.dof)

    def save_npz(self, path):
        np.savez(path, nodes=self.nodes, elements=self.elementNodeIds, boundary=self.boundary,
                 elmE=self.elmE, elmThick=self.elmThick, density=self.density, v=self.v,
                 damp=self.damp, bdyU=self.bdyU)

    @classmethod
    def from_npz(cls, path, nSmp=None):
        d = np.load(path)
        elmE = d["elmE"]
        S = elmE.shape[1] if nSmp is None else nSmp
        return cls(nodes=d["nodes"], elementNodeIds=d["elements"], boundary=d["boundary"],
                   nSmp=S, density=float(d["density"]), v=float(d["v"]), damp=float(d["damp"]),
                   bdyU=float(d["bdyU"]), elmE=elmE[:, :S], elmThick=d["elmThick"][:, :S])


def min_altitude(nodes: np.ndarray, elements: np.ndarray) -> float:
    """Smallest triangle altitude (used by the CFL rule ``0.5*h_min/sqrt(E_max/rho)``)."""
    p = nodes[elements]
    e0 = p[:, 2] - p[:, 1]
    e1 = p[:, 0] - p[:, 2]
    e2 = p[:, 1] - p[:, 0]
    area2 = np.linalg.norm(np.cross(e0, -e1), axis=1)
    longest = np.max(np.stack([np.linalg.norm(e0, axis=1), np.linalg.norm(e1, axis=1),
                               np.linalg.norm(e2, axis=1)]), axis=0)
    return float(np.min(area2 / longest))


def cfl_dt(nodes, elements, e_max: float, rho: float, safety: float = 0.5) -> float:
    """Per-tube time step ``safety * h_min / sqrt(E_max/rho)``."""
    return safety * min_altitude(nodes, elements) / math.sqrt(e_max / rho)
