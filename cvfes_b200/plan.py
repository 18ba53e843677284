"""Device-resident set-up of one membrane mesh for the sm_100a solid step.

A :class:`SolidPlan` owns (as torch CUDA tensors) everything the per-step
kernels read that does not depend on the samples' state:

* the node-centric slot layout (fan-ordered incident elements) built on the
  host by ``cvfes_mesh_incidence``;
* per-slot 3x9 rows of the unit element stiffness ``Kt_e`` (FP64, and an FP32
  copy), built on the GPU by ``cvfes_solid_templates_f64``;
* per-sample material: the stiffness coefficient ``E*h`` per element, the
  lumped mass and its FP64 inverse per node, and the unit-pressure load.

Tables (D, quadrature, lumped-mass weights) follow ``physicsSolver.py:146-197``.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr

SHEAR_K = 5.0 / 6.0
# Mid-edge quadrature of physicsSolver.py:146-148: (N_0, N_1, N_2, weight).
QUAD = np.array([[0.5, 0.5, 0.0, 1.0 / 3.0],
                 [0.5, 0.0, 0.5, 1.0 / 3.0],
                 [0.0, 0.5, 0.5, 1.0 / 3.0]])
SLAB = 28


def d_matrix(v: float, k: float = SHEAR_K) -> np.ndarray:
    """Membrane/transverse-shear constitutive matrix divided by E (physicsSolver.py:184-188)."""
    c = 1.0 - v * v
    D = np.zeros((5, 5))
    D[0, 0] = D[1, 1] = 1.0 / c
    D[0, 1] = D[1, 0] = v / c
    D[2, 2] = 0.5 * (1 - v) / c
    D[3, 3] = D[4, 4] = 0.5 * k * (1 - v) / c
    return D


def lumped_mass_weights(density: float, lumping: str = "reference") -> np.ndarray:
    """Row-sum weights ``mw[a, g]`` of the lumped mass of local node ``a``.

    ``reference``: ``rho * w_g^2 * N_g(a)`` -- the row sum of ``tM_g * w_g``
    (``tM_g = N_gᵀN_g w_g rho``, physicsSolver.py:190-197; the assembly applies
    ``w_g`` a second time, optimizedSolidAssemble.pyx:564-566), one third of
    the element mass per node.
    ``rowsum``: ``rho * w_g * N_g(a)`` -- the row sum of the consistent mass
    matrix (the full rho*h*A/3 per node); equal to ``reference`` with 3 rho.
    ``opencl``: the OpenCL class's lumping of nodal thickness (``assemble_K_M_P``,
    physicsSolverSDampGPUs.cl:174-223): node a gets ``rho A/3 sum_k W[a][k] h_k``
    with ``h_k`` the thickness of the element's node k; its rows are the sums of the
    kernel's ab terms, row 2 with the kernel's own ``ab = 22`` weights (h1/4, not h2/4,
    physicsSolverSDampGPUs.cl:218), so W[2] = (1/4, 3/8, 3/8).  With one thickness per
    element every row sums to rho h A/3, the ``rowsum`` mass."""
    if lumping == "opencl":
        W = np.array([[0.5, 0.25, 0.25], [0.25, 0.5, 0.25], [0.25, 0.375, 0.375]])
        return density * W / 3.0
    w = QUAD[:, 3:4] ** 2 if lumping == "reference" else QUAD[:, 3:4]
    if lumping not in ("reference", "rowsum"):
        raise ValueError("mass lumping must be 'reference', 'rowsum' or 'opencl'")
    return density * (QUAD[:, :3] * w).T.copy()


def incidence(elements: np.ndarray, n_nodes: int):
    """Host call of ``cvfes_mesh_incidence``: (node_ptr, slot_rec (3E,4), elem_slot (E,3))."""
    e = np.ascontiguousarray(elements, dtype=np.int64)
    E = e.shape[0]
    node_ptr = np.empty(n_nodes + 1, dtype=np.int32)
    slot_rec = np.empty((3 * E, 4), dtype=np.int32)
    elem_slot = np.empty((E, 3), dtype=np.int32)
    call("cvfes_mesh_incidence", n_nodes, E, ptr(e), ptr(node_ptr), ptr(slot_rec), ptr(elem_slot))
    return node_ptr, slot_rec, elem_slot


def color_greedy(elements: np.ndarray, n_nodes: int, max_colors: int = 23):
    """Host call of ``cvfes_mesh_color_greedy`` (meshColoring.py semantics)."""
    e = np.ascontiguousarray(elements, dtype=np.int64)
    colors = np.empty(e.shape[0], dtype=np.int32)
    n = call("cvfes_mesh_color_greedy", n_nodes, e.shape[0], ptr(e), max_colors, ptr(colors))
    return colors, n


def numbering_bandwidth(elements: np.ndarray, n_clamped: int) -> int:
    """Largest id distance between two unclamped nodes of one element: how far ahead of
    a node its neighbours' rows lie (the clamped prefix is left out; its rows are few and
    read by every end-ring node, so the step kernels keep them cached anyway)."""
    e = np.asarray(elements, dtype=np.int64)
    if e.size == 0:
        return 0
    free = e >= n_clamped
    hi = np.where(free, e, -1).max(axis=1)
    lo = np.where(free, e, np.iinfo(np.int64).max).min(axis=1)
    ok = hi >= 0
    return int(np.max(hi[ok] - lo[ok])) if ok.any() else 0


class SolidPlan:
    """Mesh-dependent device data of the solid step (one mesh, local numbering).

    ``nodes (N,3)`` and ``elements (E,3)`` must already be in the solver's local
    numbering with the clamped nodes first (``n_clamped`` of them).
    """

    def __init__(self, nodes, elements, n_clamped: int, clamp_value: float, v: float,
                 density: float, device="cuda", precisions=(32, 64), keep_full=False,
                 mass_lumping: str = "reference"):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("SolidPlan needs a CUDA device; there is no CPU path")
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        elements = np.ascontiguousarray(elements, dtype=np.int64)
        self.N = int(nodes.shape[0])
        self.E = int(elements.shape[0])
        self.n_clamped = int(n_clamped)
        self.clamp_value = float(clamp_value)
        self.v = float(v)
        self.density = float(density)
        self.mass_lumping = mass_lumping
        self.precisions = tuple(precisions)
        node_ptr, slot_rec, elem_slot = incidence(elements, self.N)
        self.host_node_ptr, self.host_slot_rec = node_ptr, slot_rec
        self.max_degree = int(np.max(np.diff(node_ptr))) if self.N > 0 else 0
        self.bandwidth = numbering_bandwidth(elements, self.n_clamped)
        dev = self.device
        self.stream = torch.cuda.current_stream(dev)
        self.nodes = torch.from_numpy(nodes).to(dev)
        self.elems = torch.from_numpy(elements.astype(np.int32)).to(dev)
        self.node_ptr = torch.from_numpy(node_ptr).to(dev)
        self.slot_rec = torch.from_numpy(slot_rec).to(dev)
        self.elem_slot = torch.from_numpy(elem_slot).to(dev)
        ns = 3 * self.E
        self.slot_k64 = torch.empty(SLAB * ns, dtype=torch.float64, device=dev) if 64 in self.precisions else None
        self.slot_k32 = torch.empty(SLAB * ns, dtype=torch.float32, device=dev) if 32 in self.precisions else None
        self.kt_full = torch.empty(self.E * 81, dtype=torch.float64, device=dev) if keep_full else None
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.area = torch.empty(self.E, dtype=torch.float64, device=dev)
        self.normal = torch.empty(3 * self.E, dtype=torch.float64, device=dev)
        D = np.ascontiguousarray(d_matrix(self.v))
        with torch.cuda.device(dev):
            call("cvfes_solid_templates_f64", self.N, self.E, ptr(self.nodes), ptr(self.elems),
                 ptr(D), ptr(self.elem_slot), ptr(self.slot_rec), ptr(self.slot_k64),
                 ptr(self.slot_k32), ptr(self.kt_full), ptr(self.area), ptr(self.normal),
                 self._s())
        self.S = None
        self.build_tiles()

    def build_tiles(self, P: int = 16, H: int = 18, W: int = 3, EH: int = 36, WE: int = 2):
        """Strip tiling for the TMA-tiled step (``cvfes_mesh_tiles``): tiles of P nodes,
        W windows of H node ids and WE windows of EH element ids per tile."""
        nt = (self.N + P - 1) // P
        tw = np.empty((nt, W + WE), dtype=np.int32)
        tr = np.empty((3 * self.E, 4), dtype=np.int32)
        nl = np.empty(self.N, dtype=np.int32)
        st = np.zeros(4, dtype=np.int64)
        call("cvfes_mesh_tiles", self.N, self.E, ptr(self.host_node_ptr), ptr(self.host_slot_rec),
             self.n_clamped, P, H, W, EH, WE, ptr(tw), ptr(tr), ptr(nl), ptr(st))
        dev = self.device
        self.tile_win = torch.from_numpy(tw).to(dev)
        self.tile_rec = torch.from_numpy(tr).to(dev)
        self.node_loc = torch.from_numpy(nl).to(dev)
        self.tile_shape = (P, H, W, EH, WE)
        self.tile_stats = dict(tiles=int(st[0]), node_outliers=int(st[1]),
                               element_outliers=int(st[2]), most_windows=int(st[3]))

    def _s(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    # ------------------------------------------------------------------ material
    def set_material(self, coefK, gthick):
        """Per-sample material: ``coefK (E,S)`` = E*h weighted at the quadrature points and
        thickness ``gthick`` as ``(E,S)`` (uniform per element) or ``(E,S,3)``."""
        dev = self.device
        coef64 = torch.as_tensor(np.ascontiguousarray(coefK, dtype=np.float64)).to(dev)
        g = np.ascontiguousarray(gthick, dtype=np.float64)
        if g.ndim == 3 and np.all(g == g[:, :, :1]):
            g = np.ascontiguousarray(g[:, :, 0])
        n_gauss = 1 if g.ndim == 2 else 3
        if coef64.shape[0] != self.E or g.shape[0] != self.E or g.shape[1] != coef64.shape[1]:
            raise ValueError("coefK/gthick must be (E,S) / (E,S[,3]) for this mesh")
        S = int(coef64.shape[1])
        self.S = S
        gth = torch.from_numpy(g).to(dev)
        self.coef64 = coef64 if 64 in self.precisions else None
        self.coef32 = coef64.to(torch.float32) if 32 in self.precisions else None
        self.lm = torch.empty((self.N, S), dtype=torch.float64, device=dev)
        self.invm64 = torch.empty((self.N, S), dtype=torch.float64, device=dev)
        self.invm32 = torch.empty((self.N, S), dtype=torch.float32, device=dev)
        self.fhat64 = torch.empty((self.N, 4), dtype=torch.float64, device=dev)
        self.fhat32 = torch.empty((self.N, 4), dtype=torch.float32, device=dev)
        mw = np.ascontiguousarray(lumped_mass_weights(self.density, self.mass_lumping))
        with torch.cuda.device(dev):
            call("cvfes_solid_mass_load_f64", self.N, self.E, S, ptr(self.node_ptr),
                 ptr(self.slot_rec), ptr(self.area), ptr(self.normal), ptr(gth), n_gauss,
                 ptr(mw), ptr(self.lm), ptr(self.invm64), ptr(self.invm32), ptr(self.fhat64),
                 ptr(self.fhat32), self._s())
        del gth
        if 64 not in self.precisions:
            self.invm64 = None
        return self

    def coef(self, precision):
        return self.coef64 if precision == 64 else self.coef32

    def invm(self, precision):
        return self.invm64 if precision == 64 else self.invm32

    def desc(self, precision: int) -> _lib.SolidMeshDesc:
        """C descriptor of this mesh for FP32 or FP64 kernels (valid while self lives)."""
        if self.S is None:
            raise RuntimeError("set_material() first")
        slab = self.slot_k64 if precision == 64 else self.slot_k32
        fhat = self.fhat64 if precision == 64 else self.fhat32
        if slab is None:
            raise RuntimeError(f"plan was built without FP{precision} templates")
        d = _lib.SolidMeshDesc(self.N, self.E, self.S, self.n_clamped, self.clamp_value,
                               ptr(self.node_ptr), ptr(self.slot_rec), ptr(slab), ptr(fhat),
                               self.max_degree, ptr(self.status))
        d.bandwidth = self.bandwidth
        if getattr(self, "tile_win", None) is not None:
            P, H, W, EH, WE = self.tile_shape
            d.tile_win, d.tile_rec, d.node_loc = (ptr(self.tile_win), ptr(self.tile_rec),
                                                  ptr(self.node_loc))
            d.tile_p, d.tile_h, d.tile_w, d.tile_eh, d.tile_we = P, H, W, EH, WE
        return d

    def check_status(self):
        """Raise if a bounded device wait gave up since the last check (syncs the stream)."""
        call("cvfes_status_read", ptr(self.status), self._s())
