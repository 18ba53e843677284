"""Mesh generator, renumbering, host preprocessing and the GMRF sampler (CPU)."""
import numpy as np
import pytest

from cvfes_b200.mesh import (SolidMesh, TubeGeometry, cfl_dt, special_assignment, sparse_pattern,
                             stenosis_radius, tube_mesh)


def test_tube_counts_and_pattern():
    for nc, na in [(8, 6), (64, 128)]:
        nodes, elems, inl, outl = tube_mesh(TubeGeometry(nc, na, 3.0))
        assert nodes.shape == (nc * na, 3)
        assert elems.shape == (2 * nc * (na - 1), 3)
        indptr, indices = sparse_pattern(elems, len(nodes))
        assert len(indices) == 7 * nc * na - 4 * nc


def test_outward_normals():
    nodes, elems, _, _ = tube_mesh(TubeGeometry(16, 5, 2.0, 0.5))
    p = nodes[elems]
    n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    c = p.mean(axis=1)
    radial = c.copy()
    radial[:, 2] = 0.0
    assert np.all(np.sum(n * radial, axis=1) > 0)


def test_stenosis_radius():
    x = np.array([0.0, 2.5, 5.0])
    r = stenosis_radius(x)
    assert abs(r[1] - 0.15) < 1e-12 and abs(r[0] - 0.3) < 1e-6


def test_special_assignment_boundary_first():
    nodes, elems, inl, outl = tube_mesh(TubeGeometry(8, 6, 3.0))
    bdy = np.concatenate([inl, outl])
    lcl, lel, lb, nb = special_assignment(elems, len(nodes), bdy)
    assert nb == 16 and np.array_equal(lcl[:16], bdy)
    assert np.array_equal(lb, np.arange(16))
    assert np.array_equal(lcl[lel], elems)


def test_incidence_fans(lib):
    from cvfes_b200.plan import incidence
    nodes, elems, _, _ = tube_mesh(TubeGeometry(8, 6, 3.0))
    node_ptr, rec, elem_slot = incidence(elems, len(nodes))
    assert node_ptr[-1] == 3 * len(elems)
    for e in range(len(elems)):
        for la in range(3):
            s = elem_slot[e, la]
            a = elems[e, la]
            assert node_ptr[a] <= s < node_ptr[a + 1]
            assert rec[s, 0] == e and (rec[s, 3] >> 8) == la
            assert {rec[s, 1], rec[s, 2]} == set(elems[e]) - {a}
    # interior nodes: closed fans of 6, every slot after the first continues the fan
    for a in range(8, 40):
        k0, k1 = node_ptr[a], node_ptr[a + 1]
        assert k1 - k0 == 6
        assert all(rec[k, 3] & 1 for k in range(k0 + 1, k1))
        assert all(rec[k, 1] == rec[k - 1, 2] for k in range(k0 + 1, k1))


def test_incidence_rejects_bad_input(lib):
    from cvfes_b200 import _lib
    from cvfes_b200.plan import incidence
    with pytest.raises(_lib.CvfesError):
        incidence(np.array([[0, 1, 7]]), 3)
    with pytest.raises(_lib.CvfesError):
        incidence(np.array([[0, 1, 1]]), 3)


def test_greedy_colouring_matches_reference_algorithm(lib):
    from cvfes_b200.plan import color_greedy
    nodes, elems, _, _ = tube_mesh(TubeGeometry(10, 7, 3.0))
    colors, n = color_greedy(elems, len(nodes))
    # pure-Python restatement of meshColoring.py:39-56
    E = len(elems)
    node_elems = [[] for _ in range(len(nodes))]
    for e in range(E):
        for a in elems[e]:
            node_elems[a].append(e)
    ref = -np.ones(E, dtype=int)
    for e in range(E):
        used = {ref[q] for a in elems[e] for q in node_elems[a] if ref[q] >= 0}
        c = 0
        while c in used:
            c += 1
        ref[e] = c
    assert np.array_equal(colors, ref) and n == ref.max() + 1
    for e in range(E):  # no two elements of one colour share a node
        for a in elems[e]:
            assert sum(colors[q] == colors[e] for q in node_elems[a]) == 1


def test_colouring_runs_out(lib):
    from cvfes_b200 import _lib
    from cvfes_b200.plan import color_greedy
    nodes, elems, _, _ = tube_mesh(TubeGeometry(10, 7, 3.0))
    with pytest.raises(_lib.CvfesError):
        color_greedy(elems, len(nodes), max_colors=3)


def test_gmrf_exact_variance_and_statistics(lib):
    from cvfes_b200.gmrf import ElementGMRF
    nodes, elems, _, _ = tube_mesh(TubeGeometry(10, 8, 3.0))
    g = ElementGMRF(elems, len(nodes))
    Qinv = np.linalg.inv(g.Q.toarray())
    assert np.abs(g.variance() - np.diag(Qinv)).max() < 1e-12
    z = g.sample(40000, 5)
    assert np.abs(z.std(axis=1) - 1.0).max() < 0.03
    s = np.sqrt(np.diag(Qinv))
    assert np.abs(np.cov(z) - Qinv / np.outer(s, s)).max() < 0.05
    # seeded: same draw twice
    assert np.array_equal(g.sample(3, 11), g.sample(3, 11))


def test_material_and_cfl(lib):
    from cvfes_b200.gmrf import material_fields
    nodes, elems, _, _ = tube_mesh(TubeGeometry(12, 9, 3.0))
    E, h, _ = material_fields(elems, len(nodes), 4)
    assert E.shape == (len(elems), 4) and np.all(E > 0) and np.all(h > 0)
    assert 5e-7 < cfl_dt(nodes, elems, E.max(), 1.0) < 1e-4


def test_solid_mesh_nodal_coefficients():
    nodes, elems, inl, outl = tube_mesh(TubeGeometry(6, 4, 1.0))
    N, S = len(nodes), 2
    m = SolidMesh(nodes, elems, np.concatenate([inl, outl]), S, vE=np.full((N, S), 3.0),
                  vthickness=np.full((N, S), 2.0))
    coefK, gthick = m.element_coefficients()
    assert np.allclose(coefK, 6.0) and np.allclose(gthick, 2.0)


def test_gmrf_matches_oracle_restatement(lib):
    """The product sampler (selected inversion and Lᵀ solve in the library) against the
    oracle's C restatement on the same SuperLU factor: marginal variances and samples."""
    from cvfes_b200.gmrf import ElementGMRF
    from oracle.gmrf_oracle import GMRFOracle, load_library
    if load_library() is None:
        pytest.skip("oracle/_ref/libgmrf_oracle.so not built (make -C oracle restatement)")
    nodes, elems, _, _ = tube_mesh(TubeGeometry(24, 20, 3.0))
    g = ElementGMRF(elems, len(nodes))
    o = GMRFOracle(elems, len(nodes))
    v, vo = g.variance(), o.marginal_variance()
    assert np.max(np.abs(v - vo) / vo) < 1e-12
    z = g.sample(12, seed=5)
    zo = o.sample(12, seed=5, columns=[0, 7, 11])
    assert np.max(np.abs(z[:, [0, 7, 11]] - zo)) < 1e-10


def _reference_module(filename):
    """Import a module of the reference checkout (CVFES_REFERENCE, else `reference` beside
    this repository) with stubs for the modules it imports at load time but the tested
    functions never use (mesh, mpi4py, parmetis).  None when the checkout is absent."""
    import importlib.util
    import os
    import sys
    import types
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    ref = os.environ.get("CVFES_REFERENCE") or os.path.join(root, "reference")
    path = os.path.join(ref, filename)
    if not os.path.exists(path):
        return None
    stubs = {"mesh": types.ModuleType("mesh"), "mpi4py": types.ModuleType("mpi4py"),
             "parmetis": types.ModuleType("parmetis")}
    stubs["mpi4py"].MPI = None
    stubs["parmetis"].PyParMETIS_V3_PartMeshKway = None
    saved = {k: sys.modules.get(k) for k in stubs}
    sys.modules.update(stubs)
    try:
        spec = importlib.util.spec_from_file_location("ref_" + filename[:-3], path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return mod


class _RaggedNumpy:
    """numpy for code written for NumPy 1.x: np.array of ragged lists gives an object
    array (NumPy 2 raises instead); everything else is numpy itself."""

    def __getattr__(self, name):
        return getattr(np, name)

    @staticmethod
    def array(x, *args, **kw):
        try:
            return np.array(x, *args, **kw)
        except ValueError:
            out = np.empty(len(x), dtype=object)
            for i, item in enumerate(x):
                out[i] = item
            return out


def test_greedy_colouring_matches_reference_module(lib, tmp_path, monkeypatch):
    """cvfes_mesh_color_greedy against the reference's own MeshColoring
    (meshColoring.py:7-63), run here on the same mesh: identical colours."""
    from cvfes_b200.plan import color_greedy
    mod = _reference_module("meshColoring.py")
    if mod is None:
        pytest.skip("reference checkout not found")
    mod.np = _RaggedNumpy()
    nodes, elems, inl, outl = tube_mesh(TubeGeometry(16, 12, 3.0))
    lcl, lel, lb, nb = special_assignment(elems, len(nodes), np.concatenate([inl, outl]))
    stub = type("M", (), dict(lclNNodes=len(nodes), nElements=len(elems), lclElmNodeIds=lel))()
    monkeypatch.chdir(tmp_path)
    assert mod.MeshColoring("colors", stub) == 0
    ours, n = color_greedy(lel, len(nodes))
    assert np.array_equal(np.asarray(stub.elmColors, dtype=np.int64), ours.astype(np.int64))
    assert n == len(stub.colorGroups)


def test_special_assignment_matches_reference_module():
    """mesh.special_assignment against the reference's SolidMeshPartition.SpecialAssignment
    (meshPartition.py:240-254), run here: identical numbering."""
    mod = _reference_module("meshPartition.py")
    if mod is None:
        pytest.skip("reference checkout not found")
    mod.np = _RaggedNumpy()
    if not hasattr(np, "in1d"):
        mod.np.in1d = np.isin
    nodes, elems, inl, outl = tube_mesh(TubeGeometry(16, 12, 3.0))
    bdy = np.concatenate([inl, outl])
    stub = type("M", (), dict(nNodes=len(nodes), boundary=bdy, elementNodeIds=elems))()
    mod.SolidMeshPartition.SpecialAssignment(None, stub)
    lcl, lel, lb, nb = special_assignment(elems, len(nodes), bdy)
    assert np.array_equal(stub.lclNodeIds, lcl) and np.array_equal(stub.lclElmNodeIds, lel)
    assert np.array_equal(stub.lclBoundary, lb) and stub.lclNSpecialHead == nb
