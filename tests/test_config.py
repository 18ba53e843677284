"""ConfigObj-subset reader and the reference's config classes."""
import os

import numpy as np
import pytest

from cvfes_b200 import config

ROOT = os.path.dirname(os.path.dirname(__file__))


def test_parse_nested_sections_lists_and_comments():
    txt = """
dimensions = 3
sample_num = 4  # inline comment
[meshes]
    [[mesh 2]]
        name = wall
        file_path = 'a.vtp'
        [[[faces]]]
            [[[[face 1]]]]
                name = boundaries
                file_path = 'in.vtp','out.vtp'
[solver]
    dt = 1.0e-5
    endtime = 0.03
    restart = 1
"""
    root = config.parse(txt)
    assert root.as_int("sample_num") == 4
    face = root["meshes"]["mesh 2"]["faces"]["face 1"]
    assert face["file_path"] == ["in.vtp", "out.vtp"]
    assert root["solver"].as_bool("restart") is True
    assert root["meshes"].sections == ["mesh 2"]


@pytest.mark.parametrize("name", sorted(os.listdir(os.path.join(ROOT, "cfg"))))
def test_shipped_cfgs_load(name):
    cfg = config.load(os.path.join(ROOT, "cfg", name))
    assert cfg.solver.dt > 0 and cfg.nSmp >= 1
    assert cfg.gpu.precision in (32, 64)
    assert "solid" in cfg.equations


def test_sample_override():
    cfg = config.load(os.path.join(ROOT, "cfg", "tube64x128.cfg"), nSmp=3)
    assert cfg.nSmp == 3 and cfg.solver.nSmp == 3


def test_legacy_vtk_round_trip_with_stress(tmp_path):
    """Displacement vectors and per-sample stress cell scalars read back unchanged."""
    from cvfes_b200.io import (STRESS_NAMES, read_legacy_vtk_cell_scalars,
                               read_legacy_vtk_vectors, save_displacement)
    from cvfes_b200.mesh import TubeGeometry, tube_mesh
    nodes, elems, inl, outl = tube_mesh(TubeGeometry(6, 4, 1.0, 0.3))
    rng = np.random.default_rng(3)
    S = 2
    u = rng.standard_normal((S, len(nodes), 3))
    stress = rng.standard_normal((len(elems), S, 5))

    class M:
        pass
    m = M()
    m.nodes, m.elementNodeIds = nodes, elems
    path = save_displacement(str(tmp_path / "wall.vtk"), 3, m, u, stress=stress)
    vec = read_legacy_vtk_vectors(path)
    cells = read_legacy_vtk_cell_scalars(path)
    for s in range(S):
        assert np.array_equal(vec[f"u_{s:03d}"], u[s])
        for c, name in enumerate(STRESS_NAMES):
            assert np.array_equal(cells[f"{name}_{s:03d}"], stress[:, s, c])
    npz = save_displacement(str(tmp_path / "wall.npz"), 3, m, u, stress=stress)
    d = np.load(npz)
    assert np.array_equal(d["stress"], stress) and np.array_equal(d["u"], u)
