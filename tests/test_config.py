"""ConfigObj-subset reader and the reference's config classes."""
import os

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
