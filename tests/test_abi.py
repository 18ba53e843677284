"""The C-ABI library loads and exports every entry point its header declares (no GPU calls)."""
import os
import re

from cvfes_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "cvfes_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cvfes_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "cvfes_solid_step_f32" in names and len(names) >= 20


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_every_declared_symbol_has_a_binding():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_version_and_error_channel(lib):
    assert lib.cvfes_version() >= 100
    rc = lib.cvfes_mesh_incidence(0, 0, None, None, None, None)
    assert rc == _lib.CVFES_ERR_ARG
    assert "cvfes_mesh_incidence" in _lib.last_error()
