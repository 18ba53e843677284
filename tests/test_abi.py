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


def test_tuning_setters_validate_and_round_trip(lib):
    """Host-only tuning knobs: arguments are checked, values read back."""
    saved = _lib.get_step_prefetch(32)
    try:
        _lib.set_step_prefetch(32, 300, 1)
        assert _lib.get_step_prefetch(32) == dict(distance=300, parts=1)
        for bad in ((32, -2, 3), (32, (1 << 20) + 1, 3), (16, 4, 3), (32, 4, 8), (32, 4, -2)):
            assert lib.cvfes_set_step_prefetch(*bad) == _lib.CVFES_ERR_ARG
            assert "cvfes_set_step_prefetch" in _lib.last_error()
        assert _lib.get_step_prefetch(32) == dict(distance=300, parts=1)
        _lib.set_step_prefetch(32)  # automatic: from the mesh's bandwidth and samples
        assert _lib.get_step_prefetch(32) == dict(distance=-1, parts=-1)
        _lib.set_step_prefetch(32, 80, 7)  # bit 2: own rows into L1
        assert _lib.get_step_prefetch(32) == dict(distance=80, parts=7)
        for bad in ((32, 4, 4, 8, 4), (32, 4, 2, 9, 2), (64, 4, 2, 3, 2)):
            assert lib.cvfes_set_step_tuning(*bad) == _lib.CVFES_ERR_ARG
        assert lib.cvfes_set_wait_probe(-1) == _lib.CVFES_ERR_ARG
        assert lib.cvfes_set_wait_probe(0) == _lib.CVFES_OK
        assert lib.cvfes_set_norms_memory(2) == _lib.CVFES_ERR_ARG
        assert lib.cvfes_set_norms_memory(1) == _lib.CVFES_OK
        assert lib.cvfes_set_norms_memory(0) == _lib.CVFES_OK
    finally:
        _lib.set_step_prefetch(32, **saved)
    t = _lib.get_step_tuning(64)
    assert lib.cvfes_set_step_tuning(64, 4, 2, 3, 2) == _lib.CVFES_ERR_ARG  # FP64 vec <= 2
    assert lib.cvfes_set_step_tuning(32, 4, 2, 9, 2) == _lib.CVFES_ERR_ARG  # no variant 9
    assert _lib.get_step_tuning(64) == t
