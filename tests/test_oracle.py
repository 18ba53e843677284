"""The CPU oracle against the reference's own kernels and the golden fixtures."""
import os

import numpy as np
import pytest

from oracle import solid_oracle as so

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["tube8x6_element.npz", "tube6x5_nodal.npz"]


def _load(name):
    return dict(np.load(os.path.join(GOLD, name)))


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("name", CASES)
def test_restatement_matches_golden_assembly(name):
    g = _load(name)
    M, C, K, f, LM, LC = so.assemble_with_damping(
        g["nodes"], g["elements"], g["coefK"], g["gthick"], float(g["density"]), float(g["v"]),
        float(g["damp"]), g["indptr"], g["indices"])
    assert _rel(K, g["K"]) < 1e-13
    assert _rel(M, g["M"]) < 1e-13
    if float(g["damp"]) > 0:
        assert _rel(C, g["C"]) < 1e-13
    assert _rel(f, g["f"]) < 1e-13
    assert _rel(LM, g["LM"]) < 1e-13


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("backend", ["numpy", "template"])
def test_restatement_matches_golden_history(name, backend):
    g = _load(name)
    o = so.OracleSolidSolver(g["nodes"], g["elements"], g["boundary"], g["coefK"], g["gthick"],
                             float(g["density"]), float(g["v"]), float(g["damp"]), float(g["dt"]),
                             backend=backend)
    assert so.rel_l2(o.up, g["up0"]) < 1e-13 or np.abs(g["up0"]).max() == 0
    hist = o.run(g["pressures"], history_every=5)
    for h, ref in zip(hist, g["hist"]):
        assert so.rel_l2(h, ref) < 1e-12


def test_pattern_matches_golden():
    g = _load(CASES[0])
    indptr, indices = so._pattern(g["elements"], len(g["nodes"]))
    assert np.array_equal(indptr, g["indptr"]) and np.array_equal(indices, g["indices"])


def test_multiply_by_vector_against_reference_module():
    ref = so.load_reference_module()
    if ref is None:
        pytest.skip("oracle/_ref not built (make -C oracle)")
    g = _load(CASES[0])
    rng = np.random.default_rng(0)
    v = rng.standard_normal(g["LM"].shape)
    res_ref = np.zeros_like(v)
    ref.MultiplyByVector(g["indptr"], g["indices"], g["K"], v, res_ref)
    res = so.multiply_by_vector(g["indptr"], g["indices"], g["K"], v)
    assert _rel(res, res_ref) < 1e-14


def test_rigid_translation_in_null_space():
    g = _load(CASES[0])
    N = len(g["nodes"])
    t = np.tile(np.array([0.3, -0.2, 0.7]), N)[:, None] * np.ones((1, g["K"].shape[1]))
    r = so.multiply_by_vector(g["indptr"], g["indices"], g["K"], t)
    scale = np.abs(g["K"]).max() * 1.0
    assert np.abs(r).max() < 1e-12 * scale


def test_closed_tube_net_pressure_force_is_axial_only():
    g = _load(CASES[0])
    f = g["f"].reshape(-1, 3)
    # radial components cancel on a closed ring; the open ends leave no axial load either
    assert np.abs(f[:, 0].sum()) < 1e-12 * np.abs(f).sum()
    assert np.abs(f[:, 1].sum()) < 1e-12 * np.abs(f).sum()


@pytest.mark.parametrize("name", ["tube8x6_geo1.npz", "tube8x6_geo3.npz"])
def test_geometric_update_restatement_matches_golden_history(name):
    """Stiffness and follower pressure rebuilt on x + u (OptimizedSolidAssembleUpdate,
    pyx:710-819) every 1 / 3 steps: the NumPy restatement against the reference run."""
    g = dict(np.load(os.path.join(GOLD, name)))
    o = so.OracleSolidSolver(g["nodes"], g["elements"], g["boundary"], g["coefK"], g["gthick"],
                             float(g["density"]), float(g["v"]), float(g["damp"]), float(g["dt"]),
                             backend="numpy", update_interval=int(g["update_interval"]))
    hist = o.run(g["pressures"], history_every=5)
    for h, ref in zip(hist, g["hist"]):
        assert _rel(h, ref) < 1e-12


@pytest.mark.parametrize("name", ["tube8x6_element.npz", "tube6x5_nodal.npz",
                                  "tube8x6_geo1.npz", "tube8x6_geo3.npz"])
def test_stress_restatement_matches_golden(name):
    """Element stresses (OptimizedCalculateStress, pyx:1116-1223) of the final state, on the
    undeformed geometry or on the geometry of the last update."""
    g = dict(np.load(os.path.join(GOLD, name)))
    o = so.OracleSolidSolver(g["nodes"], g["elements"], g["boundary"], g["coefK"], g["gthick"],
                             float(g["density"]), float(g["v"]), float(g["damp"]), float(g["dt"]),
                             backend="numpy", update_interval=int(g["update_interval"]))
    o.run(g["pressures"])
    assert _rel(o.stress(g["young"]), g["stress"]) < 1e-12
