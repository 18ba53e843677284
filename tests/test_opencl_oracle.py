"""The OpenCL-class restatement (oracle/opencl_oracle.py) pinned to the reference's
compiled CPU kernels where the two classes compute the same thing (CPU).

With one modulus and one thickness per sample (so mean(E h) over an element's nodes is
the CPU path's coefK and every lumping row sums to rho h A/3, the row-sum mass, i.e.
the CPU reference run with 3 rho), no damping (so both left-hand sides are LM) and
the stiffness and follower pressure rebuilt on x + u every step (the CPU path's
stiffness update interval 1, the OpenCL class's assemble_K_P), the two must give the
same displacement history.
"""
import numpy as np
import pytest

from cvfes_b200.mesh import TubeGeometry, tube_mesh
from oracle import solid_oracle as so
from oracle.opencl_oracle import MASS_W, OpenCLSolidOracle


@pytest.fixture(scope="module")
def tube():
    nodes, elems, inl, outl = tube_mesh(TubeGeometry(8, 6, 3.0, 0.3))
    return nodes, elems, np.concatenate([inl, outl])


def test_mass_weights_are_the_kernel_ab_sums():
    # node 0: ab 00, 01, 02; node 1: ab 01, 11, 12; node 2: ab 02, 12, 22 (kernel's weights)
    ab = {"00": (1 / 4, 1 / 8, 1 / 8), "01": (1 / 8, 1 / 8, 0), "02": (1 / 8, 0, 1 / 8),
          "11": (1 / 8, 1 / 4, 1 / 8), "12": (0, 1 / 8, 1 / 8), "22": (1 / 8, 1 / 4, 1 / 8)}
    rows = [ab["00"], ab["01"], ab["02"]], [ab["01"], ab["11"], ab["12"]], \
        [ab["02"], ab["12"], ab["22"]]
    W = np.array([np.sum(r, axis=0) for r in rows])
    assert np.array_equal(W, MASS_W)


def test_opencl_restatement_matches_reference_kernels(tube):
    if so.load_reference_module() is None:
        pytest.skip("oracle/_ref not built (make -C oracle reference)")
    nodes, elems, bdy = tube
    N, E, S = len(nodes), len(elems), 2
    rng = np.random.default_rng(3)
    Es = 7e6 * np.exp(0.2 * rng.standard_normal(S))
    hs = 0.04 * np.exp(0.1 * rng.standard_normal(S))
    vE, vh = np.tile(Es, (N, 1)), np.tile(hs, (N, 1))
    dt, rho, v = 2e-6, 1.0, 0.49
    pres = 1.33e5 * np.minimum(np.arange(25) / 10.0, 1.0)
    ocl = OpenCLSolidOracle(nodes, elems, bdy, vE, vh, rho, v, 0.0, dt)
    ref = so.OracleSolidSolver(nodes, elems, bdy, np.tile(Es * hs, (E, 1)),
                               np.repeat(np.tile(hs, (E, 1))[:, :, None], 3, axis=2), 3 * rho, v,
                               0.0, dt, backend="reference", update_interval=1)
    assert so.rel_l2(ocl.LM, ref.LM) < 1e-13
    for p in pres:
        a, b = ocl.step(p), ref.step(p)
    assert np.abs(a).max() > 0
    assert so.rel_l2(a, b) < 1e-12


def test_opencl_damping_and_start_up(tube):
    """Damping per dof and the start-up acceleration without damping, restated: one step
    from rest with damping equals the undamped step (the damping force needs a velocity),
    and with an initial velocity the damped state moves less."""
    nodes, elems, bdy = tube
    N, S = len(nodes), 2
    rng = np.random.default_rng(5)
    vE = 7e6 * np.exp(0.2 * rng.standard_normal((N, S)))
    vh = 0.04 * np.exp(0.1 * rng.standard_normal((N, S)))
    a = OpenCLSolidOracle(nodes, elems, bdy, vE, vh, 1.0, 0.49, 0.0, 2e-6)
    b = OpenCLSolidOracle(nodes, elems, bdy, vE, vh, 1.0, 0.49, 50.0, 2e-6)
    assert np.array_equal(a.up, b.up)          # calc_ddu has no damping term
    du0 = np.zeros(3 * N)
    du0[3 * np.setdiff1d(np.arange(N), bdy) + 2] = 1.0
    c = OpenCLSolidOracle(nodes, elems, bdy, vE, vh, 1.0, 0.49, 0.0, 2e-6, du0=du0)
    d = OpenCLSolidOracle(nodes, elems, bdy, vE, vh, 1.0, 0.49, 50.0, 2e-6, du0=du0)
    for _ in range(5):
        uc, ud = c.step(0.0), d.step(0.0)
    assert np.linalg.norm(ud) < np.linalg.norm(uc)
