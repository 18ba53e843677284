"""Generate the golden fixtures of the solid path with the reference's own kernels.

Runs the reference's compiled ``optimizedSolidAssemble`` (built from the
reference sources by ``oracle/Makefile`` into ``oracle/_ref``) on two tiny
synthetic tubes and stores inputs and outputs in ``tests/golden/*.npz``:

* ``tube8x6_element.npz``: per-element E and h (coefK = E*h, thickness at the 3
  quadrature points = h), 3 samples, damping 100, linear pressure ramp, 30 steps;
* ``tube6x5_nodal.npz``: nodal E and h interpolated to the quadrature points as
  ``physicsSolver.py:146-165`` does, 2 samples, no damping, 20 steps;
* ``tube8x6_geo1.npz`` / ``tube8x6_geo3.npz``: as the element tube, with the stiffness
  and the follower pressure rebuilt on x + u by ``OptimizedSolidAssembleUpdate`` every
  step / every 3 steps (``stiffness_update_interval``), 30 steps.

Stored: assembled block-CSR K, M, C (reference layout), traction f, lumped LM,
LC, u_{-1}, the displacement history every 5 steps and the element stresses of the
final state (``OptimizedCalculateStress``, with E the per-element mean modulus).

    make -C oracle && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cvfes_b200.mesh import SolidMesh, TubeGeometry, tube_mesh  # noqa: E402
from oracle.solid_oracle import OracleSolidSolver, load_reference_module  # noqa: E402


def run(name, nc, na, S, damp, steps, nodal, seed, update_interval=0):
    rng = np.random.default_rng(seed)
    nodes, elems, inl, outl = tube_mesh(TubeGeometry(nc, na, 3.0, 0.3))
    N, E = len(nodes), len(elems)
    if nodal:
        vE = 7e6 * np.exp(0.2 * rng.standard_normal((N, S)))
        vh = 0.04 * np.exp(0.1 * rng.standard_normal((N, S)))
        mesh = SolidMesh(nodes, elems, np.concatenate([inl, outl]), S, density=1.0, v=0.49,
                         damp=damp, vE=vE, vthickness=vh)
    else:
        eE = 7e6 * np.exp(0.2 * rng.standard_normal((E, S)))
        eh = 0.04 * np.exp(0.1 * rng.standard_normal((E, S)))
        mesh = SolidMesh(nodes, elems, np.concatenate([inl, outl]), S, density=1.0, v=0.49,
                         damp=damp, elmE=eE, elmThick=eh)
    coefK, gthick = mesh.element_coefficients()
    dt = 2e-6
    pres = 1.33e5 * np.minimum(np.arange(steps) / 10.0, 1.0)
    o = OracleSolidSolver(nodes, elems, mesh.boundary, coefK, gthick, 1.0, 0.49, damp, dt,
                          backend="reference", update_interval=update_interval)
    up0 = o.up.copy()
    hist = []
    for n, p in enumerate(pres):
        o.step(p)
        if (n + 1) % 5 == 0:
            hist.append(o.u.copy())
    young = mesh.element_moduli()
    stress = o.stress(young)
    out = dict(nodes=nodes, elements=elems, boundary=mesh.boundary, coefK=coefK, gthick=gthick,
               young=young, stress=stress,
               density=1.0, v=0.49, damp=damp, dt=dt, pressures=pres, indptr=o.indptr,
               indices=o.indices, K=o.K, M=o.M, C=o.C, f=o.f, LM=o.LM, LC=o.LC, up0=up0,
               hist=np.array(hist), update_interval=update_interval)
    if nodal:
        out.update(vE=mesh.vE, vthickness=mesh.vthickness)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, {k: np.shape(v) for k, v in out.items() if np.ndim(v) > 1})


if __name__ == "__main__":
    if load_reference_module() is None:
        sys.exit("oracle/_ref is not built: make -C oracle")
    run("tube8x6_element.npz", 8, 6, 3, 100.0, 30, nodal=False, seed=1)
    run("tube6x5_nodal.npz", 6, 5, 2, 0.0, 20, nodal=True, seed=2)
    run("tube8x6_geo1.npz", 8, 6, 3, 100.0, 30, nodal=False, seed=1, update_interval=1)
    run("tube8x6_geo3.npz", 8, 6, 3, 100.0, 30, nodal=False, seed=1, update_interval=3)
