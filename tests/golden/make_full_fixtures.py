"""Full-run-length fixtures of the three large workloads, from the reference's own kernels.

For each workload a seeded chunk of its sample ensemble is advanced over the
workload's whole run by the reference's CPU solid path in linear-template mode: its
compiled ``OptimizedSolidAssembleWithDamping`` and ``MultiplyByVector``
(``optimizedSolidAssemble.pyx:457-599, 1250-1274``, built from the reference sources
by ``oracle/Makefile``) driven by the update of ``physicsSolver.py:263-292``
(``oracle.solid_oracle.OracleSolidSolver(backend="reference")``).  Samples never
interact, so a chunk of the ensemble advanced alone is exactly those samples of the
whole ensemble.

* ``full_tube256x1024.npz``: the 256 x 1024 tube, 2 of its 512 samples, dt 5e-7,
  2000 steps, row-sum lumped mass (the reference's assembly run with 3 rho);
* ``full_stenosed512x2048.npz``: the stenosed 512 x 2048 tube, 2 of its 128 samples,
  the CFL time step of the whole ensemble, 1000 steps;
* ``full_batchNN.npz``: tubes of the uneven 64-tube ensemble (the largest mesh, the
  most node-samples, the largest FP32 error of each state form and a 16-sample tube),
  2 samples each, their own CFL time steps, 1000 steps.

Stored (small): the chunk's sample indices, dt, the final displacement at a seeded
subset of 2048 nodes (global numbering), the per-sample sums over ALL nodes of u^2 and
of (u_n - u_{n-1})^2 at the final step, and checksums of the material columns so a
test can confirm it regenerated the same inputs.  The material is the workload's own
GMRF ensemble (``cvfes_b200.cases``), generated identically wherever the tests run.

Beside the reference's FP64 result each fixture holds the same run in long double
(80-bit, 64-bit mantissa): the reference's update of ``physicsSolver.py:272-285`` and
block SpMV from the same assembled FP64 matrices and start-up state, evaluated in
``numpy.longdouble``.  Over 1000-2000 steps the reference's own FP64 rounding reaches
several 1e-12 on some tubes (its update forms 2 m u - m u_prev, so every step's rounding
of u enters the velocity), so a 1e-12 gate is checked against this truth.

    make -C oracle && python tests/golden/make_full_fixtures.py [names...]
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cvfes_b200.cases import CASES, batched_cases, build_mesh, case_dt  # noqa: E402
from oracle.solid_oracle import OracleSolidSolver, load_reference_module  # noqa: E402

N_SUBSET = 2048
CHUNK = 2
# tubes of the 64-tube ensemble (seed 7): 47 the largest mesh (256 x 937), 34 the most
# node-samples (256 x 847, 256 samples), 32 the largest FP32 error of the velocity-state
# form (7.4e-6), 58 the largest of the previous-displacement form (6.2e-5), 2 a
# 16-sample tube
BATCH_TUBES = (47, 34, 32, 58, 2)


def material_checksum(coefK, gthick):
    """Sum, sum of squares and three entries of each material column (E*h, h)."""
    E = coefK.shape[0]
    picks = [0, E // 2, E - 1]
    out = []
    for a in (coefK, gthick):
        a = np.asarray(a, dtype=np.float64).reshape(E, a.shape[1], -1)[:, :, 0]
        out.append(np.stack([a.sum(axis=0), (a * a).sum(axis=0), *[a[i] for i in picks]]))
    return np.concatenate(out)  # (10, chunk)


def _ld_spmv(K, indptr, indices, v):
    """``K v`` of the block-CSR matrix in the arithmetic of K's dtype."""
    N, S = len(indptr) - 1, K.shape[1]
    prod = np.einsum("nsij,njs->nis", K, v.reshape(N, 3, S)[indices])
    rows = np.zeros((N, 3, S), dtype=K.dtype)
    nz = np.diff(indptr) > 0
    rows[nz] = np.add.reduceat(prod, indptr[:-1][nz], axis=0)
    return rows.reshape(3 * N, S)


def run_case(name, case, mesh, dt, n_steps, seed):
    S = mesh.nSmp
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(S, size=min(CHUNK, S), replace=False))
    coefK, gthick = mesh.element_coefficients()
    coefK, gthick = np.ascontiguousarray(coefK[:, idx]), np.ascontiguousarray(gthick[:, idx])
    # row-sum lumping is the reference's lumping with 3 rho (the quadrature weight 1/3
    # applied once instead of twice)
    rho = mesh.density * (3.0 if getattr(mesh, "mass_lumping", "reference") == "rowsum" else 1.0)
    t0 = time.time()
    o = OracleSolidSolver(mesh.nodes, mesh.elementNodeIds, mesh.boundary, coefK, gthick, rho,
                          mesh.v, mesh.damp, dt, backend="reference")
    t1 = time.time()
    LD = np.longdouble
    K, LM, LC = o.K.astype(LD), o.LM.astype(LD), o.LC.astype(LD)
    f, dtl = o.f.astype(LD), LD(dt)
    LHS = LM + LD(0.5) * dtl * LC
    u, up = o.u.astype(LD), o.up.astype(LD)
    pres = case.pressures(n_steps)
    for n in range(n_steps):
        o.step(float(pres[n]))
        rhs = (dtl * dtl * LD(pres[n]) * f[:, None] + 2 * LM * u
               - dtl * dtl * _ld_spmv(K, o.indptr, o.indices, u) + (LD(0.5) * dtl * LC - LM) * up)
        un = np.where(LHS != 0, rhs / np.where(LHS != 0, LHS, 1), 0)
        un[o.bdyDofs, :] = o.bdyU
        up, u = u, un
    t2 = time.time()
    N = mesh.nNodes
    nodes = np.sort(np.random.default_rng(seed + 1).choice(N, size=min(N_SUBSET, N),
                                                           replace=False))
    dofs = (3 * nodes[:, None] + np.arange(3)[None, :]).ravel()
    out = dict(workload=name, samples=idx, n_samples=S, dt=dt, n_steps=n_steps,
               density=rho, nodes=nodes, u_subset=o.u[dofs], sum_u2=np.sum(o.u ** 2, axis=0),
               sum_du2=np.sum((o.u - o.up) ** 2, axis=0),
               material=material_checksum(coefK, gthick), finite=np.isfinite(o.u).all(),
               u_subset_truth=u[dofs].astype(np.float64),
               sum_u2_truth=np.sum(u.astype(np.float64) ** 2, axis=0))
    path = os.path.join(HERE, f"full_{name}.npz")
    np.savez_compressed(path, **out)
    err = np.linalg.norm(out["u_subset"] - out["u_subset_truth"]) / np.linalg.norm(
        out["u_subset_truth"])
    print(f"{name}: samples {idx.tolist()} dt {dt:.4e} steps {n_steps}: assembly {t1 - t0:.0f} s, "
          f"steps {t2 - t1:.0f} s, |u| max {np.abs(o.u).max():.3e}, reference FP64 vs long "
          f"double {err:.3e} -> {path}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="*")
    a = ap.parse_args()
    if load_reference_module() is None:
        sys.exit("oracle/_ref is not built: make -C oracle")
    todo = a.names or ["tube256x1024", "stenosed512x2048"] + [f"batch{i:02d}" for i in BATCH_TUBES]
    cases = batched_cases(64, seed=7)
    for name in todo:
        if name.startswith("batch"):
            case = cases[int(name[5:])]
            n_steps = 1000
        else:
            case = CASES[name]
            n_steps = case.n_steps
        mesh = build_mesh(case)
        dt = case_dt(case, mesh)
        run_case(name, case, mesh, dt, n_steps, seed=2024)


if __name__ == "__main__":
    main()
