"""Displacement output without VTK.

The reference writes one VTP per save with a ``displacement_%03d`` point array
per sample (``mesh.py:709-726``).  Here a save is an ``.npz`` (``u`` as
(S, N, 3), nodes and elements) and, when the file name ends in ``.vtk``, a
legacy-VTK ASCII polydata file with the same per-sample point arrays, which
ParaView reads.
"""
from __future__ import annotations

import os

import numpy as np


def _numbered(filename: str, counter: int) -> str:
    base, ext = os.path.splitext(filename)
    return "{}{}{}".format(base, counter, ext or ".npz")


def save_displacement(filename: str, counter: int, mesh, u: np.ndarray, uname: str = "u",
                      stress: np.ndarray = None) -> str:
    """Write displacement ``u`` (S, N, 3) of step ``counter`` and, when given, the element
    stresses (E, S, 5: xx, yy, xy, xz, yz, as ``mesh.py:709-726`` names them); returns the
    path written."""
    path = _numbered(filename, counter)
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    if path.endswith(".vtk"):
        write_legacy_vtk(path, mesh.nodes, mesh.elementNodeIds, u, uname, stress)
    else:
        if not path.endswith(".npz"):
            path = os.path.splitext(path)[0] + ".npz"
        extra = {} if stress is None else {"stress": stress}
        np.savez(path, u=u, nodes=mesh.nodes, elements=mesh.elementNodeIds, **extra)
    return path


STRESS_NAMES = ("xx", "yy", "xy", "xz", "yz")


def write_legacy_vtk(path, nodes, elements, u, uname="u", stress=None):
    """Legacy ASCII VTK polydata: triangles, one vector array per sample and, when given,
    one cell scalar per stress component and sample (``<comp>_<sample>``)."""
    S = u.shape[0]
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.0\ncvfes_b200 displacement\nASCII\nDATASET POLYDATA\n")
        f.write("POINTS {} double\n".format(len(nodes)))
        np.savetxt(f, nodes, fmt="%.17g")
        f.write("POLYGONS {} {}\n".format(len(elements), 4 * len(elements)))
        np.savetxt(f, np.hstack([np.full((len(elements), 1), 3), elements]), fmt="%d")
        f.write("POINT_DATA {}\n".format(len(nodes)))
        for s in range(S):
            f.write("VECTORS {}_{:03d} double\n".format(uname, s))
            np.savetxt(f, u[s], fmt="%.17g")
        if stress is not None:
            f.write("CELL_DATA {}\n".format(len(elements)))
            for s in range(stress.shape[1]):
                for c, name in enumerate(STRESS_NAMES):
                    f.write("SCALARS {}_{:03d} double 1\nLOOKUP_TABLE default\n".format(name, s))
                    np.savetxt(f, stress[:, s, c], fmt="%.17g")


def read_legacy_vtk_vectors(path):
    """Read back the per-sample vector arrays written by :func:`write_legacy_vtk`."""
    out, cur, n = {}, None, None
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("POINT_DATA"):
            n = int(ln.split()[1])
        elif ln.startswith("VECTORS"):
            name = ln.split()[1]
            out[name] = np.loadtxt(lines[i + 1:i + 1 + n]).reshape(n, 3)
            i += n
        i += 1
    return out


def read_legacy_vtk_cell_scalars(path):
    """Read back the per-sample cell scalars (stress components) of :func:`write_legacy_vtk`."""
    out, n = {}, None
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("CELL_DATA"):
            n = int(ln.split()[1])
        elif ln.startswith("SCALARS") and n is not None:
            name = ln.split()[1]
            out[name] = np.loadtxt(lines[i + 2:i + 2 + n]).reshape(n)
            i += n + 1
        i += 1
    return out
