"""cvfes_b200: the ensemble membrane solid time step of CVFES, rebuilt for NVIDIA B200.

Entry points:
* :class:`cvfes_b200.solver.GPUSolidSolver` — the reference's solver-class interface;
* :class:`cvfes_b200.transient.CVFES` / ``python -m cvfes_b200 -f cfg -s nSmp`` — cfg-driven runs;
* :mod:`cvfes_b200._lib` — ctypes binding of the C ABI in ``include/cvfes_b200.h``.
"""
__version__ = "0.1.0"
