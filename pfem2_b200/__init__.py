"""B200-native PFEM2 time-step library (host side).

The compute path is libpfem2b.so (hand-written sm_100a CUDA kernels behind
the C ABI in include/pfem2.h). This package holds the Python mirror of the
reference's pfem2Solver interface (solver.py), the programmatic meshes
(meshes.py) and the workload definitions (cases.py).
"""
from . import _abi, meshes, cases  # noqa: F401

__all__ = ["_abi", "meshes", "cases"]
