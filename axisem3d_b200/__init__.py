"""axisem3d_b200 -- B200-native (sm_100a) engine for AxiSEM3D's per-time-step loop.

The product is the C-ABI library ``libaxg.so`` (include/axg.h): fused CUDA
kernels for solid/fluid element stiffness, point assembly, boundary
conditions, mass inversion, the Newmark update, sources and stations, driven
by a C++ host engine. This package holds its sources (``csrc/``), the in-tree
build, and a thin Python mirror of the ABI (``Solver``) with the seeded model
generators used by the tests and the benchmark.
"""
from .model import Model, STF  # noqa: F401

__all__ = ["Model", "STF", "Solver", "build"]


def build(force=False):
    from .build import build as _b
    return _b(force=force)


def __getattr__(name):
    if name == "Solver":
        from .solver import Solver
        return Solver
    raise AttributeError(name)
