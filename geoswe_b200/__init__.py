"""geoswe_b200 -- GeoSWE's finite-volume time step, rebuilt for NVIDIA B200 (sm_100a).

The public names follow the reference package (Mesh2D, Config, Solver2D,
CompressedSolver, RainfallForcing, StageBoundary); the compute path is libgsw.so,
hand-written CUDA kernels behind a C ABI (include/gsw.h), called through ctypes.
"""
from .config import Config, G, H_MIN
from .mesh import Mesh2D
from .forcing import RainfallForcing, StageBoundary

__all__ = ["Config", "G", "H_MIN", "Mesh2D", "RainfallForcing", "StageBoundary", "Solver2D",
           "CompressedSolver"]


def __getattr__(name):
    # the solvers import torch and load libgsw.so; keep `import geoswe_b200` light
    if name == "Solver2D":
        from .solver import Solver2D
        return Solver2D
    if name == "CompressedSolver":
        from .compressed import CompressedSolver
        return CompressedSolver
    raise AttributeError(name)
