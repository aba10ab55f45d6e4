"""B200-native (sm_100a) per-RK-stage explicit residual path of the FooskaGPU two-phase
finite-volume solver: mesh pre-processing, device kernels behind a C ABI, Python host API."""
from .api import Mesh, Solver, default_case  # noqa: F401

__all__ = ["Mesh", "Solver", "default_case"]
