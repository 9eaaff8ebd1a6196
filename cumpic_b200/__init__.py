"""cumpic_b200 — B200-native CUMC3D hot path (ideal-MHD PPM/HLL/CT/RK3 step).

The compute path is the CUDA library ``libcumc_b200.so`` behind the C-ABI in
include/cumc.h; this package holds its ctypes binding (``_native``), the
host-side mirror of the reference driver's calls (``solver.CUMC3D``), the
initial models (``problems``) and the build recipe (``build``).
"""
from . import _native, problems  # noqa: F401
from .problems import Problem  # noqa: F401


def __getattr__(name):
    if name == "CUMC3D":
        from .solver import CUMC3D
        return CUMC3D
    raise AttributeError(name)
