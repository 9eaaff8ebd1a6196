"""ctypes binding of the CUMC3D C-ABI (include/cumc.h).

The shared library ``libcumc_b200.so`` is built in-tree by
``cumpic_b200.build.build_library``. There is no fallback: if the library is
missing or cannot load, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_longlong, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcumc_b200.so")

# status codes (include/cumc.h)
CUMC_OK = 0
CUMC_ERR_ARG = 1
CUMC_ERR_CONFIG = 2
CUMC_ERR_CUDA = 3
CUMC_ERR_NONFINITE = 4
CUMC_ERR_STATE = 5
CUMC_ERR_NOMEM = 6
CUMC_ERR_LIMIT = 7

CARTESIAN, CYLINDRICAL, SPHERICAL = 1, 2, 3
TVDMM, PPMC = 1, 4
HLL = 2
FP64, MIXED, FP64_FAST = 0, 1, 2
MODEL_NONE, MODEL_RIEMANN, MODEL_TORUS_SPH, MODEL_TORUS_CYN = 0, 1, 2, 3

OBJ_MAGNETIC, OBJ_KINETIC, OBJ_LINEAR = 1, 2, 3

K_SWEEP_X, K_SWEEP_Y, K_SWEEP_Z, K_EMF, K_COMBINE, K_UTOP, K_BOUNDARY, K_FINDDT = range(8)
K_NAMES = ["sweep_x", "sweep_y", "sweep_z", "emf", "combine", "utop", "boundary", "finddt", "ct"]


class CumcConfig(ctypes.Structure):
    """Mirror of ``cumc_config`` (include/cumc.h)."""

    _fields_ = [
        ("nx", c_int),
        ("ny", c_int),
        ("nz", c_int),
        ("xf", POINTER(c_double)),
        ("yf", POINTER(c_double)),
        ("zf", POINTER(c_double)),
        ("coordinate", c_int),
        ("boundary_flag", c_int * 6),
        ("ggas", c_double),
        ("cfl", c_double),
        ("recon", c_int),
        ("solver", c_int),
        ("precision", c_int),
        ("model", c_int),
        ("rho_floor", c_double),
        ("eps_floor", c_double),
        ("r_sh", c_double),
        ("geom_source_repeat", c_int),
        ("reserved", c_int * 7),
    ]


class CumcError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[cumc status {code}] {message}")
        self.code = code


EXPORTS = [
    "cumc_init", "cumc_free", "cumc_last_error", "cumc_upload_state", "cumc_download_state",
    "cumc_initial_update", "cumc_finddt", "cumc_rungekutta", "cumc_spatial", "cumc_download_lrk",
    "cumc_divb", "cumc_advance", "cumc_get_stream", "cumc_profile", "cumc_profile_read",
    "cumc_launch_count", "cumc_query", "cumc_cfl_dt_static", "cumc_cfl_dt_static_error", "cumc_adjoint_run",
    "cumc_snapshot_async", "cumc_snapshot_wait", "cumc_restore_state",
    "cumc_rk_stage", "cumc_rk_stage_part", "cumc_halo_doubles", "cumc_halo_pack", "cumc_halo_unpack", "cumc_model_torus",
]
BC_EXCHANGE = -1
Q_X_STAGING = 1
Q_FUSED = 2
STATE_ARRAYS = 17


class CumcTorusModel(ctypes.Structure):
    _fields_ = [(n, c_double) for n in ("r_sh", "s_in", "s_max", "q_grad", "rho_max", "rho_fac", "rho_cut", "beta",
                                        "noise")] + [("seed", ctypes.c_ulonglong)]


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    dp = POINTER(c_double)
    sig = {
        "cumc_init": (c_int, [POINTER(CumcConfig), POINTER(c_void_p)]),
        "cumc_free": (c_int, [c_void_p]),
        "cumc_last_error": (c_char_p, [c_void_p]),
        "cumc_upload_state": (c_int, [c_void_p, dp, dp]),
        "cumc_download_state": (c_int, [c_void_p, dp, dp, dp, dp]),
        "cumc_initial_update": (c_int, [c_void_p]),
        "cumc_finddt": (c_int, [c_void_p, dp]),
        "cumc_rungekutta": (c_int, [c_void_p, c_double]),
        "cumc_spatial": (c_int, [c_void_p]),
        "cumc_download_lrk": (c_int, [c_void_p, dp]),
        "cumc_divb": (c_int, [c_void_p, dp, dp]),
        "cumc_advance": (c_int, [c_void_p, c_int, c_double, dp, POINTER(c_int)]),
        "cumc_get_stream": (c_int, [c_void_p, POINTER(c_void_p)]),
        "cumc_profile": (c_int, [c_void_p, c_int]),
        "cumc_profile_read": (c_int, [c_void_p, c_int, POINTER(c_int), dp]),
        "cumc_launch_count": (c_int, [c_void_p, POINTER(c_longlong)]),
        "cumc_query": (c_int, [c_void_p, c_int, POINTER(c_longlong)]),
        "cumc_cfl_dt_static": (c_int, [c_int, c_int, c_int] + [c_void_p] * 11 + [c_int, c_void_p, c_void_p,
                                                                                   c_double, c_double, c_void_p,
                                                                                   c_void_p]),
        "cumc_cfl_dt_static_error": (c_char_p, []),
        "cumc_adjoint_run": (c_int, [c_void_p, c_int, c_int, c_int, dp, dp, dp, dp, dp, dp]),
        "cumc_rk_stage": (c_int, [c_void_p, c_int, c_double]),
        "cumc_rk_stage_part": (c_int, [c_void_p, c_int, c_double, c_int]),
        "cumc_halo_doubles": (c_int, [c_void_p, POINTER(c_longlong)]),
        "cumc_halo_pack": (c_int, [c_void_p, c_int, c_void_p]),
        "cumc_halo_unpack": (c_int, [c_void_p, c_int, c_void_p]),
        "cumc_model_torus": (c_int, [c_void_p, POINTER(CumcTorusModel)]),
        "cumc_snapshot_async": (c_int, [c_void_p, dp]),
        "cumc_snapshot_wait": (c_int, [c_void_p]),
        "cumc_restore_state": (c_int, [c_void_p, dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB
