"""ctypes binding of the FP64 CPU oracle (oracle/cumc_oracle.cpp).

Test infrastructure: the oracle is the checker the CUDA path is compared
against; it is never part of the product path. The method names mirror
cumpic_b200.solver.CUMC3D so a test can drive both with the same calls.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_void_p

import numpy as np

from cumpic_b200 import _native as N
from cumpic_b200.problems import Problem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "build", "libcumc_oracle.so")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
_LIBS: dict = {}


def ref_lib_path(model: str) -> str:
    """mechanical translation of the reference for a model (oracle/f2c_ref.py)"""
    return os.path.join(REF_DIR, f"libcumc_ref_{model}.so")


def lib(path: str = ORACLE_LIB):
    if path not in _LIBS:
        if path == ORACLE_LIB and not os.path.exists(ORACLE_LIB):
            from cumpic_b200.build import build_oracle
            build_oracle()
        L = ctypes.CDLL(path)
        dp = POINTER(c_double)
        L.orc_create.restype = c_void_p
        L.orc_create.argtypes = [POINTER(N.CumcConfig), c_char_p, c_int]
        L.orc_free.argtypes = [c_void_p]
        L.orc_set_threads.argtypes = [c_int]
        L.orc_get_threads.restype = c_int
        for name in ("orc_upload",):
            getattr(L, name).argtypes = [c_void_p, dp, dp]
        for name in ("orc_initial_update", "orc_spatial"):
            getattr(L, name).argtypes = [c_void_p]
        L.orc_finddt.argtypes = [c_void_p, dp]
        L.orc_rungekutta.argtypes = [c_void_p, c_double]
        L.orc_divb.argtypes = [c_void_p, dp]
        L.orc_download.argtypes = [c_void_p, dp, dp, dp, dp, dp]
        _LIBS[path] = L
    return _LIBS[path]


def _dp(a):
    return a.ctypes.data_as(POINTER(c_double))


class Oracle:
    def __init__(self, problem: Problem, threads: int | None = None, lib_path: str = ORACLE_LIB):
        self.problem = problem
        L = self._L = lib(lib_path)
        if threads:
            L.orc_set_threads(int(threads))
        self._cfg = problem.config()
        err = ctypes.create_string_buffer(512)
        h = L.orc_create(ctypes.byref(self._cfg), err, 512)
        if not h:
            raise ValueError(err.value.decode())
        self._h = h
        self.global_time = 0.0
        self.n_step = 0

    def close(self):
        if self._h:
            self._L.orc_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        p = self.problem
        return (p.nz + 6, p.ny + 6, p.nx + 6)

    def upload(self, prim=None, eps=None):
        prim = np.ascontiguousarray(self.problem.prim if prim is None else prim, dtype=np.float64)
        eps = np.ascontiguousarray(self.problem.eps if eps is None else eps, dtype=np.float64)
        self._L.orc_upload(self._h, _dp(prim), _dp(eps))

    def initial_update(self):
        self._L.orc_initial_update(self._h)

    def finddt(self) -> float:
        dt = c_double()
        self._L.orc_finddt(self._h, ctypes.byref(dt))
        return dt.value

    def rungekutta(self, dt: float):
        self._L.orc_rungekutta(self._h, float(dt))

    def spatial(self) -> np.ndarray:
        self._L.orc_spatial(self._h)
        out = np.zeros(self.shape + (8,))
        self._L.orc_download(self._h, None, None, None, None, _dp(out))
        return out

    def find_divb(self) -> float:
        v = c_double()
        self._L.orc_divb(self._h, ctypes.byref(v))
        return v.value

    def download(self) -> dict:
        prim = np.zeros(self.shape + (8,))
        cons = np.zeros(self.shape + (8,))
        eps = np.zeros(self.shape)
        bcell = np.zeros(self.shape + (3,))
        self._L.orc_download(self._h, _dp(prim), _dp(cons), _dp(eps), _dp(bcell), None)
        return {"prim": prim, "cons": cons, "eps": eps, "bcell": bcell}

    def step(self, total_time: float | None = None) -> float:
        dt = self.finddt()
        if total_time is not None and self.global_time + dt > total_time:
            dt = total_time - self.global_time
        self.rungekutta(dt)
        self.n_step += 1
        self.global_time += dt
        return dt

    def run(self, total_time: float, max_steps: int = 10 ** 9) -> int:
        n = 0
        while self.global_time < total_time and n < max_steps:
            self.step(total_time)
            n += 1
        return n


class TangentOracle:
    """Tangent-linear run of the oracle: the same discrete map on
    (value, direction) pairs with every branch frozen at the base point, so
    the derivative parts are the exact directional derivative of the map
    upload -> initial_update -> RK3 steps (the FP64 reference gradient the
    adjoint is checked against)."""

    def __init__(self, problem: Problem, threads: int | None = None):
        self.problem = problem
        L = self._L = lib(ORACLE_LIB)
        if not hasattr(L.orc_tl_create, "_typed"):
            dp = POINTER(c_double)
            L.orc_tl_create.restype = c_void_p
            L.orc_tl_create.argtypes = [POINTER(N.CumcConfig), c_char_p, c_int]
            L.orc_tl_free.argtypes = [c_void_p]
            L.orc_tl_upload.argtypes = [c_void_p, dp, dp, dp, dp]
            L.orc_tl_initial_update.argtypes = [c_void_p]
            L.orc_tl_rungekutta.argtypes = [c_void_p, c_double]
            L.orc_tl_download.argtypes = [c_void_p] + [dp] * 8
            L.orc_tl_create._typed = True
        if threads:
            L.orc_set_threads(int(threads))
        self._cfg = problem.config()
        err = ctypes.create_string_buffer(512)
        h = L.orc_tl_create(ctypes.byref(self._cfg), err, 512)
        if not h:
            raise ValueError(err.value.decode())
        self._h = h

    def close(self):
        if self._h:
            self._L.orc_tl_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        p = self.problem
        return (p.nz + 6, p.ny + 6, p.nx + 6)

    def run(self, dprim: np.ndarray, deps: np.ndarray, dts) -> tuple[dict, dict]:
        """initial_update and one rungekutta per dt from the problem's state
        perturbed along (dprim, deps); returns (values, derivatives)."""
        p = self.problem
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (p.prim, p.eps, dprim, deps)]
        self._L.orc_tl_upload(self._h, *[_dp(a) for a in arrs])
        self._L.orc_tl_initial_update(self._h)
        for dt in dts:
            self._L.orc_tl_rungekutta(self._h, float(dt))
        v = {"prim": np.zeros(self.shape + (8,)), "cons": np.zeros(self.shape + (8,)), "eps": np.zeros(self.shape),
             "bcell": np.zeros(self.shape + (3,))}
        d = {k: np.zeros_like(a) for k, a in v.items()}
        self._L.orc_tl_download(self._h, _dp(v["prim"]), _dp(v["cons"]), _dp(v["eps"]), _dp(v["bcell"]),
                                _dp(d["prim"]), _dp(d["cons"]), _dp(d["eps"]), _dp(d["bcell"]))
        return v, d
