"""cumc_cfl_dt_static: the CFL time step for callers that cannot allocate.

Codes that capture their time loop into a CUDA graph cannot call cudaMalloc
during the capture, and host programs whose device memory is owned by another
runtime (an OpenACC data region, a framework allocator, a fixed pool) must not
allocate behind its back. cumc_cfl_dt_static serves them: it reads device
arrays the caller already owns and keeps its reduction scratch in a fixed
array inside the library. This test hands it the same state the library's own
cumc_finddt sees, as device arrays allocated here by the test, and checks that
both give the same time step, on two calls in a row (the second after one
RK3 step, so the shared scratch is reused with new contents), on a
Cartesian, a cylindrical and a spherical grid.
"""
import ctypes
import math

import numpy as np
import pytest

from cumpic_b200 import _native as N
from cumpic_b200 import problems as P

pytestmark = pytest.mark.gpu


def _widths(f: np.ndarray) -> np.ndarray:
    """cell widths f(i) - f(i-1) for i = -3..n+3 (index i+3; entry 0 unused)"""
    d = np.zeros_like(f)
    d[1:] = f[1:] - f[:-1]
    return d


def _centres_and_sines(problem):
    """cell-centre radius 0.5 (xF(i) + xF(i-1)) and the sine of the polar cell
    centre, for i = -3..n+3 (index i+3; entry 0 unused), computed with the
    same double operations and the C library's sin, as the library's own
    tables are"""
    xc = np.zeros_like(problem.xf)
    xc[1:] = 0.5 * (problem.xf[1:] + problem.xf[:-1])
    sin_yc = np.zeros_like(problem.yf)
    for i in range(1, len(problem.yf)):
        sin_yc[i] = math.sin(0.5 * (problem.yf[i] + problem.yf[i - 1]))
    return xc, sin_yc


def _static_dt(sim, problem, torch):
    st = sim.download()
    prim, bcell = st["prim"], st["bcell"]
    dev = torch.device("cuda", 0)
    fields = [prim[..., q] for q in range(5)] + [bcell[..., q] for q in range(3)]
    arrays = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in fields]
    widths = [torch.from_numpy(_widths(f)).to(dev) for f in (problem.xf, problem.yf, problem.zf)]
    xc, sin_yc = (torch.from_numpy(a).to(dev) for a in _centres_and_sines(problem))
    curvilinear = problem.coordinate != N.CARTESIAN
    dt_out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    lib = N.lib()
    stream = torch.cuda.current_stream(dev)
    rc = lib.cumc_cfl_dt_static(problem.nx, problem.ny, problem.nz,
                                *[a.data_ptr() for a in arrays], *[w.data_ptr() for w in widths],
                                problem.coordinate, xc.data_ptr() if curvilinear else None,
                                sin_yc.data_ptr() if problem.coordinate == N.SPHERICAL else None,
                                problem.ggas, problem.cfl, dt_out.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
    assert rc == N.CUMC_OK, lib.cumc_cfl_dt_static_error()
    stream.synchronize()
    return float(dt_out.item())


GRIDS = [
    ("cartesian", lambda: P.orszag_tang(24, ny=20, nz=16)),
    ("cylindrical", lambda: P.shell(N.CYLINDRICAL, 16, 12, 10)),
    ("spherical", lambda: P.torus(24, 16, 8)),
]


@pytest.mark.parametrize("name,make", GRIDS, ids=[g[0] for g in GRIDS])
def test_static_cfl_dt_matches_finddt(name, make):
    torch = pytest.importorskip("torch")
    from cumpic_b200.solver import CUMC3D
    problem = make()
    sim = CUMC3D(problem)
    sim.upload()
    sim.initial_update()
    for _ in range(2):  # two calls in a row, the second on an advanced state
        dt_lib = sim.finddt()
        dt_static = _static_dt(sim, problem, torch)
        assert dt_static == dt_lib, (dt_static, dt_lib)  # same arithmetic: bit for bit
        sim.rungekutta(dt_lib)


def test_static_cfl_dt_rejects_oversize_grid():
    lib = N.lib()
    big = 257  # 257^3 > CUMC_STATIC_MAX_CELLS
    rc = lib.cumc_cfl_dt_static(big, big, big, *([ctypes.c_void_p(1)] * 11), N.CARTESIAN, None, None,
                                5.0 / 3.0, 0.4, ctypes.c_void_p(1), None)
    assert rc == N.CUMC_ERR_LIMIT
    assert b"256^3" in lib.cumc_cfl_dt_static_error()
