"""CPU-only checks: the oracle's physics invariants, the generators, and the
C-ABI library's exports and config validation (no compute on a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from cumpic_b200 import _native as N
from cumpic_b200 import problems as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle(problem):
    from _oracle import Oracle
    o = Oracle(problem, threads=4)
    o.upload()
    o.initial_update()
    return o


def test_header_symbols_exported():
    """every function declared in include/cumc.h is exported by the library."""
    src = open(os.path.join(ROOT, "include", "cumc.h")).read()
    names = set(re.findall(r"^\s*(?:int|const char\*)\s+(cumc_\w+)\s*\(", src, re.M))
    assert len(names) >= 16
    lib = N.load()
    for name in sorted(names):
        assert hasattr(lib, name), name
    assert set(N.EXPORTS) <= names


def test_config_validation_before_device():
    """cumc_init rejects bad configs with CUMC_ERR_CONFIG before touching CUDA."""
    lib = N.load()
    p = P.orszag_tang(8)
    for mutate, code in [
        (lambda c: setattr(c, "recon", 2), N.CUMC_ERR_CONFIG),
        (lambda c: setattr(c, "solver", 4), N.CUMC_ERR_CONFIG),
        (lambda c: c.boundary_flag.__setitem__(4, 3), N.CUMC_ERR_CONFIG),
        (lambda c: c.boundary_flag.__setitem__(0, 4), N.CUMC_ERR_CONFIG),
        (lambda c: setattr(c, "nx", 2), N.CUMC_ERR_CONFIG),
        (lambda c: setattr(c, "ggas", 1.0), N.CUMC_ERR_CONFIG),
    ]:
        cfg = p.config()
        mutate(cfg)
        h = ctypes.c_void_p()
        rc = lib.cumc_init(ctypes.byref(cfg), ctypes.byref(h))
        assert rc == code, (rc, lib.cumc_last_error(None))
        assert lib.cumc_last_error(None)


def test_init_without_device_fails_loudly():
    """on a machine without a CUDA device the library refuses (no CPU fallback)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    lib = N.load()
    p = P.orszag_tang(8)
    cfg = p.config()
    h = ctypes.c_void_p()
    assert lib.cumc_init(ctypes.byref(cfg), ctypes.byref(h)) == N.CUMC_ERR_CUDA


def test_generator_is_deterministic():
    a = P.uniform01(1, np.arange(10))
    b = P.uniform01(1, np.arange(10))
    assert np.array_equal(a, b) and np.all((a >= 0) & (a < 1))
    assert not np.array_equal(a, P.uniform01(2, np.arange(10)))


def test_orszag_tang_initial_divb_zero():
    o = _oracle(P.orszag_tang(16))
    assert abs(o.find_divb()) < 1e-15


@pytest.mark.parametrize("make", [lambda: P.torus(24, 16, 8), lambda: P.torus_cyl(24, 6, 20)],
                         ids=["torus_spherical", "torus_cylindrical"])
def test_torus_initial_divb_zero(make):
    """both tori's face fields are the discrete curl of A_phi with the grid's
    own face areas, so their divergence (find_divb) vanishes to round-off"""
    o = _oracle(make())
    assert abs(o.find_divb()) < 1e-15


def test_oracle_conservation_periodic():
    p = P.orszag_tang(12)
    o = _oracle(p)
    sl = (slice(3, 15),) * 3
    c0 = o.download()["cons"][sl].sum(axis=(0, 1, 2))
    o.run(10.0, 8)
    c1 = o.download()["cons"][sl].sum(axis=(0, 1, 2))
    scale = np.abs(o.download()["cons"][sl]).sum(axis=(0, 1, 2))
    # mass, momentum, energy: round-off only
    assert np.all(np.abs(c1[:5] - c0[:5]) <= 1e-12 * scale[:5]), (c1 - c0) / scale


def test_oracle_brio_wu_permutation_symmetry():
    out = []
    for ax in range(3):
        n = [4, 4, 4]
        n[ax] = 48
        o = _oracle(P.brio_wu(*n, axis=ax))
        o.run(0.1, 15)
        sl = [4, 4, 4]
        sl[2 - ax] = slice(3, 51)
        out.append(o.download()["prim"][tuple(sl) + (0,)])
    assert np.max(np.abs(out[0] - out[1])) <= 1e-14
    assert np.max(np.abs(out[0] - out[2])) <= 1e-14


def test_oracle_uniform_state():
    p = P.orszag_tang(8)
    sl = (slice(2, 11),) * 3
    p.prim[sl + (slice(0, 8),)] = [1.0, 0.1, -0.2, 0.3, 0.6, 0.2, 0.1, -0.3]
    p.eps[sl] = 0.6 / (p.ggas - 1.0)
    o = _oracle(p)
    o.run(1.0, 3)
    rho = o.download()["prim"][3:11, 3:11, 3:11, 0]
    assert np.all(rho == rho.flat[0])


def test_oracle_brio_wu_physics():
    """Brio-Wu at t=0.1: density stays within the initial range (up to small
    overshoot) and shows the compound-wave plateau near x~0.6."""
    p = P.brio_wu(128, 4, 4)
    o = _oracle(p)
    o.run(p.t_end)
    rho = o.download()["prim"][4, 4, 3:131, 0]
    assert 0.1 < rho.min() and rho.max() < 1.01
    assert abs(o.global_time - 0.1) == 0.0


def test_oracle_rejects_equatorial_x():
    from _oracle import Oracle
    p = P.orszag_tang(8)
    p.boundary_flag = (4, 1, 0, 0, 0, 0)
    with pytest.raises(ValueError):
        Oracle(p)
