"""Parity of the FP64 CUDA path with the FP64 oracle at the configured sizes.

The small cases of test_gpu_parity.py pin every code path; these runs pin the
configurations the throughput and the accuracy figures are quoted on:

* Orszag-Tang 256^3 (the throughput configuration), 3 main-loop steps, bit for
  bit (dt included).
* Orszag-Tang 64^3 run to its t_end = 0.5 (about 160 steps), the FP64 bar:
  relative L1 <= 1e-10 per conserved variable at t_end and normalised
  max |div B| <= 1e-12; the run is also bit for bit.
* The spherical torus at its configured grid, 192 x 128 x 64 (log-spaced r,
  floors, point-mass gravity, ghost clamps, 8x geometric source), 100 steps
  bit for bit.

The oracle runs on all host threads; each case takes well under a minute of
oracle time on a 16-core host.
"""
import os

import numpy as np
import pytest

from cumpic_b200 import problems as P
from compare import diffs, rel_l1_interior

pytestmark = pytest.mark.gpu

REL_L1_TOL = 1.0e-10  # FP64 parity bar per conserved variable at t_end
DIVB_TOL = 1.0e-12    # normalised max |div B| held by CT


def _pair(problem):
    from cumpic_b200.solver import CUMC3D
    from _oracle import Oracle
    g = CUMC3D(problem)
    o = Oracle(problem, threads=os.cpu_count())
    for s in (g, o):
        s.upload()
        s.initial_update()
    return g, o


def _steps_bitwise(g, o, nsteps):
    for n in range(nsteps):
        dg, do = g.finddt(), o.finddt()
        assert dg == do, (n, dg, do)
        g.rungekutta(dg)
        o.rungekutta(do)


def _assert_bitwise(g, o, what):
    a = g.download()
    b = o.download()
    d = diffs(a, b)
    bad = {k: v for k, v in d.items() if v != 0.0}
    assert not bad, f"{what}: {bad}"
    return a, b


def test_orszag_tang_256_three_steps_bitwise():
    p = P.orszag_tang(256)
    g, o = _pair(p)
    _steps_bitwise(g, o, 3)
    _assert_bitwise(g, o, "Orszag-Tang 256^3 after 3 steps")
    g.close()
    o.close()


def test_orszag_tang_64_to_t_end():
    p = P.orszag_tang(64)
    g, o = _pair(p)
    ng = g.run(p.t_end)
    no = o.run(p.t_end)
    assert ng == no and ng > 100
    assert g.global_time == o.global_time == p.t_end
    a, b = _assert_bitwise(g, o, "Orszag-Tang 64^3 at t_end")
    rel = rel_l1_interior(a, b)
    assert max(rel.values()) <= REL_L1_TOL, rel
    _, norm = g.find_divb()
    assert norm <= DIVB_TOL, norm
    assert np.all(np.isfinite(a["cons"]))


def test_torus_configured_grid_100_steps():
    p = P.torus()
    assert (p.nx, p.ny, p.nz) == (192, 128, 64)
    g, o = _pair(p)
    _steps_bitwise(g, o, 100)
    _assert_bitwise(g, o, "torus 192x128x64 after 100 steps")
