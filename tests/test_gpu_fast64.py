"""CUMC_FP64_FAST: the FP64 path with the HLL solve's quotients formed as
products with reciprocals (not bit-compatible with the reference).

The FP64 parity bar is relative L1 <= 1e-10 per conserved variable against
the FP64 oracle at t_end, with normalised max |div B| <= 1e-12. The fast build
meets it on Orszag-Tang 64^3 to t_end = 0.5. On the Brio-Wu configuration
(512 x 4 x 4 to t_end = 0.1) the shocks amplify its last-place differences:
rho v_x, whose own L1 norm is small, ends 3.7e-10 away, so there the test
holds it to 1e-9 and the bar is not met. A torus (spherical grid, floors,
gravity) tracks the oracle over its first steps.
"""
import os

import pytest

from cumpic_b200 import _native as N
from cumpic_b200 import problems as P
from compare import rel_l1_interior

pytestmark = pytest.mark.gpu

REL_L1_TOL = 1.0e-10
DIVB_TOL = 1.0e-12


def _fast_and_oracle(prob):
    import dataclasses
    from cumpic_b200.solver import CUMC3D
    from _oracle import Oracle
    g = CUMC3D(dataclasses.replace(prob, precision=N.FP64_FAST))
    o = Oracle(prob, threads=os.cpu_count())
    for s in (g, o):
        s.upload()
        s.initial_update()
    return g, o


@pytest.mark.parametrize("make,tol", [(lambda: P.brio_wu(512, 4, 4), 1.0e-9), (lambda: P.orszag_tang(64), REL_L1_TOL)],
                         ids=["brio_wu_512", "orszag_tang_64"])
def test_fast_fp64_to_t_end(make, tol):
    prob = make()
    g, o = _fast_and_oracle(prob)
    g.run(prob.t_end)
    o.run(prob.t_end)
    assert g.global_time == pytest.approx(prob.t_end, rel=0, abs=1e-15)
    rel = rel_l1_interior(g.download(), o.download())
    assert max(rel.values()) <= tol, rel
    assert max(rel.values()) > 0.0  # a different arithmetic, not the bitwise path
    _, norm = g.find_divb()
    assert norm <= DIVB_TOL, norm


def test_fast_fp64_torus_tracks_oracle():
    g, o = _fast_and_oracle(P.torus(24, 16, 8))
    for _ in range(10):
        g.rungekutta(o.step())
    rel = rel_l1_interior(g.download(), o.download())
    assert max(rel.values()) <= 1e-12, rel


def test_fast_fp64_refuses_adjoint():
    import dataclasses
    from cumpic_b200.solver import CUMC3D
    s = CUMC3D(dataclasses.replace(P.orszag_tang(8), precision=N.FP64_FAST))
    s.upload()
    with pytest.raises(N.CumcError) as e:
        s.adjoint(1, 1)
    assert e.value.code == N.CUMC_ERR_CONFIG
