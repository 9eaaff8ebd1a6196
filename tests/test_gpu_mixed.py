"""Mixed-precision path (CUMC_MIXED) against the FP64 path.

Bars: relative L1 of the density against the FP64 run <= 1e-5 (the accuracy
bar of the mixed form) and the normalised max |div B| of the compensated face
fields at round-off.
"""
import numpy as np
import pytest

from cumpic_b200 import _native as N
from cumpic_b200 import problems as P
from compare import rel_l1_interior

pytestmark = pytest.mark.gpu

RHO_L1_TOL = 1.0e-5
DIVB_TOL = 1.0e-12


def _run(problem, precision, steps=None, t_end=None):
    from cumpic_b200.solver import CUMC3D
    problem.precision = precision
    s = CUMC3D(problem)
    s.upload()
    s.initial_update()
    if t_end is not None:
        s.run(t_end)
    else:
        for _ in range(steps):
            s.step()
    return s


@pytest.mark.parametrize("bscale", [1.0, 10.0])
def test_orszag_tang_mixed_vs_fp64(bscale):
    a = _run(P.orszag_tang(32, bscale=bscale), N.FP64, t_end=0.05)
    b = _run(P.orszag_tang(32, bscale=bscale), N.MIXED, t_end=0.05)
    rel = rel_l1_interior(b.download(), a.download())
    assert rel[0] <= RHO_L1_TOL, rel
    assert max(rel.values()) <= 1e-3, rel
    _, norm = b.find_divb()
    assert norm <= DIVB_TOL, norm


def test_brio_wu_mixed_vs_fp64():
    p = P.brio_wu(512, 4, 4)
    a = _run(P.brio_wu(512, 4, 4), N.FP64, t_end=p.t_end)
    b = _run(P.brio_wu(512, 4, 4), N.MIXED, t_end=p.t_end)
    assert b.global_time == pytest.approx(p.t_end)
    rel = rel_l1_interior(b.download(), a.download())
    assert rel[0] <= 1e-4, rel  # shocks: FP32 fluxes move discontinuities by round-off


def test_torus_mixed_runs_and_tracks_fp64():
    a = _run(P.torus(48, 32, 16), N.FP64, steps=20)
    b = _run(P.torus(48, 32, 16), N.MIXED, steps=20)
    da, db = a.download(), b.download()
    assert np.all(np.isfinite(db["cons"]))
    rel = rel_l1_interior(db, da)
    assert rel[0] <= 1e-4, rel


def test_mixed_advance_equals_host_loop():
    from cumpic_b200.solver import CUMC3D
    p = P.orszag_tang(16, precision=N.MIXED)
    x, y = CUMC3D(p), CUMC3D(p)
    for s in (x, y):
        s.upload()
        s.initial_update()
    for _ in range(5):
        x.step()
    y.advance(5)
    assert x.global_time == y.global_time
    assert np.array_equal(x.download()["cons"], y.download()["cons"])


@pytest.mark.parametrize("make", [lambda: P.shell(N.CYLINDRICAL, 24, 20, 16), lambda: P.shell(N.SPHERICAL, 24, 20, 16),
                                  lambda: P.torus_cyl(40, 8, 40)], ids=["cyl_shell", "sph_shell", "torus_cyl"])
def test_curvilinear_mixed_vs_fp64(make):
    """geometric flux, CT and source terms (and the cylindrical torus's
    gravity, floors and ghost clamps) of the mixed path, with the FP64 run's
    dt sequence replayed"""
    a = _run(make(), N.FP64, steps=0)
    dts = [a.step() for _ in range(10)]
    b = _run(make(), N.MIXED, steps=0)
    for dt in dts:
        b.rungekutta(dt)
    db = b.download()
    assert np.all(np.isfinite(db["cons"][3:-3, 3:-3, 3:-3]))
    rel = rel_l1_interior(db, a.download())
    assert rel[0] <= RHO_L1_TOL, rel


def test_fused_stage_equals_split(monkeypatch):
    """the default mixed stage (tiled EMF + CT, combine fused with the
    conversions) agrees with the split one (k_emf, k_combine_mx, k_utop_mx)
    on a Cartesian box and on a torus with floors. Both evaluate the same
    expressions, but the mixed unit contracts to FMA and may pair a product
    with a different sum in the two forms, so they agree to FP32 round-off
    rather than bit for bit."""
    from cumpic_b200.solver import CUMC3D
    out = {}
    for mode in (None, "split"):
        if mode:
            monkeypatch.setenv("CUMC_MX_STAGE", mode)
        else:
            monkeypatch.delenv("CUMC_MX_STAGE", raising=False)
        for name, prob in (("ot", P.orszag_tang(37, ny=29, nz=40)), ("torus", P.torus(24, 16, 40))):
            prob.precision = N.MIXED
            s = CUMC3D(prob)
            s.upload()
            s.initial_update()
            s.advance(4)
            out[(mode, name)] = s.download()
            s.close()
    for name in ("ot", "torus"):
        a, b = out[(None, name)], out[("split", name)]
        rel = rel_l1_interior(a, b)
        assert max(rel.values()) <= 1.0e-6, (name, rel)
        x, y = a["cons"][3:-3, 3:-3, 3:-3], b["cons"][3:-3, 3:-3, 3:-3]
        for q in range(8):
            scale = np.max(np.abs(y[..., q])) or 1.0
            assert np.max(np.abs(x[..., q] - y[..., q])) <= 1.0e-5 * scale, (name, q)


def test_fp32_hll_form(monkeypatch):
    """CUMC_MX_HLL=fp32 (the HLL solve all in FP32) runs the same problem
    within the bar, and is a different arithmetic from the default form,
    whose hydro HLL components are combined in FP64"""
    a = _run(P.orszag_tang(32), N.FP64, t_end=0.05)
    ref = a.download()
    b = _run(P.orszag_tang(32), N.MIXED, t_end=0.05)
    monkeypatch.setenv("CUMC_MX_HLL", "fp32")
    c = _run(P.orszag_tang(32), N.MIXED, t_end=0.05)
    db, dc = b.download(), c.download()
    rel_c = rel_l1_interior(dc, ref)
    assert rel_c[0] <= RHO_L1_TOL, rel_c
    assert not np.array_equal(db["cons"], dc["cons"])
