"""Parity of the CUDA path (through the C-ABI) with the FP64 CPU oracle.

The FP64 path is compiled without FMA contraction and evaluates every
expression in the reference's order, so on the small cases below it must agree
with the oracle bit for bit (max |diff| == 0). The full Brio-Wu run is checked
against the FP64 parity bar: relative L1 <= 1e-10 per conserved variable.
"""
import numpy as np
import pytest

from cumpic_b200 import _native as N
from cumpic_b200 import problems as P
from compare import diffs, rel_l1_interior

pytestmark = pytest.mark.gpu

BITWISE = 0.0
REL_L1_TOL = 1.0e-10  # FP64 parity bar (per conserved variable, at t_end)


def _pair(problem, threads=8):
    from cumpic_b200.solver import CUMC3D
    from _oracle import Oracle
    g = CUMC3D(problem)
    o = Oracle(problem, threads=threads)
    for s in (g, o):
        s.upload()
        s.initial_update()
    return g, o


def _assert_bitwise(g, o, what=""):
    d = diffs(g.download(), o.download())
    bad = {k: v for k, v in d.items() if v > BITWISE}
    assert not bad, f"{what}: {bad}"


SMALL = [
    ("brio_wu_x", lambda: P.brio_wu(64, 4, 4, axis=0)),
    ("brio_wu_y", lambda: P.brio_wu(4, 48, 5, axis=1)),
    ("brio_wu_z", lambda: P.brio_wu(3, 4, 40, axis=2)),
    ("orszag_tang_16", lambda: P.orszag_tang(16)),
    ("orszag_tang_ragged", lambda: P.orszag_tang(12, ny=10, nz=7)),
    ("orszag_tang_tvd", lambda: P.orszag_tang(12, recon=N.TVDMM)),
    ("torus_small", lambda: P.torus(24, 16, 8)),
    ("torus_small_q1_once", lambda: P.torus(20, 12, 6, geom_source_repeat=1)),
    ("cylindrical_shell", lambda: P.shell(N.CYLINDRICAL, 16, 12, 10)),
    ("torus_cylindrical", lambda: P.torus_cyl(24, 6, 20)),
    ("spherical_shell", lambda: P.shell(N.SPHERICAL, 14, 12, 10)),
]


@pytest.mark.parametrize("name,make", SMALL, ids=[s[0] for s in SMALL])
def test_initial_update_bitwise(name, make):
    g, o = _pair(make())
    _assert_bitwise(g, o, "initial_update")


@pytest.mark.parametrize("name,make", SMALL, ids=[s[0] for s in SMALL])
def test_spatial_lrk_bitwise(name, make):
    g, o = _pair(make())
    lg, lo = g.spatial(), o.spatial()
    nz, ny, nx = (s - 6 for s in g.shape)
    sl = (slice(2, nz + 3), slice(2, ny + 3), slice(2, nx + 3))
    d = np.abs(lg[sl] - lo[sl]).max(axis=(0, 1, 2))
    assert np.all(d == 0.0), d


@pytest.mark.parametrize("name,make", SMALL, ids=[s[0] for s in SMALL])
def test_steps_bitwise(name, make):
    g, o = _pair(make())
    for n in range(5):
        dg, do = g.finddt(), o.finddt()
        assert dg == do, (n, dg, do)
        g.rungekutta(dg)
        o.rungekutta(do)
    _assert_bitwise(g, o, "after 5 steps")


def test_brio_wu_full_t_end():
    """Brio-Wu 512x4x4 to t_end=0.1 (config 1), cell by cell."""
    p = P.brio_wu(512, 4, 4)
    g, o = _pair(p)
    ng = g.run(p.t_end)
    no = o.run(p.t_end)
    assert ng == no
    assert g.global_time == o.global_time == p.t_end
    a, b = g.download(), o.download()
    rel = rel_l1_interior(a, b)
    assert max(rel.values()) <= REL_L1_TOL, rel
    d = diffs(a, b)
    assert max(d.values()) == 0.0, d


def test_advance_matches_host_loop():
    """cumc_advance (dt on the device, CUDA graph) == finddt/rungekutta from the host."""
    from cumpic_b200.solver import CUMC3D
    p = P.orszag_tang(16)
    a = CUMC3D(p)
    b = CUMC3D(p)
    for s in (a, b):
        s.upload()
        s.initial_update()
    for _ in range(6):
        a.step()
    b.advance(6)
    assert a.global_time == b.global_time
    d = diffs(a.download(), b.download())
    assert max(d.values()) == 0.0, d


def test_advance_stops_at_t_end():
    from cumpic_b200.solver import CUMC3D
    p = P.brio_wu(64, 4, 4)
    g = CUMC3D(p)
    g.upload()
    g.initial_update()
    n1 = g.run(0.02, 10000)
    assert g.global_time == 0.02
    assert g.run(0.02, 50) == 0  # the loop condition already fails: no step


def test_divb_roundoff():
    from cumpic_b200.solver import CUMC3D
    p = P.orszag_tang(24)
    g = CUMC3D(p)
    g.upload()
    g.initial_update()
    g.advance(20)
    signed, norm = g.find_divb()
    assert norm <= 1.0e-12, norm


def test_uniform_state_preserved():
    p = P.orszag_tang(8)
    sl = (slice(2, 11), slice(2, 11), slice(2, 11))
    p.prim[sl + (slice(0, 8),)] = [1.0, 0.1, -0.2, 0.3, 0.6, 0.2, 0.1, -0.3]
    p.eps[sl] = 0.6 / 1.0 / (p.ggas - 1.0)
    g, o = _pair(p)
    for _ in range(3):
        g.step()
        o.step()
    a = g.download()
    nz, ny, nx = (s - 6 for s in g.shape)
    rho = a["prim"][3:nz + 3, 3:ny + 3, 3:nx + 3, 0]
    assert np.all(rho == rho.flat[0])
    _assert_bitwise(g, o)


@pytest.mark.parametrize("flags", [(2, 2, 2, 2, 2, 2), (3, 1, 4, 2, 0, 0), (1, 2, 3, 4, 4, 2)])
def test_reflecting_axis_equatorial_boundaries(flags):
    p = P.orszag_tang(10, ny=8, nz=6)
    p.boundary_flag = flags
    g, o = _pair(p)
    for _ in range(3):
        dg, do = g.finddt(), o.finddt()
        assert dg == do
        g.rungekutta(dg)
        o.rungekutta(do)
    _assert_bitwise(g, o, f"flags {flags}")


def test_call_order_and_config_errors():
    from cumpic_b200.solver import CUMC3D
    p = P.orszag_tang(8)
    g = CUMC3D(p)
    with pytest.raises(N.CumcError) as e:
        g.rungekutta(1e-3)
    assert e.value.code == N.CUMC_ERR_STATE
    q = P.orszag_tang(8)
    q.boundary_flag = (4, 1, 0, 0, 0, 0)
    with pytest.raises(N.CumcError) as e:
        CUMC3D(q)
    assert e.value.code == N.CUMC_ERR_CONFIG
    # a dt that is negative or not finite is refused; the state is left as it was
    g.upload()
    g.initial_update()
    before = g.download()
    for bad in (-1e-3, float("nan"), float("inf")):
        with pytest.raises(N.CumcError) as e:
            g.rungekutta(bad)
        assert e.value.code == N.CUMC_ERR_ARG
    after = g.download()
    assert all(np.array_equal(before[k], after[k]) for k in before)
    g.rungekutta(0.0)  # a zero step is allowed


@pytest.mark.parametrize("precision", [N.FP64, N.MIXED])
def test_nonfinite_state_is_reported(precision):
    """A NaN injected into the uploaded model is flagged on the device and
    reported by the next finddt as CUMC_ERR_NONFINITE (the reference passes
    NaN and negative pressure through silently, solver/utop.f90:63)."""
    from cumpic_b200.solver import CUMC3D
    p = P.orszag_tang(8, precision=precision)
    p.prim[6, 6, 6, 0] = float("nan")  # eps would be floored by CUSTOM_CHECKRHO's MAX(eps, 0)
    g = CUMC3D(p)
    g.upload()
    g.initial_update()
    g.rungekutta(1e-3)
    with pytest.raises(N.CumcError) as e:
        g.finddt()
    assert e.value.code == N.CUMC_ERR_NONFINITE


SWEEP_MODES = ["simple", "tile", "walkx", "walksm", "walkreg", "xwarp", "xface", "fused", "fused_notma"]


@pytest.mark.parametrize("mode", SWEEP_MODES)
def test_sweep_variants_bitwise(mode, monkeypatch):
    """Every sweep kernel variant (CUMC_SWEEP, read at cumc_init) gives the
    default variant's bits, the fused stage (flux differences in the sweeps,
    x rows staged by TMA) included; ragged sizes exercise partial blocks,
    segments and x staging chunks, and the odd row pitch of nx = 37 the fused
    stage's directly loaded x rows."""
    from cumpic_b200.solver import CUMC3D
    out = {}
    for m in (None, mode):
        if m is None:
            monkeypatch.delenv("CUMC_SWEEP", raising=False)
        else:
            monkeypatch.setenv("CUMC_SWEEP", m)
        for name, prob in (("ot", P.orszag_tang(37, ny=29, nz=70)), ("tvd", P.orszag_tang(21, recon=N.TVDMM)),
                           ("torus", P.torus(24, 16, 8)), ("even", P.orszag_tang(58, ny=20, nz=13)),
                           ("cyl", P.shell(N.CYLINDRICAL, 30, 14, 9))):
            g = CUMC3D(prob)
            g.upload()
            g.initial_update()
            for _ in range(2):
                g.rungekutta(g.finddt())
            out[(m, name)] = g.download()
            g.close()
    for name in ("ot", "tvd", "torus", "even", "cyl"):
        d = diffs(out[(None, name)], out[(mode, name)])
        assert all(v == 0.0 for v in d.values()), (name, d)


def test_fused_stage_stages_x_rows_by_tma(monkeypatch):
    """CUMC_SWEEP=fused runs the fused sweeps, staging the x rows by bulk
    tensor copies whenever the row pitch allows (nx + 6 even)"""
    from cumpic_b200.solver import CUMC3D
    monkeypatch.delenv("CUMC_SWEEP", raising=False)
    assert CUMC3D(P.orszag_tang(16)).query(N.Q_FUSED) == 0
    assert CUMC3D(P.orszag_tang(16)).query(N.Q_X_STAGING) == -1
    monkeypatch.setenv("CUMC_SWEEP", "fused")
    assert CUMC3D(P.orszag_tang(16)).query(N.Q_FUSED) == 1
    assert CUMC3D(P.orszag_tang(16)).query(N.Q_X_STAGING) == 1
    assert CUMC3D(P.orszag_tang(17)).query(N.Q_X_STAGING) == 0
    assert CUMC3D(P.orszag_tang(16, precision=N.MIXED)).query(N.Q_FUSED) == 0
    monkeypatch.setenv("CUMC_SWEEP", "fused_notma")
    assert CUMC3D(P.orszag_tang(16)).query(N.Q_X_STAGING) == 0


def test_emf_ct_tiles_equal_the_pair(monkeypatch):
    """the tiled EMF + CT kernel (default) gives the bits of k_emf + k_ct
    (CUMC_EMF=pair) on Cartesian, cylindrical and spherical grids, ragged
    tiles and short z segments included"""
    from cumpic_b200.solver import CUMC3D
    out = {}
    for mode in (None, "pair"):
        if mode:
            monkeypatch.setenv("CUMC_EMF", mode)
        else:
            monkeypatch.delenv("CUMC_EMF", raising=False)
        for name, prob in (("ot", P.orszag_tang(37, ny=29, nz=70)), ("cyl", P.shell(N.CYLINDRICAL, 30, 14, 9)),
                           ("torus", P.torus(24, 16, 8))):
            g = CUMC3D(prob)
            g.upload()
            g.initial_update()
            for _ in range(2):
                g.rungekutta(g.finddt())
            out[(mode, name)] = g.download()
            g.close()
    for name in ("ot", "cyl", "torus"):
        d = diffs(out[(None, name)], out[("pair", name)])
        assert all(v == 0.0 for v in d.values()), (name, d)
