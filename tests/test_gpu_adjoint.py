"""The discrete adjoint (cumc_adjoint_run).

Two checks, both with the dt sequence frozen as the adjoint records it:

1. Exact: against the tangent-linear run of the FP64 oracle
   (_oracle.TangentOracle), the FP64 reference gradient. Both differentiate
   the same discrete map with the same branches (the CUDA forward pass is
   bit-identical to the oracle), so <grad, d> and the tangent derivative along
   d agree to round-off (bar 1e-9 relative) for every uploaded field, every
   objective, PPM and TVD, periodic and non-periodic boundaries. The base
   state is generic (smooth variations in every field): at a uniform field
   every limited slope sits on the limiter's kink and the map has no
   derivative there.
2. Central finite differences of the forward C-ABI along seeded random
   smooth directions of the initial velocity on the adjoint check
   configuration (periodic box, rho = p = 1, uniform B, smooth low-wavenumber
   velocity modes), step 1e-7 relative to the flow, bar 1e-6 relative.
"""
import dataclasses
import math

import numpy as np
import pytest

from cumpic_b200 import _native as N
from cumpic_b200 import problems as P

pytestmark = pytest.mark.gpu

FD_EPS = 1.0e-7  # relative to the field (directions are scaled to its amplitude)
FD_TOL = 1.0e-6
TL_TOL = 1.0e-9


def _live(shape):
    """masks of the uploaded entries the map reads: cell fields, face fields"""
    nz6, ny6, nx6 = shape
    nx, ny, nz = nx6 - 6, ny6 - 6, nz6 - 6
    cell = np.zeros(shape, bool)
    cell[3:nz + 3, 3:ny + 3, 3:nx + 3] = True
    faces = []
    for d in range(3):
        m = np.zeros(shape, bool)
        lo = [3, 3, 3]
        lo[d] = 2
        m[lo[2]:nz + 3, lo[1]:ny + 3, lo[0]:nx + 3] = True
        faces.append(m)
    return cell, faces


def generic_box(n, recon=N.PPMC, flags=(0, 0, 0, 0, 0, 0), seed=1):
    """Fourier box with smooth, seeded variations added to every field"""
    p0 = P.fourier_box(n, modes=4, kmax=1, amp=0.01)
    prim, eps = p0.prim.copy(), p0.eps.copy()
    x = (np.arange(-2, n + 4) - 0.5) / n
    X, Y, Z = x[None, None, :], x[None, :, None], x[:, None, None]
    rng = np.random.default_rng(seed)
    for q in (0, 1, 2, 3, 5, 6, 7):
        a = rng.uniform(0.05, 0.1) * (0.3 if q in (1, 2, 3) else 1.0)
        ph = rng.uniform(0, 2 * math.pi, 3)
        prim[..., q] += a * (np.sin(2 * math.pi * X + ph[0]) * np.cos(2 * math.pi * Y + ph[1]) +
                             np.sin(2 * math.pi * Z + ph[2]))
    eps *= 1 + 0.1 * np.sin(2 * math.pi * (X + 2 * Y) + 0.3) * np.cos(2 * math.pi * Z)
    keep = np.zeros(eps.shape, bool)
    keep[2:n + 3, 2:n + 3, 2:n + 3] = True
    prim[~keep] = 0.0
    eps[~keep] = 0.0
    return dataclasses.replace(p0, prim=prim, eps=eps, recon=recon, boundary_flag=tuple(flags))


def _dv(prob):
    """cell volumes of the active cells: dx dy dz, R dR dphi dz, d(r^3)/3 d(-cos) dphi"""
    nx, ny, nz = prob.nx, prob.ny, prob.nz
    # face arrays hold faces -3..n+3: cell j (1..n) spans f[j+2] .. f[j+3]
    xm, xp = prob.xf[3:nx + 3], prob.xf[4:nx + 4]
    dx = xp - xm
    dy = prob.yf[4:ny + 4] - prob.yf[3:ny + 3]
    dz = prob.zf[4:nz + 4] - prob.zf[3:nz + 3]
    if prob.coordinate == N.CYLINDRICAL:
        dx = 0.5 * (xp + xm) * dx
    elif prob.coordinate == N.SPHERICAL:
        dx = (xp ** 3 - xm ** 3) / 3.0
        dy = np.cos(prob.yf[3:ny + 3]) - np.cos(prob.yf[4:ny + 4])
    return dz[:, None, None] * dy[None, :, None] * dx[None, None, :]


def _objective(st, prob, kind, weights=None):
    a = (slice(3, prob.nz + 3), slice(3, prob.ny + 3), slice(3, prob.nx + 3))
    dv = _dv(prob)
    if kind == N.OBJ_MAGNETIC:
        return 0.5 * np.sum(np.sum(st["bcell"][a] ** 2, axis=-1) * dv)
    if kind == N.OBJ_KINETIC:
        pr = st["prim"][a]
        return 0.5 * np.sum(pr[..., 0] * np.sum(pr[..., 1:4] ** 2, axis=-1) * dv)
    cell, faces = _live(st["eps"].shape)
    J = np.sum(weights[..., :5][cell] * st["cons"][..., :5][cell])
    for d in range(3):
        J += np.sum(weights[..., 5 + d][faces[d]] * st["cons"][..., 5 + d][faces[d]])
    return J


def _objective_tangent(v, d, prob, kind, weights=None):
    """directional derivative of the objective from tangent values d at v"""
    a = (slice(3, prob.nz + 3), slice(3, prob.ny + 3), slice(3, prob.nx + 3))
    dv = _dv(prob)
    if kind == N.OBJ_MAGNETIC:
        return np.sum(np.sum(v["bcell"][a] * d["bcell"][a], axis=-1) * dv)
    if kind == N.OBJ_KINETIC:
        pv, pd = v["prim"][a], d["prim"][a]
        vsq = np.sum(pv[..., 1:4] ** 2, axis=-1)
        vdv = np.sum(pv[..., 1:4] * pd[..., 1:4], axis=-1)
        return np.sum((0.5 * pd[..., 0] * vsq + pv[..., 0] * vdv) * dv)
    return _objective({"cons": d["cons"], "eps": d["eps"]}, prob, N.OBJ_LINEAR, weights)


def _directions(prob, count, seed, fields=("rho", "v", "eps", "b")):
    shape = prob.eps.shape
    cell, faces = _live(shape)
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        dp = np.zeros(shape + (8,))
        de = np.zeros(shape)
        if "rho" in fields:
            dp[..., 0][cell] = rng.uniform(-1, 1, cell.sum())
        if "v" in fields:
            for q in (1, 2, 3):
                dp[..., q][cell] = rng.uniform(-1, 1, cell.sum())
        if "eps" in fields:
            de[cell] = rng.uniform(-1, 1, cell.sum())
        if "b" in fields:
            for d in range(3):
                dp[..., 5 + d][faces[d]] = rng.uniform(-1, 1, faces[d].sum())
        out.append((dp, de))
    return out


def _adjoint(prob, nsteps, ckpt, kind, weights=None):
    from cumpic_b200.solver import CUMC3D
    sim = CUMC3D(prob)
    sim.upload()
    return sim.adjoint(nsteps, ckpt, kind, weights=weights)


def _check_tangent(prob, nsteps, ckpt, kind, ndir=3, seed=11, weights=None):
    from _oracle import TangentOracle
    res = _adjoint(prob, nsteps, ckpt, kind, weights)
    tl = TangentOracle(prob, threads=8)
    worst = 0.0
    for dp, de in _directions(prob, ndir, seed):
        v, d = tl.run(dp, de, res["dts"])
        ref = _objective_tangent(v, d, prob, kind, weights)
        ad = float(np.sum(res["grad_prim"] * dp) + np.sum(res["grad_eps"] * de))
        rel = abs(ref - ad) / max(abs(ref), abs(ad), 1e-300)
        worst = max(worst, rel)
        assert rel <= TL_TOL, (ref, ad, rel)
    assert res["J"] == pytest.approx(_objective(v, prob, kind, weights), rel=1e-12)
    return worst


def test_adjoint_vs_tangent_linear_objective_one_step():
    prob = generic_box(10)
    w = np.random.default_rng(5).uniform(-1, 1, prob.prim.shape)
    _check_tangent(prob, 1, 1, N.OBJ_LINEAR, weights=w)


def test_adjoint_vs_tangent_magnetic_checkpointed():
    # 5 steps in segments of 2, 2 and 1: the recomputation crosses checkpoints
    _check_tangent(generic_box(12), 5, 2, N.OBJ_MAGNETIC)


def test_adjoint_vs_tangent_kinetic_tvd():
    _check_tangent(generic_box(10, recon=N.TVDMM), 3, 2, N.OBJ_KINETIC)


@pytest.mark.parametrize("flags", [(1, 1, 2, 2, 0, 0), (2, 1, 0, 0, 1, 2), (1, 2, 3, 4, 1, 1)])
def test_adjoint_vs_tangent_nonperiodic_boundaries(flags):
    prob = generic_box(10, flags=flags)
    w = np.random.default_rng(7).uniform(-1, 1, prob.prim.shape)
    _check_tangent(prob, 2, 1, N.OBJ_LINEAR, weights=w)


@pytest.mark.parametrize("coord,kind,recon", [(N.CYLINDRICAL, N.OBJ_LINEAR, N.PPMC),
                                               (N.SPHERICAL, N.OBJ_LINEAR, N.PPMC),
                                               (N.CYLINDRICAL, N.OBJ_MAGNETIC, N.TVDMM),
                                               (N.SPHERICAL, N.OBJ_KINETIC, N.PPMC)])
def test_adjoint_vs_tangent_curvilinear(coord, kind, recon):
    """flux-difference and CT factors and GEOM_SOURCE (added 8 times) of the
    cylindrical and spherical grids"""
    prob = P.shell(coord, 10, 8, 6, recon=recon)
    w = np.random.default_rng(9).uniform(-1, 1, prob.prim.shape) if kind == N.OBJ_LINEAR else None
    _check_tangent(prob, 2, 1, kind, weights=w)


def _density(st, prob, kind):
    """per-cell objective density (J is its sum)"""
    a = (slice(3, prob.nz + 3), slice(3, prob.ny + 3), slice(3, prob.nx + 3))
    if kind == N.OBJ_MAGNETIC:
        return 0.5 * np.sum(st["bcell"][a] ** 2, axis=-1) * _dv(prob)
    pr = st["prim"][a]
    return 0.5 * pr[..., 0] * np.sum(pr[..., 1:4] ** 2, axis=-1) * _dv(prob)


def smooth_velocity_directions(prob, count, seed, modes=8, kmax=2):
    """seeded random velocity directions from the box's own function space:
    sums of low-wavenumber modes e sin(2 pi k.x + phi) on the active cells,
    scaled to the velocity field's largest magnitude so that the step eps is
    relative to the flow. (A cell-by-cell random direction would seed density
    structure far below the grid scale of the flow and move limiter
    branches.)"""
    shape = prob.eps.shape
    cell, _ = _live(shape)
    n = prob.nx
    x = (np.arange(-2, n + 4) - 0.5) / n
    X, Y, Z = x[None, None, :], x[None, :, None], x[:, None, None]
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        dp = np.zeros(shape + (8,))
        for _m in range(modes):
            while True:
                kv = rng.integers(-kmax, kmax + 1, 3)
                if 0 < np.sqrt((kv ** 2).sum()) <= kmax:
                    break
            e = rng.normal(size=3)
            e /= np.linalg.norm(e)
            s = np.sin(2 * math.pi * (kv[0] * X + kv[1] * Y + kv[2] * Z) + rng.uniform(0, 2 * math.pi))
            for a in range(3):
                dp[..., 1 + a] += e[a] * s
        dp[~cell] = 0.0
        dp *= np.max(np.abs(prob.prim[..., 1:4][cell])) / np.max(np.abs(dp))
        out.append((dp, np.zeros(shape)))
    return out


# The magnetic energy of this small, short run moves by ~1e-5 of itself per
# unit velocity direction, so at the smallest step that keeps every limiter
# branch (1e-7) its central difference carries ~1e-6 of round-off; its bar is
# 2e-6. The exact check of the same gradient is the tangent comparison above.
@pytest.mark.parametrize("kind,tol", [(N.OBJ_KINETIC, FD_TOL), (N.OBJ_MAGNETIC, 2 * FD_TOL)])
def test_adjoint_finite_differences_velocity(kind, tol):
    """the adjoint check configuration (smaller box and fewer steps); the
    central difference is summed cell by cell so that the two runs' totals,
    which agree to ~1e-10 here, are not subtracted"""
    from cumpic_b200.solver import CUMC3D
    prob = P.fourier_box(24, modes=16, kmax=2)
    res = _adjoint(prob, 8, 4, kind)
    sim = CUMC3D(prob)

    def run(prim):
        sim.upload(prim, prob.eps)
        sim.initial_update()
        for dt in res["dts"]:
            sim.rungekutta(dt)
        return _density(sim.download(), prob, kind)

    assert res["J"] == pytest.approx(float(np.sum(run(prob.prim))), rel=1e-12)
    from _oracle import TangentOracle
    tl = TangentOracle(prob, threads=8)
    for dp, de in smooth_velocity_directions(prob, 4, 4):
        fd = float(np.sum(run(prob.prim + FD_EPS * dp) - run(prob.prim - FD_EPS * dp))) / (2 * FD_EPS)
        ad = float(np.sum(res["grad_prim"] * dp))
        v, d = tl.run(dp, de, res["dts"])
        ref = _objective_tangent(v, d, prob, kind)
        assert abs(ref - ad) <= TL_TOL * abs(ref), (ref, ad)
        assert abs(fd - ad) <= tol * max(abs(fd), abs(ad)), (fd, ad, ref)


def test_adjoint_checkpoint_interval_invariant_and_deterministic():
    """the gradient does not depend on the checkpoint interval and is the same
    bits on every run: the recomputed segments repeat the forward pass bit for
    bit, and every adjoint kernel adds its contributions in a fixed order (no
    atomics)"""
    from cumpic_b200.solver import CUMC3D
    prob = generic_box(10)
    grads, states = [], []
    for k in (1, 3, 7, 3):
        sim = CUMC3D(prob)
        sim.upload()
        grads.append(sim.adjoint(7, k, N.OBJ_MAGNETIC)["grad_prim"])
        states.append(sim.download()["cons"])
    for g, s in zip(grads[1:], states[1:]):
        assert np.array_equal(g, grads[0])
        assert np.array_equal(s, states[0])  # the context ends on the final state


def test_adjoint_autograd_harness():
    """torch.autograd.Function over the initial velocity, as a test harness"""
    torch = pytest.importorskip("torch")
    from cumpic_b200.solver import CUMC3D
    prob = P.fourier_box(12, modes=8, kmax=2)
    nsteps = 3

    class MagneticEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, vel):
            prim = prob.prim.copy()
            prim[..., 1:4] = vel.detach().cpu().numpy()
            sim = CUMC3D(dataclasses.replace(prob, prim=prim))
            sim.upload()
            r = sim.adjoint(nsteps, 2, N.OBJ_MAGNETIC)
            ctx.save_for_backward(torch.from_numpy(r["grad_prim"][..., 1:4].copy()))
            return torch.tensor(r["J"], dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (g,) = ctx.saved_tensors
            return gout * g

    vel = torch.tensor(prob.prim[..., 1:4], dtype=torch.float64, requires_grad=True)
    J = MagneticEnergy.apply(vel)
    J.backward()
    r = _adjoint(prob, nsteps, 2, N.OBJ_MAGNETIC)
    assert float(J.detach()) == r["J"]
    np.testing.assert_allclose(vel.grad.numpy(), r["grad_prim"][..., 1:4], rtol=1e-9, atol=1e-15)
    cell, _ = _live(prob.eps.shape)
    assert np.all(vel.grad.numpy()[~cell] == 0.0)  # ghosts are overwritten by initial_update
    assert np.any(vel.grad.numpy()[cell] != 0.0)


def test_adjoint_rejects_unsupported():
    from cumpic_b200.solver import CUMC3D
    for prob in (P.torus(12, 8, 4), dataclasses.replace(P.fourier_box(8), precision=N.MIXED)):
        sim = CUMC3D(prob)
        sim.upload()
        with pytest.raises(N.CumcError) as e:
            sim.adjoint(1, 1, N.OBJ_MAGNETIC)
        assert e.value.code == N.CUMC_ERR_CONFIG
