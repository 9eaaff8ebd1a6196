"""Initial models (the GET_MODEL step of solver/initial.f90:93) for the
workloads the hot path is measured and checked on.

Every generator returns a :class:`Problem`: the run-time configuration that the
reference fixes at compile time (solver/definition.f90:29-185,
model/<m>/src/defs.f90) plus the face coordinates (GETGRID,
solver/coords.f90:11-41) and the initial ``prim``/``eps`` arrays in the
reference's Fortran layout, here as C-ordered numpy arrays of shape
(nz+6, ny+6, nx+6, 8) and (nz+6, ny+6, nx+6). Like GET_MODEL, the generators
set indices 0:n and leave every other entry at zero.

Random inputs come from a counter-based generator (splitmix64 keyed on a seed
and the cell's global linear index), so every consumer of a problem sees the
same numbers.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import _native as N

IRHO, IVX, IVY, IVZ, ITAU, IBX, IBY, IBZ = range(8)


@dataclasses.dataclass
class Problem:
    name: str
    nx: int
    ny: int
    nz: int
    xf: np.ndarray  # faces -3..n+3
    yf: np.ndarray
    zf: np.ndarray
    coordinate: int
    boundary_flag: tuple
    ggas: float
    cfl: float
    t_end: float
    prim: np.ndarray
    eps: np.ndarray
    recon: int = N.PPMC
    model: int = N.MODEL_RIEMANN
    rho_floor: float = 0.0
    eps_floor: float = 0.0
    r_sh: float = 0.0
    geom_source_repeat: int = 8
    precision: int = N.FP64
    model_params: dict | None = None  # device-side generator parameters (cumc_model_torus)

    def config(self) -> N.CumcConfig:
        """Fill a cumc_config; the face arrays stay owned by this object."""
        c = N.CumcConfig()
        c.nx, c.ny, c.nz = self.nx, self.ny, self.nz
        for name in ("xf", "yf", "zf"):
            arr = np.ascontiguousarray(getattr(self, name), dtype=np.float64)
            setattr(self, name, arr)
            setattr(c, name, arr.ctypes.data_as(N.POINTER(N.c_double)))
        c.coordinate = self.coordinate
        for i, f in enumerate(self.boundary_flag):
            c.boundary_flag[i] = int(f)
        c.ggas = self.ggas
        c.cfl = self.cfl
        c.recon = self.recon
        c.solver = N.HLL
        c.precision = self.precision
        c.model = self.model
        c.rho_floor = self.rho_floor
        c.eps_floor = self.eps_floor
        c.r_sh = self.r_sh
        c.geom_source_repeat = self.geom_source_repeat
        return c

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def uniform_faces(start: float, end: float, n: int) -> np.ndarray:
    """GETGRID (solver/coords.f90:24-32): xF(j) = x_start + j*dx, j = -3..n+3."""
    d = (end - start) / float(n)
    return np.array([start + float(j) * d for j in range(-3, n + 4)], dtype=np.float64)


def _empty(nx: int, ny: int, nz: int):
    return (np.zeros((nz + 6, ny + 6, nx + 6, 8), dtype=np.float64),
            np.zeros((nz + 6, ny + 6, nx + 6), dtype=np.float64))


def _centres(f: np.ndarray) -> np.ndarray:
    """GET_COORD (solver/coords.f90:63-65) for indices -2..n+3 (array index i+2)."""
    return 0.5 * (f[1:] + f[:-1])


def uniform01(seed: int, index: np.ndarray) -> np.ndarray:
    """splitmix64(seed, index) mapped to [0, 1) with 53 bits."""
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) * np.uint64(0xD1B54A32D192ED03)
             + (index.astype(np.uint64) + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _linear_index(nx, ny, nz):
    """global linear index of cells 0:n in each direction (periodic image of 0 is n)."""
    j = (np.arange(0, nx + 1) - 1) % nx
    k = (np.arange(0, ny + 1) - 1) % ny
    l = (np.arange(0, nz + 1) - 1) % nz
    return (j[None, None, :] + nx * (k[None, :, None] + ny * l[:, None, None])).astype(np.int64)


def brio_wu(nx: int = 512, ny: int = 4, nz: int = 4, axis: int = 0, ggas: float = 2.0,
            cfl: float = 0.4, t_end: float = 0.1, recon: int = N.PPMC) -> Problem:
    """Brio-Wu shock tube (model/riemann/src/riemann1d.f90:54-89) along `axis`.

    The tube direction has n cells on [0, 1]; the other two directions use the
    same cell size, outflow along the tube and periodic across it.
    """
    n = (nx, ny, nz)
    L = 1.0 / n[axis]
    faces = [uniform_faces(0.0, 1.0 if a == axis else n[a] * L, n[a]) for a in range(3)]
    prim, eps = _empty(nx, ny, nz)
    c = _centres(faces[axis])  # index i+2 -> cell i
    x = c[2: n[axis] + 3]      # cells 0..n
    left = x <= 0.5
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    bt = np.where(left, 1.0, -1.0)
    ibn = IBX + axis
    ibt = IBX + (axis + 1) % 3  # By for an x tube (riemann1d.f90:66,70)
    shape = [1, 1, 1]
    shape[2 - axis] = n[axis] + 1
    sl = (slice(2, nz + 3), slice(2, ny + 3), slice(2, nx + 3))
    view = prim[sl]
    view[..., IRHO] = rho.reshape(shape)
    view[..., ITAU] = p.reshape(shape)
    view[..., ibt] = bt.reshape(shape)
    view[..., ibn] = 0.75
    eps[sl] = (p / rho / (ggas - 1.0)).reshape(shape)
    flags = [0, 0, 0, 0, 0, 0]
    flags[2 * axis] = flags[2 * axis + 1] = 1
    return Problem(f"brio_wu_{'xyz'[axis]}", nx, ny, nz, faces[0], faces[1], faces[2], N.CARTESIAN,
                   tuple(flags), ggas, cfl, t_end, prim, eps, recon=recon, model=N.MODEL_RIEMANN)


def orszag_tang(n: int = 256, ggas: float = 5.0 / 3.0, cfl: float = 0.4, t_end: float = 0.5,
                bscale: float = 1.0, seed: int = 1, ny: int | None = None, nz: int | None = None,
                recon: int = N.PPMC, precision: int = N.FP64) -> Problem:
    """3-D Orszag-Tang vortex on the periodic unit cube.

    rho = 25/(36 pi), p = 5/(12 pi), v = (-sin 2 pi y, sin 2 pi x, vz) with
    vz = 0.01 (2u - 1), u uniform from the seeded generator. The face field is
    the discrete curl of A_z = (cos 4 pi x / 4 pi + cos 2 pi y / 2 pi)/sqrt(4 pi)
    sampled on z-edges, so its discrete divergence vanishes to round-off;
    `bscale` multiplies the field (bscale=10 gives plasma beta ~0.05).
    """
    nx = n
    ny = n if ny is None else ny
    nz = n if nz is None else nz
    xf, yf, zf = uniform_faces(0.0, 1.0, nx), uniform_faces(0.0, 1.0, ny), uniform_faces(0.0, 1.0, nz)
    prim, eps = _empty(nx, ny, nz)
    xc, yc = _centres(xf)[2:nx + 3], _centres(yf)[2:ny + 3]
    rho = 25.0 / (36.0 * math.pi)
    p = 5.0 / (12.0 * math.pi)
    b0 = bscale / math.sqrt(4.0 * math.pi)
    sl = (slice(2, nz + 3), slice(2, ny + 3), slice(2, nx + 3))
    v = prim[sl]
    v[..., IRHO] = rho
    v[..., ITAU] = p
    v[..., IVX] = (-np.sin(2.0 * math.pi * yc))[None, :, None]
    v[..., IVY] = (np.sin(2.0 * math.pi * xc))[None, None, :]
    u = uniform01(seed, _linear_index(nx, ny, nz))
    v[..., IVZ] = 0.01 * (2.0 * u - 1.0)
    # A_z on z-edges (xF(j), yF(k)), j, k = -1..n
    xe, ye = xf[2:nx + 4], yf[2:ny + 4]
    az = b0 * (np.cos(4.0 * math.pi * xe)[None, :] / (4.0 * math.pi)
               + np.cos(2.0 * math.pi * ye)[:, None] / (2.0 * math.pi))  # [k+1, j+1]
    dx = (xf[3:nx + 4] - xf[2:nx + 3])  # widths of cells 0..n
    dy = (yf[3:ny + 4] - yf[2:ny + 3])
    bx = (az[1:, 1:] - az[:-1, 1:]) / dy[:, None]       # faces j=0..n, rows k=0..n
    by = -(az[1:, 1:] - az[1:, :-1]) / dx[None, :]
    v[..., IBX] = bx[None, :, :]
    v[..., IBY] = by[None, :, :]
    eps[sl] = p / rho / (ggas - 1.0)
    name = f"orszag_tang_{nx}" + (f"_b{bscale:g}" if bscale != 1.0 else "")
    return Problem(name, nx, ny, nz, xf, yf, zf, N.CARTESIAN, (0, 0, 0, 0, 0, 0), ggas, cfl, t_end,
                   prim, eps, recon=recon, model=N.MODEL_RIEMANN, precision=precision)


def fourier_box(n: int = 128, ggas: float = 5.0 / 3.0, cfl: float = 0.4, modes: int = 32, amp: float = 0.01,
                kmax: int = 4, seed: int = 3) -> Problem:
    """Smooth periodic box: rho = p = 1, B = (1, 0.5, 0.5)/sqrt(4 pi) uniform,
    v = sum over `modes` of amp * e_m * sin(2 pi k_m . x + phi_m) with integer
    0 < |k_m| <= kmax, unit e_m and phase phi_m drawn from the seeded generator."""
    xf = yf = zf = uniform_faces(0.0, 1.0, n)
    prim, eps = _empty(n, n, n)
    c = _centres(xf)[2:n + 3]
    X = c[None, None, :]
    Y = c[None, :, None]
    Z = c[:, None, None]
    draws = uniform01(seed, np.arange(64 * modes, dtype=np.int64))
    vel = np.zeros((n + 1, n + 1, n + 1, 3))
    q = 0
    for m in range(modes):
        while True:
            kv = np.floor(draws[q:q + 3] * (2 * kmax + 1)).astype(int) - kmax
            q += 3
            if 0 < np.sqrt((kv ** 2).sum()) <= kmax:
                break
        e = draws[q:q + 3] - 0.5
        q += 3
        e = e / np.linalg.norm(e)
        phi = 2.0 * math.pi * draws[q]
        q += 1
        arg = 2.0 * math.pi * (kv[0] * X + kv[1] * Y + kv[2] * Z) + phi
        s = amp * np.sin(arg)
        for a in range(3):
            vel[..., a] += e[a] * s
    sl = (slice(2, n + 3), slice(2, n + 3), slice(2, n + 3))
    v = prim[sl]
    v[..., IRHO] = 1.0
    v[..., ITAU] = 1.0
    v[..., IVX:IVZ + 1] = vel
    s4 = 1.0 / math.sqrt(4.0 * math.pi)
    v[..., IBX], v[..., IBY], v[..., IBZ] = s4, 0.5 * s4, 0.5 * s4
    eps[sl] = 1.0 / 1.0 / (ggas - 1.0)
    return Problem(f"fourier_box_{n}", n, n, n, xf, yf, zf, N.CARTESIAN, (0, 0, 0, 0, 0, 0), ggas, cfl, 0.0,
                   prim, eps, model=N.MODEL_RIEMANN)


def shell(coordinate: int, nx: int = 16, ny: int = 12, nz: int = 10, ggas: float = 5.0 / 3.0, cfl: float = 0.4,
          seed: int = 5, boundary_flag: tuple | None = None, recon: int = N.PPMC) -> Problem:
    """Smooth magnetised state on a curvilinear grid, for the geometric terms
    (flux-difference and CT factors, GEOM_SOURCE) without a model's source:
    a cylindrical annulus R in [1, 2], phi in [0, pi], z in [0, 1], or a
    spherical shell r in [1, 2], theta in [pi/4, 3pi/4], phi in [0, pi/2].
    Every field varies smoothly (seeded phases): rho, p = 1 + 0.2 s, v = 0.1 s,
    B = 0.3 + 0.1 s, with s a sum of sines of the cell's index coordinates.
    Default flags: copy at both radial ends, mirror at the theta ends, the
    rest periodic."""
    if coordinate == N.CYLINDRICAL:
        xf, yf, zf = uniform_faces(1.0, 2.0, nx), uniform_faces(0.0, math.pi, ny), uniform_faces(0.0, 1.0, nz)
        flags = (1, 1, 0, 0, 0, 0)
    elif coordinate == N.SPHERICAL:
        xf = uniform_faces(1.0, 2.0, nx)
        yf = uniform_faces(0.25 * math.pi, 0.75 * math.pi, ny)
        zf = uniform_faces(0.0, 0.5 * math.pi, nz)
        flags = (1, 1, 2, 2, 0, 0)
    else:
        raise ValueError("shell() builds a cylindrical or spherical grid")
    prim, eps = _empty(nx, ny, nz)
    X = ((np.arange(-3, nx + 3) + 0.5) / nx)[None, None, :]
    Y = ((np.arange(-3, ny + 3) + 0.5) / ny)[None, :, None]
    Z = ((np.arange(-3, nz + 3) + 0.5) / nz)[:, None, None]
    ph = 2.0 * math.pi * uniform01(seed, np.arange(24, dtype=np.int64)).reshape(8, 3)
    for q in range(8):
        s = (np.sin(2 * math.pi * X + ph[q, 0]) * np.cos(2 * math.pi * Y + ph[q, 1]) +
             np.sin(2 * math.pi * Z + ph[q, 2]))
        prim[..., q] = (1.0 + 0.2 * s if q in (IRHO, ITAU) else 0.1 * s if q <= IVZ else 0.3 + 0.1 * s)
    eps[...] = prim[..., ITAU] / prim[..., IRHO] / (ggas - 1.0)
    return Problem(f"shell_{coordinate}_{nx}x{ny}x{nz}", nx, ny, nz, xf, yf, zf, coordinate,
                   tuple(boundary_flag) if boundary_flag is not None else flags, ggas, cfl, 0.0, prim, eps,
                   recon=recon, model=N.MODEL_RIEMANN)


def torus(nr: int = 192, nth: int = 128, nph: int = 64, ggas: float = 5.0 / 3.0, cfl: float = 0.4,
          r_in: float = 2.0, r_out: float = 50.0, s_in: float = 6.0, s_max: float = 10.0, q_grad: float = 2.0,
          rho_max: float = 1.0, rho_fac: float = 1.0e-5, rho_cut: float = 0.2, beta: float = 100.0,
          noise: float = 0.01, seed: int = 2, geom_source_repeat: int = 8, host_arrays: bool = True) -> Problem:
    """Magnetised constant-angular-momentum torus on a spherical-polar grid,
    following model/torus_sph/src/model.f90:8-284 with a point-mass potential
    (r_sh = 0), log-spaced radial faces r_f(j) = r_in (r_out/r_in)^(j/nr) (the
    CUSTOM_GRID hook, solver/coords.f90:37), A_phi = max(rho - rho_cut, 0)
    (model/torus_cyn/src/model.f90:126, zero elsewhere) normalised to
    p_gas,max / p_mag,max = beta, and seeded density noise rho*(1 + noise(2u-1)).
    With host_arrays=False only the grid and configuration are built (prim
    and eps are None): the state then comes from the device-side generator
    (CUMC3D.generate_model, cumc_model_torus), which builds the same torus on
    the GPU."""
    r_sh = 0.0
    xf = np.array([r_in * (r_out / r_in) ** (j / nr) for j in range(-3, nr + 4)], dtype=np.float64)
    yf = uniform_faces(0.05 * math.pi, 0.95 * math.pi, nth)
    zf = uniform_faces(0.0, 2.0 * math.pi, nph)
    prim, eps = _empty(nr, nth, nph)

    def schw(r):
        return -1.0 / (r - r_sh)

    params = dict(r_sh=r_sh, s_in=s_in, s_max=s_max, q_grad=q_grad, rho_max=rho_max, rho_fac=rho_fac,
                  rho_cut=rho_cut, beta=beta, noise=noise, seed=seed)
    lkep2 = s_max ** (2.0 * q_grad - 1.0) / (s_max - r_sh) ** 2
    c_const = schw(s_in) - lkep2 * s_in ** (2.0 - 2.0 * q_grad) / (2.0 - 2.0 * q_grad)
    h_max = -schw(s_max) + lkep2 * s_max ** (2.0 - 2.0 * q_grad) / (2.0 - 2.0 * q_grad) + c_const
    k_poly = h_max * (ggas - 1.0) / ggas / rho_max ** (ggas - 1.0)
    if k_poly < 0.0:
        raise ValueError("the polytropic constant is negative")
    rho_floor = rho_fac * rho_max
    eps_floor = k_poly * rho_floor ** (ggas - 1.0) / (ggas - 1.0)
    if not host_arrays:
        return Problem(f"torus_{nr}x{nth}x{nph}", nr, nth, nph, xf, yf, zf, N.SPHERICAL, (1, 1, 3, 3, 0, 0), ggas,
                       cfl, 0.0, None, None, model=N.MODEL_TORUS_SPH, rho_floor=rho_floor, eps_floor=eps_floor,
                       r_sh=r_sh, geom_source_repeat=geom_source_repeat, model_params=params)
    rc = _centres(xf)   # index i+2 -> cell i
    tc = _centres(yf)
    r = rc[3:nr + 3][None, None, :]
    th = tc[3:nth + 3][None, :, None]
    s_eq = r * np.sin(th)
    h = -schw(r) + lkep2 * s_eq ** (2.0 - 2.0 * q_grad) / (2.0 - 2.0 * q_grad) + c_const
    h = np.maximum(h, 0.0)
    rho_loc = (h * (ggas - 1.0) / ggas / k_poly) ** (1.0 / (ggas - 1.0))
    rho_a = rho_fac * rho_max
    inside = (rho_loc > rho_a) & (s_eq >= s_in)
    rho = np.where(inside, rho_loc, rho_a) * np.ones((nph, 1, 1))
    vph = np.where(inside, np.sqrt(lkep2) * s_eq ** (-q_grad) * s_eq, 0.0) * np.ones((nph, 1, 1))
    sl1 = (slice(3, nph + 3), slice(3, nth + 3), slice(3, nr + 3))
    v = prim[sl1]
    v[..., IRHO] = rho
    v[..., IVZ] = vph
    v[..., ITAU] = k_poly * rho ** ggas
    eps[sl1] = k_poly * rho ** (ggas - 1.0) / (ggas - 1.0)
    # vector potential on cells 1:n, zero elsewhere (-2:n+3)
    A = np.zeros((nph + 6, nth + 6, nr + 6))
    A[sl1] = np.where(rho >= rho_cut, (rho - rho_cut) / rho_max, 0.0)
    # A_corner(j,k,l) = average over (j,j+1) x (l,l+1) on 1:n (model.f90:140-146)
    Ac = np.zeros_like(A)
    Ac[sl1] = 0.25 * (A[3:nph + 3, 3:nth + 3, 3:nr + 3] + A[3:nph + 3, 3:nth + 3, 4:nr + 4]
                      + A[4:nph + 4, 3:nth + 3, 3:nr + 3] + A[4:nph + 4, 3:nth + 3, 4:nr + 4])
    # face fields on 0:n (model.f90:153-162)
    J = np.arange(0, nr + 1)
    K = np.arange(0, nth + 1)
    xF = lambda j: xf[j + 3]  # noqa: E731
    yF = lambda k: yf[k + 3]  # noqa: E731
    Ajk = Ac[2:nph + 3][:, K + 2][:, :, J + 2]          # A_corner(j,k,l) for l=0..n
    Ajkm = Ac[2:nph + 3][:, K + 1][:, :, J + 2]         # (j,k-1,l)
    Ajmk = Ac[2:nph + 3][:, K + 2][:, :, J + 1]         # (j-1,k,l)
    sinf = np.sin(yF(K))[None, :, None]
    sinfm = np.sin(yF(K - 1))[None, :, None]
    dcos = (np.cos(yF(K - 1)) - np.cos(yF(K)))[None, :, None]
    xfj = xF(J)[None, None, :]
    xfjm = xF(J - 1)[None, None, :]
    xl = 0.5 * (xfj + xfjm)
    dxl = xfj - xfjm
    bx = (sinf * Ajk - sinfm * Ajkm) / (xfj * dcos)
    by = -(xfj * Ajk - xfjm * Ajmk) / (xl * dxl)
    sl0 = (slice(2, nph + 3), slice(2, nth + 3), slice(2, nr + 3))
    prim[sl0 + (IBX,)] = bx
    prim[sl0 + (IBY,)] = by
    # beta normalisation (model.f90:176-219)
    bcx = 0.5 * (prim[sl1 + (IBX,)] + prim[3:nph + 3, 3:nth + 3, 2:nr + 2, IBX])
    bcy = 0.5 * (prim[sl1 + (IBY,)] + prim[3:nph + 3, 2:nth + 2, 3:nr + 3, IBY])
    pgas_max = prim[sl1 + (ITAU,)].max()
    pmag_max = (0.5 * (bcx ** 2 + bcy ** 2)).max()
    norm = math.sqrt((pgas_max / pmag_max) / beta) if pmag_max > 0 else 0.0
    prim[sl0 + (IBX,)] *= norm
    prim[sl0 + (IBY,)] *= norm
    # density noise where rho > rho_floor (model.f90:256-265, seeded)
    idx = _linear_index(nr, nth, nph)[1:, 1:, 1:]
    u = uniform01(seed, idx)
    d = prim[sl1 + (IRHO,)]
    prim[sl1 + (IRHO,)] = np.where(d > rho_floor, d + d * (u - 0.5) / 0.5 * noise, d)
    return Problem(f"torus_{nr}x{nth}x{nph}", nr, nth, nph, xf, yf, zf, N.SPHERICAL, (1, 1, 3, 3, 0, 0), ggas,
                   cfl, 0.0, prim, eps, model=N.MODEL_TORUS_SPH, rho_floor=rho_floor, eps_floor=eps_floor,
                   r_sh=r_sh, geom_source_repeat=geom_source_repeat, model_params=params)


def torus_cyl(nr: int = 32, nph: int = 8, nz: int = 32, ggas: float = 5.0 / 3.0, cfl: float = 0.4,
              r_in: float = 1.5, r_out: float = 8.0, z_half: float = 3.0, r_sh: float = 1.0, s_in: float = 3.0,
              s_max: float = 4.7, q_grad: float = 2.0, rho_max: float = 1.0, rho_fac: float = 1.0e-4,
              rho_cut: float = 0.5, beta: float = 100.0, noise: float = 1.0e-4, seed: int = 4,
              geom_source_repeat: int = 8, host_arrays: bool = True) -> Problem:
    """Magnetised torus on a cylindrical grid (R, phi, z), following
    model/torus_cyn/src/model.f90:8-284: the pseudo-Newtonian potential
    -1/(sqrt(R^2 + z^2) - r_sh), angular momentum l^2 ~ R^(2-2q) from the
    Keplerian value at s_max, polytropic p = K rho^gamma with the torus
    inside R >= s_in and the floor rho_fac*rho_max outside; v_phi = sqrt(l_kep^2)
    R^(1-q); A_phi = max(rho - rho_cut, 0)/rho_max on the cells, averaged over
    (R, z) to the corners, B_R = -dA/dz and B_z = (1/R) d(R A)/dR on the faces,
    normalised to p_gas,max / p_mag,max = beta (the cell B_z of that ratio
    averages over the phi neighbour, as model.f90:166 does); then seeded
    density noise rho (1 + noise (2u - 1)) where rho > rho_floor. Faces:
    outflow in R and z (the model's ghost clamps apply there), periodic in phi.
    With host_arrays=False only the grid and configuration are built; the
    device-side generator (CUMC3D.generate_model) then builds the state."""
    xf = uniform_faces(r_in, r_out, nr)
    yf = uniform_faces(0.0, 2.0 * math.pi, nph)
    zf = uniform_faces(-z_half, z_half, nz)
    prim, eps = _empty(nr, nph, nz)

    def schw(r, z):
        return -1.0 / (np.sqrt(r ** 2 + z ** 2) - r_sh)

    lkep2 = s_max ** (2.0 * q_grad - 1.0) / (s_max - r_sh) ** 2
    c_const = float(schw(s_in, 0.0)) - lkep2 * s_in ** (2.0 - 2.0 * q_grad) / (2.0 - 2.0 * q_grad)
    h_max = -float(schw(s_max, 0.0)) + lkep2 * s_max ** (2.0 - 2.0 * q_grad) / (2.0 - 2.0 * q_grad) + c_const
    k_poly = h_max * (ggas - 1.0) / ggas / rho_max ** (ggas - 1.0)
    if k_poly < 0.0:
        raise ValueError("the polytropic constant is negative")
    params = dict(r_sh=r_sh, s_in=s_in, s_max=s_max, q_grad=q_grad, rho_max=rho_max, rho_fac=rho_fac,
                  rho_cut=rho_cut, beta=beta, noise=noise, seed=seed)
    if not host_arrays:
        rho_floor = rho_fac * rho_max
        return Problem(f"torus_cyl_{nr}x{nph}x{nz}", nr, nph, nz, xf, yf, zf, N.CYLINDRICAL, (1, 1, 0, 0, 1, 1),
                       ggas, cfl, 0.0, None, None, model=N.MODEL_TORUS_CYN, rho_floor=rho_floor,
                       eps_floor=k_poly * rho_floor ** (ggas - 1.0) / (ggas - 1.0), r_sh=r_sh,
                       geom_source_repeat=geom_source_repeat, model_params=params)
    R = _centres(xf)[3:nr + 3][None, None, :]
    Z = _centres(zf)[3:nz + 3][:, None, None]
    h = -schw(R, Z) + lkep2 * R ** (2.0 - 2.0 * q_grad) / (2.0 - 2.0 * q_grad) + c_const
    h = np.maximum(h, 0.0)
    rho_loc = (h * (ggas - 1.0) / ggas / k_poly) ** (1.0 / (ggas - 1.0))
    rho_a = rho_fac * rho_max
    inside = (rho_loc > rho_a) & (R >= s_in)
    rho = np.where(inside, rho_loc, rho_a) * np.ones((1, nph, 1))
    vph = np.where(inside, np.sqrt(lkep2) * R ** (-q_grad) * R, 0.0) * np.ones((1, nph, 1))
    sl1 = (slice(3, nz + 3), slice(3, nph + 3), slice(3, nr + 3))
    v = prim[sl1]
    v[..., IRHO] = rho
    v[..., IVY] = vph
    v[..., ITAU] = k_poly * rho ** ggas
    eps[sl1] = k_poly * rho ** (ggas - 1.0) / (ggas - 1.0)
    A = np.zeros((nz + 6, nph + 6, nr + 6))
    A[sl1] = np.where(rho >= rho_cut, (rho - rho_cut) / rho_max, 0.0)
    Ac = np.zeros_like(A)
    Ac[sl1] = 0.25 * (A[3:nz + 3, 3:nph + 3, 3:nr + 3] + A[3:nz + 3, 3:nph + 3, 4:nr + 4]
                      + A[4:nz + 4, 3:nph + 3, 3:nr + 3] + A[4:nz + 4, 3:nph + 3, 4:nr + 4])
    # faces on 0:n (model.f90:149-158)
    f0 = (slice(2, nz + 3), slice(2, nph + 3), slice(2, nr + 3))
    a = Ac[f0]
    a_lm = Ac[1:nz + 2, 2:nph + 3, 2:nr + 3]    # (j, k, l-1)
    a_jm = Ac[2:nz + 3, 2:nph + 3, 1:nr + 2]    # (j-1, k, l)
    xfj = xf[3:nr + 4][None, None, :]           # faces j = 0..n
    xfjm = xf[2:nr + 3][None, None, :]
    xl = 0.5 * (xfj + xfjm)
    dxl = xfj - xfjm
    dzl = (zf[3:nz + 4] - zf[2:nz + 3])[:, None, None]
    prim[f0 + (IBX,)] = -(a - a_lm) / dzl
    prim[f0 + (IBZ,)] = (xfj * a - xfjm * a_jm) / (xl * dxl)
    # beta normalisation (model.f90:162-214)
    bcx = 0.5 * (prim[sl1 + (IBX,)] + prim[3:nz + 3, 3:nph + 3, 2:nr + 2, IBX])
    bcz = 0.5 * (prim[sl1 + (IBZ,)] + prim[3:nz + 3, 2:nph + 2, 3:nr + 3, IBZ])
    pgas_max = prim[sl1 + (ITAU,)].max()
    pmag_max = (0.5 * (bcx ** 2 + bcz ** 2)).max()
    norm = math.sqrt((pgas_max / pmag_max) / beta) if pmag_max > 0 else 0.0
    prim[f0 + (IBX,)] *= norm
    prim[f0 + (IBZ,)] *= norm
    rho_floor = rho_fac * rho_max
    eps_floor = k_poly * rho_floor ** (ggas - 1.0) / (ggas - 1.0)
    u = uniform01(seed, _linear_index(nr, nph, nz)[1:, 1:, 1:])
    d = prim[sl1 + (IRHO,)]
    prim[sl1 + (IRHO,)] = np.where(d > rho_floor, d + d * (u - 0.5) / 0.5 * noise, d)
    return Problem(f"torus_cyl_{nr}x{nph}x{nz}", nr, nph, nz, xf, yf, zf, N.CYLINDRICAL, (1, 1, 0, 0, 1, 1), ggas,
                   cfl, 0.0, prim, eps, model=N.MODEL_TORUS_CYN, rho_floor=rho_floor, eps_floor=eps_floor,
                   r_sh=r_sh, geom_source_repeat=geom_source_repeat, model_params=params)
