#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference is Fortran; it runs here through its mechanical C translation
(oracle/f2c_ref.py + oracle/ref_harness.c, built by `make -C oracle ref`,
which reads the reference sources where they lie). For each case below the
script builds the initial model with cumpic_b200.problems, runs the
reference's initial_update, SPATIAL (l_rk) and a few steps of finddt +
RUNGEKUTTA, and stores the dt sequence and the final prim, cons, eps, bcell
arrays (Fortran layout) in <case>.npz, with a hash of the initial arrays.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from cumpic_b200 import problems as P  # noqa: E402
from _oracle import Oracle, ref_lib_path  # noqa: E402


def cylinder_flow(nr=6, nphi=5, nz=4):
    """smooth magnetised flow on a cylindrical grid, R in [1, 2], with the
    torus_cyn hooks (floors, gravity, no-inflow ghosts)."""
    p = P.orszag_tang(nr, ny=nphi, nz=nz)
    p.name = f"cylinder_{nr}x{nphi}x{nz}"
    p.coordinate = 2
    p.xf = P.uniform_faces(1.0, 2.0, nr)
    p.yf = P.uniform_faces(0.0, 2.0 * np.pi, nphi)
    p.zf = P.uniform_faces(-0.5, 0.5, nz)
    p.boundary_flag = (1, 1, 0, 0, 1, 1)
    p.model = 3
    p.rho_floor = 1.0e-4
    p.eps_floor = 1.0e-4
    p.r_sh = 0.1
    return p


def cases():
    """(name, generator, kwargs, model of the reference build, steps)"""
    out = [
        ("brio_wu_x_24", "brio_wu", dict(nx=24, ny=3, nz=3, axis=0), "riemann", 8),
        ("brio_wu_y_20", "brio_wu", dict(nx=3, ny=20, nz=4, axis=1), "riemann", 6),
        ("orszag_tang_6x5x4", "orszag_tang", dict(n=6, ny=5, nz=4), "riemann", 4),
        ("orszag_tang_6_tvd", "orszag_tang", dict(n=6, recon=1), "riemann", 4),
        ("orszag_tang_6x5x4_b10", "orszag_tang", dict(n=6, ny=5, nz=4, bscale=10.0), "riemann", 3),
        ("torus_12x8x4", "torus", dict(nr=12, nth=8, nph=4), "torus_sph", 3),
        ("cylinder_6x5x4", "cylinder_flow", dict(nr=6, nphi=5, nz=4), "torus_cyn", 3),
    ]
    flagged = [((3, 1, 4, 2, 0, 0), "ot_flags_314200"), ((1, 2, 3, 4, 4, 2), "ot_flags_123442")]
    for flags, name in flagged:
        out.append((name, "orszag_tang", dict(n=6, ny=5, nz=4, boundary_flag=flags), "riemann", 3))
    return out


def make_problem(gen: str, kw: dict):
    kw = dict(kw)
    flags = kw.pop("boundary_flag", None)
    p = cylinder_flow(**kw) if gen == "cylinder_flow" else getattr(P, gen)(**kw)
    if flags is not None:
        p.boundary_flag = tuple(flags)
    return p


def input_hash(p) -> str:
    h = hashlib.sha256()
    for a in (p.prim, p.eps, p.xf, p.yf, p.zf):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    for name, gen, kw, model, steps in cases():
        p = make_problem(gen, kw)
        r = Oracle(p, lib_path=ref_lib_path(model))
        r.upload()
        r.initial_update()
        init = r.download()
        lrk = r.spatial()
        dts = []
        for _ in range(steps):
            dt = r.finddt()
            r.rungekutta(dt)
            dts.append(dt)
        fin = r.download()
        r.close()
        meta = {"generator": gen, "kwargs": kw, "model": model, "steps": steps, "input_sha256": input_hash(p),
                "source": "reference Fortran via oracle/f2c_ref.py"}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta), dts=np.array(dts),
                            init_prim=init["prim"], init_cons=init["cons"], init_eps=init["eps"],
                            init_bcell=init["bcell"], lrk=lrk,
                            prim=fin["prim"], cons=fin["cons"], eps=fin["eps"], bcell=fin["bcell"])
        print(f"{name}: {steps} steps, dt={dts[-1]:.6e}")


if __name__ == "__main__":
    main()
