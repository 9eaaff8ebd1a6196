"""Comparison helpers shared by the parity tests.

Entries compared are the ones the reference itself defines after each step:
every ghosted cell of the hydro primitives, eps and bcell (BOUNDARY fills all
ghosts), the face fields at every position whose index along the field's own
axis lies in 0:n, and cons on (0:n)^3 except the face-field entries that the
reference overwrites through prim before they are read again (those keep an
unused value that differs by construction, see cumc_kernels.cuh k_boundary).
"""
from __future__ import annotations

import numpy as np


def face_mask(shape, axis: int) -> np.ndarray:
    """positions of the face field along `axis` (0=x) with index 0:n on that axis."""
    nz6, ny6, nx6 = shape
    m = np.zeros(shape, dtype=bool)
    n = (nx6 - 6, ny6 - 6, nz6 - 6)
    sl = [slice(None)] * 3
    sl[2 - axis] = slice(2, n[axis] + 3)
    m[tuple(sl)] = True
    return m


def cons_mask(shape, var: int) -> np.ndarray:
    nz6, ny6, nx6 = shape
    nx, ny, nz = nx6 - 6, ny6 - 6, nz6 - 6
    m = np.zeros(shape, dtype=bool)
    if var < 5:
        m[2:nz + 3, 2:ny + 3, 2:nx + 3] = True
    else:
        axis = var - 5
        lo = [3, 3, 3]          # 1:n on transverse axes
        lo[axis] = 2            # 0:n along the field's own axis
        m[lo[2]:nz + 3, lo[1]:ny + 3, lo[0]:nx + 3] = True
    return m


def maxdiff(x: np.ndarray, y: np.ndarray) -> float:
    """max |x-y|, NaN-aware: a NaN on both sides at the same position counts
    as equal (the reference leaves 0/0 in a few never-read ghost entries of
    the torus models), a NaN on one side only counts as +inf."""
    x = np.asarray(x)
    y = np.asarray(y)
    nx_, ny_ = np.isnan(x), np.isnan(y)
    d = np.abs(np.where(nx_ | ny_, 0.0, x - y))
    d = np.where(nx_ != ny_, np.inf, d)
    return float(np.max(d)) if d.size else 0.0


def diffs(a: dict, b: dict) -> dict:
    """max |a-b| per compared quantity (see maxdiff for NaN)."""
    shape = a["eps"].shape
    out = {}
    for q in range(5):
        out[f"prim{q}"] = maxdiff(a["prim"][..., q], b["prim"][..., q])
    for q in range(3):
        m = face_mask(shape, q)
        out[f"prim{5 + q}"] = maxdiff(a["prim"][..., 5 + q][m], b["prim"][..., 5 + q][m])
    for q in range(8):
        m = cons_mask(shape, q)
        out[f"cons{q}"] = maxdiff(a["cons"][..., q][m], b["cons"][..., q][m])
    out["eps"] = maxdiff(a["eps"], b["eps"])
    out["bcell"] = maxdiff(a["bcell"], b["bcell"])
    return out


def rel_l1_interior(a: dict, b: dict) -> dict:
    """relative L1 distance per conserved variable over the active cells."""
    shape = a["eps"].shape
    nz, ny, nx = (s - 6 for s in shape)
    out = {}
    for q in range(8):
        x = a["cons"][3:nz + 3, 3:ny + 3, 3:nx + 3, q]
        y = b["cons"][3:nz + 3, 3:ny + 3, 3:nx + 3, q]
        den = np.sum(np.abs(y))
        out[q] = float(np.sum(np.abs(x - y)) / den) if den > 0 else float(np.sum(np.abs(x - y)))
    return out
