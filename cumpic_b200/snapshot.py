"""Snapshot files: the reference's output datasets plus the state for an
exact restart.

The reference writes ``star_weno_data_<n>.hdf5`` (solver/dataio.f90:7-331,
print_hydroprofile) with the datasets ``prim`` (dims no_of_eq, nxtot, nytot,
nztot in Fortran order), ``eps`` and ``xf``, ``yf``, ``zf`` (the nxtot+1 face
coordinates), and has no restart. There is no HDF5 library here, so the
container is a flat little-endian file with the same datasets, plus those an
exact restart needs (``cons`` and ``bcell``; with ``prim`` and ``eps`` they
are the 17 arrays a step reads):

    header   "CUMCSNAP", u32 version, u32 ndatasets, i32 nx, ny, nz,
             coordinate, i64 step, f64 time, f64 ggas
    table    per dataset: 16-byte NUL-padded name, u32 dtype (1 = float64),
             u32 ndim, i64 dims[4], i64 byte offset
    data     each dataset in C order at its offset (64-byte aligned)

``prim`` is stored with dims (nz+6, ny+6, nx+6, 8): in C order that is the
reference's Fortran-order (8, nxtot, nytot, nztot) array byte for byte, so a
reader of the reference's layout takes it as is. Face coordinates run over
faces -3..n+3.
"""
from __future__ import annotations

import os
import struct

import numpy as np

MAGIC = b"CUMCSNAP"
VERSION = 1
_HEAD = struct.Struct("<8sII4iqdd")
_ENTRY = struct.Struct("<16sII4qq")
F64 = 1


def path_for(outdir: str, n: int) -> str:
    """the reference's file name for output number n, with this container's suffix"""
    return os.path.join(outdir, f"star_weno_data_{n}.cumcsnap")


def state_to_datasets(state: np.ndarray) -> dict:
    """the 17 state arrays (cons 1-8, prim 1-5, bcell 1-3, eps; each
    (nz+6, ny+6, nx+6)) -> prim, cons, bcell, eps in the reference's layouts"""
    cons = np.stack(state[0:8], axis=-1)
    prim = np.stack(list(state[8:13]) + list(state[5:8]), axis=-1)  # prim(ibx:ibz) is the face field
    bcell = np.stack(state[13:16], axis=-1)
    return {"prim": prim, "cons": cons, "bcell": bcell, "eps": np.array(state[16])}


def datasets_to_state(ds: dict) -> np.ndarray:
    prim, cons, bcell, eps = ds["prim"], ds["cons"], ds["bcell"], ds["eps"]
    state = np.empty((17,) + eps.shape)
    state[0:8] = np.moveaxis(cons, -1, 0)
    state[8:13] = np.moveaxis(prim[..., 0:5], -1, 0)
    state[13:16] = np.moveaxis(bcell, -1, 0)
    state[16] = eps
    return state


def write(path: str, problem, state: np.ndarray, time: float, step: int):
    """write a snapshot of `state` (17 arrays) of `problem`'s grid"""
    ds = {"xf": problem.xf, "yf": problem.yf, "zf": problem.zf}
    ds.update(state_to_datasets(state))
    names = ["xf", "yf", "zf", "prim", "eps", "cons", "bcell"]
    off = _HEAD.size + _ENTRY.size * len(names)
    table, blobs = [], []
    for name in names:
        a = np.ascontiguousarray(ds[name], dtype="<f8")
        off = (off + 63) // 64 * 64
        dims = list(a.shape) + [0] * (4 - a.ndim)
        table.append(_ENTRY.pack(name.encode(), F64, a.ndim, *dims, off))
        blobs.append((off, a))
        off += a.nbytes
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(_HEAD.pack(MAGIC, VERSION, len(names), problem.nx, problem.ny, problem.nz, problem.coordinate,
                           int(step), float(time), float(problem.ggas)))
        for e in table:
            f.write(e)
        for o, a in blobs:
            f.seek(o)
            a.tofile(f)
    os.replace(tmp, path)


def read(path: str) -> dict:
    """{"nx", "ny", "nz", "coordinate", "step", "time", "ggas", "datasets": {name: array}}"""
    with open(path, "rb") as f:
        raw = f.read()
    magic, version, nds, nx, ny, nz, coord, step, time, ggas = _HEAD.unpack_from(raw, 0)
    if magic != MAGIC or version != VERSION:
        raise ValueError(f"{path}: not a version-{VERSION} snapshot")
    ds = {}
    for i in range(nds):
        name, dtype, ndim, d0, d1, d2, d3, off = _ENTRY.unpack_from(raw, _HEAD.size + i * _ENTRY.size)
        if dtype != F64:
            raise ValueError(f"{path}: unknown dtype {dtype}")
        shape = (d0, d1, d2, d3)[:ndim]
        n = int(np.prod(shape))
        ds[name.rstrip(b"\0").decode()] = np.frombuffer(raw, dtype="<f8", count=n, offset=off).reshape(shape).copy()
    return {"nx": nx, "ny": ny, "nz": nz, "coordinate": coord, "step": step, "time": time, "ggas": ggas,
            "datasets": ds}
