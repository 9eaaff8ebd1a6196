"""The C program that drives the library through the C-ABI with the reference
main program's call sequence (cumpic_b200/driver/cumc_main.c).

It is compiled here as plain C99 with -Wall -Wextra -Werror -pedantic against
include/cumc.h and linked against libcumc_b200.so, so a prototype in the
header that drifts from the library, or a call that no longer matches one,
fails the build instead of passing silently as it could through ctypes. On a
GPU it runs the Brio-Wu configuration (512 x 4 x 4 to t_end = 0.1) with the
host loop (finddt, clip, rungekutta) and with the device loop
(cumc_advance), and its final state must equal the FP64 oracle's bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

from cumpic_b200 import problems as P
from compare import diffs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_driver_builds_warning_free():
    from cumpic_b200.build import build_driver
    exe = build_driver(force=True)
    assert os.access(exe, os.X_OK)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.skipif(_has_gpu(), reason="checks the failure path without a device")
def test_driver_without_device_fails_loudly(tmp_path):
    from cumpic_b200.build import build_driver
    r = subprocess.run([build_driver(), "16", "4", "4", "0.01", str(tmp_path / "out.bin")], capture_output=True,
                       text=True)
    assert r.returncode == 1
    assert "cumc_init" in r.stderr and "device" in r.stderr


def _read(path, nx, ny, nz):
    raw = np.fromfile(path, dtype=np.float64)
    head, body = raw[:8], raw[8:]
    shape = (nz + 6, ny + 6, nx + 6)
    nt = shape[0] * shape[1] * shape[2]
    assert body.size == 20 * nt
    out = {"prim": body[:8 * nt].reshape(shape + (8,)), "cons": body[8 * nt:16 * nt].reshape(shape + (8,)),
           "eps": body[16 * nt:17 * nt].reshape(shape), "bcell": body[17 * nt:].reshape(shape + (3,))}
    return head, out


@pytest.mark.gpu
@pytest.mark.parametrize("loop", ["host", "advance"])
def test_driver_brio_wu_matches_oracle(loop, tmp_path):
    from cumpic_b200.build import build_driver
    from _oracle import Oracle
    nx, ny, nz, t_end = 512, 4, 4, 0.1
    out = tmp_path / "state.bin"
    cmd = [build_driver(), str(nx), str(ny), str(nz), repr(t_end), str(out)] + (["advance"] if loop == "advance" else [])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    head, got = _read(out, nx, ny, nz)
    o = Oracle(P.brio_wu(nx, ny, nz), threads=os.cpu_count())
    o.upload()
    o.initial_update()
    steps = o.run(t_end)
    assert int(head[3]) == steps and head[4] == o.global_time == t_end
    d = diffs(got, o.download())
    assert all(v == 0.0 for v in d.values()), d
    assert head[6] <= 1.0e-12  # normalised max |div B|
