"""Golden fixtures produced by the reference itself (its Fortran sources run
through the mechanical C translation of oracle/f2c_ref.py, generated by
tests/golden/make_golden.py). The FP64 oracle must reproduce them bit for bit
on the CPU; the CUDA path must reproduce them bit for bit on the GPU."""
import glob
import json
import os

import numpy as np
import pytest

from compare import diffs

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
IDS = [os.path.basename(f)[:-4] for f in FIXTURES]


def _load(path):
    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    return z, meta


def _problem(meta):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import input_hash, make_problem
    p = make_problem(meta["generator"], meta["kwargs"])
    assert input_hash(p) == meta["input_sha256"], "initial model generator changed since the fixture was made"
    return p


def _state(z, prefix=""):
    return {k: z[prefix + k] for k in ("prim", "cons", "eps", "bcell")}


def _check_run(sim, z, meta):
    sim.upload()
    sim.initial_update()
    d = diffs(sim.download(), _state(z, "init_"))
    assert max(d.values()) == 0.0, ("initial_update", d)
    lrk = sim.spatial()
    nz, ny, nx = (s - 6 for s in lrk.shape[:3])
    sl = (slice(2, nz + 3), slice(2, ny + 3), slice(2, nx + 3))
    assert np.array_equal(lrk[sl], z["lrk"][sl]), "SPATIAL l_rk"
    for i, dt_ref in enumerate(z["dts"]):
        dt = sim.finddt()
        assert dt == dt_ref, (i, dt, dt_ref)
        sim.rungekutta(dt)
    d = diffs(sim.download(), _state(z))
    assert max(d.values()) == 0.0, ("final state", d)


def test_fixtures_present():
    assert len(FIXTURES) >= 8


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_oracle_matches_reference_fixture(path):
    from _oracle import Oracle
    z, meta = _load(path)
    p = _problem(meta)
    _check_run(Oracle(p, threads=4), z, meta)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_cuda_matches_reference_fixture(path):
    from cumpic_b200.solver import CUMC3D
    z, meta = _load(path)
    p = _problem(meta)
    _check_run(CUMC3D(p), z, meta)
