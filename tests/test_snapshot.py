"""Snapshot container (cumpic_b200.snapshot), on the CPU: round trip, and the
reference's prim layout (Fortran order (no_of_eq, nxtot, nytot, nztot),
solver/dataio.f90:275-331) read straight from the file's bytes."""
import struct

import numpy as np

from cumpic_b200 import _native as N
from cumpic_b200 import problems as P
from cumpic_b200 import snapshot


def _state(prob, seed=3):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((N.STATE_ARRAYS, prob.nz + 6, prob.ny + 6, prob.nx + 6))


def test_round_trip(tmp_path):
    prob = P.orszag_tang(8, ny=6, nz=5)
    st = _state(prob)
    path = snapshot.path_for(str(tmp_path), 7)
    assert path.endswith("star_weno_data_7.cumcsnap")
    snapshot.write(path, prob, st, 0.125, 42)
    s = snapshot.read(path)
    assert (s["nx"], s["ny"], s["nz"], s["coordinate"], s["step"], s["time"]) == (8, 6, 5, N.CARTESIAN, 42, 0.125)
    assert np.array_equal(snapshot.datasets_to_state(s["datasets"]), st)
    for a in ("xf", "yf", "zf"):
        assert np.array_equal(s["datasets"][a], getattr(prob, a))
    # prim carries the face fields in its magnetic slots, as the reference's prim does
    assert np.array_equal(s["datasets"]["prim"][..., 5:8], s["datasets"]["cons"][..., 5:8])


def test_prim_bytes_are_the_reference_fortran_array(tmp_path):
    prob = P.orszag_tang(6, ny=5, nz=4)
    st = _state(prob, 9)
    path = str(tmp_path / "s.cumcsnap")
    snapshot.write(path, prob, st, 0.0, 0)
    raw = open(path, "rb").read()
    nds = struct.unpack_from("<I", raw, 12)[0]
    entries = [snapshot._ENTRY.unpack_from(raw, snapshot._HEAD.size + i * snapshot._ENTRY.size) for i in range(nds)]
    e = next(e for e in entries if e[0].rstrip(b"\0") == b"prim")
    nxt, nyt, nzt = prob.nx + 6, prob.ny + 6, prob.nz + 6
    fortran = np.frombuffer(raw, "<f8", count=8 * nxt * nyt * nzt, offset=e[-1]).reshape((8, nxt, nyt, nzt),
                                                                                        order="F")
    # prim(q, i, j, k): q = 1..5 the primitives, 6..8 the face fields
    for q, src in ((0, 8), (4, 12), (5, 5), (7, 7)):
        assert np.array_equal(fortran[q], st[src].transpose(2, 1, 0))
