"""Snapshots and exact restart (cumc_snapshot_async, cumc_snapshot_wait,
cumc_restore_state): a context restored from a snapshot file continues bit
for bit; a snapshot delivers the state it was taken at while the following
steps run; a second snapshot waits for the first one's copy out."""
import numpy as np
import pytest

from cumpic_b200 import problems as P
from cumpic_b200 import snapshot

pytestmark = pytest.mark.gpu

CASES = [("orszag_tang", lambda: P.orszag_tang(16)), ("torus", lambda: P.torus(24, 16, 8)),
         ("cylindrical_shell", lambda: P.shell(2, 12, 10, 8))]


def _start(prob, steps):
    from cumpic_b200.solver import CUMC3D
    s = CUMC3D(prob)
    s.upload()
    s.initial_update()
    for _ in range(steps):
        s.step()
    return s


def _same(a, b):
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=True), k


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_restart_from_file_is_exact(name, make, tmp_path):
    from cumpic_b200.solver import CUMC3D
    ref = _start(make(), 6).download()
    b = _start(make(), 3)
    path = snapshot.path_for(str(tmp_path), 1)
    b.save_snapshot(path)
    c = CUMC3D(make())
    c.load_snapshot(path)
    assert (c.n_step, c.global_time) == (b.n_step, b.global_time)
    for _ in range(3):
        c.step()
    _same(c.download(), ref)


def test_snapshots_overlap_the_following_steps():
    make = lambda: P.orszag_tang(24)  # noqa: E731
    at2, at3 = _start(make(), 2).download(), _start(make(), 3).download()
    at5 = _start(make(), 5).download()
    s = _start(make(), 2)
    b2, b3 = s.state_buffer(), s.state_buffer()
    s.snapshot_async(b2)
    s.step()
    s.snapshot_async(b3)  # reuses the staging slab after b2's copy out
    s.step()
    s.step()
    s.snapshot_wait()
    for buf, ref in ((b2, at2), (b3, at3)):
        ds = snapshot.state_to_datasets(buf)
        _same({k: ds[k] for k in ("prim", "cons", "eps", "bcell")}, ref)
    _same(s.download(), at5)
