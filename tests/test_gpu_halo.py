"""z-slab decomposition with the halo exchange (cumc_rk_stage_part,
cumc_halo_pack/unpack, CUMC_BC_EXCHANGE): a decomposed run equals the
single-domain run bit for bit (every array, ghosts included), for slabs in
one process and for two gloo ranks (processes sharing this GPU; the planes
pass through host memory, and no kernel waits on another process), and the
FP64 oracle bit for bit. Each stage's sweeps of the active planes are queued
before the previous stage's halo is unpacked."""
import dataclasses
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cumpic_b200 import _native as N
from cumpic_b200 import halo
from cumpic_b200 import problems as P

pytestmark = pytest.mark.gpu


def _walls():
    p = P.orszag_tang(12, ny=10, nz=14)
    return dataclasses.replace(p, boundary_flag=(0, 0, 1, 1, 2, 1))


CASES = [("ot_periodic_2", lambda: P.orszag_tang(16), 2), ("ot_periodic_3", lambda: P.orszag_tang(16), 3),
         ("walls_3", _walls, 3), ("shell_2", lambda: P.shell(N.CYLINDRICAL, 12, 10, 12), 2)]


def _single(prob, steps):
    from cumpic_b200.solver import CUMC3D
    s = CUMC3D(prob)
    s.upload()
    s.initial_update()
    for _ in range(steps):
        s.step()
    return s.download(), s.global_time


def _same(a, b):
    """equal everywhere the step defines: a face field outside 0:n along its
    own axis is neither filled nor read (it keeps what was uploaded there)"""
    for k in a:
        x, y = a[k].copy(), b[k].copy()
        if k in ("prim", "cons"):
            for d, axis in ((0, 2), (1, 1), (2, 0)):
                n = x.shape[axis] - 6
                dead = np.ones(x.shape[axis], bool)
                dead[2:n + 3] = False  # faces 0..n (array index l + 2)
                sl = [slice(None)] * 3
                sl[axis] = dead
                x[tuple(sl) + (5 + d,)] = 0.0
                y[tuple(sl) + (5 + d,)] = 0.0
        assert np.array_equal(x, y, equal_nan=True), (k, np.argwhere(x != y)[:5])


@pytest.mark.parametrize("name,make,nslabs", CASES, ids=[c[0] for c in CASES])
def test_slabs_in_one_process_match_single_domain(name, make, nslabs):
    ref, t = _single(make(), 4)
    run = halo.LocalSlabs(make(), nslabs)
    run.start()
    for _ in range(4):
        run.step()
    assert run.global_time == t
    _same(run.download(), ref)


def test_slabs_match_oracle():
    """the decomposed run against the FP64 oracle directly (not only against
    the single-domain CUDA run)"""
    from _oracle import Oracle
    from compare import diffs
    prob = P.orszag_tang(18, ny=14, nz=15)
    run = halo.LocalSlabs(prob, 3)
    run.start()
    o = Oracle(P.orszag_tang(18, ny=14, nz=15), threads=os.cpu_count())
    o.upload()
    o.initial_update()
    for _ in range(4):
        dt = run.step()
        assert o.step() == dt
    d = diffs(run.download(), o.download())
    assert all(v == 0.0 for v in d.values()), d


def test_stage_parts_in_order():
    from cumpic_b200.solver import CUMC3D
    s = CUMC3D(halo.ZSlabs(P.orszag_tang(12), 2).local(0))
    s.upload()
    s.initial_update()
    with pytest.raises(N.CumcError) as e:
        s.rk_stage_part(1, 1e-3, 2)  # part 2 without part 1
    assert e.value.code == N.CUMC_ERR_STATE
    s.rk_stage_part(1, 1e-3, 1)
    with pytest.raises(N.CumcError) as e:
        s.rk_stage_part(1, 1e-3, 1)  # part 2 is due
    assert e.value.code == N.CUMC_ERR_STATE
    with pytest.raises(N.CumcError) as e:
        s.rk_stage_part(1, 1e-3, 3)
    assert e.value.code == N.CUMC_ERR_ARG
    s.rk_stage_part(1, 1e-3, 2)
    s.rk_stage(2, 0.0)


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    run = halo.SlabRun(P.orszag_tang(16), rank, world)
    run.start()
    for _ in range(3):
        run.step()
    st = run.download()
    np.savez(os.path.join(out, f"r{rank}.npz"), t=run.global_time, **st)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_match_single_domain(tmp_path):
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    ref, t = _single(P.orszag_tang(16), 3)
    parts = [dict(np.load(tmp_path / f"r{r}.npz")) for r in range(2)]
    assert all(float(p.pop("t")) == t for p in parts)
    _same(halo.ZSlabs(P.orszag_tang(16), 2).gather(parts), ref)


def test_exchange_faces_refuse_the_fused_paths():
    from cumpic_b200.solver import CUMC3D
    s = CUMC3D(halo.ZSlabs(P.orszag_tang(12), 2).local(0))
    s.upload()
    s.initial_update()
    for call in (lambda: s.rungekutta(1e-3), lambda: s.advance(1), lambda: s.adjoint(1, 1)):
        with pytest.raises(N.CumcError) as e:
            call()
        assert e.value.code in (N.CUMC_ERR_STATE, N.CUMC_ERR_CONFIG)
    with pytest.raises(N.CumcError) as e:
        s.rk_stage(2, 1e-3)  # stage 1 is due
    assert e.value.code == N.CUMC_ERR_STATE
    bad = dataclasses.replace(halo.ZSlabs(P.orszag_tang(12), 2).local(0), precision=N.MIXED)
    with pytest.raises(N.CumcError) as e:
        CUMC3D(bad)
    assert e.value.code == N.CUMC_ERR_CONFIG
