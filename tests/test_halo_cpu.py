"""z-slab decomposition (cumpic_b200.halo) on the CPU: the slabs' grids,
flags and neighbours, the gather, and the exchange over gloo with two and
three ranks (planes tagged by rank and plane arrive in the right ghost
planes, a two-slab ring included). The kernels' side is covered by
tests/test_gpu_halo.py."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cumpic_b200 import _native as N
from cumpic_b200 import halo
from cumpic_b200 import problems as P


def test_slab_grids_flags_and_gather():
    p = P.orszag_tang(8, ny=6, nz=11)
    z = halo.ZSlabs(p, 3)
    assert z.counts == [4, 4, 3] and z.offsets == [0, 4, 8] and z.periodic
    assert [z.neighbours(r) for r in range(3)] == [(2, 1), (0, 2), (1, 0)]
    for r in range(3):
        q = z.local(r)
        assert q.nz == z.counts[r] and q.boundary_flag[4:] == (N.BC_EXCHANGE, N.BC_EXCHANGE)
        assert np.array_equal(q.zf, p.zf[z.offsets[r]:z.offsets[r] + q.nz + 7])
        assert np.array_equal(q.prim[3:3 + q.nz], p.prim[3 + z.offsets[r]:3 + z.offsets[r] + q.nz])
    got = z.gather([{"prim": z.local(r).prim} for r in range(3)])
    assert np.array_equal(got["prim"], p.prim)
    walls = P.orszag_tang(8, ny=6, nz=9)
    walls.boundary_flag = (0, 0, 0, 0, 1, 2)
    zw = halo.ZSlabs(walls, 3)
    assert [zw.neighbours(r) for r in range(3)] == [(None, 1), (0, 2), (1, None)]
    assert zw.local(0).boundary_flag[4:] == (1, N.BC_EXCHANGE)
    assert zw.local(2).boundary_flag[4:] == (N.BC_EXCHANGE, 2)
    assert halo.ZSlabs(p, 1).local(0).boundary_flag == p.boundary_flag
    with pytest.raises(ValueError):
        halo.ZSlabs(p, 4)  # 11 planes: a slab of 2


class _FakeSlab:
    """planes (nz+6) x 5 values; value = 100*rank + global plane index"""

    def __init__(self, rank, nz, offset):
        self.nz = nz
        self.a = np.full((nz + 6, 5), -1.0)
        for l in range(1, nz + 1):
            self.a[l + 2] = 100 * rank + offset + l


def _worker(rank, world, port, nzs, periodic, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    offs = [sum(nzs[:r]) for r in range(world)]
    s = _FakeSlab(rank, nzs[rank], offs[rank])
    halo._device_buffers = lambda sim, count: [torch.zeros(15, dtype=torch.float64) for _ in range(count)]
    halo._sync = lambda sim: None

    def pack(sim, side, buf):
        rows = sim.a[3:6] if side == 0 else sim.a[sim.nz:sim.nz + 3]
        buf.copy_(torch.from_numpy(rows.reshape(-1)))

    def unpack(sim, side, buf):
        v = buf.numpy().reshape(3, 5)
        if side == 0:
            sim.a[0:3] = v
        else:
            sim.a[sim.nz + 3:sim.nz + 6] = v
    halo._pack, halo._unpack = pack, unpack
    lo = (rank - 1) % world if (rank > 0 or periodic) else None
    hi = (rank + 1) % world if (rank < world - 1 or periodic) else None
    halo.HaloExchange(s, lo, hi).exchange()
    np.save(os.path.join(out, f"r{rank}.npy"), s.a)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("nzs,periodic", [([4, 3], True), ([3, 4, 5], True), ([3, 4, 5], False)])
def test_exchange_over_gloo(nzs, periodic, tmp_path):
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    world = len(nzs)
    mp.spawn(_worker, args=(world, port, nzs, periodic, str(tmp_path)), nprocs=world, join=True)
    offs = [sum(nzs[:r]) for r in range(world)]
    total = sum(nzs)
    for r in range(world):
        a = np.load(tmp_path / f"r{r}.npy")
        n = nzs[r]
        for g in range(3):  # ghost planes l = -2..0 and n+1..n+3
            lo_plane, hi_plane = offs[r] - 2 + g, offs[r] + n + 1 + g
            if r > 0 or periodic:
                src = (r - 1) % world
                want = 100 * src + ((lo_plane - 1) % total + 1)
                assert np.all(a[g] == want), (r, g, a[g])
            else:
                assert np.all(a[g] == -1.0)
            if r < world - 1 or periodic:
                src = (r + 1) % world
                want = 100 * src + ((hi_plane - 1) % total + 1)
                assert np.all(a[n + 3 + g] == want), (r, g, a[n + 3 + g])
            else:
                assert np.all(a[n + 3 + g] == -1.0)
