"""The N>1 path of bench.py on CPU: world size 2 over gloo.

bench.py --gpus N runs N independent replicas (the path has no data-path
collective); the only cross-rank steps are the barrier and the max-over-ranks
reduction of the timed region. Here two gloo ranks each advance their own
replica with the CPU oracle, reduce their times through bench.make_reduce_max,
and must agree on the slowest time, on the whole-job rate and on the replicas'
final states. The reference arm's non-zero ranks exit without work.
"""
import os
import socket
import sys
import time

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path[:0] = [ROOT, HERE]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    import bench
    from cumpic_b200 import problems as P
    from _oracle import Oracle

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        prob = P.orszag_tang(12)
        o = Oracle(prob, threads=1)
        o.upload()
        o.initial_update()
        steps = 3
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            o.rungekutta(o.finddt())
        ms = 1e3 * (time.perf_counter() - t0) * (1.0 + rank)  # rank 1 reports the slower time
        dist.barrier()
        reduce_max = bench.make_reduce_max(world, "cpu")
        ms_max, rate = bench.replica_rate(world, prob.cells, steps, ms, reduce_max)
        cons = o.download()["cons"]
        chk = torch.tensor([float(np.sum(cons[3:-3, 3:-3, 3:-3, :5]))], dtype=torch.float64)
        allchk = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(allchk, chk)
        args = type("A", (), {"gpus": world, "steps": steps, "warmup": 1, "n": 8})()
        ref_rc = bench.run_reference(args, world, rank) if rank != 0 else 0
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.array([ms, ms_max, rate, prob.cells, steps] + [float(c) for c in allchk] + [ref_rc]))
    finally:
        dist.destroy_process_group()


def test_replicas_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    r = [np.load(tmp_path / f"r{k}.npy") for k in range(world)]
    ms = [x[0] for x in r]
    for x in r:
        assert x[1] == max(ms)                                        # max over ranks
        assert x[2] == pytest.approx(world * x[3] * x[4] / (max(ms) / 1e3) / 1e6)  # whole-job rate
        assert x[5] == x[6]                                           # replicas advance identically
        assert x[7] == 0                                              # reference arm: rank > 0 exits 0
    assert r[0][2] == r[1][2]
