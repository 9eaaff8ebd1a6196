#!/usr/bin/env python
"""Throughput of the CUMC3D per-step hot path on B200.

Workload: 3-D Orszag-Tang vortex, 256^3 cells, FP64, PPM + HLL + CT + SSP-RK3
at CFL 0.4 (the throughput configuration). One step = one full main-loop
iteration of solver/main.f90:127-143: finddt, then the three RK stages.
Metric: Mcell-upd/s = cells * steps / seconds / 1e6, whole job (all ranks).

  python bench.py [--gpus N --steps K --warmup W]      this library
  python bench.py --impl reference ...                  the FP64 CPU restatement
                                                        of the reference, all host
                                                        threads (rank 0 only)

N > 1 runs independent replicas, one per GPU (the hot path is one domain on
one GPU; there is no data-path collective); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-upd/s @256^3 (FP64, Orszag-Tang 3D, PPM/HLL/CT/RK3)"
UNIT = "Mcell-upd/s"
BYTES_PER_CELL_UPDATE = 512  # algorithmic HBM bytes of one cell through one RK3 step (FP64)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--decomp", choices=["replicas", "zslab"], default="replicas",
                    help="N > 1: independent replicas (weak scaling, the default) or one n^3 box cut into N z-slabs "
                         "with the halo exchange over NCCL (strong scaling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-fast", action="store_true", help="skip the CUMC_FP64_FAST section")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-snapshot", action="store_true")
    ap.add_argument("--no-adjoint-check", action="store_true",
                    help="skip the finite-difference check of the adjoint (128^3, 200 steps, 16 directions)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip Orszag-Tang 512^3 (FP64, mixed) and the torus over 2000 steps (FP64, mixed)")
    ap.add_argument("--all-configs", action="store_true",
                    help="compare the 512^3 mixed run with the FP64 run at t_end = 0.5 instead of t = 0.05")
    ap.add_argument("--no-ref-translation", action="store_true",
                    help="skip the second CPU figure (the reference's own loop structure)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_reduce_max(world: int, device):
    """max of a float over all ranks (a device tensor all-reduce; identity at world 1)."""
    def reduce_max(x: float) -> float:
        if world == 1:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return reduce_max


def replica_rate(world: int, cells_per_rank: int, steps: int, ms_local: float, reduce_max):
    """whole-job Mcell-upd/s of `world` replicas, each advancing its own box of
    cells_per_rank cells by `steps` steps: all ranks' cells over the slowest
    rank's time. Returns (ms of the slowest rank, rate)."""
    ms_max = reduce_max(ms_local)
    return ms_max, world * cells_per_rank * steps / (ms_max / 1e3) / 1e6


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dram_traffic_table():
    """per-launch DRAM bytes of each kernel at the bench workload, from the
    committed ncu summary (profiles/dram_traffic_orszag_tang_256.txt)."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_orszag_tang_256.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#"):
                try:
                    out[parts[0]] = float(parts[1])
                except ValueError:
                    pass
    return out


def algorithmic_bytes(kernel: str, nx: int, ny: int, nz: int) -> float:
    """compulsory HBM bytes of one launch (each value read or written once)."""
    n = (nx, ny, nz)
    if kernel.startswith("sweep_"):
        d = "xyz".index(kernel[-1])
        t = [n[a] + 2 for a in range(3) if a != d]
        faces = (n[d] + 1) * t[0] * t[1]
        cells = (n[d] + 6) * t[0] * t[1]
        return 8.0 * (7 * cells + faces + 7 * faces)
    box1 = (nx + 1) * (ny + 1) * (nz + 1)
    box2 = (nx + 2) * (ny + 2) * (nz + 2)
    if kernel == "emf":
        return 8.0 * (6 * box2 + 6 * box2 + 3 * box1)
    if kernel == "combine":  # hydro combine + conversions, stage 2/3 form: 15 hydro fluxes, u0 and uc
        # hydro, 3 face fields in; hydro cons, w, bcell, eps out
        return 8.0 * (15 + 5 + 5 + 3 + 5 + 5 + 3 + 1) * box1
    if kernel == "ct":  # 3 EMF, u0 and uc face fields in, face fields out (stage 2/3 form)
        return 8.0 * (3 + 3 + 3 + 3) * box1
    if kernel == "utop":
        return 8.0 * (8 + 2 + 5 + 5 + 1 + 3) * box1
    if kernel == "boundary":
        ghosts = (nx + 6) * (ny + 6) * (nz + 6) - nx * ny * nz
        return 8.0 * 2 * 12 * ghosts
    if kernel == "finddt":
        return 8.0 * 8 * nx * ny * nz
    return float("nan")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.6)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append({"sm": float(p[1]), "max": float(p[2]), "power": float(p[3]), "hw": p[5], "hwt": p[6],
                             "swt": p[7], "pcap": p[8]})
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        load = [r for r in rows if r["power"] > 250.0] or rows
        reasons = set()
        for r in load:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                              ("pcap", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in load), "sm_max_mhz": max(r["max"] for r in rows),
                "samples": len(load), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
WORKLOAD = "orszag_tang_3d n={n} fp64 ppm/hll/ct/rk3 cfl=0.4"


def cpu_port_rate(n: int, steps: int, warmup: int, threads: int | None = None):
    """FP64 CPU restatement (OpenMP, all host threads) on the full n^3
    Orszag-Tang box; returns (Mcell-upd/s, threads, seconds of the timed steps)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from cumpic_b200 import problems as P
    from _oracle import Oracle

    threads = threads or os.cpu_count() or 1
    p = P.orszag_tang(n)
    o = Oracle(p, threads=threads)
    used = o._L.orc_get_threads()
    o.upload()
    o.initial_update()
    for _ in range(warmup):
        o.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    el = time.perf_counter() - t0
    o.close()
    return p.cells * steps / el / 1e6, used, el


def _ref_worker(slab, steps, warmup, go, out):
    """one host rank of the translated reference: its own periodic
    Orszag-Tang slab, warm-up, then the timed steps once every rank is ready"""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from cumpic_b200 import problems as P
    from _oracle import Oracle, ref_lib_path

    nx, ny, nz = slab
    o = Oracle(P.orszag_tang(nx, ny=ny, nz=nz), lib_path=ref_lib_path("riemann"))
    o.upload()
    o.initial_update()
    for _ in range(warmup):
        o.step()
    out.put(("ready", 0.0))
    go.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    out.put(("done", time.perf_counter() - t0))


def ref_translation_available() -> bool:
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _oracle import ref_lib_path
    return os.path.exists(ref_lib_path("riemann"))


def cpu_ref_rate(steps: int, warmup: int, slab=(128, 128, 16), procs: int | None = None):
    """The reference's own loop structure on the host cores: the mechanical
    C translation of its Fortran (single-threaded, one configuration per
    process, as one MPI rank of the reference is), run as `procs` spawned
    processes that each advance their own slab, the way the reference's MPI
    ranks each advance a subdomain (without the halo exchange, which would
    only add time). Returns (Mcell-upd/s of all processes over the slowest
    one's time, processes, seconds)."""
    import multiprocessing as mp
    procs = procs or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    go = ctx.Event()
    out = ctx.Queue()
    ps = [ctx.Process(target=_ref_worker, args=(slab, steps, warmup, go, out)) for _ in range(procs)]
    for p in ps:
        p.start()

    def collect(kind):
        # one message of `kind` from every rank, giving up as soon as one has died
        import queue
        got = []
        while len(got) < procs:
            try:
                k, v = out.get(timeout=5)
            except queue.Empty:
                if any(p.exitcode not in (None, 0) for p in ps):
                    for p in ps:
                        if p.is_alive():
                            p.terminate()
                    raise RuntimeError(f"a reference rank exited before it was {kind}")
                continue
            assert k == kind, (k, kind)
            got.append(v)
        return got

    collect("ready")
    go.set()
    times = collect("done")
    for p in ps:
        p.join()
    el = max(times)
    cells = slab[0] * slab[1] * slab[2]
    return procs * cells * steps / el / 1e6, procs, el


def run_reference(args, world, rank):
    """The reference arm: the reference's CPU implementation of the hot path
    on all host cores (the mechanical translation of its own Fortran, one
    process per core; the FP64 restatement with OpenMP where the translation
    is absent), each step a bounded sample of the 256^3 workload."""
    if rank != 0:
        return 0
    n = args.n
    if ref_translation_available():
        slab = (128, 128, 16)
        rate, procs, el = cpu_ref_rate(args.steps, args.warmup, slab)
        base = {"value": rate, "unit": UNIT, "cores": procs, "kind": "reference",
                "sample": f"{procs} processes x one {slab[0]}x{slab[1]}x{slab[2]} periodic Orszag-Tang slab each "
                          f"({slab[0] * slab[1] * slab[2]} cells a process; a {n}^3 box split over {procs} MPI ranks "
                          f"gives each {n ** 3 // procs}), {args.steps} RK3 steps after {args.warmup} warm-up; "
                          f"mechanical C translation of the reference's Fortran (oracle/f2c_ref.py), "
                          f"single-threaded per process, gcc -O2"}
    else:
        rate, threads, el = cpu_port_rate(n, args.steps, args.warmup)
        base = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": f"Orszag-Tang {n}^3, {args.steps} RK3 steps after {args.warmup} warm-up "
                          f"(FP64 C++ restatement, OpenMP)"}
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD.format(n=n), "sample": base["sample"]},
        "cpu_baseline": base,
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def mixed_section(n: int, steps: int, warmup: int, fp64_ms_per_step: float) -> dict:
    """The mixed form (CUMC_MIXED) on the same workload: throughput, its ratio
    to the FP64 path, and its relative L1 error per conserved variable and
    normalised max |div B| against the FP64 path (bit-identical to the FP64
    oracle) at the configuration's t_end = 0.5, for B as given and B x 10
    (plasma beta ~0.05)."""
    import torch
    from cumpic_b200 import _native as NN
    from cumpic_b200 import problems as P
    from cumpic_b200.solver import CUMC3D
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from compare import rel_l1_interior

    prob = P.orszag_tang(n, precision=NN.MIXED)
    sim = CUMC3D(prob)
    sim.upload()
    sim.initial_update()
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    sim.advance(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.advance(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    sim.profile(True)  # per-kernel times of a few more steps (outside the timed region)
    sim.advance(min(steps, 10))
    prof = sim.profile_read()
    sim.profile(False)
    sim.close()
    tot = max(1e-9, sum(v[1] for v in prof.values()))
    out = {"value": prob.cells * steps / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms / steps,
           "speedup_vs_fp64": fp64_ms_per_step / (ms / steps), "accuracy_t": prob.t_end,
           "kernels_ms_per_launch": {k: round(v[1] / v[0], 4) for k, v in prof.items() if v[0]},
           "kernel_shares": {k: round(v[1] / tot, 4) for k, v in prof.items() if v[0]}, "vs_fp64": {}}
    names = ("rho", "mx", "my", "mz", "E", "bx", "by", "bz")
    for bscale in (1.0, 10.0):
        res = {}
        for prec in (NN.FP64, NN.MIXED):
            s = CUMC3D(P.orszag_tang(n, bscale=bscale, precision=prec))
            s.upload()
            s.initial_update()
            steps_run = s.run(prob.t_end)
            res[prec] = (s.download(), s.find_divb()[1], steps_run)
            s.close()
        rel = rel_l1_interior(res[NN.MIXED][0], res[NN.FP64][0])
        if bscale == 1.0:
            # the flow's own sensitivity: the FP64 run from a density perturbed by
            # a seeded 1e-12 relative noise, against the unperturbed FP64 run
            import numpy as np
            pp = P.orszag_tang(n, bscale=bscale)
            rho = pp.prim[..., 0]
            rho *= 1.0 + 1e-12 * (2.0 * np.random.default_rng(7).random(rho.shape) - 1.0)
            s = CUMC3D(pp)
            s.upload()
            s.initial_update()
            s.run(pp.t_end)
            relp = rel_l1_interior(s.download(), res[NN.FP64][0])
            s.close()
            out["fp64_perturbed_1e-12_rel_l1_at_t_end"] = {k: relp[q] for q, k in enumerate(names)}
            out["hll_fp32"] = mixed_fp32_form(n, steps, warmup, fp64_ms_per_step, res[NN.FP64][0], prob.t_end)
        out["vs_fp64"][f"bscale_{bscale:g}"] = {"rel_l1": {k: rel[q] for q, k in enumerate(names)},
                                                "max_divb_norm": res[NN.MIXED][1],
                                                "max_divb_norm_fp64": res[NN.FP64][1],
                                                "steps": {"fp64": res[NN.FP64][2], "mixed": res[NN.MIXED][2]}}
    return out


def mixed_fp32_form(n: int, steps: int, warmup: int, fp64_ms_per_step: float, fp64_state: dict,
                    t_end: float) -> dict:
    """The mixed form with its HLL solve all in FP32 (CUMC_MX_HLL=fp32, the
    reciprocal form): throughput and the density error at t_end against the
    FP64 run."""
    import torch
    from cumpic_b200 import _native as NN
    from cumpic_b200 import problems as P
    from cumpic_b200.solver import CUMC3D
    from compare import rel_l1_interior
    os.environ["CUMC_MX_HLL"] = "fp32"
    try:
        sim = CUMC3D(P.orszag_tang(n, precision=NN.MIXED))
        sim.upload()
        sim.initial_update()
        stream = torch.cuda.ExternalStream(sim.stream_handle())
        sim.advance(warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.advance(steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        sim.close()
        s = CUMC3D(P.orszag_tang(n, precision=NN.MIXED))
        s.upload()
        s.initial_update()
        s.run(t_end)
        rel = rel_l1_interior(s.download(), fp64_state)
        s.close()
    finally:
        os.environ.pop("CUMC_MX_HLL", None)
    return {"value": n ** 3 * steps / (ms / 1e3) / 1e6, "ms_per_step": ms / steps,
            "speedup_vs_fp64": fp64_ms_per_step / (ms / steps), "accuracy_t": t_end, "rel_l1_rho": rel[0],
            "what": "CUMC_MX_HLL=fp32: the HLL solve all in FP32 (reciprocal form) instead of its hydro components "
                    "combined in FP64"}


def fast_section(n: int, steps: int, warmup: int, fp64_ms_per_step: float) -> dict:
    """CUMC_FP64_FAST (the HLL solve's quotients as products with
    reciprocals) on the same workload: throughput, its ratio to the bitwise
    FP64 path, and its relative L1 per conserved variable and normalised
    max |div B| against the FP64 path (bit-identical to the FP64 oracle) at
    the configuration's t_end."""
    import torch
    from cumpic_b200 import _native as NN
    from cumpic_b200 import problems as P
    from cumpic_b200.solver import CUMC3D
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from compare import rel_l1_interior

    prob = P.orszag_tang(n, precision=NN.FP64_FAST)
    sim = CUMC3D(prob)
    sim.upload()
    sim.initial_update()
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    sim.advance(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.advance(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    sim.close()
    res = {}
    for prec in (NN.FP64, NN.FP64_FAST):
        s = CUMC3D(P.orszag_tang(n, precision=prec))
        s.upload()
        s.initial_update()
        nst = s.run(prob.t_end)
        res[prec] = (s.download(), s.find_divb()[1], nst)
        s.close()
    rel = rel_l1_interior(res[NN.FP64_FAST][0], res[NN.FP64][0])
    names = ("rho", "mx", "my", "mz", "E", "bx", "by", "bz")
    return {"value": prob.cells * steps / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms / steps,
            "speedup_vs_fp64": fp64_ms_per_step / (ms / steps), "accuracy_t": prob.t_end,
            "steps": {"fp64": res[NN.FP64][2], "fp64_fast": res[NN.FP64_FAST][2]},
            "rel_l1_vs_fp64": {k: rel[q] for q, k in enumerate(names)},
            "max_divb_norm": res[NN.FP64_FAST][1]}


def snapshot_section(n: int, steps: int = 20) -> dict:
    """cumc_snapshot_async on the workload: the steps alone, the same steps
    with a snapshot of the whole state (17 arrays) taken before them and
    copied out to pinned host memory while they run, and the copy out alone"""
    import torch
    from cumpic_b200 import problems as P
    from cumpic_b200.solver import CUMC3D
    sim = CUMC3D(P.orszag_tang(n))
    sim.upload()
    sim.initial_update()
    sim.advance(3)
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    buf = sim.state_buffer()
    sim.snapshot_async(buf)  # first call: staging slab and stream
    sim.snapshot_wait()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    sim.advance(steps)
    e1.record(stream)
    e1.synchronize()
    plain = e0.elapsed_time(e1)
    t0 = time.perf_counter()
    e0.record(stream)
    sim.snapshot_async(buf)
    sim.advance(steps)
    e1.record(stream)
    e1.synchronize()
    with_snap = e0.elapsed_time(e1)
    sim.snapshot_wait()
    wall = time.perf_counter() - t0
    t0 = time.perf_counter()
    sim.snapshot_async(buf)
    sim.snapshot_wait()
    alone = time.perf_counter() - t0
    pinned = False
    try:
        pinned = bool(torch.from_numpy(buf).is_pinned())
    except Exception:
        pass
    sim.close()
    return {"bytes": int(buf.nbytes), "pinned_host": pinned, "steps": steps, "ms_steps": plain,
            "ms_steps_with_snapshot": with_snap, "overhead_ms": with_snap - plain,
            "ms_wall_snapshot_and_steps": 1e3 * wall, "ms_copy_out_alone": 1e3 * alone,
            "what": "steps timed with CUDA events on the context stream; the copy out runs on its own stream"}


def adjoint_section(n: int = 128, steps: int = 200, ckpt: int = 20) -> dict:
    """Cost of the discrete adjoint on the adjoint check configuration
    (periodic box, rho = p = 1, uniform B, smooth velocity modes): the wall
    time of cumc_adjoint_run (checkpointed forward pass, recomputation,
    reverse sweep) over that of the same forward run with the same dt."""
    import torch
    from cumpic_b200 import _native as NN
    from cumpic_b200 import problems as P
    from cumpic_b200.solver import CUMC3D

    prob = P.fourier_box(n)
    sim = CUMC3D(prob)
    sim.upload()
    dts = sim.adjoint(steps, ckpt, NN.OBJ_MAGNETIC)["dts"]  # warm-up; records dt
    fw = CUMC3D(prob)
    fw.upload()
    fw.initial_update()
    for dt in dts[:5]:
        fw.rungekutta(dt)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fw.upload()
    fw.initial_update()
    for dt in dts:
        fw.rungekutta(dt)
    fw.find_divb()  # synchronises
    t_fwd = time.perf_counter() - t0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.upload()
    r = sim.adjoint(steps, ckpt, NN.OBJ_MAGNETIC, dts=dts)
    t_adj = time.perf_counter() - t0
    fw.close()
    sim.close()
    return {"workload": f"fourier_box n={n} steps={steps} checkpoint_every={ckpt} objective=magnetic_energy",
            "forward_s": t_fwd, "adjoint_s": t_adj, "cost_ratio": t_adj / t_fwd,
            "cost_ratio_beyond_forward": (t_adj - t_fwd) / t_fwd, "J": r["J"],
            "what": "adjoint_s: cumc_adjoint_run (initial_update, checkpointed forward pass, one recomputation "
                    "of every segment but the last, reverse sweep, gradient download); forward_s: upload, "
                    "initial_update and the same steps with the same dt"}


def config_runs(t512: float = 0.05) -> dict:
    """The remaining configurations: Orszag-Tang 512^3, FP64 and mixed
    (throughput over 10 device-loop steps after 2 warm-up, then the mixed
    run's relative L1 per variable and both runs' normalised max |div B|
    against the FP64 run at t = t512), and the spherical torus 192 x 128 x 64
    over 2000 steps in FP64 and in the mixed form (throughput, the mixed run's
    relative L1 against the FP64 run, both runs' normalised max |div B|)."""
    import torch
    from cumpic_b200 import _native as NN
    from cumpic_b200 import problems as P
    from cumpic_b200.solver import CUMC3D
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from compare import rel_l1_interior
    names = ("rho", "mx", "my", "mz", "E", "bx", "by", "bz")

    def timed(sim, fn):
        stream = torch.cuda.ExternalStream(sim.stream_handle())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    out = {}
    res = {}
    rate512 = {}
    for prec in (NN.FP64, NN.MIXED):
        prob = P.orszag_tang(512, precision=prec)
        s = CUMC3D(prob)
        s.upload()
        s.initial_update()
        s.advance(2)
        ms = timed(s, lambda: s.advance(10))
        rate512[prec] = prob.cells * 10 / (ms / 1e3) / 1e6
        s.upload()
        s.initial_update()
        s.global_time, s.n_step = 0.0, 0
        s.run(t512)
        res[prec] = (s.download(), s.find_divb()[1], s.n_step)
        s.close()
        del s
    rel = rel_l1_interior(res[NN.MIXED][0], res[NN.FP64][0])
    out[f"orszag_tang_512"] = {
        "fp64_mcell_upd_s": rate512[NN.FP64], "mixed_mcell_upd_s": rate512[NN.MIXED],
        "mixed_speedup": rate512[NN.MIXED] / rate512[NN.FP64], "accuracy_t": t512,
        "steps_to_accuracy_t": {"fp64": res[NN.FP64][2], "mixed": res[NN.MIXED][2]},
        "mixed_rel_l1_vs_fp64": {k: rel[q] for q, k in enumerate(names)},
        "max_divb_norm": {"fp64": res[NN.FP64][1], "mixed": res[NN.MIXED][1]}}
    del res
    # torus: throughput with the device-side dt, then the accuracy runs with
    # the FP64 run's dt sequence replayed by the mixed run (same times)
    rate = {}
    for prec in (NN.FP64, NN.MIXED):
        prob = P.torus()
        prob.precision = prec
        s = CUMC3D(prob)
        s.upload()
        s.initial_update()
        ms = timed(s, lambda: s.advance(2000))
        rate[prec] = prob.cells * 2000 / (ms / 1e3) / 1e6
        s.close()
    res = {}
    dts = []
    for prec in (NN.FP64, NN.MIXED):
        prob = P.torus()
        prob.precision = prec
        s = CUMC3D(prob)
        s.upload()
        s.initial_update()
        for n in range(2000):
            if prec == NN.FP64:
                dts.append(s.finddt())
            s.rungekutta(dts[n])
        res[prec] = (s.download(), s.find_divb()[1])
        s.close()
    rel = rel_l1_interior(res[NN.MIXED][0], res[NN.FP64][0])
    out["torus_192x128x64_2000_steps"] = {
        "fp64_mcell_upd_s": rate[NN.FP64], "mixed_mcell_upd_s": rate[NN.MIXED], "t_end": float(sum(dts)),
        "mixed_rel_l1_vs_fp64": {k: rel[q] for q, k in enumerate(names)},
        "max_divb_norm": {"fp64": res[NN.FP64][1], "mixed": res[NN.MIXED][1]},
        "accuracy_runs": "both with the FP64 run's 2000 dt values"}
    return out


def adjoint_check(n: int = 128, steps: int = 200, ckpt: int = 20, ndir: int = 8,
                  eps_list=(1e-6, 1e-7, 1e-8)) -> dict:
    """The adjoint check configuration in full: gradient of the final magnetic
    energy with respect to the initial velocity against central differences
    along `ndir` seeded smooth random directions, at several difference steps
    (relative to the flow), with the adjoint's dt sequence replayed."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from cumpic_b200 import _native as NN
    from cumpic_b200 import problems as P
    from cumpic_b200.solver import CUMC3D
    from test_gpu_adjoint import _density, smooth_velocity_directions

    prob = P.fourier_box(n)
    sim = CUMC3D(prob)
    sim.upload()
    res = sim.adjoint(steps, ckpt, NN.OBJ_MAGNETIC)
    fw = CUMC3D(prob)

    def run(prim):
        fw.upload(prim, prob.eps)
        fw.initial_update()
        for dt in res["dts"]:
            fw.rungekutta(dt)
        return _density(fw.download(), prob, NN.OBJ_MAGNETIC)

    out = {"workload": f"fourier_box n={n} steps={steps} checkpoint_every={ckpt}", "directions": ndir, "by_eps": {}}
    dirs = list(smooth_velocity_directions(prob, ndir, 4))
    for eps in eps_list:
        rels = []
        for dp, _ in dirs:
            fd = float(np.sum(run(prob.prim + eps * dp) - run(prob.prim - eps * dp))) / (2 * eps)
            ad = float(np.sum(res["grad_prim"] * dp))
            rels.append(abs(fd - ad) / max(abs(fd), abs(ad)))
        out["by_eps"][f"{eps:g}"] = {"max_rel_err": max(rels), "median_rel_err": statistics.median(rels),
                                     "rel_errs": rels}
    best = min(out["by_eps"].values(), key=lambda r: r["median_rel_err"])
    out["median_rel_err_best_eps"] = best["median_rel_err"]
    out["max_rel_err_best_eps"] = best["max_rel_err"]
    return out


# ---------------------------------------------------------------------------
def run_zslab(args, world, rank, local):
    """One n^3 Orszag-Tang box cut into `world` z-slabs, one per GPU, with the
    halo exchange over NCCL after every stage (overlapped with the next
    stage's sweeps of the active planes) and dt the minimum over ranks: K main-
    loop steps of the whole box, timed on the device, max over ranks
    (strong scaling)."""
    import torch
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    from cumpic_b200 import halo
    from cumpic_b200 import problems as P

    n = args.n
    prob = P.orszag_tang(n)
    run = halo.SlabRun(prob, rank, world)
    run.start()
    for _ in range(args.warmup):
        run.step()
    stream = torch.cuda.ExternalStream(run.sim.stream_handle())

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    l0 = run.sim.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        run.step()
    run.halo.finish()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = run.sim.launch_count() - l0
    barrier()
    clk = clocks.stop()
    ms_max = make_reduce_max(world, "cuda")(ms)
    value = prob.cells * args.steps / (ms_max / 1e3) / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD.format(n=n), "cells": prob.cells, "parallelism": f"zslab x{world}",
                   "slab_planes": run.slabs.counts,
                   "l2": "inputs larger than L2 (each of the 8 state arrays is %.2f GB)" % (8 * (n + 6) ** 3 / 1e9)},
        "gpu_launches": launches, "clocks": clk,
        "halo": {"bytes_per_face_per_stage": int(11 * 3 * (n + 6) ** 2 * 8),
                 "transport": "NCCL send/recv on a stream of its own, ordered by CUDA events" if world > 1
                 else "none (one slab)"},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_ours(args, world, rank, local):
    import torch
    import numpy as np

    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    from cumpic_b200 import problems as P
    from cumpic_b200.solver import CUMC3D

    n = args.n
    prob = P.orszag_tang(n)
    cells = prob.cells
    sim = CUMC3D(prob)
    sim.upload()
    sim.initial_update()
    stream = torch.cuda.ExternalStream(sim.stream_handle())
    sim.advance(args.warmup)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    max_over_ranks = make_reduce_max(world, "cuda")

    # ---- timed region: K main-loop steps, inputs resident in HBM ----------
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    sim.profile(True)
    l0 = sim.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.advance(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = sim.launch_count() - l0
    prof = sim.profile_read()
    sim.profile(False)
    barrier()
    clk = clocks.stop()
    ms_max, value = replica_rate(world, cells, args.steps, ms, max_over_ranks)

    # ---- roofline of the dominant kernel ------------------------------------
    hbm, hbm_kind = peaks()
    dom = max(prof, key=lambda k: prof[k][1])
    dom_n, dom_ms = prof[dom]
    per_launch_s = dom_ms / dom_n / 1e3
    alg = algorithmic_bytes(dom, prob.nx, prob.ny, prob.nz)
    achieved = alg / per_launch_s / 1e9
    traffic = dram_traffic_table().get(dom)
    kernels = {k: {"launches": v[0], "ms": round(v[1], 3), "share": round(v[1] / max(1e-9, sum(x[1] for x in prof.values())), 4)}
               for k, v in prof.items()}
    step_s = ms_max / 1e3 / args.steps
    step_achieved = BYTES_PER_CELL_UPDATE * cells / step_s / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD.format(n=n),
                   "cells_per_gpu": cells, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (each of the 8 state arrays is %.2f GB)" % (8 * (n + 6) ** 3 / 1e9)},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "peak_kind": hbm_kind,
                     "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg, "launch_ms": per_launch_s * 1e3,
                     "step": {"bytes_per_cell_update": BYTES_PER_CELL_UPDATE, "achieved": step_achieved,
                              "frac": step_achieved / hbm}},
        "kernels": kernels,
        "clocks": clk,
    }

    # ---- end to end through the C-ABI with host buffers ----------------------
    if not args.no_e2e:
        nz6, ny6, nx6 = prob.nz + 6, prob.ny + 6, prob.nx + 6
        hp = torch.empty((nz6, ny6, nx6, 8), dtype=torch.float64, pin_memory=True).numpy()
        he = torch.empty((nz6, ny6, nx6), dtype=torch.float64, pin_memory=True).numpy()
        hp[...] = prob.prim
        he[...] = prob.eps
        out = {k: torch.empty(s, dtype=torch.float64, pin_memory=True).numpy() for k, s in
               (("prim", (nz6, ny6, nx6, 8)), ("cons", (nz6, ny6, nx6, 8)), ("eps", (nz6, ny6, nx6)),
                ("bcell", (nz6, ny6, nx6, 3)))}
        sim2 = CUMC3D(prob)
        s2 = torch.cuda.ExternalStream(sim2.stream_handle())
        sim2.upload(hp, he)
        sim2.initial_update()
        sim2.step()  # warm-up of the host loop path
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        f0.record(s2)
        sim2.upload(hp, he)
        sim2.initial_update()
        for _ in range(args.steps):
            sim2.step()  # finddt -> dt to host -> clip -> rungekutta(dt)
        from cumpic_b200.solver import _dp
        lib = sim2._lib
        sim2._check(lib.cumc_download_state(sim2._h, _dp(out["prim"]), _dp(out["cons"]), _dp(out["eps"]),
                                            _dp(out["bcell"])))
        f1.record(s2)
        f1.synchronize()
        wall = time.perf_counter() - t0
        e_ms = max_over_ranks(max(f0.elapsed_time(f1), 1e3 * wall))
        state_in = hp.nbytes + he.nbytes
        state_out = sum(a.nbytes for a in out.values())
        line["e2e"] = {"value": world * cells * args.steps / (e_ms / 1e3) / 1e6, "unit": UNIT,
                       "h2d_bytes_per_step": int(state_in / args.steps + 8),
                       "d2h_bytes_per_step": int(state_out / args.steps + 8 + 4),
                       "what": "upload initial prim+eps (AoS, pinned) + initial_update + K x (cumc_finddt "
                               "-> dt to host -> clip -> cumc_rungekutta) + download prim/cons/eps/bcell"}
        sim2.close()

    # ---- CPU baseline: the restatement on the host cores (rank 0, N=1) -------
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, threads, el = cpu_port_rate(n, 10, 2)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"Orszag-Tang {n}^3 (the whole workload), 10 RK3 steps after 2 warm-up "
                                          f"({el:.1f} s; FP64 C++ restatement, OpenMP)"}
        if not args.no_ref_translation and ref_translation_available():
            slab = (128, 128, 16)
            rrate, procs, rel_s = cpu_ref_rate(3, 1, slab)
            line["cpu_baseline"]["reference_translation"] = {
                "value": rrate, "unit": UNIT, "cores": procs, "kind": "reference",
                "sample": f"{procs} processes x one {slab[0]}x{slab[1]}x{slab[2]} periodic Orszag-Tang slab each, "
                          f"3 RK3 steps after 1 warm-up ({rel_s:.1f} s); mechanical C translation of the "
                          f"reference's Fortran, single-threaded per process"}
    sim.close()
    if world == 1 and not args.no_mixed:
        line["mixed"] = mixed_section(n, args.steps, args.warmup, ms_max / args.steps)
    if world == 1 and not args.no_fast:
        line["fp64_fast"] = fast_section(n, args.steps, args.warmup, ms_max / args.steps)
    if world == 1 and not args.no_snapshot:
        line["snapshot"] = snapshot_section(n)
    if world == 1 and not args.no_adjoint:
        line["adjoint"] = adjoint_section()
        if not args.no_adjoint_check:
            line["adjoint"]["fd_check"] = adjoint_check()
    if world == 1 and not args.no_configs:
        line["configs"] = config_runs(0.5 if args.all_configs else 0.05)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    world, rank, local = dist_init()
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.decomp == "zslab":
        return run_zslab(args, world, rank, local)
    return run_ours(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
