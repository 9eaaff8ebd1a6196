"""z-slab decomposition and the halo exchange between slabs.

Replaces the reference's MPI path for the hot loop (solver/mpi.f90:255-501,
MPI_BOUNDARYP_Z / MPI_BOUNDARY_Z; the internal faces of
solver/boundary.f90:332-336,663-667) with one process per GPU and
torch.distributed. The domain is cut into z-slabs. A slab's internal z faces
carry the boundary flag CUMC_BC_EXCHANGE, and after cumc_initial_update and
after each RK stage every slab sends the three active planes next to each
internal face (w, bcell, eps and the face fields Bx, By; cumc_halo_pack) to
the neighbour across it, which writes them into its ghost planes
(cumc_halo_unpack). A periodic z direction closes the slabs into a ring. dt
is the minimum of the slabs' CFL steps (one all-reduce per step, as the
reference's MPI_Allreduce MIN, solver/rungekutta.f90:258).

With NCCL the planes move between device buffers. With gloo (CPU
collectives) they pass through host memory. ``LocalSlabs`` runs all slabs
of a decomposition in one process, moving the planes by device copies.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _native as N
from .problems import Problem


@dataclasses.dataclass
class ZSlabs:
    """cut of a problem into `nslabs` z-slabs of near-equal depth (>= 3 planes each)"""
    problem: Problem
    nslabs: int

    def __post_init__(self):
        nz, n = self.problem.nz, self.nslabs
        base, extra = divmod(nz, n)
        self.counts = [base + (1 if r < extra else 0) for r in range(n)]
        if min(self.counts) < 3:
            raise ValueError(f"{nz} planes do not make {n} slabs of at least 3")
        self.offsets = [sum(self.counts[:r]) for r in range(n)]
        self.periodic = self.problem.boundary_flag[4] == 0 and self.problem.boundary_flag[5] == 0

    def neighbours(self, r: int) -> tuple[int | None, int | None]:
        """(z-in neighbour, z-out neighbour) of slab r, None at a physical face"""
        n = self.nslabs
        if n == 1:
            return None, None
        lo = r - 1 if r > 0 else (n - 1 if self.periodic else None)
        hi = r + 1 if r < n - 1 else (0 if self.periodic else None)
        return lo, hi

    def local(self, r: int) -> Problem:
        """slab r as a problem of its own: planes offset+1 .. offset+count of
        the global grid, with its three ghost planes on each side"""
        p, o, n = self.problem, self.offsets[r], self.counts[r]
        lo, hi = self.neighbours(r)
        flags = list(p.boundary_flag)
        if lo is not None:
            flags[4] = N.BC_EXCHANGE
        if hi is not None:
            flags[5] = N.BC_EXCHANGE
        return dataclasses.replace(p, name=f"{p.name}_slab{r}of{self.nslabs}", nz=n,
                                   zf=np.array(p.zf[o:o + n + 7]), prim=np.array(p.prim[o:o + n + 6]),
                                   eps=np.array(p.eps[o:o + n + 6]), boundary_flag=tuple(flags))

    def gather(self, states: list[dict]) -> dict:
        """global arrays from the slabs' downloads: each slab's active planes,
        the first slab's z-in ghost planes and the last slab's z-out ones"""
        out = {}
        for key in states[0]:
            parts = [states[0][key][:3]]
            for r, st in enumerate(states):
                parts.append(st[key][3:3 + self.counts[r]])
            parts.append(states[-1][key][3 + self.counts[-1]:])
            out[key] = np.concatenate(parts, axis=0)
        return out


def _pack(sim, side: int, buf):
    sim._check(sim._lib.cumc_halo_pack(sim._h, side, ctypes.c_void_p(buf.data_ptr())))


def _unpack(sim, side: int, buf):
    sim._check(sim._lib.cumc_halo_unpack(sim._h, side, ctypes.c_void_p(buf.data_ptr())))


def _device_buffers(sim, count: int):
    import torch
    n = ctypes.c_longlong()
    sim._check(sim._lib.cumc_halo_doubles(sim._h, ctypes.byref(n)))
    return [torch.empty(n.value, dtype=torch.float64, device="cuda") for _ in range(count)]


def _sync(sim):
    import torch
    torch.cuda.ExternalStream(sim.stream_handle()).synchronize()


class HaloExchange:
    """moves the halo planes of one slab context to and from its neighbours
    over torch.distributed (ranks = slab indices within `group`).

    start() packs the planes on the context's stream and starts the transfer;
    finish() makes the context's stream wait for it and unpacks. With NCCL
    nothing waits on the host: the sends and receives run on a stream of
    their own that waits (by a CUDA event) for the packs, and the context's
    stream waits for the receives by another event, so the work queued on
    the context's stream between start() and finish() (the next stage's
    sweeps of the active planes) overlaps the transfer. With gloo the planes
    pass through host memory and start() blocks until they have arrived."""

    def __init__(self, sim, lower: int | None, upper: int | None, group=None):
        import torch
        import torch.distributed as dist
        self.sim, self.lower, self.upper, self.group = sim, lower, upper, group
        self.dist = dist
        self.send = _device_buffers(sim, 2)
        self.recv = _device_buffers(sim, 2)
        self.host = not dist.is_initialized() or dist.get_backend(group) != "nccl"
        self.pending = False
        if self.host:
            self.send_h = [b.cpu() for b in self.send]
            self.recv_h = [b.cpu() for b in self.recv]
        else:
            self.stream = torch.cuda.ExternalStream(sim.stream_handle())
            self.comm = torch.cuda.Stream()
            self.packed = torch.cuda.Event()
            self.arrived = torch.cuda.Event()

    def _ops(self, send, recv):
        # per peer, every rank issues: send z-out, receive z-in, send z-in,
        # receive z-out; so the messages of a pair match in order even when
        # both neighbours are the same rank (two slabs in a ring)
        dist, ops = self.dist, []
        if self.upper is not None:
            ops.append(dist.P2POp(dist.isend, send[1], self.upper, self.group, tag=0))
        if self.lower is not None:
            ops.append(dist.P2POp(dist.irecv, recv[0], self.lower, self.group, tag=0))
        if self.lower is not None:
            ops.append(dist.P2POp(dist.isend, send[0], self.lower, self.group, tag=1))
        if self.upper is not None:
            ops.append(dist.P2POp(dist.irecv, recv[1], self.upper, self.group, tag=1))
        return ops

    def start(self):
        import torch
        sim, dist = self.sim, self.dist
        # side 1 (z-out) planes go to the z-out neighbour's side 0, side 0 to the z-in neighbour's side 1
        if self.upper is not None:
            _pack(sim, 1, self.send[1])
        if self.lower is not None:
            _pack(sim, 0, self.send[0])
        sides = [side for side, nb in ((0, self.lower), (1, self.upper)) if nb is not None]
        if not sides:  # a single slab: nothing to exchange
            self.pending = False
            return
        if self.host:
            _sync(sim)
            for side in sides:
                self.send_h[side].copy_(self.send[side])
            for req in dist.batch_isend_irecv(self._ops(self.send_h, self.recv_h)):
                req.wait()
            for side in sides:
                self.recv[side].copy_(self.recv_h[side])
            if self.recv[0].is_cuda:
                torch.cuda.current_stream().synchronize()
        else:
            self.packed.record(self.stream)
            self.comm.wait_event(self.packed)
            with torch.cuda.stream(self.comm):
                for req in dist.batch_isend_irecv(self._ops(self.send, self.recv)):
                    req.wait()  # the comm stream waits for the transfer; the host does not
            self.arrived.record(self.comm)
        self.pending = True

    def finish(self):
        if not self.pending:
            return
        if not self.host:
            self.stream.wait_event(self.arrived)
        if self.lower is not None:
            _unpack(self.sim, 0, self.recv[0])
        if self.upper is not None:
            _unpack(self.sim, 1, self.recv[1])
        self.pending = False

    def exchange(self):
        self.start()
        self.finish()


class SlabRun:
    """one rank's slab of a z-slab decomposition: the reference's time loop
    (solver/main.f90:127-163) with the halo exchange after initial_update
    and after each stage, and dt the minimum over ranks"""

    def __init__(self, problem: Problem, rank: int, world: int, group=None):
        from .solver import CUMC3D
        self.slabs = ZSlabs(problem, world)
        self.rank, self.group = rank, group
        self.sim = CUMC3D(self.slabs.local(rank))
        lo, hi = self.slabs.neighbours(rank)
        self.halo = HaloExchange(self.sim, lo, hi, group)
        self.global_time, self.n_step = 0.0, 0

    def start(self):
        self.sim.upload()
        self.sim.initial_update()
        self.halo.start()

    def step(self, total_time: float | None = None) -> float:
        """one main-loop iteration. Each stage's sweeps of the active planes
        (part 1) run while the previous stage's halo is in flight; the rest of
        the stage (part 2) follows its unpack. finddt reads active cells only,
        so it too runs beside the last stage's exchange."""
        import torch
        import torch.distributed as dist
        dt = self.sim.finddt()
        if dist.is_initialized() and dist.get_world_size(self.group) > 1:
            t = torch.tensor([dt], dtype=torch.float64,
                             device="cuda" if dist.get_backend(self.group) == "nccl" else "cpu")
            dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
            dt = float(t.item())
        if total_time is not None and self.global_time + dt > total_time:
            dt = total_time - self.global_time
        for s in (1, 2, 3):
            self.sim.rk_stage_part(s, dt, 1)
            self.halo.finish()
            self.sim.rk_stage_part(s, dt, 2)
            self.halo.start()
        self.global_time += dt
        self.n_step += 1
        return dt

    def download(self) -> dict:
        """this slab's state, after its ghost planes are filled"""
        self.halo.finish()
        return self.sim.download()


class LocalSlabs:
    """every slab of a decomposition in this process, on one device; the
    halo planes move by device copies. As in SlabRun, each stage's sweeps of
    the active planes are queued before the previous stage's halo is
    unpacked; the slabs' streams order the packs and unpacks among
    themselves by CUDA events, with no wait on the host."""

    def __init__(self, problem: Problem, nslabs: int):
        import torch
        from .solver import CUMC3D
        self.slabs = ZSlabs(problem, nslabs)
        self.sims = [CUMC3D(self.slabs.local(r)) for r in range(nslabs)]
        self.bufs = [_device_buffers(s, 2) for s in self.sims]
        self.streams = [torch.cuda.ExternalStream(s.stream_handle()) for s in self.sims]
        self.packed = [torch.cuda.Event() for _ in self.sims]
        self.unpacked = [torch.cuda.Event() for _ in self.sims]
        self.pending = False
        self.global_time, self.n_step = 0.0, 0

    def start_exchange(self):
        """pack every slab's planes, once its neighbours have unpacked the last ones"""
        for r, s in enumerate(self.sims):
            lo, hi = self.slabs.neighbours(r)
            for nb in {lo, hi} - {None}:
                self.streams[r].wait_event(self.unpacked[nb])
            if lo is not None:
                _pack(s, 0, self.bufs[r][0])
            if hi is not None:
                _pack(s, 1, self.bufs[r][1])
            self.packed[r].record(self.streams[r])
        self.pending = True

    def finish_exchange(self):
        """unpack every slab's ghost planes from its neighbours' packs"""
        if not self.pending:
            return
        for r, s in enumerate(self.sims):
            lo, hi = self.slabs.neighbours(r)
            for nb in {lo, hi} - {None}:
                self.streams[r].wait_event(self.packed[nb])
            if lo is not None:
                _unpack(s, 0, self.bufs[lo][1])
            if hi is not None:
                _unpack(s, 1, self.bufs[hi][0])
            self.unpacked[r].record(self.streams[r])
        self.pending = False

    def exchange(self):
        self.start_exchange()
        self.finish_exchange()

    def start(self):
        for s in self.sims:
            s.upload()
            s.initial_update()
        self.start_exchange()

    def step(self) -> float:
        dt = min(s.finddt() for s in self.sims)
        for st in (1, 2, 3):
            for s in self.sims:
                s.rk_stage_part(st, dt, 1)
            self.finish_exchange()
            for s in self.sims:
                s.rk_stage_part(st, dt, 2)
            self.start_exchange()
        self.global_time += dt
        self.n_step += 1
        return dt

    def download(self) -> dict:
        self.finish_exchange()
        for s in self.sims:
            _sync(s)
        return self.slabs.gather([s.download() for s in self.sims])
