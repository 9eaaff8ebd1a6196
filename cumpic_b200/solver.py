"""Host-side mirror of the reference driver's calls into the hot path.

``CUMC3D`` exposes the argument-free Fortran subroutines that
solver/main.f90 calls (``initial_update``, ``finddt``, ``rungekutta``,
``find_divb``; SPATIAL for unit checks) as methods on one device context,
with the same order rules, and the main time loop of solver/main.f90:127-163
as :meth:`run`. Every method goes through the C-ABI of include/cumc.h.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .problems import Problem


def _dp(a: np.ndarray):
    return a.ctypes.data_as(N.POINTER(N.c_double))


class CUMC3D:
    def __init__(self, problem: Problem):
        self.problem = problem
        self._lib = N.lib()
        self._cfg = problem.config()
        h = ctypes.c_void_p()
        rc = self._lib.cumc_init(ctypes.byref(self._cfg), ctypes.byref(h))
        if rc != N.CUMC_OK:
            raise N.CumcError(rc, self._lib.cumc_last_error(None).decode())
        self._h = h
        self.global_time = 0.0
        self.n_step = 0

    # -- plumbing -----------------------------------------------------------
    def _check(self, rc: int):
        if rc != N.CUMC_OK:
            raise N.CumcError(rc, self._lib.cumc_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cumc_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def shape(self):
        p = self.problem
        return (p.nz + 6, p.ny + 6, p.nx + 6)

    # -- reference subroutines ---------------------------------------------
    def upload(self, prim: np.ndarray | None = None, eps: np.ndarray | None = None):
        """POPULATE_DEVICE (solver/openacc.f90:28-59) of the initial model."""
        prim = np.ascontiguousarray(self.problem.prim if prim is None else prim, dtype=np.float64)
        eps = np.ascontiguousarray(self.problem.eps if eps is None else eps, dtype=np.float64)
        self._check(self._lib.cumc_upload_state(self._h, _dp(prim), _dp(eps)))

    def generate_model(self):
        """the initial state built on the device (cumc_model_torus) from the
        problem's model_params, in place of upload"""
        mp = self.problem.model_params
        if not mp:
            raise ValueError("the problem has no device-side generator parameters")
        m = N.CumcTorusModel(**mp)
        self._check(self._lib.cumc_model_torus(self._h, ctypes.byref(m)))

    def initial_update(self):
        """initial_update (solver/initial.f90:83-140)."""
        self._check(self._lib.cumc_initial_update(self._h))

    def finddt(self) -> float:
        """finddt (solver/rungekutta.f90:161-265)."""
        dt = ctypes.c_double()
        self._check(self._lib.cumc_finddt(self._h, ctypes.byref(dt)))
        return dt.value

    def rungekutta(self, dt: float):
        """RUNGEKUTTA (solver/rungekutta.f90:12-148)."""
        self._check(self._lib.cumc_rungekutta(self._h, float(dt)))

    def spatial(self) -> np.ndarray:
        """SPATIAL (solver/spatial.f90:11-68); returns l_rk in the Fortran layout."""
        self._check(self._lib.cumc_spatial(self._h))
        out = np.zeros(self.shape + (8,))
        self._check(self._lib.cumc_download_lrk(self._h, _dp(out)))
        return out

    def find_divb(self):
        """find_divb (solver/mhd.f90:15-66): (signed max, normalised max |div B|)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.cumc_divb(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def download(self) -> dict:
        """UPDATE HOST (solver/dataio.f90:24): prim, cons, eps, bcell."""
        prim = np.zeros(self.shape + (8,))
        cons = np.zeros(self.shape + (8,))
        eps = np.zeros(self.shape)
        bcell = np.zeros(self.shape + (3,))
        self._check(self._lib.cumc_download_state(self._h, _dp(prim), _dp(cons), _dp(eps), _dp(bcell)))
        return {"prim": prim, "cons": cons, "eps": eps, "bcell": bcell}

    # -- drivers -------------------------------------------------------------
    def step(self, total_time: float | None = None) -> float:
        """One pass of the main loop body (solver/main.f90:130-142) with host dt."""
        dt = self.finddt()
        if total_time is not None and self.global_time + dt > total_time:
            dt = total_time - self.global_time
        self.rungekutta(dt)
        self.n_step += 1
        self.global_time += dt
        return dt

    def run(self, total_time: float, max_steps: int = 10 ** 9) -> int:
        """The main loop (solver/main.f90:127) with dt kept on the device."""
        t = ctypes.c_double(self.global_time)
        steps = ctypes.c_int(0)
        self._check(self._lib.cumc_advance(self._h, int(max_steps), float(total_time), ctypes.byref(t),
                                           ctypes.byref(steps)))
        self.global_time = t.value
        self.n_step += steps.value
        return steps.value

    def advance(self, nsteps: int, total_time: float = 1.0e300) -> int:
        """`nsteps` iterations of the main loop on the device (no host sync between)."""
        return self.run(total_time, nsteps)

    # -- discrete adjoint ------------------------------------------------------
    def adjoint(self, nsteps: int, checkpoint_every: int = 20, objective: int = N.OBJ_MAGNETIC,
                weights: np.ndarray | None = None, dts: np.ndarray | None = None) -> dict:
        """cumc_adjoint_run: from the uploaded state, initial_update and
        `nsteps` steps (dt from `dts` when given, else finddt), then the
        objective J on the final state and its gradient with respect to the
        uploaded prim (rho, v, face B; the pressure slot is 0) and eps.
        Returns {"J", "grad_prim", "grad_eps", "dts"}; the context then holds
        the final state."""
        gp = np.zeros(self.shape + (8,))
        ge = np.zeros(self.shape)
        dt_out = np.zeros(nsteps)
        J = ctypes.c_double()
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        d_in = None if dts is None else np.ascontiguousarray(dts, dtype=np.float64)
        self._check(self._lib.cumc_adjoint_run(self._h, int(nsteps), int(checkpoint_every), int(objective),
                                               None if w is None else _dp(w), None if d_in is None else _dp(d_in),
                                               _dp(dt_out), ctypes.byref(J), _dp(gp), _dp(ge)))
        self.n_step = nsteps
        self.global_time = float(np.sum(dt_out))
        return {"J": J.value, "grad_prim": gp, "grad_eps": ge, "dts": dt_out}

    def rk_stage(self, stage: int, dt: float):
        """cumc_rk_stage: one stage of RUNGEKUTTA (1, 2, 3 in order; dt read
        at stage 1), for slabs that exchange halos between stages"""
        self._check(self._lib.cumc_rk_stage(self._h, int(stage), float(dt)))

    def rk_stage_part(self, stage: int, dt: float, part: int):
        """cumc_rk_stage_part: part 1 (the sweeps that read no ghost plane) or
        part 2 (the rest) of one stage, so a halo exchange can run between"""
        self._check(self._lib.cumc_rk_stage_part(self._h, int(stage), float(dt), int(part)))

    # -- snapshots and restart -------------------------------------------------
    def state_buffer(self) -> np.ndarray:
        """a host buffer for one state (STATE_ARRAYS x shape doubles), pinned
        when torch can provide pinned memory, so that the copy out overlaps"""
        shape = (N.STATE_ARRAYS,) + self.shape
        try:
            import torch
            return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
        except Exception:
            return np.empty(shape)

    def snapshot_async(self, host_state: np.ndarray):
        """cumc_snapshot_async: the current state is copied out to host_state
        while the following steps run; host_state stays untouched until
        snapshot_wait returns"""
        if host_state.shape != (N.STATE_ARRAYS,) + self.shape or host_state.dtype != np.float64 or \
                not host_state.flags.c_contiguous:
            raise ValueError("host_state must be a C-contiguous float64 array of shape (17,) + shape")
        self._snap = host_state
        self._snap_meta = (self.global_time, self.n_step)
        self._check(self._lib.cumc_snapshot_async(self._h, _dp(host_state)))

    def snapshot_wait(self) -> tuple[float, int]:
        """cumc_snapshot_wait; returns the (time, step) the snapshot was taken at"""
        self._check(self._lib.cumc_snapshot_wait(self._h))
        return getattr(self, "_snap_meta", (self.global_time, self.n_step))

    def restore_state(self, host_state: np.ndarray, global_time: float = 0.0, n_step: int = 0):
        """cumc_restore_state: continue from a state taken by snapshot_async"""
        st = np.ascontiguousarray(host_state, dtype=np.float64)
        if st.shape != (N.STATE_ARRAYS,) + self.shape:
            raise ValueError("the state does not match this grid")
        self._check(self._lib.cumc_restore_state(self._h, _dp(st)))
        self.global_time, self.n_step = float(global_time), int(n_step)

    def save_snapshot(self, path: str):
        """the state now, with time and step, to a snapshot file"""
        from . import snapshot
        buf = self.state_buffer()
        self.snapshot_async(buf)
        t, n = self.snapshot_wait()
        snapshot.write(path, self.problem, buf, t, n)

    def load_snapshot(self, path: str):
        """continue from a snapshot file of this grid"""
        from . import snapshot
        s = snapshot.read(path)
        p = self.problem
        if (s["nx"], s["ny"], s["nz"], s["coordinate"]) != (p.nx, p.ny, p.nz, p.coordinate):
            raise ValueError(f"{path}: the snapshot's grid differs from this context's")
        self.restore_state(snapshot.datasets_to_state(s["datasets"]), s["time"], s["step"])

    # -- instrumentation -----------------------------------------------------
    def stream_handle(self) -> int:
        s = ctypes.c_void_p()
        self._check(self._lib.cumc_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def profile(self, enable: bool):
        self._check(self._lib.cumc_profile(self._h, int(enable)))

    def profile_read(self) -> dict:
        out = {}
        for i, name in enumerate(N.K_NAMES):
            n, ms = ctypes.c_int(), ctypes.c_double()
            self._check(self._lib.cumc_profile_read(self._h, i, ctypes.byref(n), ctypes.byref(ms)))
            out[name] = (n.value, ms.value)
        return out

    def query(self, what: int) -> int:
        """cumc_query: how the context runs a stage (N.Q_X_STAGING, N.Q_FUSED)"""
        v = ctypes.c_longlong()
        self._check(self._lib.cumc_query(self._h, int(what), ctypes.byref(v)))
        return v.value

    def launch_count(self) -> int:
        c = ctypes.c_longlong()
        self._check(self._lib.cumc_launch_count(self._h, ctypes.byref(c)))
        return c.value
