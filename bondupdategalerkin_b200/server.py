"""Batched and served time evolution: many chains on one GPU through the native job server.

``Server(workers, budget_bytes)`` wraps ``bug_server_*`` (``include/bug_b200.h``): worker threads
inside the library, each with its own engine context and stream, take jobs from one FIFO queue,
admitted by projected HBM footprint. A job is ``nsteps`` native BUG steps of one chain given by
host blocks; its Gaussian probes come from its own ``numpy`` generator seeded by the job, so its
result is the same whether it runs alone or among others.

``Server.submit`` returns a ``Job``; ``Server.wait`` blocks (releasing the GIL) until jobs finish;
``Job.result`` is the final state as host blocks and ``Job.stats`` the timings (submit, start, end,
per-step latencies with the worker's stream drained).
"""

from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _engine as E
from .native import DRAW_FN, StepParams, step_params
from .tensor import DT, Leg, from_blocks, to_blocks

LOAD_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                           ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int),
                           ctypes.POINTER(ctypes.c_void_p))
DONE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                           ctypes.POINTER(ctypes.c_void_p), ctypes.c_int)

JOB_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


class JobSpec(ctypes.Structure):
    _fields_ = [("tau_re", ctypes.c_double), ("tau_im", ctypes.c_double), ("nsteps", ctypes.c_int),
                ("params", StepParams), ("draw", DRAW_FN), ("draw_user", ctypes.c_void_p),
                ("load", LOAD_FN), ("done", DONE_FN), ("user", ctypes.c_void_p),
                ("footprint_bytes", ctypes.c_int64)]


class JobStats(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("status", ctypes.c_int), ("worker", ctypes.c_int),
                ("steps_done", ctypes.c_int), ("t_submit", ctypes.c_double),
                ("t_start", ctypes.c_double), ("t_end", ctypes.c_double),
                ("step_s_sum", ctypes.c_double), ("step_s_max", ctypes.c_double)]


class _Borrowed:
    """A worker's context seen from a callback: used, never owned."""

    def __init__(self, h):
        self.h = ctypes.c_void_p(h)
        self.lib = E.load()


def projected_footprint(L: int, d: int, maxdim: int, mpo_dim: int) -> int:
    """Projected HBM bytes of one chain at bond dimension ``maxdim`` (``bug_projected_footprint``)."""
    return int(E.load().bug_projected_footprint(L, d, maxdim, mpo_dim))


def host_blocks(tensors):
    """Host copies ``[(legs, blocks)]`` of device tensors (for building jobs from device states)."""
    return [to_blocks(t) for t in tensors]


class Job:
    """One submitted chain; holds its callbacks alive until the server is done with them."""

    def __init__(self, server, state, center, mpo, tau, nsteps, seed, kw):
        self.server = server
        self.state, self.center, self.mpo = state, center, mpo
        self.tau, self.nsteps, self.seed = complex(tau), int(nsteps), seed
        self.rng = np.random.default_rng(seed)
        self.result = None       # [(legs, blocks)] of the final state, and its centre
        self.result_center = None
        self.error = None
        self.id = None
        L = len(state)

        @DRAW_FN
        def draw(user, n, out):
            x = self.rng.standard_normal(int(n))
            ctypes.memmove(out, x.ctypes.data, 8 * int(n))

        @LOAD_FN
        def load(user, ctx, Lp, psi, centerp, mpop):
            try:
                c = _Borrowed(ctx)
                for i, (legs, blocks) in enumerate(self.state):
                    t = from_blocks(legs, blocks, c)
                    psi[i] = t.h.value
                    t.h = None  # the server owns the handle now
                for i, (legs, blocks) in enumerate(self.mpo):
                    t = from_blocks(legs, blocks, c)
                    mpop[i] = t.h.value
                    t.h = None
                Lp[0] = L
                centerp[0] = self.center
                return 0
            except Exception as exc:  # noqa: BLE001 - reported through the job
                self.error = repr(exc)
                return 1

        @DONE_FN
        def done(user, ctx, status, Ln, psi, center):
            if status != 0:
                return
            try:
                c = _Borrowed(ctx)
                out = []
                for i in range(Ln):
                    t = DT(c, ctypes.c_void_p(psi[i]))
                    out.append(to_blocks(t))
                    t.h = None  # borrowed: the server frees it
                self.result, self.result_center = out, int(center)
            except Exception as exc:  # noqa: BLE001
                self.error = repr(exc)

        self._cb = (draw, load, done)
        maxdim = kw.get("maxdim") or 128
        d = sum(state[0][0][1].sectors.values())                     # local dimension
        w = max(max(sum(legs[3].sectors.values()) for legs, _ in mpo), 1)  # MPO bond dimension
        self.spec = JobSpec(tau_re=self.tau.real, tau_im=self.tau.imag, nsteps=self.nsteps,
                            params=step_params(L, **kw), draw=draw, draw_user=None, load=load,
                            done=done, user=None,
                            footprint_bytes=projected_footprint(L, d, maxdim, w))

    @property
    def stats(self) -> dict:
        lib = self.server.lib
        st = JobStats()
        E.check(lib.bug_server_job_stats(self.server.h, self.id, ctypes.addressof(st)))
        n = ctypes.c_int()
        E.check(lib.bug_server_step_times(self.server.h, self.id, None, 0, ctypes.byref(n)))
        buf = (ctypes.c_double * max(n.value, 1))()
        E.check(lib.bug_server_step_times(self.server.h, self.id, buf, n.value, ctypes.byref(n)))
        msg = ctypes.create_string_buffer(512)
        E.check(lib.bug_server_job_error(self.server.h, self.id, msg, 512))
        return dict(state=JOB_STATES[st.state], status=st.status, worker=st.worker,
                    steps_done=st.steps_done, t_submit=st.t_submit, t_start=st.t_start,
                    t_end=st.t_end, step_s=list(buf[:n.value]),
                    error=self.error or (msg.value.decode(errors="replace") or None))


class Server:
    """A pool of ``workers`` native workers on ``device`` admitting jobs within ``budget_bytes``."""

    def __init__(self, workers: int = 8, budget_bytes: int = 64 << 30, device: int = 0):
        self.lib = E.load()
        self.h = ctypes.c_void_p()
        E.check(self.lib.bug_server_create(device, workers, budget_bytes, ctypes.byref(self.h)))
        self.jobs = []
        self._lock = threading.Lock()

    def submit(self, state, center, mpo, tau, nsteps, seed, **kw) -> Job:
        """Queue a chain: ``state`` / ``mpo`` as host blocks ``[(legs, blocks)]`` (site order),
        ``center`` 1-based, ``nsteps`` steps of ``tau`` with the step keywords ``kw``; the probes
        come from ``numpy.random.default_rng(seed)``."""
        job = Job(self, state, center, mpo, tau, nsteps, seed, kw)
        jid = ctypes.c_int64()
        E.check(self.lib.bug_server_submit(self.h, ctypes.addressof(job.spec), ctypes.byref(jid)))
        job.id = jid.value
        with self._lock:
            self.jobs.append(job)
        return job

    def cancel(self, job: Job) -> None:
        E.check(self.lib.bug_server_cancel(self.h, job.id))

    def wait(self, job: Job | None = None, timeout: float | None = None) -> bool:
        """Block until ``job`` (or every job) has finished; False if ``timeout`` passed first."""
        fin = ctypes.c_int()
        E.check(self.lib.bug_server_wait(self.h, job.id if job else 0,
                                         -1.0 if timeout is None else float(timeout),
                                         ctypes.byref(fin)))
        return bool(fin.value)

    def launches(self) -> int:
        """Kernel launches issued by all workers so far."""
        return int(self.lib.bug_server_launches(self.h))

    def close(self) -> None:
        if self.h:
            E.check(self.lib.bug_server_destroy(self.h))
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def latency_summary(jobs) -> dict:
    """p50 / p99 of per-step latency and of per-job latency (submit to end), in seconds."""
    steps = np.array([s for j in jobs for s in j.stats["step_s"]])
    per_job = np.array([j.stats["t_end"] - j.stats["t_submit"] for j in jobs])
    q = lambda a, p: float(np.percentile(a, p)) if a.size else None  # noqa: E731
    return {"step_p50_s": q(steps, 50), "step_p99_s": q(steps, 99),
            "job_p50_s": q(per_job, 50), "job_p99_s": q(per_job, 99),
            "steps": int(steps.size), "jobs": int(per_job.size)}


__all__ = ["Server", "Job", "projected_footprint", "host_blocks", "latency_summary", "Leg"]
