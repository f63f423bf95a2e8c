"""Batched and served forms over the C ABI (naer_batch_*, naer_server_*).

``Batch`` packs many independent networks into one engine and steps them
together; ``Server`` runs a request loop that admits simulation jobs by
device-memory footprint and steps every admitted job together.  Members and
jobs are given as ``NetSpec`` descriptions (or description-only
``Network`` handles made with device -1).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as capi
from . import spec as S


def _description(x):
    """A description-only Network for a NetSpec (the caller closes it)."""
    if isinstance(x, S.NetSpec):
        return S.describe(x, -1), True
    return x, False


class Batch:
    """Many networks of any sizes advanced by one set of persistent launches."""

    def __init__(self, members=(), device: int = 0, deterministic: bool = False, raster_capacity: int = 1 << 24,
                 exact: bool = False):
        capi.load()
        h = C.c_void_p()
        agg = capi.AGG_EXACT if exact else capi.AGG_DETERMINISTIC if deterministic else capi.AGG_ATOMIC
        capi.call("naer_batch_create", int(device), agg, int(raster_capacity), C.byref(h))
        self._h = h
        self.n = 0
        for m in members:
            self.add(m)

    def add(self, member) -> int:
        d, owned = _description(member)
        try:
            idx = C.c_uint32()
            capi.call("naer_batch_add", self._h, d.handle, C.byref(idx))
        finally:
            if owned:
                d.close()
        self.n += 1
        return idx.value

    def compile(self) -> "Batch":
        capi.call("naer_batch_compile", self._h)
        return self

    def run(self, nsteps: int) -> None:
        if nsteps < 0:
            raise ValueError("nsteps must be >= 0")
        capi.call("naer_batch_step", self._h, int(nsteps))

    def finish(self) -> None:
        capi.call("naer_batch_finish", self._h)

    def autotune(self, trial_steps: int = 64) -> dict:
        t = capi.Tuning()
        capi.call("naer_batch_autotune", self._h, int(trial_steps), C.byref(t))
        return {k: getattr(t, k) for k, _ in capi.Tuning._fields_ if k != "pad_"}

    def tuning(self) -> dict:
        t = capi.Tuning()
        capi.call("naer_batch_get_tuning", self._h, C.byref(t))
        return {k: getattr(t, k) for k, _ in capi.Tuning._fields_ if k != "pad_"}

    def set_tuning(self, blocks_per_sm=0, launch_steps=64, scatter_split=0, graph_launches=16,
                   scatter_piece=0, neuron_state=capi.STATE_AUTO, step_kernel=capi.KERNEL_SPLIT, bins=0) -> None:
        t = capi.Tuning(blocks_per_sm=blocks_per_sm, launch_steps=launch_steps, scatter_split=scatter_split,
                        graph_launches=graph_launches, scatter_piece=scatter_piece, neuron_state=neuron_state,
                        step_kernel=step_kernel, bins=bins)
        capi.call("naer_batch_set_tuning", self._h, C.byref(t))

    def stats(self) -> dict:
        st = capi.Stats()
        capi.call("naer_batch_get_stats", self._h, C.byref(st))
        return {k: getattr(st, k) for k, _ in capi.Stats._fields_}

    def phases(self) -> dict:
        """The step kernel's device time split (ms since compile, first block)."""
        ph = (C.c_double * 5)()
        capi.call("naer_batch_get_phases", self._h, C.cast(ph, C.c_void_p))
        return {k: ph[i] for i, k in enumerate(["lif", "lif_wait", "scatter", "reserved", "scatter_wait"])}

    def read_spikes(self):
        """(member, step, id) arrays of every recorded spike."""
        total = self.stats()["spikes"]
        m = np.zeros(total, np.uint32)
        st = np.zeros(total, np.uint32)
        ids = np.zeros(total, np.uint32)
        n = C.c_uint64()
        if total:
            capi.call("naer_batch_read_spikes", self._h, 0, int(total), m.ctypes.data_as(C.c_void_p),
                      st.ctypes.data_as(C.c_void_p), ids.ctypes.data_as(C.c_void_p), C.byref(n))
        return m[:n.value], st[:n.value], ids[:n.value]

    def member_spikes(self, member: int, spikes=None):
        m, st, ids = spikes if spikes is not None else self.read_spikes()
        sel = m == member
        return st[sel], ids[sel]

    def clear_spikes(self) -> None:
        capi.call("naer_batch_clear_spikes", self._h)

    def read_state(self, member: int, neurons: int):
        v = np.zeros(neurons, np.float32)
        r = np.zeros(neurons, np.uint32)
        capi.call("naer_batch_read_state", self._h, int(member), v.ctypes.data_as(C.c_void_p),
                  r.ctypes.data_as(C.c_void_p))
        return v, r

    def stream(self) -> int:
        p = C.c_void_p()
        capi.call("naer_batch_stream", self._h, C.byref(p))
        return p.value or 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            capi.call("naer_batch_destroy", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (a host thread inside the library)."""

    def __init__(self, device: int = 0, budget_bytes: int = 150 * 10**9, chunk_steps: int = 256,
                 deterministic: bool = False, max_jobs: int = 1024, raster_capacity: int = 1 << 24,
                 blocks_per_sm: int = 0, chunk_ms: float = 10.0, launch_steps: int = 0, exact: bool = False,
                 step_kernel: int = capi.KERNEL_TWO_BARRIER):
        capi.load()
        p = capi.ServerParams()
        capi.call("naer_server_params_default", C.byref(p))
        p.budget_bytes = int(budget_bytes)
        p.chunk_steps = int(chunk_steps)
        p.aggregation = capi.AGG_EXACT if exact else capi.AGG_DETERMINISTIC if deterministic else capi.AGG_ATOMIC
        p.max_jobs = int(max_jobs)
        p.raster_capacity = int(raster_capacity)
        p.blocks_per_sm = int(blocks_per_sm)
        p.chunk_ms = float(chunk_ms)
        p.launch_steps = int(launch_steps)
        p.step_kernel = int(step_kernel)
        h = C.c_void_p()
        capi.call("naer_server_create", int(device), C.byref(p), C.byref(h))
        self._h = h

    def submit(self, job, duration_steps: int) -> int:
        d, owned = _description(job)
        try:
            jid = C.c_uint64()
            capi.call("naer_server_submit", self._h, d.handle, int(duration_steps), C.byref(jid))
        finally:
            if owned:
                d.close()
        return jid.value

    def info(self, job: int) -> dict:
        i = capi.JobInfo()
        capi.call("naer_server_job_info", self._h, int(job), C.byref(i))
        return {k: getattr(i, k) for k, _ in capi.JobInfo._fields_ if k != "pad_"}

    def error(self, job: int) -> str:
        buf = C.create_string_buffer(4096)
        capi.call("naer_server_job_error", self._h, int(job), buf, len(buf))
        return buf.value.decode(errors="replace")

    def wait(self, job: int, timeout_s: float = 600.0) -> bool:
        f = C.c_int()
        capi.call("naer_server_wait", self._h, int(job), float(timeout_s), C.byref(f))
        return bool(f.value)

    def drain(self, timeout_s: float = 600.0) -> bool:
        f = C.c_int()
        capi.call("naer_server_drain", self._h, float(timeout_s), C.byref(f))
        return bool(f.value)

    def spikes(self, job: int):
        """(step, id) of a finished job, ordered by step then id."""
        n = self.info(job)["spikes"]
        st = np.zeros(n, np.uint32)
        ids = np.zeros(n, np.uint32)
        got = C.c_uint64()
        if n:
            capi.call("naer_server_read_spikes", self._h, int(job), 0, int(n), st.ctypes.data_as(C.c_void_p),
                      ids.ctypes.data_as(C.c_void_p), C.byref(got))
        return st[:got.value], ids[:got.value]

    def release(self, job: int) -> None:
        capi.call("naer_server_release", self._h, int(job))

    def preempt(self, job: int) -> None:
        """Takes a running job off the device at the next chunk boundary; it
        queues again and resumes from the step it reached."""
        capi.call("naer_server_preempt", self._h, int(job))

    def cancel(self, job: int) -> None:
        capi.call("naer_server_cancel", self._h, int(job))

    def stats(self) -> dict:
        s = capi.ServerStats()
        capi.call("naer_server_get_stats", self._h, C.byref(s))
        return {k: getattr(s, k) for k, _ in capi.ServerStats._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            capi.call("naer_server_destroy", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
