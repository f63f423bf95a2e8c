"""ctypes binding of include/naer/naer_capi.h (the library's C ABI).

The library is the in-tree ``libnaer_b200.so`` built by ``naer_b200.build``.
Loading fails loudly when it is missing: there is no fallback
implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libnaer_b200.so"
# NAER_CHECKED=1 in the environment loads the bounds-checked build instead
LIB_CHECKED_PATH = Path(__file__).resolve().parent / "libnaer_b200_checked.so"

NAER_OK = 0
NAER_E_INVALID = -1
NAER_E_OOM = -2
NAER_E_OVERFLOW = -3
NAER_E_TIMEOUT = -4
NAER_E_CUDA = -5
NAER_E_STATE = -6
NAER_E_UNSUPPORTED = -7

STATUS_NAMES = {
    NAER_E_INVALID: "NAER_E_INVALID",
    NAER_E_OOM: "NAER_E_OOM",
    NAER_E_OVERFLOW: "NAER_E_OVERFLOW",
    NAER_E_TIMEOUT: "NAER_E_TIMEOUT",
    NAER_E_CUDA: "NAER_E_CUDA",
    NAER_E_STATE: "NAER_E_STATE",
    NAER_E_UNSUPPORTED: "NAER_E_UNSUPPORTED",
}

NEURON_STDP, NEURON_NOP, NEURON_POISSON = 0, 1, 2
MODE_GRID, MODE_EVENT = 0, 1
AGG_ATOMIC, AGG_DETERMINISTIC, AGG_EXACT = 0, 1, 2
CONN_REF_BERNOULLI, CONN_FIXED_INDEGREE, CONN_FIXED_OUTDEGREE, CONN_EXPLICIT = 0, 1, 2, 3


class NetParams(C.Structure):
    _fields_ = [
        ("mode", C.c_uint32),
        ("aggregation", C.c_uint32),
        ("dt_us", C.c_uint32),
        ("record_spikes", C.c_uint32),
        ("raster_capacity", C.c_uint64),
        ("poisson_seed", C.c_uint32),
        ("stdp_enabled", C.c_uint32),
        ("tau_plus_ms", C.c_float),
        ("tau_minus_ms", C.c_float),
        ("a_plus", C.c_float),
        ("a_minus", C.c_float),
        ("w_max", C.c_float),
        ("stdp_history", C.c_uint32),
    ]


class PopParams(C.Structure):
    _fields_ = [
        ("tau_m_ms", C.c_float),
        ("v_th", C.c_float),
        ("v_reset", C.c_float),
        ("t_ref_ms", C.c_float),
        ("v_init", C.c_float),
        ("rate_hz", C.c_float),
        ("drive_rate_hz", C.c_float),
        ("drive_weight", C.c_float),
        ("drive_seed", C.c_uint32),
        ("pad_", C.c_uint32),
    ]


class ConnSpecC(C.Structure):
    _fields_ = [
        ("rule", C.c_uint32),
        ("degree", C.c_uint32),
        ("probability", C.c_double),
        ("weight", C.c_float),
        ("wmin", C.c_float),
        ("wmax", C.c_float),
        ("delay_min", C.c_uint32),
        ("delay_max", C.c_uint32),
        ("pad_", C.c_uint32),
        ("seed", C.c_uint64),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("step", C.c_uint64),
        ("events", C.c_uint64),
        ("spikes", C.c_uint64),
        ("raster_dropped", C.c_uint64),
        ("stdp_hist_overflow", C.c_uint64),
        ("synapses", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("neurons", C.c_uint32),
        ("ring_slots", C.c_uint32),
        ("kernel_launches", C.c_uint64),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("blocks_per_sm", C.c_uint32),
        ("launch_steps", C.c_uint32),
        ("scatter_split", C.c_uint32),
        ("graph_launches", C.c_uint32),
        ("best_us_per_step", C.c_double),
        ("default_us_per_step", C.c_double),
        ("trials", C.c_uint32),
        ("scatter_piece", C.c_uint32),
        ("neuron_state", C.c_uint32),
        ("step_kernel", C.c_uint32),
        ("bins", C.c_uint32),
        ("pad_", C.c_uint32),
    ]


STATE_AUTO, STATE_SHARED, STATE_GLOBAL = 0, 1, 2
KERNEL_SPLIT, KERNEL_TWO_BARRIER = 0, 1


class ServerParams(C.Structure):
    _fields_ = [
        ("budget_bytes", C.c_uint64),
        ("raster_capacity", C.c_uint64),
        ("chunk_steps", C.c_uint32),
        ("aggregation", C.c_uint32),
        ("max_jobs", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("chunk_ms", C.c_double),
        ("launch_steps", C.c_uint32),
        ("step_kernel", C.c_uint32),
    ]


class DeviceProbe(C.Structure):
    _fields_ = [
        ("ring_cells", C.c_uint64),
        ("small_cells", C.c_uint64),
        ("red_ring_per_s", C.c_double),
        ("red_small_per_s", C.c_double),
        ("store_ring_per_s", C.c_double),
        ("stream_gbs", C.c_double),
        ("barrier_us_1", C.c_double),
        ("barrier_us_2", C.c_double),
        ("grid", C.c_uint32),
        ("pad_", C.c_uint32),
    ]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = 0, 1, 2, 3, 4


class JobInfo(C.Structure):
    _fields_ = [
        ("state", C.c_uint32),
        ("preemptions", C.c_uint32),
        ("duration", C.c_uint64),
        ("steps_done", C.c_uint64),
        ("spikes", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("submit_s", C.c_double),
        ("admit_s", C.c_double),
        ("done_s", C.c_double),
    ]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "done", "failed", "running", "queued", "chunks",
                                           "engine_steps", "peak_bytes", "bytes_in_use", "raster_dropped")] + \
               [(n, C.c_double) for n in ("p50_ms", "p99_ms", "mean_ms", "sims_per_s", "build_s", "install_s",
                                          "step_s", "drain_s")]


class NaerError(RuntimeError):
    """A non-zero status from the C ABI (message from naer_last_error)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


_P = C.POINTER
_vp = C.c_void_p

# name -> argtypes (all return int status)
PROTOTYPES = {
    "naer_last_error": [C.c_char_p, C.c_size_t],
    "naer_device_count": [_P(C.c_int)],
    "naer_net_params_default": [_P(NetParams)],
    "naer_pop_params_default": [C.c_uint32, _P(PopParams)],
    "naer_net_create": [C.c_int, _P(NetParams), _P(_vp)],
    "naer_net_destroy": [_vp],
    "naer_net_add_population": [_vp, C.c_uint32, C.c_uint32, _P(PopParams), _P(C.c_uint32), _P(C.c_uint32)],
    "naer_net_add_connection": [_vp, C.c_uint32, C.c_uint32, _P(ConnSpecC)],
    "naer_net_add_connection_csr": [_vp, C.c_uint32, C.c_uint32, _vp, _vp, _vp, _vp],
    "naer_net_compile": [_vp],
    "naer_net_population_base": [_vp, C.c_uint32, _P(C.c_uint32)],
    "naer_net_step": [_vp, C.c_uint64],
    "naer_net_step_noalloc": [_vp, C.c_uint64],
    "naer_net_finish": [_vp],
    "naer_net_get_time_us": [_vp, _P(C.c_uint64)],
    "naer_net_get_synapses": [_vp, _P(C.c_uint64)],
    "naer_net_get_neurons": [_vp, _P(C.c_uint32)],
    "naer_net_get_stats": [_vp, _P(Stats)],
    "naer_net_read_spikes": [_vp, C.c_uint64, C.c_uint64, _vp, _vp, _P(C.c_uint64)],
    "naer_net_clear_spikes": [_vp],
    "naer_net_read_raster": [_vp, C.c_uint64, C.c_uint64, _vp, _P(C.c_uint64)],
    "naer_net_stream": [_vp, _P(_vp)],
    "naer_net_read_state": [_vp, _vp, _vp],
    "naer_net_write_state": [_vp, _vp, _vp],
    "naer_net_read_csr": [_vp, _vp, _vp, _vp, _vp],
    "naer_net_set_profiling": [_vp, C.c_int],
    "naer_net_get_profile": [_vp, _P(C.c_double), _P(C.c_double), _P(C.c_uint64)],
    "naer_net_get_phases": [_vp, _vp],
    "naer_net_get_launch_times": [_vp, _P(C.c_double), _P(C.c_double), _P(C.c_uint64)],
    "naer_net_set_wait_limit": [_vp, C.c_uint64],
    "naer_test_set_barrier_skew": [_vp, C.c_uint64],
    "naer_test_fail_allocation": [C.c_int64],
    "naer_build_checked": [_P(C.c_int)],
    "naer_net_check_report": [_vp, _P(C.c_uint32), _P(C.c_uint64)],
    "naer_probe_device": [C.c_int, C.c_uint64, C.c_uint64, _P(DeviceProbe)],
    "naer_probe_intervals": [C.c_int, C.c_double, C.c_uint32, C.c_uint32, C.c_uint64, _vp],
    "naer_net_autotune": [_vp, C.c_uint32, _P(Tuning)],
    "naer_net_set_tuning": [_vp, _P(Tuning)],
    "naer_net_get_tuning": [_vp, _P(Tuning)],
    "naer_batch_create": [C.c_int, C.c_uint32, C.c_uint64, _P(_vp)],
    "naer_batch_destroy": [_vp],
    "naer_batch_add": [_vp, _vp, _P(C.c_uint32)],
    "naer_batch_compile": [_vp],
    "naer_batch_step": [_vp, C.c_uint64],
    "naer_batch_finish": [_vp],
    "naer_batch_autotune": [_vp, C.c_uint32, _P(Tuning)],
    "naer_batch_set_tuning": [_vp, _P(Tuning)],
    "naer_batch_get_tuning": [_vp, _P(Tuning)],
    "naer_batch_read_spikes": [_vp, C.c_uint64, C.c_uint64, _vp, _vp, _vp, _P(C.c_uint64)],
    "naer_batch_clear_spikes": [_vp],
    "naer_batch_get_stats": [_vp, _P(Stats)],
    "naer_batch_get_phases": [_vp, _vp],
    "naer_batch_read_state": [_vp, C.c_uint32, _vp, _vp],
    "naer_batch_stream": [_vp, _P(_vp)],
    "naer_server_params_default": [_P(ServerParams)],
    "naer_server_create": [C.c_int, _P(ServerParams), _P(_vp)],
    "naer_server_destroy": [_vp],
    "naer_server_submit": [_vp, _vp, C.c_uint64, _P(C.c_uint64)],
    "naer_server_job_info": [_vp, C.c_uint64, _P(JobInfo)],
    "naer_server_job_error": [_vp, C.c_uint64, C.c_char_p, C.c_size_t],
    "naer_server_wait": [_vp, C.c_uint64, C.c_double, _P(C.c_int)],
    "naer_server_drain": [_vp, C.c_double, _P(C.c_int)],
    "naer_server_read_spikes": [_vp, C.c_uint64, C.c_uint64, C.c_uint64, _vp, _vp, _P(C.c_uint64)],
    "naer_server_release": [_vp, C.c_uint64],
    "naer_server_preempt": [_vp, C.c_uint64],
    "naer_server_cancel": [_vp, C.c_uint64],
    "naer_net_checkpoint_size": [_vp, _P(C.c_uint64)],
    "naer_net_checkpoint": [_vp, _vp, C.c_uint64],
    "naer_net_restore": [_vp, _vp, C.c_uint64],
    "naer_server_get_stats": [_vp, _P(ServerStats)],
}

_lib = None


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Loads the CUDA library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else (LIB_CHECKED_PATH if os.environ.get("NAER_CHECKED") == "1" else LIB_PATH)
    if not p.exists():
        raise RuntimeError(
            f"naer_b200 CUDA library not found at {p}; build it with `python -m naer_b200.build`")
    lib = C.CDLL(str(p))
    for name, args in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    _lib = lib
    return lib


def probe_device(device: int = 0, ring_cells: int = 17_000_000, small_cells: int = 3_000_000) -> dict:
    """naer_probe_device: the device's random-reduction, random-store,
    streaming and grid-barrier figures."""
    p = DeviceProbe()
    call("naer_probe_device", int(device), int(ring_cells), int(small_cells), C.byref(p))
    return {k: getattr(p, k) for k, _ in DeviceProbe._fields_ if k != "pad_"}


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    load().naer_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != NAER_OK:
        raise NaerError(status, last_error())


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))
