"""ORACLE — test infrastructure only: ctypes binding of oracle/liboracle.so.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the
checker; the product (naer_b200) never imports it.  See oracle.cpp for what
it restates and the parity status.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class OrPop(C.Structure):
    _fields_ = [("type", C.c_uint32), ("size", C.c_uint32), ("tau_m_ms", C.c_float), ("v_th", C.c_float),
                ("v_reset", C.c_float), ("t_ref_ms", C.c_float), ("v_init", C.c_float), ("rate_hz", C.c_float),
                ("drive_rate_hz", C.c_float), ("drive_weight", C.c_float), ("drive_seed", C.c_uint32),
                ("pad", C.c_uint32)]


class OrConn(C.Structure):
    _fields_ = [("src", C.c_uint32), ("dst", C.c_uint32), ("rule", C.c_uint32), ("degree", C.c_uint32),
                ("p", C.c_double), ("weight", C.c_float), ("wmin", C.c_float), ("wmax", C.c_float),
                ("dmin", C.c_uint32), ("dmax", C.c_uint32), ("pad", C.c_uint32), ("seed", C.c_uint64),
                ("rp", C.c_void_p), ("tg", C.c_void_p), ("wv", C.c_void_p), ("dv", C.c_void_p)]


class OrParams(C.Structure):
    _fields_ = [("dt_us", C.c_uint32), ("deterministic", C.c_uint32), ("poisson_seed", C.c_uint32),
                ("stdp_enabled", C.c_uint32), ("tau_plus_ms", C.c_float), ("tau_minus_ms", C.c_float),
                ("a_plus", C.c_float), ("a_minus", C.c_float), ("w_max", C.c_float), ("stdp_history", C.c_uint32),
                ("threads", C.c_int32)]


_vp = C.c_void_p
_lib = None


def build(force: bool = False) -> Path:
    src = HERE / "oracle.cpp"
    if force or not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "-B" if force else "liboracle.so"], check=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        sig = {
            "oracle_philox4x32_10": (None, [_vp, _vp, _vp]),
            "oracle_uniform_rand": (C.c_double, [C.c_uint32, C.c_uint32, C.c_uint32]),
            "oracle_exp_interval_us": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_double]),
            "oracle_poisson_window": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_uint32,
                                                   C.c_uint32, _vp]),
            "oracle_intervals": (None, [C.c_double, C.c_uint32, C.c_uint32, C.c_uint64, _vp]),
            "oracle_net_create": (_vp, [C.POINTER(OrParams), C.POINTER(OrPop), C.c_uint32, C.POINTER(OrConn),
                                        C.c_uint32]),
            "oracle_net_destroy": (None, [_vp]),
            "oracle_net_build": (C.c_int, [_vp]),
            "oracle_net_neurons": (C.c_uint32, [_vp]),
            "oracle_net_synapses": (C.c_uint64, [_vp]),
            "oracle_net_ring_slots": (C.c_uint32, [_vp]),
            "oracle_net_population_base": (C.c_uint32, [_vp, C.c_uint32]),
            "oracle_net_copy_csr": (None, [_vp, _vp, _vp, _vp, _vp]),
            "oracle_net_set_weights": (None, [_vp, _vp]),
            "oracle_net_run": (C.c_int, [_vp, C.c_uint64]),
            "oracle_net_step": (C.c_uint64, [_vp]),
            "oracle_net_events": (C.c_uint64, [_vp]),
            "oracle_net_hist_overflow": (C.c_uint64, [_vp]),
            "oracle_net_spike_count": (C.c_uint64, [_vp]),
            "oracle_net_copy_spikes": (None, [_vp, _vp, _vp]),
            "oracle_net_clear_spikes": (None, [_vp]),
            "oracle_net_copy_state": (None, [_vp, _vp, _vp]),
            "oracle_net_set_state": (None, [_vp, _vp, _vp]),
            "oracle_net_copy_ring": (None, [_vp, _vp]),
            "oracle_net_exact_shift": (C.c_int32, [_vp]),
            "oracle_net_copy_weights": (None, [_vp, _vp]),
            "oracle_max_threads": (C.c_int, []),
            "oracle_reintegrate_fp64": (C.c_int, [_vp, C.c_uint64, _vp, _vp, C.c_uint64, _vp, _vp,
                                                  C.POINTER(C.c_uint64)]),
            "oracle_reintegrate_fp64_ex": (C.c_int, [_vp, C.c_uint64, _vp, _vp, C.c_uint64, _vp, _vp,
                                                     C.POINTER(C.c_uint64), C.c_int, C.POINTER(C.c_uint64)]),
            "oracle_net_run_events": (C.c_int, [_vp, C.c_uint64, C.c_uint32]),
            "oracle_net_event_spike_count": (C.c_uint64, [_vp]),
            "oracle_net_event_copy": (None, [_vp, _vp, _vp, _vp, _vp, C.POINTER(C.c_uint64)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def _ptr(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


def philox4x32_10(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.empty(4, dtype=np.uint32)
    load().oracle_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return out


def uniform_rand(gid: int, seed: int, iteration: int) -> float:
    return load().oracle_uniform_rand(gid, seed, iteration)


def exp_interval_us(gid: int, seed: int, iteration: int, rate: float) -> int:
    """(uint)exprnd(rate) of random.cl:26-30 (saturated where x = 1)."""
    return load().oracle_exp_interval_us(gid, seed, iteration, rate)


def poisson_window(idx: int, n: int, seed: int, rate: float, t0: int, t1: int) -> np.ndarray:
    times = np.empty(10, dtype=np.uint32)
    c = load().oracle_poisson_window(idx, n, seed, rate, t0 & 0xFFFFFFFF, t1 & 0xFFFFFFFF, _ptr(times))
    return times[:c].copy()


class OracleNet:
    """The oracle's copy of a network described by a naer_b200.spec.NetSpec."""

    def __init__(self, spec, threads: int = 0, deterministic: bool | None = None):
        """deterministic: None follows the spec (its exact-sum mode
        included); True / False force the canonical fold / parallel adds."""
        lib = load()
        mode = (2 if getattr(spec, "exact", False) else int(spec.deterministic)) if deterministic is None \
            else int(deterministic)
        prm = OrParams(spec.dt_us, mode,
                       spec.poisson_seed, int(spec.stdp_enabled), spec.tau_plus_ms, spec.tau_minus_ms, spec.a_plus,
                       spec.a_minus, spec.w_max, spec.stdp_history, threads)
        pops = (OrPop * max(1, len(spec.pops)))()
        for i, p in enumerate(spec.pops):
            pops[i] = OrPop(p.type, p.size, p.tau_m_ms, p.v_th, p.v_reset, p.t_ref_ms, p.v_init, p.rate_hz,
                            p.drive_rate_hz, p.drive_weight, p.drive_seed, 0)
        conns = (OrConn * max(1, len(spec.conns)))()
        for i, c in enumerate(spec.conns):
            conns[i] = OrConn(c.src, c.dst, c.rule, c.degree, c.probability, c.weight, c.wmin, c.wmax, c.dmin,
                              c.dmax, 0, c.seed & 0xFFFFFFFFFFFFFFFF)
            if getattr(c, "csr", None) is not None:  # explicit synapses: arrays alive through the build below
                conns[i].rp, conns[i].tg, conns[i].wv, conns[i].dv = (a.ctypes.data for a in c.csr)
        self._lib = lib
        self._h = lib.oracle_net_create(C.byref(prm), pops, len(spec.pops), conns, len(spec.conns))
        if lib.oracle_net_build(self._h) != 0:
            lib.oracle_net_destroy(self._h)
            self._h = None
            raise ValueError("weights too large for exact-sum aggregation")
        self.n = lib.oracle_net_neurons(self._h)
        self.S = lib.oracle_net_synapses(self._h)

    def close(self):
        if self._h:
            self._lib.oracle_net_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def exact_shift(self) -> int:
        """S of the exact-sum mode: weights on the grid 2^-S."""
        return self._lib.oracle_net_exact_shift(self._h)

    def population_base(self, pop: int) -> int:
        return self._lib.oracle_net_population_base(self._h, pop)

    def csr(self):
        rp = np.empty(self.n + 1, dtype=np.uint64)
        tg = np.empty(self.S, dtype=np.uint32)
        w = np.empty(self.S, dtype=np.float32)
        d = np.empty(self.S, dtype=np.uint8)
        self._lib.oracle_net_copy_csr(self._h, _ptr(rp), _ptr(tg), _ptr(w), _ptr(d))
        return rp, tg, w, d

    def set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == self.S
        self._lib.oracle_net_set_weights(self._h, _ptr(w))

    def run(self, nsteps: int) -> None:
        self._lib.oracle_net_run(self._h, int(nsteps))

    @property
    def events(self) -> int:
        return self._lib.oracle_net_events(self._h)

    @property
    def hist_overflow(self) -> int:
        return self._lib.oracle_net_hist_overflow(self._h)

    def spikes(self):
        n = self._lib.oracle_net_spike_count(self._h)
        st = np.empty(n, dtype=np.uint32)
        ids = np.empty(n, dtype=np.uint32)
        self._lib.oracle_net_copy_spikes(self._h, _ptr(st), _ptr(ids))
        return st, ids

    def clear_spikes(self) -> None:
        self._lib.oracle_net_clear_spikes(self._h)

    def state(self):
        v = np.empty(self.n, dtype=np.float32)
        r = np.empty(self.n, dtype=np.uint32)
        self._lib.oracle_net_copy_state(self._h, _ptr(v), _ptr(r))
        return v, r

    def weights(self) -> np.ndarray:
        w = np.empty(self.S, dtype=np.float32)
        self._lib.oracle_net_copy_weights(self._h, _ptr(w))
        return w

    def run_events(self, windows: int, truncate96: bool = False) -> None:
        """Reference-compatible event mode: `windows` windows of 1500 us
        (see oracle_net_run_events)."""
        self._lib.oracle_net_run_events(self._h, int(windows), 1 if truncate96 else 0)

    def event_spikes(self):
        """(time in us, address) of every spike of the event mode so far."""
        n = self._lib.oracle_net_event_spike_count(self._h)
        t = np.empty(n, dtype=np.uint32)
        i = np.empty(n, dtype=np.uint32)
        self._lib.oracle_net_event_copy(self._h, _ptr(t), _ptr(i), None, None, None)
        return t, i

    def event_state(self):
        """(V, last update or refractory end time in us, synapses delivered)."""
        v = np.empty(self.n, dtype=np.float32)
        tl = np.empty(self.n, dtype=np.uint32)
        d = C.c_uint64()
        self._lib.oracle_net_event_copy(self._h, None, None, _ptr(v), _ptr(tl), C.byref(d))
        return v, tl, d.value

    def reintegrate_fp64(self, steps: np.ndarray, ids: np.ndarray, nsteps: int):
        """FP64 re-integration from the initial state (use a network that has
        not been run) with the spike times of a raster (steps, ids), raster
        ordered by step.  Returns (V float64 per address, weights float64 in
        address-order CSR, threshold mismatches)."""
        st = np.ascontiguousarray(steps, dtype=np.uint32)
        ii = np.ascontiguousarray(ids, dtype=np.uint32)
        v = np.empty(self.n, dtype=np.float64)
        w = np.empty(self.S, dtype=np.float64)
        mis = C.c_uint64()
        self._lib.oracle_reintegrate_fp64(self._h, int(nsteps), _ptr(st), _ptr(ii), len(st), _ptr(v), _ptr(w),
                                          C.byref(mis))
        return v, w, mis.value

    def reintegrate_fp64_uncapped(self, steps: np.ndarray, ids: np.ndarray, nsteps: int):
        """reintegrate_fp64 with lazy LTP over every post spike since the
        source's last spike (no post-history limit): the pair rule itself.
        Returns (V, weights, threshold mismatches, pairs the history limit
        drops on these spike times)."""
        st = np.ascontiguousarray(steps, dtype=np.uint32)
        ii = np.ascontiguousarray(ids, dtype=np.uint32)
        v = np.empty(self.n, dtype=np.float64)
        w = np.empty(self.S, dtype=np.float64)
        mis = C.c_uint64()
        lost = C.c_uint64()
        self._lib.oracle_reintegrate_fp64_ex(self._h, int(nsteps), _ptr(st), _ptr(ii), len(st), _ptr(v), _ptr(w),
                                             C.byref(mis), 1, C.byref(lost))
        return v, w, mis.value, lost.value


def intervals(rate: float, z_first: int, z_step: int, count: int) -> np.ndarray:
    """The Poisson interval (µs) of z = z_first + i * z_step with glibc's log."""
    out = np.empty(count, dtype=np.uint32)
    load().oracle_intervals(float(rate), int(z_first), int(z_step), int(count), out.ctypes.data_as(C.c_void_p))
    return out


def max_threads() -> int:
    return load().oracle_max_threads()
