"""The reference's own kernels, compiled from its sources under a host
work-group shim (oracle/ref/, `make -C oracle ref`) into
oracle/_ref/libref_kernels.so: the checker the oracle's restatement is
compared with.  Test infrastructure only; the product never loads it.

Wraps: random.cl's uniform_rand and exprnd, the Philox4x32 stand-in it is
built with, simulate_poisson_neurons (input_neuron_group.cl:6-45),
neuron_dynamics (lif.cl:15-34) and the connectivity kernels
(network.cl:14-107)."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libref_kernels.so"
REFERENCE_KERNELS = Path("/root/reference/include/naer/kernels")

_lib = None


def available() -> bool:
    return LIB.exists()


def build() -> Path | None:
    """Builds the library when the reference sources are present (a no-op
    otherwise: a library built earlier is used as it is)."""
    if REFERENCE_KERNELS.is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref"], check=True)
    return LIB if LIB.exists() else None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        lib = C.CDLL(str(LIB))
        u32, f32, f64, u64, vp = C.c_uint32, C.c_float, C.c_double, C.c_uint64, C.c_void_p
        lib.ref_philox4x32.argtypes = [vp, vp, vp]
        lib.ref_uniform_rand.argtypes = [u32, u32, u32]
        lib.ref_uniform_rand.restype = f64
        lib.ref_exprnd.argtypes = [u32, f64, u32, u32]
        lib.ref_exprnd.restype = f64
        lib.ref_poisson_neurons.argtypes = [u32, u32, u32, u32, u32, u32, vp, vp, u32]
        lib.ref_poisson_neurons.restype = u32
        lib.ref_bernoulli.argtypes = [u32, u32, u32, u32, f64, f32, f32, f32, vp, vp, vp, u64]
        lib.ref_bernoulli.restype = u64
        lib.ref_neuron_dynamics_run.argtypes = [vp, vp, u32, vp, vp, vp]
        _lib = lib
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


def philox4x32(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.empty(4, dtype=np.uint32)
    load().ref_philox4x32(_p(c), _p(k), _p(out))
    return out


def uniform_rand(gid: int, seed: int, iteration: int) -> float:
    return load().ref_uniform_rand(gid, seed, iteration)


def exprnd(gid: int, rate: float, seed: int, iteration: int) -> float:
    return load().ref_exprnd(gid, rate, seed, iteration)


def poisson_neurons(total: int, seed: int, t0: int, t1: int, capacity: int = 2048, local_size: int = 128):
    """Spikes (times, addresses) of one window of the reference's 20 Hz
    generators, sorted by (address, time)."""
    cap = total * 10
    t = np.empty(cap, dtype=np.uint32)
    a = np.empty(cap, dtype=np.uint32)
    n = load().ref_poisson_neurons(total, capacity, local_size, seed, t0, t1, _p(t), _p(a), cap)
    assert n <= cap
    o = np.lexsort((t[:n], a[:n]))
    return t[:n][o], a[:n][o]


def bernoulli(src_size: int, dst_size: int, seed: int, p: float, w: float, wmin: float = 0.0, wmax: float = 0.0,
              group_capacity: int = 512):
    """Synapses (source, destination, weight) of one connection, sorted by
    (source, destination)."""
    cap = src_size * dst_size
    s = np.empty(cap, dtype=np.uint32)
    d = np.empty(cap, dtype=np.uint32)
    x = np.empty(cap, dtype=np.float32)
    n = load().ref_bernoulli(src_size, dst_size, group_capacity, seed, p, w, wmin, wmax, _p(s), _p(d), _p(x), cap)
    assert n <= cap, "sizes beyond the reference build's compile-time groups"
    o = np.lexsort((d[:n], s[:n]))
    return s[:n][o], d[:n][o], x[:n][o]


def neuron_dynamics(times, weights):
    """One neuron under lif.cl's neuron_dynamics: (fired flags, final V,
    last time)."""
    t = np.ascontiguousarray(times, dtype=np.uint32)
    w = np.ascontiguousarray(weights, dtype=np.float32)
    fired = np.empty(len(t), dtype=np.uint8)
    v = C.c_float()
    tl = C.c_uint32()
    load().ref_neuron_dynamics_run(_p(t), _p(w), len(t), C.byref(v), C.byref(tl), _p(fired))
    return fired.astype(bool), np.float32(v.value), int(tl.value)
