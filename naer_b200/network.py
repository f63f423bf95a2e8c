"""Host-side mirror of the reference's C++ model-building API.

``Network``, ``NeuronType``, ``Population`` and ``Connection`` keep the
names, arguments and error behaviour of the reference
(include/naer/Network.h:15-142, Population.h, Connection.h,
src/Network.cpp): populations are added per neuron type and receive a
type-local base address that compile() shifts by the type base; the
two ``addConnection`` overloads take (weight, probability) or (weight,
min weight, max weight, probability, seed); ``step()`` advances one
1500 µs window and returns without waiting; ``finish()`` blocks; every
failure raises (the reference throws std::runtime_error).

The calls go through the C ABI (include/naer/naer_capi.h) to the CUDA
library; nothing here computes on the host.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi

REF_WINDOW_US = 1500  # NAER_AXONAL_DELAY and the step() window (naer_types.h:4, Network.cpp:125)
REF_DEFAULT_SEED = 0xBF785E3215AC7EBD  # Network.cpp:91


class NeuronType(enum.IntEnum):
    STDP = capi.NEURON_STDP
    NOP = capi.NEURON_NOP
    POISSON = capi.NEURON_POISSON


@dataclass
class Population:
    """Population.h:9-17 — type, baseAddress, size (plus the handle's id)."""

    type: NeuronType
    baseAddress: int
    size: int
    id: int = 0
    params: dict = field(default_factory=dict, repr=False)


@dataclass
class Connection:
    """Connection.h:8-30 plus the grid-mode rule, degree and delays."""

    source: Population
    destination: Population
    defaultWeights: float
    minRandomWeights: float
    maxRandomWeights: float
    probability: float
    seed: int
    rule: int = capi.CONN_REF_BERNOULLI
    degree: int = 0
    delay_min: int = 15
    delay_max: int = 15


def pop_params(neuron_type: int, **kw) -> capi.PopParams:
    p = capi.PopParams()
    capi.call("naer_pop_params_default", int(neuron_type), C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown population parameter {k!r}")
        setattr(p, k, v)
    return p


def net_params(**kw) -> capi.NetParams:
    p = capi.NetParams()
    capi.call("naer_net_params_default", C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown network parameter {k!r}")
        setattr(p, k, v)
    return p


class Network:
    """One network on one GPU (the plain form)."""

    def __init__(self, device: int = 0, **params):
        self._lib = capi.load()
        self.params = net_params(**params)
        h = C.c_void_p()
        capi.call("naer_net_create", int(device), C.byref(self.params), C.byref(h))
        self._h = h
        self._pops: list[Population] = []
        self._conns: list[Connection] = []
        self._compiled = False
        # reference profile counters (Network.h:50-55), filled by profile()
        self.nop_time = self.stdp_time = self.poisson_time = 0.0
        self.scan_time = self.scatter_time = self.offset_time = 0.0

    # -- lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            capi.call("naer_net_destroy", self._h)
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
    def handle(self) -> C.c_void_p:
        return self._h

    # -- model building (Network.cpp:77-105)
    def addPopulation(self, type: NeuronType, size: int, **params) -> Population:
        prm = pop_params(int(type), **params)
        pid = C.c_uint32()
        addr = C.c_uint32()
        capi.call("naer_net_add_population", self._h, int(type), int(size), C.byref(prm), C.byref(pid),
                  C.byref(addr))
        pop = Population(NeuronType(type), addr.value, int(size), pid.value, dict(params))
        self._pops.append(pop)
        return pop

    def addConnection(self, source: Population, destination: Population, defaultWeights: float, *args):
        """addConnection(src, dst, w, p) or addConnection(src, dst, w, wmin, wmax, p, seed)."""
        if len(args) == 1:
            (probability,) = args
            wmin, wmax, seed = 0.0, 1.0, REF_DEFAULT_SEED
        elif len(args) == 4:
            wmin, wmax, probability, seed = args
        else:
            raise TypeError("addConnection(src, dst, w, p) or (src, dst, w, wmin, wmax, p, seed)")
        d = max(1, round(REF_WINDOW_US / self.params.dt_us))
        return self.connect(source, destination, rule=capi.CONN_REF_BERNOULLI, weight=defaultWeights,
                            wmin=wmin, wmax=wmax, probability=probability, seed=seed, delay=(d, d))

    def connect(self, source: Population, destination: Population, *, rule: int, weight: float,
                probability: float = 0.0, degree: int = 0, wmin: float = 0.0, wmax: float = 1.0,
                delay=(1, 1), seed: int = REF_DEFAULT_SEED) -> Connection:
        """Any connection rule of the C ABI (NAER_CONN_*), delays in grid steps."""
        spec = capi.ConnSpecC()
        spec.rule = int(rule)
        spec.degree = int(degree)
        spec.probability = float(probability)
        spec.weight = float(weight)
        spec.wmin = float(wmin)
        spec.wmax = float(wmax)
        spec.delay_min, spec.delay_max = int(delay[0]), int(delay[1])
        spec.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        capi.call("naer_net_add_connection", self._h, source.id, destination.id, C.byref(spec))
        con = Connection(source, destination, weight, wmin, wmax, probability, int(seed), int(rule), int(degree),
                         int(delay[0]), int(delay[1]))
        self._conns.append(con)
        return con

    def connect_csr(self, source: Population, destination: Population, row_ptr, targets, weights,
                    delays) -> Connection:
        """Explicit connectivity: a CSR over the source population (row_ptr of
        size+1 entries), target indices within the destination population,
        weights and delays in grid steps."""
        rp = np.ascontiguousarray(row_ptr, dtype=np.uint64)
        tg = np.ascontiguousarray(targets, dtype=np.uint32)
        w = np.ascontiguousarray(weights, dtype=np.float32)
        d = np.ascontiguousarray(delays, dtype=np.uint8)
        if len(rp) != source.size + 1 or not (len(tg) == len(w) == len(d) == int(rp[-1])):
            raise ValueError("row_ptr needs size+1 entries and the synapse arrays row_ptr[-1] entries")
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        capi.call("naer_net_add_connection_csr", self._h, source.id, destination.id, p(rp), p(tg), p(w), p(d))
        con = Connection(source, destination, 0.0, 0.0, 0.0, 0.0, 0, capi.CONN_EXPLICIT, 0,
                         int(d.min()) if len(d) else 1, int(d.max()) if len(d) else 1)
        self._conns.append(con)
        return con

    def compile(self) -> None:
        capi.call("naer_net_compile", self._h)
        for p in self._pops:  # Network.cpp:283-285: final addresses
            b = C.c_uint32()
            capi.call("naer_net_population_base", self._h, p.id, C.byref(b))
            p.baseAddress = b.value
        self._compiled = True

    # -- simulation (Network.cpp:107-265)
    def steps_per_window(self) -> int:
        return max(1, round(REF_WINDOW_US / self.params.dt_us))

    def step(self) -> None:
        """One reference window (1500 µs) of grid steps, asynchronously."""
        capi.call("naer_net_step", self._h, self.steps_per_window())

    def run(self, nsteps: int) -> None:
        """nsteps grid steps, asynchronously."""
        if nsteps < 0:
            raise ValueError("nsteps must be >= 0")
        capi.call("naer_net_step", self._h, int(nsteps))

    def finish(self) -> None:
        capi.call("naer_net_finish", self._h)

    def autotune(self, trial_steps: int = 64) -> dict:
        """Picks the launch geometry by timing candidates on this network
        (each trial advances the simulation by trial_steps grid steps)."""
        t = capi.Tuning()
        capi.call("naer_net_autotune", self._h, int(trial_steps), C.byref(t))
        return {k: getattr(t, k) for k, _ in capi.Tuning._fields_ if k not in ("pad_", "graph_launches")}

    def set_tuning(self, blocks_per_sm: int = 0, launch_steps: int = 64, scatter_split: int = 0,
                   scatter_piece: int = 0, neuron_state: int = capi.STATE_AUTO,
                   step_kernel: int = capi.KERNEL_SPLIT, bins: int = 0) -> None:
        t = capi.Tuning(blocks_per_sm=blocks_per_sm, launch_steps=launch_steps, scatter_split=scatter_split,
                        scatter_piece=scatter_piece, neuron_state=neuron_state, step_kernel=step_kernel, bins=bins)
        capi.call("naer_net_set_tuning", self._h, C.byref(t))

    def get_tuning(self) -> dict:
        t = capi.Tuning()
        capi.call("naer_net_get_tuning", self._h, C.byref(t))
        return {k: getattr(t, k) for k, _ in capi.Tuning._fields_ if k != "pad_"}

    def getTime(self) -> int:
        t = C.c_uint64()
        capi.call("naer_net_get_time_us", self._h, C.byref(t))
        return t.value

    def getSynapses(self) -> int:
        s = C.c_uint64()
        capi.call("naer_net_get_synapses", self._h, C.byref(s))
        return s.value

    def getNeurons(self) -> int:
        n = C.c_uint32()
        capi.call("naer_net_get_neurons", self._h, C.byref(n))
        return n.value

    # -- readback
    def stats(self) -> dict:
        st = capi.Stats()
        capi.call("naer_net_get_stats", self._h, C.byref(st))
        return {k: getattr(st, k) for k, _ in capi.Stats._fields_}

    def read_spikes(self, first: int = 0, capacity: int | None = None):
        """(steps, ids) of recorded spikes, grouped by step, ascending address within a step."""
        if capacity is None:
            capacity = max(0, self.stats()["spikes"] - first)
        steps = np.empty(capacity, dtype=np.uint32)
        ids = np.empty(capacity, dtype=np.uint32)
        n = C.c_uint64()
        capi.call("naer_net_read_spikes", self._h, int(first), int(capacity), steps.ctypes.data_as(C.c_void_p),
                  ids.ctypes.data_as(C.c_void_p), C.byref(n))
        return steps[: n.value], ids[: n.value]

    def read_raster(self, out: np.ndarray, first: int = 0) -> int:
        """Raw {step, id} records into ``out`` (uint32, shape (cap, 2)); returns the count."""
        assert out.dtype == np.uint32 and out.ndim == 2 and out.shape[1] == 2 and out.flags.c_contiguous
        n = C.c_uint64()
        capi.call("naer_net_read_raster", self._h, int(first), out.shape[0], out.ctypes.data_as(C.c_void_p),
                  C.byref(n))
        return n.value

    def stream(self) -> int:
        """cudaStream_t of this network as an integer (for torch.cuda.ExternalStream)."""
        p = C.c_void_p()
        capi.call("naer_net_stream", self._h, C.byref(p))
        return p.value or 0

    def clear_spikes(self) -> None:
        capi.call("naer_net_clear_spikes", self._h)

    def read_state(self):
        n = self.getNeurons()
        v = np.empty(n, dtype=np.float32)
        r = np.empty(n, dtype=np.uint32)
        capi.call("naer_net_read_state", self._h, v.ctypes.data_as(C.c_void_p), r.ctypes.data_as(C.c_void_p))
        return v, r

    def write_state(self, v=None, refractory=None) -> None:
        vp = None
        rp = None
        if v is not None:
            v = np.ascontiguousarray(v, dtype=np.float32)
            vp = v.ctypes.data_as(C.c_void_p)
        if refractory is not None:
            refractory = np.ascontiguousarray(refractory, dtype=np.uint32)
            rp = refractory.ctypes.data_as(C.c_void_p)
        capi.call("naer_net_write_state", self._h, vp, rp)

    def read_csr(self):
        n = self.getNeurons()
        S = self.getSynapses()
        rp = np.empty(n + 1, dtype=np.uint64)
        tg = np.empty(S, dtype=np.uint32)
        w = np.empty(S, dtype=np.float32)
        d = np.empty(S, dtype=np.uint8)
        capi.call("naer_net_read_csr", self._h, rp.ctypes.data_as(C.c_void_p), tg.ctypes.data_as(C.c_void_p),
                  w.ctypes.data_as(C.c_void_p), d.ctypes.data_as(C.c_void_p))
        return rp, tg, w, d

    def checkpoint(self) -> bytes:
        """The network's whole simulation state between steps (blocks)."""
        n = C.c_uint64()
        capi.call("naer_net_checkpoint_size", self._h, C.byref(n))
        buf = C.create_string_buffer(n.value)
        capi.call("naer_net_checkpoint", self._h, buf, n.value)
        return buf.raw

    def restore(self, data: bytes) -> None:
        """Loads a checkpoint taken from a network of the same description."""
        buf = C.create_string_buffer(bytes(data), len(data))
        capi.call("naer_net_restore", self._h, buf, len(data))

    def set_profiling(self, on: bool) -> None:
        capi.call("naer_net_set_profiling", self._h, 1 if on else 0)

    def profile(self) -> dict:
        """Accumulated device time per kernel (ms) since profiling was enabled."""
        lif = C.c_double()
        sc = C.c_double()
        n = C.c_uint64()
        capi.call("naer_net_get_profile", self._h, C.byref(lif), C.byref(sc), C.byref(n))
        self.nop_time = lif.value / 1e3
        self.scatter_time = sc.value / 1e3
        ph = (C.c_double * 5)()
        capi.call("naer_net_get_phases", self._h, C.cast(ph, C.c_void_p))
        names = ["lif", "lif_wait", "scatter", "reserved", "scatter_wait"]
        dr, rk = C.c_double(), C.c_double()
        nl = C.c_uint64()
        capi.call("naer_net_get_launch_times", self._h, C.byref(dr), C.byref(rk), C.byref(nl))
        return {"lif_ms": lif.value, "scatter_ms": sc.value, "steps": n.value,
                "phases_ms": {k: ph[i] for i, k in enumerate(names)},
                "drive_kernel_ms": dr.value, "step_kernel_ms": rk.value, "step_kernel_launches": nl.value}
