"""Declarative network specification and the benchmark workloads.

A ``NetSpec`` lists populations and connections with every parameter the
C ABI takes, so one description builds the CUDA network (``build``) and
can be handed to any other consumer (the tests hand the same object to
the CPU oracle).  It plays the part of the reference's Brunel builders
(src/main.cpp:12-50) in declarative form.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

from . import _capi as capi
from .network import Network, NeuronType

STDP, NOP, POISSON = NeuronType.STDP, NeuronType.NOP, NeuronType.POISSON


@dataclass
class PopSpec:
    type: int
    size: int
    tau_m_ms: float = 20.0
    v_th: float = 20.0
    v_reset: float = 10.0
    t_ref_ms: float = 2.0
    v_init: float = 0.0
    rate_hz: float = 0.0          # POISSON populations
    drive_rate_hz: float = 0.0    # LIF populations: per-neuron Poisson drive
    drive_weight: float = 0.0
    drive_seed: int = 0


@dataclass
class ConnSpec:
    src: int
    dst: int
    rule: int
    weight: float
    probability: float = 0.0
    degree: int = 0
    wmin: float = 0.0
    wmax: float = 1.0
    dmin: int = 1
    dmax: int = 1
    seed: int = 1
    csr: tuple | None = None      # CONN_EXPLICIT: (row_ptr, targets, weights, delays) numpy arrays


@dataclass
class NetSpec:
    pops: list = field(default_factory=list)
    conns: list = field(default_factory=list)
    dt_us: int = 100
    deterministic: bool = False
    exact: bool = False           # exact-sum aggregation (fixed-point weights; deterministic at atomic speed)
    record: bool = True
    raster_capacity: int = 1 << 24
    poisson_seed: int = 0x15AC7EBD
    stdp_enabled: bool = False
    tau_plus_ms: float = 20.0
    tau_minus_ms: float = 20.0
    a_plus: float = 0.01
    a_minus: float = 0.0105
    w_max: float = 0.5
    stdp_history: int = 10
    name: str = ""

    def add_pop(self, type: int, size: int, **kw) -> int:
        self.pops.append(PopSpec(int(type), int(size), **kw))
        return len(self.pops) - 1

    def connect(self, src: int, dst: int, rule: int, weight: float, **kw) -> None:
        self.conns.append(ConnSpec(src, dst, int(rule), float(weight), **kw))

    def connect_csr(self, src: int, dst: int, row_ptr, targets, weights, delays) -> None:
        """Explicit synapses from population src to dst: a CSR over the
        source population, targets as indices within the destination."""
        import numpy as np
        arrs = (np.ascontiguousarray(row_ptr, dtype=np.uint64), np.ascontiguousarray(targets, dtype=np.uint32),
                np.ascontiguousarray(weights, dtype=np.float32), np.ascontiguousarray(delays, dtype=np.uint8))
        d = arrs[3]
        self.conns.append(ConnSpec(src, dst, capi.CONN_EXPLICIT, 0.0, dmin=int(d.min()) if len(d) else 1,
                                   dmax=int(d.max()) if len(d) else 1, csr=arrs))

    @property
    def neurons(self) -> int:
        return sum(p.size for p in self.pops)

    def with_(self, **kw) -> "NetSpec":
        return replace(self, **kw)


def build(spec: NetSpec, device: int = 0) -> Network:
    """Creates and compiles the CUDA network described by ``spec``."""
    net = describe(spec, device)
    try:
        net.compile()
    except Exception:
        net.close()
        raise
    return net


def describe(spec: NetSpec, device: int = -1) -> Network:
    """The uncompiled network of ``spec``.  With device -1 it is a
    description-only handle: the input of a batch or a server."""
    net = Network(
        device=device,
        dt_us=spec.dt_us,
        aggregation=(capi.AGG_EXACT if spec.exact else
                     capi.AGG_DETERMINISTIC if spec.deterministic else capi.AGG_ATOMIC),
        record_spikes=1 if spec.record else 0,
        raster_capacity=spec.raster_capacity,
        poisson_seed=spec.poisson_seed,
        stdp_enabled=1 if spec.stdp_enabled else 0,
        tau_plus_ms=spec.tau_plus_ms,
        tau_minus_ms=spec.tau_minus_ms,
        a_plus=spec.a_plus,
        a_minus=spec.a_minus,
        w_max=spec.w_max,
        stdp_history=spec.stdp_history,
    )
    try:
        pops = []
        for p in spec.pops:
            kw = dict(tau_m_ms=p.tau_m_ms, v_th=p.v_th, v_reset=p.v_reset, t_ref_ms=p.t_ref_ms, v_init=p.v_init,
                      rate_hz=p.rate_hz, drive_rate_hz=p.drive_rate_hz, drive_weight=p.drive_weight,
                      drive_seed=p.drive_seed)
            pops.append(net.addPopulation(NeuronType(p.type), p.size, **kw))
        for c in spec.conns:
            if c.csr is not None:
                net.connect_csr(pops[c.src], pops[c.dst], *c.csr)
                continue
            net.connect(pops[c.src], pops[c.dst], rule=c.rule, weight=c.weight, probability=c.probability,
                        degree=c.degree, wmin=c.wmin, wmax=c.wmax, delay=(c.dmin, c.dmax), seed=c.seed)
    except Exception:
        net.close()
        raise
    return net


# ---------------------------------------------------------------------------
# Workloads.  Potentials and weights in mV.  LIF: tau_m 20 ms, V_th 20 mV,
# V_reset 10 mV, t_ref 2 ms, dt 0.1 ms.  Values the workload text leaves
# open (drive weights) are fixed here and documented with their calibration.

W_E, W_I = 0.1, -0.5


def brunel_small(seed: int = 1, poisson_weight: float = W_E, steps_delay: int = 15) -> NetSpec:
    """1,000 LIF (800 E / 200 I), p = 0.02 recurrent (reference Bernoulli
    rule), w_E = +0.1 mV, w_I = -0.5 mV, delay 1.5 ms; 1,000 Poisson sources
    at 10 Hz with p = 0.1 onto every neuron.  ``poisson_weight`` 0.1 mV is the
    workload as stated (nearly silent); 1.0 mV is the driven variant."""
    s = NetSpec(name=f"brunel_small(w_P={poisson_weight})", poisson_seed=seed)
    P = s.add_pop(POISSON, 1000, rate_hz=10.0)
    E = s.add_pop(NOP, 800)
    I = s.add_pop(NOP, 200)
    R = capi.CONN_REF_BERNOULLI
    d = dict(dmin=steps_delay, dmax=steps_delay)
    s.connect(P, E, R, poisson_weight, probability=0.1, seed=seed * 7919 + 1, **d)
    s.connect(P, I, R, poisson_weight, probability=0.1, seed=seed * 7919 + 2, **d)
    s.connect(E, E, R, W_E, probability=0.02, seed=seed * 7919 + 3, **d)
    s.connect(E, I, R, W_E, probability=0.02, seed=seed * 7919 + 4, **d)
    s.connect(I, E, R, W_I, probability=0.02, seed=seed * 7919 + 5, **d)
    s.connect(I, I, R, W_I, probability=0.02, seed=seed * 7919 + 6, **d)
    return s


def plastic_indegree(n: int = 100_000, k: int = 1000, seed: int = 1, drive_rate_hz: float = 10.0,
                     drive_weight: float = 20.5, stdp: bool = True) -> NetSpec:
    """N LIF (80 % STDP-excitatory, 20 % inhibitory), fixed in-degree k
    (0.8 k from E, 0.2 k from I), delays U{1..20} steps, a per-neuron 10 Hz
    Poisson drive, pair-based STDP on E->E (tau 20 ms, A+ 0.01, A- 0.0105,
    w in [0, 0.5] mV).  The drive weight (20.5 mV) is calibrated on the
    oracle for ~5 Hz mean firing."""
    ne = n * 4 // 5
    s = NetSpec(name=f"plastic_indegree(N={n},K={k})", stdp_enabled=stdp, poisson_seed=seed)
    E = s.add_pop(STDP, ne, drive_rate_hz=drive_rate_hz, drive_weight=drive_weight, drive_seed=seed * 31 + 1)
    I = s.add_pop(NOP, n - ne, drive_rate_hz=drive_rate_hz, drive_weight=drive_weight, drive_seed=seed * 31 + 2)
    R = capi.CONN_FIXED_INDEGREE
    ke, ki = k * 4 // 5, k - k * 4 // 5
    d = dict(dmin=1, dmax=20)
    s.connect(E, E, R, W_E, degree=ke, seed=seed * 7919 + 11, **d)
    s.connect(E, I, R, W_E, degree=ke, seed=seed * 7919 + 12, **d)
    s.connect(I, E, R, W_I, degree=ki, seed=seed * 7919 + 13, **d)
    s.connect(I, I, R, W_I, degree=ki, seed=seed * 7919 + 14, **d)
    return s


def scatter_outdegree(n: int = 1_000_000, k: int = 1000, seed: int = 1, drive_rate_hz: float = 20.0,
                      drive_weight: float = 20.3) -> NetSpec:
    """N LIF (80/20), fixed out-degree k with targets uniform over all
    neurons, delays U{1..16} steps, no STDP, per-neuron Poisson drive at
    20 Hz; the drive weight (20.3 mV) is calibrated on the oracle at N = 20k
    (same in-degree statistics) for ~10 Hz mean firing."""
    ne = n * 4 // 5
    s = NetSpec(name=f"scatter_outdegree(N={n},K={k})", poisson_seed=seed)
    E = s.add_pop(NOP, ne, drive_rate_hz=drive_rate_hz, drive_weight=drive_weight, drive_seed=seed * 31 + 1)
    I = s.add_pop(NOP, n - ne, drive_rate_hz=drive_rate_hz, drive_weight=drive_weight, drive_seed=seed * 31 + 2)
    return _all_targets(s, E, I, k, seed)


def hub_readout(n: int = 200_000, k: int = 100, readout: int = 64, seed: int = 1) -> NetSpec:
    """A convergent network: N LIF (80/20) as in scatter_outdegree (fixed
    out-degree k over all neurons, delays 1-16 steps, 20 Hz drive) plus a
    readout population of `readout` LIF neurons that every neuron projects
    to with delay 1 (weight 0.01 mV).  Each step's events to the readout
    land on only `readout` ring cells: the case where shared-memory binning
    of the ring reductions pays."""
    s = scatter_outdegree(n=n, k=k, seed=seed)
    s.name = f"hub_readout(N={n},K={k},readout={readout})"
    R = s.add_pop(NOP, readout)
    for src in (0, 1):
        s.connect(src, R, capi.CONN_FIXED_OUTDEGREE, 0.01, degree=readout, dmin=1, dmax=1, seed=seed * 7919 + 31 + src)
    return s


def _all_targets(s: NetSpec, E: int, I: int, k: int, seed: int) -> NetSpec:
    # out-degree k over all neurons: split each source's k draws between the
    # E and I target populations in proportion to their sizes
    R = capi.CONN_FIXED_OUTDEGREE
    ne, ni = s.pops[E].size, s.pops[I].size
    ke = round(k * ne / (ne + ni))
    ki = k - ke
    d = dict(dmin=1, dmax=16)
    s.connect(E, E, R, W_E, degree=ke, seed=seed * 7919 + 21, **d)
    s.connect(E, I, R, W_E, degree=ki, seed=seed * 7919 + 22, **d)
    s.connect(I, E, R, W_I, degree=ke, seed=seed * 7919 + 23, **d)
    s.connect(I, I, R, W_I, degree=ki, seed=seed * 7919 + 24, **d)
    return s


def batch_members(count: int = 256, seed: int = 1, n_range=(2000, 50_000), k_range=(100, 1000),
                  rate_range=(5.0, 30.0), stdp_fraction: float = 0.5) -> list:
    """Independent networks of uneven sizes for the batched form: neuron
    counts log-uniform in n_range, in-degree uniform in k_range (80/20
    E/I), each with its own seed, a per-neuron Poisson drive rate uniform in
    rate_range and STDP on for a stdp_fraction of them (the plastic_indegree
    network family)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        k = int(rng.integers(k_range[0], k_range[1] + 1))
        rate = float(rng.uniform(*rate_range))
        stdp = bool(rng.random() < stdp_fraction)
        m = plastic_indegree(n=n, k=k, seed=seed * 100_003 + i, drive_rate_hz=rate, stdp=stdp)
        m.name = f"member{i}(N={n},K={k},rate={rate:.1f},stdp={int(stdp)})"
        out.append(m)
    return out


def served_jobs(count: int = 2000, seed: int = 1, arrivals_per_s: float = 50.0, n_range=(1000, 200_000),
                k_range=(100, 1000), duration_ms=(100.0, 2000.0), stdp_fraction: float = 0.3,
                rate_hz: float = 10.0, dt_us: int = 100) -> list:
    """Simulation jobs for the served form: (arrival time in s, NetSpec,
    duration in grid steps), Poisson arrivals at arrivals_per_s, neuron
    counts log-uniform in n_range, in-degree uniform in k_range, durations
    uniform in duration_ms, STDP on for a stdp_fraction of the jobs."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / arrivals_per_s))
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        k = int(rng.integers(k_range[0], k_range[1] + 1))
        dur = float(rng.uniform(*duration_ms))
        stdp = bool(rng.random() < stdp_fraction)
        m = plastic_indegree(n=n, k=k, seed=seed * 200_003 + i, drive_rate_hz=rate_hz, stdp=stdp)
        m.name = f"job{i}(N={n},K={k},stdp={int(stdp)})"
        out.append((t, m, max(1, int(round(dur * 1000.0 / dt_us)))))
    return out
