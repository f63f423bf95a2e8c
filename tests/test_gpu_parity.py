"""Parity of the CUDA path (through the C ABI) with the oracle.

Bit-exact: connectivity arrays, rasters, membrane potentials, refractory
counters and STDP weights in deterministic aggregation mode.  Atomic mode:
firing statistics within the stated tolerance.
"""
import numpy as np
import pytest

from naer_b200 import _capi as capi
from naer_b200 import spec as S
from naer_b200.network import NeuronType

from nets import integer_weight_net, mixed_rules, reference_brunel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def O(oracle_mod, lib):
    return oracle_mod


def assert_csr_equal(net, o):
    rp, tg, w, d = net.read_csr()
    orp, otg, ow, od = o.csr()
    assert np.array_equal(rp, orp)
    assert np.array_equal(tg, otg)
    assert np.array_equal(w.view(np.uint32), ow.view(np.uint32))
    assert np.array_equal(d, od)


@pytest.mark.parametrize("rule", [capi.CONN_REF_BERNOULLI, capi.CONN_FIXED_INDEGREE, capi.CONN_FIXED_OUTDEGREE])
def test_connectivity_bit_exact(O, rule):
    s = mixed_rules(rule)
    with S.build(s) as net:
        o = O.OracleNet(s)
        assert net.getSynapses() == o.S and net.getNeurons() == o.n
        assert_csr_equal(net, o)


def test_connectivity_reference_brunel(O):
    s = reference_brunel(2e5)
    with S.build(s) as net:
        o = O.OracleNet(s)
        assert net.getSynapses() == o.S
        assert_csr_equal(net, o)


def test_connectivity_large_rows(O):
    """Fixed out-degree rows of 1,000 (the scatter workload's row length)
    and fixed in-degree with multapses."""
    s = S.scatter_outdegree(n=3000, k=1000)
    with S.build(s) as net:
        assert_csr_equal(net, O.OracleNet(s))
    s = S.plastic_indegree(n=2000, k=300)
    with S.build(s) as net:
        assert_csr_equal(net, O.OracleNet(s))


def run_both(O, s, steps, threads=0):
    net = S.build(s.with_(deterministic=True))
    o = O.OracleNet(s, deterministic=True, threads=threads)
    net.run(steps)
    net.finish()
    o.run(steps)
    return net, o


def assert_same_run(net, o):
    st, ids = net.read_spikes()
    ost, oids = o.spikes()
    assert len(ids) == len(oids), (len(ids), len(oids))
    assert np.array_equal(st, ost) and np.array_equal(ids, oids)
    v, r = net.read_state()
    ov, orr = o.state()
    assert np.array_equal(v.view(np.uint32), ov.view(np.uint32))
    assert np.array_equal(r, orr)
    assert net.stats()["events"] == o.events
    return len(ids)


def test_poisson_population_raster(O):
    """POISSON populations alone: the reference generator's exact stream."""
    s = S.NetSpec()
    s.add_pop(S.POISSON, 5000, rate_hz=40.0)
    s.add_pop(S.POISSON, 3000, rate_hz=400.0)
    net, o = run_both(O, s, 3000)
    with net:
        n = assert_same_run(net, o)
        assert n > 5000 * 40 * 0.3 * 0.8


def test_brunel_small_driven_bit_exact(O):
    """The plain CPU-runnable workload (driven variant), first 1,000 steps."""
    net, o = run_both(O, S.brunel_small(poisson_weight=1.0), 1000)
    with net:
        n = assert_same_run(net, o)
        assert n > 1000


def test_brunel_small_as_stated(O):
    net, o = run_both(O, S.brunel_small(poisson_weight=0.1), 1000)
    with net:
        assert_same_run(net, o)


def test_reference_brunel_bit_exact(O):
    net, o = run_both(O, reference_brunel(2e5), 1000)
    with net:
        assert assert_same_run(net, o) > 0


def test_fixed_outdegree_bit_exact(O):
    net, o = run_both(O, S.scatter_outdegree(n=4000, k=400, drive_weight=24.0), 1000)
    with net:
        assert assert_same_run(net, o) > 1000


def test_stdp_bit_exact(O):
    """Plastic E->E with lazy LTP/LTD fused into the scatter."""
    s = S.plastic_indegree(n=2000, k=200, drive_weight=21.0)
    net, o = run_both(O, s, 1000)
    with net:
        assert assert_same_run(net, o) > 500
        _, _, w, _ = net.read_csr()
        ow = o.weights()
        assert np.array_equal(w.view(np.uint32), ow.view(np.uint32))
        _, _, w0, _ = O.OracleNet(s).csr()
        assert not np.array_equal(w0, ow)  # plasticity acted
        assert net.stats()["stdp_hist_overflow"] == o.hist_overflow


def test_mixed_rules_bit_exact(O):
    for rule in (capi.CONN_REF_BERNOULLI, capi.CONN_FIXED_INDEGREE, capi.CONN_FIXED_OUTDEGREE):
        s = mixed_rules(rule).with_(stdp_enabled=True)
        for p in s.pops[1:]:
            p.drive_rate_hz, p.drive_weight, p.drive_seed = 300.0, 12.0, 3
        net, o = run_both(O, s, 800)
        with net:
            assert_same_run(net, o)


def rates_and_cv(steps, ids, n, t_steps, dt_s=1e-4):
    rate = np.bincount(ids, minlength=n) / (t_steps * dt_s)
    order = np.lexsort((steps, ids))
    s, i = steps[order].astype(np.int64), ids[order]
    same = i[1:] == i[:-1]
    isi = np.diff(s)[same]
    owner = i[1:][same]
    cvs = []
    for k in np.unique(owner):
        x = isi[owner == k]
        if len(x) >= 5:
            cvs.append(x.std() / x.mean())
    return rate, float(np.mean(cvs))


def test_atomic_mode_statistics(O):
    """Atomic aggregation reorders float sums, so rasters diverge; per
    population rate and mean ISI CV stay within 2 % of the oracle over 2 s."""
    s = S.brunel_small(poisson_weight=1.0)
    steps = 20000
    with S.build(s) as net:
        net.run(steps)
        net.finish()
        st, ids = net.read_spikes()
    o = O.OracleNet(s, deterministic=True)
    o.run(steps)
    ost, oids = o.spikes()
    base_E, base_I = 0, 800  # NOP E then NOP I, POISSON last
    for lo, hi in [(base_E, 800), (base_I, 1000)]:
        m, om = (ids >= lo) & (ids < hi), (oids >= lo) & (oids < hi)
        r, cv = rates_and_cv(st[m], ids[m] - lo, hi - lo, steps)
        orr, ocv = rates_and_cv(ost[om], oids[om] - lo, hi - lo, steps)
        assert r.mean() == pytest.approx(orr.mean(), rel=0.02)
        assert cv == pytest.approx(ocv, rel=0.02)


def test_reference_api_flow(lib):
    """The reference's call sequence (src/main.cpp:94-126) and its errors."""
    from naer_b200 import Network, NaerError
    net = Network()
    P = net.addPopulation(NeuronType.POISSON, 400, rate_hz=20.0)
    E = net.addPopulation(NeuronType.NOP, 300, v_th=0.02)
    I = net.addPopulation(NeuronType.NOP, 100, v_th=0.02)
    S2 = net.addPopulation(NeuronType.STDP, 50, v_th=0.02)
    assert (P.baseAddress, E.baseAddress, I.baseAddress, S2.baseAddress) == (0, 0, 300, 0)  # type-local
    net.addConnection(P, E, 0.001, 0.1)
    net.addConnection(E, I, 0.0, 0.0, 0.001, 0.1, 1234)
    with pytest.raises(NaerError):
        net.addConnection(E, P, 0.001, 0.1)  # POISSON cannot receive: reported at compile
        net.compile()
    net.close()

    net = Network()
    P = net.addPopulation(NeuronType.POISSON, 400)
    E = net.addPopulation(NeuronType.NOP, 300, v_th=0.02)
    S2 = net.addPopulation(NeuronType.STDP, 50, v_th=0.02)
    net.addConnection(P, E, 0.001, 0.1)
    net.addConnection(E, S2, 0.001, 0.1)
    net.compile()
    # STDP, then NOP, then POISSON (Network.cpp:271-285)
    assert (S2.baseAddress, E.baseAddress, P.baseAddress) == (0, 50, 350)
    assert net.getNeurons() == 750 and net.getSynapses() > 0
    while net.getTime() < 30_000:
        net.step()
    net.finish()
    assert net.getTime() == 30_000
    assert net.stats()["step"] == 300
    with pytest.raises(NaerError):
        net.addPopulation(NeuronType.NOP, 5)
    net.close()


def test_state_roundtrip(lib):
    s = S.brunel_small(poisson_weight=1.0)
    with S.build(s) as net:
        net.run(50)
        v, r = net.read_state()
        v2 = v.copy()
        v2[:100] = 5.0
        net.write_state(v2, r)
        v3, r3 = net.read_state()
        assert np.array_equal(v3, v2) and np.array_equal(r3, r)


def test_atomic_persistent_path_exact_with_integer_weights(O):
    """The persistent atomic-mode kernel (the benchmarked path) against the
    oracle, bit for bit, where reduction order cannot matter."""
    s = integer_weight_net()
    with S.build(s) as net:
        l0 = net.stats()["kernel_launches"]
        for chunk in (1, 7, 300, 692):  # several launches of the persistent kernel
            net.run(chunk)
        net.finish()
        assert net.stats()["kernel_launches"] > l0
        o = O.OracleNet(s, deterministic=True)
        o.run(1000)
        n = assert_same_run(net, o)
        assert n > 2000


# Membrane potentials and STDP weights of the CUDA runs against an FP64
# re-integration (the oracle, double arithmetic, exact exp) driven by the
# run's own raster: |x32 - x64| <= 1e-5 * max(|x64|, floor), floor 1 mV for
# V and 1e-3 * w_max for weights.
FP64_RTOL = 1e-5


def assert_fp64(x32, x64, floor):
    x64 = np.asarray(x64, dtype=np.float64)
    err = np.abs(np.asarray(x32, dtype=np.float64) - x64) / np.maximum(np.abs(x64), floor)
    assert err.max() <= FP64_RTOL, err.max()


@pytest.mark.parametrize("deterministic", [True, False])
def test_fp64_reintegration_membrane_and_weights(O, deterministic):
    s = S.plastic_indegree(n=2000, k=200, drive_weight=21.0).with_(deterministic=deterministic)
    steps = 1500
    with S.build(s) as net:
        net.run(steps)
        net.finish()
        st, ids = net.read_spikes()
        v, _ = net.read_state()
        _, _, w, _ = net.read_csr()
    assert len(ids) > 1000
    v64, w64, _ = O.OracleNet(s).reintegrate_fp64(st, ids, steps)
    assert_fp64(v, v64, 1.0)
    assert_fp64(w, w64, 1e-3 * s.w_max)


def test_fp64_reintegration_atomic_brunel(O):
    """Atomic aggregation (unordered fp32 sums), 2 s of the driven workload."""
    s = S.brunel_small(poisson_weight=1.0)
    steps = 20000
    with S.build(s) as net:
        net.run(steps)
        net.finish()
        st, ids = net.read_spikes()
        v, _ = net.read_state()
    v64, _, _ = O.OracleNet(s).reintegrate_fp64(st, ids, steps)
    assert_fp64(v, v64, 1.0)


def test_edge_long_rows_long_delays_other_dt(O):
    """Rows longer than warps-per-spike x piece (the scatter loops over the
    row), delays up to 254 steps (255 ring slots), a 50 us grid step, a
    POISSON population of one neuron and populations whose sizes are not
    multiples of 4."""
    s = S.NetSpec(dt_us=50, poisson_seed=9)
    P = s.add_pop(S.POISSON, 1, rate_hz=2000.0)
    E = s.add_pop(S.NOP, 3001, drive_rate_hz=30.0, drive_weight=21.0, drive_seed=5)
    I = s.add_pop(S.NOP, 7, drive_rate_hz=30.0, drive_weight=21.0, drive_seed=6)
    s.connect(P, E, capi.CONN_FIXED_OUTDEGREE, 2.0, degree=6000, dmin=1, dmax=3, seed=21)
    s.connect(E, E, capi.CONN_FIXED_OUTDEGREE, 1.0, degree=40, dmin=1, dmax=254, seed=22)
    s.connect(I, E, capi.CONN_FIXED_OUTDEGREE, -2.0, degree=5000, dmin=200, dmax=254, seed=23)
    s.connect(E, I, capi.CONN_REF_BERNOULLI, 0.5, probability=0.5, dmin=1, dmax=1, seed=24)
    net, o = run_both(O, s, 1200)
    with net:
        assert_same_run(net, o)
        assert_csr_equal(net, o)
    # the atomic persistent kernel on the same integer-weight network
    with S.build(s) as net:
        net.run(1200)
        net.finish()
        o2 = O.OracleNet(s, deterministic=True)
        o2.run(1200)
        assert assert_same_run(net, o2) > 100


def test_silent_and_empty_networks(O):
    """No connections; a network whose only population never fires."""
    s = S.NetSpec()
    s.add_pop(S.NOP, 5, drive_rate_hz=0.0)
    net, o = run_both(O, s, 50)
    with net:
        assert assert_same_run(net, o) == 0
        assert net.getSynapses() == 0
    s2 = S.NetSpec()
    s2.add_pop(S.POISSON, 3, rate_hz=0.0)
    s2.add_pop(S.NOP, 9)
    s2.connect(0, 1, capi.CONN_FIXED_OUTDEGREE, 1.0, degree=2)
    with S.build(s2) as net:
        net.run(100)
        net.finish()
        assert net.stats()["spikes"] == 0 and net.stats()["events"] == 0


def explicit_net(seed=9):
    """POISSON -> E by a rule, explicit random E -> I and I -> E synapses
    (multapses, delays 1-7, weights of both signs), deterministic mode."""
    rng = np.random.default_rng(seed)
    s = S.NetSpec(poisson_seed=seed, deterministic=True)
    P = s.add_pop(S.POISSON, 500, rate_hz=40.0)
    E = s.add_pop(S.NOP, 900, drive_rate_hz=20.0, drive_weight=18.0, drive_seed=4)
    I = s.add_pop(S.NOP, 230)
    s.connect(P, E, capi.CONN_FIXED_OUTDEGREE, 3.0, degree=40, dmin=1, dmax=3, seed=seed)
    for src, n_src, dst, n_dst, sign in [(E, 900, I, 230, 1.0), (I, 230, E, 900, -1.0)]:
        lens = rng.integers(0, 60, n_src)
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
        nnz = int(rp[-1])
        s.connect_csr(src, dst, rp, rng.integers(0, n_dst, nnz), sign * rng.uniform(0.5, 4.0, nnz),
                      rng.integers(1, 8, nnz))
    return s


def test_explicit_connectivity_bit_exact(O):
    """Connectivity uploaded by the caller (naer_net_add_connection_csr)
    next to a generated one: the CSR, raster and state match the oracle."""
    s = explicit_net()
    net, o = run_both(O, s, 1500)
    with net:
        assert net.getSynapses() == o.S
        assert_csr_equal(net, o)
        assert assert_same_run(net, o) > 500


def test_explicit_connectivity_rejects_bad_input(lib):
    from naer_b200 import Network, NaerError
    with Network() as net:
        a = net.addPopulation(NeuronType.NOP, 4)
        b = net.addPopulation(NeuronType.NOP, 3)
        with pytest.raises(NaerError, match="outside the destination"):
            net.connect_csr(a, b, [0, 1, 1, 1, 1], [3], [1.0], [1])
        with pytest.raises(NaerError, match="delays"):
            net.connect_csr(a, b, [0, 1, 1, 1, 1], [0], [1.0], [0])
        with pytest.raises(NaerError, match="decrease"):
            net.connect_csr(a, b, [0, 2, 1, 1, 2], [0, 1], [1.0, 1.0], [1, 1])
