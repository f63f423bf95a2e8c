"""Parity on the launch geometries the benchmark runs, through the C ABI.

The 1M-neuron benchmark gives every persistent block three to five LIF
chunks (978 chunks over 296 blocks), which goes through the kernel's batched
multi-chunk loop; served sets past the shared-memory capacity run the
variant that keeps neuron state in global memory.  Small test networks never
reach either, so these tests force them: a 700k-neuron network at one block
per SM (684 chunks over 148 blocks: four or five per block, two batches of
the loop), and the same network with neuron state in global memory.
Integer weights make every ring sum exact in fp32, so the atomic kernel
must match the oracle bit for bit whatever the reduction order.

The configuration-shaped runs check the full-size networks themselves:
1M LIF / 1e9 synapses (the roofline workload) for per-population rate and
pooled ISI CV within 2 % of the oracle, and 100k LIF / 1e8 synapses with
STDP (the plastic workload) against the FP64 re-integration within 1e-5.
"""
import numpy as np
import pytest

from naer_b200 import _capi as capi
from naer_b200 import spec as S

from nets import integer_weight_net

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def O(oracle_mod, lib):
    return oracle_mod


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


BIG = dict(n=700_000, k=24, seed=5)
BIG_STEPS = 600


@pytest.fixture(scope="module")
def big_oracle(O):
    o = O.OracleNet(integer_weight_net(**BIG), deterministic=True)
    o.run(BIG_STEPS)
    yield o
    o.close()


@pytest.mark.parametrize("state", [capi.STATE_SHARED, capi.STATE_GLOBAL])
def test_multi_chunk_blocks_exact(big_oracle, state):
    """Four or five chunks per persistent block (one block per SM): shared
    state runs the batched prefetch / clear / update loop twice per step;
    global state runs the chunk loop of the other kernel variant."""
    s = integer_weight_net(**BIG)
    with S.build(s) as net:
        net.set_tuning(blocks_per_sm=1, neuron_state=state)
        t = net.get_tuning()
        assert t["blocks_per_sm"] == 1 and t["neuron_state"] == state
        for chunk in (64, 1, 200, 335):  # several persistent launches, one of one step
            net.run(chunk)
        net.finish()
        assert net.stats()["step"] == BIG_STEPS
        n = assert_same_run(net, big_oracle)
        assert n > 100_000


def test_default_geometry_big_exact(big_oracle):
    """The same network at the default geometry (most blocks per SM)."""
    with S.build(integer_weight_net(**BIG)) as net:
        net.run(BIG_STEPS)
        net.finish()
        assert_same_run(net, big_oracle)


def pooled_rate_cv(steps, ids, lo, hi, t_steps, dt_s=1e-4):
    m = (ids >= lo) & (ids < hi)
    s, i = steps[m].astype(np.int64), ids[m]
    rate = len(i) / ((hi - lo) * t_steps * dt_s)
    order = np.lexsort((s, i))
    s, i = s[order], i[order]
    same = i[1:] == i[:-1]
    isi = np.diff(s)[same].astype(np.float64)
    return rate, isi.std() / isi.mean(), len(isi)


def test_roofline_workload_statistics(O):
    """1M LIF (80/20), fixed out-degree 1,000 (1e9 synapses), delays 1-16,
    20 Hz drive, atomic aggregation at the benchmark's geometry: per
    population rate and pooled ISI CV within 2 % of the oracle over 3,000
    steps (the runs diverge chaotically, so rasters are not compared)."""
    s = S.scatter_outdegree()
    s.raster_capacity = 1 << 24
    steps = 3000
    with S.build(s) as net:
        assert net.getSynapses() == 1_000_000_000
        net.run(steps)
        net.finish()
        st, ids = net.read_spikes()
        ev = net.stats()["events"]
    o = O.OracleNet(s, deterministic=True)
    o.run(steps)
    ost, oids = o.spikes()
    oev = o.events
    o.close()
    assert ev == pytest.approx(oev, rel=0.02)
    for lo, hi in [(0, 800_000), (800_000, 1_000_000)]:
        r, cv, n = pooled_rate_cv(st, ids, lo, hi, steps)
        orr, ocv, on = pooled_rate_cv(ost, oids, lo, hi, steps)
        assert n > 10_000 and on > 10_000
        assert 5.0 < r < 20.0
        assert r == pytest.approx(orr, rel=0.02)
        assert cv == pytest.approx(ocv, rel=0.02)


def test_roofline_workload_deterministic_exact(O):
    """The roofline workload itself (1M LIF, 1e9 synapses) in deterministic
    aggregation: raster, membrane potentials, refractory counters and event
    count equal the oracle's bit for bit over 300 grid steps (about 3e8
    events, every per-cell fold in canonical order)."""
    s = S.scatter_outdegree().with_(deterministic=True)
    s.raster_capacity = 1 << 22
    steps = 300
    with S.build(s) as net:
        net.run(steps)
        net.finish()
        o = O.OracleNet(s, deterministic=True)
        o.run(steps)
        n = assert_same_run(net, o)
        o.close()
    assert n > 10_000


def test_plastic_workload_fp64(O):
    """100k LIF, fixed in-degree 1,000 (1e8 synapses), delays 1-20, pair
    STDP on E->E, 1,000 steps: membrane potentials and weights within 1e-5
    of the FP64 re-integration of the same spike inputs, with lazy LTP over
    every post spike (no history limit)."""
    s = S.plastic_indegree(n=100_000, k=1000)
    steps = 1000
    with S.build(s) as net:
        net.run(steps)
        net.finish()
        st, ids = net.read_spikes()
        v, _ = net.read_state()
        _, _, w, _ = net.read_csr()
    assert len(ids) > 10_000
    o = O.OracleNet(s)
    # against the pair rule itself: every post spike since the source's last
    # spike, no history limit (the limit drops no pair on this run)
    v64, w64, _, lost = o.reintegrate_fp64_uncapped(st, ids, steps)
    o.close()
    assert lost == 0
    for x32, x64, floor in [(v, v64, 1.0), (w, w64, 1e-3 * s.w_max)]:
        x64 = np.asarray(x64, dtype=np.float64)
        err = np.abs(np.asarray(x32, dtype=np.float64) - x64) / np.maximum(np.abs(x64), floor)
        assert err.max() <= 1e-5, err.max()


@pytest.mark.parametrize("bins", [64, 2048])
def test_binned_aggregation_exact(O, bins):
    """Shared-memory binning of the ring reductions: integer weights make
    every fold order give the same sums, so runs with a small (overflowing)
    and a large table match the oracle bit for bit, on a network whose
    readout population concentrates each step's events on a few cells."""
    s = integer_weight_net(n=20000, k=60, seed=6)
    R = s.add_pop(S.NOP, 32, drive_rate_hz=0.0)
    for src in (0, 1):
        s.connect(src, R, capi.CONN_FIXED_OUTDEGREE, 1.0, degree=16, dmin=1, dmax=2, seed=70 + src)
    o = O.OracleNet(s, deterministic=True)
    o.run(700)
    with S.build(s) as net:
        net.set_tuning(bins=bins)
        assert net.get_tuning()["bins"] == bins
        net.run(300)
        net.run(400)
        net.finish()
        assert assert_same_run(net, o) > 1000
    o.close()


def test_bins_validation(lib):
    from naer_b200 import NaerError
    with S.build(integer_weight_net(n=2000, k=50)) as net:
        for bad in (3, 32, 100, 16384):
            with pytest.raises(NaerError, match="bins"):
                net.set_tuning(bins=bad)
