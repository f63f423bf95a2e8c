"""Exact-sum aggregation (NAER_AGG_EXACT) on the GPU.

Every delivered weight is rounded to the network's fixed-point grid 2^-S and
the ring holds int32 sums, so the persistent atomic kernel gives the same
bits whatever the order of its reductions.  The oracle restates the same
quantization (its mode 2), so rasters, membrane potentials, refractory
counters, event counts and STDP weights must match it bit for bit on
non-integer weights, with POISSON multiplicities, with STDP and on the
multi-chunk geometry; two runs, and a batch member and its run alone, must
give identical rasters; and the result stays within 1e-5 of an FP64
integration of the same spike inputs.
"""
import numpy as np
import pytest

from naer_b200 import NaerError
from naer_b200 import _capi as capi
from naer_b200 import spec as S
from naer_b200.forms import Batch

from nets import integer_weight_net

pytestmark = pytest.mark.gpu


def run_gpu(spec, steps, tuning=None, chunks=None):
    with S.build(spec) as net:
        if tuning:
            net.set_tuning(**tuning)
        for c in (chunks or [steps]):
            net.run(c)
        net.finish()
        st, ids = net.read_spikes()
        v, r = net.read_state()
        ev = net.stats()["events"]
        w = net.read_csr()[2] if spec.stdp_enabled else None
    return st, ids, v, r, ev, w


def assert_matches_oracle(O, spec, steps, **kw):
    st, ids, v, r, ev, w = run_gpu(spec, steps, **kw)
    o = O.OracleNet(spec)
    assert o.exact_shift() > 0
    o.run(steps)
    ost, oids = o.spikes()
    ov, orr = o.state()
    oev = o.events
    ow = o.weights() if spec.stdp_enabled else None
    o.close()
    assert len(ids) > 100
    assert np.array_equal(st, ost) and np.array_equal(ids, oids)
    assert np.array_equal(v.view(np.uint32), ov.view(np.uint32)) and np.array_equal(r, orr)
    assert ev == oev
    if w is not None:
        assert np.array_equal(w.view(np.uint32), ow.view(np.uint32))
    return st, ids


def poisson_multiplicity_net():
    s = integer_weight_net(n=20000, k=80, seed=9)
    for c in s.conns:
        c.weight = c.weight * 0.137  # not integers: the float sums would depend on the order
    P = s.add_pop(S.POISSON, 3000, rate_hz=2000.0)
    s.connect(P, 0, capi.CONN_FIXED_OUTDEGREE, 0.29, degree=40, dmin=1, dmax=4, seed=77)
    s.connect(P, 1, capi.CONN_FIXED_OUTDEGREE, 0.11, degree=10, dmin=1, dmax=2, seed=78)
    return s


@pytest.mark.parametrize("make, steps", [
    (lambda: S.brunel_small(poisson_weight=1.0), 2000),
    (poisson_multiplicity_net, 600),
    (lambda: S.plastic_indegree(n=3000, k=200, drive_weight=21.0), 1500),
    (lambda: S.scatter_outdegree(n=50_000, k=200), 800),
])
def test_exact_matches_oracle(oracle_mod, lib, make, steps):
    assert_matches_oracle(oracle_mod, make().with_(exact=True), steps)


def test_exact_multi_chunk_geometry(oracle_mod, lib):
    """Several LIF chunks per block, neuron state in shared and in global
    memory, launches of assorted lengths."""
    s = S.scatter_outdegree(n=300_000, k=40).with_(exact=True)
    for state in (capi.STATE_SHARED, capi.STATE_GLOBAL):
        assert_matches_oracle(oracle_mod, s, 400, tuning=dict(blocks_per_sm=1, neuron_state=state),
                              chunks=[64, 1, 200, 135])


@pytest.mark.parametrize("make, steps", [
    (poisson_multiplicity_net, 600),
    (lambda: S.plastic_indegree(n=3000, k=200, drive_weight=21.0), 1500),
])
def test_exact_two_barrier_kernel_matches_oracle(oracle_mod, lib, make, steps):
    """The two-barrier kernel (k_run, the served form's default) reduces the
    same fixed-point integers: the same bits as the oracle."""
    assert_matches_oracle(oracle_mod, make().with_(exact=True), steps,
                          tuning=dict(step_kernel=capi.KERNEL_TWO_BARRIER), chunks=[64, 1, 300, steps - 365])


def test_exact_two_barrier_multi_chunk_geometry(oracle_mod, lib):
    s = S.scatter_outdegree(n=300_000, k=40).with_(exact=True)
    for state in (capi.STATE_SHARED, capi.STATE_GLOBAL):
        assert_matches_oracle(oracle_mod, s, 300, tuning=dict(blocks_per_sm=1, neuron_state=state,
                                                             step_kernel=capi.KERNEL_TWO_BARRIER),
                              chunks=[64, 1, 235])


def test_exact_repeats_and_batch_members(lib):
    """Two runs give the same bits, and batch members their runs alone."""
    specs = [S.scatter_outdegree(n=n, k=150, seed=sd).with_(exact=True) for n, sd in [(40_000, 3), (23_000, 4)]]
    alone = [run_gpu(s, 700) for s in specs]
    again = run_gpu(specs[0], 700)
    assert all(np.array_equal(a, b) for a, b in zip(alone[0][:3], again[:3]))
    with Batch(specs, exact=True).compile() as b:
        b.run(700)
        b.finish()
        sp = b.read_spikes()
        for m, a in enumerate(alone):
            st, ids = b.member_spikes(m, sp)
            assert len(ids) > 1000
            assert np.array_equal(st, a[0]) and np.array_equal(ids, a[1]), m


def test_exact_within_fp64(oracle_mod, lib):
    """Quantized inputs stay within 1e-5 of the FP64 integration (V and STDP
    weights), with lazy LTP over every post spike."""
    s = S.plastic_indegree(n=20_000, k=500).with_(exact=True)
    steps = 1000
    st, ids, v, _, _, w = run_gpu(s, steps)
    o = oracle_mod.OracleNet(s)
    v64, w64, _, lost = o.reintegrate_fp64_uncapped(st, ids, steps)
    o.close()
    assert lost == 0 and len(ids) > 1000
    for x32, x64, floor in [(v, v64, 1.0), (w, w64, 1e-3 * s.w_max)]:
        x64 = np.asarray(x64, dtype=np.float64)
        err = np.abs(np.asarray(x32, dtype=np.float64) - x64) / np.maximum(np.abs(x64), floor)
        assert err.max() <= 1e-5, err.max()


def test_exact_rejects_unbounded_weights(lib):
    s = S.NetSpec(exact=True)
    A = s.add_pop(S.NOP, 1000)
    s.connect(A, A, capi.CONN_FIXED_INDEGREE, 3.0e7, degree=200, dmin=1, dmax=3, seed=5)
    with pytest.raises(NaerError, match="exact-sum"):
        S.build(s).close()
