"""naer_net_step_noalloc: the deterministic step with the library's fixed
scratch arena, against naer_net_step on the same network, through the C ABI.

Deterministic aggregation is bit-exact, so the tolerance is zero: rasters,
membrane potentials, refractory counters, event counts and (plastic
networks) weights must match word for word after each of two calls in a
row.  Collected last so it also runs after every other GPU test.
"""
import ctypes as C

import numpy as np
import pytest

from naer_b200 import _capi as capi
from naer_b200 import spec as S

pytestmark = pytest.mark.gpu


def step_noalloc(net, n):
    return capi.load().naer_net_step_noalloc(net.handle, C.c_uint64(n))


def assert_same(a, b, plastic):
    sa, ia = a.read_spikes()
    sb, ib = b.read_spikes()
    assert len(ia) == len(ib)
    assert np.array_equal(sa, sb) and np.array_equal(ia, ib)
    va, ra = a.read_state()
    vb, rb = b.read_state()
    assert np.array_equal(va.view(np.uint32), vb.view(np.uint32))
    assert np.array_equal(ra, rb)
    ta, tb = a.stats(), b.stats()
    assert ta["events"] == tb["events"] and ta["step"] == tb["step"]
    if plastic:
        wa, wb = a.read_csr()[2], b.read_csr()[2]
        assert np.array_equal(wa.view(np.uint32), wb.view(np.uint32))
    return len(ia)


@pytest.mark.parametrize("name,make,plastic", [
    ("brunel_small", lambda: S.brunel_small(poisson_weight=1.0), False),
    ("plastic_indegree", lambda: S.plastic_indegree(n=2000, k=200, drive_weight=21.0), True),
])
def test_noalloc_matches_step_on_two_calls(lib, name, make, plastic):
    s = make().with_(deterministic=True)
    with S.build(s) as ref, S.build(s) as net:
        bytes0 = net.stats()["device_bytes"]
        total = 0
        for n in (150, 250):
            ref.run(n)
            ref.finish()
            assert step_noalloc(net, n) == capi.NAER_OK, capi.last_error()
            net.finish()
            total = assert_same(ref, net, plastic)
            assert net.stats()["device_bytes"] == bytes0  # nothing allocated by the engine
        assert net.stats()["step"] == 400 and total > 100


def test_noalloc_rejects_oversize_before_stepping(lib):
    """4.8 M padded synapses (8 B of scratch each) need more than the 32 MiB
    arena: refused with NAER_E_OVERFLOW and the network's state untouched;
    naer_net_step still runs it."""
    s = S.scatter_outdegree(n=12000, k=400, drive_weight=24.0).with_(deterministic=True)
    with S.build(s) as net:
        assert step_noalloc(net, 5) == capi.NAER_E_OVERFLOW
        assert "fixed arena holds 33554432 bytes" in capi.last_error()
        net.finish()
        assert net.stats()["step"] == 0 and net.getTime() == 0
        net.run(5)
        net.finish()
        assert net.stats()["step"] == 5


def test_noalloc_rejects_atomic_network(lib):
    with S.build(S.brunel_small(poisson_weight=1.0)) as net:
        assert step_noalloc(net, 1) == capi.NAER_E_STATE
        assert "deterministic aggregation" in capi.last_error()
        assert net.stats()["step"] == 0


def test_noalloc_follows_a_reinstall(lib):
    """A reinstall between calls (set_tuning to one block per SM, then back
    to the default) changes the step grid and the queue; the next call
    repartitions the arena for it.  Word-for-word equal to naer_net_step."""
    s = S.brunel_small(poisson_weight=1.0).with_(deterministic=True)
    with S.build(s) as ref, S.build(s) as net:
        for bps, n in ((1, 120), (0, 180), (1, 90)):
            net.set_tuning(blocks_per_sm=bps)
            ref.run(n)
            ref.finish()
            assert step_noalloc(net, n) == capi.NAER_OK, capi.last_error()
            net.finish()
            assert_same(ref, net, False)
        assert net.stats()["step"] == 390


def test_noalloc_largest_accepted_network(lib):
    """The largest fixed out-degree network (degree 100) the arena accepts,
    found by growing it until the first call is refused, runs word for word
    like naer_net_step on two calls in a row."""
    def make(n):
        return S.scatter_outdegree(n=n, k=100, drive_weight=24.0).with_(deterministic=True)
    best = None
    for n in range(4000, 40001, 2000):
        with S.build(make(n)) as net:
            rc = step_noalloc(net, 1)
            if rc == capi.NAER_E_OVERFLOW:
                assert net.stats()["step"] == 0
                break
            assert rc == capi.NAER_OK, capi.last_error()
            best = n
    assert best is not None and best < 40000, best
    s = make(best)
    with S.build(s) as ref, S.build(s) as net:
        for n in (200, 300):
            ref.run(n)
            ref.finish()
            assert step_noalloc(net, n) == capi.NAER_OK, capi.last_error()
            net.finish()
            assert assert_same(ref, net, False) > 100
