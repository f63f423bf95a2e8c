"""Failure paths on the GPU, made without any fault: every wait of the step
kernel is bounded, and a test makes one run out on purpose.

naer_test_set_barrier_skew raises every grid-barrier target of the next
launches, so no barrier can complete; each block's wait gives up after the
limit set by naer_net_set_wait_limit (here 1 ms), records NAER_E_TIMEOUT in
the control block and returns.  The host then sees NAER_E_TIMEOUT from
naer_net_finish, the handle refuses further steps, is destroyed normally,
and a fresh network on the same device steps bit-exact with the oracle
(the context is still usable).  The reference reports device failures by
throwing (src/Network.cpp:21-23, 146-149); here they are status codes.
"""
import numpy as np
import pytest

from naer_b200 import _capi as capi
from naer_b200 import spec as S

from nets import integer_weight_net

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_context_survives(oracle_mod, lib):
    s = integer_weight_net(n=6000, k=300, seed=3)
    net = S.build(s)
    try:
        net.run(5)
        net.finish()
        capi.call("naer_net_set_wait_limit", net.handle, 1000)  # 1 ms
        capi.call("naer_test_set_barrier_skew", net.handle, 1)
        net.run(130)  # three persistent launches, each ends at its first barrier
        rc = lib.naer_net_finish(net.handle)
        assert rc == capi.NAER_E_TIMEOUT, (rc, capi.last_error())
        assert "wait limit" in capi.last_error()
        rc = lib.naer_net_step(net.handle, 1)
        assert rc == capi.NAER_E_STATE
        assert "undefined" in capi.last_error()
    finally:
        net.close()
    # the device context is intact: a new network runs and matches the oracle
    with S.build(s) as fresh:
        fresh.run(300)
        fresh.finish()
        st, ids = fresh.read_spikes()
        v, r = fresh.read_state()
    o = oracle_mod.OracleNet(s, deterministic=True)
    o.run(300)
    ost, oids = o.spikes()
    ov, orr = o.state()
    o.close()
    assert len(ids) > 100
    assert np.array_equal(st, ost) and np.array_equal(ids, oids)
    assert np.array_equal(v.view(np.uint32), ov.view(np.uint32)) and np.array_equal(r, orr)


def test_wait_limit_validation(lib):
    with S.build(integer_weight_net(n=2000, k=50)) as net:
        assert lib.naer_net_set_wait_limit(net.handle, 4_000_000_000) == capi.NAER_E_INVALID
        capi.call("naer_net_set_wait_limit", net.handle, 0)  # default restored
        net.run(70)
        net.finish()
        assert net.stats()["step"] == 70


def test_device_probe_figures(lib):
    """The ceilings bench.py reports: positive, finite and ordered sensibly."""
    p = capi.probe_device(0, ring_cells=17_000_000, small_cells=3_000_000)
    assert p["grid"] >= 100
    for k in ("red_ring_per_s", "red_small_per_s", "store_ring_per_s"):
        assert 1e9 < p[k] < 1e14, (k, p[k])
    assert 500 < p["stream_gbs"] < 20_000
    assert 0.05 < p["barrier_us_1"] < 100 and 0.05 < p["barrier_us_2"] < 100


def test_allocation_failure_reported_and_released(lib):
    """An out-of-memory injected at every allocation of a compile in turn:
    each attempt returns NAER_E_OOM with nothing left allocated by it (the
    same handle then compiles to the footprint of a fresh one), and the
    network steps like one that never failed."""
    s = S.plastic_indegree(n=2000, k=100, drive_weight=21.0).with_(deterministic=True)
    with S.build(s) as ref:
        ref_bytes = ref.stats()["device_bytes"]
        ref.run(200)
        ref.finish()
        ref_raster = ref.read_spikes()
    hits = 0
    try:
        for k in range(400):
            net = S.describe(s, device=0)
            try:
                capi.call("naer_test_fail_allocation", k)
                rc = lib.naer_net_compile(net.handle)
                capi.call("naer_test_fail_allocation", -1)
                if rc == capi.NAER_OK:
                    break
                assert rc == capi.NAER_E_OOM, (k, rc, capi.last_error())
                assert "injected" in capi.last_error()
                hits += 1
                net.compile()  # the injection fired once: the same handle compiles now
                assert net.stats()["device_bytes"] == ref_bytes, k
                net.run(200)
                net.finish()
                st, ids = net.read_spikes()
                assert np.array_equal(st, ref_raster[0]) and np.array_equal(ids, ref_raster[1]), k
            finally:
                net.close()
    finally:
        capi.call("naer_test_fail_allocation", -1)
    assert hits > 10  # every allocation of the build, the tables and the queues was hit


@pytest.mark.parametrize("rate", [10.0, 20.0, 40.0])
def test_poisson_interval_log_agreement(lib, oracle_mod, rate):
    """The Poisson interval (uint)(log(1 - x) / -(rate * 1e-6)) on the
    device (CUDA's log) against the host (glibc's log) for 2^27 generator
    outputs spread over the whole range (every 32nd): the two logarithms
    may differ by an ulp, which changes the truncated µs only at an exact
    boundary.  The count of disagreements is printed and must stay a tiny
    fraction (the bit-exact raster tests depend on none occurring on their
    seeds)."""
    import ctypes as C
    n, step = 1 << 27, 32
    dev = np.empty(n, dtype=np.uint32)
    capi.call("naer_probe_intervals", 0, rate, 7, step, n, dev.ctypes.data_as(C.c_void_p))
    host = oracle_mod.intervals(rate, 7, step, n)
    diff = np.flatnonzero(dev != host)
    print(f"rate {rate} Hz: {len(diff)} of {n} intervals differ between CUDA log and glibc log"
          + (f" (first z {7 + int(diff[0]) * step}, device {dev[diff[0]]}, host {host[diff[0]]})" if len(diff) else ""))
    assert len(diff) <= n // 1_000_000
    assert np.all(np.abs(dev[diff].astype(np.int64) - host[diff].astype(np.int64)) <= 1)
