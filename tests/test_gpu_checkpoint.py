"""Checkpoint / restore of a network and pre-emption of served jobs.

A deterministic run checkpointed at step k and restored into a new handle
built from the same description must continue exactly like the
uninterrupted run: raster (steps >= k), membrane potentials, refractory
counters, event count and, with STDP, weights, bit for bit.  The same holds
for a served job taken off the device (pre-empted) and resumed, and a
cancelled job ends without affecting the others.  The reference keeps this
state only in its device buffers (src/Network.cpp:379-569) and has no way
to save it.
"""
import time

import numpy as np
import pytest

from naer_b200 import NaerError
from naer_b200 import _capi as capi
from naer_b200 import spec as S
from naer_b200.forms import Server

from nets import integer_weight_net

pytestmark = pytest.mark.gpu


def state_of(net):
    st, ids = net.read_spikes()
    v, r = net.read_state()
    return st, ids, v, r, net.stats()["events"]


@pytest.mark.parametrize("make", [
    lambda: S.plastic_indegree(n=3000, k=200, drive_weight=21.0).with_(deterministic=True),
    lambda: S.brunel_small(poisson_weight=1.0).with_(deterministic=True),
    lambda: integer_weight_net(n=5000, k=200),  # atomic mode, exact on integer weights
    lambda: S.plastic_indegree(n=3000, k=200, drive_weight=21.0).with_(exact=True),  # exact-sum mode
])
def test_restore_continues_the_run(lib, make):
    s = make()
    k, m = 700, 900
    with S.build(s) as a:
        a.run(k)
        ck = a.checkpoint()
        a.run(m)
        a.finish()
        st, ids, v, r, ev = state_of(a)
        w = a.read_csr()[2]
    with S.build(s) as b:
        b.run(13)  # some unrelated progress first: restore replaces it
        b.restore(ck)
        assert b.stats()["step"] == k and b.getTime() == k * s.dt_us
        b.run(m)
        b.finish()
        bst, bids, bv, br, bev = state_of(b)
        bw = b.read_csr()[2]
    sel = st >= k
    assert sel.sum() > 100
    assert np.array_equal(bst, st[sel]) and np.array_equal(bids, ids[sel])
    assert np.array_equal(bv.view(np.uint32), v.view(np.uint32)) and np.array_equal(br, r)
    assert bev == ev
    assert np.array_equal(bw.view(np.uint32), w.view(np.uint32))


def test_restore_rejects_other_layouts(lib):
    with S.build(S.brunel_small(poisson_weight=1.0)) as a, \
            S.build(S.plastic_indegree(n=2000, k=100)) as b:
        a.run(10)
        ck = a.checkpoint()
        with pytest.raises(NaerError, match="another layout"):
            b.restore(ck)
        with pytest.raises(NaerError, match="not a checkpoint"):
            a.restore(b"garbage" * 20)
    # the same layout with the ring holding fixed-point sums instead of floats
    with S.build(S.brunel_small(poisson_weight=1.0)) as a, \
            S.build(S.brunel_small(poisson_weight=1.0).with_(exact=True)) as b:
        a.run(10)
        with pytest.raises(NaerError, match="another layout"):
            b.restore(a.checkpoint())


def alone(spec, steps):
    with S.build(spec) as net:
        net.run(steps)
        net.finish()
        return net.read_spikes()


def wait_running(srv, job, min_steps=0, timeout=60.0):
    t0 = time.time()
    while time.time() - t0 < timeout:
        i = srv.info(job)
        if i["state"] == capi.JOB_RUNNING and i["steps_done"] >= min_steps:
            return
        time.sleep(0.002)
    raise AssertionError(f"job {job} did not reach {min_steps} steps")


def test_server_preempt_resume_and_cancel(lib):
    """Deterministic jobs: one pre-empted twice and resumed, one cancelled
    while running, one queued job cancelled; the others' rasters equal
    their runs alone, including the pre-empted one."""
    specs = [S.plastic_indegree(n=n, k=120, seed=sd, drive_rate_hz=30.0, stdp=(sd % 2 == 0)).with_(deterministic=True)
             for n, sd in [(4000, 31), (2500, 32), (3000, 33), (1800, 34)]]
    durations = [20000, 15000, 3000, 800]
    with Server(chunk_steps=64, launch_steps=16, deterministic=True) as srv:
        ids = [srv.submit(s, d) for s, d in zip(specs, durations)]
        wait_running(srv, ids[0], 1500)
        srv.preempt(ids[0])
        wait_running(srv, ids[1], 100)
        srv.cancel(ids[1])
        t0 = time.time()
        while srv.info(ids[0])["preemptions"] < 1 and time.time() - t0 < 60:
            time.sleep(0.002)
        wait_running(srv, ids[0], 6000)  # resumed and past where it stopped
        srv.preempt(ids[0])
        assert srv.drain(300.0)
        info = [srv.info(j) for j in ids]
        assert info[0]["state"] == capi.JOB_DONE and info[0]["preemptions"] == 2
        assert info[0]["steps_done"] == durations[0]
        assert info[1]["state"] == capi.JOB_CANCELLED
        with pytest.raises(NaerError):
            srv.cancel(ids[1])
        for j in (0, 2, 3):
            assert info[j]["state"] == capi.JOB_DONE
            st, i = srv.spikes(ids[j])
            ast, ai = alone(specs[j], durations[j])
            assert len(ai) > 100
            assert np.array_equal(st, ast) and np.array_equal(i, ai), j


def test_server_cancel_queued_job(lib):
    """A job still waiting for memory is cancelled before it is built."""
    big = S.plastic_indegree(n=20000, k=300, seed=41).with_(deterministic=True)
    # the footprint estimate of one job is about 114 MB (with the deterministic
    # aggregation's event lists): the budget holds one
    with Server(budget_bytes=150 * 10**6, chunk_steps=64, deterministic=True) as srv:
        a = srv.submit(big, 2000)
        b = srv.submit(big.with_(name="second"), 2000)  # waits: the budget holds one
        wait_running(srv, a, 1)
        assert srv.info(b)["state"] == capi.JOB_QUEUED
        srv.cancel(b)
        assert srv.info(b)["state"] == capi.JOB_CANCELLED
        assert srv.drain(300.0)
        assert srv.info(a)["state"] == capi.JOB_DONE
