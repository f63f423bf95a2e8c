"""Batched and served forms against the plain form, through the C ABI.

Deterministic aggregation: every member (job) must produce, bit for bit,
the raster and state it produces alone.  Atomic aggregation is checked on
integer-weight networks, where the order of the reductions cannot change
any sum, so the batched and served results must equal the deterministic
plain run exactly.
"""
import numpy as np
import pytest

from naer_b200 import _capi as capi
from naer_b200 import spec as S
from naer_b200.forms import Batch, Server
from naer_b200 import NaerError

from nets import integer_weight_net

pytestmark = pytest.mark.gpu


def alone(spec, steps):
    with S.build(spec.with_(deterministic=True)) as net:
        net.run(steps)
        net.finish()
        st, ids = net.read_spikes()
        v, r = net.read_state()
    return st, ids, v, r


def small_members(count=5, seed=3):
    return S.batch_members(count=count, seed=seed, n_range=(600, 4000), k_range=(50, 300), rate_range=(20.0, 60.0))


def test_batch_deterministic_matches_alone(lib):
    members = small_members()
    steps = 700
    with Batch(members, deterministic=True).compile() as b:
        b.run(300)
        b.run(400)
        b.finish()
        sp = b.read_spikes()
        assert b.stats()["step"] == steps
        for i, m in enumerate(members):
            st, ids, v, r = alone(m, steps)
            bst, bids = b.member_spikes(i, sp)
            assert len(ids) > 50, m.name
            assert np.array_equal(st, bst) and np.array_equal(ids, bids), m.name
            bv, br = b.read_state(i, m.neurons)
            assert np.array_equal(v.view(np.uint32), bv.view(np.uint32)) and np.array_equal(r, br), m.name


def test_batch_graph_atomic_exact_on_integer_weights(lib):
    """Atomic mode through the CUDA-graph replay (16 launches per replay)
    plus plain launches for the remainder."""
    members = [integer_weight_net(n=n, k=k, seed=sd) for n, k, sd in [(3000, 200, 1), (5000, 300, 2), (1500, 100, 3)]]
    with Batch(members).compile() as b:
        L = b.tuning()["launch_steps"]
        steps = 2 * 16 * L + 37  # two replays and a remainder
        l0 = b.stats()["kernel_launches"]
        b.run(steps)
        b.finish()
        assert b.stats()["kernel_launches"] - l0 == 2 * ((steps + L - 1) // L)
        sp = b.read_spikes()
        for i, m in enumerate(members):
            st, ids, v, r = alone(m, steps)
            bst, bids = b.member_spikes(i, sp)
            assert len(ids) > 1000
            assert np.array_equal(st, bst) and np.array_equal(ids, bids)
            bv, _ = b.read_state(i, m.neurons)
            assert np.array_equal(v.view(np.uint32), bv.view(np.uint32))


def test_batch_autotune_keeps_results(lib):
    members = [integer_weight_net(n=n, k=200, seed=sd) for n, sd in [(4000, 4), (2500, 5)]]
    with Batch(members).compile() as b:
        t = b.autotune(trial_steps=32)
        assert t["trials"] >= 2 and t["best_us_per_step"] > 0
        assert t["best_us_per_step"] <= t["default_us_per_step"]
        total = b.stats()["step"] + 200  # the trials advanced the simulation
        b.run(200)
        b.finish()
        sp = b.read_spikes()
        for i, m in enumerate(members):
            st, ids, _, _ = alone(m, total)
            bst, bids = b.member_spikes(i, sp)
            assert np.array_equal(st, bst) and np.array_equal(ids, bids)


def test_batch_phase_split(lib):
    """naer_batch_get_phases: the step kernel's time split accumulates while
    the batch steps (four phases, non-negative, growing with the steps)."""
    with Batch(small_members(count=3)).compile() as b:
        b.run(128)
        b.finish()
        p0 = b.phases()
        b.run(256)
        b.finish()
        p1 = b.phases()
    assert set(p1) == {"lif", "lif_wait", "scatter", "reserved", "scatter_wait"}
    assert all(v >= 0 for v in p0.values()) and p1["reserved"] == 0
    grown = {k: p1[k] - p0[k] for k in ("lif", "lif_wait", "scatter", "scatter_wait")}
    assert all(v >= 0 for v in grown.values()) and grown["lif"] > 0 and sum(grown.values()) > 0


def test_batch_rejects_bad_member(lib):
    s = S.NetSpec()
    P = s.add_pop(S.POISSON, 10, rate_hz=10.0)
    E = s.add_pop(S.NOP, 10)
    s.connect(E, P, capi.CONN_FIXED_OUTDEGREE, 0.1, degree=2)
    with Batch() as b:
        with pytest.raises(NaerError, match="POISSON"):
            b.add(s)
        with pytest.raises(NaerError):
            b.compile()  # no members


def test_server_deterministic_jobs_match_alone(lib):
    """Jobs of different sizes and durations arriving while others run, a
    budget that makes some wait for memory, admission every 64 steps: each
    job's raster equals its raster alone."""
    jobs = [(m, d) for m, d in zip(small_members(count=6, seed=7), [150, 700, 333, 64, 500, 260])]
    # an upper bound of the library's footprint estimate of each job (9 B per
    # synapse, 8 more for the deterministic aggregation's event lists,
    # per-neuron arrays with the list heads, decay tables); 1.5x the largest
    # lets one or two jobs run at a time
    est = max(17 * m.neurons * sum(c.degree for c in m.conns) // 2 + 480 * m.neurons + 170_000 for m, _ in jobs)
    with Server(budget_bytes=int(1.5 * est), chunk_steps=64, deterministic=True) as srv:
        ids = []
        for m, d in jobs:
            ids.append(srv.submit(m, d))
        assert srv.drain(300.0)
        st = srv.stats()
        assert st["done"] == len(jobs) and st["failed"] == 0
        assert st["p99_ms"] >= st["p50_ms"] > 0 and st["chunks"] > 1
        for jid, (m, d) in zip(ids, jobs):
            info = srv.info(jid)
            assert info["state"] == capi.JOB_DONE and info["steps_done"] == d
            s_st, s_ids = srv.spikes(jid)
            a_st, a_ids, _, _ = alone(m, d)
            assert np.array_equal(s_st, a_st) and np.array_equal(s_ids, a_ids), m.name
            srv.release(jid)


@pytest.mark.parametrize("launch_steps", [0, 16])
def test_server_atomic_integer_weights_exact(lib, launch_steps):
    jobs = [(integer_weight_net(n=n, k=150, seed=sd), d) for n, sd, d in [(3000, 11, 400), (2000, 12, 250),
                                                                          (4000, 13, 512)]]
    with Server(chunk_steps=128, launch_steps=launch_steps) as srv:
        ids = [srv.submit(m, d) for m, d in jobs]
        assert srv.drain(300.0)
        for jid, (m, d) in zip(ids, jobs):
            s_st, s_ids = srv.spikes(jid)
            a_st, a_ids, _, _ = alone(m, d)
            assert len(a_ids) > 500
            assert np.array_equal(s_st, a_st) and np.array_equal(s_ids, a_ids)


def test_server_rejects_oversize_and_invalid(lib):
    with Server(budget_bytes=10**6) as srv:
        with pytest.raises(NaerError, match="budget"):
            srv.submit(S.plastic_indegree(n=20000, k=500), 10)
        s = S.NetSpec()
        P = s.add_pop(S.POISSON, 10, rate_hz=10.0)
        E = s.add_pop(S.NOP, 10)
        s.connect(E, P, capi.CONN_FIXED_OUTDEGREE, 0.1, degree=2)
        with pytest.raises(NaerError, match="POISSON"):
            srv.submit(s, 10)
        assert srv.stats()["submitted"] == 0
    with pytest.raises(NaerError, match="launch_steps"):
        Server(budget_bytes=10**6, launch_steps=65)


def test_server_deterministic_set_outgrows_the_queue(lib):
    """A deterministic served set whose LIF chunks grow past the step
    grid's blocks after the first installation (one block per SM, so 148
    blocks): the queue and sort buffers sized for the first, one-chunk set
    must grow with the set.  Both jobs still match their runs alone."""
    small = S.plastic_indegree(n=1500, k=60, seed=21, drive_rate_hz=40.0)
    big = S.plastic_indegree(n=200_000, k=40, seed=22, drive_rate_hz=20.0, stdp=False)
    with Server(chunk_steps=32, blocks_per_sm=1, deterministic=True) as srv:
        a = srv.submit(small, 4000)
        import time
        t0 = time.time()
        while srv.info(a)["state"] != capi.JOB_RUNNING and time.time() - t0 < 60:
            time.sleep(0.01)  # the small job is installed alone first
        assert srv.info(a)["state"] == capi.JOB_RUNNING
        b = srv.submit(big, 120)
        assert srv.drain(300.0)
        assert srv.stats()["failed"] == 0
        assert srv.info(b)["admit_s"] < srv.info(a)["done_s"]  # the two ran together
        for jid, (m, d) in [(a, (small, 4000)), (b, (big, 120))]:
            s_st, s_ids = srv.spikes(jid)
            a_st, a_ids, _, _ = alone(m, d)
            assert len(a_ids) > 50
            assert np.array_equal(s_st, a_st) and np.array_equal(s_ids, a_ids), m.name
