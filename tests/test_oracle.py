"""The oracle against independent restatements, golden vectors and the
properties of the reference's algorithm (CPU only)."""
import json
from pathlib import Path

import numpy as np
import pytest

from naer_b200 import _capi as capi
from naer_b200 import spec as S

GOLDEN = Path(__file__).resolve().parent / "golden"
M = 0xFFFFFFFF


def py_philox(ctr, key):
    """Philox4x32-10 in plain Python (Salmon et al., SC'11), a third restatement."""
    c = [int(x) & M for x in ctr]
    k0, k1 = int(key[0]) & M, int(key[1]) & M
    for r in range(10):
        if r:
            k0 = (k0 + 0x9E3779B9) & M
            k1 = (k1 + 0xBB67AE85) & M
        p0 = 0xD2511F53 * c[0]
        p1 = 0xCD9E8D57 * c[2]
        c = [((p1 >> 32) ^ c[1] ^ k0) & M, p1 & M, ((p0 >> 32) ^ c[3] ^ k1) & M, p0 & M]
    return c


def test_philox_matches_python_restatement(oracle_mod):
    rng = np.random.default_rng(0)
    for _ in range(200):
        ctr = rng.integers(0, 2**32, 4, dtype=np.uint64)
        key = rng.integers(0, 2**32, 2, dtype=np.uint64)
        assert list(oracle_mod.philox4x32_10(ctr, key)) == py_philox(ctr, key)
    for ctr, key in [([0, 0, 0, 0], [0, 0]), ([M] * 4, [M, M])]:
        assert list(oracle_mod.philox4x32_10(ctr, key)) == py_philox(ctr, key)


# Known-answer vectors published with Random123 for philox4x32-10
# (counter, key, output), the library behind the reference's philox4x32
# (include/naer/kernels/random.cl:8-16).
RANDOM123_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([M, M, M, M], [M, M], [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


def test_philox_random123_known_answers(oracle_mod):
    for ctr, key, out in RANDOM123_KAT:
        assert list(oracle_mod.philox4x32_10(ctr, key)) == out
        assert py_philox(ctr, key) == out


def test_philox_matches_curand_golden(oracle_mod):
    """cuRAND's Philox4_32_10 outputs (generated on a B200 by
    tests/golden/gen_philox_curand.py) pin the oracle's Philox."""
    f = GOLDEN / "philox_curand.json"
    if not f.exists():
        pytest.skip("golden vectors not generated yet")
    data = json.loads(f.read_text())
    assert len(data["cases"]) >= 64
    for case in data["cases"]:
        seed, subseq, offset = case["seed"], case["subsequence"], case["offset"]
        blk = offset // 4
        ctr = [blk & M, blk >> 32, subseq & M, subseq >> 32]
        key = [seed & M, seed >> 32]
        assert list(oracle_mod.philox4x32_10(ctr, key)) == case["out"], case


def test_uniform_rand_is_reference_formula(oracle_mod):
    # random.cl:6-24: key {gid, seed}, counter {iter,0,0,0}, word z / UINT_MAX
    for gid, seed, it in [(0, 0, 0), (5, 0x15AC7EBD, 123456), (2**31, 7, 2**32 - 1)]:
        z = py_philox([it, 0, 0, 0], [gid, seed])[2]
        assert oracle_mod.uniform_rand(gid, seed, it) == z / 4294967295.0


def test_poisson_window_semantics(oracle_mod):
    # input_neuron_group.cl:29-38: first draw from t0, at most 10 spikes,
    # each time + (uint)exprnd(...) with counter time * N + idx
    import math
    n, seed, rate = 4096, 0x15AC7EBD, 20.0
    for idx in [0, 1, 127, 128, 2047, 2048, 4095]:
        for t0 in [0, 1500, 3000, 1_000_000]:
            times = oracle_mod.poisson_window(idx, n, seed, rate, t0, t0 + 1500)
            gid = (idx // 2048) * 128 + (idx % 2048) % 128
            z = py_philox([(t0 * n + idx) & M, 0, 0, 0], [gid, seed])[2]
            first = t0 + int(math.log(1.0 - z / 4294967295.0) / (-(rate / 1e6)))
            if first < t0 + 1500:
                assert len(times) >= 1 and times[0] == first
            else:
                assert len(times) == 0
            assert np.all(np.diff(times.astype(np.int64)) >= 0) and len(times) <= 10


def test_poisson_rate(oracle_mod):
    # 2000 generators x 200 windows of 1.5 ms at 20 Hz: mean count 0.03
    counts = [len(oracle_mod.poisson_window(i, 2000, 99, 20.0, t0, t0 + 1500))
              for i in range(0, 2000, 7) for t0 in range(0, 300_000, 1500)]
    assert np.mean(counts) == pytest.approx(0.03, rel=0.1)


def small_spec(rule, **kw):
    s = S.NetSpec()
    P = s.add_pop(S.POISSON, 50, rate_hz=50.0)
    E = s.add_pop(S.NOP, 120)
    I = s.add_pop(S.STDP, 37)
    s.connect(P, E, rule, 0.5, probability=0.2, degree=7, dmin=1, dmax=5, seed=11, **kw)
    s.connect(E, I, rule, 0.0, probability=0.3, degree=5, wmin=0.1, wmax=0.4, dmin=2, dmax=2, seed=12)
    s.connect(E, E, rule, -0.2, probability=0.1, degree=3, dmin=1, dmax=9, seed=13)
    return s


@pytest.mark.parametrize("rule", [capi.CONN_REF_BERNOULLI, capi.CONN_FIXED_INDEGREE, capi.CONN_FIXED_OUTDEGREE])
def test_csr_rules(oracle_mod, rule):
    s = small_spec(rule)
    o = oracle_mod.OracleNet(s)
    rp, tg, w, d = o.csr()
    assert rp[0] == 0 and rp[-1] == len(tg) == o.S
    base = {i: o.population_base(i) for i in range(3)}
    # address layout: STDP first, then NOP, then POISSON (Network.cpp:271-272)
    assert base[2] == 0 and base[1] == 37 and base[0] == 37 + 120
    assert d.min() >= 1 and d.max() <= 9
    E0, E1 = base[1], base[1] + 120
    if rule == capi.CONN_FIXED_OUTDEGREE:
        for a in range(base[0], base[0] + 50):
            assert rp[a + 1] - rp[a] == 7
        for a in range(E0, E1):
            assert rp[a + 1] - rp[a] == 5 + 3
    if rule == capi.CONN_FIXED_INDEGREE:
        # each E target appears 7 times among the Poisson rows
        rows = tg[rp[base[0]]:rp[base[0] + 50]]
        assert np.all(np.bincount(rows - E0, minlength=120) == 7)
    # canonical order: delay-1 synapses first (stable partition of the row)
    for a in range(o.n):
        dd = d[rp[a]:rp[a + 1]]
        assert np.all(np.diff((dd != 1).astype(np.int8)) >= 0)
    if rule == capi.CONN_REF_BERNOULLI:
        # within one connection and delay class, targets ascend (network.cl:88-105 in order)
        for a in range(base[0], base[0] + 50):
            row_t, row_d = tg[rp[a]:rp[a + 1]].astype(np.int64), d[rp[a]:rp[a + 1]]
            for cls in (row_d == 1, row_d != 1):
                assert np.all(np.diff(row_t[cls]) > 0)
        frac = (rp[base[0] + 50] - rp[base[0]]) / (50 * 120)
        assert frac == pytest.approx(0.2, abs=0.03)
    # random weights (weight 0) lie in [wmin, wmax)
    ei = np.concatenate([np.arange(int(rp[a]), int(rp[a + 1])) for a in range(E0, E1)]).astype(np.int64)
    ws = w[ei]
    rnd = ws[(ws >= 0.1 - 1e-7) & (ws <= 0.4)]
    assert rnd.size > 0


def test_bernoulli_is_reference_draw(oracle_mod):
    """network.cl:34-41: (s, d) connected iff uniform_rand(seed32, d) on
    work-item s*32 + d%32 is below p; weight from the same draw when 0."""
    s = S.NetSpec()
    A = s.add_pop(S.NOP, 9)
    B = s.add_pop(S.NOP, 70)
    seed = 0xBF785E3215AC7EBD
    s.connect(A, B, capi.CONN_REF_BERNOULLI, 0.0, probability=0.35, wmin=-1.0, wmax=2.0, seed=seed)
    o = oracle_mod.OracleNet(s)
    rp, tg, w, d = o.csr()
    bB = o.population_base(1)
    for a in range(9):
        exp_t, exp_w = [], []
        for dd in range(70):
            z = py_philox([dd, 0, 0, 0], [a * 32 + dd % 32, seed & M])[2]
            x = z / 4294967295.0
            if x < 0.35:
                exp_t.append(bB + dd)
                exp_w.append(np.float32(-1.0) + np.float32(3.0) * np.float32(x))
        got = slice(rp[a], rp[a + 1])
        assert list(tg[got]) == exp_t
        assert np.array_equal(w[got], np.array(exp_w, dtype=np.float32))


def test_lif_free_decay_matches_closed_form(oracle_mod):
    """No input: V_t = fp32(fp64(V_{t-1}) * exp(-dt/tau)) each step."""
    s = S.NetSpec()
    s.add_pop(S.NOP, 4, v_init=19.0, tau_m_ms=10.0)
    o = oracle_mod.OracleNet(s, deterministic=True)
    o.run(37)
    v, r = o.state()
    P = np.exp(-100.0 / 10000.0)
    x = np.float32(19.0)
    for _ in range(37):
        x = np.float32(np.float64(x) * P)
    assert np.all(v == x) and np.all(r == 0)


def test_lif_threshold_reset_refractory(oracle_mod):
    """A neuron above threshold spikes once, resets to V_reset and ignores
    input for t_ref steps (lif.cl:21-33 on the grid)."""
    s = S.NetSpec()
    s.add_pop(S.NOP, 1, v_init=25.0, v_th=20.0, v_reset=10.0, t_ref_ms=0.5, drive_rate_hz=5e4,
              drive_weight=3.0, drive_seed=5)
    o = oracle_mod.OracleNet(s, deterministic=True)
    o.run(40)
    st, ids = o.spikes()
    assert st[0] == 0
    assert np.all(np.diff(st.astype(np.int64)) >= 6)  # 5 refractory steps between spikes


def test_deterministic_rerun_is_identical(oracle_mod):
    s = S.brunel_small(poisson_weight=1.0)
    a = oracle_mod.OracleNet(s, deterministic=True, threads=3)
    b = oracle_mod.OracleNet(s, deterministic=True, threads=1)
    a.run(300)
    b.run(300)
    sa, ia = a.spikes()
    sb, ib = b.spikes()
    assert np.array_equal(sa, sb) and np.array_equal(ia, ib) and len(ia) > 100
    assert np.array_equal(a.state()[0], b.state()[0])


def test_stdp_weights_stay_clipped(oracle_mod):
    s = S.plastic_indegree(n=500, k=50, drive_weight=21.0)
    o = oracle_mod.OracleNet(s, deterministic=True)
    w0 = o.weights()
    o.run(500)
    w1 = o.weights()
    rp, tg, _, _ = o.csr()
    assert not np.array_equal(w0, w1)
    nE = 400
    src = np.repeat(np.arange(o.n), np.diff(rp).astype(np.int64))
    ee = (src < nE) & (tg < nE)
    assert np.all((w1[ee] >= 0.0) & (w1[ee] <= 0.5))
    assert np.array_equal(w0[~ee], w1[~ee])


def test_golden_oracle_fixture(oracle_mod):
    """Regression fixture of the oracle itself (tests/golden/gen_oracle_fixtures.py)."""
    f = GOLDEN / "oracle_brunel_small.npz"
    if not f.exists():
        pytest.skip("fixture not generated")
    g = np.load(f)
    o = oracle_mod.OracleNet(S.brunel_small(poisson_weight=1.0), deterministic=True)
    o.run(int(g["steps"]))
    st, ids = o.spikes()
    assert np.array_equal(st, g["spike_steps"]) and np.array_equal(ids, g["spike_ids"])
    assert np.array_equal(o.state()[0], g["v"])


# FP64 re-integration: the fp32 trajectory against double arithmetic with the
# same spike times.  Tolerance: |x32 - x64| <= 1e-5 * max(|x64|, floor), the
# floor being 1 mV for membrane potentials and 1e-3 * w_max for weights.
FP64_RTOL = 1e-5


def within_fp64(x32, x64, floor):
    x64 = np.asarray(x64, dtype=np.float64)
    return np.abs(np.asarray(x32, dtype=np.float64) - x64) <= FP64_RTOL * np.maximum(np.abs(x64), floor)


@pytest.mark.parametrize("make,steps", [(lambda: S.brunel_small(poisson_weight=1.0), 2000),
                                        (lambda: S.plastic_indegree(n=2000, k=200, drive_weight=21.0), 1000)])
def test_oracle_fp32_within_fp64_reintegration(oracle_mod, make, steps):
    O = oracle_mod
    s = make()
    o = O.OracleNet(s, deterministic=True)
    o.run(steps)
    st, ids = o.spikes()
    v, _ = o.state()
    w = o.weights()
    v64, w64, mismatch = O.OracleNet(s).reintegrate_fp64(st, ids, steps)
    assert len(ids) > 1000
    assert within_fp64(v, v64, 1.0).all()
    assert within_fp64(w, w64, 1e-3 * s.w_max).all()
    assert mismatch == 0


def test_fp64_uncapped_history(oracle_mod):
    O = oracle_mod
    """The uncapped re-integration (every post spike since the source's last
    spike) equals the capped one when the cap drops nothing, and departs
    from it when a one-entry history drops pairs."""
    s = S.plastic_indegree(n=1500, k=150, drive_weight=21.0, drive_rate_hz=20.0).with_(stdp_history=16)
    steps = 1200
    o = O.OracleNet(s)
    o.run(steps)
    st, ids = o.spikes()
    v64, w64, _ = O.OracleNet(s).reintegrate_fp64(st, ids, steps)
    u64, uw64, _, lost = O.OracleNet(s).reintegrate_fp64_uncapped(st, ids, steps)
    assert lost == 0 and o.hist_overflow == 0  # nothing lost, and the fp32 run's count agrees
    assert np.array_equal(v64, u64) and np.array_equal(w64, uw64)
    s1 = s.with_(stdp_history=1)
    o1 = O.OracleNet(s1)
    o1.run(steps)
    st1, ids1 = o1.spikes()
    _, cw, _ = O.OracleNet(s1).reintegrate_fp64(st1, ids1, steps)
    _, uw, _, lost1 = O.OracleNet(s1).reintegrate_fp64_uncapped(st1, ids1, steps)
    assert lost1 > 0 and o1.hist_overflow > 0
    assert not np.array_equal(cw, uw) and (uw >= cw - 1e-12).all()  # dropped pairs are potentiation only


# Reference-compatible event mode (oracle only): the `.cl` kernels' time model.

def _lif_event_model(times, w, tau_ms, v_th, v_reset, t_ref_ms):
    """neuron_dynamics (include/naer/kernels/lif.cl:15-34) for one neuron
    driven by one source: input times in us, fp32 potential, fp64 decay."""
    v = np.float32(0.0)
    last = 0
    out = []
    for T in times:
        if T < last:
            continue
        dt = float(T) - float(last)
        v = np.float32(float(v) * np.exp(-dt / (tau_ms * 1000.0)))
        v = np.float32(v + np.float32(w))
        last = T
        if v > np.float32(v_th):
            last = T + int(round(t_ref_ms * 1000.0))
            v = np.float32(v_reset)
            out.append(T)
    return v, out


@pytest.mark.parametrize("w", [0.008, 0.025])
def test_event_mode_single_synapse_matches_lif_cl(oracle_mod, w):
    O = oracle_mod
    s = S.NetSpec()
    P = s.add_pop(S.POISSON, 1, rate_hz=400.0)
    E = s.add_pop(S.NOP, 1, v_th=0.020, v_reset=0.0, t_ref_ms=2.0, tau_m_ms=20.0)
    s.connect(P, E, capi.CONN_FIXED_OUTDEGREE, w, degree=1)
    o = O.OracleNet(s)
    o.run_events(200)  # 0.3 s
    t, ids = o.event_spikes()
    pt = np.sort(t[ids == o.population_base(P)])
    assert len(pt) > 60
    # Poisson events are the generator's windows of 1500 us
    ref = np.concatenate([O.poisson_window(0, 1, s.poisson_seed, 400.0, 1500 * k, 1500 * (k + 1))
                          for k in range(200)])
    assert np.array_equal(pt, np.sort(ref))
    v, out = _lif_event_model(pt, w, 20.0, 0.020, 0.0, 2.0)
    et = np.sort(t[ids == o.population_base(E)])
    assert np.array_equal(et, np.array(out, dtype=np.uint32))
    ev, _, _ = o.event_state()
    # spikes emitted in the last window are delivered in the next one: V matches
    assert ev[o.population_base(E)] == v
    if w > 0.02:
        assert len(out) > 30   # every input outside the refractory period fires
    else:
        assert len(out) > 0    # summation of decayed inputs reaches threshold


def test_event_mode_delay_and_truncation(oracle_mod):
    """NOP spikes arrive 1500 us later; with the nop.cl option only 96
    synapses per (spike, 512-neuron NOP group) are delivered."""
    O = oracle_mod
    s = S.NetSpec()
    P = s.add_pop(S.POISSON, 1, rate_hz=200.0)
    A = s.add_pop(S.NOP, 1, v_th=0.020, v_reset=0.0)
    B = s.add_pop(S.NOP, 200, v_th=0.020, v_reset=0.0)
    s.connect(P, A, capi.CONN_FIXED_OUTDEGREE, 0.03, degree=1)
    s.connect(A, B, capi.CONN_FIXED_INDEGREE, 0.03, degree=1)  # every B neuron once in A's row
    full, trunc = O.OracleNet(s), O.OracleNet(s)
    full.run_events(100)
    trunc.run_events(100, truncate96=True)
    t, ids = full.event_spikes()
    a = full.population_base(A)
    ta = np.sort(t[ids == a])
    tb = t[(ids >= full.population_base(B)) & (ids < full.population_base(B) + 200)]
    assert len(ta) > 10
    # every B spike happens exactly one axonal delay after an A spike
    assert np.isin(tb, ta + 1500).all()
    # an A spike (w above threshold) makes every B neuron it reaches fire;
    # the A spikes whose arrival falls inside the simulated windows count
    n_a = int((ta + 1500 < 100 * 1500).sum())
    tt, it = trunc.event_spikes()
    b0 = full.population_base(B)
    assert len(tb) == 200 * n_a
    assert ((it >= b0) & (it < b0 + 200)).sum() == 96 * n_a


def test_event_mode_reference_brunel_deterministic(oracle_mod):
    from nets import reference_brunel
    O = oracle_mod
    s = reference_brunel(2e5)
    a, b = O.OracleNet(s), O.OracleNet(s)
    a.run_events(300)
    b.run_events(150)
    b.run_events(150)
    ta, ia = a.event_spikes()
    tb, ib = b.event_spikes()
    assert np.array_equal(ta, tb) and np.array_equal(ia, ib)
    assert len(ia) > 1000


def test_explicit_csr_reproduces_a_rule(oracle_mod):
    """A rule's connectivity given back as explicit synapses (the CSR the
    oracle generated) runs exactly like the rule-generated network."""
    O = oracle_mod
    a = S.NetSpec(poisson_seed=5)
    P = a.add_pop(S.POISSON, 400, rate_hz=60.0)
    E = a.add_pop(S.NOP, 300)
    a.connect(P, E, capi.CONN_FIXED_OUTDEGREE, 0.0, wmin=4.0, wmax=9.0, degree=30, dmin=1, dmax=6, seed=3)
    oa = O.OracleNet(a, deterministic=True)
    rp, tg, w, d = oa.csr()
    base_p, base_e = oa.population_base(P), oa.population_base(E)
    rows = rp[base_p:base_p + 401] - rp[base_p]
    lo, hi = int(rp[base_p]), int(rp[base_p + 400])
    b = S.NetSpec(poisson_seed=5)
    P2 = b.add_pop(S.POISSON, 400, rate_hz=60.0)
    E2 = b.add_pop(S.NOP, 300)
    b.connect_csr(P2, E2, rows, tg[lo:hi] - base_e, w[lo:hi], d[lo:hi])
    ob = O.OracleNet(b, deterministic=True)
    for x, y in zip(oa.csr(), ob.csr()):
        assert np.array_equal(x, y)
    oa.run(500)
    ob.run(500)
    sa, ia = oa.spikes()
    sb, ib = ob.spikes()
    assert len(ia) > 100 and np.array_equal(sa, sb) and np.array_equal(ia, ib)


def test_exact_sum_mode(oracle_mod):
    """The oracle's exact-sum mode (weights on the grid 2^-S, integer ring
    sums): S from the largest possible cell sum, parallel runs with the
    same bits, and potentials within 1e-5 of FP64 on the same spikes."""
    O = oracle_mod
    s = S.brunel_small(poisson_weight=1.0).with_(exact=True)
    a, b = O.OracleNet(s, threads=1), O.OracleNet(s)
    assert 10 <= a.exact_shift() <= 30
    a.run(1500)
    b.run(1500)
    sa, sb = a.spikes(), b.spikes()
    assert np.array_equal(sa[0], sb[0]) and np.array_equal(sa[1], sb[1]) and len(sa[1]) > 1000
    v, _ = a.state()
    assert np.array_equal(v.view(np.uint32), b.state()[0].view(np.uint32))
    v64, _, _ = O.OracleNet(s).reintegrate_fp64(sa[0], sa[1], 1500)
    err = np.abs(v.astype(np.float64) - v64) / np.maximum(np.abs(v64), 1.0)
    assert err.max() <= 1e-5
    big = S.NetSpec(exact=True)
    A = big.add_pop(S.NOP, 500)
    big.connect(A, A, capi.CONN_FIXED_INDEGREE, 3.0e7, degree=200, seed=2)
    with pytest.raises(ValueError, match="exact-sum"):
        O.OracleNet(big)
