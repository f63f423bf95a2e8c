"""The oracle against the reference's own kernels.

The reference's OpenCL C sources for the random numbers (random.cl), the
Poisson generators (input_neuron_group.cl:6-45), the neuron update
(lif.cl:15-34) and the connectivity builder (network.cl:14-107) compile
unchanged as C under a host work-group shim (oracle/ref/, `make -C oracle
ref`): every work-item a thread, `local` memory shared by the group,
barrier() a thread barrier.  Random123's philox.h, an un-vendored
submodule, is replaced by a restatement of the published algorithm,
itself checked against cuRAND here.

tests/golden/ref_kernels.npz holds the reference build's outputs
(tests/golden/gen_ref_fixtures.py), so these checks run where the
reference tree is absent; where the built library is present, fresh cases
are compared with it directly.  All bit for bit.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from naer_b200 import _capi as capi
from naer_b200 import spec as S
from oracle import ref as R

GOLDEN = Path(__file__).resolve().parent / "golden"
M = 0xFFFFFFFF


@pytest.fixture(scope="module")
def fx():
    return np.load(GOLDEN / "ref_kernels.npz")


live = pytest.mark.skipif(not R.available(), reason="reference kernels not built here (reference tree absent)")


def oracle_poisson(O, n, seed, t0, t1):
    times, addrs = [], []
    for idx in range(n):
        x = O.poisson_window(idx, n, seed, 20.0, t0, t1)
        times += list(x)
        addrs += [idx] * len(x)
    t = np.array(times, dtype=np.uint32)
    a = np.array(addrs, dtype=np.uint32)
    o = np.lexsort((t, a))
    return t[o], a[o]


def oracle_bernoulli(O, ns, nd, seed, p, w, wmin, wmax):
    s = S.NetSpec()
    A = s.add_pop(S.NOP, ns)
    B = s.add_pop(S.NOP, nd)
    s.connect(A, B, capi.CONN_REF_BERNOULLI, w, probability=p, wmin=wmin, wmax=wmax, seed=seed)
    o = O.OracleNet(s)
    rp, tg, ww, _ = o.csr()
    ba, bb = o.population_base(A), o.population_base(B)
    o.close()
    src, dst, wt = [], [], []
    for i in range(ns):
        t, x = tg[rp[ba + i]:rp[ba + i + 1]], ww[rp[ba + i]:rp[ba + i + 1]]
        m = t != 0xFFFFFFFF
        src += [i] * int(m.sum())
        dst += list(t[m] - bb)
        wt += list(x[m])
    src, dst = np.array(src, dtype=np.uint32), np.array(dst, dtype=np.uint32)
    wt = np.array(wt, dtype=np.float32)
    k = np.lexsort((dst, src))
    return src[k], dst[k], wt[k]


def test_uniform_rand_and_exprnd_match_reference(oracle_mod, fx):
    O = oracle_mod
    for (g, s, i), u in zip(fx["uniform_args"], fx["uniform_out"]):
        assert O.uniform_rand(int(g), int(s), int(i)) == u
    # (uint)exprnd(20 Hz) is the interval the generators add (input_neuron_group.cl:29,36)
    for (g, s, i), x in zip(fx["uniform_args"][:200], fx["exprnd_out"]):
        assert O.exp_interval_us(int(g), int(s), int(i), 20.0) == (int(x) if x < 2**32 else M)


def test_poisson_generators_match_reference(oracle_mod, fx):
    """Every spike of 5,000 generators in five windows (100 us and 1.5 ms,
    one past 2^31 us), as simulate_poisson_neurons emits it."""
    for k, (t0, t1) in enumerate(fx["poisson_windows"]):
        sel = fx["poisson_window"] == k
        t, a = oracle_poisson(oracle_mod, 5000, 7, int(t0), int(t1))
        assert np.array_equal(t, fx["poisson_time"][sel]) and np.array_equal(a, fx["poisson_address"][sel]), k
    assert len(fx["poisson_time"]) > 200


def test_bernoulli_connectivity_matches_reference(oracle_mod, fx):
    """count / integrate / generate_connections: the same synapses with the
    same weights, including the random weights drawn from the connection
    test's own draw (network.cl:97-100)."""
    for k, (ns, nd, seed, p, w, wmin, wmax) in enumerate(fx["bernoulli_cases"]):
        s, d, x = oracle_bernoulli(oracle_mod, int(ns), int(nd), int(seed), p, np.float32(w), np.float32(wmin),
                                   np.float32(wmax))
        assert np.array_equal(s, fx[f"bernoulli{k}_src"]) and np.array_equal(d, fx[f"bernoulli{k}_dst"]), k
        assert np.array_equal(x.view(np.uint32), fx[f"bernoulli{k}_w"].view(np.uint32)), k


@pytest.mark.parametrize("w", [0.008, 0.025])
def test_event_mode_neuron_matches_lif_cl(oracle_mod, fx, w):
    """The oracle's event mode (one 400 Hz generator, one synapse, 200
    windows of 1.5 ms) fires exactly where lif.cl's neuron_dynamics fires on
    the same input events, and ends at the same potential."""
    O = oracle_mod
    s = S.NetSpec()
    P = s.add_pop(S.POISSON, 1, rate_hz=400.0)
    E = s.add_pop(S.NOP, 1, v_th=0.020, v_reset=0.0, t_ref_ms=2.0, tau_m_ms=20.0)
    s.connect(P, E, capi.CONN_FIXED_OUTDEGREE, w, degree=1)
    o = O.OracleNet(s)
    o.run_events(200)
    t, ids = o.event_spikes()
    pt = np.sort(t[ids == o.population_base(P)])
    et = np.sort(t[ids == o.population_base(E)])
    ev, _, _ = o.event_state()
    v = ev[o.population_base(E)]
    o.close()
    assert np.array_equal(pt, fx["lif_times"])
    tag = f"{int(w * 1000):03d}"
    fired = fx[f"lif{tag}_fired"]
    assert fired.sum() > 0
    assert np.array_equal(et, pt[fired])
    assert np.float32(v) == fx[f"lif{tag}_v"]


def test_reference_philox_stand_in_matches_curand(fx):
    """The Philox4x32-10 restatement the reference build uses in place of
    Random123 reproduces cuRAND's Philox4_32_10 (vectors from a B200)."""
    if not R.available():
        pytest.skip("reference kernels not built here")
    data = json.loads((GOLDEN / "philox_curand.json").read_text())
    for case in data["cases"]:
        seed, subseq, offset = case["seed"], case["subsequence"], case["offset"]
        blk = offset // 4
        ctr = [blk & M, blk >> 32, subseq & M, subseq >> 32]
        assert list(R.philox4x32(ctr, [seed & M, seed >> 32])) == case["out"], case


@live
def test_fresh_cases_against_reference_build(oracle_mod):
    """New seeds and windows, compared with the reference build directly."""
    O = oracle_mod
    rng = np.random.default_rng(77)
    for _ in range(300):
        g, s, i = (int(x) for x in rng.integers(0, 2**32, 3, dtype=np.uint64))
        assert O.uniform_rand(g, s, i) == R.uniform_rand(g, s, i)
    for t0, t1 in [(777, 877), (10_000_000, 10_001_500)]:
        rt, ra = R.poisson_neurons(4100, 0x15AC7EBD, t0, t1)
        ot, oa = oracle_poisson(O, 4100, 0x15AC7EBD, t0, t1)
        assert np.array_equal(rt, ot) and np.array_equal(ra, oa)
    rs, rd, rw = R.bernoulli(150, 900, 4242, 0.1, 0.0, -0.2, 0.4)
    os_, od, ow = oracle_bernoulli(O, 150, 900, 4242, 0.1, np.float32(0.0), np.float32(-0.2), np.float32(0.4))
    assert np.array_equal(rs, os_) and np.array_equal(rd, od)
    assert np.array_equal(rw.view(np.uint32), ow.view(np.uint32))
