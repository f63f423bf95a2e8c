"""Small seeded networks shared by the parity tests."""
from naer_b200 import _capi as capi
from naer_b200 import spec as S


def mixed_rules(rule) -> S.NetSpec:
    """Poisson, NOP and STDP populations, three connections of one rule with
    fixed, random and delayed weights."""
    s = S.NetSpec()
    P = s.add_pop(S.POISSON, 50, rate_hz=50.0)
    E = s.add_pop(S.NOP, 120)
    I = s.add_pop(S.STDP, 37)
    s.connect(P, E, rule, 0.5, probability=0.2, degree=7, dmin=1, dmax=5, seed=11)
    s.connect(E, I, rule, 0.0, probability=0.3, degree=5, wmin=0.1, wmax=0.4, dmin=2, dmax=2, seed=12)
    s.connect(E, E, rule, -0.2, probability=0.1, degree=3, dmin=1, dmax=9, seed=13)
    return s


def reference_brunel(n_syn: float = 2e5) -> S.NetSpec:
    """The reference's brunel() builder (src/main.cpp:32-50) in reference
    units (volts): N = floor(sqrt(S / 0.05)), P/E/I = N/2, 0.4 N, 0.1 N,
    weights 2/N and -10/N, p = 0.1, the shared default seed."""
    import math
    N = math.floor(math.sqrt(n_syn / 0.05))
    s = S.NetSpec(name="reference_brunel")
    lif = dict(v_th=0.020, v_reset=0.0, t_ref_ms=2.0, tau_m_ms=20.0)
    P = s.add_pop(S.POISSON, N // 2, rate_hz=20.0)
    E = s.add_pop(S.NOP, N * 4 // 10, **lif)
    I = s.add_pop(S.NOP, N // 10, **lif)
    R = capi.CONN_REF_BERNOULLI
    seed = 0xBF785E3215AC7EBD
    d = dict(dmin=15, dmax=15, seed=seed)
    for src, dst, w in [(P, E, 2.0 / N), (P, I, 2.0 / N), (E, E, 2.0 / N), (E, I, 2.0 / N),
                        (I, E, -10.0 / N), (I, I, -10.0 / N)]:
        s.connect(src, dst, R, w, probability=0.1, **d)
    return s


def integer_weight_net(n=6000, k=300, seed=3, stdp=False) -> S.NetSpec:
    """Fixed out-degree network whose weights and drive weight are integers
    (mV): every ring sum is exact in fp32, so the order of the atomic
    reductions cannot change any result."""
    s = S.NetSpec(name="integer_weights", stdp_enabled=stdp, poisson_seed=seed)
    ne = n * 4 // 5
    E = s.add_pop(S.NOP, ne, drive_rate_hz=40.0, drive_weight=21.0, drive_seed=7 + seed)
    I = s.add_pop(S.NOP, n - ne, drive_rate_hz=40.0, drive_weight=21.0, drive_seed=8 + seed)
    R = capi.CONN_FIXED_OUTDEGREE
    for src, w, sd in [(E, 1.0, 1), (I, -3.0, 2)]:
        s.connect(src, E, R, w, degree=k * 4 // 5, dmin=1, dmax=12, seed=seed * 100 + sd)
        s.connect(src, I, R, w, degree=k // 5, dmin=1, dmax=12, seed=seed * 100 + sd + 10)
    return s
