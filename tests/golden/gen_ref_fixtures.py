"""Generates tests/golden/ref_kernels.npz from the reference's own kernels
(random.cl, input_neuron_group.cl, lif.cl, network.cl), compiled from the
reference tree under the host work-group shim (`make -C oracle ref`, which
reads the kernels at /root/reference/include/naer/kernels).

The fixture lets the oracle be checked against the reference's code where
the reference tree is absent.  Run from the repository root:
    python tests/golden/gen_ref_fixtures.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import ref as R  # noqa: E402

# the event-mode workload of the lif.cl check: one 400 Hz generator driving
# one neuron through one synapse, 200 windows of 1500 us
LIF_WEIGHTS = (0.008, 0.025)
LIF_SEED = 0x15AC7EBD  # the network spec's default Poisson seed
POISSON_N, POISSON_SEED = 5000, 7
POISSON_WINDOWS = [(0, 100), (100, 200), (1500, 3000), (123456, 124956), (2**31 + 77, 2**31 + 177)]
BERNOULLI = [  # (sources, destinations, seed, p, weight, wmin, wmax)
    (100, 600, 5, 0.05, 0.1, 0.0, 1.0),
    (80, 700, 99, 0.2, 0.0, 0.05, 0.3),
    (32, 300, 1, 0.5, -0.5, 0.0, 1.0),
]


def main():
    if R.build() is None:
        raise SystemExit("the reference kernels could not be built (reference tree absent)")
    rng = np.random.default_rng(2026)
    out = {}
    ctr = rng.integers(0, 2**32, (64, 4), dtype=np.uint64).astype(np.uint32)
    key = rng.integers(0, 2**32, (64, 2), dtype=np.uint64).astype(np.uint32)
    out["philox_ctr"], out["philox_key"] = ctr, key
    out["philox_out"] = np.stack([R.philox4x32(c, k) for c, k in zip(ctr, key)])
    u = rng.integers(0, 2**32, (500, 3), dtype=np.uint64).astype(np.uint32)
    out["uniform_args"] = u
    out["uniform_out"] = np.array([R.uniform_rand(int(g), int(s), int(i)) for g, s, i in u])
    out["exprnd_out"] = np.array([R.exprnd(int(g), 20.0, int(s), int(i)) for g, s, i in u[:200]])
    pw, pt, pa = [], [], []
    for k, (t0, t1) in enumerate(POISSON_WINDOWS):
        t, a = R.poisson_neurons(POISSON_N, POISSON_SEED, t0, t1)
        pw += [k] * len(t)
        pt.append(t)
        pa.append(a)
    out["poisson_windows"] = np.array(POISSON_WINDOWS, dtype=np.uint64)
    out["poisson_window"] = np.array(pw, dtype=np.uint32)
    out["poisson_time"] = np.concatenate(pt)
    out["poisson_address"] = np.concatenate(pa)
    for k, (ns, nd, seed, p, w, wmin, wmax) in enumerate(BERNOULLI):
        s, d, x = R.bernoulli(ns, nd, seed, p, w, wmin, wmax)
        out[f"bernoulli{k}_src"], out[f"bernoulli{k}_dst"], out[f"bernoulli{k}_w"] = s, d, x
    out["bernoulli_cases"] = np.array(BERNOULLI, dtype=np.float64)
    # lif.cl on the generator's own event times (the oracle's windows of the
    # 400 Hz source, which the Poisson check above pins to the reference)
    from oracle import oracle as O
    times = np.concatenate([O.poisson_window(0, 1, LIF_SEED, 400.0, 1500 * k, 1500 * (k + 1)) for k in range(200)])
    out["lif_times"] = times
    for w in LIF_WEIGHTS:
        fired, v, tl = R.neuron_dynamics(times, np.full(len(times), w, dtype=np.float32))
        tag = f"{int(w * 1000):03d}"
        out[f"lif{tag}_fired"] = fired
        out[f"lif{tag}_v"] = np.float32(v)
        out[f"lif{tag}_tlast"] = np.uint32(tl)
    np.savez_compressed(ROOT / "tests" / "golden" / "ref_kernels.npz", **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
