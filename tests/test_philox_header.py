"""The library's Philox header (naer_b200/csrc/philox.cuh), compiled for the
host, against the oracle: the full generator, and the form the Poisson-draw
kernel uses with the round-2 product supplied by the caller (CPU only)."""
import subprocess
from pathlib import Path

import numpy as np

from test_oracle import RANDOM123_KAT

ROOT = Path(__file__).resolve().parent.parent

CHECK = r"""
#include <cstdio>
#include "philox.cuh"
using namespace naer;
int main() {
    unsigned c0, c1, c2, c3, k0, k1;
    while (std::scanf("%u %u %u %u %u %u", &c0, &c1, &c2, &c3, &k0, &k1) == 6) {
        const u32x4 r = philox4x32_10(c0, c1, c2, c3, k0, k1);
        const uint64_t m = (uint64_t)kPhiloxM0 * k0;
        std::printf("%u %u %u %u %u %u\n", r.v[0], r.v[1], r.v[2], r.v[3], philox_ref_z(c0, k0, k1),
                    philox_ref_z_pre(c0, k0, k1, (uint32_t)(m >> 32), (uint32_t)m));
    }
    return 0;
}
"""


def test_header_philox_matches_oracle(tmp_path, oracle_mod):
    src = tmp_path / "check.cpp"
    exe = tmp_path / "check"
    src.write_text(CHECK)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "naer_b200" / "csrc"), "-o", str(exe), str(src)],
                   check=True)
    rng = np.random.default_rng(11)
    cases = [(c, k) for c, k, _ in RANDOM123_KAT]
    for _ in range(2000):
        ctr = [int(x) for x in rng.integers(0, 2**32, 4, dtype=np.uint64)]
        key = [int(x) for x in rng.integers(0, 2**32, 2, dtype=np.uint64)]
        cases.append((ctr, key))
    for i in range(64):  # the kernel's shape: counter {c0, 0, 0, 0}, small keys
        cases.append(([i * 1000 + 7, 0, 0, 0], [i, 0x15AC7EBD]))
    inp = "".join(" ".join(str(v) for v in c + k) + "\n" for c, k in cases)
    out = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    for (ctr, key), line in zip(cases, out):
        got = [int(v) for v in line.split()]
        full = list(oracle_mod.philox4x32_10(ctr, key))
        assert got[:4] == full, (ctr, key)
        z = list(oracle_mod.philox4x32_10([ctr[0], 0, 0, 0], key))[2]
        assert got[4] == z and got[5] == z, (ctr, key)
    for (ctr, key, want), line in zip(RANDOM123_KAT, out):
        assert [int(v) for v in line.split()][:4] == want
