"""Regenerates tests/golden/oracle_brunel_small.npz: the oracle's raster and
membrane potentials for the driven small Brunel network (deterministic
aggregation, 500 steps).  A regression fixture of the oracle itself."""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from naer_b200 import spec as S  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    steps = 500
    o = O.OracleNet(S.brunel_small(poisson_weight=1.0), deterministic=True)
    o.run(steps)
    st, ids = o.spikes()
    v, _ = o.state()
    out = Path(__file__).resolve().parent / "oracle_brunel_small.npz"
    np.savez_compressed(out, steps=steps, spike_steps=st, spike_ids=ids, v=v)
    print(f"wrote {out}: {len(ids)} spikes")


if __name__ == "__main__":
    main()
