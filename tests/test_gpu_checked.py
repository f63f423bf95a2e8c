"""The bounds-checked build (libnaer_b200_checked.so, NAER_CHECKED) on the
networks and forms the other tests use: every global access of the step
kernels at a computed index is checked against its buffer, and no run may
record a violation.  It stands in for a sanitizer, which does not run on
this hardware's pool.  The checked library runs in a child process
(NAER_CHECKED=1 selects it at load); its deterministic raster must still
equal the oracle's."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent

CHILD = r"""
import ctypes as C, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
from naer_b200 import _capi as capi
from naer_b200 import spec as S
from naer_b200.forms import Batch
from nets import integer_weight_net, mixed_rules
from oracle import oracle as O
lib = capi.load()
flag = C.c_int()
capi.call("naer_build_checked", C.byref(flag))
out = {"checked": flag.value, "runs": []}

def report(net, name, steps):
    code, idx = C.c_uint32(), C.c_uint64()
    capi.call("naer_net_check_report", net.handle, C.byref(code), C.byref(idx))
    out["runs"].append({"net": name, "steps": steps, "code": code.value, "index": idx.value,
                        "spikes": int(net.stats()["spikes"])})

cases = [
    ("brunel_small det", S.brunel_small(poisson_weight=1.0).with_(deterministic=True), {}),
    ("plastic_indegree atomic", S.plastic_indegree(n=3000, k=200, drive_weight=21.0), {}),
    ("plastic_indegree det", S.plastic_indegree(n=3000, k=200, drive_weight=21.0).with_(deterministic=True), {}),
    ("mixed rules stdp det", mixed_rules(capi.CONN_FIXED_INDEGREE).with_(stdp_enabled=True, deterministic=True), {}),
    ("integer 300k one block per SM", integer_weight_net(n=300_000, k=20, seed=2), {"blocks_per_sm": 1}),
    ("integer 300k global state", integer_weight_net(n=300_000, k=20, seed=2), {"blocks_per_sm": 1,
                                                                                "neuron_state": 2}),
    ("integer two-barrier kernel", integer_weight_net(n=20000, k=100, seed=3), {"step_kernel": 1}),
]
for name, s, tuning in cases:
    with S.build(s) as net:
        if tuning:
            net.set_tuning(**tuning)
        net.run(600)
        net.finish()
        report(net, name, 600)
        if name == "brunel_small det":
            o = O.OracleNet(s, deterministic=True)
            o.run(600)
            st, ids = net.read_spikes()
            ost, oids = o.spikes()
            out["brunel_matches_oracle"] = bool(np.array_equal(st, ost) and np.array_equal(ids, oids))
members = S.batch_members(count=6, seed=3, n_range=(600, 4000), k_range=(50, 300), rate_range=(20.0, 60.0))
for det in (False, True):
    with Batch(members, deterministic=det).compile() as b:
        b.run(500)
        b.finish()
        out["runs"].append({"net": f"batch of 6 det={det}", "steps": 500, "spikes": int(b.stats()["spikes"])})
print(json.dumps(out))
"""


def test_checked_build_records_no_violation(lib):
    from naer_b200 import build as b
    b.build(checked=True)
    env = dict(os.environ, NAER_CHECKED="1")
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], capture_output=True, text=True, env=env,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["checked"] == 1
    assert out["brunel_matches_oracle"]
    for run in out["runs"]:
        assert run.get("code", 0) == 0, run
        assert run["spikes"] > 0, run
