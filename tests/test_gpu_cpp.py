"""The C++ boundary, compiled, linked and run on the GPU.

A program written against include/naer/Network.h with the reference's call
sequence (src/main.cpp:94-126: addPopulation per type, both addConnection
overloads, compile, step() until getTime() reaches the end, finish) is
built with g++ against libnaer_b200.so and run.  Its raster must equal the
raster of the same network driven through the Python binding of the C ABI,
bit for bit (deterministic aggregation).  A second program uses
include/naer/Forms.h: two members in a Naer::Batch must each reproduce the
plain run of the same description.
"""
import subprocess
import textwrap
from pathlib import Path

import numpy as np
import pytest

from naer_b200 import _capi as capi
from naer_b200 import Network, NeuronType
from naer_b200 import spec as S

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent

PROGRAM = r"""
#include <cstdio>
#include <vector>
#include "naer/Network.h"

int main() {
    naer_net_params p;
    Naer::check(naer_net_params_default(&p));
    p.aggregation = NAER_AGG_DETERMINISTIC;
    Naer::Network net(0, &p);
    naer_pop_params pp;
    Naer::check(naer_pop_params_default(NAER_NEURON_POISSON, &pp));
    pp.rate_hz = 40.0f;
    auto P = net.addPopulation(Naer::NeuronType::POISSON, 600, &pp);
    Naer::check(naer_pop_params_default(NAER_NEURON_NOP, &pp));
    pp.v_th = 0.02f;
    auto E = net.addPopulation(Naer::NeuronType::NOP, 400, &pp);
    auto I = net.addPopulation(Naer::NeuronType::NOP, 100, &pp);
    net.addConnection(P, E, 0.004f, 0.3);
    net.addConnection(P, I, 0.004f, 0.3);
    net.addConnection(E, I, 0.0f, 0.001f, 0.003f, 0.2, 1234ull);
    net.addConnection(I, E, -0.01f, 0.1);
    net.compile();
    std::printf("bases %u %u %u\n", P->baseAddress, E->baseAddress, I->baseAddress);
    while (net.getTime() < 300000) net.step();  // 0.3 s of 1.5 ms windows
    net.finish();
    std::vector<uint32_t> steps, ids;
    net.readSpikes(steps, ids);
    std::printf("neurons %u synapses %u time %u spikes %zu\n", net.getNeurons(), net.getSynapses(), net.getTime(),
                ids.size());
    for (size_t i = 0; i < ids.size(); ++i) std::printf("%u %u\n", steps[i], ids[i]);
    return 0;
}
"""

BATCH_PROGRAM = r"""
#include <cstdio>
#include "naer/Forms.h"

static void describe(Naer::Network& d, uint32_t n, uint64_t seed) {
    naer_pop_params pp;
    Naer::check(naer_pop_params_default(NAER_NEURON_NOP, &pp));
    pp.v_th = 20.0f; pp.v_reset = 10.0f; pp.drive_rate_hz = 40.0f; pp.drive_weight = 21.0f;
    pp.drive_seed = (uint32_t)seed;
    auto E = d.addPopulation(Naer::NeuronType::NOP, n, &pp);
    naer_conn_spec c{};
    c.rule = NAER_CONN_FIXED_OUTDEGREE; c.degree = 50; c.weight = 1.0f; c.delay_min = 1; c.delay_max = 8;
    c.seed = seed;
    d.connect(*E, *E, c);
}

int main() {
    naer_net_params p;
    Naer::check(naer_net_params_default(&p));
    Naer::Network a(-1, &p), b(-1, &p);
    describe(a, 3000, 7);
    describe(b, 1700, 8);
    Naer::Batch batch(0, true);
    batch.add(a);
    batch.add(b);
    batch.compile();
    batch.step(500);
    batch.finish();
    for (const auto& s : batch.readSpikes()) std::printf("%u %u %u\n", s.member, s.step, s.address);
    return 0;
}
"""


def build_and_run(tmp_path, source, name):
    src = tmp_path / f"{name}.cpp"
    src.write_text(textwrap.dedent(source))
    exe = tmp_path / name
    lib = ROOT / "naer_b200"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"), "-o", str(exe), str(src),
                    "-L", str(lib), "-lnaer_b200", f"-Wl,-rpath,{lib}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    return out.stdout.splitlines()


def test_reference_call_sequence_from_cpp(lib, tmp_path):
    lines = build_and_run(tmp_path, PROGRAM, "app")
    bases = [int(x) for x in lines[0].split()[1:]]
    head = lines[1].split()
    n_cpp, syn_cpp, t_cpp, nsp = int(head[1]), int(head[3]), int(head[5]), int(head[7])
    rec = np.array([[int(a) for a in l.split()] for l in lines[2:]], dtype=np.uint32).reshape(-1, 2)
    assert len(rec) == nsp > 500
    # the same calls through the Python binding of the C ABI
    net = Network(aggregation=capi.AGG_DETERMINISTIC)
    P = net.addPopulation(NeuronType.POISSON, 600, rate_hz=40.0)
    E = net.addPopulation(NeuronType.NOP, 400, v_th=0.02)
    I = net.addPopulation(NeuronType.NOP, 100, v_th=0.02)
    net.addConnection(P, E, 0.004, 0.3)
    net.addConnection(P, I, 0.004, 0.3)
    net.addConnection(E, I, 0.0, 0.001, 0.003, 0.2, 1234)
    net.addConnection(I, E, -0.01, 0.1)
    net.compile()
    assert [P.baseAddress, E.baseAddress, I.baseAddress] == bases == [500, 0, 400]
    while net.getTime() < 300_000:
        net.step()
    net.finish()
    st, ids = net.read_spikes()
    assert (net.getNeurons(), net.getSynapses(), net.getTime()) == (n_cpp, syn_cpp, t_cpp)
    net.close()
    assert np.array_equal(rec[:, 0], st) and np.array_equal(rec[:, 1], ids)


def test_batch_from_cpp(lib, tmp_path):
    rec = np.array([[int(a) for a in l.split()] for l in build_and_run(tmp_path, BATCH_PROGRAM, "batch")],
                   dtype=np.uint32).reshape(-1, 3)
    for member, n, seed in [(0, 3000, 7), (1, 1700, 8)]:
        s = S.NetSpec(deterministic=True)
        E = s.add_pop(S.NOP, n, drive_rate_hz=40.0, drive_weight=21.0, drive_seed=seed)
        s.connect(E, E, capi.CONN_FIXED_OUTDEGREE, 1.0, degree=50, dmin=1, dmax=8, seed=seed)
        with S.build(s) as net:
            net.run(500)
            net.finish()
            st, ids = net.read_spikes()
        m = rec[rec[:, 0] == member]
        assert len(ids) > 200
        assert np.array_equal(m[:, 1], st) and np.array_equal(m[:, 2], ids)
