"""The C-ABI library loads, exports every symbol include/naer/*.h declares,
and its parameter blocks have the layout the header describes.  No compute
calls: these run without a GPU."""
import ctypes as C
import re
import subprocess
import textwrap
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include" / "naer").glob("*.h"))


def declared_symbols():
    names = []
    for h in HEADERS:
        names += re.findall(r"NAER_API\s+[\w\s\*]+?\b(naer_\w+)\s*\(", h.read_text())
    return sorted(set(names))


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "naer_net_create" in names and "naer_net_step" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_defaults_and_last_error(lib):
    from naer_b200 import _capi as capi
    p = capi.NetParams()
    assert lib.naer_net_params_default(C.byref(p)) == 0
    assert p.dt_us == 100 and p.poisson_seed == 0x15AC7EBD and p.stdp_history == 10
    q = capi.PopParams()
    assert lib.naer_pop_params_default(capi.NEURON_POISSON, C.byref(q)) == 0
    assert q.rate_hz == pytest.approx(20.0) and q.v_th == pytest.approx(0.020)
    assert lib.naer_pop_params_default(7, C.byref(q)) == capi.NAER_E_INVALID
    assert "unknown neuron type" in capi.last_error()


def test_struct_layout_matches_header(lib, tmp_path):
    """Compile a probe against the header and compare sizes and offsets."""
    from naer_b200 import _capi as capi
    src = tmp_path / "probe.c"
    structs = {"naer_net_params": capi.NetParams, "naer_pop_params": capi.PopParams,
               "naer_conn_spec": capi.ConnSpecC, "naer_stats": capi.Stats, "naer_tuning": capi.Tuning,
               "naer_server_params": capi.ServerParams, "naer_job_info": capi.JobInfo,
               "naer_server_stats": capi.ServerStats, "naer_device_probe": capi.DeviceProbe}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "naer/naer_capi.h"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                          check=True).stdout.split("\n") if l)
    for cname, py in structs.items():
        assert int(out[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(out[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"


def test_cpp_wrapper_compiles(tmp_path):
    """include/naer/Network.h (the reference-shaped C++ API) compiles."""
    src = tmp_path / "use.cpp"
    src.write_text(textwrap.dedent("""
        #include "naer/Network.h"
        int main() {
            // model building as in the reference's main.cpp:32-50
            auto build = []() {
                Naer::Network net;
                auto P = net.addPopulation(Naer::NeuronType::POISSON, 100);
                auto E = net.addPopulation(Naer::NeuronType::NOP, 80);
                net.addConnection(P, E, 0.001f, 0.1);
                net.addConnection(E, E, 0.0f, 0.0f, 0.001f, 0.1, 42ull);
                net.compile();
                while (net.getTime() < 15000) net.step();
                net.finish();
                return net.getSynapses();
            };
            (void)build;
            return 0;
        }
    """))
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", str(ROOT / "include"), str(src)], check=True)


def test_cpp_forms_compile(tmp_path):
    """include/naer/Forms.h (batched and served forms for C++) compiles."""
    src = tmp_path / "forms.cpp"
    src.write_text(textwrap.dedent("""
        #include "naer/Forms.h"
        int main() {
            auto describe = [](Naer::Network& d) {
                auto P = d.addPopulation(Naer::NeuronType::POISSON, 100);
                auto E = d.addPopulation(Naer::NeuronType::NOP, 80);
                d.addConnection(P, E, 0.001f, 0.1);
            };
            auto use = [&]() {
                Naer::Network d(-1);            // description only
                describe(d);
                Naer::Batch b(0, true);
                b.add(d);
                b.add(d);
                b.compile();
                b.autotune(32);
                b.step(1000);
                b.finish();
                auto sp = b.readSpikes();
                Naer::Server srv(0);
                uint64_t job = srv.submit(d, 500);
                srv.wait(job, 60.0);
                auto js = srv.spikes(job);
                return sp.size() + js.size() + (size_t)srv.stats().done;
            };
            (void)use;
            return 0;
        }
    """))
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", str(ROOT / "include"), str(src)], check=True)


def test_create_without_gpu_fails_cleanly(lib):
    from conftest import HAS_GPU
    if HAS_GPU:
        pytest.skip("GPU present")
    from naer_b200 import _capi as capi
    n = C.c_int(-1)
    assert lib.naer_device_count(C.byref(n)) == 0
    assert n.value == 0
    h = C.c_void_p()
    st = lib.naer_net_create(0, None, C.byref(h))
    assert st in (capi.NAER_E_CUDA, capi.NAER_E_INVALID)
    assert not h.value
    assert capi.last_error()


def test_description_only_network(lib):
    """device -1: a description without device resources (the input of the
    batched and served forms); compiling it is refused."""
    from naer_b200 import _capi as capi
    from naer_b200 import spec as S
    d = S.describe(S.brunel_small(), -1)
    try:
        assert lib.naer_net_compile(d.handle) == capi.NAER_E_STATE
        assert "description-only" in capi.last_error()
        st = capi.Stats()
        assert lib.naer_net_get_stats(d.handle, C.byref(st)) == capi.NAER_E_STATE
    finally:
        d.close()
    h = C.c_void_p()
    assert lib.naer_net_create(-2, None, C.byref(h)) == capi.NAER_E_INVALID


def test_server_defaults(lib):
    from naer_b200 import _capi as capi
    p = capi.ServerParams()
    assert lib.naer_server_params_default(C.byref(p)) == 0
    assert p.budget_bytes == 150 * 10**9 and p.chunk_steps == 256 and p.aggregation == capi.AGG_ATOMIC
    assert p.launch_steps == 0  # library default
    assert p.step_kernel == capi.KERNEL_TWO_BARRIER
    p.step_kernel = 7  # refused before any device work
    h = C.c_void_p()
    assert lib.naer_server_create(0, C.byref(p), C.byref(h)) == capi.NAER_E_INVALID and not h.value


def test_forms_workloads():
    """The batched and served workload generators follow their stated ranges."""
    from naer_b200 import spec as S
    m = S.batch_members(count=64, seed=5)
    ns = [sum(p.size for p in x.pops) for x in m]
    assert min(ns) >= 2000 and max(ns) <= 50_000 and len(set(ns)) > 50
    assert any(x.stdp_enabled for x in m) and not all(x.stdp_enabled for x in m)
    jobs = S.served_jobs(count=200, seed=5)
    t = [j[0] for j in jobs]
    assert all(b > a for a, b in zip(t, t[1:]))
    assert 2.5 < t[-1] < 6.0  # 200 arrivals at 50/s
    assert all(1000 <= j[2] <= 20000 for j in jobs)
