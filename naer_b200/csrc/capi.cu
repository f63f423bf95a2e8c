// extern "C" boundary: every entry point of include/naer/naer_capi.h.
#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/naer/naer_capi.h"
#include "engine.h"
#include "forms.h"

using naer::Error;

struct naer_net {
    std::unique_ptr<naer::Engine> eng;  // null for a description-only handle
    naer::NetHost net;
    uint32_t type_count[3] = {0, 0, 0};
};

struct naer_batch {
    std::unique_ptr<naer::Batch> b;
    uint32_t graph_launches = 16;
};

struct naer_server {
    std::unique_ptr<naer::Server> s;
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return NAER_OK;
    } catch (const Error& e) {
        return fail(e.code, e.what());
    } catch (const std::bad_alloc&) {
        return fail(NAER_E_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(NAER_E_INVALID, e.what());
    }
}

void need(bool ok, int code, const char* msg) {
    if (!ok) throw Error(code, msg);
}

void need_compiled(const naer_net* n) {
    need(n != nullptr, NAER_E_INVALID, "null network handle");
    need(n->net.compiled, NAER_E_STATE, "network is not compiled");
}

}  // namespace

extern "C" {

int naer_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return NAER_E_INVALID;
    const size_t n = std::min(len - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), n);
    buf[n] = '\0';
    return NAER_OK;
}

int naer_device_count(int* count) {
    return guarded([&] {
        need(count != nullptr, NAER_E_INVALID, "null pointer");
        int n = 0;
        const cudaError_t e = cudaGetDeviceCount(&n);
        if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) {
            (void)cudaGetLastError();
            n = 0;
        } else {
            NAER_CK(e);
        }
        *count = n;
    });
}

int naer_net_params_default(naer_net_params* p) {
    if (!p) return fail(NAER_E_INVALID, "null pointer");
    std::memset(p, 0, sizeof(*p));
    p->mode = NAER_MODE_GRID;
    p->aggregation = NAER_AGG_ATOMIC;
    p->dt_us = 100;
    p->record_spikes = 1;
    p->raster_capacity = 1ull << 24;
    p->poisson_seed = 0x15ac7ebdu;  // (uint32_t)0xbf785e3215ac7ebd, Network.cpp:124
    p->stdp_enabled = 0;
    p->tau_plus_ms = 20.0f;
    p->tau_minus_ms = 20.0f;
    p->a_plus = 0.01f;
    p->a_minus = 0.0105f;
    p->w_max = 0.5f;
    p->stdp_history = 10;  // NAER_HIST_LENGTH, stdp_group.cl:4
    return NAER_OK;
}

int naer_pop_params_default(uint32_t neuron_type, naer_pop_params* p) {
    if (!p) return fail(NAER_E_INVALID, "null pointer");
    if (neuron_type > NAER_NEURON_POISSON) return fail(NAER_E_INVALID, "unknown neuron type");
    std::memset(p, 0, sizeof(*p));
    // reference constants: lif.cl:3-6, input_neuron_group.cl:4
    p->tau_m_ms = 20.0f;
    p->v_th = 0.020f;
    p->v_reset = 0.0f;
    p->t_ref_ms = 2.0f;
    p->v_init = 0.0f;
    p->rate_hz = neuron_type == NAER_NEURON_POISSON ? 20.0f : 0.0f;
    return NAER_OK;
}

int naer_net_create(int device, const naer_net_params* params, naer_net** out) {
    return guarded([&] {
        need(out != nullptr, NAER_E_INVALID, "null output pointer");
        *out = nullptr;
        naer_net_params p;
        if (params) p = *params; else naer_net_params_default(&p);
        need(p.mode == NAER_MODE_GRID || p.mode == NAER_MODE_EVENT, NAER_E_INVALID, "unknown mode");
        need(p.aggregation <= NAER_AGG_EXACT, NAER_E_INVALID, "unknown aggregation");
        need(p.dt_us > 0, NAER_E_INVALID, "dt_us must be positive");
        if (p.mode == NAER_MODE_EVENT)
            throw Error(NAER_E_UNSUPPORTED, "event mode is not available in this build");
        need(device >= -1, NAER_E_INVALID, "device index out of range");
        auto n = std::make_unique<naer_net>();
        n->net.params = p;
        if (device >= 0) n->eng = std::make_unique<naer::Engine>(device);
        *out = n.release();
    });
}

int naer_net_destroy(naer_net* net) {
    if (!net) return NAER_OK;
    return guarded([&] {
        if (net->net.compiled) net->eng->free_net(net->net);
        delete net;
    });
}

int naer_net_add_population(naer_net* net, uint32_t neuron_type, uint32_t size,
                            const naer_pop_params* params, uint32_t* pop_id, uint32_t* type_address) {
    return guarded([&] {
        need(net != nullptr, NAER_E_INVALID, "null network handle");
        need(!net->net.compiled, NAER_E_STATE, "network already compiled");
        need(neuron_type <= NAER_NEURON_POISSON, NAER_E_INVALID, "unknown neuron type");
        uint64_t total = (uint64_t)net->type_count[0] + net->type_count[1] + net->type_count[2] + size;
        need(total < 0x7FFFFFF0ull, NAER_E_INVALID, "too many neurons");
        naer::PopSpec ps;
        ps.type = neuron_type;
        ps.size = size;
        if (params) ps.prm = *params; else naer_pop_params_default(neuron_type, &ps.prm);
        ps.type_address = net->type_count[neuron_type];
        net->type_count[neuron_type] += size;
        net->net.pops.push_back(ps);
        if (pop_id) *pop_id = (uint32_t)net->net.pops.size() - 1;
        if (type_address) *type_address = ps.type_address;
    });
}

int naer_net_add_connection(naer_net* net, uint32_t src_pop, uint32_t dst_pop,
                            const naer_conn_spec* spec) {
    return guarded([&] {
        need(net != nullptr && spec != nullptr, NAER_E_INVALID, "null argument");
        need(!net->net.compiled, NAER_E_STATE, "network already compiled");
        need(src_pop < net->net.pops.size() && dst_pop < net->net.pops.size(), NAER_E_INVALID,
             "unknown population");
        need(spec->rule != NAER_CONN_EXPLICIT, NAER_E_INVALID,
             "explicit connectivity is added with naer_net_add_connection_csr");
        naer::ConnSpec c;
        c.src = src_pop;
        c.dst = dst_pop;
        c.spec = *spec;
        net->net.conns.push_back(c);
    });
}

int naer_net_add_connection_csr(naer_net* net, uint32_t src_pop, uint32_t dst_pop, const uint64_t* row_ptr,
                                const uint32_t* targets, const float* weights, const uint8_t* delays) {
    return guarded([&] {
        need(net != nullptr && row_ptr != nullptr, NAER_E_INVALID, "null argument");
        need(!net->net.compiled, NAER_E_STATE, "network already compiled");
        need(src_pop < net->net.pops.size() && dst_pop < net->net.pops.size(), NAER_E_INVALID,
             "unknown population");
        const uint32_t ns = net->net.pops[src_pop].size, nd = net->net.pops[dst_pop].size;
        need(row_ptr[0] == 0, NAER_E_INVALID, "row_ptr[0] must be 0");
        for (uint32_t r = 0; r < ns; ++r)
            need(row_ptr[r + 1] >= row_ptr[r], NAER_E_INVALID, "row_ptr must not decrease");
        const uint64_t nnz = row_ptr[ns];
        need(nnz == 0 || (targets && weights && delays), NAER_E_INVALID, "null synapse arrays");
        need(nnz < (1ull << 40), NAER_E_INVALID, "too many synapses");
        auto x = std::make_shared<naer::ExplicitCsr>();
        x->row_ptr.assign(row_ptr, row_ptr + ns + 1);
        x->tgt.assign(targets, targets + nnz);
        x->w.assign(weights, weights + nnz);
        x->dly.assign(delays, delays + nnz);
        uint32_t dmin = 254, dmax = 1;
        for (uint64_t j = 0; j < nnz; ++j) {
            need(x->tgt[j] < nd, NAER_E_INVALID, "target index outside the destination population");
            need(x->dly[j] >= 1 && x->dly[j] <= 254, NAER_E_INVALID, "delays must be in 1..254 steps");
            dmin = std::min<uint32_t>(dmin, x->dly[j]);
            dmax = std::max<uint32_t>(dmax, x->dly[j]);
        }
        naer::ConnSpec c;
        c.src = src_pop;
        c.dst = dst_pop;
        c.spec.rule = NAER_CONN_EXPLICIT;
        c.spec.delay_min = nnz ? dmin : 1;
        c.spec.delay_max = nnz ? dmax : 1;
        c.csr = std::move(x);
        net->net.conns.push_back(std::move(c));
    });
}

int naer_net_compile(naer_net* net) {
    return guarded([&] {
        need(net != nullptr, NAER_E_INVALID, "null network handle");
        need(!net->net.compiled, NAER_E_STATE, "network already compiled");
        need(net->eng != nullptr, NAER_E_STATE,
             "description-only network (device -1): add it to a batch or submit it to a server");
        net->eng->build(net->net);
        const auto& P = net->net.params;
        try {
            net->eng->install({&net->net}, P.raster_capacity, P.record_spikes != 0, P.aggregation);
        } catch (...) {
            net->eng->free_net(net->net);  // compile either completes or leaves nothing built
            throw;
        }
    });
}

int naer_net_population_base(naer_net* net, uint32_t pop_id, uint32_t* base_address) {
    return guarded([&] {
        need_compiled(net);
        need(pop_id < net->net.pops.size() && base_address, NAER_E_INVALID, "bad argument");
        *base_address = net->net.pops[pop_id].id_base;
    });
}

int naer_net_step(naer_net* net, uint64_t nsteps) {
    return guarded([&] {
        need_compiled(net);
        net->eng->run(nsteps);
    });
}

int naer_net_step_noalloc(naer_net* net, uint64_t nsteps) {
    return guarded([&] {
        need_compiled(net);
        net->eng->run_fixed_scratch(nsteps);
    });
}

namespace {
void throw_device_status(naer::Engine& eng) {
    const int st = eng.device_status();
    if (st == NAER_E_TIMEOUT)
        throw Error(NAER_E_TIMEOUT, "a grid barrier of the step kernel ran out of its wait limit; the network's "
                                    "state is undefined");
    if (st) throw Error(st, "the device reported an error");
}
}  // namespace

int naer_net_finish(naer_net* net) {
    return guarded([&] {
        need_compiled(net);
        net->eng->sync();
        throw_device_status(*net->eng);
    });
}

namespace {
// Header of a checkpoint: the layout it was taken from (checked on restore)
// and the counters it restores.
struct CheckpointHeader {
    char magic[8];
    uint32_t version, stdp_on;
    uint64_t step, events, payload;
    uint64_t synapses, synapses_padded;
    uint32_t n_ids, n_storage, ring_slots, n_plastic, post_stride, dt_us;
    int32_t ring_shift;  // exact-sum aggregation: the ring's integer grid 2^-S; -1: float ring
    uint32_t pad_;
};
constexpr char kCheckpointMagic[8] = {'N', 'A', 'E', 'R', 'C', 'K', 'P', 'T'};

CheckpointHeader checkpoint_header(naer::Engine& eng, const naer::NetHost& n) {
    CheckpointHeader h{};
    std::memcpy(h.magic, kCheckpointMagic, 8);
    h.version = 2;
    h.stdp_on = n.dev.stdp_on;
    h.step = eng.host_step();
    h.events = eng.events_total();
    h.payload = naer::state_bytes(n);
    h.synapses = n.synapses;
    h.synapses_padded = n.synapses_padded;
    h.n_ids = n.n_ids;
    h.n_storage = n.n_storage;
    h.ring_slots = n.ring_slots;
    h.n_plastic = n.dev.stdp_on ? n.n_plastic : 0;
    h.post_stride = n.post_stride;
    h.dt_us = n.params.dt_us;
    h.ring_shift = n.params.aggregation == NAER_AGG_EXACT ? n.fx_shift : -1;
    return h;
}
}  // namespace

int naer_net_checkpoint_size(naer_net* net, uint64_t* bytes) {
    return guarded([&] {
        need_compiled(net);
        need(bytes != nullptr, NAER_E_INVALID, "null argument");
        *bytes = sizeof(CheckpointHeader) + naer::state_bytes(net->net);
    });
}

int naer_net_checkpoint(naer_net* net, void* buf, uint64_t capacity) {
    return guarded([&] {
        need_compiled(net);
        need(buf != nullptr, NAER_E_INVALID, "null buffer");
        need(capacity >= sizeof(CheckpointHeader) + naer::state_bytes(net->net), NAER_E_OVERFLOW,
             "buffer smaller than naer_net_checkpoint_size");
        net->eng->sync();
        throw_device_status(*net->eng);
        const CheckpointHeader h = checkpoint_header(*net->eng, net->net);
        std::memcpy(buf, &h, sizeof(h));
        net->eng->save_state(net->net, static_cast<uint8_t*>(buf) + sizeof(h));
    });
}

int naer_net_restore(naer_net* net, const void* buf, uint64_t size) {
    return guarded([&] {
        need_compiled(net);
        need(buf != nullptr && size >= sizeof(CheckpointHeader), NAER_E_INVALID, "not a checkpoint");
        CheckpointHeader h;
        std::memcpy(&h, buf, sizeof(h));
        need(std::memcmp(h.magic, kCheckpointMagic, 8) == 0 && h.version == 2, NAER_E_INVALID, "not a checkpoint");
        net->eng->sync();
        const CheckpointHeader mine = checkpoint_header(*net->eng, net->net);
        need(h.stdp_on == mine.stdp_on && h.payload == mine.payload && h.synapses == mine.synapses &&
                 h.synapses_padded == mine.synapses_padded && h.n_ids == mine.n_ids &&
                 h.n_storage == mine.n_storage && h.ring_slots == mine.ring_slots &&
                 h.n_plastic == mine.n_plastic && h.post_stride == mine.post_stride && h.dt_us == mine.dt_us &&
                 h.ring_shift == mine.ring_shift,
             NAER_E_INVALID, "checkpoint was taken from a network of another layout");
        need(size >= sizeof(h) + h.payload, NAER_E_INVALID, "checkpoint truncated");
        net->eng->load_state(net->net, static_cast<const uint8_t*>(buf) + sizeof(h));
        net->eng->set_step(h.step, h.events);
    });
}

int naer_net_set_wait_limit(naer_net* net, uint64_t limit_us) {
    return guarded([&] {
        need_compiled(net);
        need(limit_us <= 3600ull * 1000 * 1000, NAER_E_INVALID, "wait limit above one hour");
        net->eng->set_barrier_limit(limit_us * 1000ull);
    });
}

int naer_test_set_barrier_skew(naer_net* net, uint64_t skew) {
    return guarded([&] {
        need_compiled(net);
        net->eng->set_barrier_skew(skew);
    });
}

int naer_probe_intervals(int device, double rate_hz, uint32_t z_first, uint32_t z_step, uint64_t count,
                         uint32_t* out) {
    return guarded([&] {
        need(out != nullptr || count == 0, NAER_E_INVALID, "null argument");
        need(rate_hz > 0.0, NAER_E_INVALID, "rate must be positive");
        int n = 0;
        NAER_CK(cudaGetDeviceCount(&n));
        need(device >= 0 && device < n, NAER_E_INVALID, "device index out of range");
        naer::probe_intervals(device, rate_hz, z_first, z_step, count, out);
    });
}

int naer_build_checked(int* checked) {
    return guarded([&] {
        need(checked != nullptr, NAER_E_INVALID, "null argument");
#ifdef NAER_CHECKED
        *checked = 1;
#else
        *checked = 0;
#endif
    });
}

int naer_net_check_report(naer_net* net, uint32_t* code, uint64_t* index) {
    return guarded([&] {
        need_compiled(net);
        need(code != nullptr && index != nullptr, NAER_E_INVALID, "null argument");
        const naer::Ctl c = net->eng->read_ctl();
        *code = c.chk_code;
        *index = c.chk_index;
    });
}

int naer_test_fail_allocation(int64_t after) {
    return guarded([&] {
        need(after >= -1, NAER_E_INVALID, "after must be >= -1");
        naer::set_allocation_failure(after);
    });
}

int naer_probe_device(int device, uint64_t ring_cells, uint64_t small_cells, naer_device_probe* out) {
    return guarded([&] {
        need(out != nullptr, NAER_E_INVALID, "null argument");
        int n = 0;
        NAER_CK(cudaGetDeviceCount(&n));
        need(device >= 0 && device < n, NAER_E_INVALID, "device index out of range");
        naer::probe_device(device, ring_cells, small_cells, out);
    });
}

int naer_net_get_time_us(naer_net* net, uint64_t* time_us) {
    return guarded([&] {
        need(net && time_us, NAER_E_INVALID, "null argument");
        *time_us = net->eng->host_step() * (uint64_t)net->net.params.dt_us;
    });
}

int naer_net_get_synapses(naer_net* net, uint64_t* synapses) {
    return guarded([&] {
        need(net && synapses, NAER_E_INVALID, "null argument");
        *synapses = net->net.synapses;
    });
}

int naer_net_get_neurons(naer_net* net, uint32_t* neurons) {
    return guarded([&] {
        need(net && neurons, NAER_E_INVALID, "null argument");
        *neurons = net->type_count[0] + net->type_count[1] + net->type_count[2];
    });
}

int naer_net_get_stats(naer_net* net, naer_stats* st) {
    return guarded([&] {
        need_compiled(net);
        need(st != nullptr, NAER_E_INVALID, "null argument");
        const naer::Ctl c = net->eng->read_ctl();
        std::memset(st, 0, sizeof(*st));
        st->step = c.step;
        st->events = net->eng->events_total();
        st->spikes = std::min<uint64_t>(c.raster_next, net->net.params.raster_capacity);
        st->raster_dropped = c.raster_dropped;
        st->stdp_hist_overflow = net->eng->overflow_total();
        st->synapses = net->net.synapses;
        st->device_bytes = net->eng->device_bytes();
        st->neurons = net->net.n_ids;
        st->ring_slots = net->net.ring_slots;
        st->kernel_launches = net->eng->kernel_launches();
    });
}

int naer_net_read_spikes(naer_net* net, uint64_t first, uint64_t capacity, uint32_t* steps,
                         uint32_t* ids, uint64_t* count) {
    return guarded([&] {
        need_compiled(net);
        need(count != nullptr && (capacity == 0 || (steps && ids)), NAER_E_INVALID, "null argument");
        *count = net->eng->read_raster(first, capacity, steps, ids);
    });
}

int naer_net_read_raster(naer_net* net, uint64_t first, uint64_t capacity, uint32_t* records,
                         uint64_t* count) {
    return guarded([&] {
        need_compiled(net);
        need(count != nullptr && (capacity == 0 || records), NAER_E_INVALID, "null argument");
        *count = net->eng->read_raster_raw(first, capacity, records);
    });
}

int naer_net_stream(naer_net* net, void** stream) {
    return guarded([&] {
        need(net != nullptr && stream != nullptr, NAER_E_INVALID, "null argument");
        *stream = (void*)net->eng->stream();
    });
}

int naer_net_clear_spikes(naer_net* net) {
    return guarded([&] {
        need_compiled(net);
        net->eng->clear_raster();
    });
}

namespace {

void read_state_of(naer::Engine& eng, const naer::NetHost& n, float* v, uint32_t* refractory) {
    std::vector<float> hv(n.n_storage);
    std::vector<uint8_t> hr(n.n_storage);
    eng.sync();
    int prev = -1;
    NAER_CK(cudaGetDevice(&prev));
    NAER_CK(cudaSetDevice(eng.device()));
    const cudaError_t e1 = cudaMemcpy(hv.data(), n.v, n.n_storage * 4ull, cudaMemcpyDeviceToHost);
    const cudaError_t e2 = cudaMemcpy(hr.data(), n.refr, n.n_storage, cudaMemcpyDeviceToHost);
    cudaSetDevice(prev);
    NAER_CK(e1);
    NAER_CK(e2);
    for (const auto& p : n.pops) {
        const bool lif = p.type != naer::kPOISSON;
        for (uint32_t k = 0; k < p.size; ++k) {
            if (v) v[p.id_base + k] = lif ? hv[p.storage_base + k] : 0.0f;
            if (refractory) refractory[p.id_base + k] = lif ? hr[p.storage_base + k] : 0u;
        }
    }
}

}  // namespace

int naer_net_read_state(naer_net* net, float* v, uint32_t* refractory) {
    return guarded([&] {
        need_compiled(net);
        read_state_of(*net->eng, net->net, v, refractory);
    });
}

int naer_net_write_state(naer_net* net, const float* v, const uint32_t* refractory) {
    return guarded([&] {
        need_compiled(net);
        const auto& n = net->net;
        std::vector<float> hv(n.n_storage);
        std::vector<uint8_t> hr(n.n_storage);
        net->eng->sync();
        NAER_CK(cudaMemcpy(hv.data(), n.v, n.n_storage * 4ull, cudaMemcpyDeviceToHost));
        NAER_CK(cudaMemcpy(hr.data(), n.refr, n.n_storage, cudaMemcpyDeviceToHost));
        for (const auto& p : n.pops) {
            if (p.type == naer::kPOISSON) continue;
            for (uint32_t k = 0; k < p.size; ++k) {
                if (v) hv[p.storage_base + k] = v[p.id_base + k];
                if (refractory) {
                    need(refractory[p.id_base + k] <= 255, NAER_E_INVALID, "refractory count above 255");
                    hr[p.storage_base + k] = (uint8_t)refractory[p.id_base + k];
                }
            }
        }
        NAER_CK(cudaMemcpy(n.v, hv.data(), n.n_storage * 4ull, cudaMemcpyHostToDevice));
        NAER_CK(cudaMemcpy(n.refr, hr.data(), n.n_storage, cudaMemcpyHostToDevice));
    });
}

int naer_net_read_csr(naer_net* net, uint64_t* row_ptr, uint32_t* tgt, float* w, uint8_t* delay) {
    return guarded([&] {
        need_compiled(net);
        need(row_ptr != nullptr, NAER_E_INVALID, "null row_ptr");
        const auto& n = net->net;
        net->eng->sync();
        std::vector<uint64_t> rp(n.n_storage + 1);
        NAER_CK(cudaMemcpy(rp.data(), n.row_ptr, rp.size() * 8ull, cudaMemcpyDeviceToHost));
        const uint64_t S = n.synapses_padded;
        std::vector<uint32_t> ht(S);
        std::vector<float> hw(S);
        std::vector<uint8_t> hd(S);
        if (S) {
            NAER_CK(cudaMemcpy(ht.data(), n.tgt, S * 4ull, cudaMemcpyDeviceToHost));
            NAER_CK(cudaMemcpy(hw.data(), n.w, S * 4ull, cudaMemcpyDeviceToHost));
            NAER_CK(cudaMemcpy(hd.data(), n.dly, S, cudaMemcpyDeviceToHost));
        }
        uint64_t o = 0;
        for (uint32_t id = 0; id < n.n_ids; ++id) {
            row_ptr[id] = o;
            const uint32_t s = n.storage_of_id[id];
            for (uint64_t j = rp[s]; j < rp[s + 1]; ++j) {
                if (ht[j] == naer::kTgtSentinel) continue;
                if (tgt) tgt[o] = (uint32_t)n.id_of_storage[ht[j]];
                if (w) w[o] = hw[j];
                if (delay) delay[o] = hd[j];
                ++o;
            }
        }
        row_ptr[n.n_ids] = o;
    });
}

int naer_net_set_profiling(naer_net* net, int enable) {
    return guarded([&] {
        need_compiled(net);
        net->eng->set_profiling(enable != 0);
    });
}

int naer_net_get_profile(naer_net* net, double* lif_ms, double* scatter_ms, uint64_t* launches) {
    return guarded([&] {
        need_compiled(net);
        net->eng->get_profile(lif_ms, scatter_ms, launches);
    });
}

int naer_net_get_launch_times(naer_net* net, double* drive_ms, double* step_kernel_ms,
                              uint64_t* step_kernel_launches) {
    return guarded([&] {
        need_compiled(net);
        net->eng->get_launch_times(drive_ms, step_kernel_ms, step_kernel_launches);
    });
}

int naer_net_get_phases(naer_net* net, double* phase_ms5) {
    return guarded([&] {
        need_compiled(net);
        need(phase_ms5 != nullptr, NAER_E_INVALID, "null argument");
        net->eng->get_phases(phase_ms5);
    });
}

/* ---- batched form ---- */

int naer_batch_create(int device, uint32_t aggregation, uint64_t raster_capacity, naer_batch** out) {
    return guarded([&] {
        need(out != nullptr, NAER_E_INVALID, "null output pointer");
        *out = nullptr;
        auto b = std::make_unique<naer_batch>();
        b->b = std::make_unique<naer::Batch>(device, aggregation, raster_capacity, raster_capacity > 0);
        *out = b.release();
    });
}

int naer_batch_destroy(naer_batch* batch) {
    if (!batch) return NAER_OK;
    return guarded([&] {
        naer::Batch& b = *batch->b;
        if (b.compiled()) {
            b.engine().sync();
            for (size_t i = 0; i < b.size(); ++i) b.engine().free_net(b.member((uint32_t)i));
        }
        delete batch;
    });
}

int naer_batch_add(naer_batch* batch, const naer_net* description, uint32_t* member) {
    return guarded([&] {
        need(batch && description, NAER_E_INVALID, "null argument");
        const uint32_t m = batch->b->add(description->net);
        if (member) *member = m;
    });
}

int naer_batch_compile(naer_batch* batch) {
    return guarded([&] {
        need(batch != nullptr, NAER_E_INVALID, "null batch handle");
        batch->b->compile();
    });
}

int naer_batch_step(naer_batch* batch, uint64_t nsteps) {
    return guarded([&] {
        need(batch != nullptr, NAER_E_INVALID, "null batch handle");
        batch->b->step(nsteps, batch->graph_launches);
    });
}

int naer_batch_finish(naer_batch* batch) {
    return guarded([&] {
        need(batch != nullptr && batch->b->compiled(), NAER_E_STATE, "batch is not compiled");
        batch->b->engine().sync();
        throw_device_status(batch->b->engine());
    });
}

static void fill_tuning(naer_tuning* out, const naer::Tuning& t, uint32_t graph_launches) {
    std::memset(out, 0, sizeof(*out));
    out->blocks_per_sm = t.blocks_per_sm;
    out->launch_steps = t.launch_steps;
    out->scatter_split = t.scatter_split;
    out->scatter_piece = t.scatter_piece;
    out->neuron_state = t.neuron_state;
    out->step_kernel = t.step_kernel;
    out->bins = t.bins;
    out->graph_launches = graph_launches;
}

int naer_batch_autotune(naer_batch* batch, uint32_t trial_steps, naer_tuning* out) {
    return guarded([&] {
        need(batch != nullptr, NAER_E_INVALID, "null batch handle");
        const naer::TuneResult r = batch->b->autotune(trial_steps);
        if (out) {
            fill_tuning(out, r.best, batch->graph_launches);
            out->best_us_per_step = r.best_us_per_step;
            out->default_us_per_step = r.default_us_per_step;
            out->trials = r.trials;
        }
    });
}

int naer_net_autotune(naer_net* net, uint32_t trial_steps, naer_tuning* out) {
    return guarded([&] {
        need_compiled(net);
        const naer::TuneResult r = net->eng->autotune(trial_steps);
        if (out) {
            fill_tuning(out, r.best, 0);
            out->best_us_per_step = r.best_us_per_step;
            out->default_us_per_step = r.default_us_per_step;
            out->trials = r.trials;
        }
    });
}

int naer_net_set_tuning(naer_net* net, const naer_tuning* tuning) {
    return guarded([&] {
        need_compiled(net);
        need(tuning != nullptr, NAER_E_INVALID, "null argument");
        naer::Tuning t;
        t.blocks_per_sm = tuning->blocks_per_sm;
        t.launch_steps = tuning->launch_steps;
        t.scatter_split = tuning->scatter_split;
        t.scatter_piece = tuning->scatter_piece;
        t.neuron_state = tuning->neuron_state;
        t.step_kernel = tuning->step_kernel;
        t.bins = tuning->bins;
        net->eng->set_tuning(t);
    });
}

int naer_net_get_tuning(naer_net* net, naer_tuning* tuning) {
    return guarded([&] {
        need_compiled(net);
        need(tuning != nullptr, NAER_E_INVALID, "null argument");
        fill_tuning(tuning, net->eng->tuning(), 0);
    });
}

int naer_batch_set_tuning(naer_batch* batch, const naer_tuning* tuning) {
    return guarded([&] {
        need(batch && tuning, NAER_E_INVALID, "null argument");
        need(batch->b->compiled(), NAER_E_STATE, "batch is not compiled");
        naer::Tuning t;
        t.blocks_per_sm = tuning->blocks_per_sm;
        t.launch_steps = tuning->launch_steps;
        t.scatter_split = tuning->scatter_split;
        t.scatter_piece = tuning->scatter_piece;
        t.neuron_state = tuning->neuron_state;
        t.step_kernel = tuning->step_kernel;
        t.bins = tuning->bins;
        batch->b->engine().set_tuning(t);
        batch->graph_launches = tuning->graph_launches;
    });
}

int naer_batch_get_tuning(naer_batch* batch, naer_tuning* tuning) {
    return guarded([&] {
        need(batch && tuning, NAER_E_INVALID, "null argument");
        fill_tuning(tuning, batch->b->engine().tuning(), batch->graph_launches);
    });
}

int naer_batch_read_spikes(naer_batch* batch, uint64_t first, uint64_t capacity, uint32_t* member,
                           uint32_t* steps, uint32_t* ids, uint64_t* count) {
    return guarded([&] {
        need(batch && count && (capacity == 0 || (steps && ids)), NAER_E_INVALID, "null argument");
        *count = batch->b->read_spikes(first, capacity, member, steps, ids);
    });
}

int naer_batch_clear_spikes(naer_batch* batch) {
    return guarded([&] {
        need(batch != nullptr && batch->b->compiled(), NAER_E_STATE, "batch is not compiled");
        batch->b->engine().clear_raster();
    });
}

int naer_batch_get_phases(naer_batch* batch, double* phase_ms5) {
    return guarded([&] {
        need(batch && phase_ms5, NAER_E_INVALID, "null argument");
        need(batch->b->compiled(), NAER_E_STATE, "batch is not compiled");
        batch->b->engine().get_phases(phase_ms5);
    });
}

int naer_batch_get_stats(naer_batch* batch, naer_stats* st) {
    return guarded([&] {
        need(batch && st, NAER_E_INVALID, "null argument");
        naer::Batch& b = *batch->b;
        need(b.compiled(), NAER_E_STATE, "batch is not compiled");
        naer::Engine& eng = b.engine();
        const naer::Ctl c = eng.read_ctl();
        std::memset(st, 0, sizeof(*st));
        st->step = c.step;
        st->events = eng.events_total();
        st->spikes = c.raster_next;
        st->raster_dropped = c.raster_dropped;
        st->stdp_hist_overflow = eng.overflow_total();
        st->device_bytes = eng.device_bytes();
        for (size_t i = 0; i < b.size(); ++i) {
            st->synapses += b.member((uint32_t)i).synapses;
            st->neurons += b.member((uint32_t)i).n_ids;
            st->ring_slots = std::max(st->ring_slots, b.member((uint32_t)i).ring_slots);
        }
        st->kernel_launches = eng.kernel_launches();
    });
}

int naer_batch_read_state(naer_batch* batch, uint32_t member, float* v, uint32_t* refractory) {
    return guarded([&] {
        need(batch != nullptr, NAER_E_INVALID, "null batch handle");
        need(batch->b->compiled(), NAER_E_STATE, "batch is not compiled");
        need(member < batch->b->size(), NAER_E_INVALID, "unknown member");
        read_state_of(batch->b->engine(), batch->b->member(member), v, refractory);
    });
}

int naer_batch_stream(naer_batch* batch, void** stream) {
    return guarded([&] {
        need(batch && stream, NAER_E_INVALID, "null argument");
        *stream = (void*)batch->b->engine().stream();
    });
}

/* ---- served form ---- */

int naer_server_params_default(naer_server_params* p) {
    if (!p) return fail(NAER_E_INVALID, "null pointer");
    std::memset(p, 0, sizeof(*p));
    p->budget_bytes = 150ull * 1000 * 1000 * 1000;
    p->raster_capacity = 1ull << 24;
    p->chunk_steps = 256;
    p->aggregation = NAER_AGG_ATOMIC;
    p->max_jobs = 1024;
    p->blocks_per_sm = 0;
    p->chunk_ms = 10.0;
    p->launch_steps = 0;
    p->step_kernel = NAER_KERNEL_TWO_BARRIER;
    return NAER_OK;
}

int naer_server_create(int device, const naer_server_params* params, naer_server** out) {
    return guarded([&] {
        need(out != nullptr, NAER_E_INVALID, "null output pointer");
        *out = nullptr;
        naer_server_params p;
        if (params) p = *params; else naer_server_params_default(&p);
        naer::ServerParams sp;
        sp.budget_bytes = p.budget_bytes;
        sp.raster_capacity = p.raster_capacity;
        sp.chunk_steps = p.chunk_steps;
        sp.aggregation = p.aggregation;
        sp.max_jobs = p.max_jobs;
        sp.blocks_per_sm = p.blocks_per_sm;
        sp.chunk_ms = p.chunk_ms;
        if (p.launch_steps) sp.launch_steps = p.launch_steps;
        need(p.step_kernel <= NAER_KERNEL_TWO_BARRIER, NAER_E_INVALID, "unknown step kernel");
        sp.step_kernel = p.step_kernel;
        auto h = std::make_unique<naer_server>();
        h->s = std::make_unique<naer::Server>(device, sp);
        *out = h.release();
    });
}

int naer_server_destroy(naer_server* server) {
    if (!server) return NAER_OK;
    return guarded([&] { delete server; });
}

int naer_server_submit(naer_server* server, const naer_net* description, uint64_t duration_steps,
                       uint64_t* job) {
    return guarded([&] {
        need(server && description && job, NAER_E_INVALID, "null argument");
        *job = server->s->submit(description->net, duration_steps);
    });
}

int naer_server_job_info(naer_server* server, uint64_t job, naer_job_info* info) {
    return guarded([&] {
        need(server && info, NAER_E_INVALID, "null argument");
        const naer::JobInfo j = server->s->info(job);
        std::memset(info, 0, sizeof(*info));
        info->state = j.state;
        info->preemptions = j.preemptions;
        info->duration = j.duration;
        info->steps_done = j.steps_done;
        info->spikes = j.spikes;
        info->device_bytes = j.device_bytes;
        info->submit_s = j.submit_s;
        info->admit_s = j.admit_s;
        info->done_s = j.done_s;
    });
}

int naer_server_job_error(naer_server* server, uint64_t job, char* buf, size_t len) {
    return guarded([&] {
        need(server && buf && len > 0, NAER_E_INVALID, "null argument");
        const naer::JobInfo j = server->s->info(job);
        const size_t n = std::min(len - 1, j.error.size());
        std::memcpy(buf, j.error.data(), n);
        buf[n] = '\0';
    });
}

int naer_server_wait(naer_server* server, uint64_t job, double timeout_s, int* finished) {
    return guarded([&] {
        need(server != nullptr, NAER_E_INVALID, "null server handle");
        const bool ok = server->s->wait(job, timeout_s);
        if (finished) *finished = ok ? 1 : 0;
    });
}

int naer_server_drain(naer_server* server, double timeout_s, int* finished) {
    return guarded([&] {
        need(server != nullptr, NAER_E_INVALID, "null server handle");
        const bool ok = server->s->drain(timeout_s);
        if (finished) *finished = ok ? 1 : 0;
    });
}

int naer_server_read_spikes(naer_server* server, uint64_t job, uint64_t first, uint64_t capacity,
                            uint32_t* steps, uint32_t* ids, uint64_t* count) {
    return guarded([&] {
        need(server && count && (capacity == 0 || (steps && ids)), NAER_E_INVALID, "null argument");
        *count = server->s->read_spikes(job, first, capacity, steps, ids);
    });
}

int naer_server_release(naer_server* server, uint64_t job) {
    return guarded([&] {
        need(server != nullptr, NAER_E_INVALID, "null server handle");
        server->s->release(job);
    });
}

int naer_server_preempt(naer_server* server, uint64_t job) {
    return guarded([&] {
        need(server != nullptr, NAER_E_INVALID, "null server handle");
        server->s->preempt(job);
    });
}

int naer_server_cancel(naer_server* server, uint64_t job) {
    return guarded([&] {
        need(server != nullptr, NAER_E_INVALID, "null server handle");
        server->s->cancel(job);
    });
}

int naer_server_get_stats(naer_server* server, naer_server_stats* st) {
    return guarded([&] {
        need(server && st, NAER_E_INVALID, "null argument");
        const naer::ServerStats s = server->s->stats();
        std::memset(st, 0, sizeof(*st));
        st->submitted = s.submitted;
        st->done = s.done;
        st->failed = s.failed;
        st->running = s.running;
        st->queued = s.queued;
        st->chunks = s.chunks;
        st->engine_steps = s.engine_steps;
        st->peak_bytes = s.peak_bytes;
        st->bytes_in_use = s.bytes_in_use;
        st->raster_dropped = s.raster_dropped;
        st->p50_ms = s.p50_ms;
        st->p99_ms = s.p99_ms;
        st->mean_ms = s.mean_ms;
        st->sims_per_s = s.sims_per_s;
        st->build_s = s.build_s;
        st->install_s = s.install_s;
        st->step_s = s.step_s;
        st->drain_s = s.drain_s;
    });
}

}  // extern "C"
