// Naer::Network — the reference's C++ model-building API
// (include/naer/Network.h:15-142, Population.h:9-17, Connection.h:8-30,
// src/Network.cpp) as a header-only wrapper over the C ABI in naer_capi.h.
//
// Same names and call pattern as the reference: addPopulation per neuron
// type (baseAddress is type-local until compile() shifts it), the two
// addConnection overloads, compile(), step() (one 1500 µs window,
// asynchronous), finish() (blocks), getTime() in µs, getSynapses(),
// getNeurons(), and public profile counters.  Every non-zero status becomes
// std::runtime_error, as every OpenCL failure does in the reference.
// Link against naer_b200/libnaer_b200.so.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "naer_capi.h"

namespace Naer {

enum class NeuronType : uint32_t {
    STDP = NAER_NEURON_STDP,
    NOP = NAER_NEURON_NOP,
    POISSON = NAER_NEURON_POISSON,
};

struct Population {
    NeuronType type;
    uint32_t baseAddress;
    uint32_t size;
    uint32_t id;  // handle-local population index
    Population(NeuronType t, uint32_t base, uint32_t s, uint32_t i) : type(t), baseAddress(base), size(s), id(i) {}
};

struct Connection {
    std::shared_ptr<const Population> source;
    std::shared_ptr<const Population> destination;
    float defaultWeights;
    float minRandomWeights;
    float maxRandomWeights;
    double probability;
    uint64_t seed;
};

inline void check(int status) {
    if (status != NAER_OK) {
        char buf[1024];
        naer_last_error(buf, sizeof(buf));
        throw std::runtime_error(std::string("naer: ") + buf);
    }
}

class Network {
public:
    // Network::Network (Network.cpp:14-47); grid step of dt_us by default.
    explicit Network(int device = 0, const naer_net_params* params = nullptr) {
        naer_net_params p;
        if (params) {
            p = *params;
        } else {
            check(naer_net_params_default(&p));
        }
        m_dt = p.dt_us;
        check(naer_net_create(device, &p, &m_net));
    }
    ~Network() { naer_net_destroy(m_net); }
    Network(const Network&) = delete;
    Network& operator=(const Network&) = delete;

    std::shared_ptr<const Population> addPopulation(NeuronType type, uint32_t size,
                                                    const naer_pop_params* params = nullptr) {
        uint32_t id = 0, addr = 0;
        check(naer_net_add_population(m_net, (uint32_t)type, size, params, &id, &addr));
        auto pop = std::make_shared<Population>(type, addr, size, id);
        m_populations.push_back(pop);
        return pop;
    }

    void addConnection(std::shared_ptr<const Population> source, std::shared_ptr<const Population> destination,
                       float defaultWeights, double probability) {
        addConnection(source, destination, defaultWeights, 0.f, 1.f, probability, 0xbf785e3215ac7ebdull);
    }

    void addConnection(std::shared_ptr<const Population> source, std::shared_ptr<const Population> destination,
                       float defaultWeights, float minRandomWeights, float maxRandomWeights, double probability,
                       uint64_t seed) {
        naer_conn_spec c{};
        c.rule = NAER_CONN_REF_BERNOULLI;
        c.probability = probability;
        c.weight = defaultWeights;
        c.wmin = minRandomWeights;
        c.wmax = maxRandomWeights;
        c.delay_min = c.delay_max = windowSteps();  // one axonal delay of 1500 µs (naer_types.h:4)
        c.seed = seed;
        check(naer_net_add_connection(m_net, source->id, destination->id, &c));
        m_connections.push_back(Connection{source, destination, defaultWeights, minRandomWeights,
                                           maxRandomWeights, probability, seed});
    }

    // Any rule of the C ABI (fixed in/out-degree, delays in grid steps).
    void connect(const Population& source, const Population& destination, const naer_conn_spec& spec) {
        check(naer_net_add_connection(m_net, source.id, destination.id, &spec));
    }

    void compile() {
        check(naer_net_compile(m_net));
        for (auto& p : m_populations) check(naer_net_population_base(m_net, p->id, &p->baseAddress));
    }

    void step() { check(naer_net_step(m_net, windowSteps())); }
    void run(uint64_t gridSteps) { check(naer_net_step(m_net, gridSteps)); }
    void finish() { check(naer_net_finish(m_net)); }

    uint32_t getTime() {
        uint64_t t = 0;
        check(naer_net_get_time_us(m_net, &t));
        return (uint32_t)t;
    }
    uint32_t getSynapses() {
        uint64_t s = 0;
        check(naer_net_get_synapses(m_net, &s));
        return (uint32_t)s;
    }
    uint32_t getNeurons() {
        uint32_t n = 0;
        check(naer_net_get_neurons(m_net, &n));
        return n;
    }

    // Recorded spikes (no counterpart in the reference, which never reads
    // spikes back): grid steps and reference addresses, grouped by step,
    // ascending address within a step.  Blocks.
    void readSpikes(std::vector<uint32_t>& steps, std::vector<uint32_t>& addresses) {
        naer_stats st{};
        check(naer_net_get_stats(m_net, &st));
        steps.resize(st.spikes);
        addresses.resize(st.spikes);
        uint64_t n = 0;
        if (st.spikes) check(naer_net_read_spikes(m_net, 0, st.spikes, steps.data(), addresses.data(), &n));
        steps.resize(n);
        addresses.resize(n);
    }

    // Per-kernel device time (s) while profiling is enabled (Network.h:50-55).
    void setProfiling(bool on) { check(naer_net_set_profiling(m_net, on ? 1 : 0)); }
    void readProfile() {
        double lif = 0, sc = 0;
        uint64_t n = 0;
        check(naer_net_get_profile(m_net, &lif, &sc, &n));
        nop_time = lif / 1e3;
        scatter_time = sc / 1e3;
    }

    naer_net* handle() { return m_net; }

    double nop_time = 0;
    double stdp_time = 0;
    double poisson_time = 0;
    double scan_time = 0;
    double scatter_time = 0;
    double offset_time = 0;

private:
    uint32_t windowSteps() const { return m_dt >= 1500 ? 1u : (1500u + m_dt / 2) / m_dt; }

    naer_net* m_net = nullptr;
    uint32_t m_dt = 100;
    std::vector<std::shared_ptr<Population>> m_populations;
    std::vector<Connection> m_connections;
};

}  // namespace Naer
