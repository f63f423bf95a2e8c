// Naer::Batch and Naer::Server — the batched and served forms for C++
// users, header-only over naer_capi.h (naer_batch_*, naer_server_*).  No
// counterpart in the reference, which runs one Network per device queue.
//
// Networks are described with Naer::Network(-1) (a description-only handle:
// populations and connections, no device resources) and copied in.
// Every non-zero status becomes std::runtime_error, as in Network.h.
#pragma once

#include <cstdint>
#include <vector>

#include "Network.h"
#include "naer_capi.h"

namespace Naer {

struct BatchSpike {
    uint32_t member;
    uint32_t step;
    uint32_t address;
};

class Batch {
public:
    explicit Batch(int device = 0, bool deterministic = false, uint64_t rasterCapacity = 1ull << 24) {
        check(naer_batch_create(device, deterministic ? NAER_AGG_DETERMINISTIC : NAER_AGG_ATOMIC, rasterCapacity,
                                &m_batch));
    }
    ~Batch() { naer_batch_destroy(m_batch); }
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    // Copies a description-only network; returns its member index.
    uint32_t add(Network& description) {
        uint32_t m = 0;
        check(naer_batch_add(m_batch, description.handle(), &m));
        return m;
    }
    void compile() { check(naer_batch_compile(m_batch)); }
    void step(uint64_t gridSteps) { check(naer_batch_step(m_batch, gridSteps)); }
    void finish() { check(naer_batch_finish(m_batch)); }
    naer_tuning autotune(uint32_t trialSteps = 64) {
        naer_tuning t{};
        check(naer_batch_autotune(m_batch, trialSteps, &t));
        return t;
    }
    std::vector<BatchSpike> readSpikes() {
        naer_stats st{};
        check(naer_batch_get_stats(m_batch, &st));
        const uint64_t cap = st.spikes;
        std::vector<uint32_t> m(cap), s(cap), a(cap);
        uint64_t n = 0;
        if (cap) check(naer_batch_read_spikes(m_batch, 0, cap, m.data(), s.data(), a.data(), &n));
        std::vector<BatchSpike> out(n);
        for (uint64_t i = 0; i < n; ++i) out[i] = BatchSpike{m[i], s[i], a[i]};
        return out;
    }
    naer_batch* handle() { return m_batch; }

private:
    naer_batch* m_batch = nullptr;
};

class Server {
public:
    explicit Server(int device = 0, const naer_server_params* params = nullptr) {
        check(naer_server_create(device, params, &m_server));
    }
    ~Server() { naer_server_destroy(m_server); }
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    uint64_t submit(Network& description, uint64_t gridSteps) {
        uint64_t job = 0;
        check(naer_server_submit(m_server, description.handle(), gridSteps, &job));
        return job;
    }
    bool wait(uint64_t job, double timeoutSeconds) {
        int done = 0;
        check(naer_server_wait(m_server, job, timeoutSeconds, &done));
        return done != 0;
    }
    bool drain(double timeoutSeconds) {
        int done = 0;
        check(naer_server_drain(m_server, timeoutSeconds, &done));
        return done != 0;
    }
    naer_job_info info(uint64_t job) {
        naer_job_info i{};
        check(naer_server_job_info(m_server, job, &i));
        return i;
    }
    // (step, address) of a finished job, job-local steps
    std::vector<std::pair<uint32_t, uint32_t>> spikes(uint64_t job) {
        const naer_job_info i = info(job);
        std::vector<uint32_t> s(i.spikes), a(i.spikes);
        uint64_t n = 0;
        if (i.spikes) check(naer_server_read_spikes(m_server, job, 0, i.spikes, s.data(), a.data(), &n));
        std::vector<std::pair<uint32_t, uint32_t>> out(n);
        for (uint64_t k = 0; k < n; ++k) out[k] = {s[k], a[k]};
        return out;
    }
    void release(uint64_t job) { check(naer_server_release(m_server, job)); }
    naer_server_stats stats() {
        naer_server_stats st{};
        check(naer_server_get_stats(m_server, &st));
        return st;
    }

private:
    naer_server* m_server = nullptr;
};

}  // namespace Naer
