// Batched and served forms (see forms.h).
#include "forms.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace naer {

namespace {

std::unique_ptr<NetHost> clone_description(const NetHost& d) {
    if (d.compiled) throw Error(NAER_E_STATE, "a compiled network cannot be used as a description");
    auto n = std::make_unique<NetHost>();
    n->params = d.params;
    n->pops = d.pops;
    n->conns = d.conns;
    return n;
}

// Optional per-chunk and per-build trace of the served form, as CSV: set
// NAER_SERVER_TRACE to a file name (the builder writes <name>.build).
FILE* open_trace(const char* suffix, const char* header) {
    const char* base = std::getenv("NAER_SERVER_TRACE");
    if (!base || !*base) return nullptr;
    FILE* f = std::fopen((std::string(base) + suffix).c_str(), "w");
    if (f) std::fputs(header, f);
    return f;
}

// Member of an engine-global raster id (id offsets ascending).
uint32_t member_of(const std::vector<uint32_t>& off, uint32_t id) {
    const auto it = std::upper_bound(off.begin(), off.end(), id);
    return (uint32_t)(it - off.begin()) - 1u;
}

}  // namespace

// ---------------------------------------------------------------------------
// Batch

Batch::Batch(int device, uint32_t aggregation, uint64_t raster_capacity, bool record)
    : eng_(std::make_unique<Engine>(device)),
      aggregation_(aggregation),
      raster_capacity_(raster_capacity),
      record_(record) {
    if (aggregation > NAER_AGG_EXACT) throw Error(NAER_E_INVALID, "unknown aggregation");
}

uint32_t Batch::add(const NetHost& description) {
    if (compiled_) throw Error(NAER_E_STATE, "batch already compiled");
    auto n = clone_description(description);
    estimate_device_bytes(*n);  // validates now, not at compile
    members_.push_back(std::move(n));
    return (uint32_t)members_.size() - 1;
}

void Batch::compile() {
    if (compiled_) throw Error(NAER_E_STATE, "batch already compiled");
    if (members_.empty()) throw Error(NAER_E_STATE, "batch has no members");
    std::vector<NetHost*> nets;
    for (auto& m : members_) {
        eng_->build(*m);
        nets.push_back(m.get());
    }
    eng_->install(nets, raster_capacity_, record_, aggregation_);
    compiled_ = true;
}

void Batch::step(uint64_t nsteps, uint32_t graph_launches) {
    if (!compiled_) throw Error(NAER_E_STATE, "batch is not compiled");
    eng_->run_graph(nsteps, graph_launches);
}

TuneResult Batch::autotune(uint32_t trial_steps) {
    if (!compiled_) throw Error(NAER_E_STATE, "batch is not compiled");
    return eng_->autotune(trial_steps);
}

uint64_t Batch::read_spikes(uint64_t first, uint64_t cap, uint32_t* member, uint32_t* steps, uint32_t* ids) {
    if (!compiled_) throw Error(NAER_E_STATE, "batch is not compiled");
    const uint64_t n = eng_->read_raster(first, cap, steps, ids);
    const auto& off = eng_->id_offsets();
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t m = member_of(off, ids[i]);
        if (member) member[i] = m;
        ids[i] -= off[m];
    }
    return n;
}

// ---------------------------------------------------------------------------
// Server

Server::Server(int device, const ServerParams& p) : device_(device), prm_(p), t0_(std::chrono::steady_clock::now()) {
    if (p.aggregation > NAER_AGG_EXACT) throw Error(NAER_E_INVALID, "unknown aggregation");
    if (p.chunk_steps == 0) throw Error(NAER_E_INVALID, "chunk_steps must be positive");
    if (p.max_jobs == 0) throw Error(NAER_E_INVALID, "max_jobs must be positive");
    if (p.raster_capacity == 0) throw Error(NAER_E_INVALID, "raster_capacity must be positive");
    if (p.launch_steps == 0 || p.launch_steps > kDriveSlots)
        throw Error(NAER_E_INVALID, "launch_steps must be in 1..64");
    int n = 0;
    NAER_CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) throw Error(NAER_E_INVALID, "device index out of range");
    builder_ = std::thread([this] { build_loop(); });
    worker_ = std::thread([this] { loop(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    cv_build_.notify_all();
    if (worker_.joinable()) worker_.join();
    cv_build_.notify_all();
    if (builder_.joinable()) builder_.join();
}

double Server::now_s() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

uint64_t Server::submit(const NetHost& description, uint64_t duration_steps) {
    if (duration_steps == 0) throw Error(NAER_E_INVALID, "duration must be at least one step");
    auto j = std::make_unique<Job>();
    j->net = clone_description(description);
    j->est_bytes = estimate_device_bytes(*j->net, prm_.aggregation == NAER_AGG_DETERMINISTIC);
    j->chunks = lif_chunks(*j->net);
    if (j->est_bytes > prm_.budget_bytes)
        throw Error(NAER_E_OVERFLOW, "job needs about " + std::to_string(j->est_bytes) +
                                         " device bytes, more than the server budget of " +
                                         std::to_string(prm_.budget_bytes));
    j->info.duration = duration_steps;
    std::lock_guard<std::mutex> lk(mu_);
    if (!fatal_.empty()) throw Error(NAER_E_CUDA, "server stopped: " + fatal_);
    if (stop_) throw Error(NAER_E_STATE, "server is shutting down");
    j->id = next_id_++;
    j->info.submit_s = now_s();
    if (first_submit_s_ < 0) first_submit_s_ = j->info.submit_s;
    const uint64_t id = j->id;
    jobs_[id] = std::move(j);
    pending_.push_back(id);
    ++st_.submitted;
    cv_build_.notify_all();
    return id;
}

JobInfo Server::info(uint64_t job) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end() || it->second->released) throw Error(NAER_E_INVALID, "unknown job");
    return it->second->info;
}

uint64_t Server::read_spikes(uint64_t job, uint64_t first, uint64_t cap, uint32_t* steps, uint32_t* ids) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end() || it->second->released) throw Error(NAER_E_INVALID, "unknown job");
    const Job& j = *it->second;
    if (j.info.state != kJobDone) throw Error(NAER_E_STATE, "job has not finished");
    const uint64_t total = j.steps.size();
    if (first >= total || cap == 0) return 0;
    const uint64_t n = std::min<uint64_t>(cap, total - first);
    std::copy(j.steps.begin() + first, j.steps.begin() + first + n, steps);
    std::copy(j.ids.begin() + first, j.ids.begin() + first + n, ids);
    return n;
}

bool Server::wait(uint64_t job, double timeout_s) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end() || it->second->released) throw Error(NAER_E_INVALID, "unknown job");
    Job* j = it->second.get();
    return cv_done_.wait_for(lk, std::chrono::duration<double>(timeout_s),
                             [&] { return j->info.state >= kJobDone; });
}

bool Server::drain(double timeout_s) {
    std::unique_lock<std::mutex> lk(mu_);
    return cv_done_.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
        for (const auto& kv : jobs_)
            if (kv.second->info.state < kJobDone) return false;
        return true;
    });
}

void Server::release(uint64_t job) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end() || it->second->released) throw Error(NAER_E_INVALID, "unknown job");
    if (it->second->info.state < kJobDone) throw Error(NAER_E_STATE, "job has not finished");
    if (it->second->freed) jobs_.erase(it); else it->second->released = true;  // the builder erases it
}

void Server::preempt(uint64_t job) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end() || it->second->released) throw Error(NAER_E_INVALID, "unknown job");
    if (it->second->info.state != kJobRunning) throw Error(NAER_E_STATE, "job is not running");
    it->second->preempt_req = true;
}

void Server::cancel(uint64_t job) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end() || it->second->released) throw Error(NAER_E_INVALID, "unknown job");
    Job* j = it->second.get();
    if (j->info.state >= kJobDone) throw Error(NAER_E_STATE, "job has already ended");
    auto end_now = [&] {
        j->info.state = kJobCancelled;
        j->info.error = "cancelled";
        j->steps.clear();
        j->ids.clear();
        j->saved.clear();
        cv_done_.notify_all();
    };
    auto p = std::find(pending_.begin(), pending_.end(), job);
    if (p != pending_.end()) {  // not built: nothing on the device
        pending_.erase(p);
        if (j->preempt_req || !j->saved.empty()) j->preempt_req = false;
        end_now();
        return;
    }
    auto r = std::find(ready_.begin(), ready_.end(), j);
    if (r != ready_.end()) {  // built, never stepped: the builder frees it
        ready_.erase(r);
        to_free_.push_back(j);
        end_now();
        cv_build_.notify_all();
        return;
    }
    j->cancel_req = true;  // running: the stepper retires it at the next boundary
}

ServerStats Server::stats() {
    std::lock_guard<std::mutex> lk(mu_);
    ServerStats s = st_;
    s.queued = pending_.size() + ready_.size();
    s.bytes_in_use = used_;
    std::vector<double> l = latencies_ms_;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto q = [&](double f) { return l[std::min<size_t>(l.size() - 1, (size_t)std::floor(f * (l.size() - 1) + 0.5))]; };
        s.p50_ms = q(0.50);
        s.p99_ms = q(0.99);
        double sum = 0;
        for (double x : l) sum += x;
        s.mean_ms = sum / l.size();
        const double span = last_done_s_ - first_submit_s_;
        s.sims_per_s = span > 0 ? s.done / span : 0.0;
    }
    return s;
}

// Builder: admission by memory and job slots (first come, first served),
// device build on its own engine and stream, and the frees of retired jobs.
void Server::build_loop() {
    std::unique_ptr<Engine> eng;
    FILE* trace = open_trace(".build", "t_s,job,wait_s,build_ms,neurons,synapses,est_bytes,used_bytes,pending\n");
    try {
        NAER_CK(cudaSetDevice(device_));
        int lo = 0, hi = 0;
        NAER_CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        eng = std::make_unique<Engine>(device_, hi);
        // Reserve the budget in the stream-ordered pool up front (allocate
        // and free: the pool keeps it): later builds then reuse mapped memory
        // instead of growing the pool while step kernels run.
        {
            size_t free_b = 0, total_b = 0;
            NAER_CK(cudaMemGetInfo(&free_b, &total_b));
            const uint64_t margin = 8ull << 30;
            const uint64_t warm = std::min<uint64_t>(prm_.budget_bytes, free_b > margin ? free_b - margin : 0);
            if (warm) {
                void* p = nullptr;
                if (cudaMallocAsync(&p, warm, eng->stream()) == cudaSuccess) NAER_CK(cudaFreeAsync(p, eng->stream()));
                else (void)cudaGetLastError();
                eng->sync();
            }
        }
        for (;;) {
            Job* j = nullptr;
            std::vector<Job*> frees;
            {
                std::unique_lock<std::mutex> lk(mu_);
                auto head_fits = [&] {
                    if (stop_ || pending_.empty() || live_ >= prm_.max_jobs) return false;
                    return used_ + jobs_.at(pending_.front())->est_bytes <= prm_.budget_bytes;
                };
                cv_build_.wait(lk, [&] { return (stop_ && stepper_done_) || !to_free_.empty() || head_fits(); });
                frees.assign(to_free_.begin(), to_free_.end());
                to_free_.clear();
                if (frees.empty()) {
                    if (stop_ && stepper_done_) break;
                    if (head_fits()) {
                        j = jobs_.at(pending_.front()).get();
                        pending_.pop_front();
                        used_ += j->est_bytes;
                        ++live_;
                    }
                }
            }
            for (Job* f : frees) {
                eng->free_net(*f->net);
                std::lock_guard<std::mutex> lk(mu_);
                used_ -= f->est_bytes;
                --live_;
                f->freed = true;
                if (f->released) jobs_.erase(f->id);
            }
            if (!j) continue;
            const double t = now_s();
            try {
                eng->build(*j->net);
                if (prm_.aggregation == NAER_AGG_EXACT) {  // its fixed-point grid, off the stepper's path
                    eng->exact_shifts({j->net.get()});
                    if (j->net->fx_shift < 0)
                        throw Error(NAER_E_OVERFLOW, "weights too large for exact-sum aggregation");
                }
                if (!j->saved.empty()) {  // a pre-empted job: its state from before
                    eng->load_state(*j->net, j->saved.data());
                    std::vector<uint8_t>().swap(j->saved);
                }
                eng->sync();  // complete before another stream uses it
            } catch (const Error& e) {
                if (e.code == NAER_E_CUDA) throw;
                if (j->net->compiled) eng->free_net(*j->net);
                std::lock_guard<std::mutex> lk(mu_);
                used_ -= j->est_bytes;
                --live_;
                j->freed = true;
                j->info.state = kJobFailed;
                j->info.error = e.what();
                ++st_.failed;
                cv_done_.notify_all();
                continue;
            }
            std::lock_guard<std::mutex> lk(mu_);
            st_.build_s += now_s() - t;
            if (trace)
                std::fprintf(trace, "%.6f,%llu,%.6f,%.3f,%u,%llu,%llu,%llu,%zu\n", t, (unsigned long long)j->id,
                             t - j->info.submit_s, 1e3 * (now_s() - t), j->net->n_ids,
                             (unsigned long long)j->net->synapses, (unsigned long long)j->est_bytes,
                             (unsigned long long)used_, pending_.size());
            st_.peak_bytes = std::max<uint64_t>(st_.peak_bytes, eng->device_bytes());
            ready_.push_back(j);
            cv_work_.notify_all();
        }
        // shutting down: whatever was built but never stepped
        std::vector<Job*> rest;
        {
            std::lock_guard<std::mutex> lk(mu_);
            rest.assign(ready_.begin(), ready_.end());
            ready_.clear();
        }
        for (Job* j : rest) eng->free_net(*j->net);
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(mu_);
        fatal_ = e.what();
        for (auto& kv : jobs_) {
            if (kv.second->info.state < kJobDone) {
                kv.second->info.state = kJobFailed;
                kv.second->info.error = fatal_;
                ++st_.failed;
            }
        }
        pending_.clear();
        stop_ = true;
        cv_done_.notify_all();
        cv_work_.notify_all();
    }
    if (trace) std::fclose(trace);
}

// Stepper: one iteration per chunk of steps.  It takes built jobs in,
// collects the raster of the chunk in flight (waiting for it), retires the
// jobs whose last step that chunk ran, re-installs the tables if the set
// changed, queues the next chunk and only then hands the collected records
// to their jobs on the host, while the device runs the next chunk.
void Server::loop() {
    std::unique_ptr<Engine> eng;
    std::vector<Job*> running;        // set of the next chunk
    std::vector<Job*> inflight_set;   // set of the chunk in flight
    std::vector<uint32_t> inflight_off;
    bool inflight = false;
    bool changed = false;
    uint2* rec = nullptr;  // pinned staging of one chunk's raster
    cudaEvent_t copied = nullptr;
    std::vector<uint32_t> owner, count;
    // Chunks are bounded in device time, not only in steps: a chunk's step
    // count follows the measured time per step, so a large running set does
    // not stretch the interval between admission points (which would let
    // more jobs queue up and stretch it further).
    double ms_per_step = 0.0;
    uint64_t chunk_len = 0;
    cudaEvent_t c0 = nullptr, c1 = nullptr;  // device time of the chunk in flight
    FILE* trace = open_trace("", "t_s,running,admitted,finished,chunk_steps,chunk_ms,wait_ms,install_ms,drain_ms,"
                                 "records,pending,used_bytes,running_chunks,chunk_cap\n");
    try {
        NAER_CK(cudaSetDevice(device_));
        eng = std::make_unique<Engine>(device_);
        // short persistent launches: the builder's kernels (higher-priority
        // stream) get the device between them instead of after whole chunks
        Tuning tn;
        tn.launch_steps = prm_.launch_steps;
        tn.blocks_per_sm = prm_.blocks_per_sm;
        tn.step_kernel = prm_.step_kernel;
        eng->set_tuning(tn);
        // Admission keeps the running set within the step kernel's fastest
        // geometry (neuron state in shared memory, most blocks per SM).  A
        // larger set steps more slowly per job, so a backlog that admitted
        // everything would lower the throughput that has to clear it.
        const uint64_t chunk_cap = eng->fast_chunk_capacity(prm_.aggregation);
        NAER_CK(cudaHostAlloc(reinterpret_cast<void**>(&rec), prm_.raster_capacity * sizeof(uint2),
                              cudaHostAllocDefault));
        NAER_CK(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
        NAER_CK(cudaEventCreate(&c0));
        NAER_CK(cudaEventCreate(&c1));
        for (;;) {
            std::vector<Job*> admit;
            {
                std::unique_lock<std::mutex> lk(mu_);
                if (running.empty() && !inflight) cv_work_.wait(lk, [&] { return stop_ || !ready_.empty(); });
                if (stop_) break;
                uint64_t rc = 0;  // chunks of the jobs that stay after this boundary
                const uint64_t hs0 = eng->host_step();
                for (Job* j : running)
                    if (j->net->dev.end_step > hs0) rc += j->chunks;
                while (!ready_.empty()) {
                    Job* j = ready_.front();
                    const bool alone = rc == 0 && admit.empty();  // a job larger than the cap runs alone
                    if (!alone && chunk_cap && rc + j->chunks > chunk_cap) break;
                    admit.push_back(j);
                    ready_.pop_front();
                    rc += j->chunks;
                }
                const double t = now_s();
                for (Job* j : admit) {
                    j->info.state = kJobRunning;
                    j->info.admit_s = t;
                    j->info.device_bytes = j->net->device_bytes;
                }
            }
            double t = now_s();
            // the chunk in flight: wait, queue its raster copy
            uint64_t nrec = 0, dropped = 0;
            if (inflight) nrec = eng->harvest_raster(rec, copied, &dropped);
            const double t_step = inflight ? now_s() - t : 0.0;
            const uint64_t done_len = inflight ? chunk_len : 0;
            float done_ms = 0.0f;  // device time of the chunk just collected
            if (inflight && chunk_len > 0) {
                float ms = 0.0f;
                NAER_CK(cudaEventElapsedTime(&ms, c0, c1));
                done_ms = ms;
                const double m = (double)ms / (double)chunk_len;
                ms_per_step = ms_per_step > 0.0 ? 0.5 * (ms_per_step + m) : m;
            }
            const uint64_t hs = eng->host_step();
            // jobs whose last step has run; jobs to pre-empt or cancel (the
            // chunk in flight has been waited for, so their state is whole)
            std::vector<Job*> keep, finished, preempted, cancelled;
            {
                std::lock_guard<std::mutex> lk(mu_);
                for (Job* j : running) {
                    if (hs >= j->net->dev.end_step) finished.push_back(j);
                    else if (j->cancel_req) cancelled.push_back(j);
                    else if (j->preempt_req) preempted.push_back(j);
                    else keep.push_back(j);
                }
            }
            for (Job* j : preempted) {
                j->resume_steps = hs - j->net->dev.start_step;
                j->saved.resize(state_bytes(*j->net));
                eng->save_state(*j->net, j->saved.data());
            }
            if (!finished.empty() || !preempted.empty() || !cancelled.empty()) changed = true;
            running.swap(keep);
            for (Job* j : admit) {
                j->net->dev.start_step = hs - j->resume_steps;  // a resumed job keeps its own step count
                j->net->dev.end_step = j->net->dev.start_step + j->info.duration;
                running.push_back(j);
                changed = true;
            }
            t = now_s();
            double t_install = 0;
            if (changed && !running.empty()) {
                std::vector<NetHost*> nets;
                for (Job* j : running) nets.push_back(j->net.get());
                eng->install(nets, prm_.raster_capacity, true, prm_.aggregation);
                changed = false;
                t_install = now_s() - t;
            }
            // queue the next chunk
            std::vector<Job*> prev_set;
            std::vector<uint32_t> prev_off;
            prev_set.swap(inflight_set);
            prev_off.swap(inflight_off);
            if (!running.empty()) {
                uint64_t last_end = hs;
                for (Job* j : running) last_end = std::max<uint64_t>(last_end, j->net->dev.end_step);
                uint64_t len = prm_.chunk_steps;
                if (ms_per_step > 0.0 && prm_.chunk_ms > 0.0)
                    len = std::min<uint64_t>(len, std::max<uint64_t>(16, (uint64_t)(prm_.chunk_ms / ms_per_step)));
                chunk_len = std::min<uint64_t>(len, last_end - hs);
                NAER_CK(cudaEventRecord(c0, eng->stream()));
                eng->run(chunk_len);
                NAER_CK(cudaEventRecord(c1, eng->stream()));
                inflight = true;
                inflight_set = running;
                inflight_off = eng->id_offsets();
            } else {
                inflight = false;
            }
            // hand the collected records to their jobs while the device runs
            t = now_s();
            NAER_CK(cudaEventSynchronize(copied));
            owner.resize(nrec);
            count.assign(prev_set.size(), 0);
            for (uint64_t i = 0; i < nrec; ++i) {
                owner[i] = member_of(prev_off, rec[i].y);
                ++count[owner[i]];
            }
            std::vector<size_t> at(prev_set.size());
            for (size_t m = 0; m < prev_set.size(); ++m) {
                Job* j = prev_set[m];
                at[m] = j->steps.size();
                j->steps.resize(at[m] + count[m]);
                j->ids.resize(at[m] + count[m]);
            }
            for (uint64_t i = 0; i < nrec; ++i) {
                const uint32_t m = owner[i];
                Job* j = prev_set[m];
                j->steps[at[m]] = (uint32_t)(rec[i].x - j->net->dev.start_step);
                j->ids[at[m]] = rec[i].y - prev_off[m];
                ++at[m];
            }
            for (Job* j : finished) {
                // records arrive step by step (the raster is appended in step
                // order), unordered within a step: sort each step's ids
                size_t a = 0;
                while (a < j->steps.size()) {
                    size_t b = a + 1;
                    while (b < j->steps.size() && j->steps[b] == j->steps[a]) ++b;
                    std::sort(j->ids.begin() + a, j->ids.begin() + b);
                    a = b;
                }
            }
            const double t_drain = now_s() - t;
            {
                std::lock_guard<std::mutex> lk(mu_);
                const double tn2 = now_s();
                for (Job* j : preempted) {  // device memory freed by the builder, then rebuilt from the queue
                    j->preempt_req = false;
                    j->info.state = kJobQueued;
                    j->info.steps_done = j->resume_steps;
                    ++j->info.preemptions;
                    to_free_.push_back(j);
                    pending_.push_back(j->id);
                }
                for (Job* j : cancelled) {
                    j->cancel_req = false;
                    j->info.state = kJobCancelled;
                    j->info.error = "cancelled";
                    j->steps.clear();
                    j->ids.clear();
                    to_free_.push_back(j);
                }
                if (!preempted.empty() || !cancelled.empty()) {
                    cv_build_.notify_all();
                    cv_done_.notify_all();
                }
                for (Job* j : finished) {
                    j->info.state = kJobDone;
                    j->info.done_s = tn2;
                    j->info.steps_done = j->info.duration;
                    j->info.spikes = j->steps.size();
                    latencies_ms_.push_back(1e3 * (tn2 - j->info.submit_s));
                    last_done_s_ = tn2;
                    ++st_.done;
                    to_free_.push_back(j);  // no queued launch uses it any more
                }
                for (Job* j : running) j->info.steps_done = std::min<uint64_t>(hs - j->net->dev.start_step, j->info.duration);
                if (inflight) ++st_.chunks;
                st_.engine_steps = eng->host_step();
                st_.install_s += t_install;
                st_.step_s += t_step;
                st_.drain_s += t_drain;
                st_.raster_dropped += dropped;
                st_.running = running.size();
                if (trace && done_len) {
                    uint64_t rchunks = 0;
                    for (Job* j : running) rchunks += j->chunks;
                    std::fprintf(trace, "%.6f,%zu,%zu,%zu,%llu,%.3f,%.3f,%.3f,%.3f,%llu,%zu,%llu,%llu,%llu\n", tn2,
                                 running.size(), admit.size(), finished.size(), (unsigned long long)done_len, done_ms,
                                 1e3 * t_step, 1e3 * t_install, 1e3 * t_drain, (unsigned long long)nrec, pending_.size(),
                                 (unsigned long long)used_, (unsigned long long)rchunks, (unsigned long long)chunk_cap);
                }
                if (!finished.empty()) {
                    cv_done_.notify_all();
                    cv_build_.notify_all();
                }
            }
        }
        if (inflight) eng->sync();
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(mu_);
        fatal_ = e.what();
        for (auto& kv : jobs_) {
            if (kv.second->info.state < kJobDone) {
                kv.second->info.state = kJobFailed;
                kv.second->info.error = fatal_;
                ++st_.failed;
            }
        }
        pending_.clear();
        stop_ = true;
        cv_done_.notify_all();
    }
    if (eng) cudaStreamSynchronize(eng->stream());
    if (rec) cudaFreeHost(rec);
    if (copied) cudaEventDestroy(copied);
    if (c0) cudaEventDestroy(c0);
    if (c1) cudaEventDestroy(c1);
    if (trace) std::fclose(trace);
    // running jobs are abandoned: the builder frees them
    std::lock_guard<std::mutex> lk(mu_);
    for (Job* j : running) {
        if (j->info.state < kJobDone) {
            j->info.state = kJobFailed;
            j->info.error = "server stopped";
        }
        to_free_.push_back(j);
    }
    for (auto& kv : jobs_) {
        if (kv.second->info.state < kJobDone) {
            kv.second->info.state = kJobFailed;
            if (kv.second->info.error.empty()) kv.second->info.error = "server stopped";
        }
    }
    stepper_done_ = true;
    cv_done_.notify_all();
    cv_build_.notify_all();
}

}  // namespace naer
