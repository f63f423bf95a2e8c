// Batched and served forms (see forms.h).
#include "forms.h"

#include <algorithm>
#include <cmath>

namespace naer {

namespace {

struct CurrentDevice {
    int prev = -1;
    explicit CurrentDevice(int dev) {
        NAER_CK(cudaGetDevice(&prev));
        if (prev != dev) NAER_CK(cudaSetDevice(dev));
    }
    ~CurrentDevice() {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) cudaSetDevice(prev);
    }
};

std::unique_ptr<NetHost> clone_description(const NetHost& d) {
    if (d.compiled) throw Error(NAER_E_STATE, "a compiled network cannot be used as a description");
    auto n = std::make_unique<NetHost>();
    n->params = d.params;
    n->pops = d.pops;
    n->conns = d.conns;
    return n;
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
    if (aggregation > NAER_AGG_DETERMINISTIC) throw Error(NAER_E_INVALID, "unknown aggregation");
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
    if (aggregation_ == NAER_AGG_DETERMINISTIC)
        eng_->run(nsteps);
    else
        eng_->run_graph(nsteps, graph_launches);
}

TuneResult Batch::autotune(uint32_t trial_steps) {
    if (!compiled_) throw Error(NAER_E_STATE, "batch is not compiled");
    TuneResult r;
    r.best = eng_->tuning();
    if (aggregation_ == NAER_AGG_DETERMINISTIC || trial_steps == 0) return r;
    CurrentDevice g(eng_->device());
    cudaEvent_t e0, e1;
    NAER_CK(cudaEventCreate(&e0));
    NAER_CK(cudaEventCreate(&e1));
    auto trial = [&](const Tuning& t) {
        eng_->set_tuning(t);
        eng_->run(t.launch_steps);  // first launch of the new geometry
        NAER_CK(cudaEventRecord(e0, eng_->stream()));
        eng_->run(trial_steps);
        NAER_CK(cudaEventRecord(e1, eng_->stream()));
        NAER_CK(cudaEventSynchronize(e1));
        float ms = 0;
        NAER_CK(cudaEventElapsedTime(&ms, e0, e1));
        ++r.trials;
        return 1e3 * ms / trial_steps;
    };
    try {
        const Tuning def{};
        r.default_us_per_step = trial(def);
        r.best = def;
        r.best_us_per_step = r.default_us_per_step;
        const uint32_t auto_split = eng_->scatter_split();
        for (uint32_t bps : {0u, 1u}) {
            for (uint32_t L : {16u, 8u}) {
                for (uint32_t sp : {0u, std::max<uint32_t>(1, auto_split / 2), std::min<uint32_t>(64, auto_split * 2)}) {
                    Tuning t;
                    t.blocks_per_sm = bps;
                    t.launch_steps = L;
                    t.scatter_split = sp;
                    if (bps == 0 && L == 16 && sp == 0) continue;  // the default, timed above
                    const double us = trial(t);
                    if (us < r.best_us_per_step) {
                        r.best_us_per_step = us;
                        r.best = t;
                    }
                }
            }
        }
        eng_->set_tuning(r.best);
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    NAER_CK(cudaEventDestroy(e0));
    NAER_CK(cudaEventDestroy(e1));
    return r;
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
    if (p.aggregation > NAER_AGG_DETERMINISTIC) throw Error(NAER_E_INVALID, "unknown aggregation");
    if (p.chunk_steps == 0) throw Error(NAER_E_INVALID, "chunk_steps must be positive");
    if (p.max_jobs == 0) throw Error(NAER_E_INVALID, "max_jobs must be positive");
    if (p.raster_capacity == 0) throw Error(NAER_E_INVALID, "raster_capacity must be positive");
    int n = 0;
    NAER_CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) throw Error(NAER_E_INVALID, "device index out of range");
    worker_ = std::thread([this] { loop(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    if (worker_.joinable()) worker_.join();
}

double Server::now_s() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

uint64_t Server::submit(const NetHost& description, uint64_t duration_steps) {
    if (duration_steps == 0) throw Error(NAER_E_INVALID, "duration must be at least one step");
    auto j = std::make_unique<Job>();
    j->net = clone_description(description);
    j->est_bytes = estimate_device_bytes(*j->net);
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
    cv_work_.notify_all();
    return id;
}

JobInfo Server::info(uint64_t job) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end()) throw Error(NAER_E_INVALID, "unknown job");
    return it->second->info;
}

uint64_t Server::read_spikes(uint64_t job, uint64_t first, uint64_t cap, uint32_t* steps, uint32_t* ids) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(job);
    if (it == jobs_.end()) throw Error(NAER_E_INVALID, "unknown job");
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
    if (it == jobs_.end()) throw Error(NAER_E_INVALID, "unknown job");
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
    if (it == jobs_.end()) throw Error(NAER_E_INVALID, "unknown job");
    if (it->second->info.state < kJobDone) throw Error(NAER_E_STATE, "job has not finished");
    jobs_.erase(it);
}

ServerStats Server::stats() {
    std::lock_guard<std::mutex> lk(mu_);
    ServerStats s = st_;
    s.queued = pending_.size();
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

// Worker: admit -> build -> (re)install -> one chunk of steps -> hand the
// chunk's raster to its jobs -> retire finished jobs.
void Server::loop() {
    std::unique_ptr<Engine> eng;
    std::vector<Job*> running;
    uint64_t used = 0;
    bool changed = false;
    std::vector<uint2> rec;
    auto fail_all = [&](const std::string& why) {
        std::lock_guard<std::mutex> lk(mu_);
        fatal_ = why;
        for (auto& kv : jobs_) {
            if (kv.second->info.state < kJobDone) {
                kv.second->info.state = kJobFailed;
                kv.second->info.error = why;
                ++st_.failed;
            }
        }
        pending_.clear();
        st_.running = 0;
        cv_done_.notify_all();
    };
    try {
        NAER_CK(cudaSetDevice(device_));
        eng = std::make_unique<Engine>(device_);
        for (;;) {
            std::vector<Job*> admit;
            {
                std::unique_lock<std::mutex> lk(mu_);
                if (running.empty()) cv_work_.wait(lk, [&] { return stop_ || !pending_.empty(); });
                if (stop_) break;
                // first come, first served: the queue head waits for memory
                while (!pending_.empty() && running.size() + admit.size() < prm_.max_jobs) {
                    Job* j = jobs_.at(pending_.front()).get();
                    if (used + j->est_bytes > prm_.budget_bytes) break;
                    pending_.pop_front();
                    admit.push_back(j);
                    used += j->est_bytes;
                }
            }
            for (Job* j : admit) {
                try {
                    eng->build(*j->net);
                } catch (const Error& e) {
                    if (e.code == NAER_E_CUDA) throw;
                    if (j->net->compiled) eng->free_net(*j->net);
                    used -= j->est_bytes;
                    std::lock_guard<std::mutex> lk(mu_);
                    j->info.state = kJobFailed;
                    j->info.error = e.what();
                    ++st_.failed;
                    cv_done_.notify_all();
                    continue;
                }
                j->net->dev.start_step = eng->host_step();
                j->net->dev.end_step = eng->host_step() + j->info.duration;
                running.push_back(j);
                changed = true;
                std::lock_guard<std::mutex> lk(mu_);
                j->info.state = kJobRunning;
                j->info.admit_s = now_s();
                j->info.device_bytes = j->net->device_bytes;
            }
            if (running.empty()) continue;
            if (changed) {
                std::vector<NetHost*> nets;
                for (Job* j : running) nets.push_back(j->net.get());
                eng->install(nets, prm_.raster_capacity, true, prm_.aggregation);
                changed = false;
            }
            const uint64_t hs = eng->host_step();
            uint64_t last_end = hs;
            for (Job* j : running) last_end = std::max<uint64_t>(last_end, j->net->dev.end_step);
            eng->run(std::min<uint64_t>(prm_.chunk_steps, last_end - hs));

            // the chunk's raster, handed to the jobs it belongs to
            const Ctl c = eng->read_ctl();
            const uint64_t nrec = std::min<uint64_t>(c.raster_next, prm_.raster_capacity);
            rec.resize(nrec);
            if (nrec) eng->read_raster_raw(0, nrec, reinterpret_cast<uint32_t*>(rec.data()));
            eng->clear_raster();
            const auto& off = eng->id_offsets();
            for (const uint2& r : rec) {
                const uint32_t m = member_of(off, r.y);
                Job* j = running[m];
                j->steps.push_back((uint32_t)(r.x - j->net->dev.start_step));
                j->ids.push_back(r.y - off[m]);
            }
            const uint64_t now_step = eng->host_step();
            std::vector<Job*> keep;
            std::vector<Job*> finished;
            for (Job* j : running) {
                if (now_step >= j->net->dev.end_step) finished.push_back(j); else keep.push_back(j);
            }
            for (Job* j : finished) {
                eng->free_net(*j->net);
                used -= j->est_bytes;
                // records of one step arrive unordered: order by (step, id)
                std::vector<uint64_t> key(j->steps.size());
                for (size_t i = 0; i < key.size(); ++i) key[i] = ((uint64_t)j->steps[i] << 32) | j->ids[i];
                std::sort(key.begin(), key.end());
                for (size_t i = 0; i < key.size(); ++i) {
                    j->steps[i] = (uint32_t)(key[i] >> 32);
                    j->ids[i] = (uint32_t)key[i];
                }
            }
            if (!finished.empty()) changed = true;
            running.swap(keep);
            {
                std::lock_guard<std::mutex> lk(mu_);
                const double t = now_s();
                for (Job* j : finished) {
                    j->info.state = kJobDone;
                    j->info.done_s = t;
                    j->info.steps_done = j->info.duration;
                    j->info.spikes = j->steps.size();
                    latencies_ms_.push_back(1e3 * (t - j->info.submit_s));
                    last_done_s_ = t;
                    ++st_.done;
                }
                for (Job* j : running) j->info.steps_done = now_step - j->net->dev.start_step;
                ++st_.chunks;
                st_.engine_steps = now_step;
                st_.bytes_in_use = used;
                st_.peak_bytes = std::max<uint64_t>(st_.peak_bytes, eng->device_bytes());
                st_.raster_dropped += c.raster_dropped;
                st_.running = running.size();
                if (!finished.empty()) cv_done_.notify_all();
            }
        }
        // shutting down: abandon what is still running
        for (Job* j : running) eng->free_net(*j->net);
        std::lock_guard<std::mutex> lk(mu_);
        for (auto& kv : jobs_) {
            if (kv.second->info.state < kJobDone) {
                kv.second->info.state = kJobFailed;
                kv.second->info.error = "server stopped";
            }
        }
        cv_done_.notify_all();
    } catch (const std::exception& e) {
        fail_all(e.what());
    }
}

}  // namespace naer
