// Batched and served forms: many independent networks stepped together by
// one engine (one set of persistent launches per step chunk).
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"

namespace naer {

// Batched form: members are added as descriptions, built on one engine and
// stepped together; all start at engine step 0.
class Batch {
public:
    Batch(int device, uint32_t aggregation, uint64_t raster_capacity, bool record);
    uint32_t add(const NetHost& description);
    void compile();
    // Steps every member; atomic mode replays a CUDA graph of
    // `graph_launches` persistent launches when nsteps allows.
    void step(uint64_t nsteps, uint32_t graph_launches);
    // Times candidate launch geometries on the batch itself (each trial
    // advances the simulation by trial_steps) and keeps the fastest.
    TuneResult autotune(uint32_t trial_steps);
    // Raster records [first, first + cap) with their member index; steps are
    // engine steps (= member steps, all members start at 0).
    uint64_t read_spikes(uint64_t first, uint64_t cap, uint32_t* member, uint32_t* steps, uint32_t* ids);
    Engine& engine() { return *eng_; }
    NetHost& member(uint32_t i) { return *members_.at(i); }
    size_t size() const { return members_.size(); }
    bool compiled() const { return compiled_; }
    uint32_t aggregation() const { return aggregation_; }

private:
    std::unique_ptr<Engine> eng_;
    std::vector<std::unique_ptr<NetHost>> members_;
    uint32_t aggregation_;
    uint64_t raster_capacity_;
    bool record_;
    bool compiled_ = false;
};

struct ServerParams {
    uint64_t budget_bytes = 0;     // admitted networks' device bytes stay below this
    uint32_t chunk_steps = 256;    // grid steps between admission points
    uint32_t aggregation = 0;      // NAER_AGG_*
    uint32_t max_jobs = 1024;      // networks stepped together at most
    uint64_t raster_capacity = 1ull << 24;  // spike records per chunk
    uint32_t blocks_per_sm = 0;    // step-kernel blocks per SM (0 = most that fit)
    double chunk_ms = 10.0;        // target device time per chunk (sets its step count)
    uint32_t launch_steps = 4;     // grid steps per persistent step launch (builds run between launches)
    uint32_t step_kernel = 1;      // NAER_KERNEL_TWO_BARRIER (k_run) / NAER_KERNEL_SPLIT (k_step)
};

enum JobState : uint32_t { kJobQueued = 0, kJobRunning = 1, kJobDone = 2, kJobFailed = 3, kJobCancelled = 4 };

struct JobInfo {
    uint32_t state = kJobQueued;
    uint32_t preemptions = 0;  // times the job was taken off the device and later resumed
    uint64_t duration = 0, steps_done = 0, spikes = 0, spikes_dropped = 0;
    uint64_t device_bytes = 0;
    double submit_s = 0, admit_s = 0, done_s = 0;  // seconds since the server started
    std::string error;
};

struct ServerStats {
    uint64_t submitted = 0, done = 0, failed = 0, running = 0, queued = 0;
    uint64_t chunks = 0, engine_steps = 0, peak_bytes = 0, bytes_in_use = 0, raster_dropped = 0;
    double p50_ms = 0, p99_ms = 0, mean_ms = 0;
    double sims_per_s = 0;  // jobs done / (last done - first submit)
    // host seconds spent by the two server threads
    double build_s = 0;     // builder: networks built on the device
    double install_s = 0, step_s = 0, drain_s = 0;  // stepper: tables, chunks, rasters
};

// Served form: jobs (description, duration) are admitted as device memory
// and slots free up, stepped together with the jobs already running (their
// state stays on the device), and retired when their duration is reached.
// Two threads: the builder admits queued jobs first come, first served
// while their estimated bytes fit the budget, builds them on its own engine
// and stream (build kernels interleave with the step launches), and frees
// retired jobs; the stepper owns the step engine, takes built jobs in at
// every chunk boundary, runs the chunk, hands its raster to the jobs and
// retires those that reached their duration.  Public methods are
// thread-safe.
class Server {
public:
    Server(int device, const ServerParams& p);
    ~Server();
    uint64_t submit(const NetHost& description, uint64_t duration_steps);
    JobInfo info(uint64_t job);
    // raster of a finished job, sorted by (step, id); steps are job-local
    uint64_t read_spikes(uint64_t job, uint64_t first, uint64_t cap, uint32_t* steps, uint32_t* ids);
    bool wait(uint64_t job, double timeout_s);
    bool drain(double timeout_s);
    void release(uint64_t job);
    // Takes a running job off the device at the next chunk boundary: its
    // state is saved to host memory, its device memory freed, and it queues
    // again; when re-admitted it is rebuilt, restored and continues from the
    // same step (deterministic jobs give the raster of an uninterrupted run).
    void preempt(uint64_t job);
    // Ends a job that has not finished: queued or built jobs at once, a
    // running job at the next chunk boundary.  Its raster is discarded.
    void cancel(uint64_t job);
    ServerStats stats();

private:
    struct Job {
        uint64_t id = 0;
        std::unique_ptr<NetHost> net;
        JobInfo info;
        uint64_t est_bytes = 0;
        uint32_t chunks = 0;    // LIF chunks it adds to the stepping engine
        std::vector<uint32_t> steps, ids;
        bool freed = false;     // holds no device memory
        bool released = false;  // forgotten by the caller: erase once freed
        bool preempt_req = false, cancel_req = false;
        std::vector<uint8_t> saved;  // state of a pre-empted job until it is rebuilt
        uint64_t resume_steps = 0;   // job-local step it resumes from
    };
    void loop();
    void build_loop();
    double now_s() const;

    int device_;
    ServerParams prm_;
    std::chrono::steady_clock::time_point t0_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_, cv_build_;
    std::map<uint64_t, std::unique_ptr<Job>> jobs_;
    std::deque<uint64_t> pending_;   // submitted, not yet built
    std::deque<Job*> ready_;         // built, not yet stepping
    std::deque<Job*> to_free_;       // retired, device memory still held
    uint64_t used_ = 0;              // estimated bytes of built, unfreed jobs
    uint32_t live_ = 0;              // built, unfreed jobs
    uint64_t next_id_ = 1;
    bool stop_ = false;
    bool stepper_done_ = false;
    std::string fatal_;
    ServerStats st_{};
    std::vector<double> latencies_ms_;
    double first_submit_s_ = -1, last_done_s_ = 0;
    std::thread worker_, builder_;
};

}  // namespace naer
