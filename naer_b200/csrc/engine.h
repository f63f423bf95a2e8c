// Host engine: owns device memory, builds networks, runs the step loop.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/naer/naer_capi.h"
#include "engine_types.cuh"

namespace naer {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what);
#define NAER_CK(x) ::naer::cuda_check((x), #x)

constexpr int32_t kFxUnknown = -2;  // NetHost::fx_shift not computed yet

struct PopSpec {
    uint32_t type = kNOP;
    uint32_t size = 0;
    naer_pop_params prm{};
    uint32_t type_address = 0;  // address within its neuron type (before compile)
    // after layout
    uint32_t id_base = 0;       // reference address (net-local)
    uint32_t storage_base = 0;
};

// Synapses given explicitly (naer_net_add_connection_csr): a CSR over the
// source population, targets as indices within the destination population.
struct ExplicitCsr {
    std::vector<uint64_t> row_ptr;  // [src_size + 1]
    std::vector<uint32_t> tgt;
    std::vector<float> w;
    std::vector<uint8_t> dly;
};

struct ConnSpec {
    uint32_t src = 0, dst = 0;
    naer_conn_spec spec{};
    std::shared_ptr<const ExplicitCsr> csr;  // rule NAER_CONN_EXPLICIT
};

// One network: description, layout and device arrays.
struct NetHost {
    naer_net_params params{};
    std::vector<PopSpec> pops;
    std::vector<ConnSpec> conns;
    bool compiled = false;
    int32_t fx_shift = kFxUnknown;  // exact-sum grid shift S, computed when an exact-mode engine installs the net

    // layout
    std::vector<uint32_t> pop_order;   // pops in type order
    uint32_t n_ids = 0, n_storage = 0, n_plastic = 0, ring_slots = 0;
    uint32_t n_poisson = 0;
    uint64_t synapses = 0, synapses_padded = 0, max_row_padded = 0;
    uint64_t max_first_padded = 0, max_rest_padded = 0;  // longest delay-1 part / rest of a row, padded
    uint64_t syn_capacity = 0;  // entries allocated for tgt / w / dly (>= synapses_padded)
    std::vector<int32_t> id_of_storage;   // -1 for padding
    std::vector<uint32_t> storage_of_id;

    // device arrays (owned)
    float* v = nullptr;
    uint8_t* refr = nullptr;
    float* ring = nullptr;
    uint8_t* drive = nullptr;
    uint64_t* row_ptr = nullptr;
    uint32_t* row_mid = nullptr;
    uint32_t* tgt = nullptr;
    float* w = nullptr;
    uint8_t* dly = nullptr;
    int32_t* post = nullptr;   // [n_plastic][post_stride] packed post rows
    int2* pre = nullptr;       // [n_plastic] {last pre step, pre trace bits}
    uint32_t post_stride = 0;
    float* e_plus = nullptr;
    float* e_minus = nullptr;
    uint32_t e_len = 0;
    // deterministic-aggregation scratch (allocated by the first deterministic step)
    float* det_w = nullptr;
    uint32_t* det_next = nullptr;
    uint32_t* det_head = nullptr;
    uint64_t device_bytes = 0;

    NetDev dev{};
};

// Device bytes a network will hold once built (synapse arrays, state, ring,
// drive slots, plasticity state), from its description alone.  Also
// validates the description (the checks compile makes).
uint64_t estimate_device_bytes(const NetHost& description, bool deterministic = false);

// LIF work items (chunks of up to 1,024 neurons of one population) a
// network adds to an engine, from its description alone.
uint32_t lif_chunks(const NetHost& description);

// Test hook: the device allocation `after` allocations from now fails with
// NAER_E_OOM (once); -1 turns it off.
void set_allocation_failure(int64_t after);

// Bytes of one network's saved simulation state (Engine::save_state).
uint64_t state_bytes(const NetHost& n);

// Device probe (probe.cu), see naer_probe_device.
void probe_device(int device, uint64_t ring_cells, uint64_t small_cells, naer_device_probe* out);
void probe_intervals(int device, double rate_hz, uint32_t z_first, uint32_t z_step, uint64_t count, uint32_t* out);

// Launch geometry of the persistent step loop (all choices leave the
// simulated results unchanged).
struct Tuning {
    uint32_t blocks_per_sm = 0;            // resident step-kernel blocks per SM (0 = most that fit)
    uint32_t launch_steps = kDriveSlots;   // grid steps per persistent launch (1..kDriveSlots)
    uint32_t scatter_split = 0;            // warps per spike (0 = enough to cover the longest row)
    uint32_t scatter_piece = 0;            // synapses per warp iteration: 128, 256, 0 = 128 with STDP else 256
    uint32_t neuron_state = 0;             // NAER_STATE_AUTO / _SHARED / _GLOBAL: where the step kernel keeps V
    uint32_t step_kernel = 0;              // NAER_KERNEL_SPLIT (k_step) / NAER_KERNEL_TWO_BARRIER (k_run)
    uint32_t bins = 0;                     // k_step shared-memory binning table entries (0 = off)
};

struct TuneResult {
    Tuning best;
    double best_us_per_step = 0;
    double default_us_per_step = 0;
    uint32_t trials = 0;
};

class Engine {
public:
    // priority: CUDA stream priority of the engine's stream (lower = higher)
    explicit Engine(int device, int priority = 0);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }

    // Lays out and builds a network on the device (connectivity included).
    void build(NetHost& net);
    void free_net(NetHost& net);
    // Installs the nets' descriptor tables; nets must outlive the engine use.
    void exact_shifts(const std::vector<NetHost*>& nets);
    void install(const std::vector<NetHost*>& nets, uint64_t raster_capacity, bool record,
                 uint32_t aggregation);

    void run(uint64_t nsteps);
    // Atomic mode: the same steps, with the launch sequence of `graph_launches`
    // persistent launches recorded once in a CUDA graph and replayed (the
    // remainder runs as plain launches).  Returns the steps run by replays.
    uint64_t run_graph(uint64_t nsteps, uint32_t graph_launches);
    void set_tuning(const Tuning& t);
    // Most LIF chunks an installation can hold while the step kernel keeps
    // neuron state in shared memory at the most resident blocks per SM it
    // can have under the current tuning (its fastest geometry); beyond it
    // the step runs with fewer blocks or with state in global memory.
    uint32_t fast_chunk_capacity(uint32_t aggregation);
    // Times candidate launch geometries on the installed networks (each
    // trial advances the simulation by trial_steps grid steps) and keeps
    // the fastest.  Deterministic aggregation: nothing to tune.
    TuneResult autotune(uint32_t trial_steps);
    const Tuning& tuning() const { return tuning_; }
    uint32_t lif_grid() const { return lif_grid_; }
    uint32_t scatter_split() const { return eng_.scatter_split; }
    uint32_t blocks_per_sm() const { return lif_grid_ / (uint32_t)sm_count_; }
    // engine-global raster id of each installed net's reference address 0
    const std::vector<uint32_t>& id_offsets() const { return id_offsets_; }
    const std::vector<NetHost*>& nets() const { return nets_; }
    // Deterministic-aggregation steps whose scratch is the library's fixed
    // device arena: no device memory is allocated or freed by the call.
    void run_fixed_scratch(uint64_t nsteps);
    void sync();
    Ctl read_ctl();
    uint64_t host_step() const { return host_step_; }

    // raster records [first, first+cap) -> (step, id); returns count copied
    uint64_t read_raster(uint64_t first, uint64_t cap, uint32_t* steps, uint32_t* ids);
    uint64_t read_raster_raw(uint64_t first, uint64_t cap, uint32_t* records);
    // Waits for the queued steps, then queues the copy of all raster records
    // into `dst` (pinned, >= raster capacity), records `copied` after it and
    // clears the raster, all in stream order, so that further steps may be
    // queued before the host reads `dst` (after `copied`).  Returns the
    // record count; *dropped receives the records lost to a full raster.
    uint64_t harvest_raster(uint2* dst, cudaEvent_t copied, uint64_t* dropped);
    void clear_raster();

    void set_profiling(bool on);
    void get_profile(double* lif_ms, double* scatter_ms, uint64_t* launches);
    void get_phases(double* ms5);
    void get_launch_times(double* drive_ms, double* run_ms, uint64_t* run_launches);

    uint64_t device_bytes() const { return bytes_; }
    // launches of this library's own step kernels since creation
    uint64_t kernel_launches() const { return launches_; }
    uint64_t events_total();
    uint64_t overflow_total();

    void* dalloc(size_t bytes);
    void dfree(void* p, size_t bytes);

    // Simulation state of one network between steps (state_bytes() bytes:
    // neuron state, ring, plasticity state), to host memory and back.  The
    // network must be built; nothing may be queued that uses it.
    void save_state(const NetHost& n, uint8_t* dst);
    void load_state(NetHost& n, const uint8_t* src);
    // Sets the engine step (a restored network continues from it), empties
    // the raster and restarts the event counter at `events`.
    void set_step(uint64_t step, uint64_t events);

    // Bounded waits of the step kernel's grid barriers (0 = default) and the
    // test hook that makes every barrier unsatisfiable (see naer_capi.h).
    void set_barrier_limit(uint64_t limit_ns);
    void set_barrier_skew(uint64_t skew);
    // Device error flag of the control block, as a NAER_E_* status (0 =
    // none); once non-zero the engine refuses further steps.
    int device_status();

private:
    void build_arrays(NetHost& n);
    std::vector<std::pair<void*, size_t>>* alloc_log_ = nullptr;  // allocations of a build in progress
    void launch_run(uint32_t steps);
    void launch_drive(uint64_t s_first, uint32_t nsteps);
    void run_launches(uint64_t nsteps);
    void regrow(void*& p, size_t& have, size_t need);
    // deterministic-aggregation scratch: which one the installed tables point at
    static constexpr uint32_t kScratchNone = 0, kScratchOwn = 1, kScratchArena = 2;
    uint32_t det_scratch_ = kScratchNone;
    std::vector<float*> arena_w_;
    std::vector<uint32_t*> arena_next_, arena_head_;
    void ensure_det_scratch();
    void point_det_scratch(uint32_t mode);
    uint64_t sum_parts(const unsigned long long* d, uint32_t n);

    int device_ = 0;
    int sm_count_ = 148;
    cudaStream_t stream_ = nullptr;
    uint64_t bytes_ = 0;

    std::vector<NetHost*> nets_;
    EngineDev eng_{};
    NetDev* d_nets_ = nullptr;
    PopDev* d_pops_ = nullptr;
    ChunkDev* d_chunks_ = nullptr;
    Ctl* d_ctl_ = nullptr;
    SpikeRec* d_queue_[2] = {nullptr, nullptr};
    uint32_t* d_qid_[2] = {nullptr, nullptr};
    uint4* d_qrow_[2] = {nullptr, nullptr};
    size_t qrow_bytes_[2] = {0, 0};
    uint32_t* d_counts_[2] = {nullptr, nullptr};
    unsigned long long* d_ev_part_ = nullptr;
    unsigned long long* d_ovf_part_ = nullptr;
    uint32_t ev_part_n_ = 0;
    uint64_t events_base_ = 0, overflow_base_ = 0;
    uint2* d_raster_ = nullptr;
    size_t nets_bytes_ = 0, pops_bytes_ = 0, chunks_bytes_ = 0, raster_bytes_ = 0;
    size_t queue_bytes_[2] = {0, 0}, qid_bytes_[2] = {0, 0}, counts_bytes_[2] = {0, 0};
    size_t ev_part_bytes_ = 0, ovf_part_bytes_ = 0;
    size_t scatter_smem_ = 0;
    std::vector<NetDev> h_nets_;
    uint32_t queue_cap_ = 0;
    uint32_t aggregation_ = NAER_AGG_ATOMIC;
    uint32_t lif_grid_ = 0, scatter_grid_ = 0;
    uint32_t drive_grid_ = 0;  // resident blocks of k_drive
    uint64_t host_step_ = 0;
    uint64_t launches_ = 0;
    Tuning tuning_{};
    uint64_t inst_raster_cap_ = 0;
    bool inst_record_ = false;
    std::vector<uint32_t> id_offsets_;
    cudaGraphExec_t graph_exec_ = nullptr;
    uint32_t graph_launches_ = 0;
    void drop_graph();
    void launch_run_ex(uint32_t steps, bool from_ctl);
    uint64_t total_ring_cells_ = 0;


    uint32_t* h_pinned_ = nullptr;  // small pinned staging

    bool failed_ = false;  // a launch reported a device error: state undefined
    void check_usable() const;
    bool profiling_ = false;
    bool use_smem_state_ = false;
    bool split_kernel_ = true;  // k_step (else k_run)
    // CUDA-event timing of launches while profiling (pairs in launch order)
    std::vector<cudaEvent_t> timer_events_;
    std::vector<int> timer_kinds_;  // 0 drive, 1 step kernel
    std::vector<uint32_t> run_pairs_;
    double drive_ms_ = 0, run_ms_ = 0;
    uint64_t run_launches_ = 0;
    cudaEvent_t timer_event();
    void resolve_timers();
};

}  // namespace naer
