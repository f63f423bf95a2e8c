// Device-visible descriptors shared by the kernels and the host engine.
//
// One engine holds any number of networks ("nets").  Every kernel reads its
// work from these tables, so a plain run (one net), a packed batch and the
// served slot table all go through the same kernels.
//
// Storage index space of a net: populations are laid out in the reference's
// type order (STDP, then NOP, then POISSON; src/Network.cpp:267-285), each
// population starting on a multiple of 4 so that four neurons share one
// float4 of membrane potential.  The gaps are inert padding neurons (no
// synapses in or out, never spike).  Reference addresses ("ids") are the
// unpadded type-ordered addresses; each population records both bases.
#pragma once
#include <stdint.h>

namespace naer {

enum NeuronType : uint32_t { kSTDP = 0, kNOP = 1, kPOISSON = 2 };

constexpr uint32_t kTgtSentinel = 0xFFFFFFFFu;  // padding entry in a CSR row
constexpr uint32_t kNoEvent = 0xFFFFFFFFu;      // end of a ring cell's event list
constexpr uint32_t kRowAlign = 4;               // rows start on 16-byte boundaries
constexpr uint32_t kLifThreads = 256;
constexpr uint32_t kLifPerThread = 4;
constexpr uint32_t kLifChunk = kLifThreads * kLifPerThread;  // neurons per LIF work item
constexpr uint32_t kScatterThreads = 256;
constexpr uint32_t kScatterUnroll = 2;  // 128-synapse slices in flight per warp
constexpr uint32_t kScatterPiece = 128 * kScatterUnroll;  // synapses per warp iteration
constexpr uint32_t kPlasticPiece = 32;  // k_step: synapses per warp iteration of a plastic source's row
// Steps of Poisson counts drawn ahead (ring of slots); small enough that the
// counts and the delay ring stay resident in L2 together.
#ifndef NAER_DRIVE_SLOTS
#define NAER_DRIVE_SLOTS 64  // 64 measured fastest at 1M / 1e9 (26.5 vs 28.1 us per step with 16)
#endif
constexpr uint32_t kDriveSlots = NAER_DRIVE_SLOTS;  // Poisson-count slots = grid steps per launch, at most
// STDP post-spike history: at most this many entries per plastic neuron, so
// a packed post row (2 + history words, rounded up to 4) fits kPostWordsMax.
constexpr uint32_t kMaxStdpHistory = 16;
constexpr uint32_t kPostWordsMax = 20;
// Step argument of k_drive / k_run meaning "the engine step in Ctl::step"
// (launches recorded once in a CUDA graph and replayed).
constexpr unsigned long long kStepFromCtl = ~0ull;
constexpr uint32_t kLifBatch = 4;     // owned chunks whose loads are issued together

struct PopDev {
    uint32_t net;           // owning net slot
    uint32_t type;          // NeuronType
    uint32_t storage_base;  // first storage index (multiple of 4)
    uint32_t size;          // neurons
    uint32_t id_base;       // reference address of the first neuron (engine-global)
    uint32_t t_ref_steps;   // refractory steps after a spike
    float v_th;             // spike iff V > v_th (lif.cl:28)
    float v_reset;
    double prop;            // exp(-dt / tau_m), computed on the host
    // Poisson generator (POISSON populations: their own spikes; LIF
    // populations: per-neuron external drive).  rate_hz == 0 disables.
    double rate_hz;
    float drive_w;          // LIF drive weight per Poisson event
    uint32_t rng_seed;      // Philox key word 1
    uint32_t rng_n;         // N in the counter t0 * N + idx
    uint32_t rng_idx_base;  // idx of the first neuron in the generator's index space
    uint32_t z_hi;          // z in [z_hi, 0xFFFFFFFE] => first interval >= window
    uint32_t t0_limit;      // fast path valid while t0 <= t0_limit (no u32 wrap)
};

struct NetDev {
    float* v;               // [n_storage] membrane potential
    uint8_t* refr;          // [n_storage] refractory countdown (steps)
    float* ring;            // [ring_slots][n_storage] delayed input
    uint8_t* drive;         // [kDriveSlots][n_storage] Poisson events per step (drive or own spikes)
    const uint64_t* row_ptr;  // [n_storage + 1], row starts multiple of kRowAlign
    const uint32_t* row_mid;  // [n_storage] offset of the row's part of delay > 1 (multiple of kRowAlign)
    const uint32_t* tgt;    // [S] target storage index or kTgtSentinel
    float* w;               // [S] weight (written back by STDP)
    const uint8_t* dly;     // [S] delay in steps, 1..ring_slots-1
    // pair-based STDP state, one entry per plastic storage index
    // Packed post-synaptic row of each plastic neuron, post_stride int32
    // words (a multiple of 4, so one row is read with int4 loads): [0] step
    // of the newest post spike that has left the history (-1 = none), [1]
    // post trace right after the latest post spike (float bits), [2, 2 +
    // hist_len) post spike steps, newest first (-1 = none); [2] is the
    // latest post spike.
    int32_t* post;
    int2* pre;              // {step of the latest pre spike (-1 = none), pre trace after it (float bits)}
    const float* e_plus;    // [e_len] exp(-k dt / tau_plus) as float
    const float* e_minus;   // [e_len] exp(-k dt / tau_minus) as float
    // deterministic aggregation: per padded synapse j, the weight it delivered
    // in the current step and the next event of its ring cell's list; per
    // ring cell, the list head (kNoEvent when empty between steps)
    float* ev_w;
    uint32_t* ev_next;
    uint32_t* cell_head;
    uint64_t start_step;    // engine step at which this net's step 0 runs
    uint64_t end_step;      // first engine step at which this net no longer runs (~0 = never)
    uint64_t ring_key_base; // first ring cell of this net in the deterministic key space
    uint64_t syn_cap;       // entries of tgt / w / dly (bounds of the checked build)
    uint32_t n_storage;     // multiple of 4
    uint32_t ring_slots;    // D = max delay + 1
    uint32_t dt_us;         // grid step in microseconds
    uint32_t n_plastic;     // storage indices below this are STDP neurons
    uint32_t stdp_on;       // plasticity enabled for this net
    uint32_t hist_len;
    uint32_t post_stride;   // words per post row
    uint32_t e_len;
    float a_plus;           // A+ * w_max
    float a_minus;          // A- * w_max
    float w_max;
    uint32_t active;        // 0 = slot idle (served form)
    // exact-sum aggregation: weights delivered as integers on the grid 2^-S
    // (fx_scale = 2^S, fx_inv = 2^-S); both 0 when the ring holds floats
    float fx_scale;
    float fx_inv;
    uint32_t pad_;
};

struct ChunkDev {
    uint32_t pop;    // population index
    uint32_t first;  // first storage index (multiple of 4)
    uint32_t end;    // one past the last storage index of the population in this chunk
    uint32_t net;    // net slot of the population
};

// One spike in the device queue.  aux0/aux1 carry the source's pre-synaptic
// trace state before this spike (STDP sources), or the Poisson multiplicity
// in aux0 (POISSON sources); the reference's spike record carries the same
// pre information (previous_times, pre_traces: include/naer/naer_types.h:9-21).
struct SpikeRec {
    uint32_t net;
    uint32_t src;    // storage index
    int32_t aux0;    // old last_pre step | multiplicity
    float aux1;      // old x_pre
};

// Device control block.
//   step        engine step being simulated (read by the kernels of the
//               deterministic path; the persistent kernel takes it as an
//               argument and stores the end step)
//   raster_base raster records before the current step (deterministic path)
//   raster_next raster records kept so far
//   bar_arrive  grid barrier arrivals of the persistent kernel (zeroed per launch)
//   error       first device-side error (negated NAER status), 0 = none
//   prof_*      phase times of the persistent kernel (block 0, %globaltimer)
struct Ctl {
    unsigned long long step;
    unsigned long long raster_base;
    unsigned long long raster_next;
    unsigned long long raster_dropped;
    unsigned long long events;      // deterministic-mode events (atomic mode: per-block counters)
    unsigned long long stdp_hist_overflow;
    unsigned long long prof_lif_ns;
    unsigned long long prof_scatter_ns;
    unsigned long long prof_steps;
    unsigned long long prof_phase_ns[5];  // LIF, barrier 1, early scatter, late scatter, barrier 2
    unsigned long long bar_arrive;  // grid barrier arrivals of the running launch
    unsigned int qtail[4];          // k_step: spikes queued in step s, slot s & 3 (zeroed with bar_arrive)
    unsigned int error;
    unsigned int pad_;
    unsigned int chk_code;          // NAER_CHECKED build: first out-of-bounds access (CheckCode), 0 = none
    unsigned int pad2_;
    unsigned long long chk_index;   // its index
    unsigned long long bar_limit_ns;  // bounded wait of one grid barrier (0 = kBarrierLimitNs)
    unsigned long long bar_skew;      // added to every barrier target: 0, except when a test makes the
                                      // wait unsatisfiable to exercise the timeout (naer_test_set_barrier_skew)
};

constexpr unsigned long long kBarrierLimitNs = 2000000000ull;  // 2 s

constexpr int NAER_STATUS_OVERFLOW = -3;  // NAER_E_OVERFLOW of the C ABI
constexpr int NAER_STATUS_TIMEOUT = -4;   // NAER_E_TIMEOUT of the C ABI

// Spike queue.  k_run and the deterministic path: LIF block b compacts its
// spikes into region [b * region_cap, (b + 1) * region_cap) of the step's
// buffer and writes their number to counts[b]; the scatter prefix-sums the
// counts.  k_step: one contiguous list per step, each warp reserving its
// spikes' places with one atomic on Ctl::qtail.
struct EngineDev {
    Ctl* ctl;
    const NetDev* nets;
    const PopDev* pops;
    const ChunkDev* chunks;
    SpikeRec* queue[2];
    uint32_t* qid[2];               // reference address of each queued spike
    uint4* qrow[2];                 // k_step / k_det_step: row of each queued spike {begin lo, begin hi,
                                    // delay-1 part length, row length}, written with the record
    uint32_t* counts[2];            // [lif_grid] spikes per LIF block region
    unsigned long long* ev_part;    // [scatter_grid] events delivered, per scatter block
    unsigned long long* ovf_part;   // [scatter_grid] lazy-LTP history overflows, per block
    uint2* raster;                  // {engine step, id}
    unsigned long long raster_cap;
    uint32_t n_chunks;
    uint32_t n_nets;
    uint32_t lif_grid;
    uint32_t region_cap;
    uint32_t record;                // append spikes to the raster
    uint32_t scatter_split;         // warps per spike (row pieces of scatter_piece)
    uint32_t scatter_piece;         // synapses per warp iteration: 128 or kScatterPiece
    // k_step: warps per spike over the part of a row that must arrive
    // before the next LIF (the delay-1 part; whole rows of plastic sources)
    // and over the rest (delays >= 2 of static sources)
    uint32_t split_first;
    uint32_t split_rest;
    uint32_t queue_cap;             // entries of queue[i] / qid[i]
    uint32_t bins;                  // k_step: shared-memory binning table entries (power of 2), 0 = off
};

}  // namespace naer
