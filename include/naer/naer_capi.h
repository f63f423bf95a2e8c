/*
 * naer_capi.h — C ABI of the B200 spiking-network step.
 *
 * This is the boundary the reference's C++ `Naer::Network`
 * (include/naer/Network.h:15-142, src/Network.cpp) drives.  The reference
 * holds OpenCL objects directly; here every device object lives behind an
 * opaque handle and every entry point is a plain C function: no C++ or torch
 * types cross the boundary, so ctypes, cgo, JNI or N-API can bind it.
 *
 * Conventions
 *  - Every function returns an int status: NAER_OK (0) or a negative
 *    NAER_E_* code.  naer_last_error() returns the message of the last
 *    failure on the calling thread.  No exception crosses the ABI; the C++
 *    wrapper in include/naer/Network.h turns a non-zero status into
 *    std::runtime_error, as the reference does for every OpenCL failure
 *    (e.g. src/Network.cpp:21-23, 146-149).
 *  - Device memory is owned by the handle; host buffers are owned by the
 *    caller.  A handle is used by one host thread at a time.
 *  - Units: time in microseconds (reference: uint32 µs, Network.h:67) or in
 *    grid steps; potentials and weights in the caller's unit (the reference
 *    uses volts, lif.cl:3-6; the benchmark configurations use mV).
 */
#ifndef NAER_CAPI_H
#define NAER_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define NAER_API __attribute__((visibility("default")))
#else
#define NAER_API
#endif

/* ---- status codes ---------------------------------------------------- */
#define NAER_OK 0
#define NAER_E_INVALID (-1)     /* bad argument or specification */
#define NAER_E_OOM (-2)         /* device or host allocation failed */
#define NAER_E_OVERFLOW (-3)    /* a fixed-capacity buffer would overflow */
#define NAER_E_TIMEOUT (-4)     /* a bounded device wait gave up */
#define NAER_E_CUDA (-5)        /* CUDA runtime error */
#define NAER_E_STATE (-6)       /* call not valid in the handle's state */
#define NAER_E_UNSUPPORTED (-7) /* feature not available in this build */

/* ---- enumerations ---------------------------------------------------- */
/* Neuron kinds of the reference (NeuronType enum use: Network.h:81-119,
 * main.cpp:18-20): plastic LIF, static LIF, Poisson input. */
#define NAER_NEURON_STDP 0u
#define NAER_NEURON_NOP 1u
#define NAER_NEURON_POISSON 2u

/* Time discretisation.  GRID: fixed step dt_us with per-synapse delays and
 * a delay ring buffer.  EVENT: the reference's window semantics
 * (Network.cpp:122-256): exact per-event LIF decay in µs inside windows of
 * dt_us and one axonal delay of dt_us. */
#define NAER_MODE_GRID 0u
#define NAER_MODE_EVENT 1u

/* Spike aggregation into the ring buffer.  ATOMIC: float reductions, order
 * not fixed.  DETERMINISTIC: per step, events sorted by ring cell and summed
 * in ascending (source, synapse) order; bit-reproducible. */
#define NAER_AGG_ATOMIC 0u
#define NAER_AGG_DETERMINISTIC 1u
/* Exact-sum aggregation (no counterpart in the reference): every delivered
 * weight is rounded to the nearest multiple of 2^-S and the ring holds
 * int32 sums, which no summation order changes, so runs are bit-identical
 * at the atomic mode's speed.  S (at most 30) is chosen per network from
 * its largest possible ring-cell sum (in-degree x max |w|, w_max for STDP,
 * x 10 with POISSON sources); a network whose bound leaves no S >= 0 gets
 * NAER_E_OVERFLOW at compile.  Inputs differ from the float sums by at most
 * 2^-(S+1) per event. */
#define NAER_AGG_EXACT 2u

/* Connection rules.  REF_BERNOULLI is the reference's pairwise Philox test
 * (include/naer/kernels/network.cl:14-107); the fixed-degree rules draw
 * targets (out-degree) or sources (in-degree) uniformly with Philox. */
#define NAER_CONN_REF_BERNOULLI 0u
#define NAER_CONN_FIXED_INDEGREE 1u
#define NAER_CONN_FIXED_OUTDEGREE 2u
#define NAER_CONN_EXPLICIT 3u  /* synapses given by naer_net_add_connection_csr */

/* ---- parameter blocks ------------------------------------------------- */
typedef struct naer_net_params {
    uint32_t mode;            /* NAER_MODE_* */
    uint32_t aggregation;     /* NAER_AGG_* */
    uint32_t dt_us;           /* grid step (default 100) / event window (1500) */
    uint32_t record_spikes;   /* 1: append every spike to the device raster */
    uint64_t raster_capacity; /* raster records kept on the device */
    uint32_t poisson_seed;    /* Philox key word 1 of POISSON populations;
                                 the reference passes 0x15ac7ebd every step
                                 (Network.cpp:124) */
    uint32_t stdp_enabled;    /* pair-based STDP on STDP->STDP synapses */
    float tau_plus_ms;        /* pre trace time constant */
    float tau_minus_ms;       /* post trace time constant */
    float a_plus;             /* LTP amplitude, in units of w_max */
    float a_minus;            /* LTD amplitude, in units of w_max */
    float w_max;              /* weights clipped to [0, w_max] */
    uint32_t stdp_history;    /* post spikes remembered per neuron for lazy LTP */
} naer_net_params;

typedef struct naer_pop_params {
    float tau_m_ms;       /* membrane time constant (reference T_MEM, lif.cl:3) */
    float v_th;           /* spike iff V > v_th (lif.cl:28) */
    float v_reset;        /* V after a spike (lif.cl:32) */
    float t_ref_ms;       /* refractory time (lif.cl:4,31) */
    float v_init;         /* V at step 0 */
    float rate_hz;        /* POISSON populations: rate (input_neuron_group.cl:4) */
    float drive_rate_hz;  /* LIF populations: per-neuron Poisson drive, 0 = off */
    float drive_weight;   /* LIF populations: weight of one drive event */
    uint32_t drive_seed;  /* Philox key word 1 of the drive */
    uint32_t pad_;
} naer_pop_params;

typedef struct naer_conn_spec {
    uint32_t rule;        /* NAER_CONN_* */
    uint32_t degree;      /* K of the fixed-degree rules */
    double probability;   /* REF_BERNOULLI connection probability */
    float weight;         /* weight; 0 => uniform in [wmin, wmax) (network.cl:97-100) */
    float wmin;
    float wmax;
    uint32_t delay_min;   /* grid steps, >= 1 */
    uint32_t delay_max;   /* grid steps, >= delay_min */
    uint32_t pad_;
    uint64_t seed;        /* REF_BERNOULLI uses the low 32 bits, as the
                             reference does (Network.cpp:447,532) */
} naer_conn_spec;

typedef struct naer_stats {
    uint64_t step;              /* grid steps (or event windows) simulated */
    uint64_t events;            /* synaptic events delivered */
    uint64_t spikes;            /* spikes recorded in the raster */
    uint64_t raster_dropped;    /* spikes not recorded: raster full */
    uint64_t stdp_hist_overflow;/* lazy-LTP lookups that lost pairs: a post spike that had left the
                                   post-spike history still fell after the source's last spike */
    uint64_t synapses;          /* synapses (unpadded) */
    uint64_t device_bytes;      /* device memory held by the handle */
    uint32_t neurons;
    uint32_t ring_slots;
    uint64_t kernel_launches;   /* launches of the library's own step kernels */
} naer_stats;

typedef struct naer_net naer_net;

/* ---- library ---------------------------------------------------------- */
NAER_API int naer_last_error(char* buf, size_t len);
NAER_API int naer_device_count(int* count);
NAER_API int naer_net_params_default(naer_net_params* p);
NAER_API int naer_pop_params_default(uint32_t neuron_type, naer_pop_params* p);

/* ---- one network: the plain form --------------------------------------- */

/* Network::Network (Network.cpp:14-47): binds a device, creates the queue.
 * device = -1 makes a description-only handle (no device resources): it
 * takes populations and connections but cannot be compiled; it is the
 * input of naer_batch_add and naer_server_submit. */
NAER_API int naer_net_create(int device, const naer_net_params* params, naer_net** out);

/* Network::~Network (Network.cpp:49-75; the reference releases nothing). */
NAER_API int naer_net_destroy(naer_net* net);

/* Network::addPopulation (Network.cpp:77-83).  *type_address receives the
 * address within the neuron type, as the reference's Population::baseAddress
 * holds before compile(); naer_net_population_base gives the final address. */
NAER_API int naer_net_add_population(naer_net* net, uint32_t neuron_type, uint32_t size,
                                     const naer_pop_params* params, uint32_t* pop_id,
                                     uint32_t* type_address);

/* Network::addConnection (both overloads, Network.cpp:85-105). */
NAER_API int naer_net_add_connection(naer_net* net, uint32_t src_pop, uint32_t dst_pop,
                                     const naer_conn_spec* spec);

/* Connectivity given explicitly (no counterpart in the reference, whose
 * only generator is include/naer/kernels/network.cl:14-107): the synapses
 * from population src_pop to population dst_pop as a CSR over the source
 * population.  row_ptr has src_size + 1 entries (row_ptr[0] = 0, rows in
 * source order); per synapse: the target's index within the destination
 * population, its weight and its delay in grid steps (1..254).  The arrays
 * are copied; each row keeps the given synapse order (then, like every
 * row, a stable split puts its delay-1 synapses first).  Explicit and
 * rule-generated connections can be mixed; rows concatenate in the order
 * the connections were added. */
NAER_API int naer_net_add_connection_csr(naer_net* net, uint32_t src_pop, uint32_t dst_pop, const uint64_t* row_ptr,
                                         const uint32_t* targets, const float* weights, const uint8_t* delays);

/* Network::compile (Network.cpp:267-308): address layout, device buffers,
 * connectivity generated on the device. */
NAER_API int naer_net_compile(naer_net* net);

/* Population::baseAddress after compile() (Network.cpp:283-285). */
NAER_API int naer_net_population_base(naer_net* net, uint32_t pop_id, uint32_t* base_address);

/* Network::step (Network.cpp:122-256), asynchronous: enqueues nsteps grid
 * steps (GRID) or nsteps windows (EVENT) and returns. */
NAER_API int naer_net_step(naer_net* net, uint64_t nsteps);

/* No counterpart in the reference.  naer_net_step for a network compiled
 * with NAER_AGG_DETERMINISTIC (same kernels, same results), except that the
 * aggregation's scratch (8 bytes per padded synapse and 4 per ring cell)
 * comes from one fixed 32 MiB device array inside the library instead of
 * buffers the network allocates on its first deterministic step, so the
 * call never allocates or frees device memory.  It serves hosts that own
 * every byte of device memory through their own pool and must not see a
 * library call cudaMalloc (which also stalls the whole device) in the
 * middle of a run.
 * Limit: that scratch must fit in the array; a larger network gets
 * NAER_E_OVERFLOW from the call, before any state changes.  NAER_E_STATE
 * for an atomic-aggregation network.
 * The first call on a device looks up the array's device address; make it
 * before any stream capture begins.  Every call clears the parts of the
 * array that must start empty.
 * One array exists per device, shared by all networks on it: calls whose
 * GPU work overlaps (networks on different streams or host threads) race on
 * it and must be serialized by the caller. */
NAER_API int naer_net_step_noalloc(naer_net* net, uint64_t nsteps);

/* Network::finish (Network.cpp:258-265): blocks until the queue drains and
 * reports any device-side error. */
NAER_API int naer_net_finish(naer_net* net);

/* Network::getTime (Network.cpp:107-110), in µs, 64-bit. */
NAER_API int naer_net_get_time_us(naer_net* net, uint64_t* time_us);
/* Network::getSynapses / getNeurons (Network.cpp:112-120). */
NAER_API int naer_net_get_synapses(naer_net* net, uint64_t* synapses);
NAER_API int naer_net_get_neurons(naer_net* net, uint32_t* neurons);

/* Counters; blocks like finish(). */
NAER_API int naer_net_get_stats(naer_net* net, naer_stats* stats);

/* Raster readback (the reference never reads spikes back).  Copies records
 * [first, first + capacity) of the raster: steps[i] is the grid step (EVENT:
 * the spike time in µs), ids[i] the reference address.  Records are grouped
 * by step in increasing step order; within a step the order is arbitrary in
 * ATOMIC mode and ascending address in DETERMINISTIC mode.  Blocks. */
NAER_API int naer_net_read_spikes(naer_net* net, uint64_t first, uint64_t capacity,
                                  uint32_t* steps, uint32_t* ids, uint64_t* count);
NAER_API int naer_net_clear_spikes(naer_net* net);

/* Raw raster records [first, first + capacity) copied straight into a
 * caller buffer of 2 * capacity uint32 ({step, id} pairs, step order, no
 * ordering within a step): the zero-copy-overhead readback for streaming.
 * Blocks. */
NAER_API int naer_net_read_raster(naer_net* net, uint64_t first, uint64_t capacity, uint32_t* records,
                                  uint64_t* count);

/* The CUDA stream (cudaStream_t) every launch of this handle is issued on,
 * for callers that order their own work or record events against it. */
NAER_API int naer_net_stream(naer_net* net, void** stream);

/* Neuron state in address order (n = getNeurons()).  POISSON neurons report
 * v = 0, refractory = 0. Blocks. */
NAER_API int naer_net_read_state(naer_net* net, float* v, uint32_t* refractory);
NAER_API int naer_net_write_state(naer_net* net, const float* v, const uint32_t* refractory);

/* Connectivity in address order, unpadded: row_ptr[n+1], tgt/w/delay[S].
 * Synapses of a row appear in the order the scatter visits them. Blocks. */
NAER_API int naer_net_read_csr(naer_net* net, uint64_t* row_ptr, uint32_t* tgt, float* w,
                               uint8_t* delay);

/* Per-kernel device time accumulated while profiling is on (cudaEvent pairs
 * around each launch; the reference's PROFILING counters, Network.h:11,50-55).
 * names: "lif", "scatter". */
NAER_API int naer_net_set_profiling(naer_net* net, int enable);
NAER_API int naer_net_get_profile(naer_net* net, double* lif_ms, double* scatter_ms,
                                  uint64_t* launches);
/* Finer split of the same device time (ms): [0] LIF, [1] wait for all LIF
 * blocks, [2] scatter, [3] reserved (0), [4] wait for all scatter blocks.
 * Measured by the first block of the step kernel. */
NAER_API int naer_net_get_phases(naer_net* net, double* phase_ms5);
/* CUDA-event durations (ms) of the launches issued while profiling: the
 * Poisson-draw kernels and the persistent step kernels (and their count). */
NAER_API int naer_net_get_launch_times(naer_net* net, double* drive_ms, double* step_kernel_ms,
                                       uint64_t* step_kernel_launches);

/* Checkpoint and restore (no counterpart in the reference, whose state
 * lives only in its OpenCL buffers, src/Network.cpp:379-569).  A checkpoint
 * is the network's whole simulation state between steps: the step counter,
 * the event counter, membrane potentials, refractory counters, the delay
 * ring (inputs already on their way), and with plasticity the weights and
 * the pre/post traces and post-spike history.  Connectivity is not stored:
 * it is regenerated bit for bit from the same description at compile, and
 * the Poisson input follows from the step counter.
 * naer_net_checkpoint blocks until the queued steps end and writes
 * checkpoint_size bytes into buf.  naer_net_restore loads a checkpoint into
 * a compiled network built from the same description (NAER_E_INVALID when
 * its layout differs); stepping continues from the saved step, and a
 * deterministic network then produces the raster and state of the
 * uninterrupted run bit for bit.  The raster restarts empty. */
NAER_API int naer_net_checkpoint_size(naer_net* net, uint64_t* bytes);
NAER_API int naer_net_checkpoint(naer_net* net, void* buf, uint64_t capacity);
NAER_API int naer_net_restore(naer_net* net, const void* buf, uint64_t size);

/* Bounded device waits (no counterpart in the reference, whose OpenCL
 * queue has none).  Every grid barrier of the step kernel gives up after
 * limit_us microseconds (default 2 s), records NAER_E_TIMEOUT on the device
 * and ends the launch; naer_net_finish then returns NAER_E_TIMEOUT and the
 * network refuses further steps (NAER_E_STATE): its state is undefined, the
 * handle can only be destroyed.  0 restores the default. */
NAER_API int naer_net_set_wait_limit(naer_net* net, uint64_t limit_us);

/* Fault injection for tests of the bounded wait (no counterpart in the
 * reference).  A non-zero skew is added to every grid-barrier target of the
 * following launches, so no barrier can complete and each wait runs out
 * after the limit above; the kernel then returns normally with the error
 * recorded.  Nothing else changes on the device.  0 = normal operation. */
NAER_API int naer_test_set_barrier_skew(naer_net* net, uint64_t skew);

/* Fault injection for tests (no counterpart in the reference): the device
 * allocation `after` allocations from now (0 = the next one, in any handle
 * of this process) fails as if the device were out of memory, once; -1
 * turns it off.  The call that hits it returns NAER_E_OOM and releases
 * whatever it had allocated. */
NAER_API int naer_test_fail_allocation(int64_t after);

/* The bounds-checked build (libnaer_b200_checked.so, compiled with
 * NAER_CHECKED; no counterpart in the reference).  Its step kernels check
 * every global access at a computed index against the buffer it falls in
 * and skip it when outside; the first such index is recorded.  *checked =
 * 1 in that build, 0 in the normal one. */
NAER_API int naer_build_checked(int* checked);
/* First out-of-bounds access the checked build recorded for the network's
 * launches (*code 0 = none; 1 synapse arrays, 2 ring cell, 3 source of a
 * queued spike, 5 neuron state of a LIF chunk, 6 Poisson-count slot,
 * 8 deterministic event list) and its index.  Always 0 in the normal
 * build.  Blocks like finish(). */
NAER_API int naer_net_check_report(naer_net* net, uint32_t* code, uint64_t* index);

/* ---- device probe ------------------------------------------------------
 * No counterpart in the reference.  Measures, on `device`, the ceilings the
 * step kernel is measured against: random-address fp32 reductions
 * (red.global.add.f32, the atomic mode's ring accumulation) into
 * ring_cells and small_cells cells, random 4-byte stores into ring_cells
 * cells, a streaming read of 4 GiB with evict-first 128-bit loads, and one
 * grid barrier of the step kernel's kind at one and two blocks per SM.
 * Allocates and frees its own buffers (4 GiB plus 4 B per ring cell). */
typedef struct naer_device_probe {
    uint64_t ring_cells, small_cells;
    double red_ring_per_s;    /* reductions per second into ring_cells cells */
    double red_small_per_s;   /* reductions per second into small_cells cells */
    double store_ring_per_s;  /* random stores per second into ring_cells cells */
    double stream_gbs;        /* streaming read, GB/s */
    double barrier_us_1;      /* one grid barrier, 1 block per SM, microseconds */
    double barrier_us_2;      /* one grid barrier, 2 blocks per SM */
    uint32_t grid;            /* SMs */
    uint32_t pad_;
} naer_device_probe;

NAER_API int naer_probe_device(int device, uint64_t ring_cells, uint64_t small_cells, naer_device_probe* out);

/* The Poisson generator's inter-event interval in µs, (uint)(log(1 - x) /
 * -(rate * 1e-6)) with x = z / 0xFFFFFFFF (random.cl:26-30 and the cast of
 * input_neuron_group.cl:29,37), computed on `device` exactly as the drive
 * kernels do, for z = z_first + i * z_step (mod 2^32), i < count.  For
 * comparing the device's logarithm with a host's at the truncation
 * boundary (no counterpart in the reference). */
NAER_API int naer_probe_intervals(int device, double rate_hz, uint32_t z_first, uint32_t z_step, uint64_t count,
                                  uint32_t* out);

/* ---- batched form ------------------------------------------------------
 * No counterpart in the reference (one Network per device queue there).
 * Many independent networks of any sizes are packed, with offsets, into one
 * engine: one set of persistent step launches advances all of them.  Each
 * member keeps its own parameters, seeds and STDP switch; all start at step
 * 0.  Deterministic aggregation gives every member the raster it gets
 * alone, bit for bit. */
typedef struct naer_batch naer_batch;

/* Launch geometry of the step loop (results do not depend on it). */
typedef struct naer_tuning {
    uint32_t blocks_per_sm;   /* resident step-kernel blocks per SM, 0 = most that fit */
    uint32_t launch_steps;    /* grid steps per persistent launch, 1..64 */
    uint32_t scatter_split;   /* warps per spike, 0 = enough to cover the longest row */
    uint32_t graph_launches;  /* persistent launches per CUDA-graph replay, 0 = no graph */
    double best_us_per_step;  /* autotune: time of the chosen geometry */
    double default_us_per_step; /* autotune: time of the default geometry */
    uint32_t trials;          /* autotune: geometries timed */
    uint32_t scatter_piece;   /* synapses per warp iteration: 128, 256, 0 = 128 for plastic networks else 256 */
    uint32_t neuron_state;    /* NAER_STATE_*: where the step kernel keeps membrane potentials and
                                 refractory counters during a launch */
    uint32_t step_kernel;     /* NAER_KERNEL_*: which persistent step kernel runs */
    uint32_t bins;            /* SPLIT kernel: entries (a power of two, 64..8192) of the per-block
                                 shared-memory table that folds ring reductions to the same cell
                                 before they reach L2; 0 = every event reduces in L2 directly */
    uint32_t pad_;
} naer_tuning;

/* naer_tuning.step_kernel.  SPLIT: one contiguous spike list per step,
 * delay-1 synapses delivered before the next LIF and the rest of each row
 * while the grid waits at its barriers.  TWO_BARRIER: per-block spike
 * regions, the whole scatter between two grid barriers.  Same results; both
 * serve atomic and exact-sum aggregation (deterministic aggregation has a
 * kernel of its own). */
#define NAER_KERNEL_SPLIT 0u
#define NAER_KERNEL_TWO_BARRIER 1u

/* naer_tuning.neuron_state.  AUTO: shared memory when the installed chunks
 * fit it, else global memory.  SHARED: shared memory or NAER_E_INVALID.
 * GLOBAL: global memory (the path large served sets fall back to). */
#define NAER_STATE_AUTO 0u
#define NAER_STATE_SHARED 1u
#define NAER_STATE_GLOBAL 2u

NAER_API int naer_batch_create(int device, uint32_t aggregation, uint64_t raster_capacity,
                               naer_batch** out);
NAER_API int naer_batch_destroy(naer_batch* batch);
/* Copies a description-only network (naer_net_create(-1, ...)) into the
 * batch; *member is its index.  Validates it. */
NAER_API int naer_batch_add(naer_batch* batch, const naer_net* description, uint32_t* member);
/* Builds every member on the device (connectivity generated there). */
NAER_API int naer_batch_compile(naer_batch* batch);
/* Asynchronous: nsteps grid steps of every member.  In atomic mode the
 * launch sequence is recorded once as a CUDA graph and replayed. */
NAER_API int naer_batch_step(naer_batch* batch, uint64_t nsteps);
NAER_API int naer_batch_finish(naer_batch* batch);
/* Times candidate geometries on the batch itself, trial_steps grid steps
 * each (they advance the simulation), and keeps the fastest. */
NAER_API int naer_batch_autotune(naer_batch* batch, uint32_t trial_steps, naer_tuning* out);
NAER_API int naer_batch_set_tuning(naer_batch* batch, const naer_tuning* tuning);
NAER_API int naer_batch_get_tuning(naer_batch* batch, naer_tuning* tuning);
/* Raster records [first, first + capacity): member index, step, reference
 * address within the member.  Ordered by step, then member, then address. */
NAER_API int naer_batch_read_spikes(naer_batch* batch, uint64_t first, uint64_t capacity,
                                    uint32_t* member, uint32_t* steps, uint32_t* ids, uint64_t* count);
NAER_API int naer_batch_clear_spikes(naer_batch* batch);
/* Whole-batch counters (synapses and neurons summed over members). */
NAER_API int naer_batch_get_stats(naer_batch* batch, naer_stats* st);
/* The step kernel's phase split for the whole batch, as naer_net_get_phases
 * (ms, accumulated since compile, measured by the kernel's first block). */
NAER_API int naer_batch_get_phases(naer_batch* batch, double* phase_ms5);
NAER_API int naer_batch_read_state(naer_batch* batch, uint32_t member, float* v, uint32_t* refractory);
NAER_API int naer_batch_stream(naer_batch* batch, void** stream);

/* The same launch-geometry tuning for one network (no counterpart in the
 * reference): autotune times the candidates on the network itself, each
 * for trial_steps grid steps, which advance its simulation. */
NAER_API int naer_net_autotune(naer_net* net, uint32_t trial_steps, naer_tuning* out);
NAER_API int naer_net_set_tuning(naer_net* net, const naer_tuning* tuning);
NAER_API int naer_net_get_tuning(naer_net* net, naer_tuning* tuning);

/* ---- served form -------------------------------------------------------
 * No counterpart in the reference.  A request loop on its own host thread:
 * jobs (a description, a duration in grid steps) are admitted first come,
 * first served while the device bytes of the admitted networks stay under
 * the budget, built on the device and stepped together with the jobs
 * already running (continuous batching: admission and retirement happen
 * every chunk_steps grid steps, state stays on the device).  Each job's
 * raster is collected per chunk and returned when the job ends.  All
 * functions are thread-safe.
 *
 * Trace: with the environment variable NAER_SERVER_TRACE set to a file
 * name when the server is created, the stepper writes one CSV row per chunk
 * (running jobs, device ms, host ms waiting / installing / handing rasters
 * over, records, queue length, bytes in use) to that file and the builder
 * one row per build to <name>.build. */
typedef struct naer_server naer_server;

typedef struct naer_server_params {
    uint64_t budget_bytes;     /* device bytes of admitted networks, at most */
    uint64_t raster_capacity;  /* spike records per chunk (excess is dropped and counted) */
    uint32_t chunk_steps;      /* grid steps between admission points, at most */
    uint32_t aggregation;      /* NAER_AGG_* for every job */
    uint32_t max_jobs;         /* jobs stepped together, at most */
    uint32_t blocks_per_sm;    /* step-kernel blocks per SM (0 = most that fit) */
    double chunk_ms;           /* target device time of a chunk: fewer steps when many jobs run */
    uint32_t launch_steps;     /* grid steps per persistent step launch, 1..64 (0 = default);
                                  builds run between launches, so short launches let jobs in sooner
                                  and long ones pay less launch overhead per step */
    uint32_t step_kernel;      /* atomic and exact-sum aggregation: NAER_KERNEL_TWO_BARRIER (default; the
                                  served job mix completes more jobs per second with it) or NAER_KERNEL_SPLIT */
} naer_server_params;

#define NAER_JOB_QUEUED 0u
#define NAER_JOB_RUNNING 1u
#define NAER_JOB_DONE 2u
#define NAER_JOB_FAILED 3u
#define NAER_JOB_CANCELLED 4u

typedef struct naer_job_info {
    uint32_t state;            /* NAER_JOB_* */
    uint32_t preemptions;      /* times the job was pre-empted and resumed */
    uint64_t duration;         /* grid steps asked for */
    uint64_t steps_done;
    uint64_t spikes;           /* raster records of the job (when done) */
    uint64_t device_bytes;     /* device memory of its network while running */
    double submit_s, admit_s, done_s;  /* seconds since the server started */
} naer_job_info;

typedef struct naer_server_stats {
    uint64_t submitted, done, failed, running, queued;
    uint64_t chunks, engine_steps, peak_bytes, bytes_in_use, raster_dropped;
    double p50_ms, p99_ms, mean_ms;  /* job latency: submit to raster delivered */
    double sims_per_s;               /* jobs done / (last done - first submit) */
    double build_s;                  /* builder thread: device builds */
    double install_s, step_s, drain_s;  /* stepper thread: tables, chunks, rasters */
} naer_server_stats;

NAER_API int naer_server_params_default(naer_server_params* p);
NAER_API int naer_server_create(int device, const naer_server_params* params, naer_server** out);
/* Stops the loop after the current chunk; unfinished jobs are abandoned. */
NAER_API int naer_server_destroy(naer_server* server);
/* Copies a description-only network; NAER_E_OVERFLOW if its estimated
 * device bytes exceed the whole budget. */
NAER_API int naer_server_submit(naer_server* server, const naer_net* description,
                                uint64_t duration_steps, uint64_t* job);
NAER_API int naer_server_job_info(naer_server* server, uint64_t job, naer_job_info* info);
/* Error text of a failed job. */
NAER_API int naer_server_job_error(naer_server* server, uint64_t job, char* buf, size_t len);
/* *finished = 1 when the job (all jobs) ended within the timeout. */
NAER_API int naer_server_wait(naer_server* server, uint64_t job, double timeout_s, int* finished);
NAER_API int naer_server_drain(naer_server* server, double timeout_s, int* finished);
/* Raster of a finished job, ordered by (step, address); steps count from
 * the job's own step 0. */
NAER_API int naer_server_read_spikes(naer_server* server, uint64_t job, uint64_t first,
                                     uint64_t capacity, uint32_t* steps, uint32_t* ids,
                                     uint64_t* count);
/* Forgets a finished job and its raster. */
NAER_API int naer_server_release(naer_server* server, uint64_t job);
/* Pre-emption: takes a running job off the device at the next chunk
 * boundary (NAER_E_STATE if it is not running).  Its whole simulation state
 * (as naer_net_checkpoint) moves to host memory, its device memory is freed
 * and it queues again; when re-admitted it is rebuilt, restored and
 * continues from the step it reached, so a deterministic job's raster
 * equals its uninterrupted run. */
NAER_API int naer_server_preempt(naer_server* server, uint64_t job);
/* Cancels a job that has not ended: a queued or built job at once, a
 * running job at the next chunk boundary.  It ends in NAER_JOB_CANCELLED
 * and its raster is discarded.  NAER_E_STATE if it already ended. */
NAER_API int naer_server_cancel(naer_server* server, uint64_t job);
NAER_API int naer_server_get_stats(naer_server* server, naer_server_stats* st);

#ifdef __cplusplus
}
#endif

#endif /* NAER_CAPI_H */
