// Simulation-step kernels (grid mode) and their device helpers.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "check.cuh"
#include "engine_types.cuh"
#include "philox.cuh"

namespace naer {

// ---------------------------------------------------------------------------
// Poisson window generator.  Restates simulate_poisson_neurons
// (include/naer/kernels/input_neuron_group.cl:17-39) for one element:
//   time = t0 + (uint)exprnd(rate, seed, t0 * N + idx)
//   repeat 10 times: if time < t1 { emit; time += (uint)exprnd(rate, seed, time * N + idx) }
// with key word 0 = the reference work-item id of idx (random.cl:8).
// Returns the number of events in [t0, t1).
static __device__ __forceinline__ uint32_t poisson_exact(double rate, uint32_t seed, uint32_t n_gen,
                                               uint32_t idx, uint32_t key0, uint32_t z0,
                                               uint32_t t0, uint32_t t1) {
    uint32_t time = t0 + ref_exp_interval_us(z0, rate);
    uint32_t count = 0;
    for (int m = 0; m < 10; ++m) {
        if (!(time < t1)) break;
        ++count;
        const uint32_t z = philox_ref_z(time * n_gen + idx, key0, seed);
        time += ref_exp_interval_us(z, rate);
    }
    return count;
}

// First draw of the window (word z of Philox at counter t0 * N + idx).
__device__ __forceinline__ uint32_t poisson_z0(const PopDev& p, uint32_t idx, uint32_t t0) {
    return philox_ref_z(t0 * p.rng_n + idx, ref_global_id(idx, kPoissonCapacity, kPoissonWorkgroup), p.rng_seed);
}

// True when the first draw alone proves the window empty.
__device__ __forceinline__ bool poisson_quiet(const PopDev& p, uint32_t z0, uint32_t t0) {
    return z0 >= p.z_hi && z0 != 0xFFFFFFFFu && t0 <= p.t0_limit;
}

__device__ __forceinline__ uint32_t poisson_count(const PopDev& p, uint32_t idx, uint32_t t0,
                                                  uint32_t t1) {
    const uint32_t key0 = ref_global_id(idx, kPoissonCapacity, kPoissonWorkgroup);
    const uint32_t z0 = philox_ref_z(t0 * p.rng_n + idx, key0, p.rng_seed);
    // Fast path: the first interval already reaches past the window.  z_hi is
    // chosen on the host with a margin so that this agrees with the exact
    // path for every z in [z_hi, 0xFFFFFFFE].
    if (z0 >= p.z_hi && z0 != 0xFFFFFFFFu && t0 <= p.t0_limit) return 0;
    return poisson_exact(p.rate_hz, p.rng_seed, p.rng_n, idx, key0, z0, t0, t1);
}

// One grid step of a neuron that is not refractory: exponential decay by
// the fp64 propagator, the ring input and m Poisson drive events of weight
// dw, all in double arithmetic (m * dw is exact) and rounded to fp32 once.
// One rounding per step keeps the fp32 state within 1e-5 relative of an
// fp64 integration even when large drive weights pass through the sum.
__device__ __forceinline__ float lif_update(float v, double prop, float I, uint32_t m, float dw) {
    double x = __dmul_rn((double)v, prop);
    x = __dadd_rn(x, (double)I);
    if (m) x = __dadd_rn(x, __dmul_rn((double)m, (double)dw));
    return __double2float_rn(x);
}

__device__ __forceinline__ float decay_lookup(const float* table, uint32_t len, int32_t k) {
    return (k >= 0 && (uint32_t)k < len) ? __ldg(table + k) : 0.0f;
}

// Register copy of a net's plasticity fields (the kernels copy descriptor
// fields once per work item so that stores and atomics cannot force reloads).
struct StdpView {
    const int32_t* __restrict__ post;
    const float* __restrict__ e_plus;
    const float* __restrict__ e_minus;
    uint32_t hist_len, post_stride, e_len;
    float a_plus, a_minus, w_max;
};

__device__ __forceinline__ StdpView stdp_view(const NetDev& n) {
    StdpView v;
    v.post = n.post;
    v.e_plus = n.e_plus;
    v.e_minus = n.e_minus;
    v.hist_len = n.hist_len;
    v.post_stride = n.post_stride;
    v.e_len = n.e_len;
    v.a_plus = n.a_plus;
    v.a_minus = n.a_minus;
    v.w_max = n.w_max;
    return v;
}

// A packed post row (stride words, a multiple of 4) into registers with
// independent int4 loads at L2 (rows are rewritten by other blocks' LIF);
// words past the stride read as -1.
__device__ __forceinline__ void load_post_row(const int32_t* row, uint32_t stride, int32_t (&r)[kPostWordsMax]) {
#pragma unroll
    for (uint32_t v = 0; v < kPostWordsMax / 4; ++v) {
        int4 x = make_int4(-1, -1, -1, -1);
        if (v * 4u < stride) x = __ldcg(reinterpret_cast<const int4*>(row) + v);
        r[4 * v] = x.x;
        r[4 * v + 1] = x.y;
        r[4 * v + 2] = x.z;
        r[4 * v + 3] = x.w;
    }
}

// Pair-based STDP for one plastic synapse at the pre spike of step t
// (emission time).  Lazy LTP replays the post spikes of `tgt` in
// (pre_last, t], oldest first, with the pre trace decayed from pre_last;
// LTD uses the post trace at t.  Weights are clipped to [0, w_max] after
// every update, so the sequence equals the online rule's.  Every operation
// is an explicitly rounded fp32 op so the oracle can repeat it bit for bit.
// The target's whole post row is loaded at once and every decay-table
// lookup is issued before the sequential weight updates use them.
// Plays the role of update_synapse (include/naer/kernels/stdp.cl:8-30).
// stdp_apply takes the post row already in registers (stdp_update loads it).
__device__ __forceinline__ float stdp_apply(const StdpView& n, float w, const int32_t (&r)[kPostWordsMax], int32_t t,
                                            int32_t pre_last, float pre_x, uint32_t& overflow) {
    if (pre_last >= 0) {
        // history entries newer than pre_last form a prefix (newest first)
        uint32_t c = 0;
        bool run = true;
#pragma unroll
        for (uint32_t k = 0; k < kMaxStdpHistory; ++k) {
            run = run && k < n.hist_len && r[2 + k] > pre_last;
            c += run ? 1u : 0u;
        }
        // a pair is lost only if a post spike that left the history (the
        // newest one that did is kept in word 0) still falls after pre_last
        if (c == n.hist_len && r[0] > pre_last) ++overflow;
        float e[kMaxStdpHistory];
#pragma unroll
        for (uint32_t k = 0; k < kMaxStdpHistory; ++k)
            e[k] = k < c ? decay_lookup(n.e_plus, n.e_len, r[2 + k] - pre_last) : 0.0f;
#pragma unroll
        for (int k = (int)kMaxStdpHistory - 1; k >= 0; --k) {
            if ((uint32_t)k < c) {
                const float x = __fmul_rn(pre_x, e[k]);
                w = fminf(__fadd_rn(w, __fmul_rn(n.a_plus, x)), n.w_max);
            }
        }
    }
    const int32_t lp = r[2];  // the newest history entry is the last post spike
    if (lp >= 0) {
        const float y = __fmul_rn(__int_as_float(r[1]), decay_lookup(n.e_minus, n.e_len, t - lp));
        w = fmaxf(__fsub_rn(w, __fmul_rn(n.a_minus, y)), 0.0f);
    }
    return w;
}

__device__ __forceinline__ float stdp_update(const StdpView& n, float w, uint32_t tgt, int32_t t,
                                             int32_t pre_last, float pre_x, uint32_t& overflow) {
    int32_t r[kPostWordsMax];
    load_post_row(n.post + (size_t)tgt * n.post_stride, n.post_stride, r);
    return stdp_apply(n, w, r, t, pre_last, pre_x, overflow);
}

// Plasticity bookkeeping of plastic neuron i spiking at local step t: post
// trace and post history (row rewritten whole), pre trace.  aux0/aux1
// receive the pre state before this spike (carried by the queue record).
__device__ __forceinline__ void stdp_post_spike(const NetDev* np, uint32_t i, int32_t t, int32_t& aux0, float& aux1) {
    const uint32_t stride = np->post_stride, hist_len = np->hist_len, e_len = np->e_len;
    const float* e_plus = np->e_plus;
    const float* e_minus = np->e_minus;
    int32_t* row = np->post + (size_t)i * stride;
    int2* pre = np->pre + i;
    int32_t r[kPostWordsMax];
    load_post_row(row, stride, r);
    const int2 pq = __ldcg(pre);
    const int32_t lp = r[2];
    const float y = lp >= 0 ? __fmul_rn(__int_as_float(r[1]), decay_lookup(e_minus, e_len, t - lp)) : 0.0f;
    int32_t evicted = r[0];
#pragma unroll
    for (uint32_t q = 0; q < kMaxStdpHistory; ++q)
        if (q + 1 == hist_len && r[2 + q] >= 0) evicted = r[2 + q];  // the entry shifted out below
    r[0] = evicted;
    r[1] = __float_as_int(__fadd_rn(y, 1.0f));
#pragma unroll
    for (int q = (int)kMaxStdpHistory - 1; q > 0; --q)
        if ((uint32_t)q < hist_len) r[2 + q] = r[1 + q];
    r[2] = t;
#pragma unroll
    for (uint32_t v = 0; v < kPostWordsMax / 4; ++v)
        if (v * 4u < stride)
            __stcg(reinterpret_cast<int4*>(row) + v, make_int4(r[4 * v], r[4 * v + 1], r[4 * v + 2], r[4 * v + 3]));
    const int32_t lq = pq.x;
    const float xo = __int_as_float(pq.y);
    aux0 = lq;
    aux1 = xo;
    const float x = lq >= 0 ? __fmul_rn(xo, decay_lookup(e_plus, e_len, t - lq)) : 0.0f;
    __stcg(pre, make_int2(t, __float_as_int(__fadd_rn(x, 1.0f))));
}

__device__ __forceinline__ uint32_t ring_slot(uint32_t t_mod, uint32_t d, uint32_t slots) {
    uint32_t s = t_mod + d;
    return s >= slots ? s - slots : s;
}

// Kernels ---------------------------------------------------------------------
// Persistent step kernels (cooperative launches of up to kDriveSlots grid
// steps): k_step (atomic, one spike list per step, split scatter), k_run
// (atomic, per-block spike regions, two barriers per step), k_det_step
// (deterministic aggregation).  kSmem: neuron state in shared memory.
template <bool kSmem>
__global__ void k_run(EngineDev eng, unsigned long long s0, uint32_t nsteps);
template <bool kSmem>
__global__ void k_step(EngineDev eng, unsigned long long s0, uint32_t nsteps);
template <bool kSmem>
__global__ void k_det_step(EngineDev eng, unsigned long long s0, uint32_t nsteps);
// dynamic shared memory of k_run for a grid and a number of owned chunks per block
size_t run_smem_bytes(uint32_t grid, uint32_t own_max, bool smem_state);
// dynamic shared memory of k_step / k_det_step for a number of owned chunks
// per block and a binning table of `bins` entries (k_step only; 0 = none)
size_t step_smem_bytes(uint32_t own_max, bool smem_state, uint32_t bins = 0);
// offset of the chunk caches in that memory: 16 bytes, then the table
__host__ __device__ inline size_t step_smem_offset(uint32_t bins) {
    return 16 + ((((size_t)bins * 12) + 15) & ~(size_t)15);
}
// Poisson counts of up to kDriveSlots steps ahead
__global__ void k_drive(EngineDev eng, unsigned long long s_first, uint32_t nsteps);

}  // namespace naer
