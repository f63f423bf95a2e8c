// Grid-mode simulation step: LIF update with fused Poisson input and
// warp-ballot spike compaction, warp-per-spike CSR scatter into the delay
// ring buffer with fused pair-based STDP, and the deterministic
// (sorted segmented-reduce) aggregation kernels.
#include "sim_kernels.cuh"

namespace naer {

namespace {

__device__ __forceinline__ float4 ld_stream_f4(const float* p) {
    return __ldcs(reinterpret_cast<const float4*>(p));
}
__device__ __forceinline__ uint4 ld_stream_u4(const uint32_t* p) {
    return __ldcs(reinterpret_cast<const uint4*>(p));
}
__device__ __forceinline__ uint32_t ld_stream_u32(const uint8_t* p) {
    return __ldcs(reinterpret_cast<const unsigned int*>(p));
}

__device__ __forceinline__ float f4_get(const float4& v, int j) {
    return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w;
}
__device__ __forceinline__ uint32_t u4_get(const uint4& v, int j) {
    return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

}  // namespace

// ---------------------------------------------------------------------------
// LIF update, one work item = 1024 consecutive storage indices of one
// population, four neurons per thread (float4 membrane potential, uchar4
// refractory countdown, float4 ring slot read-and-clear).
//
// Grid-mode restatement of neuron_dynamics (include/naer/kernels/lif.cl:15-34)
// on a fixed step: V <- fp32(fp64(V) * exp(-dt/tau)); V += ring input; V +=
// drive weight once per Poisson drive event; spike iff V > v_th, then
// V = v_reset and t_ref steps of refractoriness, during which input is
// discarded.  POISSON populations run simulate_poisson_neurons
// (input_neuron_group.cl:6-45) on the step's window instead.
//
// Spikes are compacted with one ballot per neuron slot and one atomicAdd
// per warp into the step's queue (and the raster when recording).
__global__ void __launch_bounds__(kLifThreads) k_lif(EngineDev eng) {
    const unsigned long long s = eng.ctl->step;
    const uint32_t qb = (uint32_t)(s & 1ull);
    SpikeRec* __restrict__ queue = qb ? eng.queue[1] : eng.queue[0];
    unsigned int* qcount = &eng.ctl->q_count[qb];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;

    for (uint32_t c = blockIdx.x; c < eng.n_chunks; c += gridDim.x) {
        const ChunkDev ch = eng.chunks[c];
        const PopDev p = eng.pops[ch.pop];
        const NetDev& n = eng.nets[p.net];
        if (!n.active || s < n.start_step) continue;  // uniform over the block
        const uint32_t tl = (uint32_t)(s - n.start_step);
        const uint32_t t0 = tl * n.dt_us;
        const uint32_t t1 = t0 + n.dt_us;
        const uint32_t i0 = ch.first + threadIdx.x * kLifPerThread;
        const bool any = i0 < ch.end;

        bool spk[4] = {false, false, false, false};
        int32_t aux0[4] = {0, 0, 0, 0};
        float aux1[4] = {0.f, 0.f, 0.f, 0.f};

        if (p.type == kPOISSON) {
            if (any && p.rate_hz > 0.0) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const uint32_t i = i0 + j;
                    if (i < ch.end) {
                        const uint32_t m = poisson_count(p, p.rng_idx_base + (i - p.storage_base), t0, t1);
                        spk[j] = m > 0;
                        aux0[j] = (int32_t)m;
                    }
                }
            }
        } else if (any) {
            const uint32_t slot = tl % n.ring_slots;
            float4* ring4 = reinterpret_cast<float4*>(n.ring + (size_t)slot * n.n_storage) + (i0 >> 2);
            float4* v4 = reinterpret_cast<float4*>(n.v) + (i0 >> 2);
            uchar4* r4 = reinterpret_cast<uchar4*>(n.refr) + (i0 >> 2);
            const float4 I = *ring4;
            *ring4 = make_float4(0.f, 0.f, 0.f, 0.f);
            float4 V4 = *v4;
            uchar4 R4 = *r4;
            float vv[4] = {V4.x, V4.y, V4.z, V4.w};
            uint32_t rr[4] = {R4.x, R4.y, R4.z, R4.w};
            const bool plastic = (p.type == kSTDP) && n.stdp_on;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t i = i0 + j;
                if (i >= ch.end) continue;
                if (rr[j] > 0) {
                    rr[j] -= 1;
                    continue;
                }
                float v = __double2float_rn(__dmul_rn((double)vv[j], p.prop));
                v = __fadd_rn(v, f4_get(I, j));
                if (p.rate_hz > 0.0) {
                    const uint32_t m = poisson_count(p, i - p.storage_base, t0, t1);
                    for (uint32_t k = 0; k < m; ++k) v = __fadd_rn(v, p.drive_w);
                }
                if (v > p.v_th) {
                    v = p.v_reset;
                    rr[j] = p.t_ref_steps;
                    spk[j] = true;
                    if (plastic) {
                        const int32_t t = (int32_t)tl;
                        // post trace and post-spike history (newest first)
                        const int32_t lp = n.last_post[i];
                        float y = lp >= 0 ? __fmul_rn(n.y_post[i], decay_lookup(n.e_minus, n.e_len, t - lp)) : 0.0f;
                        n.y_post[i] = __fadd_rn(y, 1.0f);
                        n.last_post[i] = t;
                        int32_t* h = n.hist + (size_t)i * n.hist_len;
                        for (int k = (int)n.hist_len - 1; k > 0; --k) h[k] = h[k - 1];
                        h[0] = t;
                        // pre trace: the queue record carries the state before this spike
                        const int32_t lq = n.last_pre[i];
                        const float xo = n.x_pre[i];
                        aux0[j] = lq;
                        aux1[j] = xo;
                        float x = lq >= 0 ? __fmul_rn(xo, decay_lookup(n.e_plus, n.e_len, t - lq)) : 0.0f;
                        n.x_pre[i] = __fadd_rn(x, 1.0f);
                        n.last_pre[i] = t;
                    }
                }
                vv[j] = v;
            }
            *v4 = make_float4(vv[0], vv[1], vv[2], vv[3]);
            *r4 = make_uchar4((unsigned char)rr[0], (unsigned char)rr[1], (unsigned char)rr[2],
                              (unsigned char)rr[3]);
        }

        // warp-ballot compaction into the step queue (+ raster)
        uint32_t b[4];
        uint32_t total = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            b[j] = __ballot_sync(0xFFFFFFFFu, spk[j]);
            total += __popc(b[j]);
        }
        if (total == 0) continue;
        uint32_t qbase = 0;
        unsigned long long rbase = 0;
        if (lane == 0) {
            qbase = atomicAdd(qcount, total);
            if (eng.record) rbase = atomicAdd(&eng.ctl->raster_count, (unsigned long long)total);
        }
        qbase = __shfl_sync(0xFFFFFFFFu, qbase, 0);
        rbase = __shfl_sync(0xFFFFFFFFu, rbase, 0);
        if (eng.record && lane == 0 && rbase + total > eng.raster_cap) {
            const unsigned long long kept = rbase >= eng.raster_cap ? 0ull : eng.raster_cap - rbase;
            atomicAdd(&eng.ctl->raster_dropped, (unsigned long long)total - kept);
        }
        uint32_t run = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (spk[j]) {
                const uint32_t k = run + __popc(b[j] & lt_mask);
                const uint32_t i = i0 + j;
                SpikeRec rec;
                rec.net = p.net;
                rec.src = i;
                rec.aux0 = aux0[j];
                rec.aux1 = aux1[j];
                queue[qbase + k] = rec;
                if (eng.record && rbase + k < eng.raster_cap)
                    eng.raster[rbase + k] = make_uint2((uint32_t)s, p.id_base + (i - p.storage_base));
            }
            run += __popc(b[j]);
        }
    }
}

// ---------------------------------------------------------------------------
// Atomic-mode scatter: one warp per queued spike walks the source's CSR row
// (128-bit streaming loads of 4 targets, 4 weights and 4 delays per lane,
// kScatterUnroll slices in flight) and reduces each weight into
// ring[(t + d) mod D][target].  STDP sources update plastic synapses first
// and write the weight back.  This replaces the reference's per-group walk
// over every input spike (nop.cl:40-83, stdp.cl:66-133) and its
// histogram/scatter/offset passes (spike_aggregation.cl).
// The last block to finish advances the engine step.
__global__ void __launch_bounds__(kScatterThreads) k_scatter_atomic(EngineDev eng) {
    const unsigned long long s = eng.ctl->step;
    const uint32_t qb = (uint32_t)(s & 1ull);
    const uint32_t Q = eng.ctl->q_count[qb];
    const SpikeRec* __restrict__ queue = qb ? eng.queue[1] : eng.queue[0];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long ev = 0;
    uint32_t ovf = 0;

    for (uint32_t e = warp; e < Q; e += nwarps) {
        const SpikeRec r = queue[e];
        const NetDev& n = eng.nets[r.net];
        const uint32_t tl = (uint32_t)(s - n.start_step);
        const uint32_t tmod = tl % n.ring_slots;
        const uint32_t D = n.ring_slots;
        const uint32_t Ns = n.n_storage;
        float* __restrict__ ring = n.ring;
        const uint64_t beg = n.row_ptr[r.src];
        const uint64_t end = n.row_ptr[r.src + 1];
        const bool plastic_src = n.stdp_on && r.src < n.n_plastic;
        const float mult = (!plastic_src && r.aux0 > 1) ? (float)r.aux0 : 1.0f;

        for (uint64_t base = beg; base < end; base += 128ull * kScatterUnroll) {
            uint4 tg[kScatterUnroll];
            float4 ww[kScatterUnroll];
            uint32_t dd[kScatterUnroll];
#pragma unroll
            for (int u = 0; u < (int)kScatterUnroll; ++u) {
                const uint64_t off = base + (uint64_t)(u * 32 + lane) * 4ull;
                if (off < end) {
                    tg[u] = ld_stream_u4(n.tgt + off);
                    ww[u] = ld_stream_f4(n.w + off);
                    dd[u] = ld_stream_u32(n.dly + off);
                } else {
                    tg[u] = make_uint4(kTgtSentinel, kTgtSentinel, kTgtSentinel, kTgtSentinel);
                    ww[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                    dd[u] = 0;
                }
            }
#pragma unroll
            for (int u = 0; u < (int)kScatterUnroll; ++u) {
                const uint64_t off = base + (uint64_t)(u * 32 + lane) * 4ull;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const uint32_t tgt = u4_get(tg[u], j);
                    if (tgt == kTgtSentinel) continue;
                    float w = f4_get(ww[u], j);
                    const uint32_t d = (dd[u] >> (8 * j)) & 0xFFu;
                    if (plastic_src && tgt < n.n_plastic) {
                        w = stdp_update(n, w, tgt, (int32_t)tl, r.aux0, r.aux1, ovf);
                        n.w[off + j] = w;
                    }
                    if (mult != 1.0f) w = __fmul_rn(w, mult);
                    atomicAdd(ring + (size_t)ring_slot(tmod, d, D) * Ns + tgt, w);
                    ++ev;
                }
            }
        }
    }

    ev = warp_sum_u64(ev);
    const unsigned long long ov = warp_sum_u64((unsigned long long)ovf);
    if (lane == 0) {
        if (ev) atomicAdd(&eng.ctl->events, ev);
        if (ov) atomicAdd(&eng.ctl->stdp_hist_overflow, ov);
    }

    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int prev = atomicAdd(&eng.ctl->scatter_done, 1u);
        if (prev == gridDim.x - 1) {
            eng.ctl->scatter_done = 0;
            eng.ctl->q_count[qb ^ 1u] = 0;
            __threadfence();
            eng.ctl->step = s + 1;
        }
    }
}

// Advances the engine step when the scatter ran in deterministic mode.
__global__ void k_advance(EngineDev eng) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const unsigned long long s = eng.ctl->step;
        eng.ctl->q_count[(uint32_t)((s + 1) & 1ull)] = 0;
        eng.ctl->step = s + 1;
    }
}

// ---------------------------------------------------------------------------
// Deterministic aggregation.  Per step: sort the queue by (net, source);
// emit one (ring cell, weight) event per synapse in ascending (source,
// synapse) order; stable-sort the events by cell; fold each cell's run from
// left to right and add the sum to the ring.  The oracle performs the same
// per-(step, cell) fold, so ring contents and rasters are bit-identical.

__global__ void k_det_queue_keys(EngineDev eng, uint32_t q, unsigned long long* keys,
                                 uint32_t* vals, uint32_t count) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const SpikeRec r = (q ? eng.queue[1] : eng.queue[0])[e];
    keys[e] = ((unsigned long long)r.net << 32) | r.src;
    vals[e] = e;
}

__global__ void k_det_row_sizes(EngineDev eng, uint32_t q, const uint32_t* order, uint32_t count,
                                uint32_t* sizes) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const SpikeRec r = (q ? eng.queue[1] : eng.queue[0])[order[k]];
    const NetDev& n = eng.nets[r.net];
    sizes[k] = (uint32_t)(n.row_ptr[r.src + 1] - n.row_ptr[r.src]);
}

__global__ void __launch_bounds__(kScatterThreads) k_det_emit(EngineDev eng, uint32_t q,
                                                              const uint32_t* order, uint32_t count,
                                                              const uint32_t* offsets,
                                                              unsigned long long* keys, float* vals) {
    const unsigned long long s = eng.ctl->step;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long ev = 0;
    uint32_t ovf = 0;
    for (uint32_t k = warp; k < count; k += nwarps) {
        const SpikeRec r = (q ? eng.queue[1] : eng.queue[0])[order[k]];
        const NetDev& n = eng.nets[r.net];
        const uint32_t tl = (uint32_t)(s - n.start_step);
        const uint32_t tmod = tl % n.ring_slots;
        const uint64_t beg = n.row_ptr[r.src];
        const uint64_t end = n.row_ptr[r.src + 1];
        const bool plastic_src = n.stdp_on && r.src < n.n_plastic;
        const float mult = (!plastic_src && r.aux0 > 1) ? (float)r.aux0 : 1.0f;
        const uint32_t out0 = offsets[k];
        for (uint64_t j = beg + lane; j < end; j += 32) {
            const uint32_t tgt = n.tgt[j];
            unsigned long long key = ~0ull;
            float w = 0.0f;
            if (tgt != kTgtSentinel) {
                w = n.w[j];
                if (plastic_src && tgt < n.n_plastic) {
                    w = stdp_update(n, w, tgt, (int32_t)tl, r.aux0, r.aux1, ovf);
                    n.w[j] = w;
                }
                if (mult != 1.0f) w = __fmul_rn(w, mult);
                key = n.ring_key_base +
                      (unsigned long long)ring_slot(tmod, n.dly[j], n.ring_slots) * n.n_storage + tgt;
                ++ev;
            }
            keys[out0 + (uint32_t)(j - beg)] = key;
            vals[out0 + (uint32_t)(j - beg)] = w;
        }
    }
    ev = warp_sum_u64(ev);
    const unsigned long long ov = warp_sum_u64((unsigned long long)ovf);
    if (lane == 0) {
        if (ev) atomicAdd(&eng.ctl->events, ev);
        if (ov) atomicAdd(&eng.ctl->stdp_hist_overflow, ov);
    }
}

__global__ void k_det_fold(const NetDev* nets, uint32_t n_nets, const unsigned long long* keys,
                           const float* vals, uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const unsigned long long key = keys[i];
    if (key == ~0ull) return;
    if (i > 0 && keys[i - 1] == key) return;
    float sum = vals[i];
    for (uint32_t j = i + 1; j < count && keys[j] == key; ++j) sum = __fadd_rn(sum, vals[j]);
    // net owning this key: last net whose ring_key_base <= key
    uint32_t lo = 0, hi = n_nets;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (nets[mid].ring_key_base <= key) lo = mid; else hi = mid;
    }
    float* cell = nets[lo].ring + (key - nets[lo].ring_key_base);
    *cell = __fadd_rn(*cell, sum);
}

}  // namespace naer
