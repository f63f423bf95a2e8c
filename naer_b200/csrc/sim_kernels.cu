// Grid-mode simulation step: LIF update with fused Poisson input and
// warp-ballot spike compaction, warp-per-spike CSR scatter into the delay
// ring buffer with fused pair-based STDP, and the deterministic
// (sorted segmented-reduce) aggregation kernels.
//
// No global atomic counter sits on the hot path: each LIF block compacts
// its spikes into its own queue region (ballots plus a shared-memory
// counter) and publishes one count; each scatter block prefix-sums the
// counts in shared memory.  The only global atomics are the ring
// reductions themselves.
#include "grid_sync.cuh"
#include "sim_kernels.cuh"

namespace naer {

namespace {

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

// Fire-and-forget float reduction into global memory (no value returned,
// so the issuing warp never waits on it).
__device__ __forceinline__ void red_add_f32(float* addr, float v) {
    asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(addr), "f"(v) : "memory");
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Row [begin, end) of a source: two global loads named as such.
__device__ __forceinline__ ulonglong2 row_bounds(const uint64_t* row_ptr, uint32_t src) {
    const unsigned long long* rp = reinterpret_cast<const unsigned long long*>(row_ptr) + src;
    return make_ulonglong2(__ldg(rp), __ldg(rp + 1));
}

// Last region b in [0, n) with prefix[b] <= e (the region holding spike e).
__device__ __forceinline__ uint32_t locate(const uint32_t* prefix, uint32_t n, uint32_t e) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (prefix[mid] <= e) lo = mid; else hi = mid;
    }
    return lo;
}

}  // namespace

// ---------------------------------------------------------------------------
// Poisson draws of engine steps [s_first, s_first + nsteps): for every
// neuron of a population with a Poisson generator, the reference
// generator's event count in the step's window, one byte per neuron in slot
// (step mod kDriveSlots) of the net's drive ring (at most 10 events per
// window, input_neuron_group.cl:30).  Counter-based Philox makes the draws
// independent of the network state, so they run ahead of the simulation in
// a kernel of their own at full occupancy.  Work item = one chunk for all
// the steps (descriptors loaded once per chunk).
#ifndef NAER_DRIVE_MIN_BLOCKS
// resident blocks per SM of the Poisson-draw kernel: 3 leaves room for the
// per-neuron Philox products without spills (3.31 vs 3.51 us per step with
// 4 at 1M neurons)
#define NAER_DRIVE_MIN_BLOCKS 3
#endif

// Exact path of k_drive (a window whose first draw does not prove it
// empty), kept out of line so that the common path (one Philox per neuron)
// runs with few registers.
static __device__ __noinline__ uint32_t poisson_exact_call(double rate, uint32_t seed, uint32_t n_gen,
                                                           uint32_t idx, uint32_t z0, uint32_t t0, uint32_t t1) {
    return poisson_exact(rate, seed, n_gen, idx, ref_global_id(idx, kPoissonCapacity, kPoissonWorkgroup), z0, t0,
                         t1);
}

// A window queued for the exact path: storage index, drive slot, window
// start (us) and first draw.
struct DriveWindow {
    uint32_t i, slot, t0, z0;
};

// Windows a warp can hold: up to 31 left over plus 128 queued by one item
// (32 lanes x 4 neurons).
constexpr uint32_t kDriveQueue = 160;

// Resolves n <= 32 queued windows, one per lane, and writes their counts
// over the zero bytes the common path stored for them.  The warp barriers
// order those stores and the queue's shared-memory accesses.
__device__ __forceinline__ void drive_resolve(const PopDev& p, uint8_t* drive, uint32_t Ns, uint32_t dt_us,
                                              const DriveWindow* q, uint32_t n, uint32_t lane) {
    __syncwarp();
    if (lane < n) {
        const DriveWindow w = q[lane];
        const uint32_t idx = (p.type == kPOISSON ? p.rng_idx_base : 0u) + (w.i - p.storage_base);
        const uint32_t cnt = poisson_exact_call(p.rate_hz, p.rng_seed, p.rng_n, idx, w.z0, w.t0, w.t0 + dt_us);
        __stcg(drive + (size_t)w.slot * Ns + w.i, (unsigned char)cnt);
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kLifThreads, NAER_DRIVE_MIN_BLOCKS)
    k_drive(EngineDev eng, unsigned long long s_first, uint32_t nsteps) {
    // Windows whose first draw does not prove them empty (~rate x dt of
    // them) are queued per warp and resolved 32 at a time with every lane
    // busy, instead of by their own lanes while the rest of the warp waits.
    __shared__ DriveWindow s_q[kLifThreads / 32][kDriveQueue];
    DriveWindow* q = s_q[threadIdx.x >> 5];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t qn = 0;  // queued windows of this warp (the same in every lane)
    if (s_first == kStepFromCtl) s_first = eng.ctl->step;
    // (chunk, step) items in chunk-major order, an equal contiguous share per
    // block (the grid is the number of resident blocks): no partial last
    // wave, and a block reloads descriptors only when its chunk changes
    const uint64_t total = (uint64_t)eng.n_chunks * nsteps;
    const uint64_t per = (total + gridDim.x - 1) / gridDim.x;
    const uint64_t it_end = min(total, (uint64_t)(blockIdx.x + 1) * per);
    uint32_t cur = 0xFFFFFFFFu;
    PopDev p{};
    bool live = false;
    uint32_t i0 = 0, cend = 0, dt_us = 0, Ns = 0, idx0 = 0;
    uint32_t key[4] = {0, 0, 0, 0}, m_hi[4] = {0, 0, 0, 0}, m_lo[4] = {0, 0, 0, 0};  // per neuron, per chunk
    unsigned long long start = 0, stop = 0;
    uint8_t* drive = nullptr;
    const uint64_t it0 = (uint64_t)blockIdx.x * per;
    uint32_t c = (uint32_t)(it0 / nsteps);  // one division; then (c, k) advance incrementally
    uint32_t k = (uint32_t)(it0 - (uint64_t)c * nsteps);
    for (uint64_t it = it0; it < it_end; ++it, (++k == nsteps ? (k = 0, ++c) : 0)) {
        if (c != cur) {
            if (qn) {  // the previous chunk's windows, with its descriptors
                drive_resolve(p, drive, Ns, dt_us, q, qn, lane);
                qn = 0;
            }
            cur = c;
            const ChunkDev ch = eng.chunks[c];
            p = eng.pops[ch.pop];
            const NetDev* np = eng.nets + ch.net;
            start = np->start_step;
            stop = np->end_step;
            i0 = ch.first + threadIdx.x * kLifPerThread;
            cend = ch.end;
            live = p.rate_hz > 0.0 && np->active && i0 < cend;
            dt_us = np->dt_us;
            Ns = np->n_storage;
            drive = np->drive;
            idx0 = (p.type == kPOISSON ? p.rng_idx_base : 0u) + (i0 - p.storage_base);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                key[j] = ref_global_id(idx0 + j, kPoissonCapacity, kPoissonWorkgroup);
                mulhilo32(kPhiloxM0, key[j], m_hi[j], m_lo[j]);
            }
        }
        const unsigned long long s = s_first + k;
        const bool act = live && s >= start && s < stop;
        if (!__any_sync(0xFFFFFFFFu, act)) continue;  // the whole warp is idle on this item
        const uint32_t t0 = (uint32_t)(s - start) * dt_us;
        const uint32_t slot = (uint32_t)(s % kDriveSlots);
        uint32_t z[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            z[j] = philox_ref_z_pre(t0 * p.rng_n + idx0 + j, key[j], p.rng_seed, m_hi[j], m_lo[j]);
        uint32_t rare = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (act && i0 + j < cend && !poisson_quiet(p, z[j], t0)) rare |= 1u << j;
        if (act) __stcg(reinterpret_cast<unsigned int*>(drive + (size_t)slot * Ns + i0), 0u);
        if (__any_sync(0xFFFFFFFFu, rare != 0)) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool r = (rare >> j) & 1u;
                const uint32_t b = __ballot_sync(0xFFFFFFFFu, r);
                if (r) q[qn + __popc(b & lt_mask)] = DriveWindow{i0 + j, slot, t0, z[j]};
                qn += __popc(b);
            }
            while (qn >= 32) {
                qn -= 32;
                drive_resolve(p, drive, Ns, dt_us, q + qn, 32, lane);
            }
        }
    }
    if (qn) drive_resolve(p, drive, Ns, dt_us, q, qn, lane);
}

// ---------------------------------------------------------------------------
// LIF update of one work item = 1024 consecutive storage indices of one
// population, four neurons per thread (float4 membrane potential, uchar4
// refractory countdown, float4 ring slot read-and-clear, uchar4 Poisson
// counts).
//
// Grid-mode restatement of neuron_dynamics (include/naer/kernels/lif.cl:15-34)
// on a fixed step: V <- fp32(fp64(V) * exp(-dt/tau)); V += ring input; V +=
// drive weight once per Poisson drive event; spike iff V > v_th, then
// V = v_reset and t_ref steps of refractoriness, during which input is
// discarded.  POISSON populations emit the step's count of their reference
// generator (input_neuron_group.cl:6-45), drawn ahead by drive_chunks.
//
// Spikes are compacted with one ballot per neuron slot and one shared-memory
// atomicAdd per warp into the calling block's queue region.
__device__ __forceinline__ void lif_chunk(const EngineDev& eng, uint32_t c, unsigned long long s,
                                          SpikeRec* __restrict__ queue, uint32_t* __restrict__ qid,
                                          uint32_t* s_count) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const ChunkDev ch = eng.chunks[c];
    const PopDev p = eng.pops[ch.pop];
    const NetDev* np = eng.nets + ch.net;
    const unsigned long long start = np->start_step;
    if (!np->active || s < start || s >= np->end_step) return;  // uniform over the block
    const uint32_t tl = (uint32_t)(s - start);
    const uint32_t i0 = ch.first + threadIdx.x * kLifPerThread;
    const bool any = i0 < ch.end;

    bool spk[4] = {false, false, false, false};
    int32_t aux0[4] = {0, 0, 0, 0};
    float aux1[4] = {0.f, 0.f, 0.f, 0.f};

    const uint8_t* drive_slot = np->drive + (size_t)(s % kDriveSlots) * np->n_storage;
    if (p.type == kPOISSON) {
        if (any && p.rate_hz > 0.0) {
            const uchar4 m4 = *reinterpret_cast<const uchar4*>(drive_slot + i0);
            const uint32_t m[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (i0 + j < ch.end) {
                    spk[j] = m[j] > 0;
                    aux0[j] = (int32_t)m[j];
                }
            }
        }
    } else if (any) {
        const uint32_t Ns = np->n_storage;
        const uint32_t slot = tl % np->ring_slots;
        float4* __restrict__ ring4 = reinterpret_cast<float4*>(np->ring + (size_t)slot * Ns) + (i0 >> 2);
        float4* __restrict__ v4 = reinterpret_cast<float4*>(np->v) + (i0 >> 2);
        uchar4* __restrict__ r4 = reinterpret_cast<uchar4*>(np->refr) + (i0 >> 2);
        const bool plastic = (p.type == kSTDP) && np->stdp_on;
        uint32_t drive[4] = {0, 0, 0, 0};
        if (p.rate_hz > 0.0) {
            const uchar4 m4 = *reinterpret_cast<const uchar4*>(drive_slot + i0);
            drive[0] = m4.x;
            drive[1] = m4.y;
            drive[2] = m4.z;
            drive[3] = m4.w;
        }
        const float4 I = __ldcg(ring4);  // written by other SMs' reductions
        const float4 V4 = *v4;
        const uchar4 R4 = *r4;
        *ring4 = make_float4(0.f, 0.f, 0.f, 0.f);
        float vv[4] = {V4.x, V4.y, V4.z, V4.w};
        uint32_t rr[4] = {R4.x, R4.y, R4.z, R4.w};
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
            for (uint32_t k = 0; k < drive[j]; ++k) v = __fadd_rn(v, p.drive_w);
            if (v > p.v_th) {
                v = p.v_reset;
                rr[j] = p.t_ref_steps;
                spk[j] = true;
                if (plastic) stdp_post_spike(np, i, (int32_t)tl, aux0[j], aux1[j]);  // rare path
            }
            vv[j] = v;
        }
        *v4 = make_float4(vv[0], vv[1], vv[2], vv[3]);
        *r4 = make_uchar4((unsigned char)rr[0], (unsigned char)rr[1], (unsigned char)rr[2], (unsigned char)rr[3]);
    }

    // warp-ballot compaction into the block's queue region
    uint32_t b[4];
    uint32_t total = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        b[j] = __ballot_sync(0xFFFFFFFFu, spk[j]);
        total += __popc(b[j]);
    }
    if (total == 0) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(s_count, total);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    uint32_t run = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (spk[j]) {
            const uint32_t k = base + run + __popc(b[j] & lt_mask);
            const uint32_t i = i0 + j;
            __stcg(reinterpret_cast<int4*>(queue + k),
                   make_int4((int)ch.net, (int)i, aux0[j], __float_as_int(aux1[j])));
            __stcg(qid + k, p.id_base + (i - p.storage_base));
        }
        run += __popc(b[j]);
    }
}

// Standalone LIF pass (deterministic mode); same queue layout as k_run.
__global__ void __launch_bounds__(kLifThreads) k_lif(EngineDev eng) {
    __shared__ uint32_t s_count;
    const unsigned long long s = eng.ctl->step;
    const uint32_t qb = (uint32_t)(s & 1ull);
    const uint32_t region = blockIdx.x * eng.region_cap;
    SpikeRec* __restrict__ queue = (qb ? eng.queue[1] : eng.queue[0]) + region;
    uint32_t* __restrict__ qid = (qb ? eng.qid[1] : eng.qid[0]) + region;
    if (threadIdx.x == 0) {
        s_count = 0;
        if (blockIdx.x == 0) eng.ctl->raster_base = eng.ctl->raster_next;
    }
    __syncthreads();
    for (uint32_t c = blockIdx.x; c < eng.n_chunks; c += gridDim.x) lif_chunk(eng, c, s, queue, qid, &s_count);
    __syncthreads();
    if (threadIdx.x == 0) (qb ? eng.counts[1] : eng.counts[0])[blockIdx.x] = s_count;
}

// Exclusive prefix of the LIF blocks' spike counts into shared memory
// (prefix[0..n]); returns the total.
__device__ __forceinline__ uint32_t block_prefix_counts(const uint32_t* __restrict__ counts, uint32_t n,
                                                        uint32_t* prefix) {
    __shared__ uint32_t s_warp[kScatterThreads / 32];
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = threadIdx.x * per;
    uint32_t local = 0;
    for (uint32_t k = 0; k < per; ++k)
        if (lo + k < n) local += __ldcg(counts + lo + k);
    // inclusive scan of `local` over the block
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    uint32_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < blockDim.x / 32 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        if (lane < blockDim.x / 32) s_warp[lane] = w;
    }
    __syncthreads();
    uint32_t run = x - local + (wid ? s_warp[wid - 1] : 0);
    for (uint32_t k = 0; k < per; ++k) {
        if (lo + k < n) {
            prefix[lo + k] = run;
            run += __ldcg(counts + lo + k);
        }
    }
    if (threadIdx.x == blockDim.x - 1) prefix[n] = run;
    __syncthreads();
    return prefix[n];
}

// Atomic-mode scatter of step s over the queued spikes.  Each spike is
// served by `scatter_split` warps; warp k of a spike walks pieces k, k +
// split, ... of kScatterPiece synapses of the source's CSR row with 128-bit
// streaming loads (4 targets, 4 weights, 4 delays per lane per slice,
// kScatterUnroll slices in flight) and reduces each weight into
// ring[(t + d) mod D][target] with a fire-and-forget red.add.  STDP sources
// update plastic synapses first and write the weight back.  This replaces
// the reference's per-group walk over every input spike (nop.cl:40-83,
// stdp.cl:66-133) and its histogram/scatter/offset passes
// (spike_aggregation.cl).  The first warp of each spike appends it to the
// raster at rbase + its queue rank.
__device__ __forceinline__ void scatter_step(const EngineDev& eng, unsigned long long s, const uint32_t* prefix,
                                             uint32_t Q, unsigned long long rbase, unsigned long long& ev,
                                             uint32_t& ovf, const NetDev* net0) {
    const uint32_t qb = (uint32_t)(s & 1ull);
    const SpikeRec* __restrict__ queue = qb ? eng.queue[1] : eng.queue[0];
    const uint32_t* __restrict__ qid = qb ? eng.qid[1] : eng.qid[0];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t split = eng.scatter_split;
    const uint32_t psz = eng.scatter_piece;  // 128 or 256 synapses per warp iteration
    const uint32_t items = Q * split;
    const uint32_t G = eng.lif_grid;

    for (uint32_t it = warp; it < items; it += nwarps) {
        const uint32_t e = it / split;
        const uint32_t piece = it - e * split;
        const uint32_t reg = locate(prefix, G, e);
        const uint32_t qpos = reg * eng.region_cap + (e - prefix[reg]);
        // queue entries come from other blocks of the same launch: read at L2
        const int4 rv = __ldcg(reinterpret_cast<const int4*>(queue + qpos));
        SpikeRec r;
        r.net = (uint32_t)rv.x;
        r.src = (uint32_t)rv.y;
        r.aux0 = rv.z;
        r.aux1 = __int_as_float(rv.w);
        if (piece == 0 && lane == 0 && eng.record && rbase + e < eng.raster_cap)
            __stcg(eng.raster + rbase + e, make_uint2((uint32_t)s, __ldcg(qid + qpos)));
        const NetDev* np = (r.net == 0 && net0) ? net0 : eng.nets + r.net;
        const uint32_t tl = (uint32_t)(s - np->start_step);
        const uint32_t D = np->ring_slots;
        const uint32_t tmod = tl % D;
        const uint32_t Ns = np->n_storage;
        float* __restrict__ ring = np->ring;
        const uint32_t* __restrict__ tgt_a = np->tgt;
        float* __restrict__ w_a = np->w;
        const uint8_t* __restrict__ d_a = np->dly;
        const ulonglong2 rb = row_bounds(np->row_ptr, r.src);
        const uint64_t beg = rb.x;
        const uint64_t end = rb.y;
        const uint32_t n_plastic = np->n_plastic;
        const bool plastic_src = np->stdp_on && r.src < n_plastic;
        StdpView sv;
        if (plastic_src) sv = stdp_view(*np);
        const float mult = (!plastic_src && r.aux0 > 1) ? (float)r.aux0 : 1.0f;

        for (uint64_t base = beg + (uint64_t)piece * psz; base < end; base += (uint64_t)split * psz) {
            uint4 tg[kScatterUnroll];
            float4 ww[kScatterUnroll];
            uint32_t dd[kScatterUnroll];
#pragma unroll
            for (int u = 0; u < (int)kScatterUnroll; ++u) {
                const uint64_t off = base + (uint64_t)(u * 32 + lane) * 4ull;
                if (off < end && (uint32_t)u * 128u < psz) {
                    tg[u] = ld_stream_u4(tgt_a + off);
                    ww[u] = __ldcg(reinterpret_cast<const float4*>(w_a + off));  // STDP may rewrite
                    dd[u] = ld_stream_u32(d_a + off);
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
                    if (plastic_src && tgt < n_plastic) {
                        w = stdp_update(sv, w, tgt, (int32_t)tl, r.aux0, r.aux1, ovf);
                        __stcg(w_a + off + j, w);
                    }
                    if (mult != 1.0f) w = __fmul_rn(w, mult);
                    red_add_f32(ring + (size_t)ring_slot(tmod, d, D) * Ns + tgt, w);
                    ++ev;
                }
            }
        }
    }
}

// Descriptor of one chunk owned by a persistent block, cached in shared
// memory for the whole launch.
struct ChunkCache {
    PopDev p;
    float* ring;
    float* v;
    uint8_t* refr;
    uint8_t* drive;
    unsigned long long start, stop;
    uint32_t first, end, net, Ns;
    uint32_t slots, dt_us, active, plastic;
};

// LIF of one owned chunk with V, refractory counters and Poisson counts in
// shared memory (sV/sR/sD hold four neurons per thread per chunk).  Same
// arithmetic as lif_chunk.
// Loads of one owned chunk for step s, issued for a whole batch of chunks
// before any is processed so their latencies overlap: the ring slot (other
// SMs' reductions wrote it) and the Poisson counts.  Every access names the
// global space explicitly; the ring slot is cleared by lif_clear after the
// whole batch of loads has been issued, so no load waits behind a store.
__device__ __forceinline__ void lif_prefetch(const ChunkCache& cc, unsigned long long s, float4& I, uint32_t& Dw) {
    // predicated loads, no use of their values here: a chunk's loads never
    // wait for an earlier chunk's data
    const uint32_t i0 = cc.first + threadIdx.x * kLifPerThread;
    const bool live = cc.active && s >= cc.start && s < cc.stop && i0 < cc.end;
    const uint32_t tl = (uint32_t)(s - cc.start);
    const bool want_d = live && cc.p.rate_hz > 0.0;
    const bool want_i = live && cc.p.type != kPOISSON;
    Dw = want_d ? __ldcg(reinterpret_cast<const unsigned int*>(cc.drive + (size_t)(s % kDriveSlots) * cc.Ns + i0))
                : 0u;
    I = want_i ? __ldcg(reinterpret_cast<const float4*>(cc.ring + (size_t)(tl % cc.slots) * cc.Ns) + (i0 >> 2))
               : make_float4(0.f, 0.f, 0.f, 0.f);
}

__device__ __forceinline__ void lif_clear(const ChunkCache& cc, unsigned long long s) {
    if (!cc.active || s < cc.start || s >= cc.stop || cc.p.type == kPOISSON) return;
    const uint32_t i0 = cc.first + threadIdx.x * kLifPerThread;
    if (i0 >= cc.end) return;
    const uint32_t tl = (uint32_t)(s - cc.start);
    __stcg(reinterpret_cast<float4*>(cc.ring + (size_t)(tl % cc.slots) * cc.Ns) + (i0 >> 2),
           make_float4(0.f, 0.f, 0.f, 0.f));
}

__device__ __forceinline__ void lif_chunk_smem(const EngineDev& eng, const ChunkCache& cc, uint32_t j,
                                               unsigned long long s, float4* sV, uchar4* sR, const float4 I,
                                               const uint32_t Dw, SpikeRec* __restrict__ queue,
                                               uint32_t* __restrict__ qid, uint32_t* s_count) {
    if (!cc.active || s < cc.start || s >= cc.stop) return;  // uniform over the block
    const uchar4 D4 = make_uchar4(Dw & 0xFFu, (Dw >> 8) & 0xFFu, (Dw >> 16) & 0xFFu, Dw >> 24);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t tl = (uint32_t)(s - cc.start);
    const uint32_t i0 = cc.first + threadIdx.x * kLifPerThread;
    const uint32_t si = j * kLifThreads + threadIdx.x;
    const bool any = i0 < cc.end;
    bool spk[4] = {false, false, false, false};
    int32_t aux0[4] = {0, 0, 0, 0};
    float aux1[4] = {0.f, 0.f, 0.f, 0.f};
    const uint32_t type = cc.p.type;
    if (type == kPOISSON) {
        if (any && cc.p.rate_hz > 0.0) {
            const uchar4 m4 = D4;
            const uint32_t m[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (i0 + k < cc.end) {
                    spk[k] = m[k] > 0;
                    aux0[k] = (int32_t)m[k];
                }
            }
        }
    } else if (any) {
        const float4 V4 = sV[si];
        const uchar4 R4 = sR[si];
        float vv[4] = {V4.x, V4.y, V4.z, V4.w};
        uint32_t rr[4] = {R4.x, R4.y, R4.z, R4.w};
        const uint32_t dd[4] = {D4.x, D4.y, D4.z, D4.w};
        const double prop = cc.p.prop;
        const float v_th = cc.p.v_th, v_reset = cc.p.v_reset, dw = cc.p.drive_w;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t i = i0 + k;
            if (i >= cc.end) continue;
            if (rr[k] > 0) {
                rr[k] -= 1;
                continue;
            }
            float v = __double2float_rn(__dmul_rn((double)vv[k], prop));
            v = __fadd_rn(v, f4_get(I, k));
            for (uint32_t m = 0; m < dd[k]; ++m) v = __fadd_rn(v, dw);
            if (v > v_th) {
                v = v_reset;
                rr[k] = cc.p.t_ref_steps;
                spk[k] = true;
                if (cc.plastic) stdp_post_spike(eng.nets + cc.net, i, (int32_t)tl, aux0[k], aux1[k]);
            }
            vv[k] = v;
        }
        sV[si] = make_float4(vv[0], vv[1], vv[2], vv[3]);
        sR[si] = make_uchar4((unsigned char)rr[0], (unsigned char)rr[1], (unsigned char)rr[2], (unsigned char)rr[3]);
    }
    uint32_t b[4];
    uint32_t total = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        b[k] = __ballot_sync(0xFFFFFFFFu, spk[k]);
        total += __popc(b[k]);
    }
    if (total == 0) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(s_count, total);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    uint32_t run = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (spk[k]) {
            const uint32_t q = base + run + __popc(b[k] & lt_mask);
            const uint32_t i = i0 + k;
            __stcg(reinterpret_cast<int4*>(queue + q),
                   make_int4((int)cc.net, (int)i, aux0[k], __float_as_int(aux1[k])));
            __stcg(qid + q, cc.p.id_base + (i - cc.p.storage_base));
        }
        run += __popc(b[k]);
    }
}

// Persistent step kernel (atomic mode): nsteps grid steps from engine step
// s0 in one cooperative launch, after k_drive has drawn their Poisson
// counts.  Per step: every block runs the LIF on its chunks and publishes
// its spike count; grid barrier; every block prefix-sums the counts and
// scatters its share of the queued spikes; grid barrier.  With kSmem the
// block keeps its chunks' descriptors, membrane potentials and refractory
// counters in shared memory for the whole launch (loaded at entry, written
// back at exit); otherwise they stay in global memory.  Block 0 times the
// phases with %globaltimer.
#ifndef NAER_RUN_MIN_BLOCKS
#define NAER_RUN_MIN_BLOCKS 2  // resident blocks per SM the register budget must allow
#endif

template <bool kSmem>
__global__ void __launch_bounds__(kLifThreads, NAER_RUN_MIN_BLOCKS)
    k_run(EngineDev eng, unsigned long long s0, uint32_t nsteps) {
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ uint32_t s_count;
    __shared__ unsigned long long s_ev;
    __shared__ uint32_t s_ovf;
    __shared__ NetDev s_net0;  // descriptor of the first net (the only one in the plain form)
    const uint32_t G = gridDim.x;
    if (threadIdx.x == 0) s_net0 = eng.nets[0];
    uint32_t* s_prefix = reinterpret_cast<uint32_t*>(s_dyn);  // [G + 1]
    const uint32_t own_max = eng.region_cap / kLifChunk;
    const size_t off_cc = (((G + 1) * sizeof(uint32_t)) + 15) & ~(size_t)15;
    ChunkCache* s_cc = reinterpret_cast<ChunkCache*>(s_dyn + off_cc);
    const size_t off_v = off_cc + (((size_t)own_max * sizeof(ChunkCache) + 15) & ~(size_t)15);
    float4* sV = reinterpret_cast<float4*>(s_dyn + off_v);
    uchar4* sR = reinterpret_cast<uchar4*>(s_dyn + off_v + (size_t)own_max * kLifThreads * sizeof(float4));
    const uint32_t own = blockIdx.x < eng.n_chunks ? (eng.n_chunks - blockIdx.x + G - 1) / G : 0u;

    Ctl* ctl = eng.ctl;
    __shared__ BarrierCfg bcfg;  // read by thread 0 at each barrier; kept out of registers
    if (threadIdx.x == 0) bcfg = barrier_cfg(ctl);
    unsigned long long bar_target = 0;
    // every block reads the engine step before the first grid barrier; block 0
    // advances it only after the last one
    if (s0 == kStepFromCtl) s0 = ctl->step;
    unsigned long long rbase = ctl->raster_next;
    unsigned long long dropped = 0;
    const uint32_t region = blockIdx.x * eng.region_cap;
    unsigned long long ev = 0;
    uint32_t ovf = 0;
    unsigned long long t_lif = 0, t_sc = 0;
    unsigned long long t_ph[5] = {0, 0, 0, 0, 0};
    const bool timer = blockIdx.x == 0 && threadIdx.x == 0;
    if (threadIdx.x == 0) {
        s_ev = 0;
        s_ovf = 0;
    }
    if (kSmem) {
        for (uint32_t j = threadIdx.x; j < own; j += blockDim.x) {
            const ChunkDev ch = eng.chunks[blockIdx.x + j * G];
            const NetDev* np = eng.nets + ch.net;
            ChunkCache c;
            c.p = eng.pops[ch.pop];
            c.ring = np->ring;
            c.v = np->v;
            c.refr = np->refr;
            c.drive = np->drive;
            c.start = np->start_step;
            c.stop = np->end_step;
            c.first = ch.first;
            c.end = ch.end;
            c.net = ch.net;
            c.Ns = np->n_storage;
            c.slots = np->ring_slots;
            c.dt_us = np->dt_us;
            c.active = np->active;
            c.plastic = (c.p.type == kSTDP && np->stdp_on) ? 1u : 0u;
            s_cc[j] = c;
        }
        __syncthreads();
        for (uint32_t j = 0; j < own; ++j) {
            const uint32_t i0 = s_cc[j].first + threadIdx.x * kLifPerThread;
            if (i0 < s_cc[j].end) {
                const uint32_t si = j * kLifThreads + threadIdx.x;
                sV[si] = *reinterpret_cast<const float4*>(s_cc[j].v + i0);
                sR[si] = *reinterpret_cast<const uchar4*>(s_cc[j].refr + i0);
            }
        }
    }
    uint32_t k = 0;
    for (; k < nsteps; ++k) {
        const unsigned long long s = s0 + k;
        const uint32_t qb = (uint32_t)(s & 1ull);
        const unsigned long long ta = timer ? globaltimer_ns() : 0ull;
        if (threadIdx.x == 0) s_count = 0;
        __syncthreads();
        SpikeRec* queue = (qb ? eng.queue[1] : eng.queue[0]) + region;
        uint32_t* qid = (qb ? eng.qid[1] : eng.qid[0]) + region;
        if (kSmem) {
            for (uint32_t j0 = 0; j0 < own; j0 += kLifBatch) {
                float4 I[kLifBatch];
                uint32_t D[kLifBatch];
#pragma unroll
                for (uint32_t b = 0; b < kLifBatch; ++b)
                    if (j0 + b < own) lif_prefetch(s_cc[j0 + b], s, I[b], D[b]);
#pragma unroll
                for (uint32_t b = 0; b < kLifBatch; ++b)
                    if (j0 + b < own) lif_clear(s_cc[j0 + b], s);
#pragma unroll
                for (uint32_t b = 0; b < kLifBatch; ++b)
                    if (j0 + b < own)
                        lif_chunk_smem(eng, s_cc[j0 + b], j0 + b, s, sV, sR, I[b], D[b], queue, qid, &s_count);
            }
        } else {
            for (uint32_t c = blockIdx.x; c < eng.n_chunks; c += G) lif_chunk(eng, c, s, queue, qid, &s_count);
        }
        __syncthreads();
        if (threadIdx.x == 0) (qb ? eng.counts[1] : eng.counts[0])[blockIdx.x] = s_count;
        const unsigned long long ta2 = timer ? globaltimer_ns() : 0ull;
        bar_target += G;
        if (!grid_barrier(ctl, bar_target, bcfg)) break;
        const unsigned long long tb = timer ? globaltimer_ns() : 0ull;

        const uint32_t Q = block_prefix_counts(qb ? eng.counts[1] : eng.counts[0], G, s_prefix);
        scatter_step(eng, s, s_prefix, Q, rbase, ev, ovf, &s_net0);
        const unsigned long long tb2 = timer ? globaltimer_ns() : 0ull;
        const unsigned long long cap = eng.record ? eng.raster_cap : 0ull;
        const unsigned long long kept = rbase + Q <= cap ? Q : (rbase >= cap ? 0ull : cap - rbase);
        if (eng.record) dropped += Q - kept;
        rbase += kept;
        bar_target += G;
        if (!grid_barrier(ctl, bar_target, bcfg)) break;
        if (timer) {
            const unsigned long long tc = globaltimer_ns();
            t_lif += tb - ta;
            t_sc += tc - tb;
            t_ph[0] += ta2 - ta;
            t_ph[1] += tb - ta2;
            t_ph[2] += tb2 - tb;
            t_ph[4] += tc - tb2;
        }
    }
    if (kSmem) {
        __syncthreads();
        for (uint32_t j = 0; j < own; ++j) {
            const uint32_t i0 = s_cc[j].first + threadIdx.x * kLifPerThread;
            if (i0 < s_cc[j].end) {
                const uint32_t si = j * kLifThreads + threadIdx.x;
                *reinterpret_cast<float4*>(s_cc[j].v + i0) = sV[si];
                *reinterpret_cast<uchar4*>(s_cc[j].refr + i0) = sR[si];
            }
        }
    }

    // per-block counters: no same-address global atomics on the hot path
    ev = warp_sum_u64(ev);
    const unsigned long long ov = warp_sum_u64((unsigned long long)ovf);
    if ((threadIdx.x & 31u) == 0) {
        if (ev) atomicAdd(&s_ev, ev);
        if (ov) atomicAdd(&s_ovf, (uint32_t)ov);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_ev) eng.ev_part[blockIdx.x] += s_ev;
        if (s_ovf) eng.ovf_part[blockIdx.x] += s_ovf;
    }
    if (timer) {
        ctl->step = s0 + k;
        ctl->raster_next = rbase;
        ctl->raster_base = rbase;
        ctl->raster_dropped += dropped;
        ctl->prof_lif_ns += t_lif;
        ctl->prof_scatter_ns += t_sc;
        ctl->prof_steps += k;
        for (int q = 0; q < 5; ++q) ctl->prof_phase_ns[q] += t_ph[q];
    }
}

template __global__ void k_run<true>(EngineDev, unsigned long long, uint32_t);
template __global__ void k_run<false>(EngineDev, unsigned long long, uint32_t);

size_t run_smem_bytes(uint32_t grid, uint32_t own_max, bool smem_state) {
    const size_t off_cc = (((grid + 1) * sizeof(uint32_t)) + 15) & ~(size_t)15;
    if (!smem_state) return off_cc;
    const size_t off_v = off_cc + (((size_t)own_max * sizeof(ChunkCache) + 15) & ~(size_t)15);
    return off_v + (size_t)own_max * kLifThreads * (sizeof(float4) + sizeof(uchar4));
}

// ---------------------------------------------------------------------------
// Deterministic aggregation.  Per step: sort the queue by (net, source);
// emit one (ring cell, weight) event per synapse in ascending (source,
// synapse) order; stable-sort the events by cell; fold each cell's run from
// left to right and add the sum to the ring.  The oracle performs the same
// per-(step, cell) fold, so ring contents and rasters are bit-identical.
// `prefix` is the exclusive scan of the LIF blocks' counts (lif_grid + 1).

__global__ void k_det_queue_keys(EngineDev eng, const uint32_t* prefix, unsigned long long* keys,
                                 uint32_t* vals, uint32_t count) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const uint32_t qb = (uint32_t)(eng.ctl->step & 1ull);
    const uint32_t reg = locate(prefix, eng.lif_grid, e);
    const uint32_t qpos = reg * eng.region_cap + (e - prefix[reg]);
    const SpikeRec r = (qb ? eng.queue[1] : eng.queue[0])[qpos];
    keys[e] = ((unsigned long long)r.net << 32) | r.src;
    vals[e] = qpos;
}

__global__ void k_det_row_sizes(EngineDev eng, const uint32_t* order, uint32_t count, uint32_t* sizes) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const uint32_t qb = (uint32_t)(eng.ctl->step & 1ull);
    const SpikeRec r = (qb ? eng.queue[1] : eng.queue[0])[order[k]];
    const NetDev& n = eng.nets[r.net];
    sizes[k] = (uint32_t)(n.row_ptr[r.src + 1] - n.row_ptr[r.src]);
}

// Raster records of the sorted queue; advances the raster position.
__global__ void k_det_raster(EngineDev eng, const uint32_t* order, uint32_t count) {
    const unsigned long long s = eng.ctl->step;
    const uint32_t qb = (uint32_t)(s & 1ull);
    const unsigned long long rbase = eng.ctl->raster_base;
    const uint32_t* __restrict__ qid = qb ? eng.qid[1] : eng.qid[0];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
        if (eng.record && rbase + k < eng.raster_cap) eng.raster[rbase + k] = make_uint2((uint32_t)s, qid[order[k]]);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const unsigned long long cap = eng.record ? eng.raster_cap : 0ull;
        const unsigned long long kept = rbase + count <= cap ? count : (rbase >= cap ? 0ull : cap - rbase);
        eng.ctl->raster_next = rbase + kept;
        if (eng.record && kept < count) eng.ctl->raster_dropped += count - kept;
    }
}

__global__ void __launch_bounds__(kScatterThreads) k_det_emit(EngineDev eng, const uint32_t* order,
                                                              uint32_t count, const uint32_t* offsets,
                                                              unsigned long long* keys, float* vals) {
    const unsigned long long s = eng.ctl->step;
    const uint32_t qb = (uint32_t)(s & 1ull);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long ev = 0;
    uint32_t ovf = 0;
    for (uint32_t k = warp; k < count; k += nwarps) {
        const SpikeRec r = (qb ? eng.queue[1] : eng.queue[0])[order[k]];
        const NetDev& n = eng.nets[r.net];
        const uint32_t tl = (uint32_t)(s - n.start_step);
        const uint32_t tmod = tl % n.ring_slots;
        const uint64_t beg = n.row_ptr[r.src];
        const uint64_t end = n.row_ptr[r.src + 1];
        const bool plastic_src = n.stdp_on && r.src < n.n_plastic;
        StdpView sv;
        if (plastic_src) sv = stdp_view(n);
        const float mult = (!plastic_src && r.aux0 > 1) ? (float)r.aux0 : 1.0f;
        const uint32_t out0 = offsets[k];
        for (uint64_t j = beg + lane; j < end; j += 32) {
            const uint32_t tgt = n.tgt[j];
            unsigned long long key = ~0ull;
            float w = 0.0f;
            if (tgt != kTgtSentinel) {
                w = n.w[j];
                if (plastic_src && tgt < n.n_plastic) {
                    w = stdp_update(sv, w, tgt, (int32_t)tl, r.aux0, r.aux1, ovf);
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

// Advances the engine step after the deterministic aggregation.
__global__ void k_advance(EngineDev eng) {
    if (threadIdx.x == 0 && blockIdx.x == 0) eng.ctl->step = eng.ctl->step + 1;
}

}  // namespace naer
