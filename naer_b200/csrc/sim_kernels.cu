// Grid-mode simulation step: Poisson draws ahead of the simulation
// (k_drive), and three persistent cooperative step kernels that run up to 64
// grid steps per launch, each step = LIF with fused Poisson input and
// warp-ballot spike compaction, then a warp-per-row CSR scatter into the
// delay ring with fused pair-based STDP:
//   k_step      atomic aggregation, one spike list per step, scatter split
//               by deadline (default);
//   k_run       atomic aggregation, per-block spike regions and two grid
//               barriers per step (kept as a tuning choice);
//   k_det_step  deterministic aggregation through per-cell event lists
//               folded in canonical (source, synapse) order.
// The ring reductions and one list reservation per warp and step are the
// only global atomics on the hot path.
#include "check.cuh"
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

// Fire-and-forget integer reduction (exact-sum aggregation).
__device__ __forceinline__ void red_add_s32(float* addr, int v) {
    asm volatile("red.relaxed.gpu.global.add.s32 [%0], %1;" ::"l"(addr), "r"(v) : "memory");
}

// Ring-cell input as the neuron reads it: the float sum, or with exact-sum
// aggregation (fx_inv != 0) the cell's integer sum times 2^-S.
__device__ __forceinline__ float ring_input(float cell, float fx_inv) {
    return fx_inv != 0.0f ? __fmul_rn(__int2float_rn(__float_as_int(cell)), fx_inv) : cell;
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
                                              const DriveWindow* q, uint32_t n, uint32_t lane, Ctl* ctl) {
    __syncwarp();
    if (lane < n) {
        const DriveWindow w = q[lane];
        const uint32_t idx = (p.type == kPOISSON ? p.rng_idx_base : 0u) + (w.i - p.storage_base);
        const uint32_t cnt = poisson_exact_call(p.rate_hz, p.rng_seed, p.rng_n, idx, w.z0, w.t0, w.t0 + dt_us);
        if (NAER_IN_BOUNDS(ctl, w.i, Ns, kChkDrive)) __stcg(drive + (size_t)w.slot * Ns + w.i, (unsigned char)cnt);
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
                drive_resolve(p, drive, Ns, dt_us, q, qn, lane, eng.ctl);
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
        if (act && NAER_IN_BOUNDS(eng.ctl, i0 + 3, Ns, kChkDrive))
            __stcg(reinterpret_cast<unsigned int*>(drive + (size_t)slot * Ns + i0), 0u);
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
                drive_resolve(p, drive, Ns, dt_us, q + qn, 32, lane, eng.ctl);
            }
        }
    }
    if (qn) drive_resolve(p, drive, Ns, dt_us, q, qn, lane, eng.ctl);
}

// ---------------------------------------------------------------------------
// LIF update of one work item = 1024 consecutive storage indices of one
// population, four neurons per thread (float4 membrane potential, uchar4
// refractory countdown, float4 ring slot read-and-clear, uchar4 Poisson
// counts).
//
// Grid-mode restatement of neuron_dynamics (include/naer/kernels/lif.cl:15-34)
// on a fixed step: V <- fp32(fp64(V) * exp(-dt/tau) + ring input + m * drive
// weight) for m Poisson drive events, in double with one rounding
// (lif_update); spike iff V > v_th, then V = v_reset and t_ref steps of
// refractoriness, during which input is discarded.  POISSON populations emit the step's count of their reference
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
            float v = lif_update(vv[j], p.prop, ring_input(f4_get(I, j), np->fx_inv), drive[j], p.drive_w);
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
        const float qs = np->fx_scale;  // exact-sum aggregation: 2^S, else 0

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
                    float* cell = ring + (size_t)ring_slot(tmod, d, D) * Ns + tgt;
                    if (qs != 0.0f) red_add_s32(cell, __float2int_rn(__fmul_rn(w, qs)));
                    else red_add_f32(cell, w);
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
    const uint64_t* row_ptr;  // the net's CSR rows (queued spikes carry their bounds)
    const uint32_t* row_mid;
    float* ring;
    float* v;
    uint8_t* refr;
    uint8_t* drive;
    unsigned long long start, stop;
    uint32_t first, end, net, Ns;
    uint32_t slots, dt_us, active, plastic;
    float fx_inv;  // exact-sum aggregation: 2^-S (0: the ring holds floats)
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
            float v = lif_update(vv[k], prop, ring_input(f4_get(I, k), cc.fx_inv), dd[k], dw);
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
            c.fx_inv = np->fx_inv;
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

// ---------------------------------------------------------------------------
// k_step: the persistent step kernel (atomic mode) with one contiguous spike
// list per step and the scatter split by deadline.
//
// Per grid step s:
//  1. LIF of the block's chunks.  A warp keeps the spike flags of a batch of
//     chunks in registers and reserves their places in the step's list with
//     one atomic on Ctl::qtail[s & 3], then writes the records: no per-block
//     regions, no prefix sum of block counts, no search for a spike's region.
//  2. Grid barrier B1 (the list is complete).  While warp 0 waits for it, the
//     block's other warps deliver what is left of step s-1's deferred part.
//  3. The first part of every row: the delay-1 synapses of static sources
//     (the next LIF reads them) and the whole row of plastic sources (their
//     weight updates must see the post-synaptic state of step s).  Then any
//     deferred work of step s-1 still left: its delay-2 synapses feed the
//     LIF of step s+1.
//  4. Arrive at grid barrier B2.  While warp 0 waits for it, warps 1.. deliver
//     the rest of step s's rows (delays >= 2 of static sources); what is left
//     when B2 completes moves to step s+1 (at the latest before its B2
//     arrival, which precedes the LIF of step s+2).
// Every delivery is a red.add into the ring as in k_run; only the time at
// which a synapse is delivered moves, never its ring slot.

// Shared-memory binning of ring reductions (tuning `bins`, 0 = off).  A
// block folds events into an open-addressing table keyed by ring-cell
// address (shared-memory atomics), and a flush issues one global reduction
// per occupied entry before the block publishes its deliveries at a grid
// barrier.  Events whose probe finds no entry go to global memory directly.
// It pays where many events of a block hit the same cells (convergent or
// hub targets, whose global reductions to one address serialize in L2); on
// uniformly random targets it only adds work.
struct BinTable {
    unsigned long long* key;  // ring-cell address, 0 = empty
    float* sum;
    uint32_t mask;            // entries - 1; 0 = binning off
};

constexpr int kBinProbes = 4;

// qs != 0: exact-sum aggregation, the weight rounded to the nearest
// multiple of 1/qs = 2^-S and added as an integer (binning is off then).
__device__ __forceinline__ void ring_add(const BinTable& bt, float* addr, float w, float qs) {
    if (qs != 0.0f) {
        red_add_s32(addr, __float2int_rn(__fmul_rn(w, qs)));
        return;
    }
    if (bt.mask) {
        const unsigned long long a = (unsigned long long)addr;
        uint32_t h = (uint32_t)(((a >> 2) * 0x9E3779B97F4A7C15ull) >> 40) & bt.mask;
#pragma unroll
        for (int p = 0; p < kBinProbes; ++p) {
            const unsigned long long k = *(volatile unsigned long long*)(bt.key + h);
            if (k == a) {
                atomicAdd(bt.sum + h, w);
                return;
            }
            if (k == 0ull) {
                const unsigned long long old = atomicCAS(bt.key + h, 0ull, a);
                if (old == 0ull || old == a) {
                    atomicAdd(bt.sum + h, w);
                    return;
                }
            }
            h = (h + 1) & bt.mask;
        }
    }
    red_add_f32(addr, w);
}

// Every thread of the block: issues the table's sums and empties it.
__device__ __forceinline__ void flush_bins(const BinTable& bt) {
    if (!bt.mask) return;  // uniform over the block
    __syncthreads();
    for (uint32_t i = threadIdx.x; i <= bt.mask; i += blockDim.x) {
        const unsigned long long a = bt.key[i];
        if (a) {
            red_add_f32(reinterpret_cast<float*>(a), bt.sum[i]);
            bt.key[i] = 0ull;
            bt.sum[i] = 0.0f;
        }
    }
    __syncthreads();
}

// Delivers the synapses [lo, hi) of one spike's row: warp pieces piece,
// piece + split, ... of psz synapses, 128-bit loads, red.add into the ring
// (STDP update first for plastic synapses of plastic sources).
__device__ __forceinline__ void deliver_span(const NetDev* np, uint32_t tl, const SpikeRec& r, uint64_t lo,
                                             uint64_t hi, uint32_t piece, uint32_t split, uint32_t psz,
                                             uint32_t lane, unsigned long long& ev, uint32_t& ovf, Ctl* ctl,
                                             const BinTable& bt) {
    const uint32_t D = np->ring_slots;
    const uint32_t tmod = tl % D;
    const uint32_t Ns = np->n_storage;
    float* __restrict__ ring = np->ring;
    const float qs = np->fx_scale;  // exact-sum aggregation: 2^S, else 0
    const uint32_t* __restrict__ tgt_a = np->tgt;
    float* __restrict__ w_a = np->w;
    const uint8_t* __restrict__ d_a = np->dly;
    const uint32_t n_plastic = np->n_plastic;
    const bool plastic_src = np->stdp_on && r.src < n_plastic;
    if (plastic_src) {
        // one synapse per lane: each weight update waits on its target's
        // post row, so a lane takes one of them per piece of kPlasticPiece
        const StdpView sv = stdp_view(*np);
        for (uint64_t base = lo + (uint64_t)piece * kPlasticPiece; base < hi;
             base += (uint64_t)split * kPlasticPiece) {
            const uint64_t j = base + lane;
            if (j >= hi || !NAER_IN_BOUNDS(ctl, j, np->syn_cap, kChkSynapse)) continue;
            const uint32_t tgt = __ldcs(tgt_a + j);
            if (tgt == kTgtSentinel || !NAER_IN_BOUNDS(ctl, tgt, Ns, kChkRing)) continue;
            float w = __ldcg(w_a + j);
            const uint32_t d = __ldcs(d_a + j);
            if (tgt < n_plastic) {
                w = stdp_update(sv, w, tgt, (int32_t)tl, r.aux0, r.aux1, ovf);
                __stcg(w_a + j, w);
            }
            ring_add(bt, ring + (size_t)ring_slot(tmod, d, D) * Ns + tgt, w, qs);
            ++ev;
        }
        return;
    }
    const float mult = r.aux0 > 1 ? (float)r.aux0 : 1.0f;
    for (uint64_t base = lo + (uint64_t)piece * psz; base < hi; base += (uint64_t)split * psz) {
        uint4 tg[kScatterUnroll];
        float4 ww[kScatterUnroll];
        uint32_t dd[kScatterUnroll];
#pragma unroll
        for (int u = 0; u < (int)kScatterUnroll; ++u) {
            const uint64_t off = base + (uint64_t)(u * 32 + lane) * 4ull;
            if (off < hi && (uint32_t)u * 128u < psz && NAER_IN_BOUNDS(ctl, off + 3, np->syn_cap, kChkSynapse)) {
                tg[u] = ld_stream_u4(tgt_a + off);
                ww[u] = __ldcg(reinterpret_cast<const float4*>(w_a + off));
                dd[u] = ld_stream_u32(d_a + off);
            } else {
                tg[u] = make_uint4(kTgtSentinel, kTgtSentinel, kTgtSentinel, kTgtSentinel);
                ww[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                dd[u] = 0;
            }
        }
#pragma unroll
        for (int u = 0; u < (int)kScatterUnroll; ++u) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t tgt = u4_get(tg[u], j);
                if (tgt == kTgtSentinel || !NAER_IN_BOUNDS(ctl, tgt, Ns, kChkRing)) continue;
                float w = f4_get(ww[u], j);
                const uint32_t d = (dd[u] >> (8 * j)) & 0xFFu;
                if (mult != 1.0f) w = __fmul_rn(w, mult);
                ring_add(bt, ring + (size_t)ring_slot(tmod, d, D) * Ns + tgt, w, qs);
                ++ev;
            }
        }
    }
}

// deliver_span for a static source (no plasticity): the deferred rest.
__device__ __forceinline__ void deliver_static_span(const NetDev* np, uint32_t tl, int32_t aux0, uint64_t lo,
                                                    uint64_t hi, uint32_t piece, uint32_t split, uint32_t psz,
                                                    uint32_t lane, unsigned long long& ev, Ctl* ctl,
                                                    const BinTable& bt) {
    const uint32_t D = np->ring_slots;
    const uint32_t tmod = tl % D;
    const uint32_t Ns = np->n_storage;
    float* __restrict__ ring = np->ring;
    const float qs = np->fx_scale;  // exact-sum aggregation: 2^S, else 0
    const uint32_t* __restrict__ tgt_a = np->tgt;
    const float* __restrict__ w_a = np->w;
    const uint8_t* __restrict__ d_a = np->dly;
    const float mult = aux0 > 1 ? (float)aux0 : 1.0f;
    for (uint64_t base = lo + (uint64_t)piece * psz; base < hi; base += (uint64_t)split * psz) {
        uint4 tg[kScatterUnroll];
        float4 ww[kScatterUnroll];
        uint32_t dd[kScatterUnroll];
#pragma unroll
        for (int u = 0; u < (int)kScatterUnroll; ++u) {
            const uint64_t off = base + (uint64_t)(u * 32 + lane) * 4ull;
            if (off < hi && (uint32_t)u * 128u < psz && NAER_IN_BOUNDS(ctl, off + 3, np->syn_cap, kChkSynapse)) {
                tg[u] = ld_stream_u4(tgt_a + off);
                ww[u] = __ldcs(reinterpret_cast<const float4*>(w_a + off));
                dd[u] = ld_stream_u32(d_a + off);
            } else {
                tg[u] = make_uint4(kTgtSentinel, kTgtSentinel, kTgtSentinel, kTgtSentinel);
                ww[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                dd[u] = 0;
            }
        }
#pragma unroll
        for (int u = 0; u < (int)kScatterUnroll; ++u) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t tgt = u4_get(tg[u], j);
                if (tgt == kTgtSentinel || !NAER_IN_BOUNDS(ctl, tgt, Ns, kChkRing)) continue;
                float w = f4_get(ww[u], j);
                if (mult != 1.0f) w = __fmul_rn(w, mult);
                ring_add(bt, ring + (size_t)ring_slot(tmod, (dd[u] >> (8 * j)) & 0xFFu, D) * Ns + tgt, w, qs);
                ++ev;
            }
        }
    }
}

// LIF of one owned chunk with its state in shared memory (the arithmetic of
// lif_chunk); returns the spike flags of the thread's four neurons (bit k =
// neuron first + 4 * thread + k).  Post-spike plasticity bookkeeping is left
// to the record writer.
__device__ __forceinline__ uint32_t lif_flags_smem(const ChunkCache& cc, uint32_t j, unsigned long long s,
                                                   float4* sV, uchar4* sR, const float4 I, const uint32_t Dw) {
    if (!cc.active || s < cc.start || s >= cc.stop) return 0u;
    const uint32_t i0 = cc.first + threadIdx.x * kLifPerThread;
    if (i0 >= cc.end) return 0u;
    uint32_t f = 0;
    if (cc.p.type == kPOISSON) {
        if (cc.p.rate_hz > 0.0) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (i0 + k < cc.end && ((Dw >> (8 * k)) & 0xFFu)) f |= 1u << k;
        }
        return f;
    }
    const uint32_t si = j * kLifThreads + threadIdx.x;
    const float4 V4 = sV[si];
    const uchar4 R4 = sR[si];
    float vv[4] = {V4.x, V4.y, V4.z, V4.w};
    uint32_t rr[4] = {R4.x, R4.y, R4.z, R4.w};
    const double prop = cc.p.prop;
    const float v_th = cc.p.v_th, v_reset = cc.p.v_reset, dw = cc.p.drive_w, fx_inv = cc.fx_inv;
    const uint32_t tref = cc.p.t_ref_steps, end = cc.end;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (i0 + k >= end) continue;
        if (rr[k] > 0) {
            rr[k] -= 1;
            continue;
        }
        float v = lif_update(vv[k], prop, ring_input(f4_get(I, k), fx_inv), (Dw >> (8 * k)) & 0xFFu, dw);
        if (v > v_th) {
            v = v_reset;
            rr[k] = tref;
            f |= 1u << k;
        }
        vv[k] = v;
    }
    sV[si] = make_float4(vv[0], vv[1], vv[2], vv[3]);
    sR[si] = make_uchar4((unsigned char)rr[0], (unsigned char)rr[1], (unsigned char)rr[2], (unsigned char)rr[3]);
    return f;
}

// Reserves places for the warp's spikes (cnt per lane) in the step's list:
// one atomic per warp.  Returns the lane's first place.
__device__ __forceinline__ uint32_t reserve_places(Ctl* ctl, unsigned long long s, uint32_t cnt, uint32_t lane) {
    uint32_t x = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, x, 31);
    uint32_t base = 0;
    if (total) {
        if (lane == 31) base = atomicAdd(&ctl->qtail[s & 3ull], total);
        base = __shfl_sync(0xFFFFFFFFu, base, 31);
    }
    return base + x - cnt;
}

// Writes one spike record: POISSON sources carry their multiplicity,
// plastic neurons run their post-spike bookkeeping here.
// Row of a spiking neuron: {begin lo, begin hi, delay-1 part length, row
// length}, read once at LIF time so that the scatter's first load already
// names the synapses.
__device__ __forceinline__ uint4 row_of(const uint64_t* row_ptr, const uint32_t* row_mid, uint32_t i) {
    const unsigned long long b = __ldg(reinterpret_cast<const unsigned long long*>(row_ptr) + i);
    const unsigned long long e = __ldg(reinterpret_cast<const unsigned long long*>(row_ptr) + i + 1);
    const uint32_t m = __ldg(row_mid + i);
    return make_uint4((uint32_t)b, (uint32_t)(b >> 32), m, (uint32_t)(e - b));
}

__device__ __forceinline__ void write_spike(const EngineDev& eng, SpikeRec* __restrict__ queue,
                                            uint32_t* __restrict__ qid, uint32_t pos, uint32_t net, uint32_t i,
                                            const PopDev& p, bool plastic, uint32_t tl, uint32_t count,
                                            const uint4 row) {
    int32_t aux0 = 0;
    float aux1 = 0.0f;
    if (p.type == kPOISSON) aux0 = (int32_t)count;
    else if (plastic) stdp_post_spike(eng.nets + net, i, (int32_t)tl, aux0, aux1);
    if (pos < eng.queue_cap) {
        const uint32_t qb = (uint32_t)(queue == eng.queue[1]);
        __stcg(reinterpret_cast<int4*>(queue + pos), make_int4((int)net, (int)i, aux0, __float_as_int(aux1)));
        __stcg(qid + pos, p.id_base + (i - p.storage_base));
        __stcg(eng.qrow[qb] + pos, row);
    } else {
        atomicCAS(&eng.ctl->error, 0u, (unsigned int)(-NAER_STATUS_OVERFLOW));
    }
}

// Polls a grid barrier from warp 0, lane 0 (warp 0 does nothing else until
// it completes) and raises *flag for the block's other warps when it does.
__device__ __forceinline__ void poll_barrier(Ctl* ctl, unsigned long long target, const BarrierCfg& cfg,
                                             volatile int* flag, int* ok) {
    const unsigned long long t0 = globaltimer_ns();
    const unsigned long long goal = target + cfg.skew;
    unsigned long long cur;
    for (;;) {
        asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(cur) : "l"(&ctl->bar_arrive) : "memory");
        if (cur >= goal) break;
        if (globaltimer_ns() - t0 > cfg.limit_ns) {
            atomicCAS(&ctl->error, 0u, (unsigned int)(-NAER_STATUS_TIMEOUT));
            *ok = 0;
            break;
        }
        __nanosleep(32);
    }
    *flag = 1;
}

__device__ __forceinline__ void arrive_barrier(Ctl* ctl) {
    __threadfence();  // the block's stores and reductions (ordered by the preceding __syncthreads)
    asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(&ctl->bar_arrive) : "memory");
}

// Deferred ("rest") scatter work of one step: the step, its list's buffer
// and its item count are the same for the whole block (shared memory); each
// warp walks items it, it + WR, ... (it in a register).
struct RestWork {
    unsigned long long step;
    uint32_t n, qb;
};

__device__ __forceinline__ void rest_item(const EngineDev& eng, const RestWork& rw, uint32_t it, const NetDev* net0,
                                          uint32_t lane, unsigned long long& ev, const BinTable& bt) {
    const uint32_t split = eng.split_rest;
    const uint32_t e = it / split;
    const uint32_t piece = it - e * split;
    const int4 rv = __ldcg(reinterpret_cast<const int4*>(eng.queue[rw.qb] + e));
    const uint4 row = __ldcg(eng.qrow[rw.qb] + e);  // issued with the record: no dependent row lookup
    const uint32_t net = (uint32_t)rv.x, src = (uint32_t)rv.y;
    const NetDev* np = net == 0 ? net0 : eng.nets + net;
    if (np->stdp_on && src < np->n_plastic) return;  // plastic rows went whole with the first part
    const uint64_t beg = ((uint64_t)row.y << 32) | row.x;
    deliver_static_span(np, (uint32_t)(rw.step - np->start_step), rv.z, beg + row.z, beg + row.w, piece, split,
                        eng.scatter_piece, lane, ev, eng.ctl, bt);
}

// One first-part item of k_step (piece `piece` of spike e's due part: the
// delay-1 synapses of a static source, the whole row of a plastic one);
// the piece-0 warp appends the spike to the raster at rbase + e.
// (rv, row: spike e's record and row, already loaded)
__device__ __forceinline__ void first_item(const EngineDev& eng, const int4 rv, const uint4 row,
                                           const uint32_t* __restrict__ qid, uint32_t e,
                                           uint32_t piece, uint32_t split, unsigned long long s,
                                           unsigned long long rbase, const NetDev* net0, uint32_t lane,
                                           unsigned long long& ev, uint32_t& ovf, const BinTable& bt) {
    SpikeRec r;
    r.net = (uint32_t)rv.x;
    r.src = (uint32_t)rv.y;
    r.aux0 = rv.z;
    r.aux1 = __int_as_float(rv.w);
    if (piece == 0 && lane == 0 && eng.record && rbase + e < eng.raster_cap)
        __stcg(eng.raster + rbase + e, make_uint2((uint32_t)s, __ldcg(qid + e)));
    const NetDev* np = (r.net == 0) ? net0 : eng.nets + r.net;
    if (!NAER_IN_BOUNDS(eng.ctl, r.src, np->n_storage, kChkQueue)) return;
    const uint64_t beg = ((uint64_t)row.y << 32) | row.x;
    const bool plastic_src = np->stdp_on && r.src < np->n_plastic;
    const uint64_t hi = beg + (plastic_src ? row.w : row.z);
    deliver_span(np, (uint32_t)(s - np->start_step), r, beg, hi, piece, split, eng.scatter_piece, lane, ev, ovf,
                 eng.ctl, bt);
}

// Chunk descriptors, membrane potentials and refractory counters of the
// block's owned chunks into shared memory (start of a persistent launch) and
// back (end of it).
__device__ __forceinline__ void load_chunk_state(const EngineDev& eng, uint32_t own, ChunkCache* s_cc, float4* sV,
                                                 uchar4* sR) {
    const uint32_t G = gridDim.x;
    for (uint32_t j = threadIdx.x; j < own; j += blockDim.x) {
        const ChunkDev ch = eng.chunks[blockIdx.x + j * G];
        const NetDev* np = eng.nets + ch.net;
        ChunkCache c;
        c.p = eng.pops[ch.pop];
        c.row_ptr = np->row_ptr;
        c.row_mid = np->row_mid;
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
        c.fx_inv = np->fx_inv;
        s_cc[j] = c;
    }
    __syncthreads();
    for (uint32_t j = 0; j < own; ++j) {
        const uint32_t i0 = s_cc[j].first + threadIdx.x * kLifPerThread;
        // a chunk lies inside its net's state arrays (checked once per launch:
        // every later access of the chunk stays within [first, end))
        if (i0 < s_cc[j].end && NAER_IN_BOUNDS(eng.ctl, s_cc[j].end, (uint64_t)s_cc[j].Ns + 1, kChkState)) {
            const uint32_t si = j * kLifThreads + threadIdx.x;
            sV[si] = *reinterpret_cast<const float4*>(s_cc[j].v + i0);
            sR[si] = *reinterpret_cast<const uchar4*>(s_cc[j].refr + i0);
        }
    }
}

__device__ __forceinline__ void store_chunk_state(uint32_t own, const ChunkCache* s_cc, const float4* sV,
                                                  const uchar4* sR) {
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

// Per-thread event and history-overflow counts into the block's counters
// (no same-address global atomics on the hot path).
__device__ __forceinline__ void finish_counters(const EngineDev& eng, unsigned long long ev, uint32_t ovf,
                                                uint32_t lane, unsigned long long* s_ev, uint32_t* s_ovf) {
    ev = warp_sum_u64(ev);
    const unsigned long long ov = warp_sum_u64((unsigned long long)ovf);
    if (lane == 0) {
        if (ev) atomicAdd(s_ev, ev);
        if (ov) atomicAdd(s_ovf, (uint32_t)ov);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (*s_ev) eng.ev_part[blockIdx.x] += *s_ev;
        if (*s_ovf) eng.ovf_part[blockIdx.x] += *s_ovf;
    }
}

// LIF phase of a persistent step kernel: the block's chunks (state in shared
// memory with kSmem), spikes appended to the step's list (one reservation
// per warp and batch of chunks).
template <bool kSmem>
__device__ __forceinline__ void lif_phase(const EngineDev& eng, unsigned long long s, uint32_t own,
                                          const ChunkCache* s_cc, float4* sV, uchar4* sR,
                                          SpikeRec* __restrict__ queue, uint32_t* __restrict__ qid,
                                          uint32_t lane) {
    const uint32_t G = gridDim.x;
    Ctl* ctl = eng.ctl;
    if (kSmem) {
        for (uint32_t j0 = 0; j0 < own; j0 += kLifBatch) {
            float4 I[kLifBatch];
            uint32_t Dw[kLifBatch];
#pragma unroll
            for (uint32_t b = 0; b < kLifBatch; ++b)
                if (j0 + b < own) lif_prefetch(s_cc[j0 + b], s, I[b], Dw[b]);
#pragma unroll
            for (uint32_t b = 0; b < kLifBatch; ++b)
                if (j0 + b < own) lif_clear(s_cc[j0 + b], s);
            uint32_t mask = 0;
#pragma unroll
            for (uint32_t b = 0; b < kLifBatch; ++b)
                if (j0 + b < own) mask |= lif_flags_smem(s_cc[j0 + b], j0 + b, s, sV, sR, I[b], Dw[b]) << (4 * b);
            if (__any_sync(0xFFFFFFFFu, mask != 0)) {
                // the row of the lane's first spike is loaded while the
                // reservation's atomic is in flight (most lanes have one)
                uint4 row0 = make_uint4(0, 0, 0, 0);
                if (mask) {
                    const uint32_t bit = __ffs(mask) - 1u;
                    const ChunkCache& cc = s_cc[j0 + (bit >> 2)];
                    row0 = row_of(cc.row_ptr, cc.row_mid, cc.first + threadIdx.x * kLifPerThread + (bit & 3u));
                }
                uint32_t pos = reserve_places(ctl, s, __popc(mask), lane);
                bool first = true;
#pragma unroll
                for (uint32_t b = 0; b < kLifBatch; ++b) {
                    const uint32_t m4 = (mask >> (4 * b)) & 0xFu;
                    if (!m4) continue;
                    const ChunkCache& cc = s_cc[j0 + b];
                    const uint32_t i0 = cc.first + threadIdx.x * kLifPerThread;
                    const uint32_t tl = (uint32_t)(s - cc.start);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if ((m4 >> q) & 1u) {
                            const uint4 row = first ? row0 : row_of(cc.row_ptr, cc.row_mid, i0 + q);
                            first = false;
                            write_spike(eng, queue, qid, pos++, cc.net, i0 + q, cc.p, cc.plastic != 0, tl,
                                        (Dw[b] >> (8 * q)) & 0xFFu, row);
                        }
                }
            }
        }
    } else {
        for (uint32_t c = blockIdx.x; c < eng.n_chunks; c += G) {
            const ChunkDev ch = eng.chunks[c];
            const PopDev p = eng.pops[ch.pop];
            const NetDev* np = eng.nets + ch.net;
            const unsigned long long start = np->start_step;
            if (!np->active || s < start || s >= np->end_step) continue;  // uniform over the block
            const uint32_t tl = (uint32_t)(s - start);
            const uint32_t i0 = ch.first + threadIdx.x * kLifPerThread;
            uint32_t Dw = 0;
            uint32_t f = 0;
            if (i0 < ch.end) {
                const uint8_t* drive_slot = np->drive + (size_t)(s % kDriveSlots) * np->n_storage;
                if (p.rate_hz > 0.0) Dw = __ldcg(reinterpret_cast<const unsigned int*>(drive_slot + i0));
                if (p.type == kPOISSON) {
                    if (p.rate_hz > 0.0) {
#pragma unroll
                        for (int q = 0; q < 4; ++q)
                            if (i0 + q < ch.end && ((Dw >> (8 * q)) & 0xFFu)) f |= 1u << q;
                    }
                } else {
                    const uint32_t Ns = np->n_storage;
                    float4* ring4 = reinterpret_cast<float4*>(np->ring + (size_t)(tl % np->ring_slots) * Ns) +
                                    (i0 >> 2);
                    float4* v4 = reinterpret_cast<float4*>(np->v) + (i0 >> 2);
                    uchar4* r4 = reinterpret_cast<uchar4*>(np->refr) + (i0 >> 2);
                    const float4 Iv = __ldcg(ring4);
                    const float4 V4 = *v4;
                    const uchar4 R4 = *r4;
                    __stcg(ring4, make_float4(0.f, 0.f, 0.f, 0.f));
                    float vv[4] = {V4.x, V4.y, V4.z, V4.w};
                    uint32_t rr[4] = {R4.x, R4.y, R4.z, R4.w};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (i0 + q >= ch.end) continue;
                        if (rr[q] > 0) {
                            rr[q] -= 1;
                            continue;
                        }
                        float v = lif_update(vv[q], p.prop, ring_input(f4_get(Iv, q), np->fx_inv), (Dw >> (8 * q)) & 0xFFu,
                                             p.drive_w);
                        if (v > p.v_th) {
                            v = p.v_reset;
                            rr[q] = p.t_ref_steps;
                            f |= 1u << q;
                        }
                        vv[q] = v;
                    }
                    *v4 = make_float4(vv[0], vv[1], vv[2], vv[3]);
                    *r4 = make_uchar4((unsigned char)rr[0], (unsigned char)rr[1], (unsigned char)rr[2],
                                      (unsigned char)rr[3]);
                }
            }
            if (__any_sync(0xFFFFFFFFu, f != 0)) {
                uint32_t pos = reserve_places(ctl, s, __popc(f), lane);
                const bool plastic = p.type == kSTDP && np->stdp_on;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if ((f >> q) & 1u)
                        write_spike(eng, queue, qid, pos++, ch.net, i0 + q, p, plastic, tl, (Dw >> (8 * q)) & 0xFFu,
                                    row_of(np->row_ptr, np->row_mid, i0 + q));
            }
        }
    }
}

template <bool kSmem>
__global__ void __launch_bounds__(kLifThreads, NAER_RUN_MIN_BLOCKS)
    k_step(EngineDev eng, unsigned long long s0, uint32_t nsteps) {
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ unsigned long long s_ev;
    __shared__ uint32_t s_ovf;
    __shared__ NetDev s_net0;  // descriptor of the first net (the only one in the plain form)
    __shared__ BarrierCfg bcfg;
    __shared__ int s_flag, s_ok;
    __shared__ RestWork s_rw[2];                     // deferred work of steps by parity
    __shared__ uint32_t s_q;                         // size of the step's list
    __shared__ unsigned long long s_ph[5], s_dropped;  // thread 0 only
    __shared__ unsigned long long s_bar_target;      // thread 0 only
    const uint32_t G = gridDim.x;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t nw_block = kLifThreads / 32;
    // the whole grid's warps (first part) and the warps 1.. of every block (rest)
    const uint32_t gw = blockIdx.x * nw_block + wib, W = G * nw_block;
    // (warp 0 has no deferred items: gr is unused there)
    const uint32_t gr = blockIdx.x * (nw_block - 1) + (wib - 1), WR = G * (nw_block - 1);
    Ctl* ctl = eng.ctl;
    if (threadIdx.x == 0) {
        s_net0 = eng.nets[0];
        bcfg = barrier_cfg(ctl);
        s_ev = 0;
        s_ovf = 0;
        s_ok = 1;
        s_flag = 0;
        s_rw[0] = RestWork{0, 0, 0};  // nothing deferred at launch start
        s_rw[1] = RestWork{0, 0, 0};
        s_q = 0;
        for (int q = 0; q < 5; ++q) s_ph[q] = 0;
        s_dropped = 0;
        s_bar_target = 0;
    }
    const uint32_t own_max = eng.region_cap / kLifChunk;
    BinTable bt;
    bt.key = reinterpret_cast<unsigned long long*>(s_dyn + 16);
    bt.sum = reinterpret_cast<float*>(bt.key + eng.bins);
    bt.mask = eng.bins ? eng.bins - 1 : 0u;
    for (uint32_t i = threadIdx.x; i < eng.bins; i += blockDim.x) {
        bt.key[i] = 0ull;
        bt.sum[i] = 0.0f;
    }
    const size_t off_cc = step_smem_offset(eng.bins);
    ChunkCache* s_cc = reinterpret_cast<ChunkCache*>(s_dyn + off_cc);
    const size_t off_v = off_cc + (((size_t)own_max * sizeof(ChunkCache) + 15) & ~(size_t)15);
    float4* sV = reinterpret_cast<float4*>(s_dyn + off_v);
    uchar4* sR = reinterpret_cast<uchar4*>(s_dyn + off_v + (size_t)own_max * kLifThreads * sizeof(float4));
    const uint32_t own = blockIdx.x < eng.n_chunks ? (eng.n_chunks - blockIdx.x + G - 1) / G : 0u;

    if (s0 == kStepFromCtl) s0 = ctl->step;
    unsigned long long rbase = ctl->raster_next;
    unsigned long long ev = 0;
    uint32_t ovf = 0;
    const bool timer = blockIdx.x == 0 && threadIdx.x == 0;
    uint32_t rit = 0;  // this warp's next deferred item
    if (kSmem) load_chunk_state(eng, own, s_cc, sV, sR);
    __syncthreads();
    uint32_t k = 0;
    for (; k < nsteps; ++k) {
        const unsigned long long s = s0 + k;
        const uint32_t qb = (uint32_t)(s & 1ull);
        const unsigned long long ta = timer ? globaltimer_ns() : 0ull;
        SpikeRec* queue = eng.queue[qb];
        uint32_t* qid = eng.qid[qb];
        // ---- 1. LIF
        lif_phase<kSmem>(eng, s, own, s_cc, sV, sR, queue, qid, lane);
        __syncthreads();
        const unsigned long long ta2 = timer ? globaltimer_ns() : 0ull;
        // ---- 2. B1: the step's list is complete; warps 1.. work off step s-1's rest meanwhile
        const RestWork& rw_prev = s_rw[(s + 1) & 1ull];  // step s-1
        if (threadIdx.x == 0) {
            s_bar_target += G;
            arrive_barrier(ctl);
        }
        if (wib == 0) {
            if (lane == 0) {
                poll_barrier(ctl, s_bar_target, bcfg, &s_flag, &s_ok);
                // the list of step s is complete: its rest becomes the next deferred work
                const uint32_t Q = __ldcg(&ctl->qtail[s & 3ull]);
                s_rw[s & 1ull] = RestWork{s, Q * eng.split_rest, qb};
                s_q = Q;
            }
            __syncwarp();
        } else {
            while (rit < rw_prev.n) {
                if (*(volatile int*)&s_flag) break;
                rest_item(eng, rw_prev, rit, &s_net0, lane, ev, bt);
                rit += WR;
            }
        }
        __syncthreads();
        if (!s_ok) break;
        const unsigned long long tb = timer ? globaltimer_ns() : 0ull;
        // ---- 3. first parts of step s, then the rest of step s-1 that is left
        const uint32_t Q = s_q;
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->qtail[(s + 2) & 3ull] = 0u;  // reused by step s+2
        {
            // this warp's items it = gw, gw + W, ... 32 at a time: lane k
            // loads item k's record and row, and only the items with work in
            // them (piece 0 writes the raster entry) are delivered, so the
            // empty pieces of short parts cost one shared round trip
            const uint32_t split = eng.split_first;
            const uint64_t n1 = (uint64_t)Q * split;
            for (uint64_t it0 = gw; it0 < n1; it0 += 32ull * W) {
                const uint64_t it = it0 + (uint64_t)lane * W;
                int4 rv = make_int4(0, 0, 0, 0);
                uint4 row = make_uint4(0, 0, 0, 0);
                uint32_t e = 0, piece = 0;
                bool work = false;
                if (it < n1) {
                    e = (uint32_t)(it / split);
                    piece = (uint32_t)(it - (uint64_t)e * split);
                    rv = __ldcg(reinterpret_cast<const int4*>(queue + e));
                    row = __ldcg(eng.qrow[qb] + e);  // with the record: no dependent row lookup
                    const NetDev* np = rv.x == 0 ? &s_net0 : eng.nets + rv.x;
                    const bool plastic_src = np->stdp_on && (uint32_t)rv.y < np->n_plastic;
                    const uint64_t pw = plastic_src ? kPlasticPiece : eng.scatter_piece;
                    work = piece == 0 || (uint64_t)piece * pw < (plastic_src ? row.w : row.z);
                }
                uint32_t m = __ballot_sync(0xFFFFFFFFu, work);
                while (m) {
                    const int L = __ffs(m) - 1;
                    m &= m - 1u;
                    const int4 rvL = make_int4(__shfl_sync(0xFFFFFFFFu, rv.x, L), __shfl_sync(0xFFFFFFFFu, rv.y, L),
                                               __shfl_sync(0xFFFFFFFFu, rv.z, L), __shfl_sync(0xFFFFFFFFu, rv.w, L));
                    const uint4 rowL =
                        make_uint4(__shfl_sync(0xFFFFFFFFu, row.x, L), __shfl_sync(0xFFFFFFFFu, row.y, L),
                                   __shfl_sync(0xFFFFFFFFu, row.z, L), __shfl_sync(0xFFFFFFFFu, row.w, L));
                    first_item(eng, rvL, rowL, qid, __shfl_sync(0xFFFFFFFFu, e, L),
                               __shfl_sync(0xFFFFFFFFu, piece, L), split, s, rbase, &s_net0, lane, ev, ovf, bt);
                }
            }
        }
        if (wib != 0) {
            for (; rit < rw_prev.n; rit += WR) rest_item(eng, rw_prev, rit, &s_net0, lane, ev, bt);
        }
        {
            const unsigned long long cap = eng.record ? eng.raster_cap : 0ull;
            const unsigned long long kept = rbase + Q <= cap ? Q : (rbase >= cap ? 0ull : cap - rbase);
            if (eng.record && threadIdx.x == 0) s_dropped += Q - kept;
            rbase += kept;
        }
        flush_bins(bt);  // everything binned since the last barrier, before this block's arrival
        __syncthreads();
        const unsigned long long tb2 = timer ? globaltimer_ns() : 0ull;
        // ---- 4. B2: warps 1.. deliver step s's rest while warp 0 waits for
        // it.  (Starting that work as soon as a warp's due deliveries are
        // done was measured slower: the bulk reductions then contend in L2
        // with the delay-1 ones the barrier waits for.)
        if (threadIdx.x == 0) {
            s_flag = 0;
            s_bar_target += G;
            arrive_barrier(ctl);
        }
        rit = gr;
        __syncthreads();
        if (wib == 0) {
            if (lane == 0) poll_barrier(ctl, s_bar_target, bcfg, &s_flag, &s_ok);
            __syncwarp();
        } else {
            const RestWork& rw_cur = s_rw[s & 1ull];
            while (rit < rw_cur.n) {
                if (*(volatile int*)&s_flag) break;
                rest_item(eng, rw_cur, rit, &s_net0, lane, ev, bt);
                rit += WR;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_flag = 0;
        if (!s_ok) break;
        if (timer) {
            const unsigned long long tc = globaltimer_ns();
            s_ph[0] += ta2 - ta;
            s_ph[1] += tb - ta2;
            s_ph[2] += tb2 - tb;
            s_ph[4] += tc - tb2;
        }
    }
    // the last step's rest (the next launch's LIF reads it in stream order)
    if (s_ok && wib != 0 && k > 0) {
        const RestWork& rw_last = s_rw[(s0 + k - 1) & 1ull];
        for (; rit < rw_last.n; rit += WR) rest_item(eng, rw_last, rit, &s_net0, lane, ev, bt);
    }
    flush_bins(bt);
    if (kSmem) store_chunk_state(own, s_cc, sV, sR);
    finish_counters(eng, ev, ovf, lane, &s_ev, &s_ovf);
    if (timer) {
        ctl->step = s0 + k;
        ctl->raster_next = rbase;
        ctl->raster_base = rbase;
        ctl->raster_dropped += s_dropped;
        for (int q = 0; q < 5; ++q) ctl->prof_phase_ns[q] += s_ph[q];
        ctl->prof_lif_ns += s_ph[0] + s_ph[1];
        ctl->prof_scatter_ns += s_ph[2] + s_ph[4];
        ctl->prof_steps += k;
    }
}

template __global__ void k_step<true>(EngineDev, unsigned long long, uint32_t);
template __global__ void k_step<false>(EngineDev, unsigned long long, uint32_t);

// ---------------------------------------------------------------------------
// k_det_step: the persistent step kernel with deterministic aggregation.
//
// A source spikes at most once per step, so an event is identified by its
// synapse index j, and the order of a net's synapse array (rows in
// ascending source, each row in its canonical order) is the canonical
// (source, synapse) order.  Per grid step s:
//  1. LIF, spikes appended to the step's list (as k_step);
//  2. grid barrier; every event of the step stores the weight it delivers at
//     ev_w[j] and is linked into its ring cell's list: ev_next[j] =
//     atomicExch(cell_head[cell], j) (STDP updates first, as in the atomic
//     path: they do not depend on the order);
//  3. grid barrier; the event that started a list (ev_next == kNoEvent)
//     takes the head and empties it in one exchange, walks the list, orders
//     its events by j and adds their left fold to the ring cell (one
//     reduction: no other event adds to that cell in this pass);
//  4. grid barrier (the next LIF reads the ring).
// The oracle folds each (step, cell) in the same order, so rings, membrane
// potentials, weights and rasters are bit-identical; no sort, no host
// round trip, no allocation while stepping.
constexpr uint32_t kFoldRegs = 16;  // list length folded from a register copy

__device__ __forceinline__ float fold_cell(const float* __restrict__ ev_w, const uint32_t* __restrict__ ev_next,
                                           uint32_t head) {
    uint32_t buf[kFoldRegs];
    uint32_t n = 0;
    for (uint32_t h = head; h != kNoEvent; h = __ldcg(ev_next + h)) {
        if (n < kFoldRegs) buf[n] = h;
        ++n;
    }
    if (n <= kFoldRegs) {
        for (uint32_t a = 1; a < n; ++a) {  // insertion sort by synapse index
            const uint32_t x = buf[a];
            uint32_t b = a;
            while (b > 0 && buf[b - 1] > x) {
                buf[b] = buf[b - 1];
                --b;
            }
            buf[b] = x;
        }
        float sum = __ldcg(ev_w + buf[0]);
        for (uint32_t a = 1; a < n; ++a) sum = __fadd_rn(sum, __ldcg(ev_w + buf[a]));
        return sum;
    }
    // long list: take its events in ascending j by repeated minimum search
    float sum = 0.0f;
    uint32_t last = 0;
    for (uint32_t a = 0; a < n; ++a) {
        uint32_t best = kNoEvent;
        for (uint32_t h = head; h != kNoEvent; h = __ldcg(ev_next + h))
            if ((a == 0 || h > last) && h < best) best = h;
        const float w = __ldcg(ev_w + best);
        sum = a == 0 ? w : __fadd_rn(sum, w);
        last = best;
    }
    return sum;
}

// Fold of the list whose first event is j (weight wj), started from the
// head hd: every other event's next link and weight are loaded together, and
// the walk stops at j (its link is known to be the end), so a list of two
// costs one round trip.  Same order and result as fold_cell.
__device__ __forceinline__ float fold_from_start(const float* __restrict__ ev_w,
                                                 const uint32_t* __restrict__ ev_next, uint32_t hd, uint32_t j,
                                                 float wj) {
    uint32_t idx[kFoldRegs];
    float wv[kFoldRegs];
    uint32_t n = 0;
    for (uint32_t h = hd; h != j;) {
        if (n + 1 >= kFoldRegs || h == kNoEvent) return fold_cell(ev_w, ev_next, hd);  // long list
        const uint32_t nx = __ldcg(ev_next + h);
        wv[n] = __ldcg(ev_w + h);
        idx[n++] = h;
        h = nx;
    }
    idx[n] = j;
    wv[n++] = wj;
    for (uint32_t a = 1; a < n; ++a) {  // insertion sort by synapse index
        const uint32_t x = idx[a];
        const float y = wv[a];
        uint32_t b = a;
        while (b > 0 && idx[b - 1] > x) {
            idx[b] = idx[b - 1];
            wv[b] = wv[b - 1];
            --b;
        }
        idx[b] = x;
        wv[b] = y;
    }
    float sum = wv[0];
    for (uint32_t a = 1; a < n; ++a) sum = __fadd_rn(sum, wv[a]);
    return sum;
}

// Deterministic path over the pieces of a static source's row, kDetBatch
// synapses per lane at a time (out of line, so that it has its own register
// budget): every load of a batch is issued before any result is used, the
// batch's list exchanges are issued back to back (their results are only
// stored), and a list of one event (the usual case) is folded from the
// weight loaded with its head, so a batch costs two or three dependent
// round trips instead of that many per synapse.  Same results as the
// per-synapse loop of det_item.
constexpr uint32_t kDetBatch = 4;

__device__ __noinline__ uint32_t det_static_span(const NetDev* np, uint64_t row_lo, uint64_t row_hi, uint32_t piece,
                                                 uint32_t split, uint32_t psz, uint32_t tmod, float mult,
                                                 uint32_t lane, int pass, Ctl* ctl) {
    uint32_t ev = 0;  // events linked (pass 0)
    const uint32_t* __restrict__ tgt_a = np->tgt;
    const uint8_t* __restrict__ d_a = np->dly;
    const float* __restrict__ w_a = np->w;
    float* __restrict__ ev_w = np->ev_w;
    uint32_t* __restrict__ ev_next = np->ev_next;
    uint32_t* __restrict__ head = np->cell_head;
    float* __restrict__ ring = np->ring;
    const uint32_t D = np->ring_slots, Ns = np->n_storage;
    constexpr uint32_t kSpan = 32 * kDetBatch;  // synapses of one batch of the warp
    for (uint64_t base = row_lo + (uint64_t)piece * psz; base < row_hi; base += (uint64_t)split * psz) {
        const uint64_t top = row_hi < base + psz ? row_hi : base + psz;
        for (uint64_t b0 = base; b0 < top; b0 += kSpan) {
            uint32_t cell[kDetBatch];
            uint32_t aux[kDetBatch];  // pass 0: weight bits; pass 1: next event
            uint8_t dl[kDetBatch];
#pragma unroll
            for (uint32_t u = 0; u < kDetBatch; ++u) {
                const uint64_t j = b0 + lane + 32u * u;
                cell[u] = kTgtSentinel;
                if (j < top && NAER_IN_BOUNDS(ctl, j, np->syn_cap, kChkEventList)) {
                    // the linking pass leaves the step's synapses in L2 for the
                    // folding pass, which reads them for the last time
                    if (pass == 0) {
                        cell[u] = __ldcg(tgt_a + j);
                        dl[u] = __ldcg(d_a + j);
                        aux[u] = __float_as_uint(__ldcs(w_a + j));
                    } else {
                        cell[u] = __ldcs(tgt_a + j);
                        dl[u] = __ldcs(d_a + j);
                        aux[u] = __ldcs(ev_next + j);
                    }
                }
            }
#pragma unroll
            for (uint32_t u = 0; u < kDetBatch; ++u)
                if (cell[u] != kTgtSentinel) {
                    cell[u] = NAER_IN_BOUNDS(ctl, cell[u], Ns, kChkRing) ? ring_slot(tmod, dl[u], D) * Ns + cell[u]
                                                                       : kTgtSentinel;
                }
            if (pass == 0) {
                uint32_t old[kDetBatch];
#pragma unroll
                for (uint32_t u = 0; u < kDetBatch; ++u)
                    if (cell[u] != kTgtSentinel) {
                        const uint32_t j = (uint32_t)(b0 + lane + 32u * u);
                        float w = __uint_as_float(aux[u]);
                        if (mult != 1.0f) w = __fmul_rn(w, mult);
                        __stcg(ev_w + j, w);
                        old[u] = atomicExch(head + cell[u], j);
                    }
#pragma unroll
                for (uint32_t u = 0; u < kDetBatch; ++u)
                    if (cell[u] != kTgtSentinel) {
                        __stcg(ev_next + (b0 + lane + 32u * u), old[u]);
                        ++ev;
                    }
            } else {
                // the event that started its cell's list (next == none) takes
                // the head and empties it in one exchange, folds the list and
                // adds the fold to the cell: the only addition to that cell in
                // this pass, so a reduction gives the value a load, add and
                // store would
                uint32_t hd[kDetBatch];
                float wj[kDetBatch];
#pragma unroll
                for (uint32_t u = 0; u < kDetBatch; ++u)
                    if (cell[u] != kTgtSentinel && aux[u] == kNoEvent) {
                        hd[u] = atomicExch(head + cell[u], kNoEvent);
                        wj[u] = __ldcs(ev_w + (b0 + lane + 32u * u));
                    }
#pragma unroll
                for (uint32_t u = 0; u < kDetBatch; ++u)
                    if (cell[u] != kTgtSentinel && aux[u] == kNoEvent) {
                        const uint32_t j = (uint32_t)(b0 + lane + 32u * u);
                        // head == j: the list holds this event alone
                        const float sum = hd[u] == j ? wj[u] : fold_from_start(ev_w, ev_next, hd[u], j, wj[u]);
                        red_add_f32(ring + cell[u], sum);
                    }
            }
        }
    }
    return ev;
}

// One (spike, piece) item of the deterministic path: pass 0 links events,
// pass 1 folds the lists whose first event lies in the item.
__device__ __forceinline__ void det_item(const EngineDev& eng, const SpikeRec* __restrict__ queue, uint32_t e,
                                         uint32_t piece, uint32_t split, uint32_t psz, unsigned long long s,
                                         const NetDev* net0, uint32_t lane, int pass, unsigned long long& ev,
                                         uint32_t& ovf) {
    const int4 rv = __ldcg(reinterpret_cast<const int4*>(queue + e));
    SpikeRec r;
    r.net = (uint32_t)rv.x;
    r.src = (uint32_t)rv.y;
    r.aux0 = rv.z;
    r.aux1 = __int_as_float(rv.w);
    const NetDev* np = r.net == 0 ? net0 : eng.nets + r.net;
    const uint32_t tl = (uint32_t)(s - np->start_step);
    const uint32_t D = np->ring_slots, tmod = tl % D, Ns = np->n_storage;
    const uint4 row = __ldcg(eng.qrow[(uint32_t)(queue == eng.queue[1])] + e);
    const uint64_t row_beg = ((uint64_t)row.y << 32) | row.x;
    const ulonglong2 rb = make_ulonglong2(row_beg, row_beg + row.w);
    const uint32_t* __restrict__ tgt_a = np->tgt;
    const uint8_t* __restrict__ d_a = np->dly;
    float* __restrict__ w_a = np->w;
    float* __restrict__ ev_w = np->ev_w;
    uint32_t* __restrict__ ev_next = np->ev_next;
    uint32_t* __restrict__ head = np->cell_head;
    const bool plastic_src = np->stdp_on && r.src < np->n_plastic;
    const uint32_t n_plastic = np->n_plastic;
    StdpView sv;
    if (pass == 0 && plastic_src) sv = stdp_view(*np);
    const float mult = (!plastic_src && r.aux0 > 1) ? (float)r.aux0 : 1.0f;
    if (!plastic_src) {
        ev += det_static_span(np, rb.x, rb.y, piece, split, psz, tmod, mult, lane, pass, eng.ctl);
        return;
    }
    for (uint64_t base = rb.x + (uint64_t)piece * psz; base < rb.y; base += (uint64_t)split * psz) {
        const uint64_t top = rb.y < base + psz ? rb.y : base + psz;
        for (uint64_t j = base + lane; j < top; j += 32) {
            if (!NAER_IN_BOUNDS(eng.ctl, j, np->syn_cap, kChkEventList)) continue;
            const uint32_t tgt = __ldcg(tgt_a + j);
            if (tgt == kTgtSentinel || !NAER_IN_BOUNDS(eng.ctl, tgt, Ns, kChkRing)) continue;
            const uint32_t cell = ring_slot(tmod, __ldcg(d_a + j), D) * Ns + tgt;
            if (pass == 0) {
                float w = __ldcg(w_a + j);
                if (plastic_src && tgt < n_plastic) {
                    w = stdp_update(sv, w, tgt, (int32_t)tl, r.aux0, r.aux1, ovf);
                    __stcg(w_a + j, w);
                }
                if (mult != 1.0f) w = __fmul_rn(w, mult);
                __stcg(ev_w + j, w);
                __stcg(ev_next + j, atomicExch(head + cell, (uint32_t)j));
                ++ev;
            } else if (__ldcg(ev_next + j) == kNoEvent) {
                // as in det_static_span: take and empty the head, add the fold
                red_add_f32(np->ring + cell, fold_cell(ev_w, ev_next, atomicExch(head + cell, kNoEvent)));
            }
        }
    }
}

template <bool kSmem>
__global__ void __launch_bounds__(kLifThreads, NAER_RUN_MIN_BLOCKS)
    k_det_step(EngineDev eng, unsigned long long s0, uint32_t nsteps) {
    extern __shared__ __align__(16) unsigned char s_dyn[];
    __shared__ unsigned long long s_ev;
    __shared__ uint32_t s_ovf;
    __shared__ NetDev s_net0;
    __shared__ BarrierCfg bcfg;
    __shared__ unsigned long long s_ph[5], s_dropped, s_bar_target;  // thread 0 only
    const uint32_t G = gridDim.x;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t gw = blockIdx.x * (kLifThreads / 32) + wib, W = G * (kLifThreads / 32);
    Ctl* ctl = eng.ctl;
    if (threadIdx.x == 0) {
        s_net0 = eng.nets[0];
        bcfg = barrier_cfg(ctl);
        s_ev = 0;
        s_ovf = 0;
        for (int q = 0; q < 5; ++q) s_ph[q] = 0;
        s_dropped = 0;
        s_bar_target = 0;
    }
    const uint32_t own_max = eng.region_cap / kLifChunk;
    const size_t off_cc = 16;
    ChunkCache* s_cc = reinterpret_cast<ChunkCache*>(s_dyn + off_cc);
    const size_t off_v = off_cc + (((size_t)own_max * sizeof(ChunkCache) + 15) & ~(size_t)15);
    float4* sV = reinterpret_cast<float4*>(s_dyn + off_v);
    uchar4* sR = reinterpret_cast<uchar4*>(s_dyn + off_v + (size_t)own_max * kLifThreads * sizeof(float4));
    const uint32_t own = blockIdx.x < eng.n_chunks ? (eng.n_chunks - blockIdx.x + G - 1) / G : 0u;
    if (s0 == kStepFromCtl) s0 = ctl->step;
    unsigned long long rbase = ctl->raster_next;
    unsigned long long ev = 0;
    uint32_t ovf = 0;
    const bool timer = blockIdx.x == 0 && threadIdx.x == 0;
    if (kSmem) load_chunk_state(eng, own, s_cc, sV, sR);
    __syncthreads();
    const uint32_t split = eng.scatter_split, psz = eng.scatter_piece;
    uint32_t k = 0;
    for (; k < nsteps; ++k) {
        const unsigned long long s = s0 + k;
        const uint32_t qb = (uint32_t)(s & 1ull);
        const unsigned long long ta = timer ? globaltimer_ns() : 0ull;
        SpikeRec* queue = eng.queue[qb];
        uint32_t* qid = eng.qid[qb];
        lif_phase<kSmem>(eng, s, own, s_cc, sV, sR, queue, qid, lane);
        if (threadIdx.x == 0) s_bar_target += G;
        if (!grid_barrier(ctl, s_bar_target, bcfg)) break;
        const unsigned long long tb = timer ? globaltimer_ns() : 0ull;
        const uint32_t Q = __ldcg(&ctl->qtail[s & 3ull]);
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->qtail[(s + 2) & 3ull] = 0u;  // reused by step s+2
        const uint64_t n = (uint64_t)Q * split;
        for (uint64_t it = gw; it < n; it += W) {
            const uint32_t e = (uint32_t)(it / split);
            const uint32_t piece = (uint32_t)(it - (uint64_t)e * split);
            if (piece == 0 && lane == 0 && eng.record && rbase + e < eng.raster_cap)
                __stcg(eng.raster + rbase + e, make_uint2((uint32_t)s, __ldcg(qid + e)));
            det_item(eng, queue, e, piece, split, psz, s, &s_net0, lane, 0, ev, ovf);
        }
        if (threadIdx.x == 0) s_bar_target += G;
        if (!grid_barrier(ctl, s_bar_target, bcfg)) break;
        const unsigned long long tb2 = timer ? globaltimer_ns() : 0ull;
        for (uint64_t it = gw; it < n; it += W) {
            const uint32_t e = (uint32_t)(it / split);
            det_item(eng, queue, e, (uint32_t)(it - (uint64_t)e * split), split, psz, s, &s_net0, lane, 1, ev, ovf);
        }
        {
            const unsigned long long cap = eng.record ? eng.raster_cap : 0ull;
            const unsigned long long kept = rbase + Q <= cap ? Q : (rbase >= cap ? 0ull : cap - rbase);
            if (eng.record && threadIdx.x == 0) s_dropped += Q - kept;
            rbase += kept;
        }
        if (threadIdx.x == 0) s_bar_target += G;
        if (!grid_barrier(ctl, s_bar_target, bcfg)) break;
        if (timer) {
            const unsigned long long tc = globaltimer_ns();
            s_ph[0] += tb - ta;
            s_ph[2] += tb2 - tb;
            s_ph[4] += tc - tb2;
        }
    }
    if (kSmem) store_chunk_state(own, s_cc, sV, sR);
    finish_counters(eng, ev, ovf, lane, &s_ev, &s_ovf);
    if (timer) {
        ctl->step = s0 + k;
        ctl->raster_next = rbase;
        ctl->raster_base = rbase;
        ctl->raster_dropped += s_dropped;
        for (int q = 0; q < 5; ++q) ctl->prof_phase_ns[q] += s_ph[q];
        ctl->prof_lif_ns += s_ph[0];
        ctl->prof_scatter_ns += s_ph[2] + s_ph[4];
        ctl->prof_steps += k;
    }
}

template __global__ void k_det_step<true>(EngineDev, unsigned long long, uint32_t);
template __global__ void k_det_step<false>(EngineDev, unsigned long long, uint32_t);

size_t step_smem_bytes(uint32_t own_max, bool smem_state, uint32_t bins) {
    const size_t off_cc = step_smem_offset(bins);
    if (!smem_state) return off_cc;
    const size_t off_v = off_cc + (((size_t)own_max * sizeof(ChunkCache) + 15) & ~(size_t)15);
    return off_v + (size_t)own_max * kLifThreads * (sizeof(float4) + sizeof(uchar4));
}

size_t run_smem_bytes(uint32_t grid, uint32_t own_max, bool smem_state) {
    const size_t off_cc = (((grid + 1) * sizeof(uint32_t)) + 15) & ~(size_t)15;
    if (!smem_state) return off_cc;
    const size_t off_v = off_cc + (((size_t)own_max * sizeof(ChunkCache) + 15) & ~(size_t)15);
    return off_v + (size_t)own_max * kLifThreads * (sizeof(float4) + sizeof(uchar4));
}

}  // namespace naer
