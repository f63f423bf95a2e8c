// Host engine implementation.
#include <cub/cub.cuh>

#include <atomic>
#include <mutex>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

#include "build_kernels.cuh"
#include "engine.h"
#include "philox.cuh"
#include "sim_kernels.cuh"

namespace naer {

void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    (void)cudaGetLastError();
    const int code = e == cudaErrorMemoryAllocation ? NAER_E_OOM : NAER_E_CUDA;
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        NAER_CK(cudaGetDevice(&prev));
        if (prev != dev) NAER_CK(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) cudaSetDevice(prev);
    }
};

__global__ void k_u32_to_u64(const uint32_t* in, uint32_t n, uint64_t* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x)
        out[i] = i < n ? (uint64_t)in[i] : 0ull;
}

uint32_t round_up4(uint32_t x) { return (x + 3u) & ~3u; }

// deterministic-aggregation scratch of a net: padded synapse entries, ring cells
uint64_t det_syn_entries(const NetHost& n) {
    return std::max<uint64_t>(n.syn_capacity ? n.syn_capacity : n.synapses_padded, 4);
}
uint64_t det_cells(const NetHost& n) { return (uint64_t)n.ring_slots * n.n_storage; }

uint32_t bit_width(uint64_t x) {
    uint32_t b = 0;
    while (x) {
        ++b;
        x >>= 1;
    }
    return b;
}

// Smallest z (plus a safety margin) whose first interval reaches past a
// window of W µs; 0xFFFFFFFF disables the fast path.
uint32_t poisson_z_hi(double rate, uint32_t W) {
    if (!(rate > 0.0)) return 0xFFFFFFFFu;
    if (ref_exp_interval_us(0xFFFFFFFEu, rate) < W) return 0xFFFFFFFFu;
    uint64_t lo = 0, hi = 0xFFFFFFFEull;
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (ref_exp_interval_us((uint32_t)mid, rate) >= W) hi = mid; else lo = mid;
    }
    return hi + 16 >= 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)(hi + 16);
}

uint32_t poisson_t0_limit(double rate) {
    if (!(rate > 0.0)) return 0;
    const uint64_t imax = ref_exp_interval_us(0xFFFFFFFEu, rate);
    if (imax + 2 >= 0xFFFFFFFFull) return 0;
    return (uint32_t)(0xFFFFFFFFull - (imax + 2));
}

template <typename F>
void with_cub_tmp(Engine& eng, F&& f) {
    size_t bytes = 0;
    NAER_CK(f(nullptr, bytes));
    void* tmp = eng.dalloc(bytes ? bytes : 16);
    try {
        NAER_CK(f(tmp, bytes));
    } catch (...) {
        eng.dfree(tmp, bytes ? bytes : 16);
        throw;
    }
    eng.dfree(tmp, bytes ? bytes : 16);  // ordered after the call's kernels
}

uint32_t grid_for(uint64_t items, uint32_t threads, uint32_t max_blocks) {
    uint64_t b = (items + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (uint32_t)b;
}

}  // namespace

Engine::Engine(int device, int priority) : device_(device) {
    int n = 0;
    NAER_CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) throw Error(NAER_E_INVALID, "device index out of range");
    NAER_CK(cudaSetDevice(device));
    NAER_CK(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device));
    NAER_CK(cudaStreamCreateWithPriority(&stream_, cudaStreamNonBlocking, priority));
    // keep freed stream-ordered memory in this process's pool (rebuilding
    // networks reuses it without new mappings); ~Engine trims the pool
    cudaMemPool_t pool;
    NAER_CK(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = ~0ull;
    NAER_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    d_ctl_ = static_cast<Ctl*>(dalloc(sizeof(Ctl)));
    NAER_CK(cudaMemsetAsync(d_ctl_, 0, sizeof(Ctl), stream_));
    NAER_CK(cudaStreamSynchronize(stream_));
    NAER_CK(cudaMallocHost(&h_pinned_, 512));  // [0, 256): control block copies; [256, 512): host->device words
}

Engine::~Engine() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    auto f = [](void* p) {
        if (p) cudaFree(p);
    };
    f(d_ctl_);
    f(d_nets_);
    f(d_pops_);
    f(d_chunks_);
    for (int i = 0; i < 2; ++i) {
        f(d_queue_[i]);
        f(d_qid_[i]);
        f(d_qrow_[i]);
        f(d_counts_[i]);
    }
    f(d_ev_part_);
    f(d_ovf_part_);
    f(d_raster_);
    for (auto ev : timer_events_) cudaEventDestroy(ev);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (h_pinned_) cudaFreeHost(h_pinned_);
    cudaStreamDestroy(stream_);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device_) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    if (prev >= 0) cudaSetDevice(prev);
}

// Stream-ordered allocation: neither call synchronises the device, so an
// engine that builds networks never stalls another engine's step launches.
// Memory from dalloc is usable by work queued on this engine's stream at
// once, and by other streams or the host after this stream is synchronised
// (every engine entry point that hands memory elsewhere synchronises);
// dfree is ordered after the work already queued on this stream (callers
// free memory only when no other stream still uses it).
namespace {
// Fault injection for tests (naer_test_fail_allocation): the allocation
// this many allocations from now fails as an out-of-memory would; -1 = off.
std::atomic<int64_t> g_alloc_fail_after{-1};
}  // namespace

void set_allocation_failure(int64_t after) { g_alloc_fail_after.store(after); }

void* Engine::dalloc(size_t bytes) {
    int64_t left = g_alloc_fail_after.load();
    while (left >= 0 && !g_alloc_fail_after.compare_exchange_weak(left, left - 1)) {
    }
    if (left == 0) throw Error(NAER_E_OOM, "injected allocation failure (test hook)");
    void* p = nullptr;
    NAER_CK(cudaMallocAsync(&p, bytes ? bytes : 16, stream_));
    bytes_ += bytes;
    if (alloc_log_) alloc_log_->push_back({p, bytes});
    return p;
}

void Engine::dfree(void* p, size_t bytes) {
    if (!p) return;
    NAER_CK(cudaFreeAsync(p, stream_));
    bytes_ -= std::min<uint64_t>(bytes_, bytes);
    if (alloc_log_)
        for (auto& e : *alloc_log_)
            if (e.first == p) e.first = nullptr;
}

// ---------------------------------------------------------------------------
// network build

static void layout(NetHost& n) {
    const auto& P = n.params;
    if (P.dt_us == 0) throw Error(NAER_E_INVALID, "dt_us must be positive");
    uint32_t type_count[3] = {0, 0, 0};
    for (const auto& p : n.pops) type_count[p.type] += p.size;
    const uint32_t type_base[3] = {0, type_count[kSTDP], type_count[kSTDP] + type_count[kNOP]};
    n.n_ids = type_count[0] + type_count[1] + type_count[2];
    n.n_poisson = type_count[kPOISSON];
    n.pop_order.clear();
    for (uint32_t t = 0; t < 3; ++t)
        for (uint32_t i = 0; i < n.pops.size(); ++i)
            if (n.pops[i].type == t) n.pop_order.push_back(i);
    uint32_t s = 0;
    n.n_plastic = 0;
    for (uint32_t i : n.pop_order) {
        auto& p = n.pops[i];
        p.id_base = type_base[p.type] + p.type_address;
        p.storage_base = s;
        s += round_up4(p.size);
        if (p.type == kSTDP) n.n_plastic = s;
    }
    n.n_storage = std::max<uint32_t>(s, 4);
    n.id_of_storage.assign(n.n_storage, -1);
    n.storage_of_id.assign(n.n_ids, 0);
    for (const auto& p : n.pops)
        for (uint32_t k = 0; k < p.size; ++k) {
            n.id_of_storage[p.storage_base + k] = (int32_t)(p.id_base + k);
            n.storage_of_id[p.id_base + k] = p.storage_base + k;
        }
    uint32_t dmax = 1;
    for (const auto& c : n.conns) {
        const auto& sp = c.spec;
        if (c.src >= n.pops.size() || c.dst >= n.pops.size())
            throw Error(NAER_E_INVALID, "connection refers to an unknown population");
        if (n.pops[c.dst].type == kPOISSON)
            throw Error(NAER_E_INVALID, "POISSON populations cannot receive connections");
        if (sp.rule > NAER_CONN_EXPLICIT || (sp.rule == NAER_CONN_EXPLICIT) != (c.csr != nullptr))
            throw Error(NAER_E_INVALID, "unknown connection rule");
        if (sp.delay_min < 1 || sp.delay_max < sp.delay_min || sp.delay_max > 254)
            throw Error(NAER_E_INVALID, "delays must satisfy 1 <= delay_min <= delay_max <= 254");
        if (sp.rule == NAER_CONN_REF_BERNOULLI && !(sp.probability >= 0.0 && sp.probability <= 1.0))
            throw Error(NAER_E_INVALID, "probability must be in [0, 1]");
        dmax = std::max(dmax, sp.delay_max);
    }
    n.ring_slots = dmax + 1;
    for (const auto& p : n.pops) {
        if (p.type == kPOISSON) continue;
        const double tr = std::llround((double)p.prm.t_ref_ms * 1000.0 / P.dt_us);
        if (tr < 0 || tr > 255) throw Error(NAER_E_INVALID, "refractory period must be 0..255 steps");
        if (!(p.prm.tau_m_ms > 0.0f)) throw Error(NAER_E_INVALID, "tau_m_ms must be positive");
    }
    if (P.stdp_enabled && (P.stdp_history == 0 || P.stdp_history > kMaxStdpHistory))
        throw Error(NAER_E_INVALID, "stdp_history must be in 1..16");
}

// Device bytes of a built network, from its description: padded synapse
// arrays (each row padded to 4 entries in each of its two delay classes),
// row pointers, neuron state, ring, drive slots and plasticity state.  The
// Bernoulli rule's count is its mean plus six standard deviations.
uint32_t lif_chunks(const NetHost& description) {
    uint64_t c = 0;
    for (const PopSpec& ps : description.pops) c += (ps.size + kLifChunk - 1) / kLifChunk;
    return (uint32_t)std::min<uint64_t>(c, 0xFFFFFFFFu);
}

uint32_t Engine::fast_chunk_capacity(uint32_t aggregation) {
    DeviceGuard g(device_);
    int optin = 0;
    NAER_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
    const bool det = aggregation == NAER_AGG_DETERMINISTIC;
    const bool split = det || tuning_.step_kernel == NAER_KERNEL_SPLIT;
    const void* kern = det ? (const void*)k_det_step<true>
                           : split ? (const void*)k_step<true> : (const void*)k_run<true>;
    cudaFuncAttributes fa{};
    NAER_CK(cudaFuncGetAttributes(&fa, kern));
    optin -= (int)fa.sharedSizeBytes;
    NAER_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    const int bps_hi = tuning_.blocks_per_sm ? (int)std::min<uint32_t>(tuning_.blocks_per_sm, 4) : 4;
    auto fits = [&](int bps, uint32_t own) {
        const uint32_t grid = (uint32_t)bps * (uint32_t)sm_count_;
        const size_t smem = split ? step_smem_bytes(own, true, det ? 0u : tuning_.bins) : run_smem_bytes(grid, own, true);
        if (smem > (size_t)optin) return false;
        int occ = 0;
        NAER_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kLifThreads, smem));
        return occ >= bps;
    };
    for (int bps = bps_hi; bps >= 1; --bps) {
        if (!fits(bps, 1)) continue;
        uint32_t lo = 1, hi = 1;  // largest own chunks per block that still fits: doubling, then bisection
        while (hi < (1u << 16) && fits(bps, hi * 2)) hi *= 2;
        lo = hi;
        hi = hi * 2;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (fits(bps, mid)) lo = mid; else hi = mid;
        }
        return lo * (uint32_t)bps * (uint32_t)sm_count_;
    }
    return 0;
}

uint64_t estimate_device_bytes(const NetHost& description, bool deterministic) {
    NetHost n;
    n.params = description.params;
    n.pops = description.pops;
    n.conns = description.conns;
    layout(n);
    double syn = 0;
    uint64_t rows = 0;
    for (const auto& c : n.conns) {
        const double src = n.pops[c.src].size, dst = n.pops[c.dst].size;
        const auto& sp = c.spec;
        if (sp.rule == NAER_CONN_REF_BERNOULLI) {
            const double m = sp.probability * src * dst;
            syn += m + 6.0 * std::sqrt(std::max(m, 1.0));
        } else if (sp.rule == NAER_CONN_FIXED_OUTDEGREE) {
            syn += (double)sp.degree * src;
        } else if (sp.rule == NAER_CONN_EXPLICIT) {
            syn += (double)c.csr->tgt.size();
        } else {
            syn += (double)sp.degree * dst;
        }
        rows += n.pops[c.src].size;
    }
    const uint64_t Ns = n.n_storage;
    const uint64_t entries = (uint64_t)std::ceil(syn) + (rows + Ns) * 6ull;  // synapses + padding
    uint64_t b = entries * 9ull;
    b += (Ns + 1) * 8ull + Ns * 4ull;                                          // row_ptr, row_mid
    b += Ns * (4ull + 1ull + kDriveSlots + 4ull * n.ring_slots);                // V, refr, drive, ring
    if (n.params.stdp_enabled && n.n_plastic) {
        const uint64_t Np = n.n_plastic;
        b += Np * (8ull + 4ull * round_up4(2u + n.params.stdp_history));
        const double tmax = std::max(n.params.tau_plus_ms, n.params.tau_minus_ms) * 1000.0;
        b += 8ull * (uint64_t)std::min<double>(std::ceil(104.0 * tmax / n.params.dt_us) + 1.0, 1 << 24);
    }
    // deterministic aggregation: event weight and link per padded synapse,
    // list head per ring cell (allocated by the first deterministic step)
    if (deterministic) b += entries * 8ull + (uint64_t)n.ring_slots * Ns * 4ull;
    return b;
}

static ConnBuild make_cb(const NetHost& n, const ConnSpec& c) {
    ConnBuild cb{};
    const auto& s = c.spec;
    cb.rule = s.rule;
    cb.K = s.degree;
    cb.p = s.probability;
    cb.weight = s.weight;
    cb.wmin = s.wmin;
    cb.wmax = s.wmax;
    cb.dmin = s.delay_min;
    cb.dmax = s.delay_max;
    cb.seed_lo = (uint32_t)s.seed;
    cb.seed_hi = (uint32_t)(s.seed >> 32);
    cb.src_size = n.pops[c.src].size;
    cb.dst_size = n.pops[c.dst].size;
    cb.src_storage = n.pops[c.src].storage_base;
    cb.dst_storage = n.pops[c.dst].storage_base;
    return cb;
}

void Engine::build(NetHost& n) {
    DeviceGuard g(device_);
    // every allocation of the build is logged, so that a build that fails
    // part way (an allocation, a launch) leaves no device memory behind
    std::vector<std::pair<void*, size_t>> log;
    alloc_log_ = &log;
    try {
        build_arrays(n);
    } catch (...) {
        alloc_log_ = nullptr;
        cudaStreamSynchronize(stream_);
        for (auto& e : log)
            if (e.first) dfree(e.first, e.second);
        n.v = nullptr;
        n.refr = nullptr;
        n.ring = nullptr;
        n.drive = nullptr;
        n.row_ptr = nullptr;
        n.row_mid = nullptr;
        n.tgt = nullptr;
        n.w = nullptr;
        n.dly = nullptr;
        n.post = nullptr;
        n.pre = nullptr;
        n.e_plus = n.e_minus = nullptr;
        n.compiled = false;
        throw;
    }
    alloc_log_ = nullptr;
}

void Engine::build_arrays(NetHost& n) {
    n.fx_shift = kFxUnknown;  // new weights: the exact-sum grid is recomputed when installed
    layout(n);
    const uint32_t Ns = n.n_storage;
    const uint32_t T = 256;
    const uint32_t maxb = (uint32_t)sm_count_ * 16;
    cudaStream_t st = stream_;
    const uint64_t bytes0 = bytes_;

    unsigned long long* stats = nullptr;  // [synapses, longest padded row, padded size]

    // --- connectivity: counts per (connection, source)
    uint64_t* len = static_cast<uint64_t*>(dalloc(Ns * 8ull));
    NAER_CK(cudaMemsetAsync(len, 0, Ns * 8ull, st));
    std::vector<uint32_t*> cnt(n.conns.size(), nullptr);
    for (size_t ci = 0; ci < n.conns.size(); ++ci) {
        const ConnBuild cb = make_cb(n, n.conns[ci]);
        cnt[ci] = static_cast<uint32_t*>(dalloc(std::max<uint64_t>(cb.src_size, 1) * 4ull));
        NAER_CK(cudaMemsetAsync(cnt[ci], 0, std::max<uint64_t>(cb.src_size, 1) * 4ull, st));
        if (cb.src_size == 0 || cb.dst_size == 0) continue;
        if (cb.rule == NAER_CONN_REF_BERNOULLI) {
            k_bern_count<<<grid_for((uint64_t)cb.src_size * 32, T, maxb), T, 0, st>>>(cb, cnt[ci]);
        } else if (cb.rule == NAER_CONN_EXPLICIT) {
            const ExplicitCsr& x = *n.conns[ci].csr;
            std::vector<uint32_t> lens(cb.src_size);
            for (uint32_t r = 0; r < cb.src_size; ++r) lens[r] = (uint32_t)(x.row_ptr[r + 1] - x.row_ptr[r]);
            NAER_CK(cudaMemcpyAsync(cnt[ci], lens.data(), cb.src_size * 4ull, cudaMemcpyHostToDevice, st));
            NAER_CK(cudaStreamSynchronize(st));  // lens is pageable and local
        } else if (cb.rule == NAER_CONN_FIXED_OUTDEGREE) {
            k_fill_u32<<<grid_for(cb.src_size, T, maxb), T, 0, st>>>(cnt[ci], cb.src_size, cb.K);
        } else {
            const uint64_t items = (uint64_t)cb.dst_size * ((cb.K + 3) / 4);
            if (items) k_indeg_count<<<grid_for(items, T, maxb), T, 0, st>>>(cb, cnt[ci]);
        }
        k_row_len_add<<<grid_for(cb.src_size, T, maxb), T, 0, st>>>(cnt[ci], cb.src_size,
                                                                    cb.src_storage, len);
        NAER_CK(cudaGetLastError());
    }
    // Fixed-degree rules: the synapse count is known here, so the arrays are
    // sized by a bound (each row padded by at most 3 per padding) and the
    // whole build is queued without waiting for the device; a Bernoulli
    // connection needs the device's count first.
    bool exact = true;
    uint64_t syn_exact = 0;
    for (const auto& c : n.conns) {
        const auto& sp = c.spec;
        if (sp.rule == NAER_CONN_REF_BERNOULLI) exact = false;
        else if (sp.rule == NAER_CONN_EXPLICIT) syn_exact += c.csr->tgt.size();
        else if (sp.rule == NAER_CONN_FIXED_OUTDEGREE) syn_exact += (uint64_t)sp.degree * n.pops[c.src].size;
        else syn_exact += (uint64_t)sp.degree * n.pops[c.dst].size;
    }
    uint64_t* padded = static_cast<uint64_t*>(dalloc((Ns + 1) * 8ull));
    k_row_pad<<<grid_for(Ns + 1, T, maxb), T, 0, st>>>(len, Ns, padded);
    n.row_ptr = static_cast<uint64_t*>(dalloc((Ns + 1) * 8ull));
    with_cub_tmp(*this, [&](void* tmp, size_t& b) {
        return cub::DeviceScan::ExclusiveSum(tmp, b, padded, n.row_ptr, (int)(Ns + 1), st);
    });
    if (exact) {
        n.synapses_padded = syn_exact + 3ull * Ns;
    } else {
        NAER_CK(cudaMemcpyAsync(&n.synapses_padded, n.row_ptr + Ns, 8, cudaMemcpyDeviceToHost, st));
        NAER_CK(cudaStreamSynchronize(st));
    }
    const uint64_t S = n.synapses_padded;
    n.tgt = static_cast<uint32_t*>(dalloc(std::max<uint64_t>(S, 4) * 4ull));
    n.w = static_cast<float*>(dalloc(std::max<uint64_t>(S, 4) * 4ull));
    n.dly = static_cast<uint8_t*>(dalloc(std::max<uint64_t>(S, 16)));
    uint64_t* cursor = static_cast<uint64_t*>(dalloc(Ns * 8ull));
    NAER_CK(cudaMemcpyAsync(cursor, n.row_ptr, Ns * 8ull, cudaMemcpyDeviceToDevice, st));

    // --- fill rows, connection by connection
    for (size_t ci = 0; ci < n.conns.size(); ++ci) {
        const ConnBuild cb = make_cb(n, n.conns[ci]);
        if (cb.src_size == 0 || cb.dst_size == 0) continue;
        if (cb.rule == NAER_CONN_REF_BERNOULLI) {
            k_bern_fill<<<grid_for((uint64_t)cb.src_size * 32, T, maxb), T, 0, st>>>(cb, cursor, n.tgt,
                                                                                     n.w, n.dly);
        } else if (cb.rule == NAER_CONN_EXPLICIT) {
            const ExplicitCsr& x = *n.conns[ci].csr;
            const uint64_t nnz = x.tgt.size();
            auto* rp = static_cast<uint64_t*>(dalloc((cb.src_size + 1) * 8ull));
            auto* tg = static_cast<uint32_t*>(dalloc(std::max<uint64_t>(nnz, 1) * 4ull));
            auto* wv = static_cast<float*>(dalloc(std::max<uint64_t>(nnz, 1) * 4ull));
            auto* dv = static_cast<uint8_t*>(dalloc(std::max<uint64_t>(nnz, 1)));
            NAER_CK(cudaMemcpyAsync(rp, x.row_ptr.data(), (cb.src_size + 1) * 8ull, cudaMemcpyHostToDevice, st));
            if (nnz) {
                NAER_CK(cudaMemcpyAsync(tg, x.tgt.data(), nnz * 4ull, cudaMemcpyHostToDevice, st));
                NAER_CK(cudaMemcpyAsync(wv, x.w.data(), nnz * 4ull, cudaMemcpyHostToDevice, st));
                NAER_CK(cudaMemcpyAsync(dv, x.dly.data(), nnz, cudaMemcpyHostToDevice, st));
            }
            k_explicit_fill<<<grid_for((uint64_t)cb.src_size * 32, T, maxb), T, 0, st>>>(cb, rp, tg, wv, dv, cursor,
                                                                                         n.tgt, n.w, n.dly);
            NAER_CK(cudaGetLastError());
            dfree(rp, (cb.src_size + 1) * 8ull);
            dfree(tg, std::max<uint64_t>(nnz, 1) * 4ull);
            dfree(wv, std::max<uint64_t>(nnz, 1) * 4ull);
            dfree(dv, std::max<uint64_t>(nnz, 1));
        } else if (cb.rule == NAER_CONN_FIXED_OUTDEGREE) {
            const uint64_t items = (uint64_t)cb.src_size * ((cb.K + 3) / 4);
            if (items)
                k_outdeg_fill<<<grid_for(items, T, maxb), T, 0, st>>>(cb, cursor, n.tgt, n.w, n.dly);
        } else if (cb.K > 0) {
            uint64_t* off = static_cast<uint64_t*>(dalloc((cb.src_size + 1) * 8ull));
            uint64_t* cnt64 = static_cast<uint64_t*>(dalloc((cb.src_size + 1) * 8ull));
            k_u32_to_u64<<<grid_for(cb.src_size + 1, T, maxb), T, 0, st>>>(cnt[ci], cb.src_size, cnt64);
            with_cub_tmp(*this, [&](void* tmp, size_t& b) {
                return cub::DeviceScan::ExclusiveSum(tmp, b, cnt64, off, (int)(cb.src_size + 1), st);
            });
            const uint64_t total = (uint64_t)cb.dst_size * cb.K;  // every draw lands in some row
            if (total > 0x7FFFFFFFull)
                throw Error(NAER_E_OVERFLOW, "a FIXED_INDEGREE connection exceeds 2^31 synapses");
            // stable radix sort of the draws by source (draw order = canonical order)
            auto* kin = static_cast<uint32_t*>(dalloc(std::max<uint64_t>(total, 1) * 4ull));
            auto* kout = static_cast<uint32_t*>(dalloc(std::max<uint64_t>(total, 1) * 4ull));
            auto* vin = static_cast<uint32_t*>(dalloc(std::max<uint64_t>(total, 1) * 4ull));
            auto* vout = static_cast<uint32_t*>(dalloc(std::max<uint64_t>(total, 1) * 4ull));
            const uint64_t items = (uint64_t)cb.dst_size * ((cb.K + 3) / 4);
            k_indeg_keys<<<grid_for(items, T, maxb), T, 0, st>>>(cb, kin, vin);
            NAER_CK(cudaGetLastError());
            const int kbits = std::max<int>(1, (int)bit_width(cb.src_size - 1));
            with_cub_tmp(*this, [&](void* tmp, size_t& b) {
                return cub::DeviceRadixSort::SortPairs(tmp, b, kin, kout, vin, vout, (int)total, 0, kbits, st);
            });
            k_indeg_finalize<<<grid_for(total, T, maxb), T, 0, st>>>(cb, kout, vout, total, off, cursor, n.tgt,
                                                                     n.w, n.dly);
            NAER_CK(cudaGetLastError());
            dfree(kin, std::max<uint64_t>(total, 1) * 4ull);
            dfree(kout, std::max<uint64_t>(total, 1) * 4ull);
            dfree(vin, std::max<uint64_t>(total, 1) * 4ull);
            dfree(vout, std::max<uint64_t>(total, 1) * 4ull);
            dfree(off, (cb.src_size + 1) * 8ull);
            dfree(cnt64, (cb.src_size + 1) * 8ull);
        }
        k_cursor_advance<<<grid_for(cb.src_size, T, maxb), T, 0, st>>>(cnt[ci], cb.src_size,
                                                                       cb.src_storage, cursor);
        NAER_CK(cudaGetLastError());
    }
    k_pad_fill<<<grid_for(Ns, T, maxb), T, 0, st>>>(n.row_ptr, len, Ns, n.tgt, n.w, n.dly);
    NAER_CK(cudaGetLastError());
    // canonical order: stable partition of every row, delay-1 synapses first,
    // each part starting on a 16-byte boundary
    {
        uint32_t* n1 = static_cast<uint32_t*>(dalloc(Ns * 4ull));
        k_count_d1<<<grid_for((uint64_t)Ns * 32, T, maxb), T, 0, st>>>(n.row_ptr, len, Ns, n.dly, n1);
        uint64_t* padded2 = static_cast<uint64_t*>(dalloc((Ns + 1) * 8ull));
        k_row_pad_split<<<grid_for(Ns + 1, T, maxb), T, 0, st>>>(len, n1, Ns, padded2);
        uint64_t* row_ptr2 = static_cast<uint64_t*>(dalloc((Ns + 1) * 8ull));
        with_cub_tmp(*this, [&](void* tmp, size_t& b) {
            return cub::DeviceScan::ExclusiveSum(tmp, b, padded2, row_ptr2, (int)(Ns + 1), st);
        });
        uint64_t S2 = 0;
        if (exact) {
            S2 = syn_exact + 6ull * Ns;  // two padded parts per row
        } else {
            NAER_CK(cudaMemcpyAsync(&S2, row_ptr2 + Ns, 8, cudaMemcpyDeviceToHost, st));
            NAER_CK(cudaStreamSynchronize(st));
        }
        uint32_t* tgt2 = static_cast<uint32_t*>(dalloc(std::max<uint64_t>(S2, 4) * 4ull));
        float* w2 = static_cast<float*>(dalloc(std::max<uint64_t>(S2, 4) * 4ull));
        uint8_t* dly2 = static_cast<uint8_t*>(dalloc(std::max<uint64_t>(S2, 16)));
        n.row_mid = static_cast<uint32_t*>(dalloc(Ns * 4ull));
        k_partition_d1<<<grid_for((uint64_t)Ns * 32, T, maxb), T, 0, st>>>(
            n.row_ptr, len, n1, Ns, row_ptr2, n.tgt, n.w, n.dly, tgt2, w2, dly2, n.row_mid);
        NAER_CK(cudaGetLastError());
        // synapse count, longest padded row and the final padded size, read
        // back with the build's one synchronisation (below)
        stats = static_cast<unsigned long long*>(dalloc(5 * 8ull));
        NAER_CK(cudaMemsetAsync(stats, 0, 5 * 8ull, st));
        k_row_stats<<<grid_for(Ns, T, maxb), T, 0, st>>>(len, padded2, n1, Ns, stats);
        NAER_CK(cudaMemcpyAsync(stats + 2, row_ptr2 + Ns, 8, cudaMemcpyDeviceToDevice, st));
        NAER_CK(cudaGetLastError());
        dfree(n.tgt, std::max<uint64_t>(S, 4) * 4ull);
        dfree(n.w, std::max<uint64_t>(S, 4) * 4ull);
        dfree(n.dly, std::max<uint64_t>(S, 16));
        dfree(n.row_ptr, (Ns + 1) * 8ull);
        dfree(padded2, (Ns + 1) * 8ull);
        dfree(n1, Ns * 4ull);
        n.tgt = tgt2;
        n.w = w2;
        n.dly = dly2;
        n.row_ptr = row_ptr2;
        n.syn_capacity = S2;
    }
    for (size_t ci = 0; ci < cnt.size(); ++ci)
        dfree(cnt[ci], std::max<uint64_t>(n.pops[n.conns[ci].src].size, 1) * 4ull);
    dfree(len, Ns * 8ull);
    dfree(padded, (Ns + 1) * 8ull);
    dfree(cursor, Ns * 8ull);

    // --- neuron state
    n.v = static_cast<float*>(dalloc(Ns * 4ull));
    n.refr = static_cast<uint8_t*>(dalloc(Ns));
    n.ring = static_cast<float*>(dalloc((uint64_t)n.ring_slots * Ns * 4ull));
    n.drive = static_cast<uint8_t*>(dalloc((uint64_t)kDriveSlots * Ns));
    NAER_CK(cudaMemsetAsync(n.drive, 0, (uint64_t)kDriveSlots * Ns, st));
    std::vector<float> v0(Ns, 0.0f);
    for (const auto& p : n.pops)
        if (p.type != kPOISSON)
            for (uint32_t k = 0; k < p.size; ++k) v0[p.storage_base + k] = p.prm.v_init;
    NAER_CK(cudaMemcpyAsync(n.v, v0.data(), Ns * 4ull, cudaMemcpyHostToDevice, st));
    NAER_CK(cudaMemsetAsync(n.refr, 0, Ns, st));
    NAER_CK(cudaMemsetAsync(n.ring, 0, (uint64_t)n.ring_slots * Ns * 4ull, st));

    const auto& P = n.params;
    const bool stdp = P.stdp_enabled && n.n_plastic > 0;
    if (stdp) {
        const uint32_t Np = n.n_plastic;
        n.post_stride = round_up4(2u + P.stdp_history);
        n.post = static_cast<int32_t*>(dalloc((uint64_t)Np * n.post_stride * 4ull));
        n.pre = static_cast<int2*>(dalloc(Np * 8ull));
        // every word -1, then the post traces (word 1 of each row) 0.0f
        std::vector<int32_t> row0((uint64_t)Np * n.post_stride, -1);
        for (uint64_t r = 0; r < Np; ++r) row0[r * n.post_stride + 1] = 0;
        NAER_CK(cudaMemcpyAsync(n.post, row0.data(), row0.size() * 4ull, cudaMemcpyHostToDevice, st));
        std::vector<int2> pre0(Np, make_int2(-1, 0));
        NAER_CK(cudaMemcpyAsync(n.pre, pre0.data(), Np * 8ull, cudaMemcpyHostToDevice, st));
        NAER_CK(cudaStreamSynchronize(st));  // host staging vectors go out of scope
        // exp(-k dt / tau) as float until it underflows (k dt / tau > 104)
        const double tmax = std::max((double)P.tau_plus_ms, (double)P.tau_minus_ms) * 1000.0;
        n.e_len = (uint32_t)std::min<double>(std::ceil(104.0 * tmax / P.dt_us) + 1.0, 1 << 24);
        std::vector<float> ep(n.e_len), em(n.e_len);
        for (uint32_t k = 0; k < n.e_len; ++k) {
            ep[k] = (float)std::exp(-(double)k * P.dt_us / ((double)P.tau_plus_ms * 1000.0));
            em[k] = (float)std::exp(-(double)k * P.dt_us / ((double)P.tau_minus_ms * 1000.0));
        }
        n.e_plus = static_cast<float*>(dalloc(n.e_len * 4ull));
        n.e_minus = static_cast<float*>(dalloc(n.e_len * 4ull));
        NAER_CK(cudaMemcpyAsync(n.e_plus, ep.data(), n.e_len * 4ull, cudaMemcpyHostToDevice, st));
        NAER_CK(cudaMemcpyAsync(n.e_minus, em.data(), n.e_len * 4ull, cudaMemcpyHostToDevice, st));
    }
    unsigned long long hstats[5] = {0, 0, 0, 0, 0};
    NAER_CK(cudaMemcpyAsync(hstats, stats, sizeof(hstats), cudaMemcpyDeviceToHost, st));
    dfree(stats, 5 * 8ull);
    NAER_CK(cudaStreamSynchronize(st));
    n.synapses = hstats[0];
    n.max_row_padded = hstats[1];
    n.synapses_padded = hstats[2];
    n.max_first_padded = hstats[3];
    n.max_rest_padded = hstats[4];

    NetDev& d = n.dev;
    d = NetDev{};
    d.v = n.v;
    d.refr = n.refr;
    d.ring = n.ring;
    d.drive = n.drive;
    d.row_ptr = n.row_ptr;
    d.row_mid = n.row_mid;
    d.tgt = n.tgt;
    d.w = n.w;
    d.dly = n.dly;
    d.post = n.post;
    d.pre = n.pre;
    d.post_stride = n.post_stride;
    d.e_plus = n.e_plus;
    d.e_minus = n.e_minus;
    d.start_step = 0;
    d.end_step = ~0ull;
    d.syn_cap = std::max<uint64_t>(n.syn_capacity, n.synapses_padded);
    d.n_storage = Ns;
    d.ring_slots = n.ring_slots;
    d.dt_us = P.dt_us;
    d.n_plastic = stdp ? n.n_plastic : 0;
    d.stdp_on = stdp ? 1u : 0u;
    d.hist_len = P.stdp_history;
    d.e_len = n.e_len;
    d.a_plus = P.a_plus * P.w_max;
    d.a_minus = P.a_minus * P.w_max;
    d.w_max = P.w_max;
    d.active = 1;
    n.device_bytes = bytes_ - bytes0;
    n.compiled = true;
}

void Engine::free_net(NetHost& n) {
    DeviceGuard g(device_);
    const uint32_t Ns = n.n_storage;
    const uint64_t S = n.syn_capacity ? n.syn_capacity : n.synapses_padded;  // entries allocated
    dfree(n.v, Ns * 4ull);
    dfree(n.refr, Ns);
    dfree(n.ring, (uint64_t)n.ring_slots * Ns * 4ull);
    dfree(n.drive, (uint64_t)kDriveSlots * Ns);
    n.drive = nullptr;
    dfree(n.row_ptr, (Ns + 1) * 8ull);
    dfree(n.row_mid, Ns * 4ull);
    n.row_mid = nullptr;
    dfree(n.tgt, std::max<uint64_t>(S, 4) * 4ull);
    dfree(n.w, std::max<uint64_t>(S, 4) * 4ull);
    dfree(n.dly, std::max<uint64_t>(S, 16));
    const uint32_t Np = n.n_plastic;
    dfree(n.post, (uint64_t)Np * n.post_stride * 4ull);
    dfree(n.pre, Np * 8ull);
    dfree(n.e_plus, n.e_len * 4ull);
    dfree(n.e_minus, n.e_len * 4ull);
    if (n.det_w) {
        dfree(n.det_w, det_syn_entries(n) * 4ull);
        dfree(n.det_next, det_syn_entries(n) * 4ull);
        dfree(n.det_head, det_cells(n) * 4ull);
        n.det_w = nullptr;
        n.det_next = nullptr;
        n.det_head = nullptr;
    }
    n.v = nullptr;
    n.refr = nullptr;
    n.ring = nullptr;
    n.row_ptr = nullptr;
    n.tgt = nullptr;
    n.w = nullptr;
    n.dly = nullptr;
    n.post = nullptr;
    n.pre = nullptr;
    n.e_plus = n.e_minus = nullptr;
    n.compiled = false;
}

// ---------------------------------------------------------------------------
// descriptor tables

// Shift S of the exact-sum aggregation's grid 2^-S for built networks
// (fx_shift of each): the largest S <= 30 for which no ring-cell sum can
// leave int32.  A cell receives at most one event per synapse into its
// neuron before it is read, of magnitude at most max|w| (at least w_max in a
// plastic network) times 10 (the largest POISSON multiplicity), each
// rounded by at most half a unit.  -1: no S >= 0 holds that bound.  The
// device reductions of every network are queued first and read back with
// one synchronisation.
void Engine::exact_shifts(const std::vector<NetHost*>& nets) {
    if (nets.empty()) return;
    DeviceGuard g(device_);
    uint32_t ns_max = 1;
    for (const NetHost* n : nets) ns_max = std::max(ns_max, n->n_storage);
    const uint64_t in_bytes = (uint64_t)ns_max * 4ull;
    const uint64_t st_bytes = (uint64_t)nets.size() * 8ull;
    uint32_t* in = static_cast<uint32_t*>(dalloc(in_bytes));
    unsigned int* out = nullptr;
    try {
        out = static_cast<unsigned int*>(dalloc(st_bytes));  // per net: max |w| bits, max in-degree
        NAER_CK(cudaMemsetAsync(out, 0, st_bytes, stream_));
        const uint32_t T = 256;
        for (size_t i = 0; i < nets.size(); ++i) {
            const NetHost& n = *nets[i];
            const uint64_t S = n.synapses_padded;
            NAER_CK(cudaMemsetAsync(in, 0, (uint64_t)n.n_storage * 4ull, stream_));
            const uint32_t g1 = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((S + T - 1) / T, (uint64_t)sm_count_ * 8));
            if (S) k_exact_inputs<<<g1, T, 0, stream_>>>(n.tgt, n.w, S, in, out + 2 * i);
            const uint32_t g2 =
                (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n.n_storage + T - 1) / T, (uint64_t)sm_count_ * 4));
            if (n.n_storage) k_max_u32<<<g2, T, 0, stream_>>>(in, n.n_storage, out + 2 * i + 1);
        }
        NAER_CK(cudaGetLastError());
        std::vector<unsigned int> h(2 * nets.size());
        NAER_CK(cudaMemcpyAsync(h.data(), out, st_bytes, cudaMemcpyDeviceToHost, stream_));
        NAER_CK(cudaStreamSynchronize(stream_));
        dfree(out, st_bytes);
        out = nullptr;
        dfree(in, in_bytes);
        in = nullptr;
        for (size_t i = 0; i < nets.size(); ++i) {
            NetHost& n = *nets[i];
            float maxw;
            std::memcpy(&maxw, &h[2 * i], 4);
            if (n.params.stdp_enabled && n.n_plastic > 0) maxw = std::max(maxw, n.params.w_max);
            bool poisson = false;
            for (const PopSpec& ps : n.pops) poisson = poisson || (ps.type == kPOISSON && ps.size > 0);
            const uint32_t max_in = h[2 * i + 1];
            const double bound = (double)max_in * (double)maxw * (poisson ? 10.0 : 1.0);
            n.fx_shift = -1;
            for (int32_t sh = 30; sh >= 0; --sh)
                if (bound * std::ldexp(1.0, sh) + (double)max_in <= 2147483647.0) {
                    n.fx_shift = sh;
                    break;
                }
        }
    } catch (...) {
        if (out) dfree(out, st_bytes);
        if (in) dfree(in, in_bytes);
        throw;
    }
}

void Engine::install(const std::vector<NetHost*>& nets, uint64_t raster_capacity, bool record,
                     uint32_t aggregation) {
    DeviceGuard g(device_);
    NAER_CK(cudaStreamSynchronize(stream_));
    drop_graph();
    nets_ = nets;
    aggregation_ = aggregation;
    inst_raster_cap_ = raster_capacity;
    inst_record_ = record;
    std::vector<PopDev> pops;
    std::vector<ChunkDev> chunks;
    h_nets_.clear();
    id_offsets_.clear();
    if (aggregation == NAER_AGG_EXACT) {  // grids of the networks installed for the first time
        std::vector<NetHost*> fresh;
        for (NetHost* n : nets)
            if (n->fx_shift == kFxUnknown) fresh.push_back(n);
        exact_shifts(fresh);
    }
    uint64_t key_base = 0;
    uint64_t qcap = 0;
    uint64_t id_off = 0;
    for (uint32_t ni = 0; ni < nets.size(); ++ni) {
        NetHost& n = *nets[ni];
        NetDev d = n.dev;
        d.fx_scale = d.fx_inv = 0.0f;
        if (aggregation == NAER_AGG_EXACT) {
            if (n.fx_shift < 0)
                throw Error(NAER_E_OVERFLOW, "weights too large for exact-sum aggregation: no fixed-point grid "
                                             "holds the largest possible ring-cell sum in 32 bits");
            d.fx_scale = std::ldexp(1.0f, n.fx_shift);
            d.fx_inv = std::ldexp(1.0f, -n.fx_shift);
        }
        d.ring_key_base = key_base;
        key_base += (uint64_t)n.ring_slots * n.n_storage;
        h_nets_.push_back(d);
        qcap += n.n_storage;
        id_offsets_.push_back((uint32_t)id_off);
        const auto& P = n.params;
        for (uint32_t pi : n.pop_order) {
            const PopSpec& ps = n.pops[pi];
            if (ps.size == 0) continue;
            PopDev pd{};
            pd.net = ni;
            pd.type = ps.type;
            pd.storage_base = ps.storage_base;
            pd.size = ps.size;
            pd.id_base = (uint32_t)id_off + ps.id_base;  // raster ids are engine-global
            if (ps.type == kPOISSON) {
                pd.rate_hz = (double)ps.prm.rate_hz;
                pd.rng_seed = P.poisson_seed;
                pd.rng_n = n.n_poisson;
                pd.rng_idx_base = ps.type_address;
            } else {
                pd.t_ref_steps = (uint32_t)std::llround((double)ps.prm.t_ref_ms * 1000.0 / P.dt_us);
                pd.v_th = ps.prm.v_th;
                pd.v_reset = ps.prm.v_reset;
                pd.prop = std::exp(-(double)P.dt_us / ((double)ps.prm.tau_m_ms * 1000.0));
                pd.rate_hz = (double)ps.prm.drive_rate_hz;
                pd.drive_w = ps.prm.drive_weight;
                pd.rng_seed = ps.prm.drive_seed;
                pd.rng_n = ps.size;
                pd.rng_idx_base = 0;
            }
            pd.z_hi = poisson_z_hi(pd.rate_hz, P.dt_us);
            pd.t0_limit = poisson_t0_limit(pd.rate_hz);
            const uint32_t pidx = (uint32_t)pops.size();
            pops.push_back(pd);
            for (uint32_t f = ps.storage_base; f < ps.storage_base + ps.size; f += kLifChunk)
                chunks.push_back(ChunkDev{pidx, f, ps.storage_base + ps.size, ni});
        }
        id_off += n.n_ids;
        if (id_off > 0xFFFFFFFFull) throw Error(NAER_E_OVERFLOW, "more than 2^32 neuron addresses in one engine");
    }
    total_ring_cells_ = key_base;
    if (qcap > 0xFFFFFFFFull) throw Error(NAER_E_OVERFLOW, "more than 2^32 neurons in one engine");

    auto upload = [&](void*& dst, size_t& cap_bytes, const void* src, size_t bytes) {
        if (bytes > cap_bytes) {
            if (dst) dfree(dst, cap_bytes);
            dst = nullptr;
            cap_bytes = 0;
            dst = dalloc(bytes);
            cap_bytes = bytes;
        }
        if (bytes) NAER_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_));
    };
    upload(reinterpret_cast<void*&>(d_nets_), nets_bytes_, h_nets_.data(), h_nets_.size() * sizeof(NetDev));
    upload(reinterpret_cast<void*&>(d_pops_), pops_bytes_, pops.data(), pops.size() * sizeof(PopDev));
    upload(reinterpret_cast<void*&>(d_chunks_), chunks_bytes_, chunks.data(), chunks.size() * sizeof(ChunkDev));

    eng_ = EngineDev{};
    eng_.n_chunks = (uint32_t)chunks.size();
    eng_.n_nets = (uint32_t)nets.size();

    // launch geometry: the persistent kernel's cooperative grid (all blocks
    // resident).  Prefer the variant that keeps neuron state in shared
    // memory, with as many blocks per SM as its footprint allows; the
    // deterministic path's LIF uses the same queue regions.
    const bool det = aggregation == NAER_AGG_DETERMINISTIC;
    const bool exact = aggregation == NAER_AGG_EXACT;
    // exact-sum aggregation: integer reductions in either atomic kernel, no binning
    split_kernel_ = !det && tuning_.step_kernel == NAER_KERNEL_SPLIT;
    const bool list_kernel = det || split_kernel_;  // one contiguous spike list per step
    const void* kern_smem = det ? (const void*)k_det_step<true>
                                : split_kernel_ ? (const void*)k_step<true> : (const void*)k_run<true>;
    const void* kern_glob = det ? (const void*)k_det_step<false>
                                : split_kernel_ ? (const void*)k_step<false> : (const void*)k_run<false>;
    const uint32_t bins = split_kernel_ && !exact ? tuning_.bins : 0u;
    auto smem_of = [&](uint32_t grid, uint32_t own, bool state) {
        return list_kernel ? step_smem_bytes(own, state, bins) : run_smem_bytes(grid, own, state);
    };
    det_scratch_ = kScratchNone;  // the next deterministic call points the new tables at its scratch
    int dev_smem_optin = 0;
    NAER_CK(cudaDeviceGetAttribute(&dev_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
    cudaFuncAttributes fa{};
    NAER_CK(cudaFuncGetAttributes(&fa, kern_smem));
    dev_smem_optin -= (int)fa.sharedSizeBytes;
    NAER_CK(cudaFuncSetAttribute(kern_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_smem_optin));
    use_smem_state_ = false;
    lif_grid_ = 0;
    const int bps_hi = tuning_.blocks_per_sm ? (int)std::min<uint32_t>(tuning_.blocks_per_sm, 4) : 4;
    for (int bps = bps_hi; bps >= 1 && !use_smem_state_ && tuning_.neuron_state != NAER_STATE_GLOBAL; --bps) {
        const uint32_t grid = (uint32_t)bps * sm_count_;
        const uint32_t own = std::max<uint32_t>(1, (eng_.n_chunks + grid - 1) / grid);
        const size_t smem = smem_of(grid, own, true);
        if (smem > (size_t)dev_smem_optin) continue;
        int occ = 0;
        NAER_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern_smem, kLifThreads, smem));
        if (occ >= bps) {
            use_smem_state_ = true;
            lif_grid_ = grid;
            scatter_smem_ = smem;
        }
    }
    if (!use_smem_state_ && tuning_.neuron_state == NAER_STATE_SHARED)
        throw Error(NAER_E_INVALID, "neuron state does not fit shared memory at this geometry");
    if (!use_smem_state_) {
        int occ = 0;
        const size_t smem_bound = smem_of((uint32_t)sm_count_ * 4, 1, false);
        NAER_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern_glob, kLifThreads, smem_bound));
        if (occ < 1) throw Error(NAER_E_CUDA, "the step kernel cannot be resident on this device");
        lif_grid_ = (uint32_t)std::min(occ, bps_hi) * sm_count_;
        scatter_smem_ = smem_of(lif_grid_, 1, false);
    }
    scatter_grid_ = lif_grid_;
    const uint32_t chunks_per_block = (eng_.n_chunks + lif_grid_ - 1) / lif_grid_;
    const uint32_t region_cap = std::max<uint32_t>(1, chunks_per_block) * kLifChunk;

    // fold per-block event counters of a previous installation into the base
    if (d_ev_part_) {
        events_base_ += sum_parts(d_ev_part_, ev_part_n_);
        overflow_base_ += sum_parts(d_ovf_part_, ev_part_n_);
    }
    // per-block regions (k_run, deterministic LIF) or one list of every
    // neuron at most (k_step)
    const uint64_t qentries = std::max<uint64_t>((uint64_t)lif_grid_ * region_cap, qcap);
    if (qentries > 0xFFFFFFFFull) throw Error(NAER_E_OVERFLOW, "spike queue larger than 2^32 entries");
    for (int i = 0; i < 2; ++i) {
        regrow(reinterpret_cast<void*&>(d_queue_[i]), queue_bytes_[i], qentries * sizeof(SpikeRec));
        regrow(reinterpret_cast<void*&>(d_qid_[i]), qid_bytes_[i], qentries * sizeof(uint32_t));
        regrow(reinterpret_cast<void*&>(d_qrow_[i]), qrow_bytes_[i], qentries * sizeof(uint4));
        regrow(reinterpret_cast<void*&>(d_counts_[i]), counts_bytes_[i], (lif_grid_ + 1) * sizeof(uint32_t));
        NAER_CK(cudaMemsetAsync(d_counts_[i], 0, (lif_grid_ + 1) * sizeof(uint32_t), stream_));
    }
    regrow(reinterpret_cast<void*&>(d_ev_part_), ev_part_bytes_, scatter_grid_ * sizeof(unsigned long long));
    regrow(reinterpret_cast<void*&>(d_ovf_part_), ovf_part_bytes_, scatter_grid_ * sizeof(unsigned long long));
    NAER_CK(cudaMemsetAsync(d_ev_part_, 0, scatter_grid_ * sizeof(unsigned long long), stream_));
    NAER_CK(cudaMemsetAsync(d_ovf_part_, 0, scatter_grid_ * sizeof(unsigned long long), stream_));
    ev_part_n_ = scatter_grid_;
    queue_cap_ = (uint32_t)qentries;
    const size_t rbytes = std::max<uint64_t>(raster_capacity, 1) * sizeof(uint2);
    if (rbytes != raster_bytes_) {
        if (d_raster_) dfree(d_raster_, raster_bytes_);
        d_raster_ = nullptr;
        raster_bytes_ = 0;
        d_raster_ = static_cast<uint2*>(dalloc(rbytes));
        raster_bytes_ = rbytes;
    }

    eng_.ctl = d_ctl_;
    eng_.nets = d_nets_;
    eng_.pops = d_pops_;
    eng_.chunks = d_chunks_;
    for (int i = 0; i < 2; ++i) {
        eng_.queue[i] = d_queue_[i];
        eng_.qid[i] = d_qid_[i];
        eng_.qrow[i] = d_qrow_[i];
        eng_.counts[i] = d_counts_[i];
    }
    eng_.ev_part = d_ev_part_;
    eng_.ovf_part = d_ovf_part_;
    eng_.raster = d_raster_;
    eng_.raster_cap = raster_capacity;
    eng_.lif_grid = lif_grid_;
    eng_.region_cap = region_cap;
    eng_.record = record ? 1u : 0u;
    // pieces of 128 synapses when some net is plastic (a plastic synapse
    // costs a dependent post-row load, so more warps per row pay off), else
    // 256; warps per spike: enough pieces to cover the longest row once
    bool any_stdp = false;
    uint64_t max_row = 0;
    for (NetHost* n : nets) {
        max_row = std::max<uint64_t>(max_row, n->max_row_padded);
        any_stdp = any_stdp || n->dev.stdp_on;
    }
    eng_.scatter_piece = tuning_.scatter_piece ? tuning_.scatter_piece : (any_stdp ? 128u : kScatterPiece);
    const uint32_t psz = eng_.scatter_piece;
    eng_.scatter_split = (uint32_t)std::min<uint64_t>(any_stdp ? 32 : 16, std::max<uint64_t>(1, (max_row + psz - 1) / psz));
    if (tuning_.scatter_split) eng_.scatter_split = std::min<uint32_t>(tuning_.scatter_split, 64);
    // k_step: the part delivered before the next LIF (delay-1 synapses;
    // whole rows of plastic sources) and the deferred rest
    // (plastic rows go in pieces of kPlasticPiece: one synapse per lane)
    uint64_t first_pieces = 1, max_rest = 0;
    for (NetHost* n : nets) {
        if (n->dev.stdp_on)
            first_pieces = std::max<uint64_t>(first_pieces, (n->max_row_padded + kPlasticPiece - 1) / kPlasticPiece);
        first_pieces = std::max<uint64_t>(first_pieces, (n->max_first_padded + psz - 1) / psz);
        // (a plastic net's static sources defer their rows' rest too)
        max_rest = std::max<uint64_t>(max_rest, n->max_rest_padded);
    }
    const uint64_t cap_split = any_stdp ? 32 : 16;
    eng_.split_first = (uint32_t)std::min<uint64_t>(cap_split, first_pieces);
    eng_.split_rest = (uint32_t)std::min<uint64_t>(cap_split, std::max<uint64_t>(1, (max_rest + psz - 1) / psz));
    if (tuning_.scatter_split) eng_.split_first = eng_.split_rest = std::min<uint32_t>(tuning_.scatter_split, 64);
    eng_.queue_cap = (uint32_t)qentries;
    eng_.bins = bins;
    if (qentries * std::max(eng_.split_first, eng_.split_rest) > 0xFFFFFFFFull)
        throw Error(NAER_E_OVERFLOW, "spike list times warps per spike exceeds 2^32 work items");
    NAER_CK(cudaStreamSynchronize(stream_));  // tables and buffers complete for every stream
}

void Engine::set_tuning(const Tuning& t) {
    Tuning v = t;
    if (v.launch_steps == 0 || v.launch_steps > kDriveSlots)
        throw Error(NAER_E_INVALID, "launch_steps must be in 1.." + std::to_string(kDriveSlots));
    if (v.blocks_per_sm > 4) throw Error(NAER_E_INVALID, "blocks_per_sm must be in 0..4");
    if (v.scatter_piece != 0 && v.scatter_piece != 128 && v.scatter_piece != kScatterPiece)
        throw Error(NAER_E_INVALID, "scatter_piece must be 0, 128 or 256");
    if (v.neuron_state > NAER_STATE_GLOBAL) throw Error(NAER_E_INVALID, "unknown neuron_state");
    if (v.step_kernel > NAER_KERNEL_TWO_BARRIER) throw Error(NAER_E_INVALID, "unknown step_kernel");
    if (v.bins != 0 && (v.bins < 64 || v.bins > 8192 || (v.bins & (v.bins - 1))))
        throw Error(NAER_E_INVALID, "bins must be 0 or a power of two in 64..8192");
    tuning_ = v;
    if (!nets_.empty()) install(std::vector<NetHost*>(nets_), inst_raster_cap_, inst_record_, aggregation_);
}

TuneResult Engine::autotune(uint32_t trial_steps) {
    if (nets_.empty()) throw Error(NAER_E_STATE, "no network installed");
    TuneResult r;
    r.best = tuning_;
    if (trial_steps == 0) return r;
    DeviceGuard g(device_);
    cudaEvent_t e0, e1;
    NAER_CK(cudaEventCreate(&e0));
    NAER_CK(cudaEventCreate(&e1));
    auto trial = [&](const Tuning& t) {
        set_tuning(t);
        run(t.launch_steps);  // first launch of the new geometry
        NAER_CK(cudaEventRecord(e0, stream_));
        run(trial_steps);
        NAER_CK(cudaEventRecord(e1, stream_));
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
        const uint32_t auto_split = eng_.scatter_split;
        const uint32_t eng_piece_default = eng_.scatter_piece;
        for (uint32_t bps : {0u, 1u}) {
            for (uint32_t L : {kDriveSlots, kDriveSlots / 2}) {
                for (uint32_t sp : {0u, std::max<uint32_t>(1, auto_split / 2), std::min<uint32_t>(64, auto_split * 2)}) {
                    Tuning t;
                    t.blocks_per_sm = bps;
                    t.launch_steps = L;
                    t.scatter_split = sp;
                    // the other piece width with its own automatic split
                    t.scatter_piece = 0;
                    if (bps == 0 && L == kDriveSlots && sp == 0) {
                        t.scatter_piece = eng_piece_default == 128 ? kScatterPiece : 128u;
                    }
                    if (bps == 1 && L == kDriveSlots && sp == 0 && aggregation_ != NAER_AGG_DETERMINISTIC)
                        t.step_kernel = NAER_KERNEL_TWO_BARRIER;
                    // shared-memory binning of the ring reductions
                    if (bps == 0 && L == kDriveSlots / 2 && sp == 0 && aggregation_ == NAER_AGG_ATOMIC)
                        t.bins = 2048;
                    const double us = trial(t);
                    if (us < r.best_us_per_step) {
                        r.best_us_per_step = us;
                        r.best = t;
                    }
                }
            }
        }
        set_tuning(r.best);
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    NAER_CK(cudaEventDestroy(e0));
    NAER_CK(cudaEventDestroy(e1));
    return r;
}

void Engine::drop_graph() {
    if (graph_exec_) {
        NAER_CK(cudaStreamSynchronize(stream_));
        NAER_CK(cudaGraphExecDestroy(graph_exec_));
        graph_exec_ = nullptr;
        graph_launches_ = 0;
    }
}

void Engine::regrow(void*& p, size_t& have, size_t need) {
    need = std::max<size_t>(need, 16);
    if (need <= have && p) return;
    if (p) dfree(p, have);
    p = nullptr;  // nothing dangles if the allocation below fails
    have = 0;
    p = dalloc(need);
    have = need;
}

uint64_t Engine::sum_parts(const unsigned long long* d, uint32_t n) {
    if (!d || n == 0) return 0;
    std::vector<unsigned long long> h(n);
    NAER_CK(cudaMemcpyAsync(h.data(), d, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_));
    NAER_CK(cudaStreamSynchronize(stream_));
    uint64_t t = 0;
    for (auto x : h) t += x;
    return t;
}

uint64_t Engine::events_total() {
    DeviceGuard g(device_);
    const Ctl c = read_ctl();
    return events_base_ + c.events + sum_parts(d_ev_part_, ev_part_n_);
}

uint64_t Engine::overflow_total() {
    DeviceGuard g(device_);
    const Ctl c = read_ctl();
    return overflow_base_ + c.stdp_hist_overflow + sum_parts(d_ovf_part_, ev_part_n_);
}

// ---------------------------------------------------------------------------
// step loop

void Engine::launch_run(uint32_t steps) { launch_run_ex(steps, false); }

// One persistent launch.  from_ctl: the kernel takes its first step from
// Ctl::step (launches recorded in a CUDA graph); the cooperative attribute
// of cudaLaunchKernelEx keeps it capturable.
void Engine::launch_run_ex(uint32_t steps, bool from_ctl) {
    unsigned long long s0 = from_ctl ? kStepFromCtl : host_step_;
    static_assert(offsetof(Ctl, qtail) == offsetof(Ctl, bar_arrive) + 8, "Ctl layout");
    NAER_CK(cudaMemsetAsync(&d_ctl_->bar_arrive, 0, 8 + sizeof(d_ctl_->qtail), stream_));
    const bool timed = profiling_ && !from_ctl;
    if (timed) NAER_CK(cudaEventRecord(timer_event(), stream_));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(lif_grid_);
    cfg.blockDim = dim3(kLifThreads);
    cfg.dynamicSmemBytes = scatter_smem_;
    cfg.stream = stream_;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (aggregation_ == NAER_AGG_DETERMINISTIC) {
        if (use_smem_state_)
            NAER_CK(cudaLaunchKernelEx(&cfg, k_det_step<true>, eng_, s0, steps));
        else
            NAER_CK(cudaLaunchKernelEx(&cfg, k_det_step<false>, eng_, s0, steps));
    } else if (split_kernel_) {
        if (use_smem_state_)
            NAER_CK(cudaLaunchKernelEx(&cfg, k_step<true>, eng_, s0, steps));
        else
            NAER_CK(cudaLaunchKernelEx(&cfg, k_step<false>, eng_, s0, steps));
    } else {
        if (use_smem_state_)
            NAER_CK(cudaLaunchKernelEx(&cfg, k_run<true>, eng_, s0, steps));
        else
            NAER_CK(cudaLaunchKernelEx(&cfg, k_run<false>, eng_, s0, steps));
    }
    if (timed) {
        NAER_CK(cudaEventRecord(timer_event(), stream_));
        timer_kinds_.push_back(1);
    }
    if (!from_ctl) {
        ++launches_;
        host_step_ += steps;
    }
}

cudaEvent_t Engine::timer_event() {
    cudaEvent_t e;
    NAER_CK(cudaEventCreate(&e));
    timer_events_.push_back(e);
    return e;
}

// Sums the CUDA-event durations of the timed launches (pairs of events in
// launch order: drive kernels and persistent step kernels).
void Engine::resolve_timers() {
    if (timer_events_.empty()) return;
    NAER_CK(cudaStreamSynchronize(stream_));
    size_t e = 0;
    for (size_t i = 0; i < timer_kinds_.size(); ++i) {
        float ms = 0;
        NAER_CK(cudaEventElapsedTime(&ms, timer_events_[e], timer_events_[e + 1]));
        e += 2;
        if (timer_kinds_[i] == 0) {
            drive_ms_ += ms;
        } else {
            run_ms_ += ms;
            ++run_launches_;
        }
    }
    for (auto ev : timer_events_) cudaEventDestroy(ev);
    timer_events_.clear();
    timer_kinds_.clear();
    run_pairs_.clear();
}

void Engine::launch_drive(uint64_t s_first, uint32_t nsteps) {
    if (drive_grid_ == 0) {
        int occ = 0;
        NAER_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_drive, kLifThreads, 0));
        drive_grid_ = (uint32_t)std::max(1, occ) * (uint32_t)sm_count_;
    }
    // resident blocks only, each with an equal share of (chunk, step) items
    const uint32_t grid = std::max<uint32_t>(1, std::min<uint64_t>(drive_grid_, (uint64_t)eng_.n_chunks * nsteps));
    const bool from_ctl = s_first == kStepFromCtl;
    if (profiling_ && !from_ctl) NAER_CK(cudaEventRecord(timer_event(), stream_));
    k_drive<<<grid, kLifThreads, 0, stream_>>>(eng_, (unsigned long long)s_first, nsteps);
    if (!from_ctl) ++launches_;
    if (profiling_ && !from_ctl) {
        NAER_CK(cudaEventRecord(timer_event(), stream_));
        timer_kinds_.push_back(0);
    }
    NAER_CK(cudaGetLastError());
}

void Engine::run(uint64_t nsteps) {
    DeviceGuard g(device_);
    if (nets_.empty()) throw Error(NAER_E_STATE, "no network installed");
    check_usable();
    if (aggregation_ == NAER_AGG_DETERMINISTIC) ensure_det_scratch();
    run_launches(nsteps);
}

void Engine::run_launches(uint64_t nsteps) {
    // Poisson counts of a chunk of steps are drawn first (full occupancy),
    // then the persistent kernel simulates the chunk
    while (nsteps > 0) {
        const uint32_t n = (uint32_t)std::min<uint64_t>(nsteps, tuning_.launch_steps);
        launch_drive(host_step_, n);
        launch_run(n);
        nsteps -= n;
    }
    NAER_CK(cudaGetLastError());
}

uint64_t Engine::run_graph(uint64_t nsteps, uint32_t graph_launches) {
    DeviceGuard g(device_);
    if (nets_.empty()) throw Error(NAER_E_STATE, "no network installed");
    check_usable();
    if (graph_launches == 0) {
        run(nsteps);
        return 0;
    }
    if (aggregation_ == NAER_AGG_DETERMINISTIC) ensure_det_scratch();
    const uint32_t L = tuning_.launch_steps;
    const uint64_t per = (uint64_t)L * graph_launches;
    if (graph_exec_ && graph_launches_ != graph_launches) drop_graph();
    if (!graph_exec_ && nsteps >= per) {
        // record drive + step launches that read their first step from Ctl
        NAER_CK(cudaStreamSynchronize(stream_));
        NAER_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        cudaError_t err = cudaSuccess;
        try {
            for (uint32_t i = 0; i < graph_launches; ++i) {
                launch_drive(kStepFromCtl, L);
                launch_run_ex(L, true);
            }
        } catch (...) {
            cudaGraph_t gdrop = nullptr;
            cudaStreamEndCapture(stream_, &gdrop);
            if (gdrop) cudaGraphDestroy(gdrop);
            throw;
        }
        cudaGraph_t graph = nullptr;
        err = cudaStreamEndCapture(stream_, &graph);
        if (err == cudaSuccess) err = cudaGraphInstantiate(&graph_exec_, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        NAER_CK(err);
        graph_launches_ = graph_launches;
    }
    uint64_t done = 0;
    while (graph_exec_ && nsteps - done >= per) {
        NAER_CK(cudaGraphLaunch(graph_exec_, stream_));
        host_step_ += per;
        launches_ += 2ull * graph_launches;
        done += per;
    }
    run(nsteps - done);
    return done;
}

// ---------------------------------------------------------------------------
// Deterministic aggregation scratch (k_det_step): per net, the weight and the
// next event of every padded synapse (8 B per synapse) and the list head of
// every ring cell (4 B per cell, empty between steps).  The plain step keeps
// it in buffers each network owns, allocated by its first deterministic
// step; the fixed-scratch step carves it from one fixed device array.

void Engine::point_det_scratch(uint32_t mode) {
    for (size_t i = 0; i < nets_.size(); ++i) {
        const NetHost& n = *nets_[i];
        h_nets_[i].ev_w = n.det_w;
        h_nets_[i].ev_next = n.det_next;
        h_nets_[i].cell_head = n.det_head;
        if (mode == kScratchArena) {
            h_nets_[i].ev_w = arena_w_[i];
            h_nets_[i].ev_next = arena_next_[i];
            h_nets_[i].cell_head = arena_head_[i];
        }
    }
    NAER_CK(cudaMemcpyAsync(d_nets_, h_nets_.data(), h_nets_.size() * sizeof(NetDev), cudaMemcpyHostToDevice,
                            stream_));
    NAER_CK(cudaStreamSynchronize(stream_));  // h_nets_ is pageable host memory
    det_scratch_ = mode;
}

void Engine::ensure_det_scratch() {
    if (det_scratch_ == kScratchOwn) return;
    for (NetHost* n : nets_) {
        if (det_syn_entries(*n) >= kNoEvent || det_cells(*n) >= 0xFFFFFFFFull)
            throw Error(NAER_E_OVERFLOW, "deterministic aggregation needs fewer than 2^32 synapses and ring cells per "
                                         "network");
        if (n->det_w) continue;
        n->det_w = static_cast<float*>(dalloc(det_syn_entries(*n) * 4ull));
        n->det_next = static_cast<uint32_t*>(dalloc(det_syn_entries(*n) * 4ull));
        n->det_head = static_cast<uint32_t*>(dalloc(det_cells(*n) * 4ull));
        NAER_CK(cudaMemsetAsync(n->det_head, 0xFF, det_cells(*n) * 4ull, stream_));
        n->device_bytes += det_syn_entries(*n) * 8ull + det_cells(*n) * 4ull;
    }
    point_det_scratch(kScratchOwn);
}

// ---------------------------------------------------------------------------
// Deterministic steps with no allocation (naer_net_step_noalloc).  The
// scratch above is carved from one fixed device array of this library
// instead of buffers the network allocates.  Its size bounds the networks
// the call accepts.  One array exists per device and is shared by every
// engine on that device: calls whose GPU work overlaps race on it.

constexpr size_t kFixedScratchBytes = 32ull << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_fixed_scratch[kFixedScratchBytes];

namespace {
size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Device address of this device's copy of the array, looked up once per
// device with that device current (a host-side reference to the array is
// not a device address).
unsigned char* fixed_scratch_base(int device) {
    static std::mutex mu;
    static std::vector<unsigned char*> base;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)base.size() <= device) base.resize(device + 1, nullptr);
    if (!base[device]) {
        void* p = nullptr;
        NAER_CK(cudaGetSymbolAddress(&p, g_fixed_scratch));
        base[device] = static_cast<unsigned char*>(p);
    }
    return base[device];
}
}  // namespace

void Engine::run_fixed_scratch(uint64_t nsteps) {
    DeviceGuard g(device_);
    if (nets_.empty()) throw Error(NAER_E_STATE, "no network installed");
    check_usable();
    if (aggregation_ != NAER_AGG_DETERMINISTIC)
        throw Error(NAER_E_STATE, "the fixed-scratch step needs a network compiled with deterministic aggregation");
    // partition (sizes first: a network that does not fit is refused before
    // anything changes)
    size_t used = 0;
    std::vector<size_t> off_w, off_next, off_head;
    uint64_t syn = 0, cells = 0;
    for (const NetHost* n : nets_) {
        if (det_syn_entries(*n) >= kNoEvent || det_cells(*n) >= 0xFFFFFFFFull)
            throw Error(NAER_E_OVERFLOW, "network too large for deterministic aggregation");
        off_w.push_back(used);
        used = align256(used + det_syn_entries(*n) * 4ull);
        off_next.push_back(used);
        used = align256(used + det_syn_entries(*n) * 4ull);
        off_head.push_back(used);
        used = align256(used + det_cells(*n) * 4ull);
        syn += det_syn_entries(*n);
        cells += det_cells(*n);
    }
    if (used > kFixedScratchBytes)
        throw Error(NAER_E_OVERFLOW,
                    "network too large for the fixed-scratch step: its " + std::to_string(syn) +
                        " padded synapses and " + std::to_string(cells) + " ring cells need " +
                        std::to_string(used) + " bytes of scratch (8 per synapse, 4 per ring cell); the fixed "
                        "arena holds " + std::to_string(kFixedScratchBytes) + " bytes");
    unsigned char* a = fixed_scratch_base(device_);
    arena_w_.assign(nets_.size(), nullptr);
    arena_next_.assign(nets_.size(), nullptr);
    arena_head_.assign(nets_.size(), nullptr);
    for (size_t i = 0; i < nets_.size(); ++i) {
        arena_w_[i] = reinterpret_cast<float*>(a + off_w[i]);
        arena_next_[i] = reinterpret_cast<uint32_t*>(a + off_next[i]);
        arena_head_[i] = reinterpret_cast<uint32_t*>(a + off_head[i]);
        // the array keeps the last call's contents (any network's): every
        // list head must start empty
        NAER_CK(cudaMemsetAsync(arena_head_[i], 0xFF, det_cells(*nets_[i]) * 4ull, stream_));
    }
    point_det_scratch(kScratchArena);
    run_launches(nsteps);
}

void Engine::sync() {
    DeviceGuard g(device_);
    NAER_CK(cudaStreamSynchronize(stream_));
    NAER_CK(cudaGetLastError());
}

void Engine::set_barrier_limit(uint64_t limit_ns) {
    DeviceGuard g(device_);
    const unsigned long long v = limit_ns;
    std::memcpy(h_pinned_ + 64, &v, 8);
    NAER_CK(cudaMemcpyAsync(&d_ctl_->bar_limit_ns, h_pinned_ + 64, 8, cudaMemcpyHostToDevice, stream_));
    NAER_CK(cudaStreamSynchronize(stream_));
}

void Engine::set_barrier_skew(uint64_t skew) {
    DeviceGuard g(device_);
    const unsigned long long v = skew;
    std::memcpy(h_pinned_ + 66, &v, 8);
    NAER_CK(cudaMemcpyAsync(&d_ctl_->bar_skew, h_pinned_ + 66, 8, cudaMemcpyHostToDevice, stream_));
    NAER_CK(cudaStreamSynchronize(stream_));
}

int Engine::device_status() {
    const Ctl c = read_ctl();
    if (c.error == 0) return 0;
    failed_ = true;
    return c.error == (unsigned int)(-NAER_STATUS_TIMEOUT) ? NAER_E_TIMEOUT : NAER_E_CUDA;
}

void Engine::check_usable() const {
    if (failed_)
        throw Error(NAER_E_STATE,
                    "a previous launch reported a device error (bounded wait ran out): the network's state is "
                    "undefined; destroy the handle");
}

Ctl Engine::read_ctl() {
    DeviceGuard g(device_);
    static_assert(sizeof(Ctl) <= 256, "control block copy must fit the first half of the pinned staging");
    Ctl c;
    NAER_CK(cudaMemcpyAsync(h_pinned_, d_ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost, stream_));
    NAER_CK(cudaStreamSynchronize(stream_));
    std::memcpy(&c, h_pinned_, sizeof(Ctl));
    return c;
}

uint64_t Engine::read_raster(uint64_t first, uint64_t cap, uint32_t* steps, uint32_t* ids) {
    const Ctl c = read_ctl();
    const uint64_t total = std::min<uint64_t>(c.raster_next, eng_.raster_cap);
    if (first >= total || cap == 0) return 0;
    const uint64_t n = std::min<uint64_t>(cap, total - first);
    std::vector<uint2> rec(n);
    DeviceGuard g(device_);
    NAER_CK(cudaMemcpyAsync(rec.data(), d_raster_ + first, n * sizeof(uint2), cudaMemcpyDeviceToHost,
                            stream_));
    NAER_CK(cudaStreamSynchronize(stream_));
    // records of one step are contiguous; order them by address
    uint64_t a = 0;
    while (a < n) {
        uint64_t b = a + 1;
        while (b < n && rec[b].x == rec[a].x) ++b;
        std::sort(rec.begin() + a, rec.begin() + b,
                  [](const uint2& l, const uint2& r) { return l.y < r.y; });
        a = b;
    }
    for (uint64_t i = 0; i < n; ++i) {
        steps[i] = rec[i].x;
        ids[i] = rec[i].y;
    }
    return n;
}

// ---------------------------------------------------------------------------
// Simulation state of one network between steps: membrane potentials,
// refractory counters, the delay ring (slots in the network's own step
// time), and with plasticity the weights, post rows and pre traces.  The
// connectivity itself is regenerated bit for bit from the description and
// the Poisson drive from the step counter (counter-based Philox), so
// neither is stored.  Layout: V f32[Ns] | refr u8[Ns] (padded to 4) |
// ring f32[D * Ns] | with plasticity: w f32[S] | post i32[Np * stride] |
// pre int2[Np].

uint64_t state_bytes(const NetHost& n) {
    const uint64_t Ns = n.n_storage;
    uint64_t b = Ns * 4ull + ((Ns + 3ull) & ~3ull) + (uint64_t)n.ring_slots * Ns * 4ull;
    if (n.dev.stdp_on) {
        b += n.synapses_padded * 4ull;
        b += (uint64_t)n.n_plastic * n.post_stride * 4ull + (uint64_t)n.n_plastic * 8ull;
    }
    return b;
}

void Engine::save_state(const NetHost& n, uint8_t* dst) {
    DeviceGuard g(device_);
    const uint64_t Ns = n.n_storage;
    uint8_t* p = dst;
    auto copy = [&](const void* src, uint64_t bytes, uint64_t advance) {
        if (bytes) NAER_CK(cudaMemcpyAsync(p, src, bytes, cudaMemcpyDeviceToHost, stream_));
        p += advance;
    };
    copy(n.v, Ns * 4ull, Ns * 4ull);
    copy(n.refr, Ns, (Ns + 3ull) & ~3ull);
    copy(n.ring, (uint64_t)n.ring_slots * Ns * 4ull, (uint64_t)n.ring_slots * Ns * 4ull);
    if (n.dev.stdp_on) {
        copy(n.w, n.synapses_padded * 4ull, n.synapses_padded * 4ull);
        copy(n.post, (uint64_t)n.n_plastic * n.post_stride * 4ull, (uint64_t)n.n_plastic * n.post_stride * 4ull);
        copy(n.pre, (uint64_t)n.n_plastic * 8ull, (uint64_t)n.n_plastic * 8ull);
    }
    NAER_CK(cudaStreamSynchronize(stream_));
}

void Engine::load_state(NetHost& n, const uint8_t* src) {
    DeviceGuard g(device_);
    const uint64_t Ns = n.n_storage;
    const uint8_t* p = src;
    auto copy = [&](void* dst, uint64_t bytes, uint64_t advance) {
        if (bytes) NAER_CK(cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, stream_));
        p += advance;
    };
    copy(n.v, Ns * 4ull, Ns * 4ull);
    copy(n.refr, Ns, (Ns + 3ull) & ~3ull);
    copy(n.ring, (uint64_t)n.ring_slots * Ns * 4ull, (uint64_t)n.ring_slots * Ns * 4ull);
    if (n.dev.stdp_on) {
        copy(n.w, n.synapses_padded * 4ull, n.synapses_padded * 4ull);
        copy(n.post, (uint64_t)n.n_plastic * n.post_stride * 4ull, (uint64_t)n.n_plastic * n.post_stride * 4ull);
        copy(n.pre, (uint64_t)n.n_plastic * 8ull, (uint64_t)n.n_plastic * 8ull);
    }
    NAER_CK(cudaStreamSynchronize(stream_));  // the source is host memory the caller may reuse
}

void Engine::set_step(uint64_t step, uint64_t events) {
    DeviceGuard g(device_);
    drop_graph();
    host_step_ = step;
    // the step counter, an empty raster, the event counters restarted from
    // the saved total
    NAER_CK(cudaStreamSynchronize(stream_));
    Ctl c = read_ctl();
    c.step = step;
    c.raster_base = c.raster_next = c.raster_dropped = 0;
    c.events = 0;
    std::memcpy(h_pinned_, &c, sizeof(Ctl));
    NAER_CK(cudaMemcpyAsync(d_ctl_, h_pinned_, sizeof(Ctl), cudaMemcpyHostToDevice, stream_));
    NAER_CK(cudaMemsetAsync(d_ev_part_, 0, ev_part_n_ * sizeof(unsigned long long), stream_));
    NAER_CK(cudaStreamSynchronize(stream_));
    events_base_ = events;
}

uint64_t Engine::read_raster_raw(uint64_t first, uint64_t cap, uint32_t* records) {
    const Ctl c = read_ctl();
    const uint64_t total = std::min<uint64_t>(c.raster_next, eng_.raster_cap);
    if (first >= total || cap == 0) return 0;
    const uint64_t n = std::min<uint64_t>(cap, total - first);
    DeviceGuard g(device_);
    NAER_CK(cudaMemcpyAsync(records, d_raster_ + first, n * sizeof(uint2), cudaMemcpyDeviceToHost, stream_));
    NAER_CK(cudaStreamSynchronize(stream_));
    return n;
}

uint64_t Engine::harvest_raster(uint2* dst, cudaEvent_t copied, uint64_t* dropped) {
    const Ctl c = read_ctl();
    const uint64_t n = std::min<uint64_t>(c.raster_next, eng_.raster_cap);
    if (dropped) *dropped = c.raster_dropped;
    DeviceGuard g(device_);
    if (n) NAER_CK(cudaMemcpyAsync(dst, d_raster_, n * sizeof(uint2), cudaMemcpyDeviceToHost, stream_));
    NAER_CK(cudaEventRecord(copied, stream_));
    clear_raster();
    return n;
}

void Engine::clear_raster() {
    DeviceGuard g(device_);
    // raster_base, raster_next, raster_dropped: three adjacent words, reset
    // in stream order
    static_assert(offsetof(Ctl, raster_dropped) == offsetof(Ctl, raster_base) + 16, "Ctl layout");
    NAER_CK(cudaMemsetAsync(&d_ctl_->raster_base, 0, 24, stream_));
}

void Engine::set_profiling(bool on) {
    DeviceGuard g(device_);
    // the persistent kernel always times its phases; enabling resets the totals
    resolve_timers();
    if (on) {
        drive_ms_ = run_ms_ = 0;
        run_launches_ = 0;
        sync();
        const unsigned long long z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        NAER_CK(cudaMemcpy(&d_ctl_->prof_lif_ns, z, sizeof(z), cudaMemcpyHostToDevice));
    }
    profiling_ = on;
}

void Engine::get_launch_times(double* drive_ms, double* run_ms, uint64_t* run_launches) {
    DeviceGuard g(device_);
    resolve_timers();
    if (drive_ms) *drive_ms = drive_ms_;
    if (run_ms) *run_ms = run_ms_;
    if (run_launches) *run_launches = run_launches_;
}

void Engine::get_phases(double* ms5) {
    const Ctl c = read_ctl();
    for (int q = 0; q < 5; ++q) ms5[q] = c.prof_phase_ns[q] * 1e-6;
}

void Engine::get_profile(double* lif_ms, double* scatter_ms, uint64_t* launches) {
    const Ctl c = read_ctl();
    if (lif_ms) *lif_ms = c.prof_lif_ns * 1e-6;
    if (scatter_ms) *scatter_ms = c.prof_scatter_ns * 1e-6;
    if (launches) *launches = c.prof_steps;
}

}  // namespace naer
