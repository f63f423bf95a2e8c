// Device probe: the ceilings the step kernel is measured against, timed by
// the library itself on the device it runs on.
//
//  - random-address fp32 reductions (red.global.add.f32, one per event of the
//    scatter) into buffers of a given number of cells: the rate at which the
//    ring accumulation of the atomic mode can absorb events;
//  - random-address 4-byte stores into the same buffers (a write with no
//    read-modify-write, for comparison);
//  - one grid barrier of the persistent kernels (grid_sync.cuh), at one and
//    two resident blocks per SM, in a cooperative launch;
//  - a streaming read of a buffer larger than L2 with the scatter's
//    evict-first 128-bit loads.
//
// Addresses come from a per-thread xorshift generator; every kernel is sized
// so each launch runs for a few milliseconds.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.h"
#include "grid_sync.cuh"
#include "philox.cuh"

namespace naer {

namespace {

__device__ __forceinline__ uint32_t xorshift32(uint32_t x) {
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    return x;
}

__device__ __forceinline__ uint32_t seed_of(uint32_t tid, uint32_t salt) {
    uint32_t x = tid * 0x9E3779B9u + salt * 0x85EBCA6Bu + 0x632BE5ABu;
    x = xorshift32(x ? x : 1u);
    return xorshift32(x);
}

__device__ __forceinline__ uint32_t pick(uint32_t x, uint32_t n) { return (uint32_t)(((uint64_t)x * n) >> 32); }

__global__ void __launch_bounds__(256) k_probe_red(float* buf, uint32_t cells, uint32_t iters, uint32_t salt) {
    uint32_t x = seed_of(blockIdx.x * blockDim.x + threadIdx.x, salt);
    for (uint32_t i = 0; i < iters; i += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            x = xorshift32(x);
            asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(buf + pick(x, cells)), "f"(1.0f) : "memory");
        }
    }
}

__global__ void __launch_bounds__(256) k_probe_store(float* buf, uint32_t cells, uint32_t iters, uint32_t salt) {
    uint32_t x = seed_of(blockIdx.x * blockDim.x + threadIdx.x, salt);
    for (uint32_t i = 0; i < iters; i += 4) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            x = xorshift32(x);
            __stcg(buf + pick(x, cells), 1.0f);
        }
    }
}

__global__ void __launch_bounds__(256) k_probe_stream(const uint4* in, uint64_t n16, uint32_t* out) {
    uint32_t acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint4 v = __ldcs(in + i);
        acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if (acc == 0x9E3779B9u) out[0] = acc;  // keeps the loads; practically never taken
}

__global__ void __launch_bounds__(256) k_probe_barrier(Ctl* ctl, uint32_t n) {
    const BarrierCfg cfg = barrier_cfg(ctl);
    unsigned long long target = 0;
    for (uint32_t i = 0; i < n; ++i) {
        target += gridDim.x;
        if (!grid_barrier(ctl, target, cfg)) return;
    }
}

// The Poisson generator's interval (input_neuron_group.cl:29,37 through
// random.cl:26-30) of generator outputs z = z_first + i * z_step (mod 2^32),
// exactly as the drive kernels compute it on the device.
__global__ void k_probe_intervals(double rate, uint32_t z_first, uint32_t z_step, uint64_t count, uint32_t* out) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = ref_exp_interval_us(z_first + (uint32_t)i * z_step, rate);
}

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t st;
    explicit Timer(cudaStream_t s) : st(s) {
        NAER_CK(cudaEventCreate(&a));
        NAER_CK(cudaEventCreate(&b));
    }
    ~Timer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    void start() { NAER_CK(cudaEventRecord(a, st)); }
    double stop_ms() {
        NAER_CK(cudaEventRecord(b, st));
        NAER_CK(cudaEventSynchronize(b));
        float ms = 0;
        NAER_CK(cudaEventElapsedTime(&ms, a, b));
        return ms;
    }
};

}  // namespace

void probe_device(int device, uint64_t ring_cells, uint64_t small_cells, naer_device_probe* out) {
    int prev = -1;
    NAER_CK(cudaGetDevice(&prev));
    NAER_CK(cudaSetDevice(device));
    int sms = 0;
    NAER_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    cudaStream_t st = nullptr;
    NAER_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    float* buf = nullptr;
    uint4* big = nullptr;
    Ctl* ctl = nullptr;
    uint32_t* sink = nullptr;
    const uint64_t big_bytes = 4ull << 30;  // streamed: 4 GiB, 32x the L2
    try {
        if (ring_cells == 0 || ring_cells > 0xFFFFFFFFull || small_cells == 0 || small_cells > ring_cells)
            throw Error(NAER_E_INVALID, "probe sizes must satisfy 0 < small_cells <= ring_cells < 2^32");
        NAER_CK(cudaMalloc(&buf, ring_cells * 4ull));
        NAER_CK(cudaMemsetAsync(buf, 0, ring_cells * 4ull, st));
        NAER_CK(cudaMalloc(&big, big_bytes));
        NAER_CK(cudaMemsetAsync(big, 0, big_bytes, st));
        NAER_CK(cudaMalloc(&ctl, sizeof(Ctl)));
        NAER_CK(cudaMalloc(&sink, 4));
        Timer tm(st);
        const uint32_t grid = (uint32_t)sms * 8, threads = 256, iters = 256;
        const double ops = (double)grid * threads * iters;
        auto best_rate = [&](auto&& launch) {
            double best = 0;
            for (int rep = 0; rep < 4; ++rep) {  // first repetition warms up
                tm.start();
                launch((uint32_t)rep);
                const double ms = tm.stop_ms();
                NAER_CK(cudaGetLastError());
                if (rep > 0) best = std::max(best, ops / (ms * 1e-3));
            }
            return best;
        };
        std::memset(out, 0, sizeof(*out));
        out->ring_cells = ring_cells;
        out->small_cells = small_cells;
        out->red_ring_per_s = best_rate([&](uint32_t r) {
            k_probe_red<<<grid, threads, 0, st>>>(buf, (uint32_t)ring_cells, iters, r);
        });
        out->red_small_per_s = best_rate([&](uint32_t r) {
            k_probe_red<<<grid, threads, 0, st>>>(buf, (uint32_t)small_cells, iters, r);
        });
        out->store_ring_per_s = best_rate([&](uint32_t r) {
            k_probe_store<<<grid, threads, 0, st>>>(buf, (uint32_t)ring_cells, iters, r);
        });
        // streaming read
        {
            double best = 0;
            for (int rep = 0; rep < 3; ++rep) {
                tm.start();
                k_probe_stream<<<(uint32_t)sms * 8, 256, 0, st>>>(big, big_bytes / 16, sink);
                const double ms = tm.stop_ms();
                NAER_CK(cudaGetLastError());
                if (rep > 0) best = std::max(best, (double)big_bytes / (ms * 1e-3) / 1e9);
            }
            out->stream_gbs = best;
        }
        // grid barriers: cooperative launches of 1 and 2 blocks per SM
        const uint32_t nbar = 2000;
        for (int bps = 1; bps <= 2; ++bps) {
            double best = 1e30;
            for (int rep = 0; rep < 3; ++rep) {
                NAER_CK(cudaMemsetAsync(ctl, 0, sizeof(Ctl), st));
                cudaLaunchConfig_t cfg{};
                cfg.gridDim = dim3((uint32_t)bps * sms);
                cfg.blockDim = dim3(256);
                cfg.stream = st;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeCooperative;
                attr[0].val.cooperative = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                tm.start();
                NAER_CK(cudaLaunchKernelEx(&cfg, k_probe_barrier, ctl, nbar));
                const double ms = tm.stop_ms();
                Ctl c;
                NAER_CK(cudaMemcpy(&c, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
                if (c.error) throw Error(NAER_E_TIMEOUT, "probe barrier timed out");
                if (rep > 0) best = std::min(best, ms * 1e3 / nbar);
            }
            (bps == 1 ? out->barrier_us_1 : out->barrier_us_2) = best;
        }
        out->grid = (uint32_t)sms;
    } catch (...) {
        cudaStreamSynchronize(st);
        if (buf) cudaFree(buf);
        if (big) cudaFree(big);
        if (ctl) cudaFree(ctl);
        if (sink) cudaFree(sink);
        cudaStreamDestroy(st);
        cudaSetDevice(prev);
        throw;
    }
    cudaStreamSynchronize(st);
    cudaFree(buf);
    cudaFree(big);
    cudaFree(ctl);
    cudaFree(sink);
    cudaStreamDestroy(st);
    cudaSetDevice(prev);
}

void probe_intervals(int device, double rate_hz, uint32_t z_first, uint32_t z_step, uint64_t count,
                     uint32_t* out) {
    int prev = -1;
    NAER_CK(cudaGetDevice(&prev));
    NAER_CK(cudaSetDevice(device));
    uint32_t* d = nullptr;
    const cudaError_t e = cudaMalloc(&d, std::max<uint64_t>(count, 1) * 4ull);
    if (e != cudaSuccess) {
        cudaSetDevice(prev);
        NAER_CK(e);
    }
    k_probe_intervals<<<1184, 256>>>(rate_hz, z_first, z_step, count, d);
    cudaError_t e2 = cudaGetLastError();
    if (e2 == cudaSuccess && count) e2 = cudaMemcpy(out, d, count * 4ull, cudaMemcpyDeviceToHost);
    cudaFree(d);
    cudaSetDevice(prev);
    NAER_CK(e2);
}

}  // namespace naer
