// Grid-wide barrier of the persistent kernels, shared with the device probe.
#pragma once
#include <cuda_runtime.h>

#include "engine_types.cuh"

namespace naer {

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Limits of a launch's grid barriers, read from the control block once per
// launch (the host sets them between launches).
struct BarrierCfg {
    unsigned long long limit_ns;  // bounded wait of one barrier
    unsigned long long skew;      // added to every target (0 in normal operation)
};

__device__ __forceinline__ BarrierCfg barrier_cfg(const Ctl* ctl) {
    BarrierCfg b;
    b.limit_ns = ctl->bar_limit_ns ? ctl->bar_limit_ns : kBarrierLimitNs;
    b.skew = ctl->bar_skew;
    return b;
}

// Grid-wide barrier of the persistent kernels: every block adds one to an
// arrival counter (zeroed by the host before each launch) with a release
// reduction and waits until it reaches `target` (barrier number times the
// grid size).  The wait is bounded: after cfg.limit_ns the block records
// NAER_E_TIMEOUT in ctl->error and reports failure, and the kernel returns.
// Co-residency of all blocks is guaranteed by the cooperative launch.
__device__ __forceinline__ bool grid_barrier(Ctl* ctl, unsigned long long target, const BarrierCfg& cfg) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1;
        __threadfence();  // this block's stores and reductions are visible before it arrives
        asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(&ctl->bar_arrive) : "memory");
        const unsigned long long t0 = globaltimer_ns();
        const unsigned long long goal = target + cfg.skew;
        unsigned long long cur;
        for (;;) {
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(cur) : "l"(&ctl->bar_arrive) : "memory");
            if (cur >= goal) break;
            if (globaltimer_ns() - t0 > cfg.limit_ns) {
                atomicCAS(&ctl->error, 0u, (unsigned int)(-NAER_STATUS_TIMEOUT));
                s_ok = 0;
                break;
            }
            __nanosleep(20);
        }
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace naer
