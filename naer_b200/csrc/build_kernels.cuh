// Connectivity generation on the device.
//
// Row order of a source (the order the scatter visits synapses, which fixes
// the deterministic aggregation order): connections in declaration order;
// inside one connection, REF_BERNOULLI by ascending target, FIXED_OUTDEGREE
// by draw index k, FIXED_INDEGREE by ascending (target, k); finally a stable
// partition puts the delay-1 synapses first.  In device memory the two parts
// of a row each start on a 16-byte boundary (sentinel padding between and
// after them); row_mid holds the offset of the second part.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "engine_types.cuh"
#include "philox.cuh"

namespace naer {

struct ConnBuild {
    uint32_t rule;
    uint32_t K;
    double p;
    float weight, wmin, wmax;
    uint32_t dmin, dmax;
    uint32_t seed_lo, seed_hi;
    uint32_t src_size, dst_size;
    uint32_t src_storage, dst_storage;
};

// Uniform weight in [wmin, wmax) from x in [0, 1] as float; the reference's
// random_weight (include/naer/kernels/network.cl:4-12) with the operations
// rounded one by one (no contraction).
__host__ __device__ inline float conn_uniform_weight(float wmin, float wmax, float x) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(wmin, __fmul_rn(__fsub_rn(wmax, wmin), x));
#else
    return wmin + (wmax - wmin) * x;  // built with -ffp-contract=off
#endif
}

__host__ __device__ inline uint32_t conn_delay(uint32_t dmin, uint32_t dmax, uint32_t word) {
    if (dmax <= dmin) return dmin;
    const uint32_t span = dmax - dmin + 1u;
#if defined(__CUDA_ARCH__)
    return dmin + __umulhi(word, span);
#else
    return dmin + (uint32_t)(((uint64_t)word * span) >> 32);
#endif
}

__host__ __device__ inline uint32_t conn_pick(uint32_t word, uint32_t n) {
#if defined(__CUDA_ARCH__)
    return __umulhi(word, n);
#else
    return (uint32_t)(((uint64_t)word * n) >> 32);
#endif
}

// 24-bit uniform in [0, 1) as an exact float
__host__ __device__ inline float conn_unit_float(uint32_t word) {
    return (float)(word >> 8) * (1.0f / 16777216.0f);
}

__global__ void k_fill_u32(uint32_t* a, uint64_t n, uint32_t v);
__global__ void k_bern_count(ConnBuild cb, uint32_t* cnt);
__global__ void k_bern_fill(ConnBuild cb, const uint64_t* cursor, uint32_t* tgt, float* w,
                            uint8_t* dly);
__global__ void k_outdeg_fill(ConnBuild cb, const uint64_t* cursor, uint32_t* tgt, float* w,
                              uint8_t* dly);
__global__ void k_indeg_count(ConnBuild cb, uint32_t* cnt);
// [0] += synapses, [1] = max padded row, [3] = max padded delay-1 part, [4] = max padded rest
__global__ void k_row_stats(const uint64_t* len, const uint64_t* padded, const uint32_t* n1, uint32_t n,
                            unsigned long long* out);
__global__ void k_indeg_keys(ConnBuild cb, uint32_t* keys, uint32_t* vals);
__global__ void k_explicit_fill(ConnBuild cb, const uint64_t* rp, const uint32_t* tg, const float* wv,
                                const uint8_t* dv, const uint64_t* cursor, uint32_t* tgt, float* w, uint8_t* dly);
__global__ void k_indeg_finalize(ConnBuild cb, const uint32_t* keys, const uint32_t* vals, uint64_t total,
                                 const uint64_t* conn_off, const uint64_t* cursor, uint32_t* tgt,
                                 float* w, uint8_t* dly);
__global__ void k_row_len_add(const uint32_t* cnt, uint32_t src_size, uint32_t src_storage,
                              uint64_t* len);
__global__ void k_row_pad(const uint64_t* len, uint32_t n, uint64_t* padded);
__global__ void k_cursor_advance(const uint32_t* cnt, uint32_t src_size, uint32_t src_storage,
                                 uint64_t* cursor);
__global__ void k_pad_fill(const uint64_t* row_ptr, const uint64_t* len, uint32_t n, uint32_t* tgt,
                           float* w, uint8_t* dly);
__global__ void k_count_d1(const uint64_t* row_ptr, const uint64_t* len, uint32_t n, const uint8_t* dly,
                           uint32_t* n1);
__global__ void k_row_pad_split(const uint64_t* len, const uint32_t* n1, uint32_t n, uint64_t* padded);
__global__ void k_exact_inputs(const uint32_t* tgt, const float* w, uint64_t n, uint32_t* in,
                               unsigned int* maxw_bits);
__global__ void k_max_u32(const uint32_t* a, uint32_t n, unsigned int* out);
__global__ void k_partition_d1(const uint64_t* row_ptr, const uint64_t* len, const uint32_t* n1, uint32_t n,
                               const uint64_t* row_ptr2, const uint32_t* tgt, const float* w, const uint8_t* dly,
                               uint32_t* tgt2, float* w2, uint8_t* dly2, uint32_t* row_mid);

}  // namespace naer
