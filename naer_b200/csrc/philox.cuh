// Philox4x32-10 counter-based generator and the reference's draw helpers.
//
// Philox4x32-10 is restated from its published description (Salmon, Moraes,
// Dror, Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3", SC'11): four
// 32-bit counter words, two 32-bit key words, ten rounds.  Each round
// multiplies counter words 0 and 2 by two fixed odd constants (64-bit
// product split hi/lo), xors the high halves with the other counter words and
// the key, and permutes; the key is bumped by two Weyl constants between
// rounds.  The reference calls it through Random123's `philox4x32(c, k)`
// (include/naer/kernels/random.cl:8-16), a git submodule that is not vendored.
//
// The helpers below follow the reference's call sites exactly:
//   uniform_rand  include/naer/kernels/random.cl:6-24   key {gid, seed}, ctr {iter,0,0,0},
//                                                       word z / 4294967295.0 as double
//   exprnd        include/naer/kernels/random.cl:26-30  log(1 - x) / (-(rate / 1e6)) microseconds
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define NAER_HD __host__ __device__ __forceinline__
#else
#define NAER_HD inline
#endif

namespace naer {

struct u32x4 {
    uint32_t v[4];
};

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;  // golden ratio
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;  // sqrt(3) - 1

// One 32 x 32 -> 64-bit multiply (mul.wide.u32) gives both halves: on the
// GPU the rounds are bound by the integer-multiply pipe, so hi and lo are
// not computed by two separate multiplies.
NAER_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    lo = (uint32_t)p;
    hi = (uint32_t)(p >> 32);
}

// Full Philox4x32-10: returns all four output words.
NAER_HD u32x4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                            uint32_t k0, uint32_t k1) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += kPhiloxW0;
            k1 += kPhiloxW1;
        }
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(kPhiloxM0, c0, hi0, lo0);
        mulhilo32(kPhiloxM1, c2, hi1, lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    u32x4 out;
    out.v[0] = c0;
    out.v[1] = c1;
    out.v[2] = c2;
    out.v[3] = c3;
    return out;
}

// Word z (index 2) only, for counter {c0, 0, 0, 0}: the reference's
// uniform_rand draw (random.cl:8-23).  Same rounds as above; the compiler
// drops the dead words of the last round.
NAER_HD uint32_t philox_ref_z(uint32_t c0, uint32_t k0, uint32_t k1) {
    return philox4x32_10(c0, 0u, 0u, 0u, k0, k1).v[2];
}

// philox_ref_z(c0, k0, k1) with the one product that does not depend on
// the counter supplied by the caller: round 1 leaves key word k0 in counter
// word 0, so round 2 multiplies M0 by k0.  m_hi:m_lo = M0 * k0 (64-bit).
// A generator draws for the same neuron (same k0) at every step, so the
// product is computed once per neuron instead of once per draw.
NAER_HD uint32_t philox_ref_z_pre(uint32_t c0, uint32_t k0, uint32_t k1, uint32_t m_hi, uint32_t m_lo) {
    uint32_t h, l;
    mulhilo32(kPhiloxM0, c0, h, l);  // round 1; counter words 1-3 are zero
    uint32_t x0 = k0, x1 = 0u, x2 = h ^ k1, x3 = l;
    k0 += kPhiloxW0;
    k1 += kPhiloxW1;
    uint32_t h1, l1;
    mulhilo32(kPhiloxM1, x2, h1, l1);  // round 2; M0 * x0 is m_hi:m_lo
    {
        const uint32_t n0 = h1 ^ x1 ^ k0;
        const uint32_t n2 = m_hi ^ x3 ^ k1;
        x0 = n0;
        x1 = l1;
        x2 = n2;
        x3 = m_lo;
    }
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 2; r < 10; ++r) {
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(kPhiloxM0, x0, hi0, lo0);
        mulhilo32(kPhiloxM1, x2, hi1, lo1);
        const uint32_t n0 = hi1 ^ x1 ^ k0;
        const uint32_t n2 = hi0 ^ x3 ^ k1;
        x0 = n0;
        x1 = lo1;
        x2 = n2;
        x3 = lo0;
    }
    return x2;
}

// Work-item id the reference's kernels see for element `idx` of a type laid
// out in groups of `capacity` elements processed by workgroups of `wg` items
// with a strided loop (input_neuron_group.cl:17,26): get_global_id(0) =
// group * wg + (idx % capacity) % wg.
NAER_HD uint32_t ref_global_id(uint32_t idx, uint32_t capacity, uint32_t wg) {
    return (idx / capacity) * wg + (idx % capacity) % wg;
}

// Reference Poisson generator geometry: capacity 2048, workgroup 128
// (include/naer/Network.h:110-119).
constexpr uint32_t kPoissonCapacity = 2048;
constexpr uint32_t kPoissonWorkgroup = 128;

// The reference's exponential draw, truncated to whole microseconds as in
// input_neuron_group.cl:29,37 ((uint)exprnd_fast(...)).  z == 0xFFFFFFFF
// gives x == 1.0 and log(0) == -inf: the reference's cast of +inf is
// undefined; here it saturates to 0xFFFFFFFF (no further spike in any window).
NAER_HD uint32_t ref_exp_interval_us(uint32_t z, double rate_hz) {
    if (z == 0xFFFFFFFFu) return 0xFFFFFFFFu;
    double x = (double)z / 4294967295.0;
    double dt = log(1.0 - x) / (-(rate_hz / 1000000.0));
#if defined(__CUDA_ARCH__)
    return __double2uint_rz(dt);
#else
    if (!(dt < 4294967296.0)) return 0xFFFFFFFFu;
    return (uint32_t)dt;
#endif
}

}  // namespace naer
