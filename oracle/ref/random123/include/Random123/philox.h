/* Stand-in for Random123's philox.h, which the reference includes from an
 * un-vendored git submodule (no commit pinned): the types and the
 * philox4x32 call its random.cl:6-24 uses, restated from the published
 * algorithm (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy
 * as 1, 2, 3", SC'11): Philox4x32 with 10 rounds.  Checked against cuRAND's
 * Philox4_32_10 by the tests (test infrastructure only). */
#ifndef CLSHIM_PHILOX_H
#define CLSHIM_PHILOX_H
#include <stdint.h>

typedef struct {
    uint32_t v[4];
} philox4x32_ctr_t;
typedef struct {
    uint32_t v[2];
} philox4x32_key_t;

/* one round: two 32 x 32 -> 64-bit products, each half xored into the
 * other lane pair with the round key */
static inline philox4x32_ctr_t clshim_philox_round(philox4x32_ctr_t x, philox4x32_key_t k) {
    const uint64_t a = (uint64_t)x.v[0] * 0xD2511F53u;
    const uint64_t b = (uint64_t)x.v[2] * 0xCD9E8D57u;
    philox4x32_ctr_t y;
    y.v[0] = (uint32_t)(b >> 32) ^ x.v[1] ^ k.v[0];
    y.v[1] = (uint32_t)b;
    y.v[2] = (uint32_t)(a >> 32) ^ x.v[3] ^ k.v[1];
    y.v[3] = (uint32_t)a;
    return y;
}

static inline philox4x32_ctr_t philox4x32(philox4x32_ctr_t c, philox4x32_key_t k) {
    for (int r = 0; r < 10; ++r) {
        c = clshim_philox_round(c, k);
        k.v[0] += 0x9E3779B9u; /* Weyl key schedule */
        k.v[1] += 0xBB67AE85u;
    }
    return c;
}
#endif
