/*
 * ORACLE (test infrastructure only; never linked into the product library).
 *
 * Philox4x32-10 counter-based RNG, restated from the published description
 * (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3",
 * SC'11): ten rounds of two 32x32->64 multiplies with the round keys bumped
 * by the Weyl constants after every round.
 *
 * The reference draws its particle jitter from Julia's unseeded `rand` /
 * GPUArrays' `gpu_rand` (src/particles.jl:37-42, 78-83), so no bit parity with
 * the reference is possible; this generator only fixes a seeded stream that
 * the oracle and the CUDA kernels both reproduce exactly.
 */
#ifndef ISF_ORACLE_PHILOX_H
#define ISF_ORACLE_PHILOX_H
#include <stdint.h>

typedef struct { uint32_t v[4]; } orc_u32x4;

static inline orc_u32x4 orc_philox4x32_10(orc_u32x4 ctr, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)M0 * ctr.v[0];
        uint64_t p1 = (uint64_t)M1 * ctr.v[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        orc_u32x4 n;
        n.v[0] = hi1 ^ ctr.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ ctr.v[3] ^ k1;
        n.v[3] = lo0;
        ctr = n;
        k0 += W0;
        k1 += W1;
    }
    return ctr;
}

/* 24 high bits -> float in [0, 1); exact in float, so both sides agree. */
static inline float orc_u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

#endif
