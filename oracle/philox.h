/*
 * ORACLE-SIDE counter-based draw source (test infrastructure only).
 *
 * Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw, "Parallel
 * random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two 32x32->64
 * multiplies with the Weyl key schedule.  The library carries its own
 * implementation; this one is written separately so that the known-answer
 * vectors of the paper pin both independently.
 *
 * Stream layout shared with the library (the "tape"): draw k of the stream
 * (stream_id, step, tag) is taken from block k>>1 of
 *     philox(ctr = {stream_id, step, tag, k>>1}, key = {seed_lo, seed_hi})
 * using words (2*(k&1), 2*(k&1)+1) = (a, b).
 *   FP64 uniform: x = (a << 20) | (b >> 12)  (52 bits), U = (x + 0.5) * 2^-52,
 *                 so U lies in (0, 1) and both log(U) and log(1-U) are finite.
 */
#ifndef DSMC_ORACLE_PHILOX_H
#define DSMC_ORACLE_PHILOX_H
#include <stdint.h>

#define ORACLE_TAG_MOVE 1u
#define ORACLE_TAG_COLLIDE 2u
#define ORACLE_TAG_INIT 3u

static inline void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline double oracle_uniform64(uint64_t seed, uint32_t stream, uint32_t step, uint32_t tag, uint64_t k) {
    uint32_t ctr[4] = {stream, step, tag, (uint32_t)(k >> 1)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t w[4];
    oracle_philox4x32_10(ctr, key, w);
    uint32_t a = w[2 * (k & 1)], b = w[2 * (k & 1) + 1];
    uint64_t x = ((uint64_t)a << 20) | (uint64_t)(b >> 12);
    return ((double)x + 0.5) * (1.0 / 4503599627370496.0);
}

#endif
