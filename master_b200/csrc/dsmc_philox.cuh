// Counter-based draws for the DSMC kernels.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): ten rounds of two 32x32->64-bit multiplies
// (0xD2511F53, 0xCD9E8D57) with Weyl key increments (0x9E3779B9, 0xBB67AE85).
//
// The reference draws from one sequential ran1 stream per MPI rank
// (dsmc/random.cpp:43-68), which serialises every particle and cell.  Here
// every particle (mover) and every cell (collide) owns a stream:
//     draw k of stream (id, step, tag) = words (2(k&1), 2(k&1)+1) of
//     philox(ctr = {id, step, tag, k>>1}, key = {seed_lo, seed_hi}).
// fp64 draw: U = (((a << 20) | (b >> 12)) + 0.5) * 2^-52, in (0, 1).
// fp32 draw: U = ((a >> 9) + 0.5) * 2^-23, in (0, 1); the same words, so an
// fp32 run sees the fp64 run's draws rounded to 23 bits.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define DSMC_HD __host__ __device__ __forceinline__
#else
#define DSMC_HD inline
#endif

namespace dsmc {

DSMC_HD void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                           uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
        uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

// A stream with a one-block cache: two draws per Philox evaluation.
struct DrawStream {
    uint32_t key0, key1, id, step, tag, k;
    uint32_t w[4];

    DSMC_HD void init(uint64_t seed, uint32_t id_, uint32_t step_, uint32_t tag_) {
        key0 = (uint32_t)seed;
        key1 = (uint32_t)(seed >> 32);
        id = id_;
        step = step_;
        tag = tag_;
        k = 0;
    }
    DSMC_HD void words(uint32_t &a, uint32_t &b) {
        // constant indexes only, so the block stays in registers
        if ((k & 1u) == 0) {
            philox4x32_10(id, step, tag, k >> 1, key0, key1, w);
            a = w[0];
            b = w[1];
        } else {
            a = w[2];
            b = w[3];
        }
        ++k;
    }
    DSMC_HD double uniform64() {
        uint32_t a, b;
        words(a, b);
        uint64_t x = ((uint64_t)a << 20) | (uint64_t)(b >> 12);
        return ((double)x + 0.5) * (1.0 / 4503599627370496.0);
    }
    DSMC_HD float uniform32() {
        uint32_t a, b;
        words(a, b);
        return ((float)(a >> 9) + 0.5f) * (1.0f / 8388608.0f);
    }
    template <class T> DSMC_HD T uniform();
};
template <> DSMC_HD double DrawStream::uniform<double>() { return uniform64(); }
template <> DSMC_HD float DrawStream::uniform<float>() { return uniform32(); }

}  // namespace dsmc
