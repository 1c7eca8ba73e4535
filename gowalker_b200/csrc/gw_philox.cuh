// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC'11), written from the published
// round function: two 32x32->64 multiplies per round, key bumped by the Weyl
// constants between rounds, ten rounds.
//
// Every random decision of the engine is a pure function of a key and a
// 128-bit counter, so a walker's path does not depend on which thread, launch,
// iteration or schedule takes its steps.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define GW_HD __host__ __device__ __forceinline__
#else
#define GW_HD inline
#endif

namespace gw {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

// Counter lane 3 separates the streams that share a key.
constexpr uint32_t kTagWalk = 0u;
constexpr uint32_t kTagRmat = 0x524D4154u;  // 'RMAT'
constexpr uint32_t kTagInit = 0x494E4954u;  // 'INIT'

struct U4 {
    uint32_t x, y, z, w;
};

GW_HD uint32_t mulhi32(uint32_t a, uint32_t b)
{
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

GW_HD U4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = kPhiloxM0 * c0;
        const uint32_t hi0 = mulhi32(kPhiloxM0, c0);
        const uint32_t lo1 = kPhiloxM1 * c2;
        const uint32_t hi1 = mulhi32(kPhiloxM1, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    return U4{c0, c1, c2, c3};
}

// The same generator with the key schedule given: rk0[r], rk1[r] are the
// keys of round r (k + r * W, mod 2^32), philox_schedule() computes them.
GW_HD U4 philox4x32_10_sched(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, const uint32_t *rk0,
                             const uint32_t *rk1)
{
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = kPhiloxM0 * c0;
        const uint32_t hi0 = mulhi32(kPhiloxM0, c0);
        const uint32_t lo1 = kPhiloxM1 * c2;
        const uint32_t hi1 = mulhi32(kPhiloxM1, c2);
        const uint32_t n0 = hi1 ^ c1 ^ rk0[r];
        const uint32_t n2 = hi0 ^ c3 ^ rk1[r];
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    return U4{c0, c1, c2, c3};
}

inline void philox_schedule(uint32_t k0, uint32_t k1, uint32_t *rk0, uint32_t *rk1)
{
    for (int r = 0; r < 10; ++r) {
        rk0[r] = k0 + (uint32_t)r * kPhiloxW0;
        rk1[r] = k1 + (uint32_t)r * kPhiloxW1;
    }
}

// Exact a % d for 32-bit a and d >= 1 by direct computation (Lemire, Kaser and
// Kurz, "Faster remainder by direct computation", 2019): with the 64-bit
// fraction M = ceil(2^64 / d), a % d = high64((M * a mod 2^64) * d).  M costs one
// 64-bit division, so it pays off when one divisor serves many draws -- the
// warp-uniform degree of a cooperative step.
GW_HD uint64_t fastmod_magic(uint32_t d) { return ~0ull / d + 1; }
GW_HD uint32_t fastmod(uint32_t a, uint64_t M, uint32_t d)
{
    const uint64_t low = M * (uint64_t)a;
#if defined(__CUDA_ARCH__)
    return (uint32_t)__umul64hi(low, (uint64_t)d);
#else
    return (uint32_t)(((unsigned __int128)low * d) >> 64);
#endif
}

// FNV-1a over 32-bit words: the per-walker path hash.
constexpr uint64_t kFnvOffset = 0xcbf29ce484222325ull;
constexpr uint64_t kFnvPrime = 0x100000001b3ull;

GW_HD uint64_t hash_init(uint32_t source) { return (kFnvOffset ^ (uint64_t)source) * kFnvPrime; }
GW_HD uint64_t hash_step(uint64_t h, uint32_t v) { return (h ^ (uint64_t)v) * kFnvPrime; }

}  // namespace gw
