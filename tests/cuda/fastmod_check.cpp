// Test-only: the engine's fastmod (gw_philox.cuh) against the % operator, and
// its scheduled-key Philox against the plain one.
#include <cstdint>
#include <cstdio>
#include <initializer_list>
#include "gw_philox.cuh"

int main()
{
    uint64_t s = 0x9E3779B97F4A7C15ull, checked = 0;
    auto next = [&]() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; };
    const uint32_t edge[] = {0u, 1u, 2u, 3u, 7u, 0x7FFFFFFFu, 0x80000000u, 0xFFFFFFFEu, 0xFFFFFFFFu};
    for (uint32_t d = 1; d <= 4096; ++d) {
        const uint64_t M = gw::fastmod_magic(d);
        for (uint32_t a : edge) { if (gw::fastmod(a, M, d) != a % d) { printf("FAIL %u %u\n", a, d); return 1; } ++checked; }
        for (int k = 0; k < 2000; ++k) { const uint32_t a = (uint32_t)next(); if (gw::fastmod(a, M, d) != a % d) { printf("FAIL %u %u\n", a, d); return 1; } ++checked; }
    }
    for (int k = 0; k < 20000; ++k) {
        uint32_t d = (uint32_t)next();
        if (d == 0) d = 1;
        const uint64_t M = gw::fastmod_magic(d);
        for (uint32_t a : edge) { if (gw::fastmod(a, M, d) != a % d) { printf("FAIL %u %u\n", a, d); return 1; } ++checked; }
        for (int j = 0; j < 200; ++j) { const uint32_t a = (uint32_t)next(); if (gw::fastmod(a, M, d) != a % d) { printf("FAIL %u %u\n", a, d); return 1; } ++checked; }
    }
    for (uint32_t d : {0xFFFFFFFFu, 0x80000000u, 0x80000001u, 3u, 641u}) {
        const uint64_t M = gw::fastmod_magic(d);
        for (uint64_t a = 0; a <= 0xFFFFFFFFull; a += 65537) { if (gw::fastmod((uint32_t)a, M, d) != (uint32_t)a % d) { printf("FAIL %llu %u\n", (unsigned long long)a, d); return 1; } ++checked; }
    }
    for (int k = 0; k < 20000; ++k) {
        const uint32_t k0 = (uint32_t)next(), k1 = (uint32_t)next();
        uint32_t rk0[10], rk1[10];
        gw::philox_schedule(k0, k1, rk0, rk1);
        const uint32_t c0 = (uint32_t)next(), c1 = (uint32_t)next(), c2 = (uint32_t)next(), c3 = (uint32_t)next();
        const gw::U4 a = gw::philox4x32_10(c0, c1, c2, c3, k0, k1);
        const gw::U4 b = gw::philox4x32_10_sched(c0, c1, c2, c3, rk0, rk1);
        if (a.x != b.x || a.y != b.y || a.z != b.z || a.w != b.w) { printf("FAIL philox schedule\n"); return 1; }
        ++checked;
    }
    printf("ok %llu\n", (unsigned long long)checked);
    return 0;
}
