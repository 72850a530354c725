// Host-side seeded randomness used to derive Poseidon2 constants and
// synthetic inputs: rand 0.10's SmallRng (xoshiro256++, seeded from a u64
// through SplitMix64), and uniform Goldilocks sampling by rejection of
// 64-bit draws >= p.
#pragma once
#include <cstdint>

#include "gl.cuh"
#include "poseidon2.cuh"

namespace p3g {

struct SmallRng {
    uint64_t s[4];
    explicit SmallRng(uint64_t seed) {
        for (int i = 0; i < 4; i++) {
            seed += 0x9e3779b97f4a7c15ULL;
            uint64_t z = seed;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
            s[i] = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next_u64() {
        uint64_t r = rotl(s[0] + s[3], 23) + s[0];
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    uint64_t field() {
        for (;;) {
            uint64_t x = next_u64();
            if (x < gl::P) return x;
        }
    }
};

// Poseidon2Goldilocks<12>::new_from_rng_128 draw order: 4x12 initial
// external, 4x12 terminal external, 22 internal round constants. The
// internal diagonal is supplied separately.
inline void poseidon2_params_from_seed(uint64_t seed, const uint64_t diag[12], uint64_t out[p2::N_PARAMS]) {
    SmallRng r(seed);
    for (int i = 0; i < 48; i++) out[p2::OFF_INIT + i] = r.field();
    for (int i = 0; i < 48; i++) out[p2::OFF_TERM + i] = r.field();
    for (int i = 0; i < 22; i++) out[p2::OFF_INT + i] = r.field();
    for (int i = 0; i < 12; i++) out[p2::OFF_DIAG + i] = diag[i];
}

// Placeholder internal diagonal (12 uniform elements of
// SmallRng(0x646961675f3132)); p3-goldilocks's table is loaded by value
// through p3g_ctx_create when available.
inline void placeholder_diag(uint64_t out[12]) {
    SmallRng r(0x646961675f3132ULL);
    for (int i = 0; i < 12; i++) out[i] = r.field();
}

}  // namespace p3g
