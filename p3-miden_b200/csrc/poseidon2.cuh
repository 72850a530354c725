// Poseidon2 over Goldilocks, width 12, S-box x^7, 4 + 22 + 4 rounds:
// the permutation of the goldilocks_poseidon2 configuration
// (p3-miden-dev-utils/src/configs.rs:393-407, Poseidon2Goldilocks<12>).
//
// External linear layer: circ(2*M4, M4, M4) with M4 = circ(2,3,1,1)
// (Poseidon2 paper, eprint 2023/323, appendix B). Internal layer:
// s_i <- mu_i * s_i + sum(s). Constants are loaded by value: layout
// [rc_init 4x12 | rc_term 4x12 | rc_int 22 | diag 12] = 130 words.
// The device permutation is p2_permute_dev (merkle.cuh); this file holds the
// constants' layout and the host permutation used by the transcript.
#pragma once
#include "gl.cuh"

namespace p2 {

constexpr int N_PARAMS = 130;
constexpr int OFF_INIT = 0, OFF_TERM = 48, OFF_INT = 96, OFF_DIAG = 118;

// Host permutation with lazy reduction: words stay below 2^64 (congruent
// mod p), products and linear-layer sums are kept in 128 bits and reduced
// once; the output is canonical, the permutation of the state over F.
namespace host {
using u128 = unsigned __int128;
constexpr uint64_t EPS = 0xFFFFFFFFull;
inline uint64_t red(u128 x) {  // x < 2^128 -> below 2^64, congruent; branch-free
    const uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64), hh = hi >> 32;
    uint64_t t = lo - hh;
    t -= EPS & (0 - (uint64_t)(lo < hh));
    const uint64_t u = (hi & EPS) * EPS;
    uint64_t r = t + u;
    r += EPS & (0 - (uint64_t)(r < u));
    return r;
}
inline uint64_t mul(uint64_t a, uint64_t b) { return red((u128)a * b); }
inline uint64_t sbox(uint64_t x) {
    const uint64_t x2 = mul(x, x), x3 = mul(x2, x), x4 = mul(x2, x2);
    return mul(x3, x4);
}
inline void ext_linear(uint64_t *s) {
    u128 y[12];
    for (int c = 0; c < 12; c += 4) {
        const u128 a = s[c], b = s[c + 1], cc = s[c + 2], d = s[c + 3];
        const u128 t = a + b + cc + d;
        y[c] = t + a + 2 * b, y[c + 1] = t + b + 2 * cc, y[c + 2] = t + cc + 2 * d, y[c + 3] = t + d + 2 * a;
    }
    for (int k = 0; k < 4; k++) {
        const u128 t = y[k] + y[k + 4] + y[k + 8];
        s[k] = red(y[k] + t), s[k + 4] = red(y[k + 4] + t), s[k + 8] = red(y[k + 8] + t);
    }
}
inline uint64_t addc(uint64_t a, uint64_t c) {  // a < 2^64, c < p
    const uint64_t r = a + c;
    return r + (EPS & (0 - (uint64_t)(r < c)));
}
inline void permute(uint64_t *s, const uint64_t *c) {
    ext_linear(s);
    for (int r = 0; r < 4; r++) {
        for (int i = 0; i < 12; i++) s[i] = sbox(addc(s[i], c[OFF_INIT + 12 * r + i]));
        ext_linear(s);
    }
    for (int r = 0; r < 22; r++) {
        const u128 part = ((u128)s[1] + s[2] + s[3]) + ((u128)s[4] + s[5] + s[6]) + ((u128)s[7] + s[8] + s[9]) +
                          ((u128)s[10] + s[11]);
        s[0] = sbox(addc(s[0], c[OFF_INT + r]));
        const uint64_t sm = red(part + s[0]);
        for (int i = 0; i < 12; i++) s[i] = red((u128)s[i] * c[OFF_DIAG + i] + sm);
    }
    for (int r = 0; r < 4; r++) {
        for (int i = 0; i < 12; i++) s[i] = sbox(addc(s[i], c[OFF_TERM + 12 * r + i]));
        ext_linear(s);
    }
    for (int i = 0; i < 12; i++) s[i] = s[i] >= gl::P ? s[i] - gl::P : s[i];
}
}  // namespace host

}  // namespace p2
