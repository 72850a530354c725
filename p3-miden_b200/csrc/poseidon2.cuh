// Poseidon2 over Goldilocks, width 12, S-box x^7, 4 + 22 + 4 rounds:
// the permutation of the goldilocks_poseidon2 configuration
// (p3-miden-dev-utils/src/configs.rs:393-407, Poseidon2Goldilocks<12>).
//
// External linear layer: circ(2*M4, M4, M4) with M4 = circ(2,3,1,1)
// (Poseidon2 paper, eprint 2023/323, appendix B). Internal layer:
// s_i <- mu_i * s_i + sum(s). Constants are loaded by value: layout
// [rc_init 4x12 | rc_term 4x12 | rc_int 22 | diag 12] = 130 words.
#pragma once
#include "gl.cuh"

namespace p2 {

constexpr int N_PARAMS = 130;
constexpr int OFF_INIT = 0, OFF_TERM = 48, OFF_INT = 96, OFF_DIAG = 118;

GL_HD uint64_t sbox(uint64_t x) {
    uint64_t x2 = gl::mul(x, x);
    uint64_t x4 = gl::mul(x2, x2);
    uint64_t x3 = gl::mul(x2, x);
    return gl::mul(x4, x3);
}
GL_HD void m4(uint64_t &a, uint64_t &b, uint64_t &c, uint64_t &d) {
    // [2 3 1 1; 1 2 3 1; 1 1 2 3; 3 1 1 2]
    uint64_t ab = gl::add(a, b), cd = gl::add(c, d);
    uint64_t s = gl::add(ab, cd);
    uint64_t y0 = gl::add(gl::add(s, a), gl::dbl(b));   // 2a + 3b + c + d
    uint64_t y1 = gl::add(gl::add(s, b), gl::dbl(c));   // a + 2b + 3c + d
    uint64_t y2 = gl::add(gl::add(s, c), gl::dbl(d));   // a + b + 2c + 3d
    uint64_t y3 = gl::add(gl::add(s, d), gl::dbl(a));   // 3a + b + c + 2d
    a = y0, b = y1, c = y2, d = y3;
}
GL_HD void ext_linear(uint64_t *s) {
    m4(s[0], s[1], s[2], s[3]);
    m4(s[4], s[5], s[6], s[7]);
    m4(s[8], s[9], s[10], s[11]);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        uint64_t t = gl::add(gl::add(s[k], s[k + 4]), s[k + 8]);
        s[k] = gl::add(s[k], t);
        s[k + 4] = gl::add(s[k + 4], t);
        s[k + 8] = gl::add(s[k + 8], t);
    }
}

// Generic permutation over a constant table `c` (device: __constant__ array;
// host: ordinary array).
template <typename Tab>
GL_HD void permute(uint64_t *s, const Tab &c) {
    ext_linear(s);
#pragma unroll
    for (int r = 0; r < 4; r++) {
#pragma unroll
        for (int i = 0; i < 12; i++) s[i] = sbox(gl::add(s[i], c[OFF_INIT + 12 * r + i]));
        ext_linear(s);
    }
#pragma unroll 2
    for (int r = 0; r < 22; r++) {
        s[0] = sbox(gl::add(s[0], c[OFF_INT + r]));
        uint64_t sum = s[0];
#pragma unroll
        for (int i = 1; i < 12; i++) sum = gl::add(sum, s[i]);
#pragma unroll
        for (int i = 0; i < 12; i++) s[i] = gl::add(gl::mul(s[i], c[OFF_DIAG + i]), sum);
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
#pragma unroll
        for (int i = 0; i < 12; i++) s[i] = sbox(gl::add(s[i], c[OFF_TERM + 12 * r + i]));
        ext_linear(s);
    }
}

// Host permutation with lazy reduction: words stay below 2^64 (congruent
// mod p), products and linear-layer sums are kept in 128 bits and reduced
// once; the output is canonical and equal to permute()'s.
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
