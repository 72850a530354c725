// Host-side trace generators for the two AIRs on the measured path (the
// caller side of prove_multi): the Keccak-f[1600] AIR trace
// (p3-miden-lifted-examples/src/keccak.rs:54-56) and the synthetic cubic
// AIR trace of the lifted multi-trace workload.
#pragma once
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "gl.cuh"
#include "host_rng.cuh"

namespace p3g {

namespace keccak {
constexpr int STEP = 0, EXPORT = 24, PRE = 25, A = 125, C = 225, CP = 545, AP = 865, APP = 2465, APP00 = 2565,
              APPP00 = 2629, NCOLS = 2633, ROUNDS = 24;

struct Tables {
    int rot[5][5];
    uint64_t rc[24];
    Tables() {
        // FIPS 202: rho offsets by the (t+1)(t+2)/2 walk; iota constants from
        // the LFSR x^8 + x^6 + x^5 + x^4 + 1.
        memset(rot, 0, sizeof(rot));
        int x = 1, y = 0;
        for (int t = 0; t < 24; t++) {
            rot[x][y] = ((t + 1) * (t + 2) / 2) % 64;
            int nx = y, ny = (2 * x + 3 * y) % 5;
            x = nx, y = ny;
        }
        auto lfsr = [](int t) {
            unsigned r = 1;
            for (int i = 0; i < t % 255; i++) {
                r <<= 1;
                if (r & 0x100) r ^= 0x171;
            }
            return (int)(r & 1);
        };
        for (int i = 0; i < 24; i++) {
            uint64_t v = 0;
            for (int j = 0; j <= 6; j++)
                if (lfsr(j + 7 * i)) v |= 1ull << ((1u << j) - 1);
            rc[i] = v;
        }
    }
};
inline const Tables &tables() {
    static Tables t;
    return t;
}
inline uint64_t rotl(uint64_t v, int r) { return r ? (v << r) | (v >> (64 - r)) : v; }
inline void limbs(uint64_t *dst, uint64_t v) {
    for (int l = 0; l < 4; l++) dst[l] = (v >> (16 * l)) & 0xffff;
}

// rows of one permutation (up to 24), lane (x, y) = input[x + 5y]
inline void perm_rows(uint64_t *rows, size_t nrows, const uint64_t *input) {
    const Tables &T = tables();
    uint64_t st[5][5];
    for (int y = 0; y < 5; y++)
        for (int x = 0; x < 5; x++) st[x][y] = input[x + 5 * y];
    for (size_t r = 0; r < nrows; r++) {
        uint64_t *row = rows + r * NCOLS;
        memset(row, 0, NCOLS * 8);
        row[STEP + r] = 1;
        for (int y = 0; y < 5; y++)
            for (int x = 0; x < 5; x++) {
                limbs(row + PRE + (y * 5 + x) * 4, input[x + 5 * y]);
                limbs(row + A + (y * 5 + x) * 4, st[x][y]);
            }
        uint64_t c[5], d[5], ap[5][5], b[5][5], app[5][5];
        for (int x = 0; x < 5; x++) c[x] = st[x][0] ^ st[x][1] ^ st[x][2] ^ st[x][3] ^ st[x][4];
        for (int x = 0; x < 5; x++) d[x] = c[(x + 4) % 5] ^ rotl(c[(x + 1) % 5], 1);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) ap[x][y] = st[x][y] ^ d[x];
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) b[y][(2 * x + 3 * y) % 5] = rotl(ap[x][y], T.rot[x][y]);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) app[x][y] = b[x][y] ^ (~b[(x + 1) % 5][y] & b[(x + 2) % 5][y]);
        for (int x = 0; x < 5; x++)
            for (int z = 0; z < 64; z++) {
                row[C + x * 64 + z] = (c[x] >> z) & 1;
                row[CP + x * 64 + z] = ((c[x] ^ d[x]) >> z) & 1;
            }
        for (int y = 0; y < 5; y++)
            for (int x = 0; x < 5; x++) {
                for (int z = 0; z < 64; z++) row[AP + (y * 5 + x) * 64 + z] = (ap[x][y] >> z) & 1;
                limbs(row + APP + (y * 5 + x) * 4, app[x][y]);
            }
        for (int z = 0; z < 64; z++) row[APP00 + z] = (app[0][0] >> z) & 1;
        uint64_t a000 = app[0][0] ^ T.rc[r];
        limbs(row + APPP00, a000);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) st[x][y] = app[x][y];
        st[0][0] = a000;
    }
}
}  // namespace keccak

// generate_trace_rows(inputs, 0): 2^log_h rows; permutations past the
// inputs use the all-zero state (the last one possibly truncated).
inline void keccak_trace(const uint64_t *inputs25, uint64_t n_perms, uint32_t log_h, uint64_t *out) {
    const uint64_t h = 1ull << log_h;
    const uint64_t chunks = (h + 23) / 24;
    static const uint64_t zero[25] = {0};
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++)
        th.emplace_back([&, t] {
            for (uint64_t c = t; c < chunks; c += nt) {
                uint64_t nrows = std::min<uint64_t>(24, h - c * 24);
                keccak::perm_rows(out + c * 24 * keccak::NCOLS, nrows, c < n_perms ? inputs25 + 25 * c : zero);
            }
        });
    for (auto &x : th) x.join();
}

// SmallRng(seed).random::<[u64; 25]>() per permutation
inline void keccak_inputs(uint64_t seed, uint64_t n_perms, uint64_t *out25) {
    SmallRng r(seed);
    for (uint64_t i = 0; i < 25 * n_perms; i++) out25[i] = r.next_u64();
}

// Cubic AIR: k_0..k_{w-1} then row 0 drawn uniformly from SmallRng(seed);
// row r+1 = row_r^3 + rotate(row_r, 1) + k.
inline void cubic_trace(uint32_t log_h, uint64_t width, uint64_t seed, uint64_t *k, uint64_t *trace) {
    SmallRng r(seed);
    for (uint64_t i = 0; i < width; i++) k[i] = r.field();
    for (uint64_t i = 0; i < width; i++) trace[i] = r.field();
    const uint64_t h = 1ull << log_h;
    for (uint64_t row = 1; row < h; row++) {
        const uint64_t *p = trace + (row - 1) * width;
        uint64_t *q = trace + row * width;
        for (uint64_t i = 0; i < width; i++) {
            uint64_t x = p[i];
            q[i] = gl::add(gl::add(gl::mul(gl::sqr(x), x), p[i + 1 == width ? 0 : i + 1]), k[i]);
        }
    }
}

}  // namespace p3g
