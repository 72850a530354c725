// Quotient-numerator kernels: AIR constraint evaluation on the quotient
// coset gJ, alpha-folding, beta/cyclic accumulation across traces and the
// vanishing-polynomial division.
//
// For a trace of height h committed on the (lifted) coset s*K, gJ is the
// prefix of h*D rows of its bit-reversed LDE: natural point m of gJ
// (x_m = s * w_{hD}^m) sits at LDE row bitrev_{log hD}(m), and the "next"
// row is point (m + D) mod hD (prover/commit.rs:134-144,
// constraints/mod.rs:117-128). The folded numerator is
// sum_k alpha^{K-1-k} C_k(x_m) (constraints/mod.rs:50-56); alpha^{K-1-k} is
// precomputed per constraint, so the fold is a dot product.
#pragma once
#include "gl.cuh"
#include "ntt.cuh"

namespace quot {

struct EvalArgs {
    const uint64_t *lde;  // bit-reversed LDE of the trace, row stride w
    uint64_t w;
    uint32_t log_qh;       // log2(h * D)
    uint32_t log_h;
    uint64_t D;
    uint64_t shift;        // coset shift s of this trace
    ntt::PowTab wq;        // powers of w_{hD}
    uint64_t omega_h_inv;  // w_h^{-1}
    uint64_t zh[8];        // Z_H(x) = x^h - 1 on gJ, periodic with period D
    const uint64_t *alpha_pows;  // 2 words per constraint: alpha^{K-1-k}
    const uint64_t *consts;      // AIR constants (cubic: k[w])
    uint64_t *acc;               // EF accumulator, 2 words per point
};

struct Fold {
    uint64_t c0 = 0, c1 = 0;
    const uint64_t *ap;
    int k = 0;
    __device__ __forceinline__ explicit Fold(const uint64_t *a) : ap(a) {}
    __device__ __forceinline__ void emit(uint64_t v) {
        uint64_t a0 = __ldg(ap + 2 * k), a1 = __ldg(ap + 2 * k + 1);
        c0 = gl::add(c0, gl::mul(v, a0));
        c1 = gl::add(c1, gl::mul(v, a1));
        k++;
    }
};

__device__ __forceinline__ uint64_t point_x(const EvalArgs &a, uint64_t m) { return gl::mul(a.shift, a.wq.at(m)); }

// ---------------------------------------------------------------- cubic
// Constraint i = is_transition * (next[i] - (local[i]^3 + local[(i+1)%w] + k_i));
// the common factor is_transition is applied once per point.
// One warp per point, lanes over columns.
__global__ void __launch_bounds__(256) cubic_eval_kernel(const __grid_constant__ EvalArgs a) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const uint64_t qh = 1ull << a.log_qh;
    if (warp >= qh) return;
    const uint64_t m = warp;
    const uint64_t *L = a.lde + gl::bitrev(m, a.log_qh) * a.w;
    const uint64_t *N = a.lde + gl::bitrev((m + a.D) & (qh - 1), a.log_qh) * a.w;
    uint64_t c0 = 0, c1 = 0;
    for (uint64_t i = lane; i < a.w; i += 32) {
        uint64_t x = __ldg(L + i);
        uint64_t y = __ldg(L + (i + 1 == a.w ? 0 : i + 1));
        uint64_t rhs = gl::add(gl::add(gl::mul(gl::sqr(x), x), y), __ldg(a.consts + i));
        uint64_t v = gl::sub(__ldg(N + i), rhs);
        c0 = gl::add(c0, gl::mul(v, __ldg(a.alpha_pows + 2 * i)));
        c1 = gl::add(c1, gl::mul(v, __ldg(a.alpha_pows + 2 * i + 1)));
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        c0 = gl::add(c0, __shfl_xor_sync(0xffffffffu, c0, off));
        c1 = gl::add(c1, __shfl_xor_sync(0xffffffffu, c1, off));
    }
    if (lane == 0) {
        uint64_t trans = gl::sub(point_x(a, m), a.omega_h_inv);
        uint64_t *o = a.acc + 2 * m;
        o[0] = gl::add(o[0], gl::mul(c0, trans));
        o[1] = gl::add(o[1], gl::mul(c1, trans));
    }
}

// --------------------------------------------------------------- keccak
// Column layout of the Keccak-f[1600] AIR (2633 columns).
constexpr int KC_STEP = 0, KC_EXPORT = 24, KC_PRE = 25, KC_A = 125, KC_C = 225, KC_CP = 545, KC_AP = 865,
              KC_APP = 2465, KC_APP00 = 2565, KC_APPP00 = 2629, KC_NCOLS = 2633;

__constant__ uint64_t c_keccak_rc[24];
__constant__ int c_keccak_rot[25];  // rot[x*5+y]

__device__ __forceinline__ uint64_t kxor2(uint64_t a, uint64_t b) { return gl::sub(gl::add(a, b), gl::dbl(gl::mul(a, b))); }
__device__ __forceinline__ uint64_t kxor3(uint64_t a, uint64_t b, uint64_t c) { return kxor2(a, kxor2(b, c)); }
__device__ __forceinline__ uint64_t kandn(uint64_t a, uint64_t b) { return gl::mul(gl::sub(1, a), b); }
__device__ __forceinline__ uint64_t kbool(uint64_t a) { return gl::mul(a, gl::sub(a, 1)); }

// All constraints of one row pair in emission order; the same list as the
// oracle's restatement of the KeccakAir arithmetization.
__device__ void keccak_constraints(const uint64_t *L, const uint64_t *N, uint64_t first, uint64_t trans, Fold &f) {
    f.emit(gl::mul(first, gl::sub(__ldg(L + KC_STEP), 1)));
    for (int i = 1; i < 24; i++) f.emit(gl::mul(first, __ldg(L + KC_STEP + i)));
    for (int i = 0; i < 24; i++)
        f.emit(gl::mul(trans, gl::sub(__ldg(N + KC_STEP + (i + 1) % 24), __ldg(L + KC_STEP + i))));
    const uint64_t first_step = __ldg(L + KC_STEP), not_final = gl::sub(1, __ldg(L + KC_STEP + 23));
    for (int o = 0; o < 100; o++) f.emit(gl::mul(first_step, gl::sub(__ldg(L + KC_PRE + o), __ldg(L + KC_A + o))));
    const uint64_t ex = __ldg(L + KC_EXPORT);
    f.emit(kbool(ex));
    f.emit(gl::mul(not_final, ex));
    const uint64_t nf_t = gl::mul(not_final, trans);
    for (int o = 0; o < 100; o++) f.emit(gl::mul(nf_t, gl::sub(__ldg(L + KC_PRE + o), __ldg(N + KC_PRE + o))));
    for (int x = 0; x < 5; x++)
        for (int z = 0; z < 64; z++) {
            uint64_t cxz = __ldg(L + KC_C + x * 64 + z);
            f.emit(kbool(cxz));
            uint64_t v = kxor3(cxz, __ldg(L + KC_C + ((x + 4) % 5) * 64 + z), __ldg(L + KC_C + ((x + 1) % 5) * 64 + (z + 63) % 64));
            f.emit(gl::sub(__ldg(L + KC_CP + x * 64 + z), v));
        }
    for (int y = 0; y < 5; y++)
        for (int x = 0; x < 5; x++)
            for (int l = 0; l < 4; l++) {
                uint64_t acc = 0;
                for (int z = l * 16 + 15; z >= l * 16; z--) {
                    uint64_t ap = __ldg(L + KC_AP + (y * 5 + x) * 64 + z);
                    f.emit(kbool(ap));
                    acc = gl::add(gl::dbl(acc), kxor3(ap, __ldg(L + KC_C + x * 64 + z), __ldg(L + KC_CP + x * 64 + z)));
                }
                f.emit(gl::sub(acc, __ldg(L + KC_A + (y * 5 + x) * 4 + l)));
            }
    for (int x = 0; x < 5; x++)
        for (int z = 0; z < 64; z++) {
            uint64_t s = 0;
            for (int y = 0; y < 5; y++) s = gl::add(s, __ldg(L + KC_AP + (y * 5 + x) * 64 + z));
            uint64_t d = gl::sub(s, __ldg(L + KC_CP + x * 64 + z));
            f.emit(gl::mul(gl::mul(d, gl::sub(d, 2)), gl::sub(d, 4)));
        }
    for (int y = 0; y < 5; y++)
        for (int x = 0; x < 5; x++)
            for (int l = 0; l < 4; l++) {
                uint64_t acc = 0;
                for (int z = l * 16 + 15; z >= l * 16; z--) {
                    uint64_t b[3];
#pragma unroll
                    for (int u = 0; u < 3; u++) {
                        int bx = (x + u) % 5, ax = (bx + 3 * y) % 5;
                        int rot = c_keccak_rot[ax * 5 + bx];
                        b[u] = __ldg(L + KC_AP + (bx * 5 + ax) * 64 + (z + 64 - rot) % 64);
                    }
                    acc = gl::add(gl::dbl(acc), kxor2(b[0], kandn(b[1], b[2])));
                }
                f.emit(gl::sub(acc, __ldg(L + KC_APP + (y * 5 + x) * 4 + l)));
            }
    for (int l = 0; l < 4; l++) {
        uint64_t acc = 0;
        for (int z = l * 16 + 15; z >= l * 16; z--) {
            uint64_t bit = __ldg(L + KC_APP00 + z);
            f.emit(kbool(bit));
            acc = gl::add(gl::dbl(acc), bit);
        }
        f.emit(gl::sub(acc, __ldg(L + KC_APP + l)));
    }
    for (int l = 0; l < 4; l++) {
        uint64_t acc = 0;
        for (int z = l * 16 + 15; z >= l * 16; z--) {
            uint64_t rcb = 0;
            for (int r = 0; r < 24; r++)
                if ((c_keccak_rc[r] >> z) & 1) rcb = gl::add(rcb, __ldg(L + KC_STEP + r));
            acc = gl::add(gl::dbl(acc), kxor2(__ldg(L + KC_APP00 + z), rcb));
        }
        f.emit(gl::sub(acc, __ldg(L + KC_APPP00 + l)));
    }
    for (int x = 0; x < 5; x++)
        for (int y = 0; y < 5; y++)
            for (int l = 0; l < 4; l++) {
                uint64_t outv = (x == 0 && y == 0) ? __ldg(L + KC_APPP00 + l) : __ldg(L + KC_APP + (y * 5 + x) * 4 + l);
                f.emit(gl::mul(nf_t, gl::sub(outv, __ldg(N + KC_A + (y * 5 + x) * 4 + l))));
            }
}

// One thread per quotient point.
__global__ void __launch_bounds__(128) keccak_eval_kernel(const __grid_constant__ EvalArgs a) {
    const uint64_t m = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t qh = 1ull << a.log_qh;
    if (m >= qh) return;
    const uint64_t *L = a.lde + gl::bitrev(m, a.log_qh) * a.w;
    const uint64_t *N = a.lde + gl::bitrev((m + a.D) & (qh - 1), a.log_qh) * a.w;
    uint64_t x = point_x(a, m);
    uint64_t zh = a.zh[m & (a.D - 1)];
    uint64_t first = gl::mul(zh, gl::inv(gl::sub(x, 1)));
    uint64_t trans = gl::sub(x, a.omega_h_inv);
    Fold f(a.alpha_pows);
    keccak_constraints(L, N, first, trans, f);
    uint64_t *o = a.acc + 2 * m;
    o[0] = gl::add(o[0], f.c0);
    o[1] = gl::add(o[1], f.c1);
}

// acc[0..old) *= beta (EF); then acc[i] = acc[i mod old] for i in [old, new)
__global__ void scale_ef_kernel(uint64_t *acc, uint64_t n, gl::ef beta) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gl::ef v = gl::ef_mul(gl::ef{acc[2 * i], acc[2 * i + 1]}, beta);
    acc[2 * i] = v.c0;
    acc[2 * i + 1] = v.c1;
}
__global__ void tile_ef_kernel(uint64_t *acc, uint64_t old_n, uint64_t new_n) {
    uint64_t i = old_n + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= new_n) return;
    uint64_t s = i & (old_n - 1);
    acc[2 * i] = acc[2 * s];
    acc[2 * i + 1] = acc[2 * s + 1];
}
// numerator[i] *= 1 / Z_H(x_i), Z_H periodic with period D (quotient.rs:380-409)
struct VanArgs {
    uint64_t inv_van[8];
    uint64_t D;
};
__global__ void divide_vanishing_kernel(uint64_t *acc, uint64_t n, const __grid_constant__ VanArgs v) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t s = v.inv_van[i & (v.D - 1)];
    acc[2 * i] = gl::mul(acc[2 * i], s);
    acc[2 * i + 1] = gl::mul(acc[2 * i + 1], s);
}

}  // namespace quot
