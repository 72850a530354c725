// Lifted Merkle tree (LMCS) kernels: leaf sponge absorption with virtual
// lifting, and layer compression.
//
// Leaf semantics (p3-miden-lmcs/src/lifted_tree.rs:385-483): leaf j of a tree
// of height H absorbs, for every matrix m in ascending-height order, row
// j >> log2(H/h_m) of m, each row in its own absorb call (overwrite mode,
// rate 8, zero-padded partial chunk; field_sponge.rs:164-182), then squeezes
// state[0..4]. Matrices are processed one height class at a time: the
// states of a class of height h are computed from the states of the
// previous class at index j >> log2(h/h_prev); nothing is upsampled in
// memory.
//
// Digest layers of a tree of height H live in one buffer of 2H-1 digests
// (4 words each), layer l (H >> l digests) at digest offset 2H - 2(H >> l).
#pragma once
#include "gl.cuh"
#include "poseidon2.cuh"

__constant__ uint64_t c_p2[p2::N_PARAMS];

// Device permutation: one looped copy of the round body per call site, so
// that kernels stay small enough for the instruction cache (the fully
// unrolled form stalled on instruction fetch). Rounds 0-3 and 26-29 are
// external, 4-25 internal; constants come from the __constant__ table.
//
// Arithmetic is lazy: state words are kept weakly reduced (any value below
// 2^64 congruent mod p); the linear layers accumulate in 96 bits and reduce
// once per output; s*mu + sum is reduced once from 128 bits. Callers
// canonicalise words that leave the permutation (p2w::canon).
namespace p2w {
constexpr uint64_t EPS = 0xFFFFFFFFull;
struct W {  // lo + hi * 2^64
    uint64_t lo;
    uint32_t hi;
};
__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) { return gl::mul_weak(a, b); }
__device__ __forceinline__ uint64_t canon(uint64_t a) { return gl::canon_dev(a); }
// weak + canonical: one wrap at most (a + c - 2^64 + eps < 2^64)
__device__ __forceinline__ uint64_t add_c(uint64_t a, uint64_t c) {
    uint32_t r0, r1;
    asm("{\n\t.reg .u32 k;\n\t"
        "add.cc.u32 %0, %2, %4;\n\t"
        "addc.cc.u32 %1, %3, %5;\n\t"
        "addc.u32 k, 0, 0;\n\t"
        "neg.s32 k, k;\n\t"
        "add.cc.u32 %0, %0, k;\n\t"
        "addc.u32 %1, %1, 0;\n\t}"
        : "=&r"(r0), "=&r"(r1)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)c), "r"((uint32_t)(c >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}
__device__ __forceinline__ W wide(uint64_t a) { return W{a, 0}; }
__device__ __forceinline__ W wadd(W a, W b) {
    uint32_t r0, r1, h;
    asm("add.cc.u32 %0, %3, %6;\n\t"
        "addc.cc.u32 %1, %4, %7;\n\t"
        "addc.u32 %2, %5, %8;"
        : "=&r"(r0), "=&r"(r1), "=&r"(h)
        : "r"((uint32_t)a.lo), "r"((uint32_t)(a.lo >> 32)), "r"(a.hi), "r"((uint32_t)b.lo),
          "r"((uint32_t)(b.lo >> 32)), "r"(b.hi));
    return W{((uint64_t)r1 << 32) | r0, h};
}
__device__ __forceinline__ W wadd1(W a, uint64_t b) {
    uint32_t r0, r1, h;
    asm("add.cc.u32 %0, %3, %6;\n\t"
        "addc.cc.u32 %1, %4, %7;\n\t"
        "addc.u32 %2, %5, 0;"
        : "=&r"(r0), "=&r"(r1), "=&r"(h)
        : "r"((uint32_t)a.lo), "r"((uint32_t)(a.lo >> 32)), "r"(a.hi), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return W{((uint64_t)r1 << 32) | r0, h};
}
__device__ __forceinline__ W wdbl(uint64_t a) { return wadd1(wide(a), a); }
// lo + hi * 2^64 with hi < 2^32: lo + hi * eps, one wrap at most
__device__ __forceinline__ uint64_t wreduce(W a) {
    uint32_t r0, r1;
    asm("{\n\t.reg .u32 u0, u1, c;\n\t"
        "sub.cc.u32 u0, 0, %4;\n\t"  // hi*eps = (hi << 32) - hi
        "subc.u32 u1, %4, 0;\n\t"
        "add.cc.u32 %0, %2, u0;\n\t"
        "addc.cc.u32 %1, %3, u1;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 c, c;\n\t"          // on carry add eps
        "add.cc.u32 %0, %0, c;\n\t"
        "addc.u32 %1, %1, 0;\n\t}"
        : "=&r"(r0), "=&r"(r1)
        : "r"((uint32_t)a.lo), "r"((uint32_t)(a.lo >> 32)), "r"(a.hi));
    return ((uint64_t)r1 << 32) | r0;
}
__device__ __forceinline__ uint64_t sbox(uint64_t x) {
    uint64_t x2 = mul(x, x), x4 = mul(x2, x2), x3 = mul(x2, x);
    return mul(x4, x3);
}
// a*b + c for a, b < 2^64 and a 96-bit c below 2^68: c enters the product's
// carry chain whole (its top word on the third limb, where the product chain
// starts from zero), so a sum shared by several products is never reduced on
// its own. a*b + c <= (2^64-1)^2 + 2^68 < 2^128; weakly reduced.
__device__ __forceinline__ uint64_t mul_add_w(uint64_t a, uint64_t b, W c) {
    uint32_t r0, r1, r2, r3;
    asm("mad.lo.cc.u32 %0, %4, %6, %8;\n\t"
        "madc.hi.cc.u32 %1, %4, %6, %9;\n\t"
        "addc.u32 %2, %10, 0;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.cc.u32 %2, %4, %7, %2;\n\t"
        "addc.u32 %3, 0, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "addc.u32 %3, %3, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, %3;"
        : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)),
          "r"((uint32_t)c.lo), "r"((uint32_t)(c.lo >> 32)), "r"(c.hi));
    return gl::reduce4_dev(r0, r1, r2, r3);
}
// circ(2*M4, M4, M4), M4 = circ(2,3,1,1): 96-bit accumulation, one reduction per
// output. With rc_off >= 0 the next round's constants c_p2[rc_off + i] join the
// 96-bit sums before the reduction (the same value mod p as adding them after it,
// in 3 instructions instead of 6).
__device__ __forceinline__ void ext_linear(uint64_t *s, int rc_off = -1) {
    W y[12];
#pragma unroll
    for (int c = 0; c < 12; c += 4) {
        uint64_t x0 = s[c], x1 = s[c + 1], x2 = s[c + 2], x3 = s[c + 3];
        W t01 = wadd1(wide(x0), x1), t23 = wadd1(wide(x2), x3);
        W t0123 = wadd(t01, t23);
        W t01123 = wadd1(t0123, x1), t01233 = wadd1(t0123, x3);
        y[c + 0] = wadd(t01123, t01);           // 2x0 + 3x1 + x2 + x3
        y[c + 1] = wadd(t01123, wdbl(x2));      // x0 + 2x1 + 3x2 + x3
        y[c + 2] = wadd(t01233, t23);           // x0 + x1 + 2x2 + 3x3
        y[c + 3] = wadd(t01233, wdbl(x0));      // 3x0 + x1 + x2 + 2x3
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        W t = wadd(wadd(y[k], y[k + 4]), y[k + 8]);
        W a = wadd(y[k], t), b = wadd(y[k + 4], t), c = wadd(y[k + 8], t);
        if (rc_off >= 0) {
            a = wadd1(a, c_p2[rc_off + k]);
            b = wadd1(b, c_p2[rc_off + k + 4]);
            c = wadd1(c, c_p2[rc_off + k + 8]);
        }
        s[k] = wreduce(a);
        s[k + 4] = wreduce(b);
        s[k + 8] = wreduce(c);
    }
}
}  // namespace p2w

// External rounds take their constants inside the preceding linear layer
// (rounds 0-3 and 27-29); round 26 follows the internal rounds and adds its own.
__device__ __forceinline__ void p2_permute_dev(uint64_t *s) {
    p2w::ext_linear(s, p2::OFF_INIT);
#pragma unroll 1
    for (int r = 0; r < 30; r++) {
        if (r < 4 || r >= 26) {
            if (r == 26) {
#pragma unroll
                for (int i = 0; i < 12; i++) s[i] = p2w::add_c(s[i], c_p2[p2::OFF_TERM + i]);
            }
#pragma unroll
            for (int i = 0; i < 12; i++) s[i] = p2w::sbox(s[i]);
            p2w::ext_linear(s, r < 3 ? p2::OFF_INIT + 12 * (r + 1) : (r >= 26 && r < 29) ? p2::OFF_TERM + 12 * (r - 25) : -1);
        } else {
            s[0] = p2w::sbox(p2w::add_c(s[0], c_p2[p2::OFF_INT + r - 4]));
            p2w::W acc = p2w::wide(s[0]);
#pragma unroll
            for (int i = 1; i < 12; i++) acc = p2w::wadd1(acc, s[i]);  // below 12 * 2^64
#pragma unroll
            for (int i = 0; i < 12; i++) s[i] = p2w::mul_add_w(s[i], c_p2[p2::OFF_DIAG + i], acc);
        }
    }
}


// Permutation shared by 16 lanes, for latency-bound work (a few states at a
// time; about a third of the single-thread latency). Lane l < 12 holds word
// l, lanes 12..15 hold zero between rounds. External rounds run one S-box per
// lane and move the M4 and cross-block sums through shuffles. In the internal
// rounds every lane carries a copy z of s_0: the S-box runs on z while the
// sum R of s_1..s_11 is formed by a 4-step butterfly, and
// s_0 <- (mu_0 + 1) * S(z) + R, so only the S-box and one product lie on the
// round's critical path. Same lazy arithmetic as p2_permute_dev (results
// agree mod p). Two states per warp; all 32 lanes must call it. `sc` is the
// constant table staged in shared memory (stage_consts).
namespace p2x {
// copy the constant table into shared memory (all threads of the block call it)
__device__ __forceinline__ void stage_consts(uint64_t *sc) {
    for (int i = threadIdx.x; i < p2::N_PARAMS; i += blockDim.x) sc[i] = c_p2[i];
    __syncthreads();
}
__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
    const uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)v, src, 16);
    const uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(v >> 32), src, 16);
    return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ p2w::W shflW(p2w::W v, int src) {
    return p2w::W{shfl64(v.lo, src), __shfl_sync(0xffffffffu, v.hi, src, 16)};
}
__device__ __forceinline__ p2w::W shflW_xor(p2w::W v, int m) {
    const uint32_t lo = __shfl_xor_sync(0xffffffffu, (uint32_t)v.lo, m, 16);
    const uint32_t hi = __shfl_xor_sync(0xffffffffu, (uint32_t)(v.lo >> 32), m, 16);
    return p2w::W{((uint64_t)hi << 32) | lo, __shfl_xor_sync(0xffffffffu, v.hi, m, 16)};
}
struct Lane {
    uint64_t mu;     // diagonal word l (0 for l >= 12)
    uint64_t mu0p1;  // mu_0 + 1 mod p
};
__device__ __forceinline__ Lane lane_consts(const uint64_t *sc, int l) {
    return Lane{l < 12 ? sc[p2::OFF_DIAG + l] : 0, gl::add_dev(sc[p2::OFF_DIAG], 1)};
}
// circ(2*M4, M4, M4) for word l: M4 row (l mod 4) of its block, plus the sum
// over the three blocks of that row; lanes 12..15 return 0
// rc: the lane's constant of the next round (0 for none), added to the
// 96-bit sum before the reduction
__device__ __forceinline__ uint64_t ext_linear(uint64_t x, int l, uint64_t rc = 0) {
    using namespace p2w;
    const int base = l & ~3, j = l & 3;
    const uint64_t x0 = shfl64(x, base), x1 = shfl64(x, base + 1), x2 = shfl64(x, base + 2), x3 = shfl64(x, base + 3);
    const W t01 = wadd1(wide(x0), x1), t23 = wadd1(wide(x2), x3);
    const W t0123 = wadd(t01, t23);
    const uint64_t e = j < 2 ? x1 : x3;
    const W f = j == 0 ? t01 : j == 1 ? wdbl(x2) : j == 2 ? t23 : wdbl(x0);
    const W y = wadd(wadd1(t0123, e), f);
    const W t = wadd(wadd(shflW(y, j), shflW(y, j + 4)), shflW(y, j + 8));
    return l < 12 ? wreduce(wadd1(wadd(y, t), rc)) : 0;
}
// four external rounds whose first constant is already in x; each linear
// layer takes in the next round's constant
__device__ __forceinline__ uint64_t ext_rounds(uint64_t x, int l, const uint64_t *rc) {
    const int li = l < 12 ? l : 11;
#pragma unroll 1
    for (int r = 0; r < 4; r++) x = ext_linear(p2w::sbox(x), l, r < 3 ? rc[12 * (r + 1) + li] : 0);
    return x;
}
__device__ __forceinline__ uint64_t permute(uint64_t x, int l, const uint64_t *sc, const Lane &k) {
    using namespace p2w;
    const int li = l < 12 ? l : 11;
    x = ext_rounds(ext_linear(x, l, sc[p2::OFF_INIT + li]), l, sc + p2::OFF_INIT);
    uint64_t z = shfl64(x, 0);
    const bool rest = l >= 1 && l < 12;
#pragma unroll 1
    for (int r = 0; r < 22; r++) {
        const uint64_t zs = sbox(add_c(z, sc[p2::OFF_INT + r]));
        W P = wide(rest ? x : 0);
#pragma unroll
        for (int m = 1; m < 16; m <<= 1) P = wadd(P, shflW_xor(P, m));
        z = mul_add_w(zs, k.mu0p1, P);                       // P < 11 * 2^64
        x = rest ? mul_add_w(x, k.mu, wadd1(P, zs)) : 0;     // sum < 12 * 2^64
    }
    if (l == 0) x = z;
    return ext_rounds(add_c(x, sc[p2::OFF_TERM + li]), l, sc + p2::OFF_TERM);
}
}  // namespace p2x

namespace merkle {

constexpr int MAX_MATS = 8;

struct ClassArgs {
    const uint64_t *data[MAX_MATS];
    uint64_t width[MAX_MATS];
    uint64_t ld[MAX_MATS];  // row stride in words (>= width; a column slab of a wider matrix)
    int n_mats;
    uint32_t log_h;         // height of this class
    const uint64_t *prev;   // states of the previous class (12 words each), or null
    uint32_t prev_log_h;
    uint64_t *states_out;   // 12 words per leaf, or null when squeezing
    uint64_t *digests_out;  // 4 words per leaf, or null
    // optional column-major copy of the absorbed rows (n_mats == 1): word c
    // of row j < cm_rows is also written to cm[c * cm_ld + j] (the cells the
    // generated constraint kernels read; a warp's 32 rows make one 256-byte run)
    uint64_t *cm;
    uint64_t cm_ld, cm_rows;
};

// absorb one row (rate 8, overwrite mode, zero-padded last chunk); a single
// permutation call site
// permutation call site; with CM, each word is also stored at cmj[c * cm_ld]
// (cmj = cm + row index, or null for rows past cm_rows)
template <bool CM>
__device__ __forceinline__ void absorb_row(uint64_t *s, const uint64_t *row, uint64_t w, uint64_t *cmj,
                                           uint64_t cm_ld) {
#pragma unroll 1
    for (uint64_t i = 0; i < w; i += 8) {
        if (i + 8 <= w) {
#pragma unroll
            for (int j = 0; j < 8; j++) s[j] = __ldg(row + i + j);
            if (CM && cmj) {
#pragma unroll
                for (int j = 0; j < 8; j++) cmj[(i + j) * cm_ld] = s[j];
            }
        } else {
#pragma unroll
            for (int j = 0; j < 8; j++) s[j] = i + j < w ? __ldg(row + i + j) : 0;
            if (CM && cmj) {
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if (i + j < w) cmj[(i + j) * cm_ld] = s[j];
            }
        }
        p2_permute_dev(s);
    }
}

// At most 64 registers: eight 128-thread blocks per SM (measured: 66
// registers, seven blocks, made the slab's tree 9 % slower).
template <bool CM>
__global__ void __launch_bounds__(128, 8) leaf_class_kernel(const __grid_constant__ ClassArgs a) {
    uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >> a.log_h) return;
    uint64_t s[12];
    if (a.prev) {
        const uint64_t *p = a.prev + (j >> (a.log_h - a.prev_log_h)) * 12;
#pragma unroll
        for (int i = 0; i < 12; i++) s[i] = p[i];
    } else {
#pragma unroll
        for (int i = 0; i < 12; i++) s[i] = 0;
    }
    for (int m = 0; m < a.n_mats; m++)
        absorb_row<CM>(s, a.data[m] + j * a.ld[m], a.width[m], CM && j < a.cm_rows ? a.cm + j : nullptr, a.cm_ld);
    if (a.digests_out) {
#pragma unroll
        for (int i = 0; i < 4; i++) a.digests_out[j * 4 + i] = p2w::canon(s[i]);
    } else {
#pragma unroll
        for (int i = 0; i < 12; i++) a.states_out[j * 12 + i] = s[i];
    }
}

// The same leaf sponge with one 16-lane group per leaf (p2x), for classes
// with few leaves, where one thread per leaf leaves the GPU nearly empty and
// each of a row's chained permutations costs the full single-thread latency.
// States are weakly reduced like leaf_class_kernel's (congruent mod p, not
// always the same words), so classes may mix the two kernels.
constexpr uint64_t kCoopLeaves = 4096;
template <bool CM>
__global__ void __launch_bounds__(128) leaf_class_coop_kernel(const __grid_constant__ ClassArgs a) {
    __shared__ uint64_t sc[p2::N_PARAMS];
    p2x::stage_consts(sc);
    const int l = threadIdx.x & 15;
    const p2x::Lane k = p2x::lane_consts(sc, l);
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (((t & ~31ull) >> 4) >> a.log_h) return;  // warp-uniform: the warp's first leaf is past the class
    const uint64_t j = t >> 4;
    const bool ok = (j >> a.log_h) == 0;
    uint64_t x = 0;
    if (ok && a.prev && l < 12) x = a.prev[(j >> (a.log_h - a.prev_log_h)) * 12 + l];
    for (int m = 0; m < a.n_mats; m++) {
        const uint64_t w = a.width[m];
        const uint64_t *row = a.data[m] + (ok ? j : 0) * a.ld[m];
#pragma unroll 1
        for (uint64_t i = 0; i < w; i += 8) {
            if (l < 8) x = ok && i + l < w ? __ldg(row + i + l) : 0;
            if (CM && l < 8 && ok && i + l < w && j < a.cm_rows) a.cm[(i + l) * a.cm_ld + j] = x;
            x = p2x::permute(x, l, sc, k);
        }
    }
    if (!ok) return;
    if (a.digests_out) {
        if (l < 4) a.digests_out[j * 4 + l] = p2w::canon(x);
    } else if (l < 12) {
        a.states_out[j * 12 + l] = x;
    }
}

__device__ __forceinline__ void compress2(const uint64_t *l, const uint64_t *r, uint64_t *out) {
    uint64_t s[12];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        s[i] = l[i];
        s[4 + i] = r[i];
        s[8 + i] = 0;
    }
    p2_permute_dev(s);
#pragma unroll
    for (int i = 0; i < 4; i++) out[i] = p2w::canon(s[i]);
}

// One block compresses 2*blockDim.x digests of layer `l_in` through `levels`
// layers (2^levels <= 2*blockDim.x), writing every produced layer.
__global__ void __launch_bounds__(256) compress_kernel(uint64_t *layers, uint64_t H, uint32_t l_in, uint32_t levels) {
    __shared__ uint64_t sm[256 * 4];
    const uint64_t n_in = H >> l_in;
    const uint64_t off_in = 2 * H - 2 * (H >> l_in);
    const uint32_t t = threadIdx.x;
    const uint64_t parent = (uint64_t)blockIdx.x * blockDim.x + t;  // index in layer l_in+1
    uint64_t d[4];
    if (2 * parent + 1 < n_in) {
        compress2(layers + 4 * (off_in + 2 * parent), layers + 4 * (off_in + 2 * parent + 1), d);
        uint64_t off1 = 2 * H - 2 * (H >> (l_in + 1));
#pragma unroll
        for (int i = 0; i < 4; i++) {
            layers[4 * (off1 + parent) + i] = d[i];
            sm[4 * t + i] = d[i];
        }
    }
    __syncthreads();
    uint32_t active = blockDim.x;
    for (uint32_t lv = 1; lv < levels; lv++) {
        active >>= 1;
        uint64_t n_l = H >> (l_in + lv + 1);
        uint64_t pidx = (uint64_t)blockIdx.x * active + t;
        if (t < active && pidx < n_l) {
            compress2(sm + 4 * (2 * t), sm + 4 * (2 * t + 1), d);
            uint64_t off = 2 * H - 2 * (H >> (l_in + lv + 1));
#pragma unroll
            for (int i = 0; i < 4; i++) layers[4 * (off + pidx) + i] = d[i];
        }
        __syncthreads();
        if (t < active && pidx < n_l) {
#pragma unroll
            for (int i = 0; i < 4; i++) sm[4 * t + i] = d[i];
        }
        __syncthreads();
    }
}

// Levels with few parents are bound by the latency of one permutation, not
// by throughput: there one 16-lane group compresses one parent (p2x), about
// a third of the single-thread latency. Children 2p and 2p + 1 are adjacent
// digests, so lanes 0..7 load the eight input words with one access each.
__device__ __forceinline__ void compress_parent_coop(uint64_t *layers, uint64_t off_in, uint64_t off_out, uint64_t p,
                                                     bool ok, int l, const uint64_t *sc, const p2x::Lane &k) {
    uint64_t x = 0;
    if (ok && l < 8) x = __ldcg(layers + 4 * (off_in + 2 * p) + l);
    x = p2x::permute(x, l, sc, k);
    if (ok && l < 4) layers[4 * (off_out + p) + l] = p2w::canon(x);
}

// One level: parents of layer l_in + 1, one 16-lane group each.
__global__ void __launch_bounds__(128) compress_level_coop_kernel(uint64_t *layers, uint64_t H, uint32_t l_in) {
    __shared__ uint64_t sc[p2::N_PARAMS];
    p2x::stage_consts(sc);
    const int l = threadIdx.x & 15;
    const p2x::Lane k = p2x::lane_consts(sc, l);
    const uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const uint64_t n = H >> (l_in + 1);
    compress_parent_coop(layers, 2 * H - 2 * (H >> l_in), 2 * H - 2 * (H >> (l_in + 1)), p, p < n, l, sc, k);
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// The top of a tree, layer l_in up to the root, in one launch of one
// 8-CTA cluster (4 warps per CTA: one per scheduler, 64 groups): a level's
// parents are spread over the groups, and the hardware cluster barrier
// (release / acquire) orders one level's stores before the next level's
// loads, which read L2 (__ldcg). Warps without a parent in a pass skip it.
constexpr uint32_t kTopCtas = 8, kTopThreads = 128, kTopGroups = kTopCtas * kTopThreads / 16;
__global__ void __cluster_dims__(kTopCtas, 1, 1) __launch_bounds__(kTopThreads)
    compress_top_kernel(uint64_t *layers, uint64_t H, uint32_t l_in, uint32_t depth) {
    __shared__ uint64_t sc[p2::N_PARAMS];
    p2x::stage_consts(sc);
    const int l = threadIdx.x & 15;
    const p2x::Lane k = p2x::lane_consts(sc, l);
    const uint32_t gid = (blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    for (uint32_t lv = l_in; lv < depth; lv++) {
        const uint64_t n = H >> (lv + 1);
        const uint64_t off_in = 2 * H - 2 * (H >> lv), off_out = 2 * H - 2 * (H >> (lv + 1));
        for (uint64_t base = 0; base < n; base += kTopGroups)
            if (base + (gid & ~1u) < n)  // warp-uniform: the warp's first group has a parent
                compress_parent_coop(layers, off_in, off_out, base + gid, base + gid < n, l, sc, k);
        cluster_sync();
    }
}

// Digest layers of a tree whose layer l holds one digest c_l repeated:
// digest g (0 <= g < 2H - 1) belongs to layer l with H >> l = 2^(ceil(log2(2H - g)) - 1).
__global__ void fill_const_layers_kernel(uint64_t *layers, uint64_t H, uint32_t depth, const uint64_t *c) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= 2 * H - 1) return;
    const uint64_t r1 = 2 * H - g;  // >= 2
    const uint32_t lg = 64 - __clzll(r1 - 1);
    const uint32_t l = depth - (lg - 1);
#pragma unroll
    for (int k = 0; k < 4; k++) layers[4 * g + k] = c[4 * l + k];
}

}  // namespace merkle
