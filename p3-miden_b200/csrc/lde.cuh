// Coset LDE kernels: radix-8 rounds over groups of rows staged in shared
// memory, three global trips per transform of up to 2^20 rows.
//
// A matrix is h x w, row-major, one polynomial per column; h = 2^L. The
// bit positions [0, L) of a row index are split into ranges of at most 10
// bits. For a range [blo, blo + k) a block loads one group (the 2^k rows
// whose index agrees outside the range; stride 2^blo) for a tile of C
// columns, runs the k radix-2 stages of that range as rounds of up to three
// stages, and stores the group back.
//
// The LDE of a trace on s*K, |K| = h*B (p3-dft/src/traits.rs coset_lde_batch
// semantics: natural-order evaluations in, bit-reversed coset evaluations
// out) is
//   - inverse transform, decimation in time, ranges in ascending order; the
//     first range reads row bitrev_L(i) for position i, so the result is in
//     natural coefficient order (times h);
//   - for every coset c of K over H, (s*w_{hB}^c)*H: coefficient i times
//     (s*w_{hB}^c)^i / h, then a forward transform, decimation in frequency,
//     ranges in descending order, whose bit-reversed output is exactly the
//     committed layout of coset c (rows [bitrev_B(c)*h, +h)).
// The top range is the same set of rows for the last inverse range and the
// first forward range, so one kernel does both: it keeps the group's
// coefficients in shared memory and runs the forward range once per coset
// (lde_fused_kernel). A transform of L <= 10 is that kernel alone; L <= 20 is
// three launches (inverse low range, fused top range, forward low range over
// all cosets).
//
// Round arithmetic. For a round over global bits [b, b+R) and positions
// x_j = a[hi + j*2^b + l] (l = position mod 2^b), the R stages of
// decimation in frequency equal a size-2^R transform with the small root
// w_{2^R} followed by multiplying output p by t^{bitrev_R(p)},
// t = w_{2^{b+R}}^l; decimation in time is the transpose (multiply input p
// by t^{bitrev_R(p)}, then the small transform). The small roots are powers
// of two modulo p: w_8 = 2^120 = -2^24, w_4 = 2^48 (forward) and
// w_8^-1 = 2^72, w_4^-1 = -2^48 (inverse), so the small transforms cost
// shifts, not multiplications. The powers t^e of every round are built once
// per block in a shared table (2^k - 1 entries per direction).
//
// All values stay canonical (< p).
#pragma once
#include "gl.cuh"
#include "ntt.cuh"

namespace lde {

__device__ __forceinline__ uint64_t add(uint64_t a, uint64_t b) { return gl::add_dev(a, b); }
__device__ __forceinline__ uint64_t sub(uint64_t a, uint64_t b) { return gl::sub_dev(a, b); }
__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) { return gl::mul(a, b); }

// x * 2^S mod p (canonical) for x < 2^64 and S in {24, 48}: the 128-bit
// product (x >> (64 - S)) * 2^64 + (x << S) reduced with 2^64 = eps and
// 2^96 = -1 on carry chains; the last step folds the carry and the
// comparison with p into one select.
template <int S>
__device__ __forceinline__ uint64_t shl(uint64_t x) {
    static_assert(S == 24 || S == 48, "shift");
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
    uint32_t l0, l1, h0, h1;  // x << S = (l1:l0), x >> (64 - S) = (h1:h0)
    if (S == 24) {
        l0 = x0 << 24;
        l1 = __funnelshift_l(x0, x1, 24);
        h0 = x1 >> 8;
        h1 = 0;
    } else {
        l0 = 0;
        l1 = x0 << 16;
        h0 = __funnelshift_r(x0, x1, 16);
        h1 = x1 >> 16;
    }
    uint32_t r0, r1;
    if (S == 24) {  // h1 = 0: the generic form's first five instructions do nothing
        asm("{\n\t.reg .u32 m, u0, u1, t0, t1;\n\t.reg .pred q;\n\t"
            "sub.cc.u32 u0, 0, %4;\n\t"    // h0*eps
            "subc.u32 u1, %4, 0;\n\t"
            "add.cc.u32 %0, %2, u0;\n\t"
            "addc.cc.u32 %1, %3, u1;\n\t"
            "addc.u32 m, 0, 0;\n\t"
            "add.cc.u32 t0, %0, 0xFFFFFFFF;\n\t"  // r + eps: r - p, or the value of a wrapped sum
            "addc.cc.u32 t1, %1, 0;\n\t"
            "addc.u32 m, m, 0;\n\t"
            "setp.ne.u32 q, m, 0;\n\t"
            "selp.b32 %0, t0, %0, q;\n\t"
            "selp.b32 %1, t1, %1, q;\n\t}"
            : "=&r"(r0), "=&r"(r1)
            : "r"(l0), "r"(l1), "r"(h0));
        return ((uint64_t)r1 << 32) | r0;
    }
    asm("{\n\t.reg .u32 m, u0, u1, t0, t1;\n\t.reg .pred q;\n\t"
        "sub.cc.u32 %0, %2, %5;\n\t"   // (l1:l0) - h1
        "subc.cc.u32 %1, %3, 0;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"    // on borrow subtract eps
        "subc.u32 %1, %1, 0;\n\t"
        "sub.cc.u32 u0, 0, %4;\n\t"    // + h0*eps
        "subc.u32 u1, %4, 0;\n\t"
        "add.cc.u32 %0, %0, u0;\n\t"
        "addc.cc.u32 %1, %1, u1;\n\t"
        "addc.u32 m, 0, 0;\n\t"
        "add.cc.u32 t0, %0, 0xFFFFFFFF;\n\t"  // r + eps: r - p, or the value of a wrapped sum
        "addc.cc.u32 t1, %1, 0;\n\t"
        "addc.u32 m, m, 0;\n\t"
        "setp.ne.u32 q, m, 0;\n\t"
        "selp.b32 %0, t0, %0, q;\n\t"
        "selp.b32 %1, t1, %1, q;\n\t}"
        : "=&r"(r0), "=&r"(r1)
        : "r"(l0), "r"(l1), "r"(h0), "r"(h1));
    return ((uint64_t)r1 << 32) | r0;
}

// x * 2^72 mod p (canonical) for x < 2^64. With (a1:a0) = (x << 8) mod 2^64
// and y = x >> 56, x * 2^72 = (x << 8) * 2^64 = (a0 - y) * 2^32 - (a0 + a1)
// mod p (2^64 = eps, 2^128 = -2^32). That value lies in (-2^41, p), so the
// borrow of one subtraction decides the only correction (+p). Ten
// instructions in place of shl<48>(shl<24>(x)).
__device__ __forceinline__ uint64_t shl72(uint64_t x) {
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
    const uint32_t a0 = x0 << 8, a1 = __funnelshift_l(x0, x1, 8), y = x1 >> 24;
    uint32_t r0, r1;
    asm("{\n\t.reg .u32 s0, s1, m;\n\t"
        "add.cc.u32 s0, %2, %3;\n\t"   // s = a0 + a1 + y * 2^32
        "addc.u32 s1, %4, 0;\n\t"
        "sub.cc.u32 %0, 0, s0;\n\t"    // (a0 : 0) - s, borrow when negative
        "subc.cc.u32 %1, %2, s1;\n\t"
        "subc.u32 m, 0, 0;\n\t"        // borrow: m = 0xFFFFFFFF = eps
        "sub.cc.u32 %0, %0, m;\n\t"    // negative: + p = - eps (mod 2^64)
        "subc.u32 %1, %1, 0;\n\t}"
        : "=&r"(r0), "=&r"(r1)
        : "r"(a0), "r"(a1), "r"(y));
    return ((uint64_t)r1 << 32) | r0;
}

__host__ __device__ constexpr uint32_t brev(uint32_t p, int R) {
    return R == 3 ? ((p & 1) << 2) | (p & 2) | ((p >> 2) & 1) : R == 2 ? ((p & 1) << 1) | ((p >> 1) & 1) : p;
}

// Size-2^R transforms with power-of-two roots. dif: natural input, output
// position p holds frequency bitrev_R(p) (forward roots). dit: input
// position p holds bitrev_R(p), natural output (inverse roots).
template <int R>
__device__ __forceinline__ void dft_dif(uint64_t *x) {
    if (R == 3) {
        const uint64_t a0 = add(x[0], x[4]), a4 = sub(x[0], x[4]);
        const uint64_t a1 = add(x[1], x[5]), a5 = shl<24>(sub(x[5], x[1]));          // * w8 = -2^24
        const uint64_t a2 = add(x[2], x[6]), a6 = shl<48>(sub(x[2], x[6]));          // * w8^2 = 2^48
        const uint64_t a3 = add(x[3], x[7]), a7 = shl72(sub(x[7], x[3]));  // * w8^3 = -2^72
        const uint64_t b0 = add(a0, a2), b2 = sub(a0, a2);
        const uint64_t b1 = add(a1, a3), b3 = shl<48>(sub(a1, a3));
        const uint64_t b4 = add(a4, a6), b6 = sub(a4, a6);
        const uint64_t b5 = add(a5, a7), b7 = shl<48>(sub(a5, a7));
        x[0] = add(b0, b1), x[1] = sub(b0, b1);
        x[2] = add(b2, b3), x[3] = sub(b2, b3);
        x[4] = add(b4, b5), x[5] = sub(b4, b5);
        x[6] = add(b6, b7), x[7] = sub(b6, b7);
    } else if (R == 2) {
        const uint64_t a0 = add(x[0], x[2]), a2 = sub(x[0], x[2]);
        const uint64_t a1 = add(x[1], x[3]), a3 = shl<48>(sub(x[1], x[3]));  // * w4 = 2^48
        x[0] = add(a0, a1), x[1] = sub(a0, a1);
        x[2] = add(a2, a3), x[3] = sub(a2, a3);
    } else {
        const uint64_t a0 = add(x[0], x[1]), a1 = sub(x[0], x[1]);
        x[0] = a0, x[1] = a1;
    }
}
template <int R>
__device__ __forceinline__ void dft_dit(uint64_t *x) {
    if (R == 3) {
        const uint64_t a0 = add(x[0], x[1]), a1 = sub(x[0], x[1]);
        const uint64_t a2 = add(x[2], x[3]), a3 = sub(x[2], x[3]);
        const uint64_t a4 = add(x[4], x[5]), a5 = sub(x[4], x[5]);
        const uint64_t a6 = add(x[6], x[7]), a7 = sub(x[6], x[7]);
        uint64_t v = shl<48>(a3);  // * w4^-1 = -2^48
        const uint64_t c0 = add(a0, a2), c2 = sub(a0, a2);
        const uint64_t c1 = sub(a1, v), c3 = add(a1, v);
        v = shl<48>(a7);
        const uint64_t c4 = add(a4, a6), c6 = sub(a4, a6);
        const uint64_t c5 = sub(a5, v), c7 = add(a5, v);
        x[0] = add(c0, c4), x[4] = sub(c0, c4);
        v = shl72(c5);  // * w8^-1 = 2^72
        x[1] = add(c1, v), x[5] = sub(c1, v);
        v = shl<48>(c6);  // * w8^-2 = -2^48
        x[2] = sub(c2, v), x[6] = add(c2, v);
        v = shl<24>(c7);  // * w8^-3 = 2^24
        x[3] = add(c3, v), x[7] = sub(c3, v);
    } else if (R == 2) {
        const uint64_t a0 = add(x[0], x[1]), a1 = sub(x[0], x[1]);
        const uint64_t a2 = add(x[2], x[3]), a3 = sub(x[2], x[3]);
        const uint64_t v = shl<48>(a3);  // * w4^-1 = -2^48
        x[0] = add(a0, a2), x[2] = sub(a0, a2);
        x[1] = sub(a1, v), x[3] = add(a1, v);
    } else {
        const uint64_t a0 = add(x[0], x[1]), a1 = sub(x[0], x[1]);
        x[0] = a0, x[1] = a1;
    }
}

// Rounds of a k-bit range: decimation in time ascends from bit 0 in rounds
// of 3 (the last one shorter), decimation in frequency descends from bit k
// (the last one, at bit 0, shorter).
__device__ __forceinline__ void round_bits(bool dif, uint32_t k, uint32_t rd, uint32_t &q_lo, uint32_t &r) {
    if (dif) {
        const int hi = (int)k - 3 * (int)rd;
        q_lo = hi >= 3 ? hi - 3 : 0;
        r = hi - q_lo;
    } else {
        q_lo = 3 * rd;
        r = k - q_lo < 3 ? k - q_lo : 3;
    }
}

// Shared twiddle table of a k-bit range at global bit blo for a group with
// low position bits base_lo: the round at local bit q_lo with R bits
// occupies entries [2^q_lo - 1, 2^(q_lo+R) - 1); entry (l, e), e in
// [1, 2^R), is t_l^e with t_l = w_{2^(b+R)}^(base_lo + l*2^blo), b = blo + q_lo.
template <bool DIF>
__device__ void fill_table(uint64_t *T, uint32_t k, uint32_t blo, uint64_t base_lo, uint32_t L,
                           const ntt::PowTab &root, uint32_t tid, uint32_t nthreads) {
    const uint32_t nr = (k + 2) / 3;
    for (uint32_t rd = 0; rd < nr; rd++) {
        uint32_t q_lo, r;
        round_bits(DIF, k, rd, q_lo, r);
        const uint32_t em1 = (1u << r) - 1, b = blo + q_lo;
        const uint64_t emask = (1ull << (b + r)) - 1;
        uint64_t *Tr = T + ((1u << q_lo) - 1);
        for (uint32_t rel = tid; rel < (em1 << q_lo); rel += nthreads) {
            const uint32_t li = r == 3 ? rel / 7 : r == 2 ? rel / 3 : rel;
            const uint32_t e = rel - li * em1 + 1;
            const uint64_t l = base_lo + ((uint64_t)li << blo);
            Tr[rel] = root.at(((l * e) & emask) << (L - b - r));
        }
    }
}

// One round over the group in shared memory (element m of column c at
// sm[m*C + c]); T is the round's table, or null when every t is 1.
template <int C, int R, bool DIF>
__device__ __forceinline__ void round(uint64_t *sm, const uint64_t *T, uint32_t q_lo, uint32_t k, uint32_t c,
                                      uint32_t t, uint32_t TPC) {
    constexpr uint32_t E = 1u << R;
    const uint32_t tasks = (1u << k) >> R;
    const uint32_t stride = C << q_lo;
    for (uint32_t task = t; task < tasks; task += TPC) {
        const uint32_t low = task & ((1u << q_lo) - 1);
        const uint32_t mb = low | ((task >> q_lo) << (q_lo + R));
        uint64_t *px = sm + mb * C + c;
        uint64_t x[E];
#pragma unroll
        for (uint32_t j = 0; j < E; j++) x[j] = px[j * stride];
        const uint64_t *Tl = T ? T + low * (E - 1) : nullptr;
        if (!DIF && Tl) {
#pragma unroll
            for (uint32_t p = 1; p < E; p++) x[p] = mul(x[p], Tl[brev(p, R) - 1]);
        }
        if (DIF) dft_dif<R>(x);
        else dft_dit<R>(x);
        if (DIF && Tl) {
#pragma unroll
            for (uint32_t p = 1; p < E; p++) x[p] = mul(x[p], Tl[brev(p, R) - 1]);
        }
#pragma unroll
        for (uint32_t j = 0; j < E; j++) px[j * stride] = x[j];
    }
}

// All rounds of a k-bit range; every round ends with a block barrier.
// tw_low: whether the round at bit 0 has a nontrivial table (base_lo != 0).
template <int C, bool DIF, int KT = 0>
__device__ __forceinline__ void run_rounds(uint64_t *sm, const uint64_t *T, bool tw_low, uint32_t k_rt, uint32_t c,
                                           uint32_t t, uint32_t TPC_rt) {
    const uint32_t k = KT ? (uint32_t)KT : k_rt;
    const uint32_t TPC = KT ? (1u << KT) / 8 : TPC_rt;
    const uint32_t nr = (k + 2) / 3;
#pragma unroll
    for (uint32_t rd = 0; rd < nr; rd++) {
        uint32_t q_lo, r;
        round_bits(DIF, k, rd, q_lo, r);
        const uint64_t *Tr = (q_lo == 0 && !tw_low) ? nullptr : T + ((1u << q_lo) - 1);
        if (r == 3) round<C, 3, DIF>(sm, Tr, q_lo, k, c, t, TPC);
        else if (r == 2) round<C, 2, DIF>(sm, Tr, q_lo, k, c, t, TPC);
        else round<C, 1, DIF>(sm, Tr, q_lo, k, c, t, TPC);
        __syncthreads();
    }
}

struct PassArgs {
    const uint64_t *src;
    uint64_t *dst;
    uint64_t ld_src, ld_dst;      // row strides in words
    uint64_t src_blk, dst_blk;    // words between the blocks of blockIdx.y (cosets of forward passes)
    uint64_t w;                   // columns
    uint32_t L, blo, k;           // transform size 2^L; range [blo, blo + k)
    uint32_t n_tiles;             // column tiles; blockIdx.x = group * n_tiles + tile
    uint32_t src_bitrev;          // position i is read from row bitrev_L(i)
    ntt::PowTab root;             // powers of w_h (forward) or w_h^-1 (inverse)
};

struct FusedArgs {
    const uint64_t *src;
    uint64_t *dst;
    uint64_t ld_src, ld_dst;
    uint64_t w;
    uint32_t L, blo, k, n_tiles, src_bitrev;
    uint32_t log_cosets;          // B = 2^log_cosets output cosets of h rows each
    ntt::PowTab inv_root, fwd_root;
    // scale of coset c: coefficient i times scale_lo[c*2^lo_bits + (i mod 2^lo_bits)] *
    // scale_hi[c*scale_hi_len + (i >> lo_bits)] = (s*w_{hB}^c)^i / h
    const uint64_t *scale_lo, *scale_hi;
    uint32_t scale_lo_bits;
    uint64_t scale_hi_len;
    // optional per-column factor: coefficient i of column col times
    // colpow(col/2)^i (quotient chunks); null when absent
    const uint64_t *cp_lo, *cp_hi;
    uint32_t cp_lo_bits;
    uint64_t cp_hi_len;
};

__device__ __forceinline__ void group_of(uint64_t g, uint32_t blo, uint32_t k, uint64_t &base, uint64_t &base_lo) {
    const uint64_t S = 1ull << blo;
    base = (g & (S - 1)) | ((g >> blo) << (blo + k));
    base_lo = base & (S - 1);
}

// One range of the inverse (DIF = false) or forward (DIF = true) transform;
// KT != 0 fixes the range's bit count at compile time (blockDim = 2^KT / 8 * C).
template <int C, bool DIF, int KT = 0>
__global__ void __launch_bounds__(1024) lde_pass_kernel(const __grid_constant__ PassArgs a) {
    extern __shared__ uint64_t sm[];
    const uint32_t kk = KT ? (uint32_t)KT : a.k;
    const uint32_t G = 1u << kk;
    uint64_t *T = sm + (size_t)G * C;
    const uint32_t tile = blockIdx.x % a.n_tiles;
    uint64_t base, base_lo;
    group_of(blockIdx.x / a.n_tiles, a.blo, kk, base, base_lo);
    const uint64_t col0 = (uint64_t)tile * C;
    const uint32_t tid = threadIdx.x, c = tid % C, t = tid / C, TPC = KT ? G / 8 : blockDim.x / C;
    const bool col_ok = col0 + c < a.w;
    const uint64_t *src = a.src + blockIdx.y * a.src_blk + col0 + c;
    uint64_t *dst = a.dst + blockIdx.y * a.dst_blk + col0 + c;
    for (uint32_t m = t; m < G; m += TPC) {
        const uint64_t P = base + ((uint64_t)m << a.blo);
        const uint64_t row = a.src_bitrev ? gl::bitrev(P, a.L) : P;
        sm[m * C + c] = col_ok ? __ldg(src + row * a.ld_src) : 0;
    }
    fill_table<DIF>(T, kk, a.blo, base_lo, a.L, a.root, tid, blockDim.x);
    __syncthreads();
    run_rounds<C, DIF, KT>(sm, T, base_lo != 0, kk, c, t, TPC);
    if (!col_ok) return;
    for (uint32_t m = t; m < G; m += TPC) {
        const uint64_t P = base + ((uint64_t)m << a.blo);
        dst[P * a.ld_dst] = sm[m * C + c];
    }
}

// The top range: inverse rounds, then per coset the scale and the forward
// rounds, written to the coset's block of the output.
template <int C, int KT = 0>
__global__ void __launch_bounds__(1024) lde_fused_kernel(const __grid_constant__ FusedArgs a) {
    extern __shared__ uint64_t sm[];
    const uint32_t kk = KT ? (uint32_t)KT : a.k;
    const uint32_t G = 1u << kk;
    uint64_t *A = sm, *Bf = A + (size_t)G * C, *Ti = Bf + (size_t)G * C, *Tf = Ti + G, *sc = Tf + G;
    const uint32_t tile = blockIdx.x % a.n_tiles;
    uint64_t base, base_lo;
    group_of(blockIdx.x / a.n_tiles, a.blo, kk, base, base_lo);
    const uint64_t col0 = (uint64_t)tile * C;
    const uint32_t tid = threadIdx.x, c = tid % C, t = tid / C, TPC = KT ? G / 8 : blockDim.x / C;
    const uint64_t col = col0 + c;
    const bool col_ok = col < a.w;
    for (uint32_t m = t; m < G; m += TPC) {
        const uint64_t P = base + ((uint64_t)m << a.blo);
        const uint64_t row = a.src_bitrev ? gl::bitrev(P, a.L) : P;
        A[m * C + c] = col_ok ? __ldg(a.src + row * a.ld_src + col) : 0;
    }
    fill_table<false>(Ti, kk, a.blo, base_lo, a.L, a.inv_root, tid, blockDim.x);
    fill_table<true>(Tf, kk, a.blo, base_lo, a.L, a.fwd_root, tid, blockDim.x);
    __syncthreads();
    run_rounds<C, false, KT>(A, Ti, base_lo != 0, kk, c, t, TPC);
    const uint64_t h = 1ull << a.L;
    const uint32_t B = 1u << a.log_cosets;
    const uint64_t lo_mask = (1ull << a.scale_lo_bits) - 1;
    for (uint32_t cs = 0; cs < B; cs++) {
        const uint64_t *slo = a.scale_lo + ((uint64_t)cs << a.scale_lo_bits);
        const uint64_t *shi = a.scale_hi + cs * a.scale_hi_len;
        for (uint32_t m = tid; m < G; m += blockDim.x) {
            const uint64_t P = base + ((uint64_t)m << a.blo);
            sc[m] = mul(__ldg(slo + (P & lo_mask)), __ldg(shi + (P >> a.scale_lo_bits)));
        }
        __syncthreads();
        for (uint32_t m = t; m < G; m += TPC) {
            uint64_t v = mul(A[m * C + c], sc[m]);
            if (a.cp_lo && col_ok) {
                const uint64_t P = base + ((uint64_t)m << a.blo), tc = col / 2;
                const uint64_t f = mul(__ldg(a.cp_lo + (tc << a.cp_lo_bits) + (P & ((1ull << a.cp_lo_bits) - 1))),
                                       __ldg(a.cp_hi + tc * a.cp_hi_len + (P >> a.cp_lo_bits)));
                v = mul(v, f);
            }
            Bf[m * C + c] = v;
        }
        __syncthreads();
        run_rounds<C, true, KT>(Bf, Tf, base_lo != 0, kk, c, t, TPC);
        if (col_ok) {
            uint64_t *dst = a.dst + (uint64_t)gl::bitrev(cs, a.log_cosets) * h * a.ld_dst + col;
            for (uint32_t m = t; m < G; m += TPC) {
                const uint64_t P = base + ((uint64_t)m << a.blo);
                dst[P * a.ld_dst] = Bf[m * C + c];
            }
        }
        // the next coset writes sc (not read by the stores) and, after a
        // barrier, Bf
    }
}

}  // namespace lde
