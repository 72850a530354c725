// Goldilocks field F (p = 2^64 - 2^32 + 1) and its quadratic extension
// EF = F[x]/(x^2 - 7), for device kernels and the host-side transcript.
//
// All values are kept canonical (< p). Multiplication reduces the 128-bit
// product with 2^64 = 2^32 - 1 and 2^96 = -1 (mod p).
#pragma once
#if defined(__CUDACC_RTC__)
// compiled at run time by NVRTC as the prelude of generated constraint
// kernels (symair.cuh): no standard headers there
typedef unsigned long long uint64_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef int int32_t;
#else
#include <cstdint>
#endif

#if defined(__CUDACC__)
#define GL_HD __host__ __device__ __forceinline__
#else
#define GL_HD inline
#endif

namespace gl {

constexpr uint64_t P = 0xFFFFFFFF00000001ULL;
constexpr uint64_t EPS = 0xFFFFFFFFULL;  // 2^64 mod p
constexpr uint64_t W = 7;                // EF non-residue
constexpr uint64_t GEN = 7;              // multiplicative generator

#if defined(__CUDACC__)
// Device forms on 32-bit carry chains: no 64-bit compares or selects on the
// carries. Inputs and outputs as the host forms below.
__device__ __forceinline__ uint64_t add_dev(uint64_t a, uint64_t b) {  // a, b < p
    uint32_t r0, r1;
    asm("{\n\t.reg .u32 t0, t1, c;\n\t.reg .pred q;\n\t"
        "add.cc.u32 %0, %2, %4;\n\t"
        "addc.cc.u32 %1, %3, %5;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "add.cc.u32 t0, %0, 0xFFFFFFFF;\n\t"  // sum + eps = sum - p (mod 2^64)
        "addc.cc.u32 t1, %1, 0;\n\t"
        "addc.u32 c, c, 0;\n\t"                // sum >= 2^64 or sum >= p (never both)
        "setp.ne.u32 q, c, 0;\n\t"
        "selp.b32 %0, t0, %0, q;\n\t"
        "selp.b32 %1, t1, %1, q;\n\t}"
        : "=&r"(r0), "=&r"(r1)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}
// b < p: a - b mod p, below p when a < p, below 2^64 (weak) when a < 2^64
__device__ __forceinline__ uint64_t sub_dev(uint64_t a, uint64_t b) {
    uint32_t r0, r1;
    asm("{\n\t.reg .u32 m;\n\t"
        "sub.cc.u32 %0, %2, %4;\n\t"
        "subc.cc.u32 %1, %3, %5;\n\t"
        "subc.u32 m, 0, 0;\n\t"    // borrow: 0xFFFFFFFF = eps
        "sub.cc.u32 %0, %0, m;\n\t"  // a - b + 2^64 - eps = a - b + p
        "subc.u32 %1, %1, 0;\n\t}"
        : "=&r"(r0), "=&r"(r1)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}
// x < 2^64 -> x mod p (x >= p iff x + eps carries)
__device__ __forceinline__ uint64_t canon_dev(uint64_t x) {
    uint32_t r0, r1;
    asm("{\n\t.reg .u32 t0, t1, c;\n\t.reg .pred q;\n\t"
        "add.cc.u32 t0, %2, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 t1, %3, 0;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "setp.ne.u32 q, c, 0;\n\t"
        "selp.b32 %0, t0, %2, q;\n\t"
        "selp.b32 %1, t1, %3, q;\n\t}"
        : "=&r"(r0), "=&r"(r1)
        : "r"((uint32_t)x), "r"((uint32_t)(x >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}
#endif
GL_HD uint64_t add(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return add_dev(a, b);
#else
    uint64_t r = a + b;
    if (r < a || r >= P) r -= P;
    return r;
#endif
}
GL_HD uint64_t sub(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return sub_dev(a, b);
#else
    uint64_t r = a - b;
    if (a < b) r += P;
    return r;
#endif
}
GL_HD uint64_t neg(uint64_t a) { return a ? P - a : 0; }
GL_HD uint64_t dbl(uint64_t a) { return add(a, a); }

GL_HD uint64_t mulhi(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}
// reduce hi*2^64 + lo
GL_HD uint64_t reduce128(uint64_t hi, uint64_t lo) {
    uint64_t hh = hi >> 32, hl = hi & EPS;
    uint64_t t = lo - hh;
    if (lo < hh) t -= EPS;
    uint64_t t1 = hl * EPS;
    uint64_t r = t + t1;
    if (r < t1) r += EPS;
    if (r >= P) r -= P;
    return r;
}
#if defined(__CUDACC__)
// r0 + r1*2^32 + r2*2^64 + r3*2^96 -> a value below 2^64 congruent mod p
// (weakly reduced). With 2^64 = 2^32 - 1 and 2^96 = -1 the value is
// V = r0 + 2^32 (r1 + r2) - (r2 + r3), in (-2^33, 2^65 + 2^32): one carry
// chain forms (r1 + r2 : r0) - (r2 + r3) mod 2^64 and k = carry - borrow in
// {-1, 0, 1}, then k * eps (2^64 = eps) is added; neither direction wraps again.
__device__ __forceinline__ uint64_t reduce4_dev(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
    uint32_t o0, o1;
    asm("{\n\t.reg .u32 s0, s1, h, c, k;\n\t"
        "add.cc.u32 s0, %4, %5;\n\t"  // s = r2 + r3 (33 bits)
        "addc.u32 s1, 0, 0;\n\t"
        "add.cc.u32 h, %3, %4;\n\t"   // h = r1 + r2, carry c
        "addc.u32 c, 0, 0;\n\t"
        "sub.cc.u32 %0, %2, s0;\n\t"  // (h:r0) - (s1:s0), borrow b
        "subc.cc.u32 %1, h, s1;\n\t"
        "subc.u32 k, c, 0;\n\t"       // k = c - b
        "neg.s32 s0, k;\n\t"          // k * eps = (k >> 31 : -k)
        "shr.s32 s1, k, 31;\n\t"
        "add.cc.u32 %0, %0, s0;\n\t"
        "addc.u32 %1, %1, s1;\n\t}"
        : "=&r"(o0), "=&r"(o1)
        : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
    return ((uint64_t)o1 << 32) | o0;
}
// 64x64 -> 128 product by 32-bit partial products on carry chains.
__device__ __forceinline__ void mul128_dev(uint64_t a, uint64_t b, uint32_t &r0, uint32_t &r1, uint32_t &r2,
                                           uint32_t &r3) {
    asm("mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.u32 %2, %4, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "addc.u32 %3, %3, 0;"
        : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
}
// a*b for a, b < 2^64, weakly reduced.
__device__ __forceinline__ uint64_t mul_weak(uint64_t a, uint64_t b) {
    uint32_t r0, r1, r2, r3;
    mul128_dev(a, b, r0, r1, r2, r3);
    return reduce4_dev(r0, r1, r2, r3);
}
// Wide value lo + hi * 2^64 (below 2^96), an integer congruent mod p: a chain
// of sums and differences accumulates here and is reduced once at its end.
struct Wide {
    uint64_t lo;
    uint32_t hi;
};
__device__ __forceinline__ Wide wide_add(Wide a, Wide b) {  // the caller keeps a + b below 2^96
    uint32_t r0, r1, h;
    asm("add.cc.u32 %0, %3, %6;\n\t"
        "addc.cc.u32 %1, %4, %7;\n\t"
        "addc.u32 %2, %5, %8;"
        : "=&r"(r0), "=&r"(r1), "=&r"(h)
        : "r"((uint32_t)a.lo), "r"((uint32_t)(a.lo >> 32)), "r"(a.hi), "r"((uint32_t)b.lo),
          "r"((uint32_t)(b.lo >> 32)), "r"(b.hi));
    return Wide{((uint64_t)r1 << 32) | r0, h};
}
// C - b for a constant multiple C = (c_hi : c_lo) of p with C >= b
__device__ __forceinline__ Wide wide_neg(Wide b, uint64_t c_lo, uint32_t c_hi) {
    uint32_t r0, r1, h;
    asm("sub.cc.u32 %0, %6, %3;\n\t"
        "subc.cc.u32 %1, %7, %4;\n\t"
        "subc.u32 %2, %8, %5;"
        : "=&r"(r0), "=&r"(r1), "=&r"(h)
        : "r"((uint32_t)b.lo), "r"((uint32_t)(b.lo >> 32)), "r"(b.hi), "r"((uint32_t)c_lo),
          "r"((uint32_t)(c_lo >> 32)), "r"(c_hi));
    return Wide{((uint64_t)r1 << 32) | r0, h};
}
// a + (C - b) = a - b (mod p), C as in wide_neg
__device__ __forceinline__ Wide wide_sub(Wide a, Wide b, uint64_t c_lo, uint32_t c_hi) {
    return wide_add(a, wide_neg(b, c_lo, c_hi));
}
// canonical value of a: lo + hi * eps (2^64 = eps mod p) with one wrap at
// most, then one conditional subtraction of p
__device__ __forceinline__ uint64_t wide_canon(Wide a) {
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
    return canon_dev(((uint64_t)r1 << 32) | r0);
}
#endif
#if defined(__CUDACC__)
// Lazy sum of products: sum a_i * b_i held in 160 bits (r4 counts the
// overflows past 2^128, so up to 2^32 products), reduced once.
struct Acc {
    uint32_t r0 = 0, r1 = 0, r2 = 0, r3 = 0, r4 = 0;
    __device__ __forceinline__ void mac(uint64_t a, uint64_t b) {  // += a*b, a, b < 2^64
        asm("mad.lo.cc.u32 %0, %5, %7, %0;\n\t"
            "madc.hi.cc.u32 %1, %5, %7, %1;\n\t"
            "madc.lo.cc.u32 %2, %6, %8, %2;\n\t"
            "madc.hi.cc.u32 %3, %6, %8, %3;\n\t"
            "addc.u32 %4, %4, 0;\n\t"
            "mad.lo.cc.u32 %1, %5, %8, %1;\n\t"
            "madc.hi.cc.u32 %2, %5, %8, %2;\n\t"
            "addc.cc.u32 %3, %3, 0;\n\t"
            "addc.u32 %4, %4, 0;\n\t"
            "mad.lo.cc.u32 %1, %6, %7, %1;\n\t"
            "madc.hi.cc.u32 %2, %6, %7, %2;\n\t"
            "addc.cc.u32 %3, %3, 0;\n\t"
            "addc.u32 %4, %4, 0;"
            : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(r4)
            : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    }
    __device__ __forceinline__ void add(uint64_t a) {  // += a, a < 2^64
        asm("add.cc.u32 %0, %0, %5;\n\t"
            "addc.cc.u32 %1, %1, %6;\n\t"
            "addc.cc.u32 %2, %2, 0;\n\t"
            "addc.cc.u32 %3, %3, 0;\n\t"
            "addc.u32 %4, %4, 0;"
            : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(r4)
            : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)));
    }
    // canonical value: 2^128 = -2^32 (mod p), and r4 * 2^32 < p
    __device__ __forceinline__ uint64_t reduce() const {
        return sub_dev(canon_dev(reduce4_dev(r0, r1, r2, r3)), (uint64_t)r4 << 32);
    }
};
#endif
GL_HD uint64_t mul(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return canon_dev(mul_weak(a, b));
#else
    return reduce128(mulhi(a, b), a * b);
#endif
}
GL_HD uint64_t sqr(uint64_t a) { return mul(a, a); }
GL_HD uint64_t pow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = mul(r, b);
        b = mul(b, b);
        e >>= 1;
    }
    return r;
}
GL_HD uint64_t inv(uint64_t a) { return pow(a, P - 2); }
GL_HD uint64_t exp2k(uint64_t a, unsigned k) {
    while (k--) a = mul(a, a);
    return a;
}
// primitive 2^k-th root of unity, 7^((p-1)/2^k)
GL_HD uint64_t root(unsigned k) { return pow(GEN, (P - 1) >> k); }
GL_HD uint64_t mul7(uint64_t a) {
    uint64_t a2 = add(a, a), a4 = add(a2, a2);
    return add(add(a4, a2), a);
}

struct ef {
    uint64_t c0, c1;
};
GL_HD ef ef_make(uint64_t a, uint64_t b) { return ef{a, b}; }
GL_HD ef ef_zero() { return ef{0, 0}; }
GL_HD ef ef_one() { return ef{1, 0}; }
GL_HD ef ef_add(ef a, ef b) { return ef{add(a.c0, b.c0), add(a.c1, b.c1)}; }
GL_HD ef ef_sub(ef a, ef b) { return ef{sub(a.c0, b.c0), sub(a.c1, b.c1)}; }
GL_HD ef ef_neg(ef a) { return ef{neg(a.c0), neg(a.c1)}; }
GL_HD ef ef_mulf(ef a, uint64_t b) { return ef{mul(a.c0, b), mul(a.c1, b)}; }
GL_HD ef ef_mul(ef a, ef b) {
    uint64_t m0 = mul(a.c0, b.c0), m1 = mul(a.c1, b.c1);
    uint64_t m2 = mul(add(a.c0, a.c1), add(b.c0, b.c1));
    return ef{add(m0, mul7(m1)), sub(sub(m2, m0), m1)};
}
GL_HD ef ef_sqr(ef a) { return ef_mul(a, a); }
GL_HD ef ef_inv(ef a) {
    uint64_t n = sub(mul(a.c0, a.c0), mul7(mul(a.c1, a.c1)));
    uint64_t ni = inv(n);
    return ef{mul(a.c0, ni), mul(neg(a.c1), ni)};
}
GL_HD bool ef_eq(ef a, ef b) { return a.c0 == b.c0 && a.c1 == b.c1; }
GL_HD ef ef_pow(ef b, uint64_t e) {
    ef r = ef_one();
    while (e) {
        if (e & 1) r = ef_mul(r, b);
        b = ef_mul(b, b);
        e >>= 1;
    }
    return r;
}
GL_HD ef ef_exp2k(ef a, unsigned k) {
    while (k--) a = ef_mul(a, a);
    return a;
}

GL_HD uint64_t bitrev(uint64_t x, unsigned bits) {
#if defined(__CUDA_ARCH__)
    return bits ? (__brevll(x) >> (64 - bits)) : 0;
#else
    uint64_t r = 0;
    for (unsigned i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
#endif
}

}  // namespace gl
