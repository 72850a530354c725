// Goldilocks field F (p = 2^64 - 2^32 + 1) and its quadratic extension
// EF = F[x]/(x^2 - 7), for device kernels and the host-side transcript.
//
// All values are kept canonical (< p). Multiplication reduces the 128-bit
// product with 2^64 = 2^32 - 1 and 2^96 = -1 (mod p).
#pragma once
#include <cstdint>

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

GL_HD uint64_t add(uint64_t a, uint64_t b) {
    uint64_t r = a + b;
    if (r < a || r >= P) r -= P;
    return r;
}
GL_HD uint64_t sub(uint64_t a, uint64_t b) {
    uint64_t r = a - b;
    if (a < b) r += P;
    return r;
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
// 64x64 -> 128 product by 32-bit partial products on carry chains, then the
// reduction 2^64 = 2^32 - 1, 2^96 = -1 on the same chains. The result is
// weakly reduced: below 2^64 and congruent mod p (not necessarily < p).
__device__ __forceinline__ uint64_t mul_weak(uint64_t a, uint64_t b) {
    uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    uint32_t r0, r1, r2, r3, t, ul, uh;
    asm("mul.lo.u32 %0, %7, %9;\n\t"
        "mul.hi.u32 %1, %7, %9;\n\t"
        "mad.lo.cc.u32 %1, %7, %10, %1;\n\t"
        "madc.hi.u32 %2, %7, %10, 0;\n\t"
        "mad.lo.cc.u32 %1, %8, %9, %1;\n\t"
        "madc.hi.cc.u32 %2, %8, %9, %2;\n\t"
        "madc.hi.u32 %3, %8, %10, 0;\n\t"
        "mad.lo.cc.u32 %2, %8, %10, %2;\n\t"
        "addc.u32 %3, %3, 0;\n\t"
        // (r1:r0) - r3, on borrow subtract eps
        "sub.cc.u32 %0, %0, %3;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32 %4, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, %4;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        // + r2 * eps = (r2 << 32) - r2, on carry add eps
        "sub.cc.u32 %5, 0, %2;\n\t"
        "subc.u32 %6, %2, 0;\n\t"
        "add.cc.u32 %0, %0, %5;\n\t"
        "addc.cc.u32 %1, %1, %6;\n\t"
        "addc.u32 %4, 0, 0;\n\t"
        "neg.s32 %4, %4;\n\t"
        "add.cc.u32 %0, %0, %4;\n\t"
        "addc.u32 %1, %1, 0;"
        : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3), "=&r"(t), "=&r"(ul), "=&r"(uh)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
    return ((uint64_t)r1 << 32) | r0;
}
#endif
GL_HD uint64_t mul(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    uint64_t r = mul_weak(a, b);
    return r >= P ? r - P : r;
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
