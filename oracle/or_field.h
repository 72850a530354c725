/*
 * ORACLE (test infrastructure only): Goldilocks field and its quadratic
 * extension, written for obviousness rather than speed.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg may use this
 * code, and only as the checker. The product never links it.
 *
 * Field: p = 2^64 - 2^32 + 1 (Goldilocks), the base field F of the
 * goldilocks_poseidon2 configuration (p3-miden-dev-utils/src/configs.rs:393-407).
 * Extension: EF = F[x]/(x^2 - 7). 7 is the smallest quadratic non-residue
 * mod p, which makes x^2 - 7 irreducible. The configuration's
 * BinomialExtensionField<F, 2> is this field (p3-field 0.5.0, not vendored).
 * Multiplicative generator: 7 (7^((p-1)/2) = -1 and 7 generates F*).
 * Two-adic generators: w_k = 7^((p-1)/2^k). w_32 = 0x185629dcda58878c.
 */
#ifndef OR_FIELD_H
#define OR_FIELD_H
#include <stdint.h>
#include <stddef.h>

#define OR_P 0xFFFFFFFF00000001ULL
#define OR_W 7ULL
#define OR_GEN 7ULL

typedef unsigned __int128 or_u128;

static inline uint64_t or_add(uint64_t a, uint64_t b) {
    or_u128 s = (or_u128)a + b;
    if (s >= OR_P) s -= OR_P;
    return (uint64_t)s;
}
static inline uint64_t or_sub(uint64_t a, uint64_t b) {
    return a >= b ? a - b : (uint64_t)((or_u128)a + OR_P - b);
}
static inline uint64_t or_neg(uint64_t a) { return a ? OR_P - a : 0; }
/* reference product: exact 128-bit remainder */
static inline uint64_t or_mul_ref(uint64_t a, uint64_t b) {
    return (uint64_t)(((or_u128)a * b) % OR_P);
}
/* product via 2^64 = 2^32 - 1 and 2^96 = -1 (mod p); equal to or_mul_ref */
static inline uint64_t or_mul(uint64_t a, uint64_t b) {
    or_u128 x = (or_u128)a * b;
    uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
    uint64_t hh = hi >> 32, hl = hi & 0xffffffffULL;
    uint64_t t = lo - hh;
    if (lo < hh) t -= 0xffffffffULL;
    uint64_t t1 = (hl << 32) - hl;
    uint64_t r = t + t1;
    if (r < t1) r += 0xffffffffULL;
    if (r >= OR_P) r -= OR_P;
    return r;
}
static inline uint64_t or_canon(uint64_t a) { return a >= OR_P ? a - OR_P : a; }
static inline uint64_t or_pow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = or_mul(r, b);
        b = or_mul(b, b);
        e >>= 1;
    }
    return r;
}
static inline uint64_t or_inv(uint64_t a) { return or_pow(a, OR_P - 2); }
/* primitive 2^k-th root of unity, the convention 7^((p-1)/2^k) */
static inline uint64_t or_root(unsigned k) { return or_pow(OR_GEN, (OR_P - 1) >> k); }
static inline uint64_t or_exp2(uint64_t a, unsigned k) {
    while (k--) a = or_mul(a, a);
    return a;
}

typedef struct { uint64_t c0, c1; } or_ef;

static inline or_ef or_ef_make(uint64_t a, uint64_t b) { or_ef r = {a, b}; return r; }
static inline or_ef or_ef_from(uint64_t a) { or_ef r = {a, 0}; return r; }
static inline or_ef or_ef_add(or_ef a, or_ef b) { return or_ef_make(or_add(a.c0, b.c0), or_add(a.c1, b.c1)); }
static inline or_ef or_ef_sub(or_ef a, or_ef b) { return or_ef_make(or_sub(a.c0, b.c0), or_sub(a.c1, b.c1)); }
static inline or_ef or_ef_neg(or_ef a) { return or_ef_make(or_neg(a.c0), or_neg(a.c1)); }
static inline or_ef or_ef_mul(or_ef a, or_ef b) {
    uint64_t c0 = or_add(or_mul(a.c0, b.c0), or_mul(OR_W, or_mul(a.c1, b.c1)));
    uint64_t c1 = or_add(or_mul(a.c0, b.c1), or_mul(a.c1, b.c0));
    return or_ef_make(c0, c1);
}
static inline or_ef or_ef_mulf(or_ef a, uint64_t b) { return or_ef_make(or_mul(a.c0, b), or_mul(a.c1, b)); }
static inline int or_ef_eq(or_ef a, or_ef b) { return a.c0 == b.c0 && a.c1 == b.c1; }
static inline or_ef or_ef_inv(or_ef a) {
    /* (a0 + a1 x)^-1 = (a0 - a1 x) / (a0^2 - W a1^2) */
    uint64_t n = or_sub(or_mul(a.c0, a.c0), or_mul(OR_W, or_mul(a.c1, a.c1)));
    uint64_t ni = or_inv(n);
    return or_ef_make(or_mul(a.c0, ni), or_mul(or_neg(a.c1), ni));
}
static inline or_ef or_ef_pow(or_ef b, uint64_t e) {
    or_ef r = or_ef_from(1);
    while (e) {
        if (e & 1) r = or_ef_mul(r, b);
        b = or_ef_mul(b, b);
        e >>= 1;
    }
    return r;
}
static inline or_ef or_ef_exp2(or_ef a, unsigned k) {
    while (k--) a = or_ef_mul(a, a);
    return a;
}

static inline size_t or_bitrev(size_t i, unsigned bits) {
    size_t r = 0;
    for (unsigned b = 0; b < bits; b++) r |= ((i >> b) & 1) << (bits - 1 - b);
    return r;
}
static inline unsigned or_log2(size_t n) {
    unsigned l = 0;
    while (((size_t)1 << l) < n) l++;
    return l;
}

#endif
