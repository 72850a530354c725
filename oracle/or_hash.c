/*
 * ORACLE (test infrastructure only): seeded RNG, the Poseidon2 permutation
 * over Goldilocks with width 12, the stateful sponge, the 2-to-1 truncated
 * compression and the duplex Fiat-Shamir challenger.
 *
 * Parity status: the permutation's round constants are generated by
 * restating the published algorithms the reference's configuration uses;
 * its internal diagonal is a placeholder loaded by value (see
 * or_p2_default_params), so hash outputs are "parity unpinned" against
 * p3-goldilocks 0.5.0 until real constants are supplied.
 */
#include <string.h>
#include <stdlib.h>
#include "oracle.h"

/* ---------------------------------------------------------------- RNG ---
 * rand 0.10 SmallRng = xoshiro256++ (Blackman & Vigna), seeded from a u64
 * through SplitMix64, as in p3-miden-dev-utils/src/configs.rs:215-218
 * (SmallRng::seed_from_u64(TEST_SEED)) and
 * p3-miden-lifted-examples/src/bin/lifted_keccak.rs:167.
 */
void or_rng_seed(or_rng *r, uint64_t seed) {
    const uint64_t PHI = 0x9e3779b97f4a7c15ULL;
    for (int i = 0; i < 4; i++) {
        seed += PHI;
        uint64_t z = seed;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        r->s[i] = z ^ (z >> 31);
    }
}
static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
uint64_t or_rng_next(or_rng *r) {
    uint64_t *s = r->s;
    uint64_t res = rotl64(s[0] + s[3], 23) + s[0];
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return res;
}
/* Uniform field element: rejection of u64 draws >= p. */
uint64_t or_rng_field(or_rng *r) {
    for (;;) {
        uint64_t x = or_rng_next(r);
        if (x < OR_P) return x;
    }
}

/* ---------------------------------------------------------- Poseidon2 ---
 * Poseidon2 (Grassi, Khovratovich, Schofnegger; eprint 2023/323) over
 * Goldilocks, t = 12, S-box x^7, R_F = 8 (4 + 4), R_P = 22.
 * External layer M_E = circ(2*M4, M4, M4) with M4 = circ(2,3,1,1);
 * internal layer M_I = 1*1^T + diag(mu).
 * Round constants: Poseidon2Goldilocks<12>::new_from_rng_128 draws, in order,
 * 4 initial external rounds x 12, 4 terminal external rounds x 12, then 22
 * internal constants, each a uniform field element.
 */
void or_p2_params_from_seed(or_p2_params *pp, uint64_t seed, const uint64_t diag[12]) {
    or_rng r;
    or_rng_seed(&r, seed);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 12; j++) pp->rc_init[i][j] = or_rng_field(&r);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 12; j++) pp->rc_term[i][j] = or_rng_field(&r);
    for (int i = 0; i < 22; i++) pp->rc_int[i] = or_rng_field(&r);
    for (int j = 0; j < 12; j++) pp->diag[j] = diag[j];
}

static void m4(uint64_t *x) {
    uint64_t a = x[0], b = x[1], c = x[2], d = x[3];
    uint64_t two_a = or_add(a, a), two_b = or_add(b, b), two_c = or_add(c, c), two_d = or_add(d, d);
    uint64_t three_a = or_add(two_a, a), three_b = or_add(two_b, b), three_c = or_add(two_c, c), three_d = or_add(two_d, d);
    x[0] = or_add(or_add(two_a, three_b), or_add(c, d));
    x[1] = or_add(or_add(a, two_b), or_add(three_c, d));
    x[2] = or_add(or_add(a, b), or_add(two_c, three_d));
    x[3] = or_add(or_add(three_a, b), or_add(c, two_d));
}
static void ext_linear(uint64_t *s) {
    for (int c = 0; c < 12; c += 4) m4(s + c);
    uint64_t sums[4];
    for (int k = 0; k < 4; k++) sums[k] = or_add(or_add(s[k], s[k + 4]), s[k + 8]);
    for (int i = 0; i < 12; i++) s[i] = or_add(s[i], sums[i & 3]);
}
static inline uint64_t sbox7(uint64_t x) {
    uint64_t x2 = or_mul(x, x), x4 = or_mul(x2, x2), x3 = or_mul(x2, x);
    return or_mul(x4, x3);
}
void or_p2_permute(const or_p2_params *pp, uint64_t *s) {
    ext_linear(s);
    for (int r = 0; r < 4; r++) {
        for (int i = 0; i < 12; i++) s[i] = sbox7(or_add(s[i], pp->rc_init[r][i]));
        ext_linear(s);
    }
    for (int r = 0; r < 22; r++) {
        s[0] = sbox7(or_add(s[0], pp->rc_int[r]));
        uint64_t sum = 0;
        for (int i = 0; i < 12; i++) sum = or_add(sum, s[i]);
        for (int i = 0; i < 12; i++) s[i] = or_add(or_mul(s[i], pp->diag[i]), sum);
    }
    for (int r = 0; r < 4; r++) {
        for (int i = 0; i < 12; i++) s[i] = sbox7(or_add(s[i], pp->rc_term[r][i]));
        ext_linear(s);
    }
}

/* ------------------------------------------------------------- sponge ---
 * StatefulSponge<Perm, 12, 8, 4>::absorb_into
 * (p3-miden-stateful-hasher/src/field_sponge.rs:164-182): overwrite the rate
 * with the next 8 inputs and permute; a partial final chunk is zero-filled up
 * to the rate and permuted; an empty input (or one that ends on a rate
 * boundary) adds no permutation. Squeeze = state[0..4] (:184-187).
 */
void or_sponge_absorb(const or_p2_params *pp, uint64_t *st, const uint64_t *in, size_t n) {
    size_t i = 0;
    while (i < n) {
        size_t take = n - i < 8 ? n - i : 8;
        for (size_t j = 0; j < take; j++) st[j] = in[i + j];
        for (size_t j = take; j < 8; j++) st[j] = 0;
        or_p2_permute(pp, st);
        i += take;
    }
}
/* TruncatedPermutation<Perm, 2, 4, 12> (p3-miden-dev-utils/src/configs.rs:202):
 * permute [left || right || 0^4] and keep the first 4 words. */
void or_compress(const or_p2_params *pp, const uint64_t *l, const uint64_t *r, uint64_t *out) {
    uint64_t s[12] = {0};
    memcpy(s, l, 32);
    memcpy(s + 4, r, 32);
    or_p2_permute(pp, s);
    memcpy(out, s, 32);
}

/* --------------------------------------------------------- challenger ---
 * DuplexChallenger<F, Perm, 12, 8> (p3-challenger 0.5.0) as driven by
 * ProverTranscript (p3-miden-transcript/src/prover.rs:97-145):
 *  observe: clear outputs, buffer the input, duplex when 8 are buffered;
 *  sample: duplex if inputs are pending or outputs are exhausted, then pop
 *          the LAST output word;
 *  duplex: overwrite state[0..k] with the k pending inputs, permute,
 *          outputs = state[0..8];
 *  sample_bits(b) = canonical(sample()) & (2^b - 1);
 *  grind(b): smallest witness w (scanning 0,1,2,...) such that observing w
 *          then sample_bits(b) gives 0; the real challenger then performs that
 *          observe + sample. b = 0 returns w = 0 and leaves the state alone;
 *  finalize: one more duplex, digest = the full 12-word state.
 */
void or_ch_init(or_challenger *c, const or_p2_params *pp) {
    memset(c, 0, sizeof(*c));
    c->pp = pp;
}
static void ch_duplex(or_challenger *c) {
    for (int i = 0; i < c->n_in; i++) c->state[i] = c->in[i];
    c->n_in = 0;
    or_p2_permute(c->pp, c->state);
    for (int i = 0; i < 8; i++) c->out[i] = c->state[i];
    c->n_out = 8;
}
void or_ch_observe(or_challenger *c, uint64_t x) {
    c->n_out = 0;
    c->in[c->n_in++] = x;
    if (c->n_in == 8) ch_duplex(c);
}
uint64_t or_ch_sample(or_challenger *c) {
    if (c->n_in > 0 || c->n_out == 0) ch_duplex(c);
    return c->out[--c->n_out];
}
uint64_t or_ch_sample_bits(or_challenger *c, unsigned bits) {
    uint64_t v = or_ch_sample(c);
    return bits >= 64 ? v : (v & ((1ULL << bits) - 1));
}
or_ef or_ch_sample_ef(or_challenger *c) {
    uint64_t a = or_ch_sample(c);
    uint64_t b = or_ch_sample(c);
    return or_ef_make(a, b);
}
uint64_t or_ch_grind(or_challenger *c, unsigned bits) {
    if (bits == 0) return 0;
    for (uint64_t w = 0;; w++) {
        or_challenger t = *c;
        or_ch_observe(&t, w);
        if (or_ch_sample_bits(&t, bits) == 0) {
            or_ch_observe(c, w);
            (void)or_ch_sample_bits(c, bits);
            return w;
        }
    }
}
void or_ch_finalize(or_challenger *c, uint64_t digest[12]) {
    ch_duplex(c);
    memcpy(digest, c->state, 96);
}

/* ------------------------------------------------------------ transcript
 * ProverTranscript (p3-miden-transcript/src/prover.rs:122-145): send_* records
 * and observes, hint_* records only, grind records the witness.
 */
void or_tr_init(or_transcript *t, const or_p2_params *pp) {
    memset(t, 0, sizeof(*t));
    or_ch_init(&t->ch, pp);
}
static void push_field(or_transcript *t, uint64_t v) {
    if (t->n_fields == t->cap_fields) {
        t->cap_fields = t->cap_fields ? 2 * t->cap_fields : 1024;
        t->fields = (uint64_t *)realloc(t->fields, t->cap_fields * 8);
    }
    t->fields[t->n_fields++] = v;
}
static void push_commit(or_transcript *t, const uint64_t *d) {
    if (t->n_commits == t->cap_commits) {
        t->cap_commits = t->cap_commits ? 2 * t->cap_commits : 256;
        t->commits = (uint64_t *)realloc(t->commits, t->cap_commits * 32);
    }
    memcpy(t->commits + 4 * t->n_commits, d, 32);
    t->n_commits++;
}
void or_tr_send_field(or_transcript *t, uint64_t v) {
    push_field(t, v);
    or_ch_observe(&t->ch, v);
}
void or_tr_send_ef(or_transcript *t, or_ef v) {
    or_tr_send_field(t, v.c0);
    or_tr_send_field(t, v.c1);
}
void or_tr_send_commit(or_transcript *t, const uint64_t *d) {
    push_commit(t, d);
    for (int i = 0; i < 4; i++) or_ch_observe(&t->ch, d[i]);
}
void or_tr_hint_field(or_transcript *t, uint64_t v) { push_field(t, v); }
void or_tr_hint_commit(or_transcript *t, const uint64_t *d) { push_commit(t, d); }
uint64_t or_tr_grind(or_transcript *t, unsigned bits) {
    uint64_t w = or_ch_grind(&t->ch, bits);
    push_field(t, w);
    return w;
}
void or_tr_free(or_transcript *t) {
    free(t->fields);
    free(t->commits);
    memset(t, 0, sizeof(*t));
}
