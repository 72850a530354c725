/*
 * ORACLE (test infrastructure only): two-adic DFTs, the bit-reversed coset
 * LDE and the lifted Merkle tree (LMCS) with its batch-opening hints.
 */
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

/* ------------------------------------------------------------------ DFT
 * Values, not algorithms, are what the reference fixes: the DFT of size n
 * maps coefficients a_k to evaluations sum_k a_k w_n^{ik} at the natural
 * points w_n^i, with w_n = 7^((p-1)/n). Here: iterative radix-2 DIT. */
static void bitrev_permute(uint64_t *a, size_t n) {
    unsigned L = or_log2(n);
    for (size_t i = 0; i < n; i++) {
        size_t j = or_bitrev(i, L);
        if (i < j) {
            uint64_t t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
}
static void ntt_with_root(uint64_t *a, size_t n, uint64_t root_n) {
    if (n <= 1) return;
    bitrev_permute(a, n);
    unsigned L = or_log2(n);
    for (unsigned s = 1; s <= L; s++) {
        size_t m = (size_t)1 << s, half = m >> 1;
        uint64_t wm = or_exp2(root_n, L - s); /* primitive m-th root */
        uint64_t *tw = (uint64_t *)malloc(half * 8);
        tw[0] = 1;
        for (size_t j = 1; j < half; j++) tw[j] = or_mul(tw[j - 1], wm);
        for (size_t k = 0; k < n; k += m)
            for (size_t j = 0; j < half; j++) {
                uint64_t u = a[k + j], v = or_mul(a[k + j + half], tw[j]);
                a[k + j] = or_add(u, v);
                a[k + j + half] = or_sub(u, v);
            }
        free(tw);
    }
}
void or_ntt(uint64_t *a, size_t n) { ntt_with_root(a, n, or_root(or_log2(n))); }
void or_intt(uint64_t *a, size_t n) {
    unsigned L = or_log2(n);
    ntt_with_root(a, n, or_inv(or_root(L)));
    uint64_t ninv = or_inv((uint64_t)n % OR_P);
    for (size_t i = 0; i < n; i++) a[i] = or_mul(a[i], ninv);
}

/* Radix2DitParallel::coset_lde_batch(trace, log_blowup, shift) followed by
 * bit_reverse_rows (p3-miden-lifted-stark/src/prover/commit.rs:217-222):
 * row bitrev(i) of the output holds the evaluation at shift * w_{hB}^i. */
void or_coset_lde_bitrev(const uint64_t *in, size_t h, size_t w, unsigned log_blowup, uint64_t shift,
                         uint64_t *out) {
    size_t n = h << log_blowup;
    unsigned L = or_log2(n);
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t c = 0; c < w; c++) {
        uint64_t *col = (uint64_t *)calloc(n, 8);
        for (size_t r = 0; r < h; r++) col[r] = in[r * w + c];
        or_intt(col, h);
        uint64_t s = 1;
        for (size_t k = 0; k < h; k++) {
            col[k] = or_mul(col[k], s);
            s = or_mul(s, shift);
        }
        or_ntt(col, n);
        for (size_t i = 0; i < n; i++) out[or_bitrev(i, L) * w + c] = col[i];
        free(col);
    }
}

/* ----------------------------------------------------------------- LMCS
 * LiftedMerkleTree::build_with_alignment (p3-miden-lmcs/src/lifted_tree.rs:244-310):
 * one zeroed sponge state per leaf of the tallest matrix; matrices are
 * absorbed in (ascending-height) order, each row with its own absorb call;
 * when the height grows, each state is duplicated into a contiguous block
 * (nearest-neighbour upsampling, :385-437); squeeze; then compress pairs
 * layer by layer (:494-539). The alignment only affects hints. */
static void tree_build(const or_p2_params *pp, or_tree *t, const or_matrix *mats, size_t n, size_t alignment,
                       const uint64_t *salt, size_t salt_width) {
    memset(t, 0, sizeof(*t));
    t->salt = salt;
    t->salt_width = salt ? salt_width : 0;
    t->n_mats = n;
    for (size_t i = 0; i < n; i++) t->mats[i] = mats[i];
    t->alignment = alignment ? alignment : 1;
    size_t H = mats[n - 1].height;
    t->depth = or_log2(H);
    uint64_t *states = (uint64_t *)calloc(H * 12, 8);
    size_t active = mats[0].height;
    for (size_t m = 0; m < n; m++) {
        size_t h = mats[m].height;
        if (h > active) {
            size_t f = h / active;
            for (size_t i = active; i-- > 0;)
                for (size_t k = f; k-- > 0;)
                    memcpy(states + (i * f + k) * 12, states + i * 12, 96);
        }
        const uint64_t *d = mats[m].data;
        size_t w = mats[m].width;
#pragma omp parallel for schedule(static)
        for (size_t r = 0; r < h; r++) or_sponge_absorb(pp, states + r * 12, d + r * w, w);
        active = h;
    }
    /* hiding: the salt row, one more absorb call per leaf
     * (p3-miden-lmcs/src/lifted_tree.rs:271-279) */
    if (t->salt_width) {
#pragma omp parallel for schedule(static)
        for (size_t r = 0; r < H; r++) or_sponge_absorb(pp, states + r * 12, salt + r * salt_width, salt_width);
    }
    size_t total = 2 * H - 1;
    t->layers = (uint64_t *)malloc(total * 32);
    for (size_t i = 0; i < H; i++) memcpy(t->layers + 4 * i, states + 12 * i, 32);
    free(states);
    size_t off = 0, len = H;
    t->layer_off[0] = 0;
    for (unsigned l = 1; l <= t->depth; l++) {
        size_t noff = off + len, nlen = len / 2;
        const uint64_t *prev = t->layers + 4 * off;
        uint64_t *next = t->layers + 4 * noff;
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < nlen; i++) or_compress(pp, prev + 8 * i, prev + 8 * i + 4, next + 4 * i);
        t->layer_off[l] = noff;
        off = noff;
        len = nlen;
    }
}
void or_tree_build(const or_p2_params *pp, or_tree *t, const or_matrix *mats, size_t n, size_t alignment) {
    tree_build(pp, t, mats, n, alignment, NULL, 0);
}
/* HidingLmcsConfig::build_tree / build_aligned_tree (hiding_lmcs.rs:112-145)
 * with the caller's salt matrix in place of the config's RNG draw */
void or_tree_build_hiding(const or_p2_params *pp, or_tree *t, const or_matrix *mats, size_t n, size_t alignment,
                          const uint64_t *salt, size_t salt_width) {
    tree_build(pp, t, mats, n, alignment, salt, salt_width);
}
void or_tree_root(const or_tree *t, uint64_t out[4]) { memcpy(out, t->layers + 4 * t->layer_off[t->depth], 32); }
void or_tree_free(or_tree *t) {
    free(t->layers);
    t->layers = NULL;
}

/* LmcsTree::prove_batch (p3-miden-lmcs/src/lifted_tree.rs:157-224): for each
 * unique index in ascending order, one row per matrix (row index >> the
 * matrix's lift), zero-padded to the alignment; then, level by level from
 * the leaves, the sibling digest of every pair with exactly one known child,
 * left to right. Hints are recorded, not observed. */
void or_tree_prove_batch(const or_tree *t, const size_t *idx, size_t n_idx, or_transcript *tr) {
    size_t H = (size_t)1 << t->depth;
    for (size_t q = 0; q < n_idx; q++) {
        for (size_t m = 0; m < t->n_mats; m++) {
            const or_matrix *M = &t->mats[m];
            unsigned lift = t->depth - or_log2(M->height);
            size_t row = idx[q] >> lift;
            size_t w = M->width, aw = (w + t->alignment - 1) / t->alignment * t->alignment;
            for (size_t c = 0; c < aw; c++) or_tr_hint_field(tr, c < w ? M->data[row * w + c] : 0);
        }
        /* hiding: the leaf's salt, unpadded (lifted_tree.rs:189-192) */
        for (size_t c = 0; c < t->salt_width; c++) or_tr_hint_field(tr, t->salt[idx[q] * t->salt_width + c]);
    }
    (void)H;
    size_t *known = (size_t *)malloc((n_idx + 1) * sizeof(size_t));
    size_t nk = n_idx;
    memcpy(known, idx, n_idx * sizeof(size_t));
    for (unsigned l = 0; l < t->depth; l++) {
        size_t np = 0;
        for (size_t i = 0; i < nk; i++) {
            size_t pos = known[i], parent = pos >> 1;
            if (np > 0 && known[np - 1] == parent) continue; /* pair handled */
            int have_left = 0, have_right = 0;
            size_t left = parent * 2, right = left + 1;
            /* known is sorted: look at neighbours */
            if (pos == left) {
                have_left = 1;
                have_right = (i + 1 < nk && known[i + 1] == right);
            } else {
                have_right = 1;
            }
            const uint64_t *layer = t->layers + 4 * t->layer_off[l];
            if (have_left && !have_right) or_tr_hint_commit(tr, layer + 4 * right);
            else if (!have_left && have_right) or_tr_hint_commit(tr, layer + 4 * left);
            known[np++] = parent; /* safe: np <= i */
        }
        nk = np;
    }
    free(known);
}

/* PeriodicLde::build (p3-miden-lifted-stark/src/prover/periodic.rs:49-81):
 * NaiveDft::coset_lde_batch of the columns repeated to the largest period p
 * (p x w, row-major) on the coset of period_shift = lde_shift^(2^(log_h -
 * log p)) (periodic.rs:66-71), natural order, (p << log_blowup) x w. Restated
 * from the defining sums, O(p * pB) per column: interpolate on the subgroup
 * of order p, then evaluate at period_shift * w_{pB}^i. */
void or_periodic_lde(const uint64_t *repeated, size_t p, size_t w, unsigned log_blowup, unsigned log_trace_height,
                     uint64_t lde_shift, uint64_t *out) {
    unsigned lp = or_log2(p);
    size_t n = p << log_blowup;
    uint64_t ps = or_exp2(lde_shift % OR_P, log_trace_height - lp);
    uint64_t wp_inv = or_inv(or_root(lp)), wn = or_root(lp + log_blowup), pinv = or_inv((uint64_t)p % OR_P);
    uint64_t *coef = (uint64_t *)malloc(p * 8);
    for (size_t c = 0; c < w; c++) {
        for (size_t k = 0; k < p; k++) { /* a_k = (1/p) sum_j v_j w_p^{-jk} */
            uint64_t s = 0;
            for (size_t j = 0; j < p; j++) s = or_add(s, or_mul(repeated[j * w + c], or_pow(wp_inv, (j * k) % p)));
            coef[k] = or_mul(s, pinv);
        }
        for (size_t i = 0; i < n; i++) { /* f(ps * w_n^i) by Horner */
            uint64_t x = or_mul(ps, or_pow(wn, i)), acc = 0;
            for (size_t k = p; k-- > 0;) acc = or_add(or_mul(acc, x), coef[k]);
            out[i * w + c] = acc;
        }
    }
    free(coef);
}
