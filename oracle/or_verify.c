/*
 * ORACLE (test infrastructure only): a CPU restatement of the lifted-STARK
 * verifier, the acceptance check for proofs made by the CUDA product (and by
 * the oracle prover). It replays the transcript, verifies every LMCS opening,
 * the DEEP and FRI query checks, the final polynomial and the quotient
 * identity at the out-of-domain point, and the transcript digest.
 *
 * Restated from:
 *   verify_multi            p3-miden-lifted-stark/src/verifier/mod.rs:170-364
 *   ConstraintFolder,       p3-miden-lifted-stark/src/verifier/constraints.rs
 *   reconstruct_quotient
 *   selectors_at,           p3-miden-lifted-stark/src/coset.rs (selectors_at,
 *   vanishing_at                vanishing_at, lde_shift)
 *   verify / verify_aligned p3-miden-lifted-fri/src/verifier.rs
 *   DeepOracle              p3-miden-lifted-fri/src/deep/verifier.rs
 *   FriOracle               p3-miden-lifted-fri/src/fri/verifier.rs
 *   LMCS open_batch         p3-miden-lmcs/src/lmcs.rs:167-290
 *   VerifierTranscript      p3-miden-transcript/src/verifier.rs
 * The challenger's check_witness with bits = 0 accepts without observing,
 * the convention of or_ch_grind.
 */
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

typedef struct {
    or_challenger ch;
    const uint64_t *fields;
    size_t nf, pf;
    const uint64_t *commits;
    size_t nc, pc;
    int short_read;
} vch;

/* received (observed) and hinted (recorded only) values */
static uint64_t v_field(vch *v) {
    if (v->pf >= v->nf) {
        v->short_read = 1;
        return 0;
    }
    uint64_t x = v->fields[v->pf++];
    or_ch_observe(&v->ch, x);
    return x;
}
static or_ef v_ef(vch *v) {
    uint64_t a = v_field(v);
    uint64_t b = v_field(v);
    return or_ef_make(a, b);
}
static uint64_t v_hint_field(vch *v) {
    if (v->pf >= v->nf) {
        v->short_read = 1;
        return 0;
    }
    return v->fields[v->pf++];
}
static void v_commit(vch *v, uint64_t out[4], int observe) {
    if (v->pc >= v->nc) {
        v->short_read = 1;
        memset(out, 0, 32);
        return;
    }
    memcpy(out, v->commits + 4 * v->pc++, 32);
    if (observe)
        for (int i = 0; i < 4; i++) or_ch_observe(&v->ch, out[i]);
}
static int v_grind(vch *v, unsigned bits) {
    uint64_t w = v_hint_field(v);
    if (bits == 0) return 1;
    or_ch_observe(&v->ch, w);
    return or_ch_sample_bits(&v->ch, bits) == 0;
}

static int cmp_size(const void *a, const void *b) {
    size_t x = *(const size_t *)a, y = *(const size_t *)b;
    return x < y ? -1 : x > y;
}
static size_t sort_unique(size_t *v, size_t n) {
    qsort(v, n, sizeof(size_t), cmp_size);
    size_t u = 0;
    for (size_t i = 0; i < n; i++)
        if (u == 0 || v[u - 1] != v[i]) v[u++] = v[i];
    return u;
}

/* LMCS open_batch: for each sorted unique index read the concatenated rows
 * (widths[]), hash them (one absorb per matrix row), then rebuild the root
 * from the known nodes and the hinted siblings, bottom-up and left to right.
 * rows_out: n_idx x sum(widths). Returns 0 or an OR_VERR code. */
static int lmcs_open_batch(const or_p2_params *pp, vch *v, const uint64_t commit[4], const size_t *widths,
                           size_t n_w, unsigned log_h, const size_t *idx, size_t n_idx, uint64_t *rows_out) {
    size_t tw = 0;
    for (size_t m = 0; m < n_w; m++) tw += widths[m];
    size_t *pos = (size_t *)malloc(n_idx * sizeof(size_t));
    uint64_t *hash = (uint64_t *)malloc(n_idx * 32);
    for (size_t q = 0; q < n_idx; q++) {
        if (idx[q] >> log_h) {
            free(pos);
            free(hash);
            return OR_VERR_OPENING;
        }
        uint64_t *row = rows_out + q * tw;
        for (size_t c = 0; c < tw; c++) row[c] = v_hint_field(v);
        uint64_t st[12] = {0};
        size_t off = 0;
        for (size_t m = 0; m < n_w; m++) {
            or_sponge_absorb(pp, st, row + off, widths[m]);
            off += widths[m];
        }
        pos[q] = idx[q];
        memcpy(hash + 4 * q, st, 32);
    }
    size_t n = n_idx;
    for (unsigned l = 0; l < log_h; l++) {
        size_t np = 0;
        for (size_t i = 0; i < n;) {
            const size_t p = pos[i];
            uint64_t mine[4], sib[4], left[4], right[4];
            memcpy(mine, hash + 4 * i, 32);
            if (i + 1 < n && pos[i + 1] == (p ^ 1)) { /* both children known */
                memcpy(sib, hash + 4 * (i + 1), 32);
                i += 2;
            } else { /* sibling streamed from the proof */
                v_commit(v, sib, 0);
                i += 1;
            }
            if (p & 1) {
                memcpy(left, sib, 32);
                memcpy(right, mine, 32);
            } else {
                memcpy(left, mine, 32);
                memcpy(right, sib, 32);
            }
            or_compress(pp, left, right, hash + 4 * np); /* np < i: entries already read */
            pos[np++] = p >> 1;
        }
        n = np;
    }
    int ok = n == 1 && pos[0] == 0 && memcmp(hash, commit, 32) == 0;
    free(pos);
    free(hash);
    return ok ? 0 : OR_VERR_ROOT;
}

static or_ef horner_acc(or_ef acc, or_ef x, const uint64_t *vals, size_t n) {
    for (size_t i = 0; i < n; i++) acc = or_ef_add(or_ef_mul(acc, x), or_ef_from(vals[i]));
    return acc;
}

/* arity-a fold of one row of bit-reversed coset evaluations
 * (fri/fold/arity{2,4,8}.rs): (1/a) sum_j (beta * s_inv)^j sum_k y_k w_a^{-jk} */
static or_ef fold_evals(const or_ef *ev, unsigned log_a, uint64_t s_inv, or_ef beta) {
    size_t a = (size_t)1 << log_a;
    uint64_t winv = or_inv(or_root(log_a));
    or_ef x = or_ef_mulf(beta, s_inv), xp = or_ef_from(1), res = or_ef_from(0);
    for (size_t j = 0; j < a; j++) {
        or_ef u = or_ef_from(0);
        for (size_t k = 0; k < a; k++) u = or_ef_add(u, or_ef_mulf(ev[or_bitrev(k, log_a)], or_pow(winv, (j * k) % a)));
        res = or_ef_add(res, or_ef_mul(u, xp));
        xp = or_ef_mul(xp, x);
    }
    return or_ef_mulf(res, or_inv((uint64_t)a));
}

int or_verify(const or_p2_params *pp, const or_pcs_params *pcs, const or_instance *inst, size_t n_inst,
              const uint64_t *fields, size_t n_fields, const uint64_t *commits, size_t n_commits,
              const uint64_t digest[12]) {
    if (n_inst == 0 || n_inst > 8) return OR_VERR_SHAPE;
    for (size_t i = 0; i < n_inst; i++)
        if (inst[i].height == 0 || (inst[i].height & (inst[i].height - 1)) ||
            (i && inst[i].height < inst[i - 1].height))
            return OR_VERR_SHAPE;
    vch v;
    memset(&v, 0, sizeof(v));
    or_ch_init(&v.ch, pp);
    v.fields = fields, v.nf = n_fields, v.commits = commits, v.nc = n_commits;
    int err = 0;
    const unsigned lb = pcs->log_blowup;
    const unsigned log_max_h = or_log2(inst[n_inst - 1].height);
    unsigned log_qd = 0;
    size_t n_rand = 0;
    for (size_t i = 0; i < n_inst; i++) {
        if (inst[i].air == OR_AIR_SYMBOLIC && (!inst[i].sym || or_sym_validate(inst[i].sym))) return OR_VERR_SHAPE;
        unsigned d = or_inst_log_qd(&inst[i]);
        if (d > log_qd) log_qd = d;
        if (or_inst_num_randomness(&inst[i]) > n_rand) n_rand = or_inst_num_randomness(&inst[i]);
    }
    if (log_qd > lb) return OR_VERR_SHAPE;
    const size_t D = (size_t)1 << log_qd;
    const unsigned log_lde = log_max_h + lb;

    /* 1.-5. commitments and challenges in prover order */
    uint64_t main_c[4], aux_c[4], quot_c[4];
    v_commit(&v, main_c, 1);
    or_ef rnd[64];
    for (size_t r = 0; r < n_rand && r < 64; r++) rnd[r] = or_ch_sample_ef(&v.ch); /* aux randomness */
    v_commit(&v, aux_c, 1);
    /* aux values per instance (verifier/mod.rs:230-239) */
    size_t n_auxv = 0;
    for (size_t i = 0; i < n_inst; i++) n_auxv += or_inst_num_aux_values(&inst[i]);
    or_ef *auxv = (or_ef *)malloc((n_auxv + 1) * sizeof(or_ef));
    for (size_t k = 0; k < n_auxv; k++) auxv[k] = v_ef(&v);
    or_ef alpha = or_ch_sample_ef(&v.ch);
    or_ef beta = or_ch_sample_ef(&v.ch);
    v_commit(&v, quot_c, 1);
    /* 6. OOD point outside H and gK */
    or_ef z;
    for (;;) {
        z = or_ch_sample_ef(&v.ch);
        int in_h = or_ef_eq(or_ef_exp2(z, log_max_h), or_ef_from(1));
        int in_gk = or_ef_eq(or_ef_exp2(or_ef_mulf(z, or_inv(OR_GEN)), log_lde), or_ef_from(1));
        if (!in_h && !in_gk) break;
    }
    const or_ef zs[2] = {z, or_ef_mulf(z, or_root(log_max_h))};

    /* 7. groups: main (one matrix per instance), aux (2 columns each),
     * quotient (2D columns); LMCS alignment 8 */
    size_t n_mats = 2 * n_inst + 1, aw[17], ow[17], grp_first[4] = {0, n_inst, 2 * n_inst, 2 * n_inst + 1};
    for (size_t i = 0; i < n_inst; i++) {
        ow[i] = inst[i].width;
        ow[n_inst + i] = 2 * or_inst_aux_width(&inst[i]);
    }
    ow[2 * n_inst] = 2 * D;
    size_t total_aligned = 0;
    for (size_t m = 0; m < n_mats; m++) {
        aw[m] = (ow[m] + 7) / 8 * 8;
        total_aligned += aw[m];
    }
    const uint64_t *gcommit[3] = {main_c, aux_c, quot_c};

    /* 8a. DEEP oracle: the aligned OOD evaluations per point, grind, alpha_c, beta_p */
    or_ef *evals = (or_ef *)malloc(2 * total_aligned * sizeof(or_ef)); /* [point][col] */
    for (int p = 0; p < 2; p++)
        for (size_t c = 0; c < total_aligned; c++) evals[p * total_aligned + c] = v_ef(&v);
    if (!v_grind(&v, pcs->deep_pow_bits)) err = OR_VERR_POW;
    or_ef ac = or_ch_sample_ef(&v.ch);
    or_ef bp = or_ch_sample_ef(&v.ch);
    or_ef red_open[2];
    for (int p = 0; p < 2; p++) {
        or_ef acc = or_ef_from(0);
        for (size_t c = 0; c < total_aligned; c++) acc = or_ef_add(or_ef_mul(acc, ac), evals[p * total_aligned + c]);
        red_open[p] = acc;
    }
    /* 8b. FRI oracle: round commitments, grinds, betas, final polynomial */
    const unsigned log_a = pcs->log_folding_arity;
    const size_t arity = (size_t)1 << log_a;
    const unsigned log_max_final = pcs->log_final_degree + lb;
    const size_t rounds = log_lde > log_max_final ? (log_lde - log_max_final + log_a - 1) / log_a : 0;
    const unsigned log_final_size = log_lde - (unsigned)rounds * log_a;
    const size_t final_deg = (size_t)1 << (log_final_size > lb ? log_final_size - lb : 0);
    uint64_t(*fri_c)[4] = (uint64_t(*)[4])malloc((rounds + 1) * 32);
    or_ef *fri_beta = (or_ef *)malloc((rounds + 1) * sizeof(or_ef));
    for (size_t r = 0; r < rounds; r++) {
        v_commit(&v, fri_c[r], 1);
        if (!v_grind(&v, pcs->folding_pow_bits) && !err) err = OR_VERR_POW;
        fri_beta[r] = or_ch_sample_ef(&v.ch);
    }
    or_ef *final_poly = (or_ef *)malloc(final_deg * sizeof(or_ef));
    for (size_t i = 0; i < final_deg; i++) final_poly[i] = v_ef(&v);
    /* 8c. query pow, indices */
    if (!v_grind(&v, pcs->query_pow_bits) && !err) err = OR_VERR_POW;
    size_t *idx = (size_t *)malloc((pcs->num_queries + 1) * sizeof(size_t));
    for (unsigned q = 0; q < pcs->num_queries; q++) idx[q] = or_bitrev(or_ch_sample_bits(&v.ch, log_lde), log_lde);
    const size_t nq = sort_unique(idx, pcs->num_queries);
    /* 8d. DEEP open_batch: openings of the three trace trees, reduced rows */
    or_ef *red_row = (or_ef *)calloc(nq ? nq : 1, sizeof(or_ef));
    for (int g = 0; g < 3 && !err; g++) {
        size_t m0 = grp_first[g], m1 = grp_first[g + 1], tw = 0;
        for (size_t m = m0; m < m1; m++) tw += aw[m];
        uint64_t *rows = (uint64_t *)malloc((nq ? nq : 1) * tw * 8);
        err = lmcs_open_batch(pp, &v, gcommit[g], aw + m0, m1 - m0, log_lde, idx, nq, rows);
        for (size_t q = 0; q < nq && !err; q++) red_row[q] = horner_acc(red_row[q], ac, rows + q * tw, tw);
        free(rows);
    }
    or_ef *cur = (or_ef *)malloc((nq ? nq : 1) * sizeof(or_ef));
    size_t *cur_idx = (size_t *)malloc((nq ? nq : 1) * sizeof(size_t));
    size_t ncur = nq;
    if (!err) {
        const uint64_t gen = or_root(log_lde);
        for (size_t q = 0; q < nq && !err; q++) {
            uint64_t x = or_mul(OR_GEN, or_pow(gen, or_bitrev(idx[q], log_lde)));
            or_ef de = or_ef_from(0), bpow = or_ef_from(1);
            for (int p = 0; p < 2; p++) {
                or_ef den = or_ef_sub(zs[p], or_ef_from(x));
                if (den.c0 == 0 && den.c1 == 0) {
                    err = OR_VERR_DEEP;
                    break;
                }
                de = or_ef_add(de, or_ef_mul(bpow, or_ef_mul(or_ef_sub(red_open[p], red_row[q]), or_ef_inv(den))));
                bpow = or_ef_mul(bpow, bp);
            }
            cur[q] = de;
            cur_idx[q] = idx[q];
        }
    }
    /* 8e. FRI low-degree test */
    unsigned log_dom = log_lde;
    uint64_t g_inv = or_inv(or_root(log_lde));
    for (size_t r = 0; r < rounds && !err; r++) {
        const unsigned log_folded = log_dom - log_a;
        size_t *ridx = (size_t *)malloc((ncur ? ncur : 1) * sizeof(size_t));
        for (size_t q = 0; q < ncur; q++) ridx[q] = cur_idx[q] >> log_a;
        size_t nr = sort_unique(ridx, ncur);
        size_t w = 2 * arity;
        uint64_t *rows = (uint64_t *)malloc((nr ? nr : 1) * w * 8);
        err = lmcs_open_batch(pp, &v, fri_c[r], &w, 1, log_folded, ridx, nr, rows);
        or_ef *next = (or_ef *)malloc((nr ? nr : 1) * sizeof(or_ef));
        or_ef *rowv = (or_ef *)malloc(arity * sizeof(or_ef));
        for (size_t k = 0; k < nr && !err; k++) {
            for (size_t j = 0; j < arity; j++) rowv[j] = or_ef_make(rows[k * w + 2 * j], rows[k * w + 2 * j + 1]);
            /* every query falling in this row must match its position */
            for (size_t q = 0; q < ncur; q++)
                if ((cur_idx[q] >> log_a) == ridx[k] && !or_ef_eq(rowv[cur_idx[q] & (arity - 1)], cur[q]))
                    err = OR_VERR_FRI;
            uint64_t s_inv = or_pow(g_inv, or_bitrev(ridx[k], log_folded));
            next[k] = fold_evals(rowv, log_a, s_inv, fri_beta[r]);
        }
        free(rowv);
        free(rows);
        memcpy(cur, next, nr * sizeof(or_ef));
        memcpy(cur_idx, ridx, nr * sizeof(size_t));
        ncur = nr;
        free(next);
        free(ridx);
        log_dom = log_folded;
        g_inv = or_exp2(g_inv, log_a);
    }
    if (!err) {
        const uint64_t gen = or_root(log_dom);
        for (size_t q = 0; q < ncur && !err; q++) {
            uint64_t x = or_pow(gen, or_bitrev(cur_idx[q], log_dom));
            or_ef e = or_ef_from(0);
            for (size_t i = 0; i < final_deg; i++) e = or_ef_add(or_ef_mulf(e, x), final_poly[i]);
            if (!or_ef_eq(e, cur[q])) err = OR_VERR_FINAL;
        }
    }
    free(cur);
    free(cur_idx);
    free(red_row);
    free(idx);
    free(final_poly);
    free(fri_beta);
    free(fri_c);

    /* 10. constraints at z (local) and z * w (next) per instance, beta accumulation */
    or_ef accumulated = or_ef_from(0);
    if (!err) {
        size_t off = 0, aux_off = 0, auxv_off = 0;
        for (size_t m = 0; m < n_inst; m++) aux_off += aw[m];
        for (size_t i = 0; i < n_inst; i++) {
            if (inst[i].air == OR_AIR_SYMBOLIC) {
                /* ConstraintFolder over the DAG at z (verifier/mod.rs:286-339) */
                const or_sym_air *A = inst[i].sym;
                const size_t w = inst[i].width, awi = A->aux_width;
                const unsigned log_h = or_log2(inst[i].height), lift = log_max_h - log_h;
                or_ef *ml = (or_ef *)malloc((w + 1) * sizeof(or_ef)), *mn = (or_ef *)malloc((w + 1) * sizeof(or_ef));
                or_ef *al = (or_ef *)malloc((awi + 1) * sizeof(or_ef)), *an = (or_ef *)malloc((awi + 1) * sizeof(or_ef));
                or_ef *per = (or_ef *)malloc((A->num_periodic + 1) * sizeof(or_ef));
                or_ef *nodes = (or_ef *)malloc((A->n_nodes + 1) * sizeof(or_ef));
                or_ef *cons = (or_ef *)malloc((A->n_constraints + 1) * sizeof(or_ef));
                for (size_t c = 0; c < w; c++) ml[c] = evals[off + c], mn[c] = evals[total_aligned + off + c];
                /* aux EF column c = its two base coordinates (row_to_packed_ext) */
                const or_ef X = or_ef_make(0, 1);
                for (size_t c = 0; c < awi; c++) {
                    al[c] = or_ef_add(evals[aux_off + 2 * c], or_ef_mul(X, evals[aux_off + 2 * c + 1]));
                    an[c] = or_ef_add(evals[total_aligned + aux_off + 2 * c],
                                      or_ef_mul(X, evals[total_aligned + aux_off + 2 * c + 1]));
                }
                or_sym_periodic_at(A, inst[n_inst - 1].height, z, per);
                or_ef zl = or_ef_exp2(z, lift);
                or_ef van = or_ef_sub(or_ef_exp2(zl, log_h), or_ef_from(1));
                uint64_t oinv = or_inv(or_root(log_h));
                or_sym_point pt;
                pt.sel[0] = or_ef_mul(van, or_ef_inv(or_ef_sub(zl, or_ef_from(1))));
                pt.sel[1] = or_ef_mul(van, or_ef_inv(or_ef_sub(zl, or_ef_from(oinv))));
                pt.sel[2] = or_ef_sub(zl, or_ef_from(oinv));
                pt.main_local = ml, pt.main_next = mn, pt.aux_local = al, pt.aux_next = an;
                pt.pub = inst[i].public_values, pt.rand = rnd, pt.auxv = auxv + auxv_off, pt.periodic = per;
                or_sym_eval(A, &pt, nodes, cons);
                or_ef folded = or_ef_from(0);
                for (size_t k = 0; k < A->n_constraints; k++) folded = or_ef_add(or_ef_mul(folded, alpha), cons[k]);
                accumulated = or_ef_add(or_ef_mul(accumulated, beta), folded);
                free(ml), free(mn), free(al), free(an), free(per), free(nodes), free(cons);
                off += aw[i];
                aux_off += aw[n_inst + i];
                auxv_off += A->num_aux_values;
                continue;
            }
            aux_off += aw[n_inst + i];
            const size_t w = inst[i].width;
            const unsigned log_h = or_log2(inst[i].height), lift = log_max_h - log_h;
            or_ef *L = (or_ef *)malloc(w * sizeof(or_ef)), *N = (or_ef *)malloc(w * sizeof(or_ef));
            for (size_t c = 0; c < w; c++) {
                L[c] = evals[off + c];
                N[c] = evals[total_aligned + off + c];
            }
            off += aw[i];
            or_ef zl = or_ef_exp2(z, lift);
            or_ef van = or_ef_sub(or_ef_exp2(zl, log_h), or_ef_from(1));
            uint64_t oinv = or_inv(or_root(log_h));
            or_ef sel[3];
            sel[0] = or_ef_mul(van, or_ef_inv(or_ef_sub(zl, or_ef_from(1))));
            sel[1] = or_ef_mul(van, or_ef_inv(or_ef_sub(zl, or_ef_from(oinv))));
            sel[2] = or_ef_sub(zl, or_ef_from(oinv));
            size_t K = or_air_num_constraints(inst[i].air, w);
            or_ef *cons = (or_ef *)malloc((K ? K : 1) * sizeof(or_ef));
            or_air_eval_ef(inst[i].air, w, inst[i].consts, L, N, sel, cons);
            or_ef folded = or_ef_from(0);
            for (size_t k = 0; k < K; k++) folded = or_ef_add(or_ef_mul(folded, alpha), cons[k]);
            accumulated = or_ef_add(or_ef_mul(accumulated, beta), folded);
            free(cons);
            free(L);
            free(N);
        }
        /* 11. Q(z) from the D chunks (columns 2t, 2t+1 are the basis
         * coordinates of chunk t) and the quotient identity */
        size_t qoff = 0;
        for (size_t m = 0; m < 2 * n_inst; m++) qoff += aw[m];
        const or_ef X = or_ef_make(0, 1);
        or_ef u = or_ef_exp2(or_ef_mulf(z, or_inv(OR_GEN)), log_max_h);
        uint64_t ws = or_root(log_qd), wt = 1;
        or_ef num = or_ef_from(0), den = or_ef_from(0);
        for (size_t t = 0; t < D; t++) {
            or_ef qt = or_ef_add(evals[qoff + 2 * t], or_ef_mul(X, evals[qoff + 2 * t + 1]));
            or_ef wgt = or_ef_mulf(or_ef_inv(or_ef_sub(u, or_ef_from(wt))), wt);
            num = or_ef_add(num, or_ef_mul(wgt, qt));
            den = or_ef_add(den, wgt);
            wt = or_mul(wt, ws);
        }
        or_ef qz = or_ef_mul(num, or_ef_inv(den));
        or_ef vanish = or_ef_sub(or_ef_exp2(z, log_max_h), or_ef_from(1));
        if (!or_ef_eq(accumulated, or_ef_mul(qz, vanish))) err = OR_VERR_QUOTIENT;
    }
    free(evals);
    free(auxv);
    if (!err && v.short_read) err = OR_VERR_TRANSCRIPT;
    /* 13. transcript fully consumed, digest */
    if (!err && (v.pf != v.nf || v.pc != v.nc)) err = OR_VERR_TRANSCRIPT;
    if (!err) {
        uint64_t dg[12];
        or_ch_finalize(&v.ch, dg);
        if (memcmp(dg, digest, 96) != 0) err = OR_VERR_DIGEST;
    }
    return err;
}
