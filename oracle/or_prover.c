/*
 * ORACLE (test infrastructure only): prove_multi for the Goldilocks/Poseidon2
 * configuration, restated step by step from
 *   p3-miden-lifted-stark/src/prover/mod.rs:223-461        (protocol order)
 *   p3-miden-lifted-stark/src/prover/commit.rs:175-228     (trace commitment)
 *   p3-miden-lifted-stark/src/prover/quotient.rs:40-238    (quotient)
 *   p3-miden-lifted-stark/src/prover/constraints/mod.rs:63-179 (constraint fold)
 *   p3-miden-lifted-stark/src/coset.rs:210-342             (selectors, OOD point)
 *   p3-miden-lifted-fri/src/prover.rs:35-116               (PCS opening)
 *   p3-miden-lifted-fri/src/deep/{interpolate,prover}.rs   (DEEP)
 *   p3-miden-lifted-fri/src/fri/{mod,prover}.rs, fri/fold/arity{2,4,8}.rs (FRI)
 */
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "oracle.h"

static double g_stage[16];
static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
double or_last_stage_seconds(int stage) { return (stage >= 0 && stage < 16) ? g_stage[stage] : 0.0; }

typedef struct {
    or_tree tree;
    uint64_t *ldes[8];
    size_t n;
} committed;

/* commit_traces: per trace, coset LDE on the nested coset g^(2^lift) and
 * bit-reversed rows; then an aligned LMCS tree (commit.rs:198-227). */
static void commit_traces(const or_p2_params *pp, committed *c, const uint64_t *const *traces, const size_t *h,
                          const size_t *w, size_t n, unsigned log_blowup) {
    unsigned log_max = or_log2(h[n - 1]);
    or_matrix mats[8];
    c->n = n;
    for (size_t i = 0; i < n; i++) {
        unsigned lift = log_max - or_log2(h[i]);
        uint64_t shift = or_exp2(OR_GEN, lift);
        size_t lh = h[i] << log_blowup;
        c->ldes[i] = (uint64_t *)malloc(lh * w[i] * 8 + 8);
        or_coset_lde_bitrev(traces[i], h[i], w[i], log_blowup, shift, c->ldes[i]);
        mats[i].data = c->ldes[i];
        mats[i].height = lh;
        mats[i].width = w[i];
    }
    or_tree_build(pp, &c->tree, mats, n, 8);
}
static void committed_free(committed *c) {
    for (size_t i = 0; i < c->n; i++) free(c->ldes[i]);
    or_tree_free(&c->tree);
}

/* arity-a fold of one coset row (fri/fold/arity{2,4,8}.rs): evals are
 * bit-reversed samples y_k = f(s w_a^k); result (1/a) sum_j (beta/s)^j
 * sum_k y_k w_a^{-jk}. */
static or_ef fold_row(const or_ef *ev, unsigned log_a, uint64_t s_inv, or_ef beta) {
    size_t a = (size_t)1 << log_a;
    uint64_t winv = or_inv(or_root(log_a));
    or_ef x = or_ef_mulf(beta, s_inv), xp = or_ef_from(1), res = or_ef_from(0);
    for (size_t j = 0; j < a; j++) {
        or_ef u = or_ef_from(0);
        for (size_t k = 0; k < a; k++) {
            uint64_t wk = or_pow(winv, (j * k) % a);
            u = or_ef_add(u, or_ef_mulf(ev[or_bitrev(k, log_a)], wk));
        }
        res = or_ef_add(res, or_ef_mul(u, xp));
        xp = or_ef_mul(xp, x);
    }
    return or_ef_mulf(res, or_inv((uint64_t)a));
}

static int cmp_size(const void *a, const void *b) {
    size_t x = *(const size_t *)a, y = *(const size_t *)b;
    return x < y ? -1 : x > y;
}

/* LiftedAir properties of an instance: the built-in AIRs declare the
 * examples' dummy aux (one EF column, one challenge, no aux values,
 * p3-miden-lifted-examples/src/lib.rs:93-103); symbolic AIRs their own. */
size_t or_inst_aux_width(const or_instance *I) { return I->air == OR_AIR_SYMBOLIC ? I->sym->aux_width : 1; }
size_t or_inst_num_randomness(const or_instance *I) { return I->air == OR_AIR_SYMBOLIC ? I->sym->num_randomness : 1; }
size_t or_inst_num_aux_values(const or_instance *I) { return I->air == OR_AIR_SYMBOLIC ? I->sym->num_aux_values : 0; }
unsigned or_inst_log_qd(const or_instance *I) {
    return I->air == OR_AIR_SYMBOLIC ? or_sym_log_quotient_degree(I->sym) : or_air_log_quotient_degree(I->air);
}
size_t or_inst_num_constraints(const or_instance *I) {
    return I->air == OR_AIR_SYMBOLIC ? I->sym->n_constraints : or_air_num_constraints(I->air, I->width);
}

/* DEEP openings (PointQuotients::new, p3-miden-lifted-fri/src/deep/interpolate.rs:81-109,
 * and batch_eval_lifted, :123-201): f(z_j) of every column of every matrix
 * (bit-reversed LDEs on g*K, ascending heights, the largest the LDE domain),
 * matrix by matrix, 4 words per column: z_0 (c0, c1), z_1 (c0, c1). The first
 * d_m = h_m / B rows of a bit-reversed LDE are the trace domain's points in
 * bit-reversed order, so f(z) = s(z) sum_i w_i(z) f(x_i) with barycentric
 * weights folded by blocks for shorter matrices. */
void or_deep_evals(const or_matrix *mats, size_t n_mats, unsigned log_blowup, const or_ef zs[2], uint64_t *out) {
    const size_t n_lde = mats[n_mats - 1].height;
    const unsigned log_lde = or_log2(n_lde);
    uint64_t *xs = (uint64_t *)malloc(n_lde * 8);
    uint64_t wn = or_root(log_lde);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n_lde; i++) xs[i] = or_mul(OR_GEN, or_pow(wn, or_bitrev(i, log_lde)));
    size_t d = n_lde >> log_blowup;
    or_ef *q = (or_ef *)malloc(d * 2 * sizeof(or_ef));
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < d; i++)
        for (int j = 0; j < 2; j++) q[2 * i + j] = or_ef_inv(or_ef_sub(zs[j], or_ef_from(xs[i])));
    unsigned log_d = or_log2(d);
    or_ef sj[2];
    for (int j = 0; j < 2; j++) {
        or_ef t = or_ef_sub(or_ef_exp2(or_ef_mulf(zs[j], or_inv(OR_GEN)), log_d), or_ef_from(1));
        sj[j] = or_ef_mulf(t, or_inv((uint64_t)d));
    }
    or_ef *wts = (or_ef *)malloc(d * 2 * sizeof(or_ef));
    size_t off = 0;
    for (size_t m = 0; m < n_mats; m++) {
        const or_matrix *M = &mats[m];
        size_t dm = M->height >> log_blowup, ratio = d / dm;
        for (size_t i = 0; i < dm; i++)
            for (int j = 0; j < 2; j++) {
                or_ef s = or_ef_from(0);
                for (size_t c = 0; c < ratio; c++) {
                    size_t ii = i * ratio + c;
                    s = or_ef_add(s, or_ef_mulf(q[2 * ii + j], xs[ii]));
                }
                wts[2 * i + j] = s;
            }
#pragma omp parallel for schedule(static)
        for (size_t col = 0; col < M->width; col++)
            for (int j = 0; j < 2; j++) {
                or_ef s = or_ef_from(0);
                for (size_t i = 0; i < dm; i++) s = or_ef_add(s, or_ef_mulf(wts[2 * i + j], M->data[i * M->width + col]));
                or_ef e = or_ef_mul(s, sj[j]);
                out[4 * (off + col) + 2 * j] = e.c0;
                out[4 * (off + col) + 2 * j + 1] = e.c1;
            }
        off += M->width;
    }
    free(wts);
    free(q);
    free(xs);
}

/* The DEEP quotient (DeepPoly::from_evals + accumulate_matrices,
 * p3-miden-lifted-fri/src/deep/prover.rs:106-364): columns padded to
 * `alignment` with zeros; f_red(z_j) = Horner in ac over the padded
 * evaluations (z_j), coefficients -ac^{W-1-c}; for each LDE point x_i
 * (bit-reversed), Q = sum_j bp^j (f_red(z_j) - f_red(x_i)) / (z_j - x_i),
 * rows of shorter matrices read lifted (i >> lift). out: 2 words per point. */
void or_deep_quotient(const or_matrix *mats, size_t n_mats, unsigned log_blowup, size_t alignment, const or_ef zs[2],
                      const uint64_t *evals4, or_ef ac, or_ef bp, uint64_t *out) {
    (void)log_blowup;
    const size_t n_lde = mats[n_mats - 1].height;
    const unsigned log_lde = or_log2(n_lde);
    size_t total_aligned = 0;
    size_t *aligned_w = (size_t *)malloc(n_mats * sizeof(size_t));
    for (size_t m = 0; m < n_mats; m++) {
        aligned_w[m] = (mats[m].width + alignment - 1) / alignment * alignment;
        total_aligned += aligned_w[m];
    }
    or_ef fred[2] = {or_ef_from(0), or_ef_from(0)};
    size_t src = 0;
    for (size_t m = 0; m < n_mats; m++)
        for (size_t c = 0; c < aligned_w[m]; c++) {
            for (int j = 0; j < 2; j++) {
                or_ef v = c < mats[m].width ? or_ef_make(evals4[4 * (src + c) + 2 * j], evals4[4 * (src + c) + 2 * j + 1])
                                            : or_ef_from(0);
                fred[j] = or_ef_add(or_ef_mul(fred[j], ac), v);
            }
            if (c + 1 == aligned_w[m]) src += mats[m].width;
        }
    or_ef *coef = (or_ef *)malloc((total_aligned + 1) * sizeof(or_ef));
    {
        or_ef p = or_ef_from(OR_P - 1);
        for (size_t c = total_aligned; c-- > 0;) {
            coef[c] = p;
            p = or_ef_mul(p, ac);
        }
    }
    uint64_t wn = or_root(log_lde);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n_lde; i++) {
        uint64_t x = or_mul(OR_GEN, or_pow(wn, or_bitrev(i, log_lde)));
        or_ef negf = or_ef_from(0);
        size_t off = 0;
        for (size_t m = 0; m < n_mats; m++) {
            const or_matrix *M = &mats[m];
            unsigned liftm = log_lde - or_log2(M->height);
            const uint64_t *row = M->data + (i >> liftm) * M->width;
            for (size_t col = 0; col < M->width; col++) negf = or_ef_add(negf, or_ef_mulf(coef[off + col], row[col]));
            off += aligned_w[m];
        }
        or_ef q0 = or_ef_inv(or_ef_sub(zs[0], or_ef_from(x))), q1 = or_ef_inv(or_ef_sub(zs[1], or_ef_from(x)));
        or_ef r = or_ef_mul(q0, or_ef_add(fred[0], negf));
        r = or_ef_add(r, or_ef_mul(bp, or_ef_mul(q1, or_ef_add(fred[1], negf))));
        out[2 * i] = r.c0;
        out[2 * i + 1] = r.c1;
    }
    free(coef);
    free(aligned_w);
}

/* FriFold::fold_matrix (p3-miden-lifted-fri/src/fri/fold/mod.rs:119-181): a
 * layer of n = 2^log_n EF values (bit-reversed), rows of a = 2^log_a values;
 * row k is the coset s*<w_a>, s = w_n^{bitrev_{log n - log a}(k)}. */
void or_fri_fold(const uint64_t *in, unsigned log_n, unsigned log_a, const uint64_t beta2[2], uint64_t *out) {
    const size_t a = (size_t)1 << log_a, nf = ((size_t)1 << log_n) / a;
    const unsigned ls = log_n - log_a;
    const uint64_t ginv = or_inv(or_root(log_n));
    const or_ef b = or_ef_make(beta2[0], beta2[1]);
    or_ef *row = (or_ef *)malloc(a * sizeof(or_ef));
    for (size_t k = 0; k < nf; k++) {
        for (size_t t = 0; t < a; t++) row[t] = or_ef_make(in[2 * (k * a + t)], in[2 * (k * a + t) + 1]);
        or_ef r = fold_row(row, log_a, or_pow(ginv, or_bitrev(k, ls)), b);
        out[2 * k] = r.c0;
        out[2 * k + 1] = r.c1;
    }
    free(row);
}

int or_prove(const or_p2_params *pp, const or_pcs_params *pcs, const or_instance *inst, size_t n_inst,
             or_proof *out) {
    memset(out, 0, sizeof(*out));
    memset(g_stage, 0, sizeof(g_stage));
    if (n_inst == 0 || n_inst > 8) return 1;
    for (size_t i = 0; i < n_inst; i++) {
        if (inst[i].height < 2 || (inst[i].height & (inst[i].height - 1))) return 2;
        if (i && inst[i].height < inst[i - 1].height) return 3;
        if (inst[i].air == OR_AIR_SYMBOLIC &&
            (!inst[i].sym || or_sym_validate(inst[i].sym) || inst[i].sym->main_width != inst[i].width))
            return 5;
    }
    const unsigned log_blowup = pcs->log_blowup;
    const unsigned log_max_h = or_log2(inst[n_inst - 1].height);
    unsigned log_qd = 0;
    for (size_t i = 0; i < n_inst; i++) {
        unsigned l = or_inst_log_qd(&inst[i]);
        if (l > log_qd) log_qd = l;
    }
    if (log_qd > log_blowup) return 4;
    const unsigned log_lde = log_max_h + log_blowup;
    const size_t n_lde = (size_t)1 << log_lde;
    const size_t D = (size_t)1 << log_qd;
    double t0 = now_s(), t1;

    or_transcript tr;
    or_tr_init(&tr, pp);

    /* 1. main traces */
    const uint64_t *traces[8];
    size_t hs[8], ws[8];
    for (size_t i = 0; i < n_inst; i++) {
        traces[i] = inst[i].trace;
        hs[i] = inst[i].height;
        ws[i] = inst[i].width;
    }
    committed mainc, auxc, quotc;
    commit_traces(pp, &mainc, traces, hs, ws, n_inst, log_blowup);
    or_tree_root(&mainc.tree, out->main_root);
    or_tr_send_commit(&tr, out->main_root);
    t1 = now_s();
    g_stage[0] = t1 - t0;
    t0 = t1;

    /* 2. randomness (max over the AIRs of num_randomness) and the aux
     * traces from each instance's AuxBuilder, flattened EF -> 2 base columns
     * (prover/mod.rs:285-345); without a builder the aux trace is all zero
     * (the examples' dummy builder, p3-miden-lifted-examples/src/lib.rs:93-103). */
    size_t n_rand = 0;
    for (size_t i = 0; i < n_inst; i++)
        if (or_inst_num_randomness(&inst[i]) > n_rand) n_rand = or_inst_num_randomness(&inst[i]);
    uint64_t *rnd = (uint64_t *)calloc(2 * n_rand + 2, 8);
    for (size_t r = 0; r < n_rand; r++) {
        or_ef e = or_ch_sample_ef(&tr.ch);
        rnd[2 * r] = e.c0, rnd[2 * r + 1] = e.c1;
    }
    uint64_t *auxt[8], *auxv[8];
    size_t aw[8];
    for (size_t i = 0; i < n_inst; i++) {
        aw[i] = 2 * or_inst_aux_width(&inst[i]);
        auxt[i] = (uint64_t *)calloc(hs[i] * aw[i] + 1, 8);
        auxv[i] = (uint64_t *)calloc(2 * or_inst_num_aux_values(&inst[i]) + 2, 8);
        if (inst[i].aux_build &&
            inst[i].aux_build(inst[i].aux_user, i, inst[i].trace, rnd, or_inst_num_randomness(&inst[i]), hs[i],
                              auxt[i], auxv[i]) != 0) {
            for (size_t k = 0; k <= i; k++) free(auxt[k]), free(auxv[k]);
            free(rnd);
            or_tr_free(&tr);
            committed_free(&mainc);
            return 6;
        }
    }
    commit_traces(pp, &auxc, (const uint64_t *const *)auxt, hs, aw, n_inst, log_blowup);
    for (size_t i = 0; i < n_inst; i++) free(auxt[i]);
    or_tree_root(&auxc.tree, out->aux_root);
    or_tr_send_commit(&tr, out->aux_root);
    /* aux values, per instance in order (prover/mod.rs:347-353) */
    for (size_t i = 0; i < n_inst; i++)
        for (size_t k = 0; k < or_inst_num_aux_values(&inst[i]); k++)
            or_tr_send_ef(&tr, or_ef_make(auxv[i][2 * k], auxv[i][2 * k + 1]));
    t1 = now_s();
    g_stage[1] = t1 - t0;
    t0 = t1;

    /* 4. constraint folding alpha, accumulation beta */
    or_ef alpha = or_ch_sample_ef(&tr.ch);
    or_ef beta = or_ch_sample_ef(&tr.ch);
    out->alpha[0] = alpha.c0, out->alpha[1] = alpha.c1;
    out->beta[0] = beta.c0, out->beta[1] = beta.c1;

    /* 5. constraints, ascending heights, cyclic extension + beta Horner */
    const size_t max_qh = inst[n_inst - 1].height * D;
    or_ef *acc = (or_ef *)calloc(max_qh, sizeof(or_ef));
    size_t acc_len = 0;
    for (size_t ii = 0; ii < n_inst; ii++) {
        const or_instance *I = &inst[ii];
        unsigned log_h = or_log2(I->height);
        unsigned lift = log_max_h - log_h;
        uint64_t shift = or_exp2(OR_GEN, lift);
        size_t qh = I->height * D;
        unsigned log_qh = log_h + log_qd;
        /* cyclic_extend_and_scale (quotient.rs:348-363) */
        if (acc_len == 0) {
            memset(acc, 0, qh * sizeof(or_ef));
        } else {
            for (size_t i = 0; i < acc_len; i++) acc[i] = or_ef_mul(acc[i], beta);
            while (acc_len < qh) {
                memcpy(acc + acc_len, acc, acc_len * sizeof(or_ef));
                acc_len *= 2;
            }
        }
        acc_len = qh;
        /* selectors on the quotient coset (coset.rs:210-247) */
        uint64_t omega_h_inv = or_inv(or_root(log_h));
        uint64_t omega_q = or_root(log_qh);
        size_t K = or_inst_num_constraints(I);
        const uint64_t *lde = mainc.ldes[ii];
        size_t w = I->width;
        if (I->air == OR_AIR_SYMBOLIC) {
            /* symbolic AIR: the DAG evaluated per point of gJ (constraints/mod.rs:63-179);
             * aux rows as EF, periodic values from PeriodicLde on the
             * quotient coset (periodic.rs:49-98, coset D, read at m mod its height) */
            const or_sym_air *A = I->sym;
            const uint64_t *alde = auxc.ldes[ii];
            const size_t aux_w = A->aux_width, nper = A->num_periodic;
            size_t max_p = 0;
            uint64_t *rep = or_sym_periodic_matrix(A, &max_p);
            uint64_t *plde = NULL;
            size_t ph = 0;
            if (rep) {
                ph = max_p << log_qd;
                plde = (uint64_t *)malloc(ph * nper * 8);
                or_periodic_lde(rep, max_p, nper, log_qd, log_h, shift, plde);
                free(rep);
            }
            or_ef *rand_ef = (or_ef *)malloc((A->num_randomness + 1) * sizeof(or_ef));
            or_ef *auxv_ef = (or_ef *)malloc((A->num_aux_values + 1) * sizeof(or_ef));
            for (size_t r = 0; r < A->num_randomness; r++) rand_ef[r] = or_ef_make(rnd[2 * r], rnd[2 * r + 1]);
            for (size_t r = 0; r < A->num_aux_values; r++) auxv_ef[r] = or_ef_make(auxv[ii][2 * r], auxv[ii][2 * r + 1]);
#pragma omp parallel
            {
                or_ef *ml = (or_ef *)malloc((w + 1) * sizeof(or_ef)), *mn = (or_ef *)malloc((w + 1) * sizeof(or_ef));
                or_ef *al = (or_ef *)malloc((aux_w + 1) * sizeof(or_ef)), *an = (or_ef *)malloc((aux_w + 1) * sizeof(or_ef));
                or_ef *per = (or_ef *)malloc((nper + 1) * sizeof(or_ef));
                or_ef *nodes = (or_ef *)malloc((A->n_nodes + 1) * sizeof(or_ef));
                or_ef *cons = (or_ef *)malloc((K + 1) * sizeof(or_ef));
#pragma omp for schedule(static)
                for (size_t m = 0; m < qh; m++) {
                    uint64_t x = or_mul(shift, or_pow(omega_q, m));
                    uint64_t zh = or_sub(or_exp2(x, log_h), 1);
                    or_sym_point pt;
                    pt.sel[0] = or_ef_from(or_mul(zh, or_inv(or_sub(x, 1))));
                    pt.sel[1] = or_ef_from(or_mul(zh, or_inv(or_sub(x, omega_h_inv))));
                    pt.sel[2] = or_ef_from(or_sub(x, omega_h_inv));
                    size_t rl = or_bitrev(m, log_qh), rn = or_bitrev((m + D) % qh, log_qh);
                    for (size_t c = 0; c < w; c++) ml[c] = or_ef_from(lde[rl * w + c]), mn[c] = or_ef_from(lde[rn * w + c]);
                    for (size_t c = 0; c < aux_w; c++) {
                        al[c] = or_ef_make(alde[rl * 2 * aux_w + 2 * c], alde[rl * 2 * aux_w + 2 * c + 1]);
                        an[c] = or_ef_make(alde[rn * 2 * aux_w + 2 * c], alde[rn * 2 * aux_w + 2 * c + 1]);
                    }
                    for (size_t c = 0; c < nper; c++) per[c] = or_ef_from(plde[(m % ph) * nper + c]);
                    pt.main_local = ml, pt.main_next = mn, pt.aux_local = al, pt.aux_next = an;
                    pt.pub = I->public_values, pt.rand = rand_ef, pt.auxv = auxv_ef, pt.periodic = per;
                    or_sym_eval(A, &pt, nodes, cons);
                    or_ef f = or_ef_from(0);
                    for (size_t k = 0; k < K; k++) f = or_ef_add(or_ef_mul(f, alpha), cons[k]);
                    acc[m] = or_ef_add(acc[m], f);
                }
                free(ml), free(mn), free(al), free(an), free(per), free(nodes), free(cons);
            }
            free(plde), free(rand_ef), free(auxv_ef);
            continue;
        }
#pragma omp parallel
        {
            uint64_t *cons = (uint64_t *)malloc(K * 8);
#pragma omp for schedule(static)
            for (size_t m = 0; m < qh; m++) {
                uint64_t x = or_mul(shift, or_pow(omega_q, m));
                uint64_t zh = or_sub(or_exp2(x, log_h), 1);
                uint64_t sel[3];
                sel[0] = or_mul(zh, or_inv(or_sub(x, 1)));
                sel[1] = or_mul(zh, or_inv(or_sub(x, omega_h_inv)));
                sel[2] = or_sub(x, omega_h_inv);
                const uint64_t *L = lde + or_bitrev(m, log_qh) * w;
                const uint64_t *N = lde + or_bitrev((m + D) % qh, log_qh) * w;
                or_air_eval(I->air, w, I->consts, L, N, sel, cons);
                or_ef f = or_ef_from(0);
                for (size_t k = 0; k < K; k++) f = or_ef_add(or_ef_mul(f, alpha), or_ef_from(cons[k]));
                acc[m] = or_ef_add(acc[m], f);
            }
            free(cons);
        }
    }
    for (size_t i = 0; i < n_inst; i++) free(auxv[i]);
    free(rnd);
    /* 6. divide by Z_H on the max quotient coset (quotient.rs:380-409) */
    {
        uint64_t s_pow_n = or_exp2(OR_GEN, log_max_h);
        uint64_t wd = or_root(log_qd), p = 1;
        uint64_t inv_van[64];
        for (size_t t = 0; t < D; t++) {
            inv_van[t] = or_inv(or_sub(or_mul(s_pow_n, p), 1));
            p = or_mul(p, wd);
        }
        for (size_t i = 0; i < max_qh; i++) acc[i] = or_ef_mulf(acc[i], inv_van[i & (D - 1)]);
    }
    t1 = now_s();
    g_stage[2] = t1 - t0;
    t0 = t1;

    /* 7. commit_quotient (quotient.rs:441-546) */
    {
        size_t N = inst[n_inst - 1].height, NB = N << log_blowup, qw = 2 * D;
        uint64_t *qm = (uint64_t *)malloc(NB * qw * 8);
        uint64_t omega_j_inv = or_inv(or_root(log_max_h + log_qd));
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t col = 0; col < qw; col++) {
            size_t t = col / 2, comp = col & 1;
            uint64_t *v = (uint64_t *)calloc(NB, 8);
            for (size_t r = 0; r < N; r++) v[r] = comp ? acc[r * D + t].c1 : acc[r * D + t].c0;
            or_intt(v, N);
            uint64_t rb = 1; /* (omega_j^-k)^t */
            uint64_t step = or_pow(omega_j_inv, t);
            for (size_t k = 0; k < N; k++) {
                v[k] = or_mul(v[k], rb);
                rb = or_mul(rb, step);
            }
            or_ntt(v, NB);
            for (size_t i = 0; i < NB; i++) qm[or_bitrev(i, log_lde) * qw + col] = v[i];
            free(v);
        }
        or_matrix m = {qm, NB, qw};
        or_tree_build(pp, &quotc.tree, &m, 1, 8);
        quotc.ldes[0] = qm;
        quotc.n = 1;
        or_tree_root(&quotc.tree, out->quot_root);
        or_tr_send_commit(&tr, out->quot_root);
    }
    free(acc);
    t1 = now_s();
    g_stage[3] = t1 - t0;
    t0 = t1;

    /* 8. OOD point outside H and gK (coset.rs:329-342), z_next = z * w_N */
    or_ef z;
    for (;;) {
        z = or_ch_sample_ef(&tr.ch);
        int in_h = or_ef_eq(or_ef_exp2(z, log_max_h), or_ef_from(1));
        int in_gk = or_ef_eq(or_ef_exp2(or_ef_mulf(z, or_inv(OR_GEN)), log_lde), or_ef_from(1));
        if (!in_h && !in_gk) break;
    }
    or_ef zs[2] = {z, or_ef_mulf(z, or_root(log_max_h))};
    out->z[0] = z.c0, out->z[1] = z.c1;

    /* 9. PCS opening: DEEP (deep/prover.rs:171-409, interpolate.rs:81-201) */
    committed *trees[3] = {&mainc, &auxc, &quotc};
    size_t n_mats_total = 0;
    const or_matrix *allm[24];
    for (int g = 0; g < 3; g++)
        for (size_t m = 0; m < trees[g]->tree.n_mats; m++) allm[n_mats_total++] = &trees[g]->tree.mats[m];
    size_t total_aligned = 0;
    for (size_t m = 0; m < n_mats_total; m++) total_aligned += (allm[m]->width + 7) / 8 * 8;
    or_matrix mats_flat[24];
    for (size_t m = 0; m < n_mats_total; m++) mats_flat[m] = *allm[m];
    size_t total_w = 0;
    for (size_t m = 0; m < n_mats_total; m++) total_w += allm[m]->width;
    uint64_t *ev4 = (uint64_t *)malloc((total_w + 1) * 32);
    or_deep_evals(mats_flat, n_mats_total, log_blowup, zs, ev4);
    /* the aligned flat columns [col][j]: zero beyond each matrix's width */
    or_ef *evals = (or_ef *)calloc(total_aligned * 2 + 2, sizeof(or_ef));
    {
        size_t off = 0, src = 0;
        for (size_t m = 0; m < n_mats_total; m++) {
            for (size_t col = 0; col < allm[m]->width; col++, src++)
                for (int j = 0; j < 2; j++) evals[2 * (off + col) + j] = or_ef_make(ev4[4 * src + 2 * j], ev4[4 * src + 2 * j + 1]);
            off += (allm[m]->width + 7) / 8 * 8;
        }
    }
    for (int j = 0; j < 2; j++)
        for (size_t c = 0; c < total_aligned; c++) or_tr_send_ef(&tr, evals[2 * c + j]);
    or_tr_grind(&tr, pcs->deep_pow_bits);
    or_ef ac = or_ch_sample_ef(&tr.ch);
    or_ef bp = or_ch_sample_ef(&tr.ch);
    out->deep_alpha[0] = ac.c0, out->deep_alpha[1] = ac.c1;
    out->deep_beta[0] = bp.c0, out->deep_beta[1] = bp.c1;
    or_ef *deep = (or_ef *)malloc(n_lde * sizeof(or_ef));
    or_deep_quotient(mats_flat, n_mats_total, log_blowup, 8, zs, ev4, ac, bp, (uint64_t *)deep);
    free(ev4);
    free(evals);
    t1 = now_s();
    g_stage[4] = t1 - t0;
    t0 = t1;

    /* FRI commit phase (fri/prover.rs:190-323) */
    const unsigned log_a = pcs->log_folding_arity;
    const size_t arity = (size_t)1 << log_a;
    size_t dom = n_lde;
    unsigned log_max_final = pcs->log_final_degree + log_blowup;
    size_t rounds = log_lde > log_max_final ? (log_lde - log_max_final + log_a - 1) / log_a : 0;
    unsigned log_final_size = log_lde - (unsigned)rounds * log_a;
    size_t final_deg = (size_t)1 << (log_final_size > log_blowup ? log_final_size - log_blowup : 0);
    size_t final_dom = final_deg << log_blowup;
    or_tree *fri_trees = (or_tree *)calloc(rounds + 1, sizeof(or_tree));
    uint64_t **fri_data = (uint64_t **)calloc(rounds + 1, sizeof(uint64_t *));
    size_t nfri = 0;
    uint64_t *s_inv = (uint64_t *)malloc((n_lde / arity) * 8);
    {
        uint64_t ginv = or_inv(or_root(log_lde)), p = 1;
        size_t ns = n_lde / arity;
        uint64_t *tmp = (uint64_t *)malloc(ns * 8);
        for (size_t k = 0; k < ns; k++) {
            tmp[k] = p;
            p = or_mul(p, ginv);
        }
        unsigned ls = or_log2(ns);
        for (size_t k = 0; k < ns; k++) s_inv[k] = tmp[or_bitrev(k, ls)];
        free(tmp);
    }
    or_ef *cur = deep;
    while (dom > final_dom) {
        size_t fd = dom / arity;
        /* flattened (dom/arity) x (2*arity) base matrix, unaligned tree */
        uint64_t *flat = (uint64_t *)malloc(dom * 2 * 8);
        for (size_t i = 0; i < dom; i++) {
            flat[2 * i] = cur[i].c0;
            flat[2 * i + 1] = cur[i].c1;
        }
        or_matrix m = {flat, fd, 2 * arity};
        or_tree_build(pp, &fri_trees[nfri], &m, 1, 1);
        fri_data[nfri] = flat;
        uint64_t root[4];
        or_tree_root(&fri_trees[nfri], root);
        or_tr_send_commit(&tr, root);
        nfri++;
        or_tr_grind(&tr, pcs->folding_pow_bits);
        or_ef b = or_ch_sample_ef(&tr.ch);
        or_ef *nxt = (or_ef *)malloc(fd * sizeof(or_ef));
#pragma omp parallel for schedule(static)
        for (size_t k = 0; k < fd; k++) nxt[k] = fold_row(cur + k * arity, log_a, s_inv[k], b);
        free(cur);
        cur = nxt;
        dom = fd;
        size_t nn = dom / arity;
        for (size_t k = 0; k < nn; k++) s_inv[k] = or_exp2(s_inv[k * arity], log_a);
    }
    free(s_inv);
    /* final polynomial: truncate, bit-reverse, iDFT, descending order */
    {
        unsigned lf = or_log2(final_deg);
        or_ef *v = (or_ef *)malloc(final_deg * sizeof(or_ef));
        for (size_t i = 0; i < final_deg; i++) v[i] = cur[or_bitrev(i, lf)];
        uint64_t *c0 = (uint64_t *)malloc(final_deg * 8), *c1 = (uint64_t *)malloc(final_deg * 8);
        for (size_t i = 0; i < final_deg; i++) c0[i] = v[i].c0, c1[i] = v[i].c1;
        or_intt(c0, final_deg);
        or_intt(c1, final_deg);
        for (size_t i = final_deg; i-- > 0;) or_tr_send_ef(&tr, or_ef_make(c0[i], c1[i]));
        free(c0);
        free(c1);
        free(v);
    }
    free(cur);
    t1 = now_s();
    g_stage[5] = t1 - t0;
    t0 = t1;

    /* query phase (prover.rs:85-115) */
    or_tr_grind(&tr, pcs->query_pow_bits);
    size_t *idx = (size_t *)malloc(pcs->num_queries * sizeof(size_t));
    for (unsigned qi = 0; qi < pcs->num_queries; qi++) idx[qi] = or_bitrev(or_ch_sample_bits(&tr.ch, log_lde), log_lde);
    qsort(idx, pcs->num_queries, sizeof(size_t), cmp_size);
    size_t nu = 0;
    for (size_t i = 0; i < pcs->num_queries; i++)
        if (nu == 0 || idx[nu - 1] != idx[i]) idx[nu++] = idx[i];
    for (int g = 0; g < 3; g++) or_tree_prove_batch(&trees[g]->tree, idx, nu, &tr);
    size_t *ridx = (size_t *)malloc(nu * sizeof(size_t));
    for (size_t r = 0; r < nfri; r++) {
        size_t nr = 0;
        for (size_t i = 0; i < nu; i++) {
            size_t v = idx[i] >> (log_a * (r + 1));
            if (nr == 0 || ridx[nr - 1] != v) ridx[nr++] = v;
        }
        or_tree_prove_batch(&fri_trees[r], ridx, nr, &tr);
    }
    free(ridx);
    free(idx);
    for (size_t r = 0; r < nfri; r++) {
        or_tree_free(&fri_trees[r]);
        free(fri_data[r]);
    }
    free(fri_trees);
    free(fri_data);
    committed_free(&mainc);
    committed_free(&auxc);
    committed_free(&quotc);
    or_ch_finalize(&tr.ch, out->digest);
    out->fields = tr.fields;
    out->n_fields = tr.n_fields;
    out->commits = tr.commits;
    out->n_commits = tr.n_commits;
    t1 = now_s();
    g_stage[6] = t1 - t0;
    return 0;
}
void or_proof_free(or_proof *p) {
    free(p->fields);
    free(p->commits);
    p->fields = p->commits = NULL;
}
