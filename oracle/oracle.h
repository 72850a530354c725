/*
 * ORACLE (test infrastructure only) — a CPU restatement, in plain C, of the
 * lifted-STARK prover path of adr1anh/p3-miden v0.5.0 for the Goldilocks +
 * Poseidon2 configuration. It is the checker for the CUDA product: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference leg
 * may load it. The product library never links or calls it.
 *
 * Each function cites the reference file:line it restates. Third-party
 * pieces (Plonky3 0.5.0 crates, rand 0.10) are restated from their published
 * algorithms; where a constant could not be obtained (the Poseidon2 internal
 * diagonal, the exact Keccak AIR constraint order) the oracle is
 * "parity unpinned" for that piece.
 */
#ifndef ORACLE_H
#define ORACLE_H
#include <stddef.h>
#include <stdint.h>
#include "or_field.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ hashing */
typedef struct { uint64_t s[4]; } or_rng;
void or_rng_seed(or_rng *r, uint64_t seed);
uint64_t or_rng_next(or_rng *r);
uint64_t or_rng_field(or_rng *r);

typedef struct {
    uint64_t rc_init[4][12];
    uint64_t rc_term[4][12];
    uint64_t rc_int[22];
    uint64_t diag[12];
} or_p2_params;

void or_p2_params_from_seed(or_p2_params *pp, uint64_t seed, const uint64_t diag[12]);
void or_p2_permute(const or_p2_params *pp, uint64_t *state12);
void or_sponge_absorb(const or_p2_params *pp, uint64_t *st, const uint64_t *in, size_t n);
void or_compress(const or_p2_params *pp, const uint64_t *l, const uint64_t *r, uint64_t *out);

typedef struct {
    const or_p2_params *pp;
    uint64_t state[12];
    uint64_t in[8];
    uint64_t out[8];
    int n_in, n_out;
} or_challenger;
void or_ch_init(or_challenger *c, const or_p2_params *pp);
void or_ch_observe(or_challenger *c, uint64_t x);
uint64_t or_ch_sample(or_challenger *c);
uint64_t or_ch_sample_bits(or_challenger *c, unsigned bits);
or_ef or_ch_sample_ef(or_challenger *c);
uint64_t or_ch_grind(or_challenger *c, unsigned bits);
void or_ch_finalize(or_challenger *c, uint64_t digest[12]);

typedef struct {
    or_challenger ch;
    uint64_t *fields;
    size_t n_fields, cap_fields;
    uint64_t *commits; /* 4 words each */
    size_t n_commits, cap_commits;
} or_transcript;
void or_tr_init(or_transcript *t, const or_p2_params *pp);
void or_tr_send_field(or_transcript *t, uint64_t v);
void or_tr_send_ef(or_transcript *t, or_ef v);
void or_tr_send_commit(or_transcript *t, const uint64_t *d);
void or_tr_hint_field(or_transcript *t, uint64_t v);
void or_tr_hint_commit(or_transcript *t, const uint64_t *d);
uint64_t or_tr_grind(or_transcript *t, unsigned bits);
void or_tr_free(or_transcript *t);

/* ------------------------------------------------------------------ DFT */
void or_ntt(uint64_t *a, size_t n);  /* natural in, natural out: a_i -> sum_k a_k w_n^{ik} */
void or_intt(uint64_t *a, size_t n); /* inverse, includes 1/n */
/* Coset LDE of a row-major h x w matrix to (h<<log_blowup) x w on shift*K,
 * rows stored bit-reversed (p3-miden-lifted-stark/src/prover/commit.rs:217-222). */
void or_coset_lde_bitrev(const uint64_t *in, size_t h, size_t w, unsigned log_blowup,
                         uint64_t shift, uint64_t *out);

/* PeriodicLde::build (p3-miden-lifted-stark/src/prover/periodic.rs:49-81):
 * natural-order coset LDE of the repeated periodic columns (NaiveDft). */
void or_periodic_lde(const uint64_t *repeated, size_t p, size_t w, unsigned log_blowup, unsigned log_trace_height,
                     uint64_t lde_shift, uint64_t *out);

/* ----------------------------------------------------------------- LMCS */
typedef struct {
    const uint64_t *data; /* row-major */
    size_t height, width;
} or_matrix;
typedef struct {
    size_t n_mats;
    or_matrix mats[8];
    size_t alignment;
    unsigned depth;       /* log2 of the tree height */
    uint64_t *layers;     /* all digest layers, leaves first, 4 words each */
    size_t layer_off[40]; /* offset (in digests) of layer l */
    const uint64_t *salt; /* hiding LMCS: height x salt_width, or NULL */
    size_t salt_width;
} or_tree;
void or_tree_build(const or_p2_params *pp, or_tree *t, const or_matrix *mats, size_t n, size_t alignment);
/* HidingLmcsConfig: each leaf absorbs its salt row after the matrices */
void or_tree_build_hiding(const or_p2_params *pp, or_tree *t, const or_matrix *mats, size_t n, size_t alignment,
                          const uint64_t *salt, size_t salt_width);
void or_tree_root(const or_tree *t, uint64_t out[4]);
void or_tree_free(or_tree *t);
void or_tree_prove_batch(const or_tree *t, const size_t *sorted_unique_idx, size_t n_idx, or_transcript *tr);

/* --------------------------------------------------------------- AIRs */
enum { OR_AIR_CUBIC = 1, OR_AIR_KECCAK = 2 };
size_t or_air_num_constraints(int air, size_t width);
unsigned or_air_log_quotient_degree(int air);
/* Evaluate all constraints of one row pair, in the AIR's emission order.
 * sel = {is_first_row, is_last_row, is_transition}. */
void or_air_eval(int air, size_t width, const uint64_t *consts, const uint64_t *local,
                 const uint64_t *next, const uint64_t sel[3], uint64_t *out);
void or_air_eval_ef(int air, size_t width, const uint64_t *consts, const or_ef *local, const or_ef *next,
                    const or_ef sel[3], or_ef *out);
/* Trace generators (the caller side of the reference path). */
void or_cubic_trace(size_t log_h, size_t width, uint64_t seed, uint64_t *consts_out, uint64_t *trace_out);
size_t or_keccak_num_cols(void);
void or_keccak_trace(const uint64_t *inputs25, size_t n_perms, size_t log_h, uint64_t *trace_out);
void or_keccak_inputs(uint64_t seed, size_t n_perms, uint64_t *out25);
/* debug check: returns index of first failing (row*K + constraint) + 1, or 0 */
size_t or_check_constraints(int air, size_t height, size_t width, const uint64_t *consts, const uint64_t *trace);

/* ------------------------------------------------------- symbolic AIRs
 * (or_sym.c) constraint DAGs from p3-air's SymbolicAirBuilder */
enum {
    OR_SYM_CONST = 0,         /* value */
    OR_SYM_MAIN = 1,          /* main column a, row offset b (0 local, 1 next) */
    OR_SYM_AUX = 2,           /* aux EF column a, row offset b */
    OR_SYM_PUBLIC = 3,        /* public value a */
    OR_SYM_RANDOMNESS = 4,    /* aux randomness a (EF) */
    OR_SYM_AUX_VALUE = 5,     /* aux value a (EF) */
    OR_SYM_PERIODIC = 6,      /* periodic column a */
    OR_SYM_IS_FIRST_ROW = 7,
    OR_SYM_IS_LAST_ROW = 8,
    OR_SYM_IS_TRANSITION = 9,
    OR_SYM_ADD = 10,
    OR_SYM_SUB = 11,
    OR_SYM_MUL = 12,
    OR_SYM_NEG = 13
};
typedef struct {
    uint32_t op, a, b, pad;
    uint64_t value;
} or_sym_node;
typedef struct {
    uint32_t main_width, aux_width, num_randomness, num_aux_values, num_public_values, num_periodic;
    const uint64_t *periodic_lengths; /* num_periodic powers of two */
    const uint64_t *periodic_values;  /* the columns, concatenated */
    const or_sym_node *nodes;
    size_t n_nodes;
    const uint32_t *constraints; /* node per constraint, emission order */
    const uint8_t *is_ext;       /* assert_zero_ext (1) or assert_zero (0) */
    size_t n_constraints;
} or_sym_air;
typedef struct {
    const or_ef *main_local, *main_next, *aux_local, *aux_next;
    const uint64_t *pub;
    const or_ef *rand, *auxv, *periodic;
    or_ef sel[3]; /* is_first_row, is_last_row, is_transition */
} or_sym_point;
int or_sym_validate(const or_sym_air *a);
unsigned or_sym_max_degree(const or_sym_air *a);
unsigned or_sym_log_quotient_degree(const or_sym_air *a);
void or_sym_eval(const or_sym_air *a, const or_sym_point *pt, or_ef *scratch_nodes, or_ef *out_constraints);
uint64_t *or_sym_periodic_matrix(const or_sym_air *a, size_t *max_p);
void or_sym_periodic_at(const or_sym_air *a, size_t max_trace_height, or_ef z, or_ef *out);

/* --------------------------------------------------------------- prover */
typedef struct {
    unsigned log_blowup, log_folding_arity, log_final_degree;
    unsigned folding_pow_bits, deep_pow_bits, num_queries, query_pow_bits;
} or_pcs_params;

/* AuxBuilder::build_aux_trace (p3-miden-lifted-air/src/auxiliary/builder.rs:16-37):
 * writes the aux trace (height x aux_width EF, 2 words each, row-major) and
 * num_aux_values EF values; 0 = success. */
typedef int (*or_aux_fn)(void *user, uint64_t instance, const uint64_t *main_trace, const uint64_t *randomness,
                         uint64_t n_randomness, uint64_t height, uint64_t *aux_out, uint64_t *aux_values_out);

enum { OR_AIR_SYMBOLIC = 3 };
typedef struct {
    int air;
    size_t height, width;
    const uint64_t *trace;  /* row-major height x width */
    const uint64_t *consts; /* AIR constants (cubic: k[width]) */
    const or_sym_air *sym;  /* OR_AIR_SYMBOLIC */
    const uint64_t *public_values;
    or_aux_fn aux_build;    /* NULL: the all-zero aux trace */
    void *aux_user;
} or_instance;

typedef struct {
    uint64_t *fields;
    size_t n_fields;
    uint64_t *commits;
    size_t n_commits;
    uint64_t digest[12];
    /* intermediate values exposed for stage-by-stage parity tests */
    uint64_t main_root[4], aux_root[4], quot_root[4];
    uint64_t alpha[2], beta[2], z[2];
    uint64_t deep_alpha[2], deep_beta[2];
} or_proof;

int or_prove(const or_p2_params *pp, const or_pcs_params *pcs, const or_instance *inst, size_t n_inst,
             or_proof *out);
void or_deep_evals(const or_matrix *mats, size_t n_mats, unsigned log_blowup, const or_ef zs[2], uint64_t *out);
void or_deep_quotient(const or_matrix *mats, size_t n_mats, unsigned log_blowup, size_t alignment, const or_ef zs[2],
                      const uint64_t *evals4, or_ef ac, or_ef bp, uint64_t *out);
void or_fri_fold(const uint64_t *in, unsigned log_n, unsigned log_a, const uint64_t beta2[2], uint64_t *out);
size_t or_inst_aux_width(const or_instance *I);
size_t or_inst_num_randomness(const or_instance *I);
size_t or_inst_num_aux_values(const or_instance *I);
unsigned or_inst_log_qd(const or_instance *I);
size_t or_inst_num_constraints(const or_instance *I);
void or_proof_free(or_proof *p);

/* --------------------------------------------------------------- verifier */
enum {
    OR_VERR_SHAPE = 1,   /* instances not ascending / not powers of two, degree > blowup */
    OR_VERR_OPENING,     /* query index outside the tree */
    OR_VERR_ROOT,        /* an LMCS opening does not reproduce its commitment */
    OR_VERR_POW,         /* a proof-of-work witness fails */
    OR_VERR_DEEP,        /* an evaluation point lies on the LDE domain */
    OR_VERR_FRI,         /* an FRI row does not contain the folded value */
    OR_VERR_FINAL,       /* the final polynomial disagrees with the last fold */
    OR_VERR_QUOTIENT,    /* folded constraints != Q(z) * Z_H(z) */
    OR_VERR_TRANSCRIPT,  /* transcript too short or not fully consumed */
    OR_VERR_DIGEST,      /* final challenger state differs from the proof's digest */
};
/* Verify a proof (fields, commitments, digest) for the given instances
 * (air, height, width, consts; traces are not read). 0 = accepted. */
int or_verify(const or_p2_params *pp, const or_pcs_params *pcs, const or_instance *inst, size_t n_inst,
              const uint64_t *fields, size_t n_fields, const uint64_t *commits, size_t n_commits,
              const uint64_t digest[12]);
/* Stage timers of the last or_prove call (seconds), by stage index. */
double or_last_stage_seconds(int stage);

#ifdef __cplusplus
}
#endif
#endif
