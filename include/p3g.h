/*
 * p3g.h — C ABI of libp3miden_b200.so, the B200 (sm_100a) implementation of
 * the lifted-STARK prover hot path of adr1anh/p3-miden v0.5.0 for the
 * Goldilocks + Poseidon2 configuration (goldilocks_poseidon2:
 * p3-miden-dev-utils/src/configs.rs:393-407).
 *
 * Conventions
 *  - Field elements are canonical Goldilocks values (< 2^64 - 2^32 + 1) in
 *    uint64_t. Extension elements (F[x]/(x^2 - 7)) are two words (c0, c1).
 *  - Matrices are row-major, height x width, one polynomial per column.
 *  - "d_" pointers are device pointers on the context's device; all others
 *    are host pointers.
 *  - Every call returns a status (P3G_OK = 0) and never aborts the process
 *    or traps the GPU; p3g_last_error() describes the last failure of a
 *    context. Calls on one context must come from one host thread at a time.
 *  - Results are bit-identical to the oracle's (oracle/, a CPU restatement of
 *    the reference prover) on the same inputs and permutation table. The
 *    pieces the reference takes from third-party crates that are not in its
 *    source tree are restated, not pinned: the Poseidon2 internal diagonal
 *    (a placeholder by default; the real table is a p3g_ctx_create
 *    argument), DuplexChallenger::finalize, the grind witness choice and the
 *    Keccak AIR's constraint order.
 */
#ifndef P3G_H
#define P3G_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum p3g_status {
    P3G_OK = 0,
    P3G_ERR_INVALID = 1,    /* bad argument: null pointer, size, unsupported parameter */
    P3G_ERR_VALIDATION = 2, /* ProverError / AirValidationError equivalents */
    P3G_ERR_OOM = 3,        /* device allocation refused */
    P3G_ERR_TIMEOUT = 4,    /* a bounded search gave up (proof-of-work) */
    P3G_ERR_CUDA = 5,       /* other CUDA runtime error */
    P3G_ERR_REJECTED = 6    /* a served proof failed the server's self-check (p3g_server_set_self_check) */
};

enum p3g_air {
    P3G_AIR_CUBIC = 1,   /* c_i[r+1] = c_i[r]^3 + c_{(i+1) mod w}[r] + k_i, degree 3 */
    P3G_AIR_KECCAK = 2,  /* Keccak-f[1600] AIR, 2633 columns, 24 rows per permutation */
    P3G_AIR_SYMBOLIC = 3 /* any AIR given as symbolic constraints (p3g_air_create) */
};

typedef struct p3g_ctx p3g_ctx;
typedef struct p3g_tree p3g_tree;
typedef struct p3g_sym_air p3g_sym_air;

/* ------------------------------------------------------- symbolic AIRs
 * LiftedAir (p3-miden-lifted-air/src/air.rs:42-319) through its symbolic
 * form: the expression DAG p3-air's SymbolicAirBuilder records when eval()
 * runs on it (the reference's own symbolic pass, air.rs:225-247; the types
 * are re-exported at p3-miden-lifted-air/src/lib.rs:34-37). Nodes are in
 * topological order (operands before the node). Leaves: constants, main
 * trace cells (column a, row offset b: 0 local, 1 next), aux (permutation)
 * trace cells (extension field), public values, aux randomness (permutation
 * challenges, extension), aux values (permutation values, extension),
 * periodic columns and the three selectors; inner nodes: +, -, *, negation.
 * The constraint list gives the node each assert_zero (is_ext 0) or
 * assert_zero_ext (is_ext 1) asserted, in emission order. */
enum p3g_sym_op {
    P3G_SYM_CONST = 0, P3G_SYM_MAIN = 1, P3G_SYM_AUX = 2, P3G_SYM_PUBLIC = 3, P3G_SYM_RANDOMNESS = 4,
    P3G_SYM_AUX_VALUE = 5, P3G_SYM_PERIODIC = 6, P3G_SYM_IS_FIRST_ROW = 7, P3G_SYM_IS_LAST_ROW = 8,
    P3G_SYM_IS_TRANSITION = 9, P3G_SYM_ADD = 10, P3G_SYM_SUB = 11, P3G_SYM_MUL = 12, P3G_SYM_NEG = 13
};
typedef struct {
    uint32_t op, a, b, pad; /* enum p3g_sym_op; operands or variable index / row offset */
    uint64_t value;         /* P3G_SYM_CONST: a canonical field element */
} p3g_sym_node;
/* AirLayout (air.rs:150-163) plus the periodic columns (LiftedAir::
 * periodic_columns, air.rs:51-57) and the constraint DAG. */
typedef struct {
    uint32_t main_width, aux_width, num_randomness, num_aux_values, num_public_values, num_periodic;
    const uint64_t *periodic_lengths; /* num_periodic powers of two */
    const uint64_t *periodic_values;  /* the periodic columns, concatenated */
    const p3g_sym_node *nodes;
    uint64_t n_nodes;
    const uint32_t *constraints; /* node per constraint, emission order */
    const uint8_t *is_ext;       /* 1: assert_zero_ext, 0: assert_zero */
    uint64_t n_constraints;
} p3g_air_desc;
/* Validates the DAG (operand order; variable indices inside the declared
 * dimensions, the bounds LiftedAir::is_valid_builder checks), derives the
 * degree multiples and log_quotient_degree = log2_ceil(max(M, 2) - 1)
 * (air.rs:225-247) and the base/extension ConstraintLayout
 * (constraints/layout.rs:27-37), generates the constraint kernel for gJ
 * (constraints/mod.rs:63-179) and compiles it with NVRTC for the context's
 * device. P3G_ERR_VALIDATION for a malformed DAG (p3g_last_error says why). */
int p3g_air_create(p3g_ctx *ctx, const p3g_air_desc *desc, p3g_sym_air **out);
void p3g_air_free(p3g_sym_air *air);
uint32_t p3g_air_log_quotient_degree(const p3g_sym_air *air);
uint32_t p3g_air_max_degree(const p3g_sym_air *air);
uint64_t p3g_air_num_constraints_of(const p3g_sym_air *air);
/* Generated constraint kernels (chunks) of the AIR. */
uint64_t p3g_air_num_kernels(const p3g_sym_air *air);
/* ConstraintLayout: base_indices / ext_indices; *n_base and *n_ext are
 * capacities on entry and counts on return. */
int p3g_air_layout(const p3g_sym_air *air, uint64_t *base_idx, uint64_t *n_base, uint64_t *ext_idx, uint64_t *n_ext);
/* No device needed: the analysis, the generated kernel source (*len = size
 * with the terminating zero), and an NVRTC compile for sm_<cc>a. */
int p3g_air_analyse(const p3g_air_desc *desc, uint32_t *max_degree, uint32_t *log_quotient_degree,
                    uint64_t *n_base, uint64_t *n_ext);
int p3g_air_generate_source(const p3g_air_desc *desc, char *buf, uint64_t cap, uint64_t *len);
int p3g_air_compile_check(const p3g_air_desc *desc, int32_t cc, uint64_t *cubin_bytes);

/* AuxBuilder::build_aux_trace (p3-miden-lifted-air/src/auxiliary/builder.rs:
 * 16-37), called once per instance after the main commitment with the
 * instance's num_randomness challenges (2 words each). It writes the aux
 * trace, height x aux_width extension elements (2 words each, row-major)
 * into aux_out and num_aux_values extension elements into aux_values_out
 * (host memory the library provides), and returns 0; any other value ends
 * the proof with P3G_ERR_VALIDATION. main_trace is the instance's trace
 * pointer as given (host or device). */
typedef int (*p3g_aux_build_fn)(void *user, uint64_t instance, const uint64_t *main_trace, const uint64_t *randomness,
                                uint64_t n_randomness, uint64_t height, uint64_t *aux_out, uint64_t *aux_values_out);

/* PcsParams::new(log_blowup, log_folding_arity, log_final_degree,
 * folding_pow_bits, deep_pow_bits, num_queries, query_pow_bits)
 * (p3-miden-lifted-fri/src/params.rs:170-204). */
typedef struct {
    uint32_t log_blowup, log_folding_arity, log_final_degree;
    uint32_t folding_pow_bits, deep_pow_bits, num_queries, query_pow_bits;
} p3g_pcs_params;

/* One (AIR, AirWitness) pair of prove_multi (p3-miden-lifted-stark/src/
 * prover/mod.rs:223-227; AirWitness: p3-miden-lifted-air/src/instance.rs:17-24).
 * The trace is borrowed for the duration of the call. */
typedef struct {
    int32_t air;             /* enum p3g_air */
    int32_t trace_on_device; /* 0: host memory (pinned is fastest), 1: device memory */
    uint64_t height, width;  /* power-of-two height; instances in ascending height order */
    const uint64_t *trace;   /* row-major height x width */
    const uint64_t *consts;  /* host; cubic AIR: k[width]; Keccak: NULL */
    uint64_t n_consts;
    const p3g_sym_air *sym;      /* P3G_AIR_SYMBOLIC: the compiled AIR */
    const uint64_t *public_values; /* AirWitness::public_values (host) */
    uint64_t n_public_values;
    /* The instance's AuxBuilder; NULL: an all-zero aux trace (the examples'
     * dummy builder: one EF column for the built-in AIRs, aux_width columns
     * and num_aux_values zero values for a symbolic AIR). The built-in AIRs
     * declare aux_width 1, num_randomness 1, num_aux_values 0. */
    p3g_aux_build_fn aux_build;
    void *aux_user;
} p3g_instance;

/* StarkOutput { digest, proof: TranscriptData { fields, commitments } }
 * (p3-miden-lifted-stark/src/proof.rs:39-44, p3-miden-transcript/src/data.rs:11-14).
 * Buffers are malloc'ed by the library; release with p3g_proof_free. */
typedef struct {
    uint64_t *fields;
    uint64_t n_fields;
    uint64_t *commits; /* 4 words per commitment */
    uint64_t n_commits;
    uint64_t digest[12];
    double stage_ms[12]; /* device time per protocol stage [0..7]; [8] main-trace LDE kernels;
                            [9] main-tree leaf-sponge launches (span on the prover stream);
                            [10] number of those launches; [11] = whole proof */
    uint64_t gpu_launches;
    uint64_t h2d_bytes, d2h_bytes;
} p3g_proof;

/* ------------------------------------------------------------ context */
/* Creates a context on `device` with the Poseidon2 constants
 * [rc_init 4x12 | rc_term 4x12 | rc_int 22 | diag 12] (130 words): the
 * StarkConfig's permutation (config.rs:26-42, configs.rs:214-233). */
int p3g_ctx_create(int device, const uint64_t *poseidon2_params130, p3g_ctx **out);
void p3g_ctx_destroy(p3g_ctx *ctx);
const char *p3g_last_error(const p3g_ctx *ctx);

/* Poseidon2Goldilocks<12>::new_from_rng_128(SmallRng::seed_from_u64(2025))
 * round constants (configs.rs:215-218) with this build's placeholder
 * internal diagonal. */
void p3g_default_poseidon2_params(uint64_t *out130);
void p3g_poseidon2_params_from_seed(uint64_t seed, const uint64_t *diag12, uint64_t *out130);

/* ------------------------------------------------------------- prover */
/* prove_multi (p3-miden-lifted-stark/src/prover/mod.rs:223-461) with a fresh
 * challenger (configs.rs:231-233). */
int p3g_prove(p3g_ctx *ctx, const p3g_pcs_params *pcs, const p3g_instance *instances, uint64_t n,
              p3g_proof *out);
void p3g_proof_free(p3g_proof *proof);
/* Wire format of a proof (digest + TranscriptData, p3-miden-transcript/src/
 * data.rs:11-49), little-endian: "P3GPROOF", u32 version 1, u32 0,
 * u64 n_fields, u64 n_commits, the 12 digest words (128-byte header), then the
 * field words, then the commitment words (the payload TranscriptData::
 * size_in_bytes counts). p3g_proof_serialize sets *len to the size and fails
 * with P3G_ERR_INVALID when cap is smaller; p3g_proof_deserialize checks the
 * header, the length and that every word is canonical, and fills malloc'ed
 * buffers (release with p3g_proof_free; timing fields are zero). */
uint64_t p3g_proof_wire_size(const p3g_proof *proof);
int p3g_proof_serialize(const p3g_proof *proof, uint8_t *buf, uint64_t cap, uint64_t *len);
int p3g_proof_deserialize(const uint8_t *buf, uint64_t len, p3g_proof *out);

/* ------------------------------------------------------- stage seams */
/* TwoAdicSubgroupDft::coset_lde_batch(trace, log_blowup, shift) followed by
 * bit_reverse_rows (p3-miden-lifted-stark/src/prover/commit.rs:217-222;
 * trait from p3-dft 0.5.0). d_in: height x width, d_out: (height << log_blowup) x width. */
int p3g_coset_lde(p3g_ctx *ctx, const uint64_t *d_in, uint64_t height, uint64_t width, uint32_t log_blowup,
                  uint64_t shift, uint64_t *d_out);

/* PeriodicLde::build (p3-miden-lifted-stark/src/prover/periodic.rs:49-81):
 * d_repeated holds the periodic columns repeated to the largest period
 * (max_period x width); d_out receives their LDE on the coset of shift
 * lde_shift^(2^log_trace_height / max_period), (max_period << log_blowup) x
 * width in natural order, read at row i mod that height (periodic.rs:88-98). */
int p3g_periodic_lde(p3g_ctx *ctx, const uint64_t *d_repeated, uint64_t max_period, uint64_t width,
                     uint32_t log_blowup, uint32_t log_trace_height, uint64_t lde_shift, uint64_t *d_out);
/* Lmcs::build_tree / build_aligned_tree (p3-miden-lmcs/src/lib.rs:191-197,
 * lmcs.rs:412-440) over device matrices sorted by ascending height;
 * alignment 1 = build_tree, 8 = build_aligned_tree (the sponge rate). */
int p3g_lmcs_build(p3g_ctx *ctx, const uint64_t *const *d_mats, const uint64_t *heights, const uint64_t *widths,
                   uint64_t n, uint32_t alignment, p3g_tree **out);
/* HidingLmcsConfig::build_tree / build_aligned_tree (p3-miden-lmcs/src/
 * hiding_lmcs.rs:112-145): as p3g_lmcs_build, and after the matrices every
 * leaf absorbs its row of d_salt (tree height x salt_width, row-major, on the
 * device; the config draws it from its RNG, here the caller supplies it and
 * it stays borrowed). p3g_lmcs_prove_batch then hints each index's salt,
 * unpadded, after its rows (lifted_tree.rs:189-192). */
int p3g_lmcs_build_hiding(p3g_ctx *ctx, const uint64_t *const *d_mats, const uint64_t *heights,
                          const uint64_t *widths, uint64_t n, uint32_t alignment, const uint64_t *d_salt,
                          uint64_t salt_width, p3g_tree **out);
/* Lmcs::open_batch (p3-miden-lmcs/src/lmcs.rs:167-290), hashed on the
 * device: checks the hints of p3g_lmcs_prove_batch (fields: each index's
 * rows padded to the alignment, then salt_width salt words for a hiding
 * tree; commits: the streamed siblings) against commit4 for strictly
 * ascending indices. *verdict: P3G_ACCEPT, P3G_VERR_OPENING (an index outside
 * the tree), P3G_VERR_ROOT or P3G_VERR_TRANSCRIPT (hints too short or left
 * over). */
int p3g_lmcs_open_batch(p3g_ctx *ctx, const uint64_t *commit4, const uint64_t *widths, uint64_t n_mats,
                        uint32_t alignment, uint64_t salt_width, uint32_t log_height, const uint64_t *indices,
                        uint64_t n_idx, const uint64_t *fields, uint64_t n_fields, const uint64_t *commits,
                        uint64_t n_commits, int32_t *verdict);
/* LmcsTree::root (lib.rs:264) */
int p3g_lmcs_root(const p3g_tree *tree, uint64_t *out4);
/* digest layer `level` (0 = leaves) copied to host: (height >> level) x 4 words */
int p3g_lmcs_layer(p3g_ctx *ctx, const p3g_tree *tree, uint32_t level, uint64_t *host_out);
/* LmcsTree::prove_batch hints (lifted_tree.rs:157-224) for strictly
 * ascending indices: rows (padded to the alignment) into fields_out, sibling
 * digests into commits_out; *n_fields / *n_commits are capacities on entry
 * and counts on return. */
int p3g_lmcs_prove_batch(p3g_ctx *ctx, const p3g_tree *tree, const uint64_t *indices, uint64_t n,
                         uint64_t *fields_out, uint64_t *n_fields, uint64_t *commits_out, uint64_t *n_commits);
void p3g_lmcs_free(p3g_tree *tree);

/* LmcsTree::rows (p3-miden-lmcs/src/lib.rs:277, lifted_tree.rs:127-138): the
 * row of each committed matrix at leaf `index` (lifted), each zero-padded to
 * the tree's alignment, concatenated; *n_words is the capacity on entry and
 * the count on return. */
int p3g_lmcs_rows(p3g_ctx *ctx, const p3g_tree *tree, uint64_t index, uint64_t *out, uint64_t *n_words);

/* One FRI round's fold (FriFold::fold_matrix, p3-miden-lifted-fri/src/fri/
 * fold/mod.rs:119-181, arity{2,4,8}.rs:32-148): d_in holds a layer of 2^log_n
 * EF values, bit-reversed; d_out receives the 2^(log_n - log_arity) folded
 * values with challenge beta2. The round's commitment (FriPolys::new,
 * fri/prover.rs:143-150) is p3g_lmcs_build of d_in viewed as
 * (n / a) x 2a base words with alignment 1. */
int p3g_fri_fold(p3g_ctx *ctx, const uint64_t *d_in, uint32_t log_n, uint32_t log_arity, const uint64_t *beta2,
                 uint64_t *d_out);

/* DEEP at the stage seam, over committed matrices (bit-reversed LDEs on g*K,
 * ascending heights; the tallest is the LDE domain), at the points
 * z4 = (z_0, z_1) (2 EF). p3g_deep_evals: PointQuotients::new and
 * batch_eval_lifted (p3-miden-lifted-fri/src/deep/interpolate.rs:81-201),
 * f(z_0), f(z_1) of every column into evals_out (host, 4 words per column,
 * matrix by matrix). p3g_deep_quotient: DeepPoly::from_evals +
 * accumulate_matrices (deep/prover.rs:106-364) with the column challenge
 * alpha2 and the point challenge beta2, columns padded to `alignment`
 * (the LMCS alignment); d_out receives the quotient's n EF values
 * (bit-reversed), the first FRI layer. */
int p3g_deep_evals(p3g_ctx *ctx, const uint64_t *const *d_mats, const uint64_t *heights, const uint64_t *widths,
                   uint64_t n_mats, uint32_t log_blowup, const uint64_t *z4, uint64_t *evals_out);
int p3g_deep_quotient(p3g_ctx *ctx, const uint64_t *const *d_mats, const uint64_t *heights, const uint64_t *widths,
                      uint64_t n_mats, uint32_t log_blowup, uint32_t alignment, const uint64_t *z4,
                      const uint64_t *evals, const uint64_t *alpha2, const uint64_t *beta2, uint64_t *d_out);

/* The configuration's permutation (Poseidon2Goldilocks<12>::permute_mut) on
 * n device states of 12 words, in place. */
int p3g_poseidon2_permute_batch(p3g_ctx *ctx, uint64_t *d_states, uint64_t n);

/* GrindingChallenger::grind (p3-miden-transcript/src/prover.rs:140-144;
 * DuplexChallenger, p3-challenger 0.5.0): the smallest witness w such that a
 * challenger with sponge state `state12` and `n_pending` buffered inputs,
 * after observing w, samples a word whose low `bits` bits are zero. */
int p3g_grind(p3g_ctx *ctx, const uint64_t *state12, const uint64_t *pending, uint32_t n_pending, uint32_t bits,
              uint64_t *witness);

/* No counterpart in the reference. The coset LDE of p3g_coset_lde for
 * callers that cannot allocate device memory (a fixed, pre-reserved HBM
 * budget, or a host runtime whose allocator forbids cudaMalloc/cudaFree on
 * its hot path): it allocates nothing, using a 16.1 MiB static device array
 * inside the library (held by every GPU that loads it). Limits: height <=
 * 2^22 and height * width <= 2^21 words (p3g_coset_lde_noalloc_max_words),
 * else P3G_ERR_INVALID. Asynchronous on `stream`; the first call on a device
 * does a one-time set-up and should come before any stream capture; calls
 * that overlap on the GPU share the array and race. */
int p3g_coset_lde_noalloc(const uint64_t *d_in, uint64_t height, uint64_t width, uint32_t log_blowup, uint64_t shift,
                          uint64_t *d_out, void *stream);
uint64_t p3g_coset_lde_noalloc_max_words(void);

/* ------------------------------------------------------------ autotuning */
/* No counterpart in the reference. Launch shapes of this library timed on
 * the context's device with CUDA events; every choice computes the same
 * values, so only the time changes. p3g_autotune_lde times the candidate
 * splits of a 2^log_height-row coset LDE into bit ranges of at most 10 bits
 * (each range is one shared-memory pass) on random data, keeps the fastest
 * for this context and returns it (best_sizes, *n_sizes capacity on entry,
 * count on return) with its time per LDE and the default split's.
 * p3g_autotune_slabs does the same for the column-slab width of the main
 * commit (LDE + leaf sponge + tree of a device trace; the tuned width
 * applies to device-resident traces, host traces keep about 8 slabs so their
 * upload overlaps the hash). The setters load a
 * saved choice (n = 0 / cols = 0 restore the defaults; a split must have
 * ranges of 1..10 bits adding up to log_height, a slab width must be a
 * multiple of 8, the sponge rate). */
int p3g_autotune_lde(p3g_ctx *ctx, uint32_t log_height, uint64_t width, uint32_t log_blowup, uint32_t reps,
                     uint32_t *best_sizes, uint32_t *n_sizes, double *best_ms, double *default_ms);
int p3g_autotune_slabs(p3g_ctx *ctx, uint32_t log_height, uint64_t width, uint32_t log_blowup, uint32_t reps,
                       uint64_t *best_cols, double *best_ms, double *default_ms);
int p3g_ctx_set_lde_split(p3g_ctx *ctx, uint32_t log_height, const uint32_t *sizes, uint32_t n);
int p3g_ctx_set_slab_columns(p3g_ctx *ctx, uint64_t cols);
/* No counterpart in the reference: the context's memory pool, bytes reserved
 * from the device and in use, and the host time spent in allocation calls
 * since creation (growth of the pool maps device memory inside them). */
/* No counterpart in the reference: DAG nodes per generated constraint kernel
 * for symbolic AIRs created on this context afterwards (0: default 500;
 * otherwise at least 16). Results do not depend on it. */
int p3g_ctx_set_air_chunk_nodes(p3g_ctx *ctx, uint64_t nodes);
int p3g_ctx_memory_stats(p3g_ctx *ctx, uint64_t *reserved_bytes, uint64_t *used_bytes, double *alloc_ms);

/* ------------------------------------------------------------ verifier */
/* verify_multi (p3-miden-lifted-stark/src/verifier/mod.rs:170-364) of a
 * proof made by p3g_prove, with the LMCS openings, the DEEP and the FRI
 * query checks on the device and the transcript replay on the host.
 * `instances` give the shapes only (air, height, width, consts; trace and
 * trace_on_device are ignored). Returns P3G_OK when the check ran, with
 * *verdict = P3G_ACCEPT or the first failing check in verify_multi's order
 * (VerifierError, verifier/mod.rs:75-98; PcsError, p3-miden-lifted-fri/src/
 * verifier.rs:165; FriError, fri/verifier.rs:232; DeepError,
 * deep/verifier.rs:220; LmcsError, p3-miden-lmcs/src/lib.rs:303).
 * P3G_ERR_INVALID for a null pointer, an unsupported parameter or a
 * transcript word that is not a canonical field element. */
enum p3g_verdict {
    P3G_ACCEPT = 0,
    P3G_VERR_SHAPE = 1,      /* instance shapes, ConstraintDegreeTooHigh */
    P3G_VERR_OPENING = 2,    /* an opened index outside its tree */
    P3G_VERR_ROOT = 3,       /* an opening does not hash to its commitment */
    P3G_VERR_POW = 4,        /* a proof-of-work witness fails its bits */
    P3G_VERR_DEEP = 5,       /* a query point equals an out-of-domain point */
    P3G_VERR_FRI = 6,        /* a fold does not match the next round's opening */
    P3G_VERR_FINAL = 7,      /* the final polynomial disagrees with the last fold */
    P3G_VERR_QUOTIENT = 8,   /* ConstraintMismatch at the out-of-domain point */
    P3G_VERR_TRANSCRIPT = 9, /* transcript too short or not fully consumed */
    P3G_VERR_DIGEST = 10     /* transcript digest differs */
};
typedef struct {
    double host_ms;   /* transcript replay and opening layout */
    double device_ms; /* uploads, kernels and read-back */
    uint64_t gpu_launches;
} p3g_verify_stats;
int p3g_verify(p3g_ctx *ctx, const p3g_pcs_params *pcs, const p3g_instance *instances, uint64_t n,
               const uint64_t *fields, uint64_t n_fields, const uint64_t *commits, uint64_t n_commits,
               const uint64_t *digest12, int32_t *verdict, p3g_verify_stats *stats);
/* No counterpart in the reference: verify_multi of n proofs in one call. The
 * transcript replays run on up to host_threads host threads (0: one per
 * hardware thread); then one device pass hashes every proof's openings
 * (one launch for all leaves, one per tree level) and runs the DEEP and FRI
 * checks. verdicts[i] belongs to jobs[i]; stats cover the whole call. */
typedef struct {
    p3g_pcs_params pcs;
    const p3g_instance *instances;
    uint64_t n_instances;
    const uint64_t *fields;
    uint64_t n_fields;
    const uint64_t *commits;
    uint64_t n_commits;
    const uint64_t *digest12;
} p3g_verify_job;
int p3g_verify_batch(p3g_ctx *ctx, const p3g_verify_job *jobs, uint64_t n, uint32_t host_threads, int32_t *verdicts,
                     p3g_verify_stats *stats);
/* ------------------------------------------- batched and served proving */
/* No counterpart in the reference: a job queue in front of p3g_prove
 * (prove_multi, p3-miden-lifted-stark/src/prover/mod.rs:223). n_workers
 * workers on one device, each with its own stream and context, prove jobs
 * concurrently; a job is admitted, in arrival order, when its device
 * footprint (p3g_job_footprint_bytes) fits in what is left of
 * hbm_budget_bytes, or when nothing else runs. Each job's proof is the one
 * p3g_prove returns for it alone. Traces are borrowed until the job is
 * awaited. */
typedef struct p3g_server p3g_server;
typedef struct {
    p3g_pcs_params pcs;
    const p3g_instance *instances;
    uint64_t n_instances;
    double arrival_s;  /* p3g_server_run: submit this many seconds after the call starts */
} p3g_job;
typedef struct {
    int32_t status;    /* the job's own status; other jobs are unaffected by it */
    int32_t verdict;   /* self-check verdict (enum p3g_verdict), -1 when not checked */
    p3g_proof proof;   /* valid when status == P3G_OK; release with p3g_proof_free */
    double submit_s, start_s, end_s;
    double verify_ms;  /* self-check wall time */
} p3g_job_result;

int p3g_server_create(int device, const uint64_t *poseidon2_params130, uint32_t n_workers,
                      uint64_t hbm_budget_bytes, p3g_server **out);
/* No counterpart in the reference. With self-check on, each worker verifies
 * its proof with p3g_verify's checks, on its own stream, before the job ends;
 * a rejected proof ends the job with P3G_ERR_REJECTED and its verdict. */
int p3g_server_set_self_check(p3g_server *srv, int32_t enabled);
/* No counterpart in the reference: saved launch shapes (as
 * p3g_ctx_set_lde_split / p3g_ctx_set_slab_columns) for every worker; call
 * before submitting jobs. */
int p3g_server_set_lde_split(p3g_server *srv, uint32_t log_height, const uint32_t *sizes, uint32_t n);
int p3g_server_set_slab_columns(p3g_server *srv, uint64_t cols);
/* No counterpart in the reference: at most n heavy jobs (LDEs above 2^26
 * words) run at a time; 0 lifts the limit (default 1). */
int p3g_server_set_max_heavy(p3g_server *srv, uint32_t n);
/* Waits for every submitted job, then releases the workers. */
void p3g_server_destroy(p3g_server *srv);
int p3g_server_submit(p3g_server *srv, const p3g_job *job, uint64_t *ticket);
/* Blocks until the ticket's job ends; returns its status. */
int p3g_server_wait(p3g_server *srv, uint64_t ticket, p3g_job_result *out);
/* Submits each job at its arrival time, then waits for all; results[i]
 * belongs to jobs[i]. Returns P3G_OK unless an argument is invalid. */
int p3g_server_run(p3g_server *srv, const p3g_job *jobs, uint64_t n, p3g_job_result *results);
uint64_t p3g_server_peak_admitted_bytes(const p3g_server *srv);
/* Upper bound of the device bytes p3g_prove allocates for these instances. */
uint64_t p3g_job_footprint_bytes(const p3g_pcs_params *pcs, const p3g_instance *instances, uint64_t n);

/* ------------------------------------------------- caller-side helpers */
/* generate_keccak_trace (p3-miden-lifted-examples/src/keccak.rs:54-56):
 * 2^log_height x 2633, n_perms * 24 <= 2^log_height. */
int p3g_keccak_trace(const uint64_t *inputs25, uint64_t n_perms, uint32_t log_height, uint64_t *out);
/* The same rows generated on the device (generate_trace_rows,
 * p3-miden-lifted-examples/src/keccak.rs:54-56): d_inputs25 (device,
 * n_perms x 25) -> d_out (device, 2^log_height x 2633, row-major), on the
 * context's stream; returns when the trace is written. A caller holding only
 * the permutation inputs uploads 200 bytes per permutation instead of the
 * 505 KB of its 24 trace rows. */
int p3g_keccak_trace_device(p3g_ctx *ctx, const uint64_t *d_inputs25, uint64_t n_perms, uint32_t log_height,
                            uint64_t *d_out);
/* SmallRng::seed_from_u64(seed).random::<[u64; 25]>() per permutation
 * (p3-miden-lifted-examples/src/bin/lifted_keccak.rs:167-170) */
int p3g_keccak_inputs(uint64_t seed, uint64_t n_perms, uint64_t *out25);
/* Cubic AIR trace: k then row 0 drawn from SmallRng(seed), forward iteration. */
int p3g_cubic_trace(uint32_t log_height, uint64_t width, uint64_t seed, uint64_t *consts_out, uint64_t *trace_out);
uint64_t p3g_air_num_constraints(int32_t air, uint64_t width);
/* The cubic AIR's trace generated on the device: k and row 0 from
 * SmallRng(seed) (as p3g_cubic_trace), the forward iteration on the device
 * into d_out (device, 2^log_height x width, row-major, width <= 8192);
 * consts_out (host) receives k. Bit-identical to p3g_cubic_trace; the caller
 * uploads nothing. */
int p3g_cubic_trace_device(p3g_ctx *ctx, uint32_t log_height, uint64_t width, uint64_t seed, uint64_t *consts_out,
                           uint64_t *d_out);

#ifdef __cplusplus
}
#endif
#endif /* P3G_H */
