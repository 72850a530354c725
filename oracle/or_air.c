/*
 * ORACLE (test infrastructure only): the two AIRs on the measured path and
 * their trace generators.
 *
 * 1. Cubic AIR (synthetic degree-3 AIR of the lifted multi-trace workload):
 *    column i obeys c_i[r+1] = c_i[r]^3 + c_{(i+1) mod w}[r] + k_i on every
 *    row but the last. Constraint i (emission order i = 0..w-1) is
 *    is_transition * (next[i] - (local[i]^3 + local[(i+1) mod w] + k_i)).
 *    Trace: SmallRng(seed) draws k_0..k_{w-1}, then row 0; later rows by
 *    forward iteration.
 *
 * 2. Keccak-f[1600] AIR, the AIR LiftedKeccakAir delegates to
 *    (p3-miden-lifted-examples/src/keccak.rs:13-59; KeccakAir from
 *    p3-keccak-air 0.5.0, not vendored). One row per round, 24 rows per
 *    permutation, 2633 columns laid out as
 *      step_flags[24] | export | preimage[y][x][4] | a[y][x][4] | c[x][64] |
 *      c'[x][64] | a'[y][x][64] | a''[y][x][4] | a''[0][0] bits[64] |
 *      a'''[0][0] limbs[4]            (16-bit limbs, little-endian)
 *    The constraint list restates the published KeccakAir arithmetization;
 *    its emission order is "parity unpinned" against p3-keccak-air 0.5.0.
 */
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

/* ------------------------------------------------------------ cubic --- */
void or_cubic_trace(size_t log_h, size_t width, uint64_t seed, uint64_t *k, uint64_t *trace) {
    or_rng r;
    or_rng_seed(&r, seed);
    for (size_t i = 0; i < width; i++) k[i] = or_rng_field(&r);
    for (size_t i = 0; i < width; i++) trace[i] = or_rng_field(&r);
    size_t h = (size_t)1 << log_h;
    for (size_t row = 1; row < h; row++) {
        const uint64_t *p = trace + (row - 1) * width;
        uint64_t *q = trace + row * width;
        for (size_t i = 0; i < width; i++) {
            uint64_t x = p[i];
            q[i] = or_add(or_add(or_mul(or_mul(x, x), x), p[(i + 1) % width]), k[i]);
        }
    }
}

/* ----------------------------------------------------------- keccak --- */
#define KC_STEP 0
#define KC_EXPORT 24
#define KC_PRE 25
#define KC_A 125
#define KC_C 225
#define KC_CP 545
#define KC_AP 865
#define KC_APP 2465
#define KC_APP00 2565
#define KC_APPP00 2629
#define KC_NCOLS 2633

size_t or_keccak_num_cols(void) { return KC_NCOLS; }

static int rot_r[5][5]; /* rot_r[x][y] */
static uint64_t rc64[24];
static int keccak_tables_ready = 0;

/* FIPS 202: rotation offsets by the (t+1)(t+2)/2 walk; round constants from
 * the degree-8 LFSR rc(t). */
static int lfsr_rc(int t) {
    if (t % 255 == 0) return 1;
    unsigned R = 1;
    for (int i = 1; i <= t % 255; i++) {
        R <<= 1;
        if (R & 0x100) R ^= 0x171;
    }
    return R & 1;
}
static void keccak_tables(void) {
    if (keccak_tables_ready) return;
    memset(rot_r, 0, sizeof(rot_r));
    int x = 1, y = 0;
    for (int t = 0; t < 24; t++) {
        rot_r[x][y] = ((t + 1) * (t + 2) / 2) % 64;
        int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
    for (int i = 0; i < 24; i++) {
        uint64_t rc = 0;
        for (int j = 0; j <= 6; j++)
            if (lfsr_rc(j + 7 * i)) rc |= 1ULL << ((1u << j) - 1);
        rc64[i] = rc;
    }
    keccak_tables_ready = 1;
}
static inline uint64_t rotl(uint64_t v, int r) { return r ? (v << r) | (v >> (64 - r)) : v; }

/* Keccak-f[1600] input states: SmallRng(seed).random::<[u64; 25]>() per
 * permutation (p3-miden-lifted-examples/src/bin/lifted_keccak.rs:167-170),
 * lane (x, y) = state[x + 5y]. */
void or_keccak_inputs(uint64_t seed, size_t n_perms, uint64_t *out25) {
    or_rng r;
    or_rng_seed(&r, seed);
    for (size_t i = 0; i < 25 * n_perms; i++) out25[i] = or_rng_next(&r);
}

static void put_limbs(uint64_t *dst, uint64_t v) {
    for (int l = 0; l < 4; l++) dst[l] = (v >> (16 * l)) & 0xffff;
}
static void gen_perm_rows(uint64_t *rows, size_t nrows, const uint64_t *input) {
    uint64_t A[5][5]; /* A[x][y] */
    for (int y = 0; y < 5; y++)
        for (int x = 0; x < 5; x++) A[x][y] = input[x + 5 * y];
    for (size_t r = 0; r < nrows; r++) {
        uint64_t *row = rows + r * KC_NCOLS;
        row[KC_STEP + r] = 1;
        for (int y = 0; y < 5; y++)
            for (int x = 0; x < 5; x++) {
                put_limbs(row + KC_PRE + (y * 5 + x) * 4, input[x + 5 * y]);
                put_limbs(row + KC_A + (y * 5 + x) * 4, A[x][y]);
            }
        uint64_t C[5], Cp[5], Ap[5][5], B[5][5], App[5][5];
        for (int x = 0; x < 5; x++) C[x] = A[x][0] ^ A[x][1] ^ A[x][2] ^ A[x][3] ^ A[x][4];
        for (int x = 0; x < 5; x++) Cp[x] = C[x] ^ C[(x + 4) % 5] ^ rotl(C[(x + 1) % 5], 1);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) Ap[x][y] = A[x][y] ^ C[(x + 4) % 5] ^ rotl(C[(x + 1) % 5], 1);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) B[y][(2 * x + 3 * y) % 5] = rotl(Ap[x][y], rot_r[x][y]);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) App[x][y] = B[x][y] ^ (~B[(x + 1) % 5][y] & B[(x + 2) % 5][y]);
        for (int x = 0; x < 5; x++)
            for (int z = 0; z < 64; z++) {
                row[KC_C + x * 64 + z] = (C[x] >> z) & 1;
                row[KC_CP + x * 64 + z] = (Cp[x] >> z) & 1;
            }
        for (int y = 0; y < 5; y++)
            for (int x = 0; x < 5; x++) {
                for (int z = 0; z < 64; z++) row[KC_AP + (y * 5 + x) * 64 + z] = (Ap[x][y] >> z) & 1;
                put_limbs(row + KC_APP + (y * 5 + x) * 4, App[x][y]);
            }
        for (int z = 0; z < 64; z++) row[KC_APP00 + z] = (App[0][0] >> z) & 1;
        uint64_t a000 = App[0][0] ^ rc64[r];
        put_limbs(row + KC_APPP00, a000);
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++) A[x][y] = App[x][y];
        A[0][0] = a000;
    }
}
/* generate_trace_rows(inputs, 0): 2^log_h rows (the next power of two of
 * 24 * n_perms); the rows past the inputs hold (possibly truncated)
 * permutations of the all-zero state. */
void or_keccak_trace(const uint64_t *inputs25, size_t n_perms, size_t log_h, uint64_t *trace) {
    keccak_tables();
    size_t h = (size_t)1 << log_h;
    memset(trace, 0, h * KC_NCOLS * 8);
    size_t n_chunks = (h + 23) / 24;
    static const uint64_t zero[25] = {0};
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < n_chunks; c++) {
        size_t nrows = (c + 1) * 24 <= h ? 24 : h - c * 24;
        gen_perm_rows(trace + c * 24 * KC_NCOLS, nrows, c < n_perms ? inputs25 + 25 * c : zero);
    }
}

/* The constraint list, instantiated over F (quotient domain) and over EF
 * (the verifier's out-of-domain point). */
#define KT uint64_t
#define K_ADD or_add
#define K_SUB or_sub
#define K_MUL or_mul
#define K_C(u) ((uint64_t)(u))
#define K_FN(name) name
#include "or_keccak_cons.inc"
#undef KT
#undef K_ADD
#undef K_SUB
#undef K_MUL
#undef K_C
#undef K_FN
#define KT or_ef
#define K_ADD or_ef_add
#define K_SUB or_ef_sub
#define K_MUL or_ef_mul
#define K_C(u) or_ef_from((uint64_t)(u))
#define K_FN(name) name##_ef
#include "or_keccak_cons.inc"
#undef KT
#undef K_ADD
#undef K_SUB
#undef K_MUL
#undef K_C
#undef K_FN

size_t or_air_num_constraints(int air, size_t width) {
    if (air == OR_AIR_CUBIC) return width;
    if (air == OR_AIR_KECCAK) {
        uint64_t dummy[KC_NCOLS] = {0}, sel[3] = {0, 0, 0};
        return keccak_eval(dummy, dummy, sel, NULL);
    }
    return 0;
}
/* Both AIRs have maximal constraint degree 3 (is_transition counts 0,
 * is_first_row 1), so log2_ceil(3 - 1) = 1
 * (p3-miden-lifted-air/src/air.rs:267-289). */
unsigned or_air_log_quotient_degree(int air) {
    (void)air;
    return 1;
}
void or_air_eval(int air, size_t width, const uint64_t *consts, const uint64_t *L, const uint64_t *N,
                 const uint64_t sel[3], uint64_t *out) {
    if (air == OR_AIR_CUBIC) {
        for (size_t i = 0; i < width; i++) {
            uint64_t x = L[i];
            uint64_t rhs = or_add(or_add(or_mul(or_mul(x, x), x), L[(i + 1) % width]), consts[i]);
            out[i] = or_mul(sel[2], or_sub(N[i], rhs));
        }
    } else if (air == OR_AIR_KECCAK) {
        keccak_eval(L, N, sel, out);
    }
}

/* Constraints of one row pair over EF (the verifier's local/next openings
 * at z and z*w), in emission order; sel as in or_air_eval. */
void or_air_eval_ef(int air, size_t width, const uint64_t *consts, const or_ef *L, const or_ef *N, const or_ef sel[3],
                    or_ef *out) {
    if (air == OR_AIR_CUBIC) {
        for (size_t i = 0; i < width; i++) {
            or_ef x = L[i];
            or_ef rhs = or_ef_add(or_ef_add(or_ef_mul(or_ef_mul(x, x), x), L[(i + 1) % width]), or_ef_from(consts[i]));
            out[i] = or_ef_mul(sel[2], or_ef_sub(N[i], rhs));
        }
    } else if (air == OR_AIR_KECCAK) {
        keccak_eval_ef(L, N, sel, out);
    }
}

/* Row-by-row check on the trace domain (selectors as field values there),
 * mirroring the debug checker p3-miden-lifted-stark/src/debug.rs:44. */
size_t or_check_constraints(int air, size_t height, size_t width, const uint64_t *consts, const uint64_t *trace) {
    size_t K = or_air_num_constraints(air, width);
    uint64_t *out = (uint64_t *)malloc(K * 8);
    size_t bad = 0;
    for (size_t r = 0; r < height && !bad; r++) {
        uint64_t sel[3] = {r == 0, r == height - 1, r != height - 1};
        or_air_eval(air, width, consts, trace + r * width, trace + ((r + 1) % height) * width, sel, out);
        for (size_t k = 0; k < K; k++)
            if (out[k]) {
                bad = r * K + k + 1;
                break;
            }
    }
    free(out);
    return bad;
}
