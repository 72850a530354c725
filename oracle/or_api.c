/*
 * ORACLE (test infrastructure only): exported wrappers so tests can call the
 * oracle's inline field arithmetic and parameter set-up through ctypes.
 */
#include <string.h>
#include "oracle.h"

uint64_t or_x_add(uint64_t a, uint64_t b) { return or_add(a, b); }
uint64_t or_x_sub(uint64_t a, uint64_t b) { return or_sub(a, b); }
uint64_t or_x_mul(uint64_t a, uint64_t b) { return or_mul(a, b); }
uint64_t or_x_mul_ref(uint64_t a, uint64_t b) { return or_mul_ref(a, b); }
uint64_t or_x_inv(uint64_t a) { return or_inv(a); }
uint64_t or_x_root(unsigned k) { return or_root(k); }
void or_x_ef_mul(const uint64_t *a, const uint64_t *b, uint64_t *out) {
    or_ef r = or_ef_mul(or_ef_make(a[0], a[1]), or_ef_make(b[0], b[1]));
    out[0] = r.c0;
    out[1] = r.c1;
}
void or_x_ef_inv(const uint64_t *a, uint64_t *out) {
    or_ef r = or_ef_inv(or_ef_make(a[0], a[1]));
    out[0] = r.c0;
    out[1] = r.c1;
}

/* Placeholder internal diagonal for Poseidon2 width 12: 12 uniform field
 * elements from SmallRng::seed_from_u64(0x646961675f3132). p3-goldilocks
 * 0.5.0's MATRIX_DIAG_12 is not available here; hashes are parity-unpinned
 * until a caller loads the real diagonal. */
void or_p2_placeholder_diag(uint64_t out[12]) {
    or_rng r;
    or_rng_seed(&r, 0x646961675f3132ULL);
    for (int i = 0; i < 12; i++) out[i] = or_rng_field(&r);
}
/* The configuration's permutation: constants from SmallRng(2025)
 * (p3-miden-dev-utils/src/configs.rs:215-218, fixtures.rs:15). */
void or_p2_default_params(or_p2_params *pp) {
    uint64_t diag[12];
    or_p2_placeholder_diag(diag);
    or_p2_params_from_seed(pp, 2025, diag);
}
size_t or_p2_params_size(void) { return sizeof(or_p2_params); }
size_t or_proof_struct_size(void) { return sizeof(or_proof); }
