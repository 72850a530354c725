/*
 * ORACLE (test infrastructure only): AIRs given as symbolic constraint
 * expressions, the output of p3-air 0.5.0's SymbolicAirBuilder that the
 * reference runs its AIRs through (p3-miden-lifted-air/src/air.rs:225-247,
 * re-exported at p3-miden-lifted-air/src/lib.rs:34-37).
 *
 * An expression is a DAG of nodes in topological order. Leaves are
 * constants, trace variables (main columns and aux EF columns at the local or
 * next row), public values, aux randomness, aux values, periodic columns and
 * the three selectors; inner nodes are +, -, * and negation. The constraint
 * list gives, in emission order, the node each assert_zero / assert_zero_ext
 * asserted.
 *
 * Degree multiples follow p3-air's SymbolicExpression::degree_multiple:
 * trace variables and periodic columns 1, is_first_row / is_last_row 1,
 * is_transition 0, constants, public values, randomness and aux values 0;
 * a sum takes the maximum, a product the sum. log_quotient_degree is
 * log2_ceil(max(M, 2) - 1) (air.rs:225-247).
 *
 * Evaluation runs every node in the extension field: base-field values are
 * embedded (c1 = 0), which gives the same values as base-field arithmetic.
 */
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

unsigned or_sym_max_degree(const or_sym_air *a) {
    unsigned *deg = (unsigned *)calloc(a->n_nodes ? a->n_nodes : 1, sizeof(unsigned));
    for (size_t i = 0; i < a->n_nodes; i++) {
        const or_sym_node *n = &a->nodes[i];
        switch (n->op) {
            case OR_SYM_MAIN: case OR_SYM_AUX: case OR_SYM_PERIODIC:
            case OR_SYM_IS_FIRST_ROW: case OR_SYM_IS_LAST_ROW: deg[i] = 1; break;
            case OR_SYM_ADD: case OR_SYM_SUB: deg[i] = deg[n->a] > deg[n->b] ? deg[n->a] : deg[n->b]; break;
            case OR_SYM_MUL: deg[i] = deg[n->a] + deg[n->b]; break;
            case OR_SYM_NEG: deg[i] = deg[n->a]; break;
            default: deg[i] = 0; break;
        }
    }
    unsigned m = 0;
    for (size_t k = 0; k < a->n_constraints; k++)
        if (deg[a->constraints[k]] > m) m = deg[a->constraints[k]];
    free(deg);
    return m;
}

unsigned or_sym_log_quotient_degree(const or_sym_air *a) {
    unsigned m = or_sym_max_degree(a);
    if (m < 2) m = 2;
    unsigned l = 0;
    while (((size_t)1 << l) < (size_t)(m - 1)) l++;
    return l;
}

void or_sym_eval(const or_sym_air *a, const or_sym_point *pt, or_ef *v, or_ef *out) {
    for (size_t i = 0; i < a->n_nodes; i++) {
        const or_sym_node *n = &a->nodes[i];
        or_ef r;
        switch (n->op) {
            case OR_SYM_CONST: r = or_ef_from(n->value); break;
            case OR_SYM_MAIN: r = n->b ? pt->main_next[n->a] : pt->main_local[n->a]; break;
            case OR_SYM_AUX: r = n->b ? pt->aux_next[n->a] : pt->aux_local[n->a]; break;
            case OR_SYM_PUBLIC: r = or_ef_from(pt->pub[n->a]); break;
            case OR_SYM_RANDOMNESS: r = pt->rand[n->a]; break;
            case OR_SYM_AUX_VALUE: r = pt->auxv[n->a]; break;
            case OR_SYM_PERIODIC: r = pt->periodic[n->a]; break;
            case OR_SYM_IS_FIRST_ROW: r = pt->sel[0]; break;
            case OR_SYM_IS_LAST_ROW: r = pt->sel[1]; break;
            case OR_SYM_IS_TRANSITION: r = pt->sel[2]; break;
            case OR_SYM_ADD: r = or_ef_add(v[n->a], v[n->b]); break;
            case OR_SYM_SUB: r = or_ef_sub(v[n->a], v[n->b]); break;
            case OR_SYM_MUL: r = or_ef_mul(v[n->a], v[n->b]); break;
            default: r = or_ef_neg(v[n->a]); break; /* OR_SYM_NEG */
        }
        v[i] = r;
    }
    for (size_t k = 0; k < a->n_constraints; k++) out[k] = v[a->constraints[k]];
}

/* Shape checks: operands precede their node, variable indices inside the
 * declared dimensions (the guarantee LiftedAir::is_valid_builder gives the
 * reference, air.rs:268-319). 0 = valid. */
int or_sym_validate(const or_sym_air *a) {
    for (size_t i = 0; i < a->n_nodes; i++) {
        const or_sym_node *n = &a->nodes[i];
        switch (n->op) {
            case OR_SYM_CONST: if (n->value >= OR_P) return 1; break;
            case OR_SYM_MAIN: if (n->a >= a->main_width || n->b > 1) return 1; break;
            case OR_SYM_AUX: if (n->a >= a->aux_width || n->b > 1) return 1; break;
            case OR_SYM_PUBLIC: if (n->a >= a->num_public_values) return 1; break;
            case OR_SYM_RANDOMNESS: if (n->a >= a->num_randomness) return 1; break;
            case OR_SYM_AUX_VALUE: if (n->a >= a->num_aux_values) return 1; break;
            case OR_SYM_PERIODIC: if (n->a >= a->num_periodic) return 1; break;
            case OR_SYM_IS_FIRST_ROW: case OR_SYM_IS_LAST_ROW: case OR_SYM_IS_TRANSITION: break;
            case OR_SYM_ADD: case OR_SYM_SUB: case OR_SYM_MUL: if (n->a >= i || n->b >= i) return 1; break;
            case OR_SYM_NEG: if (n->a >= i) return 1; break;
            default: return 1;
        }
    }
    for (size_t k = 0; k < a->n_constraints; k++)
        if (a->constraints[k] >= a->n_nodes) return 1;
    for (uint32_t c = 0; c < a->num_periodic; c++) {
        uint64_t p = a->periodic_lengths[c];
        if (p == 0 || (p & (p - 1))) return 1;
    }
    return 0;
}

/* The periodic columns repeated to the largest period (max_p x num_periodic),
 * as periodic_columns_matrix builds them (air.rs:64-84). */
uint64_t *or_sym_periodic_matrix(const or_sym_air *a, size_t *max_p) {
    size_t mp = 0, off = 0;
    for (uint32_t c = 0; c < a->num_periodic; c++)
        if (a->periodic_lengths[c] > mp) mp = a->periodic_lengths[c];
    *max_p = mp;
    if (!mp) return NULL;
    uint64_t *m = (uint64_t *)malloc(mp * a->num_periodic * 8);
    for (uint32_t c = 0; c < a->num_periodic; c++) {
        size_t p = a->periodic_lengths[c];
        for (size_t r = 0; r < mp; r++) m[r * a->num_periodic + c] = a->periodic_values[off + r % p];
        off += p;
    }
    return m;
}

/* PeriodicPolys::eval_at (p3-miden-lifted-stark/src/verifier/periodic.rs:31-80):
 * coefficients by an inverse DFT on the subgroup of order p, evaluated at
 * z^(max_trace_height / p) by Horner. */
void or_sym_periodic_at(const or_sym_air *a, size_t max_trace_height, or_ef z, or_ef *out) {
    size_t off = 0;
    for (uint32_t c = 0; c < a->num_periodic; c++) {
        size_t p = a->periodic_lengths[c];
        unsigned lp = or_log2(p);
        uint64_t winv = or_inv(or_root(lp)), pinv = or_inv((uint64_t)p % OR_P);
        or_ef y = or_ef_pow(z, max_trace_height / p), acc = or_ef_from(0);
        for (size_t k = p; k-- > 0;) {
            uint64_t s = 0;
            for (size_t j = 0; j < p; j++) s = or_add(s, or_mul(a->periodic_values[off + j], or_pow(winv, (j * k) % p)));
            acc = or_ef_add(or_ef_mul(acc, y), or_ef_from(or_mul(s, pinv)));
        }
        out[c] = acc;
        off += p;
    }
}
