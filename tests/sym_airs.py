"""AIRs of the reference's own tests and examples, written against the
symbolic AirBuilder (p3_miden_b200.symbolic), with their trace and aux
builders, for the symbolic-AIR parity tests. Arithmetic here is plain Python
integers (Goldilocks and its quadratic extension F[x]/(x^2 - 7))."""
from __future__ import annotations

import numpy as np

P = 0xFFFFFFFF00000001
W = 7


def ef_mul(a, b):
    return ((a[0] * b[0] + W * a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def ef_add(a, b):
    return ((a[0] + b[0]) % P, (a[1] + b[1]) % P)


def ef_inv(a):
    n = (a[0] * a[0] - W * a[1] * a[1]) % P
    ni = pow(n, P - 2, P)
    return (a[0] * ni % P, (P - a[1]) * ni % P)


# ------------------------------------------------------------------ cubic
def cubic_eval(k):
    """The cubic synthetic AIR: c_i[r+1] = c_i[r]^3 + c_{(i+1) mod w}[r] + k_i
    on every row but the last, one constraint per column in column order."""
    def ev(b):
        local, nxt = b.main()
        w = len(local)
        for i in range(w):
            b.when_transition().assert_eq(nxt[i], local[i] * local[i] * local[i] + local[(i + 1) % w] + int(k[i]))
    return ev


# ------------------------------------------------------------------- tiny
def tiny_eval(b):
    """TinyAir (p3-miden-lifted-stark/tests/tiny_air.rs:60-110): main[0]
    starts at public value 0 and is raised to the 4th power each row; every
    periodic column reads 1 on the first and the last row; the aux column
    starts at the challenge and is raised to the 4th power each row."""
    local, nxt = b.main()
    start = b.public_values()[0]
    b.when_first_row().assert_eq(local[0], start)
    b.when_transition().assert_eq(nxt[0], local[0].exp_power_of_2(2))
    for p in b.periodic_values():
        b.when_first_row().assert_one(p)
        b.when_last_row().assert_one(p)
    aux_l, aux_n = b.permutation()
    ch = b.permutation_randomness()[0]
    b.when_first_row().assert_eq_ext(aux_l[0], ch)
    b.when_transition().assert_eq_ext(aux_n[0], aux_l[0].exp_power_of_2(2))


def tiny_periodic(periods):
    cols = []
    for p in periods:
        c = [0] * p
        c[0] = 1
        c[p - 1] = 1
        cols.append(c)
    return cols


def tiny_trace(start: int, height: int) -> np.ndarray:
    v, out = start % P, []
    for _ in range(height):
        out.append(v)
        v = pow(v, 4, P)
    return np.array(out, dtype=np.uint64).reshape(-1, 1)


def tiny_aux(instance, randomness, height):
    """TinyAuxBuilder: aux column challenge^(4^row); aux value = the last row."""
    cur, rows = randomness[0], []
    for _ in range(height):
        rows.append(cur)
        cur = ef_mul(cur, cur)
        cur = ef_mul(cur, cur)
    aux = np.array(rows, dtype=np.uint64).reshape(height, 2)
    return aux, np.array(rows[-1], dtype=np.uint64)


# -------------------------------------------------------------------- bus
def bus_eval(b):
    """BusTestAir (p3-miden-lifted-stark/tests/bus_test.rs:92-150): a
    power-of-4 chain, and two constant aux columns tied to the challenges,
    the public values and the aux values."""
    pv0, pv1, pv2 = b.public_values()
    local, nxt = b.main()
    b.when_first_row().assert_eq(local[0], pv0)
    b.when_transition().assert_eq(nxt[0], local[0].exp_power_of_2(2))
    c0, c1 = b.permutation_randomness()
    av0, av1 = b.permutation_values()
    aux_l, aux_n = b.permutation()
    b.when_first_row().assert_eq_ext(aux_l[0] * (pv1 + c0), 1)
    b.when_first_row().assert_eq_ext(aux_l[1], pv2 + c1)
    b.when_transition().assert_eq_ext(aux_n[0], aux_l[0])
    b.when_transition().assert_eq_ext(aux_n[1], aux_l[1])
    b.when_last_row().assert_eq_ext(aux_l[0], av0)
    b.when_last_row().assert_eq_ext(aux_l[1], av1)


def bus_aux(pi0, pi1):
    """BusTestAuxBuilder: col 0 = 1/(pi_0 + c0), col 1 = pi_1 + c1 on every
    row; the aux values are those two constants."""
    def build(instance, randomness, height):
        v0 = ef_inv(ef_add((pi0, 0), randomness[0]))
        v1 = ef_add((pi1, 0), randomness[1])
        aux = np.tile(np.array([v0[0], v0[1], v1[0], v1[1]], dtype=np.uint64), (height, 1))
        return aux, np.array([v0[0], v0[1], v1[0], v1[1]], dtype=np.uint64)
    return build


# ------------------------------------------------------------ miden dummy
def miden_eval(b):
    """DummyMidenAir (p3-miden-lifted-examples/src/miden.rs:57-62): the
    product of the first nine main columns is zero (degree 9: eight
    quotient chunks)."""
    local, _ = b.main()
    prod = local[0]
    for j in range(1, 9):
        prod = prod * local[j]
    b.assert_zero(prod)


def miden_trace(width: int, log_h: int, seed: int) -> np.ndarray:
    """Column 0 zero, the other columns seeded uniform (generate_dummy_trace)."""
    rng = np.random.default_rng(seed)
    t = rng.integers(0, P, size=(1 << log_h, width), dtype=np.uint64)
    t[:, 0] = 0
    return t


# ---------------------------------------------------------------- chains
def chains_eval(b):
    """Linear chains for the code generator's rewrites: a 60-step Horner chain
    over differences (its 96-bit accumulation reaches the 2^95 bound and is
    closed and restarted), the XOR form a + b - (c + c), a negation inside a
    chain and a product read only by a product; column 7 holds their
    combination."""
    L, _ = b.main()
    acc = b.const(0)
    for k in range(60):
        acc = acc + acc + (L[k % 7] - L[(k + 2) % 7])
    prod = L[0] * L[1]
    x = L[0] + L[1] - (prod + prod)
    y = -(L[2] - L[3]) + L[4] + L[4]
    z = (L[5] * L[6]) * L[5]  # a product read only by a product
    b.assert_zero(L[7] - acc - x * y - z)


def chains_trace(log_h: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = rng.integers(0, P, size=(1 << log_h, 8), dtype=np.uint64)
    for r in range(1 << log_h):
        c = [int(v) for v in t[r, :7]]
        acc = 0
        for k in range(60):
            acc = (2 * acc + c[k % 7] - c[(k + 2) % 7]) % P
        x = (c[0] + c[1] - 2 * c[0] * c[1]) % P
        y = (-(c[2] - c[3]) + 2 * c[4]) % P
        t[r, 7] = (acc + x * y + c[5] * c[6] * c[5]) % P
    return t


# ---------------------------------------------------------------- keccak
# The Keccak AIR's symbolic form is part of the package (p3_miden_b200.airs),
# where the bench also takes it from.
from conftest import load_product as _load_product

_load_product()
from p3_miden_b200.airs import (KC_A, KC_AP, KC_APP, KC_APP00, KC_APPP00, KC_C, KC_CP,  # noqa: E402,F401
                                KC_EXPORT, KC_NCOLS, KC_PRE, KC_STEP, keccak_eval, keccak_tables)
