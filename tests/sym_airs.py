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


# ---------------------------------------------------------------- keccak
# Column layout of the Keccak-f[1600] AIR (2633 columns): step flags (24),
# export, preimage (100 limbs), A (100 limbs), C (320 bits), C' (320 bits),
# A' (1600 bits), A'' (100 limbs), A''[0][0] bits (64), A'''[0][0] (4 limbs).
KC_STEP, KC_EXPORT, KC_PRE, KC_A, KC_C, KC_CP = 0, 24, 25, 125, 225, 545
KC_AP, KC_APP, KC_APP00, KC_APPP00, KC_NCOLS = 865, 2465, 2565, 2629, 2633


def keccak_tables():
    """FIPS 202: rho offsets rot[x][y] by the (t+1)(t+2)/2 walk, round
    constants from the degree-8 LFSR."""
    rot = [[0] * 5 for _ in range(5)]
    x, y = 1, 0
    for t in range(24):
        rot[x][y] = ((t + 1) * (t + 2) // 2) % 64
        x, y = y, (2 * x + 3 * y) % 5

    def rc_bit(t):
        if t % 255 == 0:
            return 1
        r = 1
        for _ in range(t % 255):
            r <<= 1
            if r & 0x100:
                r ^= 0x171
        return r & 1

    rc = []
    for i in range(24):
        v = 0
        for j in range(7):
            if rc_bit(j + 7 * i):
                v |= 1 << ((1 << j) - 1)
        rc.append(v)
    return rot, rc


def keccak_eval(b):
    """The Keccak-f[1600] AIR's 3182 constraints in the emission order the
    oracle's restatement uses (one row per round: step flags, preimage, the
    theta/rho/pi/chi/iota relations bit by bit and limb by limb)."""
    rot, rc = keccak_tables()
    L, N = b.main()
    first, trans = b.is_first_row(), b.is_transition()

    def xor2(p, q):
        return p + q - (p * q + p * q)

    def xor3(p, q, r):
        return xor2(p, xor2(q, r))

    def andn(p, q):
        return (1 - p) * q

    def isbool(p):
        return p * (p - 1)

    b.assert_zero(first * (L[KC_STEP] - 1))
    for i in range(1, 24):
        b.assert_zero(first * L[KC_STEP + i])
    for i in range(24):
        b.assert_zero(trans * (N[KC_STEP + (i + 1) % 24] - L[KC_STEP + i]))
    first_step, not_final = L[KC_STEP], 1 - L[KC_STEP + 23]
    for y in range(5):
        for x in range(5):
            for l in range(4):
                o = (y * 5 + x) * 4 + l
                b.assert_zero(first_step * (L[KC_PRE + o] - L[KC_A + o]))
    b.assert_zero(isbool(L[KC_EXPORT]))
    b.assert_zero(not_final * L[KC_EXPORT])
    for y in range(5):
        for x in range(5):
            for l in range(4):
                o = (y * 5 + x) * 4 + l
                b.assert_zero(not_final * (trans * (L[KC_PRE + o] - N[KC_PRE + o])))
    for x in range(5):
        for z in range(64):
            b.assert_zero(isbool(L[KC_C + x * 64 + z]))
            v = xor3(L[KC_C + x * 64 + z], L[KC_C + ((x + 4) % 5) * 64 + z], L[KC_C + ((x + 1) % 5) * 64 + (z + 63) % 64])
            b.assert_zero(L[KC_CP + x * 64 + z] - v)
    for y in range(5):
        for x in range(5):
            for l in range(4):
                acc = b.const(0)
                for z in range(l * 16 + 15, l * 16 - 1, -1):
                    ap = L[KC_AP + (y * 5 + x) * 64 + z]
                    b.assert_zero(isbool(ap))
                    acc = acc + acc + xor3(ap, L[KC_C + x * 64 + z], L[KC_CP + x * 64 + z])
                b.assert_zero(acc - L[KC_A + (y * 5 + x) * 4 + l])
    for x in range(5):
        for z in range(64):
            s = b.const(0)
            for y in range(5):
                s = s + L[KC_AP + (y * 5 + x) * 64 + z]
            d = s - L[KC_CP + x * 64 + z]
            b.assert_zero(d * (d - 2) * (d - 4))

    def bbit(bx, by, bz):
        ax = (bx + 3 * by) % 5
        return L[KC_AP + (bx * 5 + ax) * 64 + (bz + 64 - rot[ax][bx]) % 64]

    for y in range(5):
        for x in range(5):
            for l in range(4):
                acc = b.const(0)
                for z in range(l * 16 + 15, l * 16 - 1, -1):
                    acc = acc + acc + xor2(bbit(x, y, z), andn(bbit((x + 1) % 5, y, z), bbit((x + 2) % 5, y, z)))
                b.assert_zero(acc - L[KC_APP + (y * 5 + x) * 4 + l])
    for l in range(4):
        acc = b.const(0)
        for z in range(l * 16 + 15, l * 16 - 1, -1):
            b.assert_zero(isbool(L[KC_APP00 + z]))
            acc = acc + acc + L[KC_APP00 + z]
        b.assert_zero(acc - L[KC_APP + l])
    for l in range(4):
        acc = b.const(0)
        for z in range(l * 16 + 15, l * 16 - 1, -1):
            rcb = b.const(0)
            for r in range(24):
                if (rc[r] >> z) & 1:
                    rcb = rcb + L[KC_STEP + r]
            acc = acc + acc + xor2(L[KC_APP00 + z], rcb)
        b.assert_zero(acc - L[KC_APPP00 + l])
    for x in range(5):
        for y in range(5):
            for l in range(4):
                outv = L[KC_APPP00 + l] if (x == 0 and y == 0) else L[KC_APP + (y * 5 + x) * 4 + l]
                b.assert_zero(trans * (not_final * (outv - N[KC_A + (y * 5 + x) * 4 + l])))
