"""The Keccak-f[1600] AIR written against the symbolic AirBuilder
(p3_miden_b200.symbolic): the AIR of the reference's lifted Keccak example
(p3-miden-lifted-examples/src/bin/lifted_keccak.rs, KeccakAir from the
p3-keccak-air crate), given to the library as a constraint DAG so that its
constraint kernels are generated (p3g_air_create). The same constraints, in the
same emission order, as the built-in AIR (P3G_AIR_KECCAK) and the oracle's
restatement: both produce the same proof.

Usage::

    air = Air(ctx, build_air(keccak_eval, KC_NCOLS))
    prove_multi(ctx, pcs, [AirWitness(air, trace)])
"""
from __future__ import annotations

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
