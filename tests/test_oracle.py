"""CPU checks of the oracle itself: arithmetic, DFT definition, Keccak-f
against SHA3 (hashlib), constraint vanishing on generated traces, the
sponge padding rule (field_sponge.rs:196-267) and challenger semantics."""
import hashlib
import random

import numpy as np
import pytest

import oracle_ffi as O

P = O.P
L = O.lib()


def test_mul_matches_exact_remainder():
    r = random.Random(1)
    cases = [(P - 1, P - 1), (0, P - 1), (2**64 - 2**32, 2**32), (1, 1)]
    cases += [(r.randrange(P), r.randrange(P)) for _ in range(20000)]
    for a, b in cases:
        assert L.or_x_mul(a, b) == (a * b) % P


def test_extension_field():
    r = random.Random(2)
    for _ in range(200):
        a = [r.randrange(P), r.randrange(P)]
        b = [r.randrange(P), r.randrange(P)]
        out = (O.C.c_uint64 * 2)()
        L.or_x_ef_mul((O.C.c_uint64 * 2)(*a), (O.C.c_uint64 * 2)(*b), out)
        assert out[0] == (a[0] * b[0] + 7 * a[1] * b[1]) % P
        assert out[1] == (a[0] * b[1] + a[1] * b[0]) % P
        inv = (O.C.c_uint64 * 2)()
        L.or_x_ef_inv((O.C.c_uint64 * 2)(*a), inv)
        one = (O.C.c_uint64 * 2)()
        L.or_x_ef_mul((O.C.c_uint64 * 2)(*a), inv, one)
        assert list(one) == [1, 0]


def test_two_adic_roots():
    assert L.or_x_root(32) == 0x185629DCDA58878C
    for k in range(1, 33):
        w = L.or_x_root(k)
        assert pow(w, 2**k, P) == 1 and pow(w, 2 ** (k - 1), P) == P - 1
    assert L.or_x_root(2) == 2**48  # w_4 = 2^48


def test_ntt_definition_and_inverse():
    r = random.Random(3)
    for n in (1, 2, 8, 32):
        a = np.array([r.randrange(P) for _ in range(n)], dtype=np.uint64)
        b = a.copy()
        L.or_ntt(O.ptr(b), n)
        w = L.or_x_root(n.bit_length() - 1)
        for i in range(n):
            assert int(b[i]) == sum(int(a[k]) * pow(w, i * k, P) for k in range(n)) % P
        L.or_intt(O.ptr(b), n)
        assert np.array_equal(a, b)


def test_coset_lde_is_evaluation_on_coset():
    r = np.random.default_rng(4)
    h, w, lb = 8, 3, 2
    t = r.integers(0, P, size=(h, w), dtype=np.uint64)
    shift = 7
    lde = O.coset_lde_bitrev(t, lb, shift)
    # interpolate column 0 on H, evaluate at shift * w_{hB}^i
    c = t[:, 0].copy()
    L.or_intt(O.ptr(c), h)
    wn = L.or_x_root(5)
    for i in range(h << lb):
        x = shift * pow(wn, i, P) % P
        v = sum(int(c[k]) * pow(x, k, P) for k in range(h)) % P
        row = int("{:05b}".format(i)[::-1], 2)
        assert int(lde[row, 0]) == v


def test_keccak_rounds_match_sha3():
    st = np.zeros((1, 25), dtype=np.uint64)
    st[0, 0] = 0x06
    st[0, 16] = 0x8000000000000000
    t = O.keccak_trace(st, 5)
    row = t[23]

    def lane(x, y):
        base = 2629 if (x, y) == (0, 0) else 2465 + (y * 5 + x) * 4
        return sum(int(row[base + l]) << (16 * l) for l in range(4))

    out = b"".join(lane(i % 5, i // 5).to_bytes(8, "little") for i in range(4))
    assert out == hashlib.sha3_256(b"").digest()


def test_keccak_trace_satisfies_constraints():
    inp = O.keccak_inputs(1, 42)
    t = O.keccak_trace(inp, 10)
    assert t.shape == (1024, 2633)
    assert O.check_constraints(O.AIR_KECCAK, t) == 0
    assert L.or_air_num_constraints(O.AIR_KECCAK, 2633) == 3182
    bad = t.copy()
    bad[5, 300] ^= 1  # flip a c bit
    assert O.check_constraints(O.AIR_KECCAK, bad) != 0


def test_cubic_trace_satisfies_constraints():
    k, t = O.cubic_trace(7, 16, 11)
    assert O.check_constraints(O.AIR_CUBIC, t, k) == 0
    t[3, 2] = (int(t[3, 2]) + 1) % P
    assert O.check_constraints(O.AIR_CUBIC, t, k) != 0


def test_sponge_zero_padding_equivalence():
    pp = O.default_p2()
    for n in range(1, 25):
        x = np.arange(1, n + 1, dtype=np.uint64)
        pad = np.concatenate([x, np.zeros((-n) % 8, dtype=np.uint64)])
        s1 = np.zeros(12, dtype=np.uint64)
        s2 = np.zeros(12, dtype=np.uint64)
        L.or_sponge_absorb(O.C.byref(pp), O.ptr(s1), O.ptr(x), n)
        L.or_sponge_absorb(O.C.byref(pp), O.ptr(s2), O.ptr(pad), len(pad))
        assert np.array_equal(s1, s2)
    s = np.zeros(12, dtype=np.uint64)
    L.or_sponge_absorb(O.C.byref(pp), O.ptr(s), O.ptr(np.zeros(1, np.uint64)), 0)
    assert not s.any()  # empty input is a no-op


def test_challenger_sampling_order():
    pp = O.default_p2()
    ch = O.Challenger()
    L.or_ch_init(O.C.byref(ch), O.C.byref(pp))
    for v in (1, 2, 3):
        L.or_ch_observe(O.C.byref(ch), v)
    s = [L.or_ch_sample(O.C.byref(ch)) for _ in range(9)]
    st = np.zeros(12, dtype=np.uint64)
    st[:3] = [1, 2, 3]
    st = O.permute(pp, st)
    # outputs pop from the end of the rate; a fresh duplex after 8 samples
    assert s[:8] == [int(st[i]) for i in range(7, -1, -1)]
    st2 = O.permute(pp, st)
    assert s[8] == int(st2[7])


def test_grind_finds_smallest_witness():
    pp = O.default_p2()
    ch = O.Challenger()
    L.or_ch_init(O.C.byref(ch), O.C.byref(pp))
    L.or_ch_observe(O.C.byref(ch), 42)
    bits = 6
    base = O.Challenger.from_buffer_copy(ch)
    w = L.or_ch_grind(O.C.byref(ch), bits)
    for cand in range(w + 1):
        t = O.Challenger.from_buffer_copy(base)
        L.or_ch_observe(O.C.byref(t), cand)
        ok = L.or_ch_sample_bits(O.C.byref(t), bits) == 0
        assert ok == (cand == w)
    assert L.or_ch_grind(O.C.byref(O.Challenger.from_buffer_copy(base)), 0) == 0


def test_oracle_prove_is_deterministic():
    pp = O.default_p2()
    k, t = O.cubic_trace(5, 8, 3)
    pcs = dict(log_blowup=1, log_folding_arity=1, log_final_degree=0, folding_pow_bits=2,
               deep_pow_bits=0, num_queries=4, query_pow_bits=0)
    a = O.prove(pp, pcs, [(O.AIR_CUBIC, t, k)])
    b = O.prove(pp, pcs, [(O.AIR_CUBIC, t, k)])
    assert np.array_equal(a["fields"], b["fields"]) and np.array_equal(a["commits"], b["commits"])
    assert np.array_equal(a["digest"], b["digest"])


# ----------------------------------------------------------- verifier
def _prove_and_meta(pcs, insts):
    pp = O.default_p2()
    pr = O.prove(pp, pcs, insts)
    meta = [(a, t.shape[0], t.shape[1], k) for a, t, k in insts]
    return pp, pr, meta


BASE_PCS = dict(log_blowup=1, log_folding_arity=1, log_final_degree=0, folding_pow_bits=4, deep_pow_bits=0,
                num_queries=20, query_pow_bits=0)


@pytest.mark.parametrize("log_a,log_b", [(1, 1), (2, 2), (3, 3), (1, 3), (3, 1)])
def test_verifier_accepts_oracle_proofs(log_a, log_b):
    """verify_multi restatement (verifier/mod.rs:170-364) accepts the oracle
    prover's proofs across FRI arities and blowups."""
    k, t = O.cubic_trace(6, 9, 3)
    pcs = dict(BASE_PCS, log_folding_arity=log_a, log_blowup=log_b)
    pp, pr, meta = _prove_and_meta(pcs, [(O.AIR_CUBIC, t, k)])
    assert O.verify(pp, pcs, meta, pr["fields"], pr["commits"], pr["digest"]) == 0


def test_verifier_accepts_lifted_keccak_and_pow():
    ins = []
    for lh, w, s in [(3, 20, 1), (5, 9, 2), (7, 5, 3)]:
        kk, tt = O.cubic_trace(lh, w, s)
        ins.append((O.AIR_CUBIC, tt, kk))
    pcs = dict(BASE_PCS, log_blowup=2, log_folding_arity=2, log_final_degree=2, deep_pow_bits=3, query_pow_bits=5)
    pp, pr, meta = _prove_and_meta(pcs, ins)
    assert O.verify(pp, pcs, meta, pr["fields"], pr["commits"], pr["digest"]) == 0
    t = O.keccak_trace(O.keccak_inputs(1, 5), 7)
    pp, pr, meta = _prove_and_meta(BASE_PCS, [(O.AIR_KECCAK, t, None)])
    assert O.verify(pp, BASE_PCS, meta, pr["fields"], pr["commits"], pr["digest"]) == 0


def test_verifier_rejects_tampering():
    """Any changed field, commitment or digest, a truncated transcript, or a
    wrong statement (other AIR constants) is rejected."""
    k, t = O.cubic_trace(6, 9, 3)
    pcs = dict(BASE_PCS, folding_pow_bits=0, log_blowup=2, log_folding_arity=2)
    pp, pr, meta = _prove_and_meta(pcs, [(O.AIR_CUBIC, t, k)])
    f, c, d = pr["fields"], pr["commits"], pr["digest"]
    n = len(f)
    for i in [0, 1, 7, n // 4, n // 2, n - 2, n - 1]:
        g = f.copy()
        g[i] = (int(g[i]) + 1) % (2**64 - 2**32 + 1)
        assert O.verify(pp, pcs, meta, g, c, d) != 0, i
    for i in range(len(c)):
        cc = c.copy()
        cc[i][0] ^= 1
        assert O.verify(pp, pcs, meta, f, cc, d) != 0, i
    dd = d.copy()
    dd[3] ^= 1
    assert O.verify(pp, pcs, meta, f, c, dd) == 10
    assert O.verify(pp, pcs, meta, f[:-1], c, d) != 0
    k2 = k.copy()
    k2[0] = (int(k2[0]) + 1) % (2**64 - 2**32 + 1)
    assert O.verify(pp, pcs, [(O.AIR_CUBIC, t.shape[0], t.shape[1], k2)], f, c, d) == 8  # quotient identity


def test_hiding_tree_is_one_more_absorb():
    """Hiding LMCS (p3-miden-lmcs/src/lifted_tree.rs:271-279): the salt row is
    one more absorb call per leaf, so the root equals the plain tree's over
    the matrices plus the salt as a last full-height matrix; the salt is
    hinted unpadded after each index's rows."""
    rng = np.random.default_rng(4)
    pp = O.default_p2()
    mats = [rng.integers(0, O.P, size=(h, w), dtype=np.uint64) for h, w in [(4, 7), (8, 8), (16, 11)]]
    salt = rng.integers(0, O.P, size=(16, 5), dtype=np.uint64)
    hid = O.OracleTree(pp, mats, 8, salt)
    assert np.array_equal(hid.root(), O.OracleTree(pp, mats + [salt], 1).root())
    assert not np.array_equal(hid.root(), O.OracleTree(pp, mats, 8).root())
    f, c = hid.prove_batch([3, 9])
    assert f.size == 2 * (8 + 8 + 16 + 5)
    assert np.array_equal(f[8 + 8 + 16:8 + 8 + 16 + 5], salt[3])


def test_deep_evals_are_polynomial_evaluations():
    """The oracle's batch_eval_lifted restatement returns p(z) for the
    polynomial p interpolating each trace column on the trace domain, also
    for a lifted (shorter) matrix, which reads z^(lift ratio)."""
    import sym_airs as S
    rng = np.random.default_rng(3)
    lb = 2
    t_small, t_big = rng.integers(0, O.P, size=(8, 2), dtype=np.uint64), rng.integers(0, O.P, size=(32, 3), dtype=np.uint64)
    mats = [O.coset_lde_bitrev(t_small, lb, pow(7, 4, O.P)), O.coset_lde_bitrev(t_big, lb, 7)]
    z = (int(rng.integers(0, O.P, dtype=np.uint64)), int(rng.integers(0, O.P, dtype=np.uint64)))
    w = pow(7, (O.P - 1) // 32, O.P)
    zs = [z, (z[0] * w % O.P, z[1] * w % O.P)]
    ev = O.deep_evals(mats, lb, zs)

    def ef_pow(a, e):
        r = (1, 0)
        while e:
            if e & 1:
                r = S.ef_mul(r, a)
            a = S.ef_mul(a, a)
            e >>= 1
        return r

    def poly_at(col, x):
        c = np.ascontiguousarray(col, dtype=np.uint64).copy()
        O.lib().or_intt(O.ptr(c), c.size)
        acc = (0, 0)
        for k in reversed(range(c.size)):
            acc = S.ef_add(S.ef_mul(acc, x), (int(c[k]), 0))
        return acc

    k = 0
    for t, ratio in ((t_small, 4), (t_big, 1)):
        for col in range(t.shape[1]):
            for j in range(2):
                assert tuple(int(v) for v in ev[k, j]) == poly_at(t[:, col], ef_pow(zs[j], ratio)), (k, j)
            k += 1
