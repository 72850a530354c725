"""Stage-by-stage parity of the CUDA kernels against the CPU oracle
(bit-exact: all arithmetic is exact modular integer arithmetic)."""
import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu
P = O.P


def rand_mat(rng, h, w):
    return rng.integers(0, P, size=(h, w), dtype=np.uint64)


@pytest.mark.parametrize("log_h,w,log_blowup", [(0, 3, 1), (1, 1, 1), (3, 5, 2), (6, 9, 1), (10, 33, 1),
                                                (11, 2, 3), (12, 64, 3), (13, 17, 1), (21, 3, 1),
                                                # the headline trace's kernel instances (2^18 rows: two
                                                # 9-bit ranges, 8-column tiles, blowup 2) and the lifted
                                                # workload's tallest trace (2^20 rows, blowup 8)
                                                (18, 16, 1), (20, 8, 3)])
def test_coset_lde_matches_oracle(product, gpu_ctx, log_h, w, log_blowup):
    rng = np.random.default_rng(log_h * 100 + w)
    t = rand_mat(rng, 1 << log_h, w)
    shift = int(rng.integers(1, P, dtype=np.uint64))
    want = O.coset_lde_bitrev(t, log_blowup, shift)
    got = product.to_host(product.coset_lde(gpu_ctx, product.to_device(t), log_blowup, shift))
    assert got.shape == want.shape
    assert np.array_equal(got, want)


def test_poseidon2_params_match_oracle(product):
    pp = O.default_p2()
    assert np.array_equal(product.default_poseidon2_params(), O.p2_to_array(pp))


def test_poseidon2_permutation_matches_oracle(product, gpu_ctx):
    pp = O.default_p2()
    rng = np.random.default_rng(5)
    st = rng.integers(0, P, size=(300, 12), dtype=np.uint64)
    st[0] = 0
    st[1] = P - 1  # every word at the top of the field: exercises every wrap
    st[2, ::2] = P - 1
    st[3] = np.arange(12, dtype=np.uint64) * np.uint64(0xFFFFFFFF)
    want = np.stack([O.permute(pp, s) for s in st])
    got = product.to_host(product.poseidon2_permute_batch(gpu_ctx, product.to_device(st)))
    assert np.array_equal(got, want)


SCENARIOS = [
    [(1, 1)], [(1, 7)], [(2, 3), (4, 5), (8, 8)],
    [(1, 5), (1, 3), (2, 7), (4, 1), (8, 9)],
    [(4, 7), (8, 8), (16, 11)], [(8, 13), (16, 25)],
    [(1, 16), (4, 15), (8, 16), (16, 22)],
    [(4, 7), (4, 8), (8, 11), (8, 16)], [(16, 7)],
    [(1024, 3), (4096, 20), (1 << 15, 9)],
]


@pytest.mark.parametrize("scenario", range(len(SCENARIOS)))
@pytest.mark.parametrize("alignment", [1, 8])
def test_lmcs_tree_matches_oracle(product, gpu_ctx, scenario, alignment):
    """Matrix scenarios of p3-miden-dev-utils/src/fixtures.rs:54-81 (rate 8)."""
    rng = np.random.default_rng(scenario)
    mats = [rand_mat(rng, h, w) for h, w in SCENARIOS[scenario]]
    pp = O.default_p2()
    ot = O.OracleTree(pp, mats, alignment)
    gt = product.LmcsTree(gpu_ctx, [product.to_device(m) for m in mats], alignment)
    assert np.array_equal(gt.root(), ot.root())
    for l in range(gt.depth + 1):
        assert np.array_equal(gt.layer(l), ot.layer(l))


@pytest.mark.parametrize("n_perms,log_h", [(0, 0), (1, 5), (5, 7), (10, 8), (42, 10), (2730, 16)])
def test_keccak_trace_device_matches_host(product, gpu_ctx, n_perms, log_h):
    """Device generate_trace_rows equals the host generator bit for bit,
    including truncated last permutations and zero padding permutations."""
    import torch
    inputs = product.keccak_inputs(9, n_perms)
    host = np.zeros((1 << log_h, product.KECCAK_NUM_COLS), dtype=np.uint64)
    product.lib().p3g_keccak_trace(inputs.ctypes.data_as(product.u64p) if n_perms else None, n_perms, log_h,
                                   host.ctypes.data_as(product.u64p))
    d_in = product.to_device(inputs.reshape(-1, 25)) if n_perms else torch.empty((0, 25), dtype=torch.int64,
                                                                                  device="cuda:0")
    dev = product.generate_keccak_trace_device(gpu_ctx, d_in, log_h)
    assert np.array_equal(product.to_host(dev), host)


@pytest.mark.parametrize("scenario", [0, 2, 3, 6, 9])
@pytest.mark.parametrize("alignment", [1, 8])
@pytest.mark.parametrize("salt_w", [0, 1, 4, 9])
def test_lmcs_prove_batch_and_hiding_match_oracle(product, gpu_ctx, scenario, alignment, salt_w):
    """LmcsTree::prove_batch hints (rows padded to the alignment, then the
    siblings) and the hiding LMCS (a per-leaf salt absorbed last, hinted
    unpadded after the rows) equal the oracle's."""
    rng = np.random.default_rng(100 + scenario)
    mats = [rand_mat(rng, h, w) for h, w in SCENARIOS[scenario]]
    H = mats[-1].shape[0]
    salt = rand_mat(rng, H, salt_w) if salt_w else None
    pp = O.default_p2()
    ot = O.OracleTree(pp, mats, alignment, salt)
    gt = product.LmcsTree(gpu_ctx, [product.to_device(m) for m in mats], alignment,
                          product.to_device(salt) if salt_w else None)
    assert np.array_equal(gt.root(), ot.root())
    for l in range(gt.depth + 1):
        assert np.array_equal(gt.layer(l), ot.layer(l))
    idx = sorted(set(rng.integers(0, H, size=min(H, 13)).tolist()))
    fg, cg = gt.prove_batch(idx)
    fo, co = ot.prove_batch(idx)
    assert np.array_equal(fg, fo) and np.array_equal(cg, co)


@pytest.mark.parametrize("salt_w", [0, 4])
@pytest.mark.parametrize("alignment", [1, 8])
def test_lmcs_open_batch_roundtrip(product, gpu_ctx, salt_w, alignment):
    """Lmcs::open_batch on the device (p3g_lmcs_open_batch) accepts the hints
    of prove_batch, for plain and hiding trees (the hiding round trip of
    p3-miden-lmcs/src/tests.rs:203-221), and rejects changed rows, salts,
    siblings and commitments and truncated or extended hints."""
    rng = np.random.default_rng(7 + salt_w + alignment)
    mats = [rand_mat(rng, h, w) for h, w in [(4, 3), (8, 5), (16, 9)]]
    salt = rand_mat(rng, 16, salt_w) if salt_w else None
    gt = product.LmcsTree(gpu_ctx, [product.to_device(m) for m in mats], alignment,
                          product.to_device(salt) if salt_w else None)
    for idx in ([1, 3, 5], [0, 15], list(range(16)), [7]):
        f, c = gt.prove_batch(idx)
        assert gt.open_batch(idx, f, c) == 0
        f2 = f.copy()
        f2[-1] = (int(f2[-1]) + 1) % O.P  # the last index's salt, or its last row word
        assert product.VERDICTS[gt.open_batch(idx, f2, c)] == "root"
        if len(c):
            c2 = c.copy()
            c2[0, 0] = (int(c2[0, 0]) + 1) % O.P
            assert product.VERDICTS[gt.open_batch(idx, f, c2)] == "root"
        assert product.VERDICTS[gt.open_batch(idx, f, c, commitment=gt.root() ^ np.uint64(1))] == "root"
        assert gt.open_batch(idx, f[:-1], c) != 0
        assert product.VERDICTS[gt.open_batch(idx, np.append(f, np.uint64(0)), c)] == "transcript"
    # different salts, different commitments (tests.rs:223-238)
    if salt_w:
        other = product.LmcsTree(gpu_ctx, [product.to_device(m) for m in mats], alignment,
                                 product.to_device(rand_mat(rng, 16, salt_w)))
        assert not np.array_equal(other.root(), gt.root())


def _bitrev(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


@pytest.mark.parametrize("log_h,log_blowup,periods", [(6, 1, [1, 2, 4, 8]), (6, 3, [4, 2]), (3, 2, [8, 1]),
                                                      (5, 2, [1])])
def test_periodic_lde_matches_full_lde(product, gpu_ctx, log_h, log_blowup, periods):
    """PeriodicLde (p3-miden-lifted-stark/src/prover/periodic.rs; its own test
    assert_periodic_lde_matches_full): row i of the full coset LDE of the
    columns repeated to the trace height equals row i mod the periodic LDE's
    height, in natural order."""
    rng = np.random.default_rng(log_h * 10 + log_blowup)
    cols = [rng.integers(0, O.P, size=p, dtype=np.uint64) for p in periods]
    max_p = max(periods)
    repeated = np.array([[c[r % len(c)] for c in cols] for r in range(max_p)], dtype=np.uint64)
    h = 1 << log_h
    full = np.array([[c[i % len(c)] for c in cols] for i in range(h)], dtype=np.uint64)
    per = product.to_host(product.periodic_lde(gpu_ctx, product.to_device(repeated), log_blowup, log_h, 7))
    assert per.shape == (max_p << log_blowup, len(periods))
    brev = product.to_host(product.coset_lde(gpu_ctx, product.to_device(full), log_blowup, 7))
    L = log_h + log_blowup
    nat = brev[[_bitrev(i, L) for i in range(h << log_blowup)]]
    for i in range(h << log_blowup):
        assert np.array_equal(nat[i], per[i % per.shape[0]]), i


@pytest.mark.parametrize("log_h,log_blowup,periods,shift", [(6, 1, [1, 2, 4, 8], 7), (10, 3, [16, 4], 7),
                                                            (8, 2, [64, 1, 32], 11), (4, 1, [1], 7)])
def test_periodic_lde_matches_oracle(product, gpu_ctx, log_h, log_blowup, periods, shift):
    """p3g_periodic_lde against the oracle's NaiveDft restatement of
    PeriodicLde::build (periodic.rs:49-81), bit for bit."""
    rng = np.random.default_rng(log_h * 7 + sum(periods))
    cols = [rng.integers(0, O.P, size=p, dtype=np.uint64) for p in periods]
    max_p = max(periods)
    repeated = np.array([[c[r % len(c)] for c in cols] for r in range(max_p)], dtype=np.uint64)
    got = product.to_host(product.periodic_lde(gpu_ctx, product.to_device(repeated), log_blowup, log_h, shift))
    want = O.periodic_lde(repeated, log_blowup, log_h, shift)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("log_h,w", [(1, 1), (4, 1), (8, 3), (10, 64), (12, 1024), (16, 2), (6, 3000)])
def test_cubic_trace_device_matches_host(product, gpu_ctx, log_h, w):
    """The cubic AIR's forward iteration on the device equals the host
    generator (k and every row), including widths above one block's threads."""
    k_d, t_d = product.generate_cubic_trace_device(gpu_ctx, log_h, w, 40 + w)
    k_h, t_h = O.cubic_trace(log_h, w, 40 + w)
    assert np.array_equal(k_d, k_h)
    assert np.array_equal(product.to_host(t_d), t_h)


def test_proof_from_device_cubic_trace(product, gpu_ctx):
    k, t = product.generate_cubic_trace_device(gpu_ctx, 10, 16, 9)
    pcs = product.PcsParams(3, 2, 0, 6, 0, 20, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_CUBIC, t, k)])
    kh, th = O.cubic_trace(10, 16, 9)
    orc = O.prove(O.default_p2(), dict(log_blowup=3, log_folding_arity=2, log_final_degree=0, folding_pow_bits=6,
                                       deep_pow_bits=0, num_queries=20, query_pow_bits=0), [(O.AIR_CUBIC, th, kh)])
    assert np.array_equal(gpu.proof.fields, orc["fields"]) and np.array_equal(gpu.digest, orc["digest"])


@pytest.mark.parametrize("split", [(6, 6), (4, 8), (10, 2), (3, 3, 3, 3), (2, 10)])
def test_lde_split_does_not_change_values(product, gpu_ctx, split):
    """Any split of the transform's bits into passes computes the same LDE
    (the autotuner only changes the time)."""
    rng = np.random.default_rng(sum(split))
    t = rand_mat(rng, 1 << 12, 24)
    want = O.coset_lde_bitrev(t, 2, 7)
    gpu_ctx.set_lde_split(12, list(split))
    try:
        got = product.to_host(product.coset_lde(gpu_ctx, product.to_device(t), 2, 7))
    finally:
        gpu_ctx.set_lde_split(12, [])
    assert np.array_equal(got, want)


def test_autotuner_keeps_a_valid_split(product, gpu_ctx):
    r = gpu_ctx.autotune_lde(14, 16, 1, 1)
    assert sum(r["split"]) == 14 and all(1 <= k <= 10 for k in r["split"]) and r["ms"] <= r["default_ms"] + 1e-9
    rng = np.random.default_rng(3)
    t = rand_mat(rng, 1 << 14, 16)
    try:
        got = product.to_host(product.coset_lde(gpu_ctx, product.to_device(t), 1, 7))
    finally:
        gpu_ctx.set_lde_split(14, [])
    assert np.array_equal(got, O.coset_lde_bitrev(t, 1, 7))
    s = gpu_ctx.autotune_slabs(12, 64, 1, 1)
    assert s["slab_cols"] % 8 == 0
    gpu_ctx.set_slab_columns(0)
    with pytest.raises(product.P3gError):
        gpu_ctx.set_lde_split(12, [11, 1])
