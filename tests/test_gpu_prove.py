"""Whole-proof parity and acceptance: the GPU prover's transcript (fields,
commitments, digest) is bit-identical to the oracle's on the same traces and
parameters, and the verifier restatement (oracle/or_verify.c) accepts it,
including at the full sizes of the headline and lifted workloads, where only
the (cheap) verifier runs on the CPU."""
import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu


def pcs_dict(p):
    return dict(log_blowup=p.log_blowup, log_folding_arity=p.log_folding_arity,
                log_final_degree=p.log_final_degree, folding_pow_bits=p.folding_pow_bits,
                deep_pow_bits=p.deep_pow_bits, num_queries=p.num_queries, query_pow_bits=p.query_pow_bits)


def check_verifies(gpu, pcs, instances):
    """instances: (air, height, width, consts|None) in ascending height order."""
    rc = O.verify(O.default_p2(), pcs_dict(pcs), instances, gpu.proof.fields, gpu.proof.commitments, gpu.digest)
    assert rc == 0, f"verifier rejected the GPU proof: {O.VERIFY_ERRORS.get(rc, rc)}"


def check_same(gpu, orc):
    assert np.array_equal(gpu.proof.commitments, orc["commits"]), "commitments differ"
    assert len(gpu.proof.fields) == len(orc["fields"])
    diff = np.nonzero(gpu.proof.fields != orc["fields"])[0]
    assert diff.size == 0, f"first differing field at {diff[:5]}"
    assert np.array_equal(gpu.digest, orc["digest"])


@pytest.mark.parametrize("arity", [1, 2, 3])
def test_cubic_single_trace(product, gpu_ctx, arity):
    k, t = O.cubic_trace(8, 12, 21)
    pcs = product.PcsParams(2, arity, 0, 4, 0, 12, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_CUBIC, t, k)])
    orc = O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_CUBIC, t, k)])
    check_same(gpu, orc)
    check_verifies(gpu, pcs, [(O.AIR_CUBIC, t.shape[0], t.shape[1], k)])


def test_cubic_lifted_three_traces(product, gpu_ctx):
    """Lifted multi-trace: three traces of ascending heights in one tree."""
    specs = [(4, 32, 1), (7, 8, 2), (9, 4, 3)]
    inst, oinst = [], []
    for log_h, w, seed in specs:
        k, t = O.cubic_trace(log_h, w, seed)
        inst.append(product.AirWitness(product.AIR_CUBIC, t, k))
        oinst.append((O.AIR_CUBIC, t, k))
    pcs = product.PcsParams(3, 2, 0, 5, 2, 20, 3)
    gpu = product.prove_multi(gpu_ctx, pcs, inst)
    orc = O.prove(O.default_p2(), pcs_dict(pcs), oinst)
    check_same(gpu, orc)
    check_verifies(gpu, pcs, [(a, t.shape[0], t.shape[1], k) for a, t, k in oinst])


def test_keccak_small(product, gpu_ctx):
    inputs = O.keccak_inputs(1, 5)
    t = O.keccak_trace(inputs, 7)
    pcs = product.PcsParams(1, 1, 0, 6, 0, 16, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_KECCAK, t)])
    orc = O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_KECCAK, t, None)])
    check_same(gpu, orc)
    check_verifies(gpu, pcs, [(O.AIR_KECCAK, t.shape[0], t.shape[1], None)])


def test_keccak_42_perms_config(product, gpu_ctx):
    """The CPU-runnable Keccak workload: 42 permutations, 2^10 rows, the
    example's parameters (log_blowup 1, arity 2, final degree 0, folding PoW
    16, 100 queries)."""
    inputs = O.keccak_inputs(1, 42)
    t = O.keccak_trace(inputs, 10)
    pcs = product.PcsParams(1, 1, 0, 16, 0, 100, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_KECCAK, t)])
    orc = O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_KECCAK, t, None)])
    check_same(gpu, orc)
    check_verifies(gpu, pcs, [(O.AIR_KECCAK, t.shape[0], t.shape[1], None)])


def test_keccak_2e13_bit_exact(product, gpu_ctx):
    """341 permutations (8184 rows, padded to 2^13) with the headline's
    parameters: the smallest whole proof whose main tree runs the
    throughput leaf kernel (2^14 leaves, above the cooperative kernel's
    4096) over the slab-carried sponge states, the multi-level compression
    and the two-range LDE; bit-identical to the oracle."""
    inputs = O.keccak_inputs(3, 341)
    t = O.keccak_trace(inputs, 13)
    pcs = product.PcsParams(1, 1, 0, 16, 0, 100, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_KECCAK, t)])
    orc = O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_KECCAK, t, None)])
    check_same(gpu, orc)
    check_verifies(gpu, pcs, [(O.AIR_KECCAK, t.shape[0], t.shape[1], None)])


def test_non_default_poseidon2_table(product, gpu_ctx):
    """The prover is parametric in the 130-word permutation table the
    StarkConfig supplies (configs.rs:215-217): with other round constants
    and a random internal diagonal, GPU and oracle still agree bit for bit,
    and the proof differs from the default table's. A context with the
    default table used afterwards is unaffected."""
    rng = np.random.default_rng(77)
    diag = rng.integers(0, O.P, size=12, dtype=np.uint64)
    table = product.poseidon2_params_from_seed(99, diag)
    pp = O.p2_from_array(table)
    k, t = O.cubic_trace(7, 12, 4)
    k2, t2 = O.cubic_trace(9, 5, 6)
    pcs = product.PcsParams(2, 2, 0, 5, 1, 16, 2)
    inst = [product.AirWitness(product.AIR_CUBIC, t, k), product.AirWitness(product.AIR_CUBIC, t2, k2)]
    oinst = [(O.AIR_CUBIC, t, k), (O.AIR_CUBIC, t2, k2)]
    ctx = product.Context(0, table)
    try:
        gpu = product.prove_multi(ctx, pcs, inst)
        kt = O.keccak_trace(O.keccak_inputs(5, 3), 7)
        pcs_k = product.PcsParams(1, 1, 0, 6, 0, 12, 0)
        gk = product.prove_multi(ctx, pcs_k, [product.AirWitness(product.AIR_KECCAK, kt)])
    finally:
        ctx.close()
    check_same(gpu, O.prove(pp, pcs_dict(pcs), oinst))
    check_same(gk, O.prove(pp, pcs_dict(pcs_k), [(O.AIR_KECCAK, kt, None)]))
    assert O.verify(pp, pcs_dict(pcs), [(a, tt.shape[0], tt.shape[1], kk) for a, tt, kk in oinst],
                    gpu.proof.fields, gpu.proof.commitments, gpu.digest) == 0
    default = product.prove_multi(gpu_ctx, pcs, inst)
    assert not np.array_equal(default.digest, gpu.digest)
    check_same(default, O.prove(O.default_p2(), pcs_dict(pcs), oinst))


def test_device_resident_trace(product, gpu_ctx):
    k, t = O.cubic_trace(6, 8, 5)
    pcs = product.PcsParams(1, 1, 0, 3, 0, 8, 0)
    host = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_CUBIC, t, k)])
    dev = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_CUBIC, product.to_device(t), k)])
    assert np.array_equal(host.proof.fields, dev.proof.fields)
    assert np.array_equal(host.digest, dev.digest)


def test_keccak_headline_2e18_verifies(product, gpu_ctx):
    """The headline workload at full size (10922 permutations, 2^18 x 2633):
    the GPU proof is accepted by the verifier restatement."""
    t = product.generate_keccak_trace(product.keccak_inputs(1, 10922))
    assert t.shape == (1 << 18, 2633)
    pcs = product.PcsParams(1, 1, 0, 16, 0, 100, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_KECCAK, product.to_device(t))])
    check_verifies(gpu, pcs, [(O.AIR_KECCAK, t.shape[0], t.shape[1], None)])
    # a proof for other inputs does not verify against this statement's transcript
    bad = gpu.proof.fields.copy()
    bad[len(bad) // 2] ^= 1
    rc = O.verify(O.default_p2(), pcs_dict(pcs), [(O.AIR_KECCAK, t.shape[0], t.shape[1], None)], bad,
                  gpu.proof.commitments, gpu.digest)
    assert rc != 0
    # the device verifier: accepts the proof, and agrees on the perturbed one
    shapes = [product.AirShape(product.AIR_KECCAK, t.shape[0], t.shape[1])]
    assert product.verify_output(gpu_ctx, pcs, shapes, gpu).ok
    assert product.verify_multi(gpu_ctx, pcs, shapes, bad, gpu.proof.commitments, gpu.digest).verdict == rc


def test_lifted_config_full_size_verifies(product, gpu_ctx):
    """Three cubic-AIR traces 2^12 x 1024, 2^16 x 256, 2^20 x 64 lifted to
    2^20, log_blowup 3, FRI arity 4: accepted by the verifier restatement."""
    inst, meta = [], []
    for i, (lh, w) in enumerate([(12, 1024), (16, 256), (20, 64)]):
        k, t = product.generate_cubic_trace(lh, w, 300 + i)
        inst.append(product.AirWitness(product.AIR_CUBIC, product.to_device(t), k))
        meta.append((O.AIR_CUBIC, t.shape[0], t.shape[1], k))
    pcs = product.PcsParams(3, 2, 0, 16, 0, 100, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, inst)
    check_verifies(gpu, pcs, meta)
    assert product.verify_output(gpu_ctx, pcs, [product.AirShape(*m) for m in meta], gpu).ok
