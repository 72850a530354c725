"""Symbolic AIRs on the GPU: proofs made with the generated constraint
kernels (NVRTC, sm_100a) and caller-built aux traces are bit-identical to the
oracle's, and the device verifier accepts them. The AIRs are the reference's
own test and example AIRs (TinyAir, BusTestAir, DummyMidenAir) and the cubic
AIR written symbolically, which must also reproduce the hand-written cubic
kernel's proof."""
import numpy as np
import pytest

import oracle_ffi as O
import sym_airs as S

pytestmark = pytest.mark.gpu


def pcs_dict(p):
    return dict(log_blowup=p.log_blowup, log_folding_arity=p.log_folding_arity,
                log_final_degree=p.log_final_degree, folding_pow_bits=p.folding_pow_bits,
                deep_pow_bits=p.deep_pow_bits, num_queries=p.num_queries, query_pow_bits=p.query_pow_bits)


def check_same(gpu, orc):
    assert np.array_equal(gpu.proof.commitments, orc["commits"]), "commitments differ"
    assert len(gpu.proof.fields) == len(orc["fields"])
    diff = np.nonzero(gpu.proof.fields != orc["fields"])[0]
    assert diff.size == 0, f"first differing field at {diff[:5]}"
    assert np.array_equal(gpu.digest, orc["digest"])


def test_symbolic_cubic_matches_builtin_kernel(product, gpu_ctx):
    k, t = O.cubic_trace(7, 16, 31)
    k2, t2 = O.cubic_trace(9, 8, 32)
    pcs = product.PcsParams(2, 2, 0, 4, 1, 16, 1)
    a1 = product.Air(gpu_ctx, product.build_air(S.cubic_eval(k), 16))
    a2 = product.Air(gpu_ctx, product.build_air(S.cubic_eval(k2), 8))
    assert (a1.log_quotient_degree, a1.max_degree) == (1, 3)
    sym = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(a1, t), product.AirWitness(a2, t2)])
    builtin = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_CUBIC, t, k),
                                                 product.AirWitness(product.AIR_CUBIC, t2, k2)])
    assert np.array_equal(sym.proof.fields, builtin.proof.fields)
    assert np.array_equal(sym.digest, builtin.digest)
    check_same(sym, O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_CUBIC, t, k), (O.AIR_CUBIC, t2, k2)]))
    shapes = [product.AirShape(a1, t.shape[0], 16), product.AirShape(a2, t2.shape[0], 8)]
    assert product.verify_output(gpu_ctx, pcs, shapes, sym).ok


@pytest.mark.parametrize("periods,heights", [((), (8,)), ((4,), (16,)), ((2, 4), (4, 8)),
                                             ((2, 4), (4, 8, 16)), ((8,), (1024, 4096))])
def test_tiny_air_matches_oracle(product, gpu_ctx, periods, heights):
    """TinyAir (tests/tiny_air.rs): periodic columns, an aux trace from a
    caller's AuxBuilder (challenge^(4^row), extension field), an aux value,
    a public value per instance; lifted traces of several heights."""
    desc = product.build_air(S.tiny_eval, 1, num_public_values=1, num_aux_values=1,
                             periodic_columns=S.tiny_periodic(periods))
    air = product.Air(gpu_ctx, desc)
    assert air.log_quotient_degree == 2
    wits, oinst, shapes = [], [], []
    for i, h in enumerate(heights):
        t = S.tiny_trace(i + 2, h)
        pv = np.array([i + 2], dtype=np.uint64)
        wits.append(product.AirWitness(air, t, public_values=pv, aux_builder=S.tiny_aux))
        oinst.append((O.AIR_SYMBOLIC, t, None, {"sym": desc, "public_values": pv, "aux_builder": S.tiny_aux}))
        shapes.append(product.AirShape(air, h, 1, public_values=pv))
    pcs = product.PcsParams(2, 1, 0, 3, 0, 12, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, wits)
    check_same(gpu, O.prove(O.default_p2(), pcs_dict(pcs), oinst))
    assert product.verify_output(gpu_ctx, pcs, shapes, gpu).ok
    bad = gpu.proof.fields.copy()
    bad[3] = (int(bad[3]) + 1) % O.P
    assert not product.verify_multi(gpu_ctx, pcs, shapes, bad, gpu.proof.commitments, gpu.digest).ok


def test_bus_air_matches_oracle(product, gpu_ctx):
    """BusTestAir (tests/bus_test.rs): extension-field constraints on two aux
    columns built from two challenges, three public values, two aux values."""
    desc = product.build_air(S.bus_eval, 1, aux_width=2, num_randomness=2, num_aux_values=2, num_public_values=3)
    air = product.Air(gpu_ctx, desc)
    base, ext = air.layout()
    assert base.size == 2 and ext.size == 6
    pv = np.array([2, 42, 67], dtype=np.uint64)
    t = S.tiny_trace(2, 64)
    pcs = product.PcsParams(2, 2, 0, 4, 0, 20, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(air, t, public_values=pv,
                                                                aux_builder=S.bus_aux(42, 67))])
    extra = {"sym": desc, "public_values": pv, "aux_builder": S.bus_aux(42, 67)}
    check_same(gpu, O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_SYMBOLIC, t, None, extra)]))
    assert product.verify_output(gpu_ctx, pcs, [product.AirShape(air, 64, 1, public_values=pv)], gpu).ok


def test_miden_dummy_air_matches_oracle(product, gpu_ctx):
    """DummyMidenAir (p3-miden-lifted-examples/src/miden.rs): a degree-9
    constraint, eight quotient chunks (log_blowup 3), eight all-zero aux EF
    columns and aux values, two traces of 51 and 20 columns (the example's
    widths) at reduced heights."""
    d1 = product.build_air(S.miden_eval, 51, aux_width=8, num_randomness=2, num_aux_values=8)
    d2 = product.build_air(S.miden_eval, 20, aux_width=8, num_randomness=2, num_aux_values=8)
    a1, a2 = product.Air(gpu_ctx, d1), product.Air(gpu_ctx, d2)
    assert a1.log_quotient_degree == 3
    t1, t2 = S.miden_trace(51, 10, 1), S.miden_trace(20, 11, 2)
    pcs = product.PcsParams(3, 2, 0, 8, 0, 24, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(a1, t1), product.AirWitness(a2, t2)])
    check_same(gpu, O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_SYMBOLIC, t1, None, {"sym": d1}),
                                                               (O.AIR_SYMBOLIC, t2, None, {"sym": d2})]))
    shapes = [product.AirShape(a1, 1 << 10, 51), product.AirShape(a2, 1 << 11, 20)]
    assert product.verify_output(gpu_ctx, pcs, shapes, gpu).ok


def test_mixed_builtin_and_symbolic_instances(product, gpu_ctx):
    """A Keccak instance (hand-written kernel, dummy aux) lifted with a
    TinyAir instance (generated kernel, caller aux) in one proof."""
    desc = product.build_air(S.tiny_eval, 1, num_public_values=1, num_aux_values=1,
                             periodic_columns=S.tiny_periodic((4,)))
    air = product.Air(gpu_ctx, desc)
    tt = S.tiny_trace(5, 64)
    pv = np.array([5], dtype=np.uint64)
    kt = O.keccak_trace(O.keccak_inputs(4, 5), 7)
    pcs = product.PcsParams(2, 1, 0, 4, 0, 16, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(air, tt, public_values=pv, aux_builder=S.tiny_aux),
                                             product.AirWitness(product.AIR_KECCAK, kt)])
    orc = O.prove(O.default_p2(), pcs_dict(pcs), [
        (O.AIR_SYMBOLIC, tt, None, {"sym": desc, "public_values": pv, "aux_builder": S.tiny_aux}),
        (O.AIR_KECCAK, kt, None)])
    check_same(gpu, orc)
    shapes = [product.AirShape(air, 64, 1, public_values=pv), product.AirShape(product.AIR_KECCAK, 128, kt.shape[1])]
    assert product.verify_output(gpu_ctx, pcs, shapes, gpu).ok


def test_symbolic_keccak_generated_kernels(product, gpu_ctx):
    """The Keccak-f[1600] AIR through the generated path: 3182 constraints
    compiled as chunked kernels (NVRTC, one program per group of chunks,
    compiled in parallel), bit-identical to the oracle and to the
    hand-written Keccak kernel's proof."""
    desc = product.build_air(S.keccak_eval, S.KC_NCOLS)
    air = product.Air(gpu_ctx, desc)
    assert air.log_quotient_degree == 1
    t = O.keccak_trace(O.keccak_inputs(1, 42), 10)
    pcs = product.PcsParams(1, 1, 0, 8, 0, 30, 0)
    sym = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(air, t)])
    hand = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(product.AIR_KECCAK, t)])
    assert np.array_equal(sym.proof.fields, hand.proof.fields)
    assert np.array_equal(sym.digest, hand.digest)
    check_same(sym, O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_KECCAK, t, None)]))
    assert product.verify_output(gpu_ctx, pcs, [product.AirShape(air, 1024, S.KC_NCOLS)], sym).ok


def test_symbolic_keccak_2e13_matches_oracle(product, gpu_ctx):
    """The headline's path at 2^13 rows (341 permutations, the example's
    parameters: blowup 2, 100 queries, 16-bit folding PoW): 2^14 leaves run the
    one-thread-per-leaf sponge that also writes the column-major copy the
    generated kernels read, the multi-range LDE, and the 500-node chunk
    kernels over 2^14 points; fields, commitments and digest equal the
    oracle's proof of the same trace."""
    air = product.Air(gpu_ctx, product.build_air(S.keccak_eval, S.KC_NCOLS))
    t = O.keccak_trace(O.keccak_inputs(3, 341), 13)
    pcs = product.PcsParams(1, 1, 0, 16, 0, 100, 0)
    sym = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(air, t)])
    check_same(sym, O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_KECCAK, t, None)]))
    # a device-resident trace and a host trace (slab pipeline) give the same proof
    import torch
    dev = torch.from_numpy(t.view(np.int64)).to("cuda:0")
    again = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(air, dev)])
    assert np.array_equal(again.digest, sym.digest)


def test_chunk_size_does_not_change_the_proof(product):
    """The chunk size of the generated kernels is a launch-shape choice: the
    cubic AIR (w = 24) cut into 16-node chunks (many kernels, each adding its
    part of the fold) gives the built-in kernel's proof. The context's memory
    statistics stay consistent across repeated proofs (large buffers come
    back from the context's cache)."""
    ctx = product.Context(0)
    try:
        ctx.set_air_chunk_nodes(16)
        k, t = O.cubic_trace(12, 24, 77)
        air = product.Air(ctx, product.build_air(S.cubic_eval(k), 24))
        assert air.num_kernels > 4
        pcs = product.PcsParams(1, 1, 0, 8, 0, 30, 0)
        sym = product.prove_multi(ctx, pcs, [product.AirWitness(air, t)])
        builtin = product.prove_multi(ctx, pcs, [product.AirWitness(product.AIR_CUBIC, t, k)])
        assert np.array_equal(sym.proof.fields, builtin.proof.fields)
        assert np.array_equal(sym.digest, builtin.digest)
        m0 = ctx.memory_stats()
        again = [product.prove_multi(ctx, pcs, [product.AirWitness(air, t)]) for _ in range(3)]
        m1 = ctx.memory_stats()
        assert all(np.array_equal(a.digest, sym.digest) for a in again)
        assert m1["reserved_bytes"] >= m1["used_bytes"] > 0
        assert m1["reserved_bytes"] == m0["reserved_bytes"]  # repeated proofs do not grow the pool
        assert m1["alloc_ms"] >= m0["alloc_ms"] >= 0
        with pytest.raises(product.P3gError):
            ctx.set_air_chunk_nodes(3)
    finally:
        ctx.close()


def test_linear_chain_rewrites_match_oracle(product, gpu_ctx):
    """The generated code's rewrites (96-bit chains closed at the 2^95 bound,
    the XOR form, weakly reduced products) give the oracle's proof."""
    desc = product.build_air(S.chains_eval, 8)
    src = product.air_source(desc)
    assert "gl::wide_canon(" in src and "gl::add(gl::sub(" in src and "gl::mul_weak(" in src
    air = product.Air(gpu_ctx, desc)
    t = S.chains_trace(8, 5)
    pcs = product.PcsParams(1, 1, 0, 8, 0, 24, 0)
    gpu = product.prove_multi(gpu_ctx, pcs, [product.AirWitness(air, t)])
    check_same(gpu, O.prove(O.default_p2(), pcs_dict(pcs), [(O.AIR_SYMBOLIC, t, None, {"sym": desc})]))
    assert product.verify_output(gpu_ctx, pcs, [product.AirShape(air, 256, 8)], gpu).ok
