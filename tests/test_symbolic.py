"""Symbolic AIRs on the CPU: the degree analysis of the product and of the
oracle agree with each other and with the reference's rule
(log2_ceil(max(M, 2) - 1), p3-miden-lifted-air/src/air.rs:225-247); the
oracle's symbolic path reproduces its built-in cubic AIR bit for bit; the
oracle proves and verifies the reference's test AIRs (TinyAir with periodic
columns and an aux trace, BusTestAir with extension constraints and aux
values, DummyMidenAir of degree 9); the generated constraint kernels compile
with NVRTC for sm_100a; malformed DAGs are rejected."""
import numpy as np
import pytest

import oracle_ffi as O
import sym_airs as S


def pcs_d(lb, arity=1, final=0, fpow=4, dpow=0, nq=12, qpow=0):
    return dict(log_blowup=lb, log_folding_arity=arity, log_final_degree=final, folding_pow_bits=fpow,
                deep_pow_bits=dpow, num_queries=nq, query_pow_bits=qpow)


def tiny_desc(product, periods=()):
    return product.build_air(S.tiny_eval, 1, num_public_values=1, num_aux_values=1,
                             periodic_columns=S.tiny_periodic(periods))


def bus_desc(product):
    return product.build_air(S.bus_eval, 1, aux_width=2, num_randomness=2, num_aux_values=2, num_public_values=3)


def miden_desc(product, width, n_aux=8):
    return product.build_air(S.miden_eval, width, aux_width=n_aux, num_randomness=2, num_aux_values=n_aux)


def test_degree_analysis(product):
    k = np.arange(1, 9, dtype=np.uint64)
    cases = [(product.build_air(S.cubic_eval(k), 8), 3, 1), (tiny_desc(product), 4, 2),
             (tiny_desc(product, (2, 4)), 4, 2), (bus_desc(product), 4, 2), (miden_desc(product, 12), 9, 3)]
    for desc, deg, lqd in cases:
        got = product.air_analyse(desc)
        assert (got["max_degree"], got["log_quotient_degree"]) == (deg, lqd)
        assert O.sym_degree(desc) == (deg, lqd)
        assert got["n_base"] + got["n_ext"] == desc.num_constraints
    lay = product.air_analyse(bus_desc(product))
    assert (lay["n_base"], lay["n_ext"]) == (2, 6)


def test_oracle_symbolic_cubic_equals_builtin():
    """The symbolic path of the oracle against its hand-written cubic AIR:
    same constraints in the same order, so the same proof."""
    import conftest
    product = conftest.load_product()
    k, t = O.cubic_trace(6, 5, 11)
    k2, t2 = O.cubic_trace(8, 3, 12)
    pcs = pcs_d(2, 2, fpow=3, dpow=1, nq=10, qpow=1)
    builtin = O.prove(O.default_p2(), pcs, [(O.AIR_CUBIC, t, k), (O.AIR_CUBIC, t2, k2)])
    d1, d2 = product.build_air(S.cubic_eval(k), 5), product.build_air(S.cubic_eval(k2), 3)
    sym = O.prove(O.default_p2(), pcs, [(O.AIR_CUBIC, t, None, {"sym": d1}), (O.AIR_CUBIC, t2, None, {"sym": d2})])
    for key in ("fields", "commits", "digest"):
        assert np.array_equal(builtin[key], sym[key]), key
    assert O.verify(O.default_p2(), pcs, [(O.AIR_CUBIC, 64, 5, None, {"sym": d1}), (O.AIR_CUBIC, 256, 3, None, {"sym": d2})],
                    sym["fields"], sym["commits"], sym["digest"]) == 0


@pytest.mark.parametrize("periods,heights", [((), (8,)), ((4,), (8,)), ((2, 4), (4, 8)), ((2, 4), (4, 8, 16))])
def test_oracle_tiny_air_proves_and_verifies(product, periods, heights):
    """TinyAir's own cases (tests/tiny_air.rs): periodic columns, several
    traces of different heights, aux trace challenge^(4^row)."""
    desc = tiny_desc(product, periods)
    inst, shapes = [], []
    for i, h in enumerate(heights):
        t = S.tiny_trace(i + 2, h)
        extra = {"sym": desc, "public_values": np.array([i + 2], dtype=np.uint64), "aux_builder": S.tiny_aux}
        inst.append((O.AIR_SYMBOLIC, t, None, extra))
        shapes.append((O.AIR_SYMBOLIC, h, 1, None, extra))
    pcs = pcs_d(2, 1, fpow=2, nq=8)
    pr = O.prove(O.default_p2(), pcs, inst)
    assert O.verify(O.default_p2(), pcs, shapes, pr["fields"], pr["commits"], pr["digest"]) == 0
    bad = pr["fields"].copy()
    bad[5] = (int(bad[5]) + 1) % O.P
    assert O.verify(O.default_p2(), pcs, shapes, bad, pr["commits"], pr["digest"]) != 0
    # a statement with another public value does not verify
    wrong = [(a, h, w, c, dict(e, public_values=np.array([99], dtype=np.uint64))) for a, h, w, c, e in shapes]
    assert O.verify(O.default_p2(), pcs, wrong, pr["fields"], pr["commits"], pr["digest"]) == O.VERIFY_ERRORS_CODE[
        "quotient identity"]


def test_oracle_bus_air_proves_and_verifies(product):
    desc = bus_desc(product)
    pv = np.array([2, 42, 67], dtype=np.uint64)
    t = S.tiny_trace(2, 8)
    extra = {"sym": desc, "public_values": pv, "aux_builder": S.bus_aux(42, 67)}
    pcs = pcs_d(2, 1, fpow=2, nq=8)
    pr = O.prove(O.default_p2(), pcs, [(O.AIR_SYMBOLIC, t, None, extra)])
    assert O.verify(O.default_p2(), pcs, [(O.AIR_SYMBOLIC, 8, 1, None, extra)], pr["fields"], pr["commits"],
                    pr["digest"]) == 0


def test_oracle_miden_dummy_air(product):
    """DummyMidenAir: one degree-9 constraint (eight quotient chunks, so
    log_blowup 3), 8 all-zero aux EF columns, two traces of different widths."""
    d1, d2 = miden_desc(product, 12), miden_desc(product, 10)
    t1, t2 = S.miden_trace(12, 5, 1), S.miden_trace(10, 6, 2)
    pcs = pcs_d(3, 2, fpow=2, nq=8)
    pr = O.prove(O.default_p2(), pcs, [(O.AIR_SYMBOLIC, t1, None, {"sym": d1}), (O.AIR_SYMBOLIC, t2, None, {"sym": d2})])
    assert O.verify(O.default_p2(), pcs, [(O.AIR_SYMBOLIC, 32, 12, None, {"sym": d1}),
                                          (O.AIR_SYMBOLIC, 64, 10, None, {"sym": d2})],
                    pr["fields"], pr["commits"], pr["digest"]) == 0


def test_generated_kernels_compile_for_sm100a(product):
    k = np.arange(3, 67, dtype=np.uint64)
    for desc in (product.build_air(S.cubic_eval(k), 64), tiny_desc(product, (2, 4)), bus_desc(product),
                 miden_desc(product, 51)):
        assert product.air_compile_check(desc, 100) > 0
    src = product.air_source(bus_desc(product))
    assert "p3g_sym_eval" in src and "gl::ef_mul" in src


def test_malformed_dags_rejected(product):
    desc = tiny_desc(product)
    bad = product.AirDesc(**{**desc.__dict__})
    bad.nodes = desc.nodes.copy()
    # an operand after its node
    i = int(np.nonzero(bad.nodes["op"] == product.symbolic.MUL)[0][0])
    bad.nodes[i]["a"] = len(bad.nodes) - 1
    with pytest.raises(product.P3gError):
        product.air_analyse(bad)
    # a main column outside the width
    bad2 = product.AirDesc(**{**desc.__dict__})
    bad2.nodes = desc.nodes.copy()
    j = int(np.nonzero(bad2.nodes["op"] == product.symbolic.MAIN)[0][0])
    bad2.nodes[j]["a"] = 5
    with pytest.raises(product.P3gError):
        product.air_analyse(bad2)


def test_oracle_symbolic_keccak_equals_builtin(product):
    """The Keccak-f[1600] AIR written against the symbolic builder (3182
    constraints, degree 3) drives the oracle to its hand-written Keccak
    AIR's proof, bit for bit: the DAG carries the same constraints in the
    same order."""
    desc = product.build_air(S.keccak_eval, S.KC_NCOLS)
    assert desc.num_constraints == 3182
    assert product.air_analyse(desc)["log_quotient_degree"] == 1
    t = O.keccak_trace(O.keccak_inputs(1, 5), 7)
    pcs = pcs_d(1, 1, fpow=4, nq=10)
    a = O.prove(O.default_p2(), pcs, [(O.AIR_KECCAK, t, None)])
    b = O.prove(O.default_p2(), pcs, [(O.AIR_KECCAK, t, None, {"sym": desc})])
    for key in ("fields", "commits", "digest"):
        assert np.array_equal(a[key], b[key]), key


def test_chains_air_holds_on_its_trace(product):
    """The rewrite test AIR's trace satisfies its constraint (oracle's
    symbolic evaluation on the CPU), so its GPU proof must verify."""
    desc = product.build_air(S.chains_eval, 8)
    t = S.chains_trace(4, 5)
    pcs = dict(log_blowup=1, log_folding_arity=1, log_final_degree=0, folding_pow_bits=4, deep_pow_bits=0,
               num_queries=8, query_pow_bits=0)
    out = O.prove(O.default_p2(), pcs, [(O.AIR_SYMBOLIC, t, None, {"sym": desc})])
    assert O.verify(O.default_p2(), pcs, [(O.AIR_SYMBOLIC, t.shape[0], t.shape[1], None, {"sym": desc})],
                    out["fields"], out["commits"], out["digest"]) == 0
    # the generated source of this AIR compiles for sm_100a without a device
    assert product.air_compile_check(desc) > 0
