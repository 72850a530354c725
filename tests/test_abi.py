"""CPU checks of the C ABI: the library loads without a GPU, exports every
function include/p3g.h declares, the host-side helpers (trace generators,
Poseidon2 constants) agree with the oracle, and argument validation fails
cleanly."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

import oracle_ffi as O

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    src = (ROOT / "include" / "p3g.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(p3g_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported(product):
    lib = C.CDLL(str(product.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_poseidon2_constants_match_oracle(product):
    assert np.array_equal(product.default_poseidon2_params(), O.p2_to_array(O.default_p2()))


def test_keccak_trace_generator_matches_oracle(product):
    inp = product.keccak_inputs(1, 42)
    assert np.array_equal(inp, O.keccak_inputs(1, 42))
    t = product.generate_keccak_trace(inp)
    assert t.shape == (1024, 2633)
    assert np.array_equal(t, O.keccak_trace(inp, 10))
    # partial last permutation and exact fits
    for n in (1, 2, 5, 11):
        inp = product.keccak_inputs(7, n)
        t = product.generate_keccak_trace(inp)
        h = t.shape[0]
        assert np.array_equal(t, O.keccak_trace(inp, h.bit_length() - 1))


def test_cubic_trace_generator_matches_oracle(product):
    for log_h, w, seed in [(1, 1, 0), (5, 7, 3), (9, 64, 11)]:
        k, t = product.generate_cubic_trace(log_h, w, seed)
        ko, to = O.cubic_trace(log_h, w, seed)
        assert np.array_equal(k, ko) and np.array_equal(t, to)


def test_constraint_counts(product):
    assert product.lib().p3g_air_num_constraints(product.AIR_KECCAK, 2633) == \
        O.lib().or_air_num_constraints(O.AIR_KECCAK, 2633) == 3182
    assert product.lib().p3g_air_num_constraints(product.AIR_CUBIC, 77) == 77


def test_invalid_arguments_are_rejected_without_a_device(product):
    lib = product.lib()
    assert lib.p3g_ctx_create(0, None, None) == product.ERR_INVALID
    out = np.zeros(4, dtype=np.uint64)
    assert lib.p3g_keccak_trace(None, 3, 4, out.ctypes.data_as(product.u64p)) == product.ERR_INVALID
    # 2 permutations need 48 rows: 2^5 is too small
    inp = np.zeros(50, dtype=np.uint64)
    assert lib.p3g_keccak_trace(inp.ctypes.data_as(product.u64p), 2, 5, out.ctypes.data_as(product.u64p)) \
        == product.ERR_INVALID
    assert lib.p3g_coset_lde(None, None, 4, 1, 1, 7, None) == product.ERR_INVALID


def test_proof_wire_format_roundtrip(product):
    """p3g_proof_serialize / p3g_proof_deserialize: a 128-byte header, then
    8 bytes per field element and 32 per commitment (TranscriptData's
    size_in_bytes); malformed buffers are rejected."""
    rng = np.random.default_rng(5)
    P = O.P
    for n_f, n_c in [(0, 0), (1, 0), (0, 3), (1000, 37)]:
        digest = rng.integers(0, P, size=12, dtype=np.uint64)
        proof = product.TranscriptData(rng.integers(0, P, size=n_f, dtype=np.uint64),
                                       rng.integers(0, P, size=(n_c, 4), dtype=np.uint64))
        wire = product.proof_to_wire(digest, proof)
        assert len(wire) == 128 + 8 * n_f + 32 * n_c
        assert wire[:8] == b"P3GPROOF"
        assert wire[128:] == proof.to_bytes()
        d2, p2 = product.proof_from_wire(wire)
        assert np.array_equal(d2, digest)
        assert np.array_equal(p2.fields, proof.fields) and np.array_equal(p2.commitments, proof.commitments)
    bad = [b"", wire[:127], b"X" + wire[1:], wire[:-1], wire + b"\0" * 8]
    nc = bytearray(wire)
    nc[128:136] = (P).to_bytes(8, "little")  # a field word equal to p
    bad.append(bytes(nc))
    for b in bad:
        try:
            product.proof_from_wire(b)
        except product.P3gError:
            continue
        raise AssertionError(f"accepted a malformed buffer of {len(b)} bytes")
