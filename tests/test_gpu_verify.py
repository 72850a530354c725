"""Device-side verifier (p3g_verify, verify_multi with the openings, DEEP and
FRI query checks on the GPU): it accepts every GPU proof, and on perturbed
proofs it returns the same verdict as the verifier restatement
(oracle/or_verify.c). Perturbations are spread over the whole transcript
(field words, commitments, digest, length), so each failing check of
verify_multi is reached: an early field changes the challenges, a late one
an opened row or sibling."""
import numpy as np
import pytest

import oracle_ffi as O
from test_gpu_prove import pcs_dict

pytestmark = pytest.mark.gpu

P = (1 << 64) - (1 << 32) + 1


def _keccak_cfg(product):
    t = O.keccak_trace(O.keccak_inputs(1, 42), 10)
    pcs = product.PcsParams(1, 1, 0, 16, 0, 100, 0)
    return pcs, [product.AirWitness(product.AIR_KECCAK, t)], [(O.AIR_KECCAK, t.shape[0], t.shape[1], None)]


def _cubic_lifted(product):
    inst, oinst = [], []
    for log_h, w, seed in [(4, 32, 1), (7, 8, 2), (9, 4, 3)]:
        k, t = O.cubic_trace(log_h, w, seed)
        inst.append(product.AirWitness(product.AIR_CUBIC, t, k))
        oinst.append((O.AIR_CUBIC, t.shape[0], t.shape[1], k))
    return product.PcsParams(3, 2, 0, 5, 2, 20, 3), inst, oinst


def _cubic_arity8_final(product):
    k, t = O.cubic_trace(9, 12, 5)
    pcs = product.PcsParams(2, 3, 1, 3, 1, 24, 2)
    return pcs, [product.AirWitness(product.AIR_CUBIC, t, k)], [(O.AIR_CUBIC, t.shape[0], t.shape[1], k)]


def _mixed(product):
    k, tc = O.cubic_trace(7, 16, 9)
    tk = O.keccak_trace(O.keccak_inputs(3, 10), 8)
    inst = [product.AirWitness(product.AIR_CUBIC, tc, k), product.AirWitness(product.AIR_KECCAK, tk)]
    oinst = [(O.AIR_CUBIC, tc.shape[0], tc.shape[1], k), (O.AIR_KECCAK, tk.shape[0], tk.shape[1], None)]
    return product.PcsParams(1, 1, 0, 4, 0, 30, 0), inst, oinst


CASES = {"keccak_42_perms": _keccak_cfg, "cubic_lifted": _cubic_lifted, "cubic_arity8_final": _cubic_arity8_final,
         "cubic_keccak_mixed": _mixed}


@pytest.fixture(scope="module", params=list(CASES))
def case(request, product, gpu_ctx):
    pcs, inst, oinst = CASES[request.param](product)
    out = product.prove_multi(gpu_ctx, pcs, inst)
    return request.param, pcs, oinst, out


def _verdicts(product, ctx, pcs, oinst, fields, commits, digest):
    shapes = [product.AirShape(a, h, w, k) for a, h, w, k in oinst]
    g = product.verify_multi(ctx, pcs, shapes, fields, commits, digest)
    o = O.verify(O.default_p2(), pcs_dict(pcs), oinst, fields, commits, digest)
    return g, o


def test_accepts_gpu_proofs(product, gpu_ctx, case):
    name, pcs, oinst, out = case
    g, o = _verdicts(product, gpu_ctx, pcs, oinst, out.proof.fields, out.proof.commitments, out.digest)
    assert o == 0, name
    assert g.verdict == 0, f"{name}: device verifier rejected a valid proof ({g.name})"
    assert g.gpu_launches > 0


def test_perturbed_fields_match_oracle(product, gpu_ctx, case):
    name, pcs, oinst, out = case
    f0 = out.proof.fields
    n = f0.size
    positions = sorted(set(np.linspace(0, n - 1, 24).astype(int).tolist() + [n - 1, n - 2, n // 2]))
    seen = set()
    for pos in positions:
        f = f0.copy()
        f[pos] = (int(f[pos]) + 1) % P
        g, o = _verdicts(product, gpu_ctx, pcs, oinst, f, out.proof.commitments, out.digest)
        assert g.verdict == o, f"{name}: field {pos}: device {g.name}, oracle {O.VERIFY_ERRORS[o]}"
        assert g.verdict != 0
        seen.add(g.verdict)
    assert len(seen) >= 2, seen


def test_perturbed_commitments_match_oracle(product, gpu_ctx, case):
    name, pcs, oinst, out = case
    c0 = out.proof.commitments
    rows = sorted(set(np.linspace(0, c0.shape[0] - 1, 16).astype(int).tolist()))
    for r in rows:
        c = c0.copy()
        c[r, r % 4] = (int(c[r, r % 4]) + 1) % P
        g, o = _verdicts(product, gpu_ctx, pcs, oinst, out.proof.fields, c, out.digest)
        assert g.verdict == o, f"{name}: commitment {r}: device {g.name}, oracle {O.VERIFY_ERRORS[o]}"
        assert g.verdict != 0


def test_digest_and_length(product, gpu_ctx, case):
    name, pcs, oinst, out = case
    f, c, d = out.proof.fields, out.proof.commitments, out.digest
    d2 = d.copy()
    d2[5] = (int(d2[5]) + 1) % P
    variants = {"digest": (f, c, d2), "short": (f[:-1], c, d), "long": (np.append(f, np.uint64(3)), c, d),
                "commit short": (f, c[:-1], d), "commit long": (f, np.vstack([c, c[:1]]), d)}
    for label, (ff, cc, dd) in variants.items():
        g, o = _verdicts(product, gpu_ctx, pcs, oinst, ff, cc, dd)
        assert g.verdict == o, f"{name}: {label}: device {g.name}, oracle {O.VERIFY_ERRORS[o]}"
        assert g.verdict != 0
    g, _ = _verdicts(product, gpu_ctx, pcs, oinst, f, c, d2)
    assert g.name == "digest"


def test_noncanonical_word_is_an_error(product, gpu_ctx, case):
    name, pcs, oinst, out = case
    f = out.proof.fields.copy()
    f[0] = np.uint64(P)
    with pytest.raises(Exception):
        product.verify_multi(gpu_ctx, pcs, [product.AirShape(a, h, w, k) for a, h, w, k in oinst], f,
                             out.proof.commitments, out.digest)


def test_batch_matches_single(product, gpu_ctx):
    """p3g_verify_batch: one device pass for proofs of different shapes,
    valid and perturbed, gives each proof its single-call verdict."""
    items, want = [], []
    for i, make in enumerate(CASES.values()):
        pcs, inst, oinst = make(product)
        out = product.prove_multi(gpu_ctx, pcs, inst)
        shapes = [product.AirShape(a, h, w, k) for a, h, w, k in oinst]
        f, c, d = out.proof.fields, out.proof.commitments, out.digest
        variants = [(f, c, d)]
        bad = f.copy()
        k = (len(bad) * (i + 1)) // 5
        bad[k] = (int(bad[k]) + 1) % P
        variants.append((bad, c, d))
        d2 = d.copy()
        d2[0] = (int(d2[0]) + 1) % P
        variants.append((f, c, d2))
        variants.append((f[:-3], c, d))
        for ff, cc, dd in variants:
            items.append((pcs, shapes, ff, cc, dd))
            want.append(product.verify_multi(gpu_ctx, pcs, shapes, ff, cc, dd).verdict)
    for threads in (1, 0):
        got, stats = product.verify_batch(gpu_ctx, items, threads)
        assert got == want
        assert stats.gpu_launches > 0
    assert want.count(0) == len(CASES)


def test_wire_roundtrip_verifies(product, gpu_ctx, case):
    """A proof sent through the wire format verifies like the original."""
    name, pcs, oinst, out = case
    digest, proof = product.proof_from_wire(product.proof_to_wire(out.digest, out.proof))
    shapes = [product.AirShape(a, h, w, k) for a, h, w, k in oinst]
    assert product.verify_multi(gpu_ctx, pcs, shapes, proof.fields, proof.commitments, digest).ok, name
