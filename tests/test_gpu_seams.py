"""The per-stage seams of the reference's PCS and LMCS traits, each against
the oracle bit for bit: LmcsTree::rows, one FRI fold (FriFold::fold_matrix,
arities 2, 4, 8), and the two halves of DEEP (batch_eval_lifted and the DEEP
quotient) over lifted matrices of several heights and widths."""
import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu
P = O.P


def rand_mat(rng, h, w):
    return rng.integers(0, P, size=(h, w), dtype=np.uint64)


@pytest.mark.parametrize("scenario,alignment", [([(4, 7), (8, 8), (16, 11)], 8), ([(1, 5), (8, 3)], 1),
                                                ([(16, 7)], 8), ([(2, 3), (4, 9), (64, 20)], 4)])
def test_lmcs_rows(product, gpu_ctx, scenario, alignment):
    """LmcsTree::rows (lifted_tree.rs:127-138): each matrix's row at the
    lifted index, zero-padded to the alignment."""
    rng = np.random.default_rng(len(scenario) + alignment)
    mats = [rand_mat(rng, h, w) for h, w in scenario]
    tree = product.LmcsTree(gpu_ctx, [product.to_device(m) for m in mats], alignment)
    H = scenario[-1][0]
    for idx in sorted({0, 1, H // 2, H - 1}):
        want = []
        for m in mats:
            r = m[idx >> ((H // m.shape[0]).bit_length() - 1)]
            pad = (-m.shape[1]) % alignment
            want.append(np.concatenate([r, np.zeros(pad, dtype=np.uint64)]))
        assert np.array_equal(tree.rows(idx), np.concatenate(want)), idx


@pytest.mark.parametrize("log_n,log_a", [(1, 1), (4, 1), (10, 1), (6, 2), (13, 2), (3, 3), (12, 3)])
def test_fri_fold_matches_oracle(product, gpu_ctx, log_n, log_a):
    rng = np.random.default_rng(log_n * 8 + log_a)
    layer = rand_mat(rng, 1 << log_n, 2)
    beta = (int(rng.integers(0, P, dtype=np.uint64)), int(rng.integers(0, P, dtype=np.uint64)))
    got = product.to_host(product.fri_fold(gpu_ctx, product.to_device(layer), log_a, beta))
    assert np.array_equal(got, O.fri_fold(layer, log_a, beta))


@pytest.mark.parametrize("shapes,log_blowup,alignment", [([(16, 5)], 1, 8), ([(8, 3), (32, 7), (32, 2)], 1, 8),
                                                         ([(64, 9), (256, 4), (1024, 12)], 3, 8),
                                                         ([(128, 16), (128, 1)], 2, 1)])
def test_deep_matches_oracle(product, gpu_ctx, shapes, log_blowup, alignment):
    """DEEP at the stage seam: the out-of-domain evaluations of every column
    (lifted matrices), then the quotient with given challenges."""
    rng = np.random.default_rng(sum(h * w for h, w in shapes))
    # columns of bit-reversed LDEs: low-degree data so the evaluations are meaningful
    mats = []
    for h, w in shapes:
        t = rand_mat(rng, h >> log_blowup, w)
        mats.append(O.coset_lde_bitrev(t, log_blowup, pow(7, 1 << ((shapes[-1][0] // h).bit_length() - 1), P)))
    ef = lambda: (int(rng.integers(0, P, dtype=np.uint64)), int(rng.integers(0, P, dtype=np.uint64)))
    z0 = ef()
    zs = [z0, (z0[0] * pow(7, (P - 1) // (shapes[-1][0] >> log_blowup), P) % P,
               z0[1] * pow(7, (P - 1) // (shapes[-1][0] >> log_blowup), P) % P)]
    dev = [product.to_device(m) for m in mats]
    ev = product.deep_evals(gpu_ctx, dev, log_blowup, zs)
    want = O.deep_evals(mats, log_blowup, zs)
    assert np.array_equal(ev, want)
    alpha, beta = ef(), ef()
    q = product.to_host(product.deep_quotient(gpu_ctx, dev, log_blowup, alignment, zs, ev, alpha, beta))
    assert np.array_equal(q, O.deep_quotient(mats, log_blowup, alignment, zs, want, alpha, beta))
