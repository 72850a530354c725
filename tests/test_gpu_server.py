"""Batched and served proving: every proof produced inside a mix of
concurrent jobs is bit-identical to the same job proven alone, a failing job
reports its own status without disturbing the others, and admission respects
the HBM budget."""
import numpy as np
import pytest

import oracle_ffi as O

pytestmark = pytest.mark.gpu


def mix(product, n=9, seed=3):
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        if i % 3 == 2:
            perms = int(rng.integers(3, 20))
            t = product.generate_keccak_trace(product.keccak_inputs(100 + i, perms))
            w = [product.AirWitness(product.AIR_KECCAK, t)]
        else:
            log_h = int(rng.integers(4, 10))
            width = int(rng.choice([8, 16, 32, 64]))
            k, t = product.generate_cubic_trace(log_h, width, 1000 + i)
            w = [product.AirWitness(product.AIR_CUBIC, t, k)]
        pcs = product.PcsParams(int(rng.choice([1, 2, 3])), int(rng.choice([1, 2])), 0, 8, 0, 20, 0)
        jobs.append(product.Job(pcs, w))
    return jobs


def test_mix_matches_alone(product, gpu_ctx):
    jobs = mix(product)
    alone = [product.prove_multi(gpu_ctx, j.pcs, j.instances) for j in jobs]
    srv = product.ProofServer(0, n_workers=4)
    try:
        res = srv.run(jobs)
    finally:
        srv.close()
    for a, r in zip(alone, res):
        assert r.status == product.OK
        assert np.array_equal(a.proof.fields, r.output.proof.fields)
        assert np.array_equal(a.proof.commitments, r.output.proof.commitments)
        assert np.array_equal(a.digest, r.output.digest)


def test_failing_job_is_isolated(product, gpu_ctx):
    jobs = mix(product, n=4, seed=5)
    k1, t1 = product.generate_cubic_trace(6, 8, 1)
    k2, t2 = product.generate_cubic_trace(5, 8, 2)
    bad = product.Job(product.PcsParams(1, 1, 0, 4, 0, 8, 0),
                      [product.AirWitness(product.AIR_CUBIC, t1, k1), product.AirWitness(product.AIR_CUBIC, t2, k2)])
    jobs.insert(2, bad)  # descending heights: AirValidationError::NotAscending
    srv = product.ProofServer(0, n_workers=2)
    try:
        res = srv.run(jobs)
    finally:
        srv.close()
    assert res[2].status == product.ERR_VALIDATION and res[2].output is None
    for i, r in enumerate(res):
        if i == 2:
            continue
        alone = product.prove_multi(gpu_ctx, jobs[i].pcs, jobs[i].instances)
        assert r.status == product.OK
        assert np.array_equal(alone.proof.fields, r.output.proof.fields)


def test_arrivals_and_budget(product):
    jobs = mix(product, n=6, seed=7)
    for i, j in enumerate(jobs):
        j.arrival_s = 0.01 * i
    fps = [product.ProofServer.footprint_bytes(j.pcs, j.instances) for j in jobs]
    # a budget below any single job still runs every job, one at a time
    srv = product.ProofServer(0, n_workers=3, hbm_budget=1)
    try:
        res = srv.run(jobs)
        peak = srv.peak_admitted_bytes()
    finally:
        srv.close()
    assert all(r.status == product.OK for r in res)
    assert peak == max(fps)
    for r, j in zip(res, jobs):
        assert r.submit_s >= j.arrival_s - 1e-3 and r.start_s >= r.submit_s and r.end_s >= r.start_s
    # serialized by the budget: no two jobs overlap
    spans = sorted((r.start_s, r.end_s) for r in res)
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 1e-6


def test_submit_wait_from_python(product, gpu_ctx):
    jobs = mix(product, n=3, seed=9)
    srv = product.ProofServer(0, n_workers=2)
    try:
        tickets = [srv.submit(j) for j in jobs]
        res = [srv.wait(t) for t in tickets]
    finally:
        srv.close()
    for j, r in zip(jobs, res):
        alone = product.prove_multi(gpu_ctx, j.pcs, j.instances)
        assert r.status == product.OK and np.array_equal(alone.digest, r.output.digest)


def test_self_check(product, gpu_ctx):
    """With self-check on, every served proof is verified on the device
    before its job ends; the proofs are the same as without it."""
    jobs = mix(product, n=6, seed=11)
    srv = product.ProofServer(0, n_workers=3, self_check=True)
    try:
        res = srv.run(jobs)
    finally:
        srv.close()
    for j, r in zip(jobs, res):
        assert r.status == product.OK and r.verdict == 0 and r.verify_ms > 0
        alone = product.prove_multi(gpu_ctx, j.pcs, j.instances)
        assert np.array_equal(alone.digest, r.output.digest)
    srv = product.ProofServer(0, n_workers=2)
    try:
        plain = srv.run(jobs[:2])
    finally:
        srv.close()
    assert all(r.verdict == -1 for r in plain)


def test_heavy_and_symbolic_jobs(product, gpu_ctx):
    """Heavy jobs (LDEs above 2^26 words: Keccak 2^12 rows at blowup 8), with
    two allowed at once, beside light built-in and symbolic jobs (the
    symbolic ones use the worker's workspace for their column-major rows):
    every proof equals the same job proven alone."""
    import sym_airs as S
    jobs = []
    pcs_h = product.PcsParams(3, 1, 0, 8, 0, 20, 0)
    for i in range(2):
        t = product.generate_keccak_trace(product.keccak_inputs(300 + i, 170))
        jobs.append(product.Job(pcs_h, [product.AirWitness(product.AIR_KECCAK, t)]))
    for i in range(3):
        k, t = product.generate_cubic_trace(8 + i, 16, 400 + i)
        air = product.Air(gpu_ctx, product.build_air(S.cubic_eval(k), 16))
        jobs.append(product.Job(product.PcsParams(2, 1, 0, 8, 0, 20, 0), [product.AirWitness(air, t)]))
    alone = [product.prove_multi(gpu_ctx, j.pcs, j.instances) for j in jobs]
    srv = product.ProofServer(0, n_workers=3, max_heavy=2)
    try:
        res = srv.run(jobs)
    finally:
        srv.close()
    for a, r in zip(alone, res):
        assert r.status == product.OK
        assert np.array_equal(a.proof.fields, r.output.proof.fields)
        assert np.array_equal(a.digest, r.output.digest)
