"""p3g_coset_lde_noalloc: the coset LDE for callers that cannot allocate
device memory (a fixed, pre-reserved HBM budget, or a runtime whose own
allocator forbids cudaMalloc/cudaFree on its hot path). Its scratch is a
static device array inside the library, so its output must equal the
allocating entry point's (p3g_coset_lde) bit for bit, call after call: the
array keeps the previous call's contents and every call must overwrite what
it reads. Collected last so that a failure here stops a -x run only after
every other test has run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
P = 0xFFFFFFFF00000001


def noalloc_fn(product):
    lib = C.CDLL(str(product.LIB_PATH))
    fn = lib.p3g_coset_lde_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint64, C.c_void_p, C.c_void_p]
    mx = lib.p3g_coset_lde_noalloc_max_words
    mx.restype = C.c_uint64
    return fn, int(mx())


def run_noalloc(product, fn, trace, log_blowup, shift):
    import torch
    d_in = product.to_device(trace)
    h, w = trace.shape
    d_out = product.empty_device((h << log_blowup, w))
    d_out.fill_(-1)  # poison: every output word must be written
    torch.cuda.synchronize()
    rc = fn(d_in.data_ptr(), h, w, log_blowup, shift, d_out.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    return product.to_host(d_out)


def test_noalloc_lde_matches_allocating_entry_point(product, gpu_ctx):
    fn, max_words = noalloc_fn(product)
    assert max_words == 1 << 21
    rng = np.random.default_rng(2025)
    # two calls in a row with different shapes, then a repeat of the first;
    # then the edges of the pass layout: height 1 (a pass of zero bits),
    # blowup 1 (log_blowup 0), and the widest inputs the scratch admits
    # (more column tiles than one launch's grid.y holds)
    cases = [(12, 96, 1), (7, 5, 3), (12, 96, 1), (20, 2, 1),
             (0, 3, 2), (10, 7, 0), (2, 1 << 19, 1), (1, 1 << 20, 1)]
    for log_h, w, lb in cases:
        t = rng.integers(0, P, size=(1 << log_h, w), dtype=np.uint64)
        shift = int(rng.integers(1, P, dtype=np.uint64))
        got = run_noalloc(product, fn, t, lb, shift)
        want = product.to_host(product.coset_lde(gpu_ctx, product.to_device(t), lb, shift))
        assert np.array_equal(got, want), (log_h, w, lb)


def test_noalloc_rejects_sizes_beyond_its_scratch(product):
    import torch
    fn, max_words = noalloc_fn(product)
    small = product.empty_device((4, 4))
    out = product.empty_device((8, 4))
    torch.cuda.synchronize()
    # height * width over the static scratch, and a height beyond 2^22
    assert fn(small.data_ptr(), 1 << 20, 4, 1, 7, out.data_ptr(), None) == product.ERR_INVALID
    assert fn(small.data_ptr(), 1 << 23, 1, 1, 7, out.data_ptr(), None) == product.ERR_INVALID
    assert fn(small.data_ptr(), 3, 4, 1, 7, out.data_ptr(), None) == product.ERR_INVALID
