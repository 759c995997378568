"""The search entry point that allocates nothing, against the allocating one (needs a B200).

nndex_cuda_search_batch_device_noalloc is for callers that cannot call cudaMalloc while they
search — a process whose HBM another allocator has reserved in full, or a latency-critical path
that cannot take cudaMalloc's implicit synchronisation. It runs the same kernels in a fixed
file-scope device array, so its results must equal nndex_cuda_search_batch_device's. This file is
collected last so that a run stopping at the first failure has run every other test first; it
also passes alone in a fresh process (the first call on the device does the array's set-up).
"""
import ctypes as C

import numpy as np
import pytest

from nndex_b200 import NNdex, _lib

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _call(fn, index, q, k, torch):
    n, dims = q.shape
    kk = min(k, index.rows)
    idx = torch.zeros((n, kk), dtype=torch.int64, device="cuda")
    sim = torch.zeros((n, kk), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    if fn == "noalloc":
        st = _lib.lib().nndex_cuda_search_batch_device_noalloc(index.handle, q.data_ptr(), n, dims, k,
                                                               idx.data_ptr(), sim.data_ptr(), cnt.data_ptr(),
                                                               None)
    else:
        st = _lib.lib().nndex_cuda_search_batch_device(index.handle, q.data_ptr(), n, dims, k, idx.data_ptr(),
                                                       sim.data_ptr(), cnt.data_ptr(), None, 1)
    assert st == 0, _lib.last_error()
    return idx.cpu().numpy(), sim.cpu().numpy(), cnt.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2024)
    m = rng.normal(size=(120_000, 96)).astype(np.float32)
    index = NNdex(m)
    # two calls in a row with different batch shapes and k: the shared array keeps the previous
    # call's contents, which must not leak into the next result
    for n, k in [(16, 100), (5, 7)]:
        q = torch.from_numpy(rng.normal(size=(n, 96)).astype(np.float32)).cuda()
        ai, asim, acnt = _call("alloc", index, q, k, torch)
        ni, nsim, ncnt = _call("noalloc", index, q, k, torch)
        assert np.array_equal(ni, ai)
        assert np.max(np.abs(nsim - asim)) <= TOL
        assert np.array_equal(ncnt, acnt) and np.all(ncnt == k)


def test_noalloc_rejects_batches_beyond_its_array():
    torch = pytest.importorskip("torch")
    index = NNdex(np.random.default_rng(1).normal(size=(4096, 768)).astype(np.float32))
    n = _lib.NNDEX_NOALLOC_SCRATCH_BYTES // (768 * 4) + 1  # the normalised queries alone overflow it
    q = torch.ones((n, 768), dtype=torch.float32, device="cuda")
    out_i = torch.zeros((n, 10), dtype=torch.int64, device="cuda")
    out_s = torch.zeros((n, 10), dtype=torch.float32, device="cuda")
    st = _lib.lib().nndex_cuda_search_batch_device_noalloc(index.handle, q.data_ptr(), n, 768, 10,
                                                           out_i.data_ptr(), out_s.data_ptr(), None, None)
    assert st == _lib.NNDEX_ERR_UNSUPPORTED
    assert "no-allocation entry point" in _lib.last_error()


def test_noalloc_reports_query_errors():
    torch = pytest.importorskip("torch")
    index = NNdex(np.eye(4, 8, dtype=np.float32))
    q = torch.zeros((2, 8), dtype=torch.float32, device="cuda")
    q[0, 0] = 1.0
    out_i = torch.zeros((2, 2), dtype=torch.int64, device="cuda")
    out_s = torch.zeros((2, 2), dtype=torch.float32, device="cuda")
    st = _lib.lib().nndex_cuda_search_batch_device_noalloc(index.handle, q.data_ptr(), 2, 8, 2, out_i.data_ptr(),
                                                           out_s.data_ptr(), None, None)
    assert st == _lib.NNDEX_ERR_ZERO_NORM
    q[1, 1] = 1.0
    st = _lib.lib().nndex_cuda_search_batch_device_noalloc(index.handle, q.data_ptr(), 2, 8, 2, out_i.data_ptr(),
                                                           out_s.data_ptr(), None, None)
    assert st == 0, _lib.last_error()
    assert out_i.cpu().numpy()[:, 0].tolist() == [0, 1]


def test_noalloc_large_low_dim_batch_runs_in_pieces():
    """70,000 queries of 8 dims at k = 1 fit the array but exceed one launch's row of merge blocks
    (65,535): the batch runs in pieces of 16,384 queries like the allocating entry point's, with
    the same results, and the call's statistics describe this call."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(77)
    index = NNdex(rng.normal(size=(3000, 8)).astype(np.float32))
    q = torch.from_numpy(rng.normal(size=(70_000, 8)).astype(np.float32)).cuda()
    ai, asim, acnt = _call("alloc", index, q, 1, torch)
    ni, nsim, ncnt = _call("noalloc", index, q, 1, torch)
    assert np.array_equal(ni, ai)
    assert np.max(np.abs(nsim - asim)) <= TOL
    assert np.array_equal(ncnt, acnt) and np.all(ncnt == 1)
    st = _lib.SearchStats()
    assert _lib.lib().nndex_cuda_last_search_stats(index.handle, C.byref(st)) == 0
    assert st.path == 1
    assert st.kernel_launches == 3 * 5  # prep, scan and merge for each of 5 pieces
    assert st.rows_scanned == 3000 * 70_000
