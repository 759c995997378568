"""Exact-search parity of the CUDA backend against the CPU oracle (needs a B200).

Every call goes through nndex_b200.NNdex → libnndex_cuda.so's C ABI. Acceptance rule:
scores within 1e-5 absolute of the FP64 score of the returned row, and indices bit-exact wherever
the FP64 gap between neighbouring ranks exceeds 1e-5 (ties → lower index); see tests/_parity.py.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from nndex_b200 import NNdex, kernel_launch_count, list_gpu_devices
from nndex_b200 import _lib
from oracle import oracle as O
from tests._parity import assert_topk_matches

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _oracle_storage(m, normalized):
    st, base = O.prepare_index(m, normalized)
    assert st == 0
    return base


def _check_batch(index, m, queries, k, normalized=False, what=""):
    base = _oracle_storage(m, normalized)
    idx, sim = index.search(queries, k=k)
    st, qn = O.prepare_queries(queries, normalized, base.shape[1])
    assert st == 0
    for i in range(queries.shape[0]):
        s64 = O.scores_f64(base, qn[i])
        assert_topk_matches(idx[i], sim[i], s64, k, what=f"{what} q{i}")
    return idx, sim


def test_device_listed():
    devs = list_gpu_devices()
    assert devs and devs[0]["backend"] == "Cuda"
    assert devs[0]["compute_capability"] == "10.0"


def test_demo_seed42_golden():
    g = json.load(open(os.path.join(GOLD, "demo_seed42.json")))
    rng = np.random.default_rng(42)
    m = rng.normal(size=(g["rows"], g["dims"])).astype(np.float32)
    q = rng.normal(size=(g["dims"],)).astype(np.float32)
    queries = rng.normal(size=(4, g["dims"])).astype(np.float32)
    index = NNdex(m, normalized=False, approx=False, backend="cuda")
    idx, sim = index.search(q, k=5)
    assert idx.dtype == np.uint64 and sim.dtype == np.float32
    assert idx.tolist() == g["indices"]
    np.testing.assert_allclose(sim, np.array(g["similarities"], np.float32), atol=1e-5)
    idx10, _ = index.search(q, k=10)
    assert idx10.tolist() == g["numpy_f64_top10"]
    bi, bs = index.search(queries, k=5)
    assert bi.shape == (4, 5) and bs.shape == (4, 5)
    _check_batch(index, m, queries, 5, what="demo batch")


def test_config1_batch64_k10():
    rng = np.random.default_rng(42)
    m = rng.normal(size=(50_000, 128)).astype(np.float32)
    queries = rng.normal(size=(64, 128)).astype(np.float32)
    index = NNdex(m)
    _check_batch(index, m, queries, 10, what="c1 b64")


def test_known_answer():
    m = np.array([[1, 0, 0, 0, 0, 0, 0, 0], [0, 1, 0, 0, 0, 0, 0, 0], [1, 1, 0, 0, 0, 0, 0, 0]], np.float32)
    index = NNdex(m, normalized=False)
    idx, sim = index.search(np.array([0.8, 0.6, 0, 0, 0, 0, 0, 0], np.float32), k=2)
    assert idx.tolist() == [2, 0]
    assert abs(sim[0] - 0.98994946) <= 1e-5 and abs(sim[1] - 0.8) <= 1e-6


def test_batch_matches_single_query_results():
    m = np.eye(3, 8, dtype=np.float32)
    index = NNdex(m, normalized=True)
    queries = np.eye(2, 8, dtype=np.float32)
    bi, bs = index.search(queries, k=2)
    for r in range(2):
        si, ss = index.search(queries[r], k=2)
        assert bi[r].tolist() == si.tolist()
        assert bs[r].tolist() == ss.tolist()


def test_padding_non_multiple_of_8():
    index = NNdex(np.ones((3, 7), np.float32))
    assert index.dims == 7
    idx, _ = index.search(np.ones(7, np.float32), k=1)
    assert idx.shape == (1,)


PARITY = [
    # rows, dims, nq, k
    (1, 8, 1, 1), (5, 8, 3, 3), (127, 16, 2, 10), (128, 31, 4, 128), (129, 33, 5, 7),
    (1000, 1, 1, 5), (1000, 7, 16, 100), (1000, 64, 17, 1000), (4096, 128, 1, 25),
    (5000, 200, 8, 64), (20000, 96, 16, 100), (20000, 768, 4, 100), (3000, 256, 40, 10),
    (2500, 48, 33, 2048), (70000, 32, 16, 300),
]


def _away_from_zero(x):
    # rows whose squared norm is at or below f32::EPSILON are ZeroNorm errors (as in the
    # reference); keep random test rows clear of that threshold
    small = np.sum(x.astype(np.float64) ** 2, axis=1) < 1e-3
    x[small] += np.float32(0.5)
    return x


@pytest.mark.parametrize("rows,dims,nq,k", PARITY)
def test_random_parity(rows, dims, nq, k):
    rng = np.random.default_rng(rows * 131 + dims * 7 + nq)
    m = _away_from_zero(rng.normal(size=(rows, dims)).astype(np.float32))
    queries = _away_from_zero(rng.normal(size=(nq, dims)).astype(np.float32))
    index = NNdex(m)
    if nq == 1:
        idx, sim = index.search(queries[0], k=k)
        base = _oracle_storage(m, False)
        st, qn = O.prepare_query(queries[0], False, base.shape[1])
        assert_topk_matches(idx, sim, O.scores_f64(base, qn), k, what="single")
    else:
        _check_batch(index, m, queries, k, what=f"{rows}x{dims}")


def test_exact_vs_numpy_4096x128():
    # tests_python/test_accuracy_vs_numpy.py:15-26
    rng = np.random.default_rng(123)
    m = rng.normal(size=(4096, 128)).astype(np.float32)
    q = rng.normal(size=(128,)).astype(np.float32)
    idx, sim = NNdex(m, normalized=False).search(q, k=25)
    mn = m / np.maximum(np.linalg.norm(m, axis=1, keepdims=True), 1e-12)
    qq = q / max(float(np.linalg.norm(q)), 1e-12)
    s = mn @ qq
    top = np.argpartition(s, -25)[-25:]
    ordered = top[np.argsort(s[top])[::-1]]
    assert np.array_equal(idx, ordered)
    assert np.allclose(sim, s[ordered], atol=1e-5)


def test_matches_oracle_exactly_without_near_ties():
    rng = np.random.default_rng(5)
    m = rng.normal(size=(30000, 128)).astype(np.float32)
    queries = rng.normal(size=(16, 128)).astype(np.float32)
    index = NNdex(m)
    idx, sim = index.search(queries, k=50)
    base = _oracle_storage(m, False)
    _, qn = O.prepare_queries(queries, False, base.shape[1])
    oi, osim = O.search_exact(base, qn, 50)
    assert np.array_equal(idx.astype(np.int64), oi.astype(np.int64))
    assert np.max(np.abs(sim - osim)) <= 1e-5


def test_k_larger_than_rows_returns_all_rows():
    m = np.eye(2, 8, dtype=np.float32)
    idx, _ = NNdex(m).search(np.eye(1, 8, dtype=np.float32)[0], k=100)
    assert idx.shape == (2,)


def test_single_row():
    m = np.eye(1, 8, dtype=np.float32)
    idx, sim = NNdex(m, normalized=True).search(m[0], k=1)
    assert idx.tolist() == [0] and abs(sim[0] - 1.0) <= 1e-5
    m2 = np.zeros((1, 8), np.float32)
    m2[0, 1] = 1.0
    idx, sim = NNdex(m2, normalized=True).search(m2[0], k=5)
    assert idx.tolist() == [0] and abs(sim[0] - 1.0) <= 1e-5


def test_batch_k_one_matches_single():
    rng = np.random.default_rng(42)
    m = (rng.random(size=(100, 16)) - 0.5).astype(np.float32)
    queries = (rng.random(size=(8, 16)) - 0.5).astype(np.float32)
    index = NNdex(m)
    bi, bs = index.search(queries, k=1)
    for r in range(8):
        si, ss = index.search(queries[r], k=1)
        assert bi[r, 0] == si[0] and abs(bs[r, 0] - ss[0]) <= 1e-5


def test_all_negative_scores():
    m = np.zeros((5, 8), np.float32)
    m[:, 0] = 1.0
    index = NNdex(m, normalized=True)
    q = np.zeros((4, 8), np.float32)
    q[:, 0] = -1.0
    idx, sim = index.search(q, k=3)
    assert idx.shape == (4, 3)
    assert np.all(idx < 5) and np.allclose(sim, -1.0, atol=1e-5)
    # identical scores: the canonical order keeps the lowest rows
    assert idx.tolist() == [[0, 1, 2]] * 4


def test_identical_rows_tie_break_by_index():
    m = np.tile(np.arange(1, 17, dtype=np.float32), (3000, 1))
    index = NNdex(m)
    idx, sim = index.search(np.arange(1, 17, dtype=np.float32), k=100)
    assert idx.tolist() == list(range(100))
    assert np.allclose(sim, 1.0, atol=1e-5)


def _batch_via_abi(index, q, k):
    q = np.ascontiguousarray(q, dtype=np.float32)
    n = q.shape[0]
    kk = min(k, index.rows)
    idx = np.zeros((n, kk), np.uint64)
    sim = np.zeros((n, kk), np.float32)
    cnt = np.zeros(n, np.uint64)
    st = _lib.lib().nndex_cuda_search_batch(index.handle, q.ctypes.data, q.size, n, k, idx.ctypes.data,
                                            sim.ctypes.data, cnt.ctypes.data)
    assert st == 0, _lib.last_error()
    return idx, sim


def test_alone_equals_in_batch_bitwise():
    # The scan's FMA order per (row, query) does not depend on the batch's composition, so a
    # query scored alone (batch of one) and inside any batch gives bit-identical results.
    rng = np.random.default_rng(9)
    m = rng.normal(size=(50000, 96)).astype(np.float32)
    queries = rng.normal(size=(16, 96)).astype(np.float32)
    index = NNdex(m)
    bi, bs = _batch_via_abi(index, queries, 20)
    for r in [0, 5, 15]:
        ai, as_ = _batch_via_abi(index, queries[r:r + 1], 20)
        assert ai[0].tolist() == bi[r].tolist()
        assert as_[0].tobytes() == bs[r].tobytes()
        lo = min(r, 13)
        si, ss = _batch_via_abi(index, queries[lo:lo + 3], 20)
        assert si[r - lo].tolist() == bi[r].tolist()
        assert ss[r - lo].tobytes() == bs[r].tobytes()
    # NNdex::search normalises a single query with sequential FP32 (src/lib.rs:558-569) while
    # search_batch uses the FP64-accumulated row norm (src/lib.rs:525-532): same indices, scores
    # within the tolerance.
    for r in [0, 5, 15]:
        ai, as_ = index.search(queries[r], k=20)
        assert ai.tolist() == bi[r].tolist()
        assert np.max(np.abs(as_ - bs[r])) <= 1e-5


def test_normalized_flag_skips_normalization():
    rng = np.random.default_rng(11)
    m = rng.normal(size=(2000, 64)).astype(np.float32)
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    queries = rng.normal(size=(6, 64)).astype(np.float32)
    queries /= np.linalg.norm(queries, axis=1, keepdims=True)
    index = NNdex(m, normalized=True)
    _check_batch(index, m, queries, 10, normalized=True, what="normalized")


def test_error_paths():
    with pytest.raises(ValueError, match="all input values must be finite"):
        NNdex(np.array([[1.0, np.nan] + [0.0] * 6], np.float32))
    with pytest.raises(ValueError, match="all input values must be finite"):
        NNdex(np.array([[np.inf] + [0.0] * 7], np.float32))
    with pytest.raises(ValueError, match="zero-norm"):
        NNdex(np.zeros((1, 8), np.float32))
    with pytest.raises(ValueError, match="all input values must be finite"):
        NNdex(np.array([[np.nan] * 8], np.float32), normalized=True)
    index = NNdex(np.eye(1, 8, dtype=np.float32))
    with pytest.raises(RuntimeError, match="top-k must be greater than zero"):
        index.search(np.ones(8, np.float32), k=0)
    with pytest.raises(ValueError, match="query dims mismatch"):
        index.search(np.ones(4, np.float32), k=1)
    with pytest.raises(RuntimeError, match="all input values must be finite"):
        index.search(np.array([np.nan] + [0.0] * 7, np.float32), k=1)
    with pytest.raises(RuntimeError, match="zero-norm"):
        index.search(np.zeros(8, np.float32), k=1)
    index2 = NNdex(np.ones((2, 8), np.float32))
    with pytest.raises(RuntimeError, match="top-k must be greater than zero"):
        index2.search(np.ones((2, 8), np.float32), k=0)
    with pytest.raises(RuntimeError, match="zero-norm"):
        index2.search(np.array([[1.0] * 8, [0.0] * 8], np.float32), k=1)


def test_c_abi_shape_and_order_checks():
    L = _lib.lib()
    index = NNdex(np.ones((2, 8), np.float32))
    q = np.ones(16, np.float32)
    out_i = np.zeros(16, np.uint64)
    out_s = np.zeros(16, np.float32)
    cnt = np.zeros(3, np.uint64)
    # search_batch: shape before k (src/lib.rs:378-381)
    st = L.nndex_cuda_search_batch(index.handle, q.ctypes.data, 16, 3, 0, out_i.ctypes.data, out_s.ctypes.data,
                                   cnt.ctypes.data)
    assert st == _lib.NNDEX_ERR_SHAPE_MISMATCH
    assert "matrix shape mismatch: rows=3, dims=8, values=16" in _lib.last_error()
    # search: k before dims (src/lib.rs:336-344)
    c = C.c_uint64(0)
    st = L.nndex_cuda_search(index.handle, q.ctypes.data, 4, 0, out_i.ctypes.data, out_s.ctypes.data, C.byref(c))
    assert st == _lib.NNDEX_ERR_INVALID_TOPK
    st = L.nndex_cuda_search(index.handle, q.ctypes.data, 4, 1, out_i.ctypes.data, out_s.ctypes.data, C.byref(c))
    assert st == _lib.NNDEX_ERR_QUERY_DIMS
    assert "expected 8, found 4" in _lib.last_error()
    h = C.c_void_p()
    st = L.nndex_cuda_create(q.ctypes.data, 10, 3, 4, 0, None, C.byref(h))
    assert st == _lib.NNDEX_ERR_SHAPE_MISMATCH
    st = L.nndex_cuda_create(q.ctypes.data, 0, 0, 8, 0, None, C.byref(h))
    assert st == _lib.NNDEX_ERR_SHAPE_MISMATCH
    opts = _lib.Opts()
    opts.device = 9999
    st = L.nndex_cuda_create(q.ctypes.data, 16, 2, 8, 0, C.byref(opts), C.byref(h))
    assert st == _lib.NNDEX_ERR_DEVICE_INDEX


def test_device_api_and_fp64_report():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    m = rng.normal(size=(40000, 128)).astype(np.float32)
    queries = rng.normal(size=(12, 128)).astype(np.float32)
    index = NNdex(m)
    k = 32
    dq = torch.from_numpy(queries).cuda()
    di = torch.zeros((12, k), dtype=torch.int64, device="cuda")
    ds = torch.zeros((12, k), dtype=torch.float32, device="cuda")
    dc = torch.zeros(12, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = _lib.lib().nndex_cuda_search_batch_device(index.handle, dq.data_ptr(), 12, 128, k, di.data_ptr(),
                                                   ds.data_ptr(), dc.data_ptr(), None, 1)
    assert st == 0, _lib.last_error()
    hi, hs = index.search(queries, k=k)
    assert np.array_equal(di.cpu().numpy().astype(np.uint64), hi)
    assert np.array_equal(ds.cpu().numpy(), hs)
    assert dc.cpu().tolist() == [k] * 12
    # FP64 oracle on the device for the returned pairs
    base = _oracle_storage(m, False)
    _, qn = O.prepare_queries(queries, False, base.shape[1])
    pq = torch.arange(12, device="cuda").repeat_interleave(k).to(torch.int64)
    pr = di.reshape(-1)
    out = torch.zeros(12 * k, dtype=torch.float64, device="cuda")
    dqn = torch.from_numpy(np.ascontiguousarray(qn[:, :128])).cuda()
    st = _lib.lib().nndex_cuda_fp64_scores(index.handle, dqn.data_ptr(), 12, pq.data_ptr(), pr.data_ptr(), 12 * k,
                                           out.data_ptr())
    assert st == 0, _lib.last_error()
    got = out.cpu().numpy().reshape(12, k)
    for i in range(12):
        ref = O.scores_f64(base, qn[i])[hi[i].astype(np.int64)]
        np.testing.assert_allclose(got[i], ref, rtol=0, atol=1e-12)
        assert np.max(np.abs(hs[i] - got[i])) <= 1e-5


def test_launch_counter_and_stats():
    rng = np.random.default_rng(1)
    index = NNdex(rng.normal(size=(5000, 64)).astype(np.float32))
    before = kernel_launch_count()
    index.search(rng.normal(size=(4, 64)).astype(np.float32), k=10)
    after = kernel_launch_count()
    st = index.last_search_stats()
    assert after - before == st["kernel_launches"] == 3
    assert st["path"] == 1
    info = index.gpu_info
    assert info["backend"] == "Cuda" and info["sm_count"] >= 100


def test_large_multi_cta_flushes():
    rng = np.random.default_rng(21)
    m = rng.normal(size=(300_000, 64)).astype(np.float32)
    queries = rng.normal(size=(16, 64)).astype(np.float32)
    index = NNdex(m)
    idx, sim = index.search(queries, k=100)
    base = _oracle_storage(m, False)
    _, qn = O.prepare_queries(queries, False, base.shape[1])
    oi, osim = O.search_exact(base, qn, 100)
    for i in range(16):
        assert_topk_matches(idx[i], sim[i], O.scores_f64(base, qn[i]), 100, what=f"q{i}")


def test_create_from_device_waits_for_pending_writes():
    # The matrix is still being written asynchronously (no synchronize) when the index is built.
    torch = pytest.importorskip("torch")
    rows, dims = 2_000_000, 128
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    x = torch.randn((rows, dims), generator=g, device="cuda")
    x = x / torch.linalg.vector_norm(x, dim=1, keepdim=True)
    h = C.c_void_p()
    opts = _lib.Opts()
    opts.device = 0
    st = _lib.lib().nndex_cuda_create_from_device(x.data_ptr(), x.numel(), rows, dims, _lib.NNDEX_FLAG_NORMALIZED,
                                                  C.byref(opts), C.byref(h))
    assert st == 0, _lib.last_error()
    try:
        q = x[[0, rows // 2, rows - 1]].clone()
        pq = torch.arange(3, device="cuda", dtype=torch.int64)
        pr = torch.tensor([0, rows // 2, rows - 1], device="cuda", dtype=torch.int64)
        out = torch.zeros(3, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert _lib.lib().nndex_cuda_fp64_scores(h, q.data_ptr(), 3, pq.data_ptr(), pr.data_ptr(), 3,
                                                 out.data_ptr()) == 0
        assert np.allclose(out.cpu().numpy(), 1.0, atol=1e-5)
    finally:
        _lib.lib().nndex_cuda_destroy(h)
