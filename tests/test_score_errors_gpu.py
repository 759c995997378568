"""Per-result score errors against the FP64 oracle (needs a B200).

With the error report on, every search records, for each returned (query, row), |returned score −
FP64 score of the stored row with the normalised query|. The expected value comes from the CPU
oracle's own normalisation of the same matrix and queries (bit-identical to the index's), scored in
FP64 here; the two FP64 sums differ only in order, far below the reported errors' 1e-12 tolerance.
"""
import numpy as np
import pytest

from nndex_b200 import NNdex
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _expected(m, q, idx, sim, normalized=False):
    st, base = O.prepare_index(m, normalized)
    assert st == 0
    _, qn = O.prepare_queries(q, normalized, base.shape[1])
    s64 = np.einsum("qkd,qd->qk", base[idx.astype(np.int64)].astype(np.float64), qn.astype(np.float64))
    return np.abs(sim.astype(np.float64) - s64)


def _check(index, m, q, k, path):
    idx, sim = index.search(q, k=k)
    st = index.last_search_stats()
    assert st["path"] == path and st["score_errors"] == 1, st
    got = index.last_score_errors(q.shape[0], k)
    want = _expected(m, q, idx, sim)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
    assert abs(st["max_score_error"] - want.max()) <= 1e-12
    assert abs(st["mean_score_error"] - want.mean()) <= 1e-12
    assert want.max() <= 1e-5  # the acceptance tolerance of every path
    return got


@pytest.mark.parametrize("nq,path", [(4, 1), (16, 6)])
def test_fp32_paths_report_their_errors(nq, path):
    rng = np.random.default_rng(5)
    m = rng.normal(size=(30_000, 200)).astype(np.float32)
    q = rng.normal(size=(nq, 200)).astype(np.float32)
    index = NNdex(m, autotune=False)
    index.set_error_report(True)
    got = _check(index, m, q, 25, path)
    assert np.count_nonzero(got) > 0  # FP32 accumulation leaves some error
    # off again: the next search records nothing
    index.set_error_report(False)
    index.search(q, k=25)
    assert index.last_search_stats()["score_errors"] == 0


def test_tensor_core_path_reports_its_errors():
    rng = np.random.default_rng(6)
    m = rng.normal(size=(40_000, 128)).astype(np.float32)
    q = rng.normal(size=(96, 128)).astype(np.float32)
    index = NNdex(m, precision="bf16", autotune=False)
    index.set_error_report(True)
    _check(index, m, q, 10, 2)


def test_ivf_path_reports_its_errors_and_short_lists_give_zero():
    rng = np.random.default_rng(7)
    m = rng.normal(size=(20_000, 64)).astype(np.float32)
    q = rng.normal(size=(8, 64)).astype(np.float32)
    index = NNdex(m, approx=True, nlist=64, kmeans_iters=3, seed=1, autotune=False)
    index.set_error_report(True)
    idx, sim = index.search(q, k=10)
    st = index.last_search_stats()
    assert st["path"] == 4 and st["score_errors"] == 1
    got = index.last_score_errors(8, 10)
    np.testing.assert_allclose(got, _expected(m, q, idx, sim), rtol=0, atol=1e-12)
