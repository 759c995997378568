"""TF32 candidate scan (batches of 9-16 queries of an FP32 index) against the FP32 scan and the
FP64 oracle (needs a B200).

Batches of 9 to 16 queries take the tensor-core candidate scan (one TF32 product per row and
query, ranked by an upper bound) with the exact rerank; batches of 8 or fewer take the FP32 scan. A
certified query's rows and scores are the FP32 scan's, bit for bit (the rerank sums in the FP32
scan's order); an uncertified one is re-run on the FP32 scan. So each query of a 16-query batch
must equal its result from two 8-query batches, bit for bit.
"""
import numpy as np
import pytest

from nndex_b200 import NNdex
from oracle import oracle as O
from tests._parity import assert_topk_matches

pytestmark = pytest.mark.gpu


def mixture(rng, rows, dims, centers, sigma, center_seed=77):
    c = np.random.default_rng(center_seed).normal(size=(centers, dims)).astype(np.float32)
    a = rng.integers(0, centers, size=rows)
    return (c[a] + np.float32(sigma) * rng.normal(size=(rows, dims)).astype(np.float32)).astype(np.float32)


CASES = [
    # rows, dims, nq, k, data
    (200_000, 768, 16, 100, "mixture"),
    (100_003, 256, 16, 10, "mixture"),
    (50_000, 100, 9, 1, "gauss"),      # dims padded to 128, 9 queries
    (30_001, 128, 13, 128, "gauss"),   # rows not a multiple of the 128-row tile, largest k
]


@pytest.mark.parametrize("rows,dims,nq,k,data", CASES)
def test_tf32_scan_equals_fp32_scan(rows, dims, nq, k, data):
    rng = np.random.default_rng(rows + dims)
    if data == "mixture":
        m = mixture(rng, rows, dims, 256, 0.3)
        q = mixture(np.random.default_rng(5), nq, dims, 256, 0.3)
    else:
        m = rng.normal(size=(rows, dims)).astype(np.float32)
        q = rng.normal(size=(nq, dims)).astype(np.float32)
    index = NNdex(m, autotune=False)
    ti, ts = index.search(q, k=k)
    st = index.last_search_stats()
    assert st["path"] == 6, st
    assert st["rerank_width"] >= k
    parts = [index.search(q[lo:lo + 8].copy(), k=k) for lo in range(0, nq, 8)]
    assert index.last_search_stats()["path"] == 1
    fi = np.vstack([p[0] for p in parts])
    fs = np.vstack([p[1] for p in parts])
    np.testing.assert_array_equal(ti, fi)
    np.testing.assert_array_equal(ts.view(np.uint32), fs.view(np.uint32))
    # and against the FP64 oracle on a few queries
    _, base = O.prepare_index(m, False)
    _, qn = O.prepare_queries(q, False, base.shape[1])
    for i in range(0, nq, 4):
        assert_topk_matches(ti[i], ts[i], O.scores_f64(base, qn[i]), k, what=f"tf32 q{i}")


def test_tf32_scan_certifies_the_benchmark_mixture():
    # the C2 distribution (1,024 centres, sigma 0.3, unit rows) at k = 100: every query certifies,
    # so no FP32 re-run
    rng = np.random.default_rng(12)
    m = mixture(rng, 300_000, 768, 1024, 0.3, center_seed=1)
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    q = mixture(np.random.default_rng(13), 16, 768, 1024, 0.3, center_seed=1)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    index = NNdex(m, normalized=True, autotune=False)
    index.search(q, k=100)
    st = index.last_search_stats()
    assert st["path"] == 6 and st["fp32_fallback_queries"] == 0, st


def _equal_to_fp32_scan(index, q, k):
    ti, ts = index.search(q, k=k)
    st = index.last_search_stats()
    parts = [index.search(q[lo:lo + 8].copy(), k=k) for lo in range(0, len(q), 8)]
    assert index.last_search_stats()["path"] == 1
    np.testing.assert_array_equal(ti, np.vstack([p[0] for p in parts]))
    np.testing.assert_array_equal(ts.view(np.uint32), np.vstack([p[1] for p in parts]).view(np.uint32))
    return st


def test_tf32_scan_bound_follows_row_and_query_norms():
    # normalized=true keeps the caller's rows and queries as they are: norms from 0.01 to 100, so
    # the bound must scale with ‖q‖‖x‖ (a unit-norm bound would drop true neighbours)
    rng = np.random.default_rng(31)
    m = mixture(rng, 60_000, 192, 128, 0.3)
    m *= (10.0 ** rng.uniform(-2, 2, size=(60_000, 1))).astype(np.float32)
    q = mixture(np.random.default_rng(32), 16, 192, 128, 0.3)
    q *= (10.0 ** np.random.default_rng(33).uniform(-2, 2, size=(16, 1))).astype(np.float32)
    index = NNdex(m, normalized=True, autotune=False)
    st = _equal_to_fp32_scan(index, q, 50)
    assert st["path"] == 6, st


def test_tf32_scan_ties_fall_back_to_the_fp32_scan():
    # 3,000 copies of one row: the k-th and the k'-th scores are equal, the certificate cannot
    # hold, and the queries are re-run on the FP32 scan (lowest row index first among the ties)
    rng = np.random.default_rng(41)
    m = rng.normal(size=(20_000, 64)).astype(np.float32)
    m[5_000:8_000] = m[5_000]
    q = np.repeat(m[5_000:5_001], 12, axis=0) + np.float32(1e-3) * rng.normal(size=(12, 64)).astype(np.float32)
    index = NNdex(m, autotune=False)
    st = _equal_to_fp32_scan(index, q, 20)
    assert st["path"] == 6 and st["fp32_fallback_queries"] == 12, st
    ti, _ = index.search(q, k=20)
    assert ti[0].tolist() == list(range(5_000, 5_020))


@pytest.mark.parametrize("k", [10, 100])
def test_tf32_scan_rows_sorted_by_cluster(k):
    # Each CTA lists a quarter of k′ per query; rows outside the lists are covered by the floor
    # (the largest full-list minimum) in the certificate. With the base sorted by cluster, a query's
    # neighbours crowd into a few CTAs, whose lists leave true candidates out: the results must
    # still equal the FP32 scan's, bit for bit, certified or re-run.
    rng = np.random.default_rng(61 + k)
    centers = np.random.default_rng(62).normal(size=(64, 256)).astype(np.float32)
    assign = np.sort(rng.integers(0, 64, size=150_000))
    m = (centers[assign] + np.float32(0.2) * rng.normal(size=(150_000, 256)).astype(np.float32)).astype(np.float32)
    q = (centers[rng.integers(0, 64, size=16)] + np.float32(0.2) * rng.normal(size=(16, 256))).astype(np.float32)
    index = NNdex(m, autotune=False)
    st = _equal_to_fp32_scan(index, q, k)
    assert st["path"] == 6, st
    # and against the FP64 oracle
    idx, sim = index.search(q, k=k)
    stb, base = O.prepare_index(m, False)
    assert stb == 0
    _, qn = O.prepare_queries(q, False, base.shape[1])
    for i in range(q.shape[0]):
        assert_topk_matches(idx[i], sim[i], O.scores_f64(base, qn[i]), k, what=f"sorted k={k} q{i}")
