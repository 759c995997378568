"""Tensor-core (BF16 / FP8) scan + exact FP32 rerank against the oracle (needs a B200).

The low-precision paths must return the exact FP32 top-k (same acceptance rule as the FP32 path):
candidates are re-scored in FP32 and queries whose certificate fails are re-run on the FP32 scan.
The approximate candidate scores themselves must stay within the certificate's error bound.
"""
import numpy as np
import pytest

from nndex_b200 import NNdex
from oracle import oracle as O
from tests._parity import assert_topk_matches

pytestmark = pytest.mark.gpu


def mixture(rng, rows, dims, centers, sigma, center_seed=1234):
    # base and queries share the centres (same center_seed), as in the benchmark workloads
    c = np.random.default_rng(center_seed).normal(size=(centers, dims)).astype(np.float32)
    a = rng.integers(0, centers, size=rows)
    x = c[a] + np.float32(sigma) * rng.normal(size=(rows, dims)).astype(np.float32)
    return x.astype(np.float32)


def _check(index, m, queries, k, what):
    st, base = O.prepare_index(m, False)
    assert st == 0
    idx, sim = index.search(queries, k=k)
    _, qn = O.prepare_queries(queries, False, base.shape[1])
    for i in range(queries.shape[0]):
        assert_topk_matches(idx[i], sim[i], O.scores_f64(base, qn[i]), k, what=f"{what} q{i}")
    return base, qn, idx, sim


CASES = [
    # precision, rows, dims, nq, k, data
    ("bf16", 20_000, 128, 128, 10, "mixture"),
    ("bf16", 50_000, 256, 300, 10, "mixture"),
    ("bf16", 7_777, 100, 65, 5, "mixture"),
    ("bf16", 30_000, 64, 129, 16, "gauss"),
    ("fp8", 20_000, 128, 128, 10, "mixture"),
    ("fp8", 40_000, 256, 200, 10, "mixture"),
    ("fp8", 9_000, 200, 40, 8, "gauss"),
    # large D × large k: the pass-1 heaps only fit with the query slabs streamed per ring stage
    ("bf16", 20_000, 512, 100, 100, "mixture"),
    ("fp8", 20_000, 512, 100, 100, "mixture"),
    # D = 768: pass 2 streams the query slabs too
    ("bf16", 12_000, 768, 70, 100, "mixture"),
]


@pytest.mark.parametrize("precision,rows,dims,nq,k,data", CASES)
def test_low_precision_exact_topk(precision, rows, dims, nq, k, data):
    rng = np.random.default_rng(rows + dims + nq)
    if data == "mixture":
        m = mixture(rng, rows, dims, 256, 0.25)
        q = mixture(np.random.default_rng(7), nq, dims, 256, 0.25)
    else:
        m = rng.normal(size=(rows, dims)).astype(np.float32)
        q = rng.normal(size=(nq, dims)).astype(np.float32)
    index = NNdex(m, precision=precision)
    base, qn, idx, sim = _check(index, m, q, k, f"{precision} {rows}x{dims}")
    st = index.last_search_stats()
    assert st["path"] == (2 if precision == "bf16" else 3)
    assert st["rerank_width"] >= k
    # The certificate's premise: every candidate's ranking score is an upper bound of its exact
    # score, and not a loose one (within the worst-case bound of the quantisation).
    cidx, cbound, eps, cert = index.last_candidates(nq)
    assert eps > 0
    for i in range(min(nq, 32)):
        exact = O.scores_f64(base, qn[i])[cidx[i].astype(np.int64)]
        gap = cbound[i].astype(np.float64) - exact
        assert gap.min() >= -1e-6, (precision, gap.min())
        assert gap.max() <= 4 * eps + 1e-3, (precision, gap.max(), eps)


def test_bf16_threshold_pass_avoids_fp32_fallback():
    # Queries that pass 1 cannot certify are finished by the threshold pass, not the FP32 scan.
    rng = np.random.default_rng(3)
    m = mixture(rng, 60_000, 256, 512, 0.25)
    q = mixture(np.random.default_rng(4), 256, 256, 512, 0.25)
    index = NNdex(m, precision="bf16")
    _check(index, m, q, 10, "bf16 two-pass")
    st = index.last_search_stats()
    assert st["path"] == 2
    assert st["fp32_fallback_queries"] == 0, st


def test_fp8_exact_with_threshold_pass():
    # FP8's bound is wide: most queries take the threshold pass; results stay exact.
    rng = np.random.default_rng(11)
    m = rng.normal(size=(20_000, 64)).astype(np.float32)
    q = rng.normal(size=(64, 64)).astype(np.float32)
    index = NNdex(m, precision="fp8")
    _check(index, m, q, 10, "fp8 fallback")


def test_tc_matches_fp32_path():
    # the exact rerank and the FP32 scan select the same rows; scores agree within the tolerance
    rng = np.random.default_rng(5)
    m = mixture(rng, 30_000, 128, 128, 0.25)
    q = mixture(np.random.default_rng(6), 150, 128, 128, 0.25)
    index = NNdex(m, precision="bf16")
    ti, ts = index.search(q, k=10)
    index.set_precision("fp32")
    fi, fs = index.search(q, k=10)
    assert np.array_equal(ti, fi)
    assert np.max(np.abs(ts - fs)) <= 1e-5


def test_tc_alone_equals_in_batch():
    rng = np.random.default_rng(8)
    m = mixture(rng, 40_000, 128, 128, 0.25)
    q = mixture(np.random.default_rng(9), 200, 128, 128, 0.25)
    index = NNdex(m, precision="bf16")
    bi, bs = index.search(q, k=10)
    for lo in (0, 70, 190):
        si, ss = index.search(q[lo:lo + 5].copy(), k=10)
        assert np.array_equal(si, bi[lo:lo + 5])
        assert np.array_equal(ss, bs[lo:lo + 5])


def test_pass2_padding_lanes_ignore_stale_memory():
    # Pass 2 scores whole 128-query blocks; the lanes past the last uncertified query are padding.
    # Device memory freed by earlier work is refilled with BF16 +inf patterns first, so that new
    # scratch buffers are likely to start with them. Against a base of strictly positive values a
    # +inf query row scores +inf on every row. The padding lanes must still never survive: the
    # result equals the FP32 path's.
    import torch

    rng = np.random.default_rng(21)
    m = np.abs(mixture(rng, 40_000, 128, 128, 0.25)) + np.float32(0.05)
    q = np.abs(mixture(np.random.default_rng(22), 200, 128, 128, 0.25)) + np.float32(0.05)
    index = NNdex(m, precision="bf16", autotune=False)
    index.set_precision("fp32")
    fi, fs = index.search(q, k=10)
    junk = torch.full((1 << 29,), 0x7F80, dtype=torch.int16, device="cuda")  # 1 GiB of BF16 +inf
    torch.cuda.synchronize()
    del junk
    torch.cuda.empty_cache()
    index.set_precision("bf16", rerank_width=10)  # k' = k: most queries need pass 2
    ti, ts = index.search(q, k=10)
    st = index.last_search_stats()
    assert st["path"] == 2 and st["second_pass_queries"] > 0, st
    assert np.array_equal(ti, fi)
    assert np.max(np.abs(ts - fs)) <= 1e-5


def test_overflowing_collection_reruns_on_the_fp32_scan():
    # 10,000 copies of one row: pass 1 cannot certify (the k-th and k'-th scores tie), pass 2
    # collects every copy — more than its 8,192-row buffer — so the device marks each query for the
    # FP32 scan, which returns the lowest rows among the ties
    rng = np.random.default_rng(31)
    m = rng.normal(size=(30_000, 64)).astype(np.float32)
    m[10_000:20_000] = m[10_000]
    q = (np.repeat(m[10_000:10_001], 130, axis=0) + np.float32(1e-3) * rng.normal(size=(130, 64))).astype(np.float32)
    index = NNdex(m, precision="bf16", autotune=False)
    ti, ts = index.search(q, k=10)
    st = index.last_search_stats()
    assert st["path"] == 2 and st["second_pass_queries"] == 130 and st["fp32_fallback_queries"] == 130, st
    assert ti[0].tolist() == list(range(10_000, 10_010))
    index.set_precision("fp32")
    fi, fs = index.search(q, k=10)
    np.testing.assert_array_equal(ti, fi)
    np.testing.assert_array_equal(ts.view(np.uint32), fs.view(np.uint32))


@pytest.mark.parametrize("precision,certifying,uncertified,qb", [
    ("bf16", 250, 50, 2),    # 50 live queries of 300: the CTA's second query block is empty
    ("bf16", 100, 200, 2),   # 200 live: the second block is partly filled
    ("bf16", 100, 600, 2),   # 600 live: three CTA query pairs, the last with one block
    ("bf16", 100, 200, 1),
    ("fp8", 150, 170, 2),
    ("fp8", 150, 170, 1),
    ("bf16", 250, 50, 3),    # CTA pairs: one pair, the odd CTA's block empty
    ("bf16", 100, 200, 3),   # one pair, both blocks partly filled
    ("bf16", 100, 600, 3),   # five blocks: three pairs, the last CTA's block empty
    ("fp8", 150, 170, 3),
])
def test_pass2_query_blocks_per_cta(precision, certifying, uncertified, qb):
    # Pass 2 of a batch of more than 128 queries can put two query blocks in each CTA against
    # 128-row base tiles, or run CTA pairs (qb 3: one block per CTA, M = 256 MMAs over both CTAs'
    # shared memory, each CTA loading half of every 256-row tile) — the plan's qb, fixed here
    # through the autotuner's cache. The number of live queries decides on the device how many
    # blocks (or pairs) there are; a block without queries still loads its half of the tiles. Queries equal
    # to a base row of a mixture certify in pass 1 (their top-1 scores 1, their cluster about 0.94);
    # a query with 40 near-duplicate rows (scores about 1e-4 apart, inside the bound slack) cannot
    # certify with k' = 32 and takes pass 2. Results equal the oracle's and the FP32 path's.
    rng = np.random.default_rng(certifying + uncertified)
    dims = 128
    mix = mixture(rng, 8_000, dims, 256, 0.25)
    vs = rng.normal(size=(100, dims)).astype(np.float32)
    groups = (np.repeat(vs, 40, axis=0) + np.float32(1e-2) * rng.normal(size=(4_000, dims))).astype(np.float32)
    m = np.concatenate([mix, groups]).astype(np.float32)
    q = np.concatenate([mix[rng.choice(8_000, certifying, replace=False)],
                        vs[rng.integers(0, 100, size=uncertified)]]).astype(np.float32)
    q = q[rng.permutation(q.shape[0])].copy()
    index = NNdex(m, precision=precision)
    code = 2 if precision == "bf16" else 3
    nqb = 1 << (q.shape[0] - 1).bit_length()
    index.autotune_import(index.autotune_export() +
                          f"shape ivf=0 nq={nqb} k=1 precision={code} nprobe=0 plan path={code} stride=1 qb={qb} ms=0\n")
    _check(index, m, q, 1, f"{precision} pass 2 with {qb} query blocks per CTA")
    st = index.last_search_stats()
    # (FP8's wider bound may leave a few of the other queries uncertified too)
    if precision == "bf16":
        assert st["second_pass_queries"] == uncertified, st
    else:
        assert uncertified <= st["second_pass_queries"] <= uncertified + certifying // 10, st
    assert st["pass2_query_blocks"] == qb and st["tuned"] == 2, st
    assert st["fp32_fallback_queries"] == 0, st
    ti, ts = index.search(q, k=1)
    index.set_precision("fp32")
    fi, fs = index.search(q, k=1)
    np.testing.assert_array_equal(ti, fi)
    np.testing.assert_array_equal(ts.view(np.uint32), fs.view(np.uint32))
