"""Parity at the benchmark shapes themselves (needs a B200; each case holds a few to ~40 GB of HBM).

The smaller parity tests fix the algorithms; these check that the numbers the benchmark reports
rest on correct results at their own sizes:

* 1,000,000 × 768 mixture (1,024 centres, sigma 0.3, unit rows, normalized=true), k = 100, batches
  of 1, 4 and 16: every query against the FP64 scores of the whole base (the acceptance rule of
  tests/_parity.py).
* 10,000,000 × 256 mixture (4,096 centres, sigma 0.25) with BF16 and FP8-E4M3 scoring copies, one
  batch of 4,096 queries, k = 10: both tensor-core paths return the FP32 scan's rows and scores bit
  for bit, and every query meets the acceptance rule against an FP64 brute force (recall@10 = 1).
* 2,000,000 × 384 Zipf(1.1) mixture (8,192 centres), IVF nlist 1,414, 10 k-means iterations,
  seed 42: the k-means++ picks against the restated reference, the last assignment of every row
  against the restated argmax over the ninth iteration's centroids, the centroids bit for bit
  against the restated update, the list layout against a stable counting sort, and approx
  searches at nprobe 8, 32 and 64 against the restated reference search over the same lists.

Data comes from the benchmark's own seeded generator (bench.make_mixture) on the GPU.
"""
import ctypes as C

import numpy as np
import pytest

from nndex_b200 import NNdex, _lib
from nndex_b200._lib import NNDEX_FLAG_APPROX, NNDEX_FLAG_BF16, NNDEX_FLAG_FP8, NNDEX_FLAG_NORMALIZED
from oracle import oracle as O
from tests._parity import TOL, assert_topk_matches

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _mixture(rows, dims, centers, sigma, seed, zipf=None):
    import bench
    return bench.make_mixture(rows, dims, centers, sigma, seed, torch.device("cuda", 0), center_seed=seed,
                              zipf=zipf)


def _index_from_device(base, flags, nlist=0, iters=0, seed=None):
    rows, dims = base.shape
    opts = _lib.Opts()
    opts.device = 0
    opts.nlist = nlist
    opts.kmeans_iters = iters
    opts.has_seed = 0 if seed is None else 1
    opts.seed = 0 if seed is None else seed
    h = C.c_void_p()
    st = _lib.lib().nndex_cuda_create_from_device(base.data_ptr(), base.numel(), rows, dims, flags, C.byref(opts),
                                                  C.byref(h))
    assert st == 0, _lib.last_error()
    ix = NNdex.__new__(NNdex)
    ix._h = None
    ix._adopt(h, rows, dims, bool(flags & NNDEX_FLAG_NORMALIZED), bool(flags & NNDEX_FLAG_APPROX), True)
    return ix


def _fp64_topk(base, queries, width, chunk=1 << 17):
    """FP64 brute force on the GPU: the `width` best rows of every query (scores descending)."""
    q64 = queries.double()
    best_s = best_i = None
    for r0 in range(0, base.shape[0], chunk):
        s = q64 @ base[r0:r0 + chunk].double().T
        v, i = torch.topk(s, min(width, s.shape[1]), dim=1)
        i += r0
        if best_s is None:
            best_s, best_i = v, i
        else:
            v2, j = torch.topk(torch.cat([best_s, v], 1), width, dim=1)
            best_i = torch.gather(torch.cat([best_i, i], 1), 1, j)
            best_s = v2
        del s
    return best_s.cpu().numpy(), best_i.cpu().numpy()


def _fp64_scores_of(base, queries, idx):
    """FP64 score of each (query, returned row) pair."""
    rows = base[torch.from_numpy(idx.astype(np.int64)).to(base.device)].double()  # nq × k × D
    return torch.einsum("qkd,qd->qk", rows, queries.double()).cpu().numpy()


def _assert_sparse_rule(gidx, gsim, ret64, ref_s, ref_i, k, what):
    """The acceptance rule of tests/_parity.py from the FP64 top-(k + extra) and the FP64 scores of
    the returned rows: scores within TOL, result order, no row below the k-th, every row clearly in
    the top-k returned, and isolated ranks at their exact position."""
    gidx = np.asarray(gidx, np.int64)
    gsim = np.asarray(gsim, np.float64)
    assert len(set(gidx.tolist())) == k, f"{what}: duplicate rows"
    err = np.abs(gsim - ret64)
    assert np.all(err <= TOL), f"{what}: score error {err.max():.3g}"
    for j in range(k - 1):
        a, b = gsim[j], gsim[j + 1]
        assert a > b or (a == b and gidx[j] < gidx[j + 1]), f"{what}: order broken at {j}"
    kth, nxt = ref_s[k - 1], ref_s[k]
    assert np.all(ret64 >= kth - TOL), f"{what}: a returned row is below the k-th score"
    must = ref_i[:k][ref_s[:k] > nxt + TOL]
    missing = set(must.tolist()) - set(gidx.tolist())
    assert not missing, f"{what}: rows {sorted(missing)[:10]} missing"
    for j in range(k):
        lo_ok = j == 0 or ref_s[j - 1] - ref_s[j] > TOL
        hi_ok = ref_s[j] - ref_s[j + 1] > TOL
        if lo_ok and hi_ok:
            assert gidx[j] == ref_i[j], f"{what}: position {j}: row {gidx[j]}, expected {ref_i[j]}"


def test_exact_fp32_1M_x_768_k100_batches_1_4_16():
    rows, dims, k = 1_000_000, 768, 100
    base = _mixture(rows, dims, 1024, 0.3, 42)
    index = _index_from_device(base, NNDEX_FLAG_NORMALIZED)
    # the benchmark draws its queries from a second generator over the same centres
    import bench
    qall = bench.make_mixture(21, dims, 1024, 0.3, 49, torch.device("cuda", 0), center_seed=42)
    s64 = (base.double() @ qall.double().T).cpu().numpy()  # rows × 21
    qh = qall.cpu().numpy()
    lo = 0
    paths = {}
    for b in (1, 4, 16):
        gi, gs = index.search(qh[lo:lo + b] if b > 1 else qh[lo], k=k)
        paths[b] = index.last_search_stats()["path"]
        gi = np.atleast_2d(gi)
        gs = np.atleast_2d(gs)
        for j in range(b):
            assert_topk_matches(gi[j], gs[j], s64[:, lo + j], k, what=f"batch {b} query {j}")
        lo += b
    assert paths[16] in (1, 6), paths


@pytest.mark.parametrize("precision", ["bf16", "fp8"])
def test_mixed_precision_10M_x_256_4096_queries(precision, c3_case):
    index, base, q, fp32_idx, fp32_sim, ref_s, ref_i = c3_case
    index.set_precision(precision)
    gi, gs = index.search(q.cpu().numpy(), k=10)
    st = index.last_search_stats()
    assert st["path"] == (2 if precision == "bf16" else 3), st
    # the certified results and the second pass rerank in the FP32 scan's order: identical bits
    np.testing.assert_array_equal(gi, fp32_idx)
    np.testing.assert_array_equal(gs.view(np.uint32), fp32_sim.view(np.uint32))


@pytest.fixture(scope="module")
def c3_case():
    rows, dims, nq, k = 10_000_000, 256, 4096, 10
    base = _mixture(rows, dims, 4096, 0.25, 42)
    index = _index_from_device(base, NNDEX_FLAG_NORMALIZED | NNDEX_FLAG_BF16 | NNDEX_FLAG_FP8)
    import bench
    q = bench.make_mixture(nq, dims, 4096, 0.25, 49, torch.device("cuda", 0), center_seed=42)
    index.set_precision("fp32")
    fi, fs = index.search(q.cpu().numpy(), k=k)
    ref_s, ref_i = _fp64_topk(base, q, k + 6)
    ret64 = _fp64_scores_of(base, q, fi)
    # the FP32 scan itself against FP64, every query: recall@10 = 1 wherever the gap rule applies
    for j in range(nq):
        _assert_sparse_rule(fi[j], fs[j], ret64[j], ref_s[j], ref_i[j], k, what=f"fp32 query {j}")
    yield index, base, q, fi, fs, ref_s, ref_i
    del index, base


def _ivf_index(base, iters):
    return _index_from_device(base, NNDEX_FLAG_NORMALIZED | NNDEX_FLAG_APPROX, nlist=1414, iters=iters, seed=42)


def test_ivf_build_2M_x_384_nlist1414_matches_reference_steps():
    rows, dims, nlist = 2_000_000, 384, 1414
    base = _mixture(rows, dims, 8192, 0.25, 42, zipf=1.1)
    ix10 = _ivf_index(base, 10)
    lay10 = ix10.ivf_layout()
    del ix10
    ix9 = _ivf_index(base, 9)
    lay9 = ix9.ivf_layout()
    del ix9
    host = base.cpu().numpy()
    assert lay10["centroids"].shape == (nlist, dims)
    # k-means++: both builds pick the same rows; the first 16 picks are the restated reference's
    np.testing.assert_array_equal(lay10["init_rows"], lay9["init_rows"])
    chosen, _ = O.kmeans_plusplus_init(host, 16, seed=42)
    np.testing.assert_array_equal(lay10["init_rows"][:16], chosen)
    # the last assignment (iteration 10) against the ninth iteration's centroids, every row:
    # FP64 scores on the GPU rounded to f32 decide rows whose best two differ by more than two
    # ulps (the restated dot can differ from them by one ulp); the rest run the restated argmax
    assign = np.empty(rows, np.uint32)
    off = lay10["cluster_offsets"].astype(np.int64)
    orig = lay10["original_indices"].astype(np.int64)
    for c in range(nlist):
        assign[orig[off[c]:off[c + 1]]] = c
    c9 = torch.from_numpy(lay9["centroids"]).cuda().double()
    ambiguous = []
    for r0 in range(0, rows, 1 << 17):
        s = (base[r0:r0 + (1 << 17)].double() @ c9.T).float()
        top2, arg = torch.topk(s, 2, dim=1)
        first = torch.argmax(s, dim=1)  # the lowest index among equal maxima
        gap = top2[:, 0] - top2[:, 1]
        ulp = torch.abs(top2[:, 0]) * 2.0 ** -23 + 2.0 ** -149
        sure = gap > 2 * ulp
        got = torch.from_numpy(assign[r0:r0 + (1 << 17)].astype(np.int64)).cuda()
        bad = sure & (first != got)
        assert not bool(bad.any()), f"rows {(torch.nonzero(bad)[:5, 0] + r0).tolist()} assigned off the argmax"
        ambiguous.append((torch.nonzero(~sure)[:, 0] + r0).cpu().numpy())
    amb = np.concatenate(ambiguous)
    if amb.size:
        exact = O.kmeans_assign_rows(host, amb, lay9["centroids"])
        np.testing.assert_array_equal(exact, assign[amb])
    # the centroids after the last update, bit for bit
    cent = O.kmeans_update(host, assign, nlist)
    np.testing.assert_array_equal(lay10["centroids"].view(np.uint32), cent.view(np.uint32))
    # the list layout: a stable counting sort of the assignment
    np.testing.assert_array_equal(orig, np.argsort(assign, kind="stable"))
    np.testing.assert_array_equal(off, np.concatenate([[0], np.cumsum(np.bincount(assign, minlength=nlist))]))

    # approx searches over the same lists: the restated reference search on the GPU's layout
    ix = _ivf_index(base, 10)
    import bench
    q = bench.make_mixture(48, dims, 8192, 0.25, 49, torch.device("cuda", 0), center_seed=42, zipf=1.1)
    qh = q.cpu().numpy()
    ref = O.IvfIndex(host, layout=lay10)
    exact_s, exact_i = _fp64_topk(base, q, 10)
    for nprobe in (8, 32, 64):
        ix.set_nprobe(nprobe)
        gi, gs = ix.search(qh, k=10)
        ri, rs, _ = ref.search(qh, 10, nprobe=nprobe)
        rec_gpu = rec_ref = 0
        for j in range(len(qh)):
            probed, _ = ref.probe(qh[j], nprobe)
            rows_p = np.concatenate([orig[off[c]:off[c + 1]] for c in probed.astype(np.int64)])
            s64 = np.full(rows, -np.inf)
            s64[rows_p] = host[rows_p].astype(np.float64) @ qh[j].astype(np.float64)
            assert_topk_matches(gi[j], gs[j], s64, 10, what=f"nprobe {nprobe} query {j}")
            rec_gpu += len(set(gi[j].tolist()) & set(exact_i[j].tolist()))
            rec_ref += len(set(ri[j].astype(np.int64).tolist()) & set(exact_i[j].tolist()))
        assert rec_gpu >= rec_ref, (nprobe, rec_gpu, rec_ref)
