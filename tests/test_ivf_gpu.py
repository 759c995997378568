"""IVF build and search on the GPU against the oracle's restatement of src/approx.rs (needs a B200).

The build must reproduce the reference's index exactly: the rows k-means++ picks, every centroid
(bit for bit), the cluster offsets and the reordered row order. Searches then probe the same lists,
and the returned rows must be the exact top-k of the probed rows (scores within 1e-5 of FP64,
indices exact wherever the FP64 gap exceeds 1e-5).
"""
import numpy as np
import pytest

from nndex_b200 import NNdex
from oracle import oracle as O
from tests._parity import assert_topk_matches

pytestmark = pytest.mark.gpu


def mixture(rng, rows, dims, centers, sigma, zipf=None, center_seed=99):
    c = np.random.default_rng(center_seed).normal(size=(centers, dims)).astype(np.float32)
    if zipf:
        w = 1.0 / np.arange(1, centers + 1) ** zipf
        a = rng.choice(centers, size=rows, p=w / w.sum())
    else:
        a = rng.integers(0, centers, size=rows)
    return (c[a] + np.float32(sigma) * rng.normal(size=(rows, dims)).astype(np.float32)).astype(np.float32)


def unit(x):
    return (x / np.linalg.norm(x.astype(np.float64), axis=1, keepdims=True)).astype(np.float32)


BUILD_CASES = [
    # name, rows, dims, nlist, iters, seed, normalized, data
    ("mixture", 20_000, 64, 64, 5, 42, False, "mixture"),
    ("policy", 12_000, 100, 0, 3, None, False, "gauss"),
    ("prenormalized", 8_000, 48, 40, 4, 7, True, "mixture"),
    ("zipf", 30_000, 96, 150, 4, 42, False, "zipf"),
    ("duplicates", 600, 32, 16, 3, 5, False, "dups"),
]


def make_data(kind, rows, dims, seed=0):
    rng = np.random.default_rng(seed + rows + dims)
    if kind == "mixture":
        return mixture(rng, rows, dims, 128, 0.3)
    if kind == "zipf":
        return mixture(rng, rows, dims, 512, 0.25, zipf=1.1)
    if kind == "dups":
        base = rng.normal(size=(5, dims)).astype(np.float32)
        return base[rng.integers(0, 5, size=rows)]
    return rng.normal(size=(rows, dims)).astype(np.float32)


_cache = {}


def built(case):
    name, rows, dims, nlist, iters, seed, normalized, kind = case
    if name not in _cache:
        m = make_data(kind, rows, dims)
        if normalized:
            m = unit(m)
        index = NNdex(m, normalized=normalized, approx=True, nlist=nlist, kmeans_iters=iters, seed=seed)
        st, storage = O.prepare_index(m, normalized)
        assert st == 0
        ref = O.IvfIndex(storage, nlist=nlist, iters=iters, seed=seed)
        _cache[name] = (m, index, storage, ref)
    return _cache[name]


@pytest.mark.parametrize("case", BUILD_CASES, ids=[c[0] for c in BUILD_CASES])
def test_ivf_build_matches_oracle(case):
    m, index, storage, ref = built(case)
    lay = index.ivf_layout()
    assert lay is not None
    assert lay["centroids"].shape[0] == ref.nlist
    np.testing.assert_array_equal(lay["init_rows"], ref.init_rows)
    np.testing.assert_array_equal(lay["cluster_offsets"], ref.offsets)
    np.testing.assert_array_equal(lay["original_indices"], ref.original_indices)
    # bit-for-bit centroids (FP64 sums in row order, Rust's rounding of every step)
    np.testing.assert_array_equal(lay["centroids"].view(np.uint32), ref.centroids.view(np.uint32))
    st = index.ivf_stats()
    assert st["nlist"] == ref.nlist and st["build_ms"] > 0


def probed_rows(ref, q, nprobe):
    cl, _ = ref.probe(q, nprobe)
    off, orig = ref.offsets, ref.original_indices
    rows = np.concatenate([orig[int(off[c]):int(off[c + 1])] for c in cl]) if len(cl) else np.zeros(0, np.uint64)
    return np.sort(rows.astype(np.int64))


def check_against_probed(ref, storage, qn, idx, sim, cnt, k, nprobe, what):
    cand = probed_rows(ref, qn, nprobe)
    s64 = O.scores_f64(storage, qn)[cand]
    n = min(k, cand.shape[0])
    assert int(cnt) == n, f"{what}: count {cnt} vs {n} probed-limited results"
    pos = np.searchsorted(cand, idx[:n].astype(np.int64))
    assert np.all(cand[np.minimum(pos, len(cand) - 1)] == idx[:n].astype(np.int64)), f"{what}: row outside the probed lists"
    assert_topk_matches(pos, sim[:n], s64, k, what=what)


@pytest.mark.parametrize("name", ["mixture", "policy", "zipf"])
@pytest.mark.parametrize("nprobe", [0, 3, 9])
@pytest.mark.parametrize("k", [1, 10])
def test_ivf_search_matches_oracle(name, nprobe, k):
    case = next(c for c in BUILD_CASES if c[0] == name)
    m, index, storage, ref = built(case)
    q = make_data("mixture" if name != "policy" else "gauss", 37, m.shape[1], seed=5)
    index.set_nprobe(nprobe)
    try:
        gi, gs = index.search(q, k=k)
        st = index.last_search_stats()
    finally:
        index.set_nprobe(0)
    assert st["path"] == 4
    assert st["ivf_rows_union"] <= st["ivf_rows_streamed"] and st["rows_scanned"] > 0
    eff_np = nprobe if nprobe else O.choose_nprobe(ref.nlist, min(k, m.shape[0]), m.shape[0])
    assert st["nprobe"] == min(eff_np, ref.nlist)
    _, qn = O.prepare_queries(q, False, storage.shape[1])
    ri, rs, rc = ref.search(qn, k, nprobe)
    for i in range(q.shape[0]):
        cnt = int(rc[i])
        check_against_probed(ref, storage, qn[i], gi[i], gs[i], cnt, k, min(eff_np, ref.nlist), f"{name} q{i}")


def test_ivf_scores_bitwise_equal_to_exact_path():
    case = BUILD_CASES[0]
    m, index, storage, ref = built(case)
    exact = NNdex(m)
    q = make_data("mixture", 25, m.shape[1], seed=11)
    ai, asim = index.search(q, k=10)
    ei, esim = exact.search(q, k=10)
    shared = 0
    for i in range(q.shape[0]):
        e = dict(zip(ei[i].tolist(), esim[i].tolist()))
        for r, s in zip(ai[i].tolist(), asim[i].tolist()):
            if r in e:
                assert np.float32(s).view(np.uint32) == np.float32(e[r]).view(np.uint32)
                shared += 1
    assert shared > 100


def test_ivf_batch_equals_single():
    # src/lib.rs:1205-1297 batch_approx_matches_single_approx_results
    case = BUILD_CASES[0]
    m, index, storage, ref = built(case)
    q = make_data("mixture", 12, m.shape[1], seed=23)
    bi, bs = index.search(q, k=10)
    for i in range(q.shape[0]):
        si, ss = index.search(q[i], k=10)
        # same rows in the same order; scores within the reference's 1e-4 (a single query is
        # normalised by normalize_vector, a batch by normalize_rows: they may differ by an ulp)
        np.testing.assert_array_equal(si, bi[i])
        assert np.max(np.abs(ss - bs[i])) < 1e-4


def test_ivf_recall_equals_reference_approx():
    # src/lib.rs:962-1021 (4096 × 64 uniform(-1, 1), k = 20, reference nlist/nprobe policy). The
    # reference asserts ≥ 14 of 20 for one ChaCha8 draw, which numpy cannot reproduce; on numpy draws
    # of the same distribution the restated reference IVF keeps ≈ 11 of 20 on average. The GPU index
    # is the same index, so its overlap equals the restatement's on every draw (the acceptance bar:
    # recall no lower than the reference approx mode at the same nlist/nprobe/seed).
    gpu, ref_ov = [], []
    for seed in range(6):
        rng = np.random.default_rng(seed)
        m = rng.uniform(-1, 1, size=(4096, 64)).astype(np.float32)
        q = rng.uniform(-1, 1, size=(64,)).astype(np.float32)
        ai, _ = NNdex(m, approx=True).search(q, k=20)
        ei, _ = NNdex(m).search(q, k=20)
        st, storage = O.prepare_index(m, False)
        ref = O.IvfIndex(storage)
        _, qn = O.prepare_queries(q.reshape(1, -1), False, storage.shape[1])
        ri, _, _ = ref.search(qn, 20, 0)
        exact = set(ei.tolist())
        gpu.append(len(set(ai.tolist()) & exact))
        ref_ov.append(len(set(ri[0].tolist()) & exact))
        assert ai[0] in exact
    assert gpu == ref_ov, (gpu, ref_ov)
    assert np.mean(gpu) >= 10


def test_ivf_small_index_answers_exactly():
    # rows < 256: a single list, no speedup → exact results (src/approx.rs:49-59, src/cpu.rs:399-407)
    rng = np.random.default_rng(3)
    m = rng.normal(size=(200, 16)).astype(np.float32)
    q = rng.normal(size=(5, 16)).astype(np.float32)
    a = NNdex(m, approx=True)
    assert a.ivf_layout() is None
    ai, asim = a.search(q, k=7)
    ei, esim = NNdex(m).search(q, k=7)
    np.testing.assert_array_equal(ai, ei)
    np.testing.assert_array_equal(asim, esim)
    assert a.last_search_stats()["path"] == 1


def test_ivf_probed_fewer_rows_than_k():
    # one probed list smaller than k: the result holds the probed rows only (count < k)
    case = BUILD_CASES[0]
    m, _, storage, ref = built(case)
    # nprobe given at construction (an option the reference's IndexOptions does not have)
    idx_obj = NNdex(m, approx=True, nlist=case[3], kmeans_iters=case[4], seed=case[5], nprobe=1)
    sizes = np.diff(ref.offsets.astype(np.int64))
    k = int(sizes.max()) + 5
    q = make_data("mixture", 4, m.shape[1], seed=31)
    _, qn = O.prepare_queries(q, False, storage.shape[1])
    ri, rs, rc = ref.search(qn, k, 1)
    for i in range(4):
        gi, gs = idx_obj.search(q[i], k=k)
        n = int(rc[i])
        assert n < k and gi.shape[0] == n
        check_against_probed(ref, storage, qn[i], gi, gs, n, k, 1, f"small-list q{i}")


TC_CASES = [
    # name, rows, dims, nlist, nq, k, nprobe
    ("mixture", 20_000, 64, 64, 300, 10, 0),  # ≈ 14 queries per probed list: the tensor-core scan
    ("mixture", 20_000, 64, 64, 150, 1, 9),
    ("zipf", 30_000, 96, 150, 300, 100, 0),
    ("multichunk", 60_000, 128, 8, 96, 10, 3),  # lists of ≈ 7,500 rows: two 4,096-row chunks each
]


@pytest.mark.parametrize("name,rows,dims,nlist,nq,k,nprobe", TC_CASES)
def test_ivf_tensor_core_scan_equals_fp32_scan(name, rows, dims, nlist, nq, k, nprobe):
    # the tensor-core list scan (certified BF16 candidates + exact FP32 rerank) returns the FP32 list
    # scan's result: the same probed rows, the same exact scores, bit for bit
    m = make_data("zipf" if name == "zipf" else "mixture", rows, dims)
    index = NNdex(m, approx=True, precision="auto", nlist=nlist, kmeans_iters=3, seed=42, nprobe=nprobe, autotune=False)
    q = make_data("mixture", nq, dims, seed=13)
    ti, ts = index.search(q, k=k)
    st = index.last_search_stats()
    assert st["path"] == 5, st
    # again: pass 1 may now run on a sample of each list's tiles (autotuned); same result
    ti2, ts2 = index.search(q, k=k)
    index.set_precision("fp32")
    fi, fs = index.search(q, k=k)
    assert index.last_search_stats()["path"] == 4
    for gi, gs in ((ti, ts), (ti2, ts2)):
        np.testing.assert_array_equal(gi, fi)
        np.testing.assert_array_equal(gs.view(np.uint32), fs.view(np.uint32))
    # and against the oracle's probed lists
    st_, storage = O.prepare_index(m, False)
    ref = O.IvfIndex(storage, nlist=nlist, iters=3, seed=42)
    _, qn = O.prepare_queries(q, False, storage.shape[1])
    eff = nprobe if nprobe else O.choose_nprobe(ref.nlist, k, rows)
    _, _, rc = ref.search(qn, k, nprobe)
    for i in range(0, nq, 7):
        check_against_probed(ref, storage, qn[i], ti[i], ts[i], int(rc[i]), k, min(eff, ref.nlist), f"{name} q{i}")
