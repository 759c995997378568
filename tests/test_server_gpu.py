"""Serving loop (continuous batching) on the GPU: every request's result is the same alone and in the
mix; admission by memory and queue bounds; a bad request fails alone (needs a B200)."""
import numpy as np
import pytest

from nndex_b200 import NNdex, NNdexError, Server
from nndex_b200._lib import NNDEX_ERR_ADMISSION, NNDEX_ERR_NON_FINITE

pytestmark = pytest.mark.gpu


def mixture(rng, rows, dims, centers=64, sigma=0.3, center_seed=5):
    c = np.random.default_rng(center_seed).normal(size=(centers, dims)).astype(np.float32)
    a = rng.integers(0, centers, size=rows)
    return (c[a] + np.float32(sigma) * rng.normal(size=(rows, dims)).astype(np.float32)).astype(np.float32)


@pytest.fixture(scope="module")
def index():
    rng = np.random.default_rng(1)
    m = mixture(rng, 60_000, 96)
    # approx builds the IVF; precision "auto" keeps a BF16 copy (tensor-core path at large batches)
    return NNdex(m, approx=True, precision="auto", nlist=64, kmeans_iters=4, seed=3)


def requests(n, dims, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        size = int(rng.integers(1, 257))
        out.append((mixture(rng, size, dims), int(rng.choice([1, 10, 100])), bool(rng.integers(0, 2))))
    return out


def test_alone_equals_mix(index):
    reqs = requests(40, index.dims)
    alone = []
    with Server(index, slots=1) as s:
        for q, k, approx in reqs:
            alone.append(s.result(s.submit(q, k=k, approx=approx)))
    with Server(index, slots=3) as s:
        tickets = [s.submit(q, k=k, approx=approx) for q, k, approx in reqs]
        mixed = [s.result(t, with_info=True) for t in tickets]
        st = s.stats()
    shared = 0
    for (q, k, approx), (ai, asim), ((mi, msim), info) in zip(reqs, alone, mixed):
        np.testing.assert_array_equal(mi, ai)
        np.testing.assert_array_equal(msim.view(np.uint32), asim.view(np.uint32))
        shared += info["batch_queries"] > q.shape[0]
    assert shared > 0, "no request shared a batch"
    assert st["requests_done"] == len(reqs) and st["batches"] < len(reqs)


def test_server_matches_search_batch(index):
    # a served request of ≥ 2 queries is a search_batch: same rows and scores
    q, k, _ = requests(1, index.dims, seed=11)[0]
    q = np.vstack([q, q[:1]]) if q.shape[0] == 1 else q
    with Server(index) as s:
        si, ss = s.result(s.submit(q, k=k, approx=False))
    index.set_precision("auto")
    bi, bs = index.search(q, k=k)
    np.testing.assert_array_equal(si[:, :bi.shape[1]], bi)
    np.testing.assert_array_equal(ss[:, :bs.shape[1]], bs)


def test_admission_refuses_what_cannot_fit(index):
    q = mixture(np.random.default_rng(2), 40, index.dims)
    with Server(index, max_batch_queries=32) as s:
        with pytest.raises(NNdexError) as e:
            s.submit(q, k=10)
        assert e.value.code == NNDEX_ERR_ADMISSION
        assert s.stats()["refused"] == 1
    with Server(index, queue_capacity=30) as s:
        with pytest.raises(NNdexError) as e:
            s.submit(q, k=10)  # 40 queries > 30 waiting allowed
        assert e.value.code == NNDEX_ERR_ADMISSION
    with Server(index, slot_bytes=1 << 16) as s:  # 64 KiB per slot: not even one query at k = 100
        with pytest.raises(NNdexError) as e:
            s.submit(q[:1], k=100)
        assert e.value.code == NNDEX_ERR_ADMISSION


def test_bad_request_fails_alone(index):
    rng = np.random.default_rng(4)
    big = mixture(rng, 256, index.dims)
    good = mixture(rng, 7, index.dims)
    bad = mixture(rng, 5, index.dims)
    bad[2, 3] = np.nan
    with Server(index, slots=1) as s:
        t0 = s.submit(big, k=10)
        t1 = s.submit(bad, k=10)
        t2 = s.submit(good, k=10)
        s.result(t0)
        with pytest.raises(NNdexError) as e:
            s.result(t1)
        assert e.value.code == NNDEX_ERR_NON_FINITE
        gi, gs = s.result(t2)
    with Server(index, slots=1) as s:
        ai, asim = s.result(s.submit(good, k=10))
    np.testing.assert_array_equal(gi, ai)
    np.testing.assert_array_equal(gs, asim)


def test_poll_without_waiting_and_unknown_ticket(index):
    q = mixture(np.random.default_rng(9), 3, index.dims)
    with Server(index) as s:
        t = s.submit(q, k=5)
        r = None
        while r is None:
            r = s.poll(t, timeout=0.05)
        assert r[0].shape == (3, 5)
        with pytest.raises(KeyError):
            s.poll(t)


def test_latency_budget_refuses_while_the_queue_is_backed_up(index):
    # one slot taking 64 queries per batch and a burst of 1,000 requests of 64: the queue takes
    # many batches to drain, so a few tens of milliseconds later its oldest request has waited
    # longer than a 10 ms budget and new requests are refused; the admitted ones still get the
    # answers they get alone, and once the queue has drained requests are admitted again
    import time
    rng = np.random.default_rng(11)
    qs = [mixture(rng, 64, index.dims) for _ in range(1000)]

    def submit_or_refused(s, q):
        try:
            return s.submit(q, k=10)
        except NNdexError as e:
            assert e.code == NNDEX_ERR_ADMISSION and "latency budget" in str(e), str(e)
            return None

    with Server(index, slots=1, max_batch_queries=64, latency_budget_ms=10) as s:
        s.result(s.submit(qs[0], k=10))  # any one-off set-up runs alone
        tickets = [submit_or_refused(s, q) for q in qs]
        time.sleep(0.03)
        late = submit_or_refused(s, qs[0])
        results = {j: s.result(t) for j, t in enumerate(tickets) if t is not None}
        if late is not None:
            s.result(late)
        st = s.stats()
        assert st["refused_latency"] >= 1, st
        assert st["refused_latency"] == st["refused"] == sum(t is None for t in tickets) + (late is None)
        s.result(s.submit(qs[1], k=10))  # drained: admitted again
    assert results, "nothing admitted"
    with Server(index, slots=1) as alone:
        for j in list(results)[:3]:
            ai, asim = alone.result(alone.submit(qs[j], k=10))
            np.testing.assert_array_equal(results[j][0], ai)
            np.testing.assert_array_equal(results[j][1].view(np.uint32), asim.view(np.uint32))



def test_warm_up_leaves_no_trace_but_loaded_kernels(index):
    # Server start runs one batch of every kind on each slot (exact and approximate; k = 1, 10 and
    # 100; small to the largest admitted batch) before it takes requests. None of them shows in the
    # request statistics; each slot then serves both kinds with the request's own mode and nprobe
    # (the warm-up restores the slot's), so results equal later ones and the index's own approximate
    # search. The first batch's time is bounded well below the ~130 ms a fresh process's first
    # tensor-core batch spends loading kernels (here earlier tests may have loaded them already).
    q, _, _ = requests(1, index.dims, seed=13)[0]
    q = np.vstack([q] * (200 // q.shape[0] + 1))[:200]  # 200 queries: the tensor-core path
    with Server(index, slots=2, max_batch_queries=512) as s:
        st = s.stats()
        assert st["batches"] == 0 and st["queries_done"] == 0 and st["requests_done"] == 0, st
        (ei, es), info = s.result(s.submit(q, k=10, approx=False), with_info=True)
        ai, asim = s.result(s.submit(q, k=10, approx=True, nprobe=8))
        assert (info["done_ns"] - info["start_ns"]) / 1e6 < 100.0, info
        ei2, es2 = s.result(s.submit(q, k=10, approx=False))
    np.testing.assert_array_equal(ei, ei2)
    np.testing.assert_array_equal(es.view(np.uint32), es2.view(np.uint32))
    index.set_nprobe(8)
    try:
        xi, xs = index.search(q, k=10)  # an approx index searches its IVF
    finally:
        index.set_nprobe(0)
    np.testing.assert_array_equal(ai, xi)
    np.testing.assert_array_equal(asim.view(np.uint32), xs.view(np.uint32))
