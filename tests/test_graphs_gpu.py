"""CUDA-graph replay of the host-buffer search: a shape repeated in a row is captured once and
replayed; results must equal direct launches bit for bit, for new query values every call, and
after nprobe / precision changes (which drop the cached graphs)."""
import ctypes as C

import numpy as np
import pytest

from nndex_b200 import NNdex, _lib, kernel_launch_count

pytestmark = pytest.mark.gpu


def _bits(a, b):
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


def _mixture(rows, dims, seed):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(200, dims)).astype(np.float32)
    x = c[rng.integers(0, 200, rows)] + 0.3 * rng.normal(size=(rows, dims)).astype(np.float32)
    return x.astype(np.float32), rng


@pytest.mark.parametrize("batch,k", [(1, 10), (16, 100), (40, 7)])
def test_replayed_graphs_equal_direct_launches(batch, k):
    base, rng = _mixture(50_000, 192, 1)
    a = NNdex(base)
    b = NNdex(base)
    _lib.lib().nndex_cuda_set_graphs(b.handle, 0)
    kinds = []
    for step in range(6):
        q = rng.normal(size=(batch, 192)).astype(np.float32)
        ra, rb = a.search(q, k=k), b.search(q, k=k)
        _bits(ra, rb)
        kinds.append(a.last_search_stats()["graph"])
        assert b.last_search_stats()["graph"] == 0
    assert 1 in kinds and kinds[-1] == 2, kinds


def test_replay_counts_its_kernels():
    base, rng = _mixture(20_000, 64, 2)
    a = NNdex(base)
    q = rng.normal(size=(8, 64)).astype(np.float32)
    for _ in range(4):  # the first call allocates, the next captures, then replays
        a.search(q, k=5)
    assert a.last_search_stats()["graph"] == 2
    n0 = kernel_launch_count()
    a.search(q, k=5)
    assert kernel_launch_count() - n0 == a.last_search_stats()["kernel_launches"] > 0


def test_ivf_list_scan_graphs_follow_nprobe():
    base, rng = _mixture(60_000, 96, 3)
    a = NNdex(base, approx=True, precision="fp32", seed=5)
    b = NNdex(base, approx=True, precision="fp32", seed=5)
    _lib.lib().nndex_cuda_set_graphs(b.handle, 0)
    for nprobe in (4, 4, 4, 12, 12, 12, 4):
        a.set_nprobe(nprobe) if nprobe != a.__dict__.get("_np") else None
        a.__dict__["_np"] = nprobe
        b.set_nprobe(nprobe)
        q = rng.normal(size=(32, 96)).astype(np.float32)
        _bits(a.search(q, k=10), b.search(q, k=10))
        assert a.last_search_stats()["path"] == 4
    assert a.last_search_stats()["graph"] in (0, 1, 2)


def test_graphs_off_and_on_again():
    base, rng = _mixture(10_000, 32, 4)
    a = NNdex(base)
    L = _lib.lib()
    q = rng.normal(size=(4, 32)).astype(np.float32)
    ref = a.search(q, k=3)
    for _ in range(4):
        _bits(a.search(q, k=3), ref)
    assert a.last_search_stats()["graph"] == 2
    assert L.nndex_cuda_set_graphs(a.handle, 0) == 0
    _bits(a.search(q, k=3), ref)
    assert a.last_search_stats()["graph"] == 0
    assert L.nndex_cuda_set_graphs(a.handle, 1) == 0
    for _ in range(3):
        _bits(a.search(q, k=3), ref)
    assert a.last_search_stats()["graph"] == 2


@pytest.mark.parametrize("precision,batch,path", [("fp32", 16, 6), ("bf16", 200, 2), ("fp8", 200, 3)])
def test_certified_paths_are_captured_and_replayed(precision, batch, path):
    # the TF32 candidate scan and the tensor-core scans decide their fallbacks on the device, so
    # their host-buffer batches are captured too; replays equal direct launches bit for bit
    base, rng = _mixture(60_000, 128, 5)
    a = NNdex(base, precision=precision, autotune=False)
    b = NNdex(base, precision=precision, autotune=False)
    _lib.lib().nndex_cuda_set_graphs(b.handle, 0)
    centres, _ = _mixture(200, 128, 5)  # points near the base's clusters
    kinds = []
    for step in range(6):
        q = (centres[rng.integers(0, 200, batch)] + 0.3 * rng.normal(size=(batch, 128))).astype(np.float32)
        _bits(a.search(q, k=10), b.search(q, k=10))
        st = a.last_search_stats()
        assert st["path"] == path, st
        kinds.append(st["graph"])
    assert 2 in kinds, kinds


def test_ivf_tensor_core_batches_are_captured_and_replayed():
    # the tensor-core IVF list scan plans, certifies and collects on the device too
    base, rng = _mixture(60_000, 128, 6)
    kw = dict(approx=True, precision="auto", nlist=32, kmeans_iters=3, seed=2, nprobe=8, autotune=False)
    a = NNdex(base, **kw)
    b = NNdex(base, **kw)
    _lib.lib().nndex_cuda_set_graphs(b.handle, 0)
    centres, _ = _mixture(200, 128, 6)
    kinds = []
    for step in range(6):
        q = (centres[rng.integers(0, 200, 200)] + 0.3 * rng.normal(size=(200, 128))).astype(np.float32)
        _bits(a.search(q, k=10), b.search(q, k=10))
        st = a.last_search_stats()
        assert st["path"] == 5, st
        kinds.append(st["graph"])
    assert 2 in kinds, kinds
