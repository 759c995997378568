"""The autotuner on the GPU: the first batch of a shape times the candidate plans, later batches
reuse the winner, the cache travels as text to another index over the same matrix, and no plan
changes a result (needs a B200)."""
import numpy as np
import pytest

from nndex_b200 import NNdex, NNdexError

pytestmark = pytest.mark.gpu


def _bits(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


def test_tuned_plans_return_the_rules_results_and_are_cached():
    rng = np.random.default_rng(3)
    m = rng.normal(size=(80_000, 256)).astype(np.float32)
    q = rng.normal(size=(16, 256)).astype(np.float32)
    tuned = NNdex(m)
    rules = NNdex(m, autotune=False)
    first = tuned.search(q, k=20)
    st = tuned.last_search_stats()
    assert st["tuned"] == 1 and st["tune_candidates"] == 2, st  # the FP32 scan and the TF32 scan
    _bits(first, rules.search(q, k=20))
    assert rules.last_search_stats()["tuned"] == 0
    again = tuned.search(rng.normal(size=(13, 256)).astype(np.float32), k=20)  # same shape bucket
    assert tuned.last_search_stats()["tuned"] == 2
    assert again[0].shape == (13, 20)
    text = tuned.autotune_export()
    assert text.startswith("nndex-autotune v2 ") and "nq=16 k=32" in text, text
    other = NNdex(m)
    other.autotune_import(text)
    _bits(other.search(q, k=20), first)
    assert other.last_search_stats()["tuned"] == 2
    # a cache made for another matrix shape is refused
    small = NNdex(m[:1000])
    with pytest.raises(NNdexError):
        small.autotune_import(text)


def test_tensor_core_strides_and_ivf_paths_are_tuned_without_changing_results():
    rng = np.random.default_rng(4)
    centres = rng.normal(size=(64, 128)).astype(np.float32)
    m = (centres[rng.integers(0, 64, 200_000)] + 0.3 * rng.normal(size=(200_000, 128))).astype(np.float32)
    q = (centres[rng.integers(0, 64, 256)] + 0.3 * rng.normal(size=(256, 128))).astype(np.float32)
    tuned = NNdex(m, precision="bf16")
    rules = NNdex(m, precision="bf16", autotune=False)
    _bits(tuned.search(q, k=10), rules.search(q, k=10))
    st = tuned.last_search_stats()
    # pass-1 strides 1, 8, 32, each with one or two query blocks per CTA in pass 2
    assert st["tuned"] == 1 and st["tune_candidates"] == 6 and st["path"] == 2, st
    a_tuned = NNdex(m, approx=True, precision="auto", nlist=128, kmeans_iters=3, seed=9)
    a_rules = NNdex(m, approx=True, precision="auto", nlist=128, kmeans_iters=3, seed=9, autotune=False)
    for nprobe in (4, 16):
        a_tuned.set_nprobe(nprobe)
        a_rules.set_nprobe(nprobe)
        _bits(a_tuned.search(q, k=10), a_rules.search(q, k=10))
        st = a_tuned.last_search_stats()
        # the FP32 list scan, and the tensor-core list scan with pass-1 strides 1, 2, 4 and 16
        assert st["tuned"] == 1 and st["tune_candidates"] == 5 and st["path"] in (4, 5), st
