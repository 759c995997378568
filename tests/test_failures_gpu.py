"""Failure handling without a GPU fault: a device wait that runs out of its budget reports
NNDEX_ERR_TIMEOUT and leaves the index usable; allocation failures injected on the host make the
call that needed the memory fail with NNDEX_ERR_OUT_OF_MEMORY, and the next call succeeds."""
import numpy as np
import pytest

from nndex_b200 import NNdex, _lib

pytestmark = pytest.mark.gpu


def _data(seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(20_000, 64)).astype(np.float32), rng.normal(size=(12, 64)).astype(np.float32)


def _bits(a, b):
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


def test_bounded_wait_reports_timeout_and_index_stays_usable():
    base, q = _data()
    ix = NNdex(base)
    ref = ix.search(q, k=10)
    L = _lib.lib()
    st = L.nndex_cuda_check_bounded_wait(ix.handle, 2_000_000)  # ≈ 1 ms of clock cycles
    assert st == _lib.NNDEX_ERR_TIMEOUT
    assert "timed out" in _lib.last_error()
    _bits(ix.search(q, k=10), ref)
    assert L.nndex_cuda_check_bounded_wait(ix.handle, 0) == _lib.NNDEX_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("approx", [False, True])
def test_injected_allocation_failure_fails_one_call(approx):
    base, q = _data(1)
    L = _lib.lib()
    ref = NNdex(base, approx=approx).search(q, k=7)
    ix = NNdex(base, approx=approx)
    try:
        L.nndex_cuda_inject_alloc_failures(1)
        with pytest.raises(RuntimeError, match="out of device memory"):
            ix.search(q, k=7)  # the first batch search allocates its scratch
    finally:
        L.nndex_cuda_inject_alloc_failures(0)
    _bits(ix.search(q, k=7), ref)
