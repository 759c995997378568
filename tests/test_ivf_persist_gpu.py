"""A saved IVF layout (centroids, offsets, permutation; src/approx.rs:11-25) installed into a new
index over the same matrix skips the build and answers every approx search exactly as the index it
was saved from — FP32 and tensor-core list scans, any k and nprobe."""
import numpy as np
import pytest

from nndex_b200 import NNdex, NNdexError, _lib

pytestmark = pytest.mark.gpu


def _mixture(rows, dims, centres, seed):
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(centres, dims)).astype(np.float32)
    x = c[rng.integers(0, centres, rows)] + 0.35 * rng.normal(size=(rows, dims)).astype(np.float32)
    q = x[rng.integers(0, rows, 300)] + 0.1 * rng.normal(size=(300, dims)).astype(np.float32)
    return x.astype(np.float32), q.astype(np.float32)


def _bitwise(a, b):
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


@pytest.mark.parametrize("precision", ["fp32", "auto"])
def test_restored_index_answers_like_the_built_one(tmp_path, precision):
    base, q = _mixture(60_000, 128, 300, seed=11)
    built = NNdex(base, approx=True, precision=precision, seed=7, autotune=False)
    path = tmp_path / "ivf.npz"
    built.save_ivf(str(path))
    restored = NNdex(base, approx=True, precision=precision, ivf=str(path), autotune=False)
    la, lb = built.ivf_layout(), restored.ivf_layout()
    for key in la:
        assert np.array_equal(la[key], lb[key]), key
    for k in (1, 10, 100):
        _bitwise(built.search(q, k=k), restored.search(q, k=k))
        _bitwise(built.search(q[0], k=k), restored.search(q[0], k=k))
    for nprobe in (4, 32):
        built.set_nprobe(nprobe)
        restored.set_nprobe(nprobe)
        _bitwise(built.search(q, k=10), restored.search(q, k=10))
    assert built.last_search_stats()["path"] == restored.last_search_stats()["path"]


def test_from_file_with_saved_ivf(tmp_path):
    base, q = _mixture(20_000, 96, 100, seed=12)
    np.save(tmp_path / "m.npy", base)
    built = NNdex.from_file(str(tmp_path / "m.npy"), approx=True)
    built.save_ivf(str(tmp_path / "ivf.npz"))
    again = NNdex.from_file(str(tmp_path / "m.npy"), approx=True, ivf=str(tmp_path / "ivf.npz"))
    _bitwise(built.search(q, k=10), again.search(q, k=10))


def test_saved_ivf_is_tied_to_its_matrix(tmp_path):
    base, _ = _mixture(5_000, 64, 50, seed=13)
    built = NNdex(base, approx=True)
    path = str(tmp_path / "ivf.npz")
    built.save_ivf(path)
    other = base.copy()
    other[[10, 11]] = other[[11, 10]]  # same values, two rows swapped
    with pytest.raises(ValueError, match="different matrix"):
        NNdex(other, approx=True, ivf=path)
    with pytest.raises(ValueError, match="was saved for a 5000 x 64 matrix"):
        NNdex(base[:4_000], approx=True, ivf=path)
    with pytest.raises(ValueError, match="needs approx=True"):
        NNdex(base, ivf=path)
    assert NNdex(base).checksum() == built.checksum() != NNdex(other).checksum()


def test_restore_validates_the_layout():
    base, _ = _mixture(4_000, 32, 40, seed=14)
    built = NNdex(base, approx=True)
    lay = built.ivf_layout()
    target = NNdex(base)
    bad = dict(lay, original_indices=lay["original_indices"].copy())
    bad["original_indices"][5] = bad["original_indices"][6]
    with pytest.raises(NNdexError, match="permutation") as e:
        target.load_ivf(bad)
    assert e.value.code == _lib.NNDEX_ERR_INVALID_ARGUMENT
    bad = dict(lay, cluster_offsets=lay["cluster_offsets"].copy())
    bad["cluster_offsets"][-1] -= 1
    with pytest.raises(NNdexError, match="offsets"):
        target.load_ivf(bad)
    bad = dict(lay, centroids=lay["centroids"].copy())
    bad["centroids"][3, 2] = np.inf
    with pytest.raises(NNdexError, match="non-finite"):
        target.load_ivf(bad)
    # a failed restore leaves the index as it was; a good one makes it approximate
    q = base[:50]
    _bitwise(target.search(q, k=5), NNdex(base).search(q, k=5))
    target.load_ivf(lay)
    _bitwise(target.search(q, k=5), built.search(q, k=5))


def test_small_index_saves_no_ivf(tmp_path):
    base, q = _mixture(200, 16, 5, seed=15)
    built = NNdex(base, approx=True)
    assert built.ivf_layout() is None
    built.save_ivf(str(tmp_path / "ivf.npz"))
    restored = NNdex(base, approx=True, ivf=str(tmp_path / "ivf.npz"))
    _bitwise(built.search(q, k=7), restored.search(q, k=7))
