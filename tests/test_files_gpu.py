"""Streaming construction on a B200: NNdex.from_file (.npy / .npz / .parquet) and the C ABI's
builder give the same index as NNdex(array) on the concatenated rows — the same scores bit for
bit, the same IVF — with the same errors in the same order (src/lib.rs:185-278,
src/python_io.rs:80-377, tests_python/test_bindings.py:189-226)."""
import ctypes as C

import numpy as np
import pytest

from nndex_b200 import NNdex, _lib

pytestmark = pytest.mark.gpu


def _same_results(a: NNdex, b: NNdex, queries: np.ndarray, k: int):
    ia, sa = a.search(queries, k=k)
    ib, sb = b.search(queries, k=k)
    assert np.array_equal(ia, ib)
    assert np.array_equal(sa.view(np.uint32), sb.view(np.uint32))


def _data(rows, dims, seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(rows, dims)).astype(np.float32), rng.normal(size=(32, dims)).astype(np.float32)


def test_reference_binding_cases(tmp_path):
    """tests_python/test_bindings.py:189-226 on the CUDA backend."""
    eye = np.eye(8, dtype=np.float32)
    np.save(tmp_path / "matrix.npy", eye)
    m = NNdex.from_file(str(tmp_path / "matrix.npy"), normalized=True)
    i, s = m.search(eye[0], k=1)
    assert int(i[0]) == 0 and float(s[0]) == pytest.approx(1.0, rel=1e-6)
    np.savez(tmp_path / "matrix.npz", embeddings=eye)
    m = NNdex.from_file(str(tmp_path / "matrix.npz"), key="embeddings", normalized=True)
    assert int(m.search(eye[3], k=1)[0][0]) == 3
    pa = pytest.importorskip("pyarrow")
    pq = pytest.importorskip("pyarrow.parquet")
    pq.write_table(pa.table({"embedding": pa.array(eye.tolist(), type=pa.list_(pa.float32(), 8))}),
                   tmp_path / "matrix.parquet")
    m = NNdex.from_file(str(tmp_path / "matrix.parquet"), key="embedding", normalized=True)
    assert int(m.search(eye[5], k=1)[0][0]) == 5
    assert (m.rows, m.dims) == (8, 8)


@pytest.mark.parametrize("normalized", [False, True])
def test_npy_layouts_equal_array(tmp_path, normalized):
    base, q = _data(70_001, 200)
    ref = NNdex(base, normalized=normalized)
    for name, arr in [("c.npy", base), ("big.npy", base.astype(">f4")), ("f.npy", np.asfortranarray(base))]:
        p = tmp_path / name
        np.save(p, arr)
        m = NNdex.from_file(str(p), normalized=normalized)
        assert (m.rows, m.dims) == base.shape
        _same_results(ref, m, q, 10)


def test_npz_equal_array(tmp_path):
    base, q = _data(30_000, 96, seed=1)
    ref = NNdex(base)
    np.savez(tmp_path / "a.npz", vecs=base, junk=np.zeros(3))
    np.savez_compressed(tmp_path / "b.npz", vecs=base)
    for name, key in [("a.npz", "vecs"), ("a.npz", "vecs.npy"), ("b.npz", "vecs")]:
        _same_results(ref, NNdex.from_file(str(tmp_path / name), key=key), q, 16)


def test_parquet_equal_array(tmp_path):
    pa = pytest.importorskip("pyarrow")
    pq = pytest.importorskip("pyarrow.parquet")
    base, q = _data(20_000, 64, seed=2)
    ref = NNdex(base)
    flat = pa.array(base.reshape(-1))
    for kind, col in [("fixed", pa.FixedSizeListArray.from_arrays(flat, 64)),
                      ("list", pa.ListArray.from_arrays(pa.array(np.arange(0, base.size + 1, 64, dtype=np.int32)),
                                                        flat))]:
        p = tmp_path / f"{kind}.parquet"
        pq.write_table(pa.table({"id": pa.array(range(len(base))), "embedding": col}), p, row_group_size=3_001)
        m = NNdex.from_file(str(p), key="embedding")
        assert (m.rows, m.dims) == base.shape
        _same_results(ref, m, q, 10)


def test_approx_from_file_builds_the_same_ivf(tmp_path):
    base, q = _data(40_000, 128, seed=3)
    np.save(tmp_path / "m.npy", base)
    a = NNdex(base, approx=True)
    b = NNdex.from_file(str(tmp_path / "m.npy"), approx=True)
    la, lb = a.ivf_layout(), b.ivf_layout()
    for key in la:
        assert np.array_equal(la[key], lb[key]), key
    _same_results(a, b, q, 10)


def test_index_errors_after_the_file_is_read(tmp_path):
    base, _ = _data(5_000, 32, seed=4)
    base[4_321, 7] = np.nan
    np.save(tmp_path / "nan.npy", base)
    with pytest.raises(ValueError) as ea:
        NNdex(base)
    with pytest.raises(ValueError) as eb:
        NNdex.from_file(str(tmp_path / "nan.npy"))
    assert str(ea.value) == str(eb.value)
    base[4_321, 7] = 1.0
    base[77] = 0.0
    np.savez(tmp_path / "zero.npz", m=base)
    with pytest.raises(ValueError) as ea:
        NNdex(base)
    with pytest.raises(ValueError) as eb:
        NNdex.from_file(str(tmp_path / "zero.npz"), key="m")
    assert str(ea.value) == str(eb.value)


def _begin(rows, dims, flags=0):
    L = _lib.lib()
    opts = _lib.Opts()
    opts.device = -1
    h = C.c_void_p()
    assert L.nndex_cuda_builder_begin(rows, dims, flags, C.byref(opts), C.byref(h)) == 0, _lib.last_error()
    return L, h


def _wrap(h, rows, dims):
    m = NNdex.__new__(NNdex)
    m._h = None
    m._adopt(h, rows, dims, False, False, True)
    return m


def test_builder_ragged_pieces_cross_staging_buffers():
    # 90,000 × 256 floats = 92 MB: two staging buffers of 64 MB, pieces that end mid-row
    base, q = _data(90_000, 256, seed=5)
    flat = base.reshape(-1)
    L, h = _begin(*base.shape)
    rng = np.random.default_rng(9)
    pos = 0
    while pos < flat.size:
        n = int(min(flat.size - pos, rng.integers(1, 3_000_000)))
        piece = np.ascontiguousarray(flat[pos:pos + n])
        assert L.nndex_cuda_builder_append(h, piece.ctypes.data, n) == 0, _lib.last_error()
        pos += n
    out = C.c_void_p()
    assert L.nndex_cuda_builder_finish(h, C.byref(out)) == 0, _lib.last_error()
    _same_results(NNdex(base), _wrap(out, *base.shape), q, 32)


def test_builder_shape_errors_match_create():
    base, _ = _data(1_000, 16, seed=6)
    flat = base.reshape(-1)
    # too few values: the reference's ShapeMismatch text with the count received
    L, h = _begin(1_000, 16)
    assert L.nndex_cuda_builder_append(h, flat.ctypes.data, flat.size - 5) == 0
    out = C.c_void_p()
    assert L.nndex_cuda_builder_finish(h, C.byref(out)) == _lib.NNDEX_ERR_SHAPE_MISMATCH
    assert _lib.last_error() == "matrix shape mismatch: rows=1000, dims=16, values=15995"
    assert not out.value
    # too many values: refused at the append, reported again at finish
    L, h = _begin(1_000, 16)
    assert L.nndex_cuda_builder_append(h, flat.ctypes.data, flat.size) == 0
    assert L.nndex_cuda_builder_append(h, flat.ctypes.data, 1) == _lib.NNDEX_ERR_SHAPE_MISMATCH
    assert L.nndex_cuda_builder_finish(h, C.byref(out)) == _lib.NNDEX_ERR_SHAPE_MISMATCH
    # abort of a half-filled builder frees it
    L, h = _begin(1_000, 16)
    assert L.nndex_cuda_builder_append(h, flat.ctypes.data, 100) == 0
    L.nndex_cuda_builder_abort(h)
    L.nndex_cuda_builder_abort(None)
