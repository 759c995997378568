"""NNdex.from_file dispatch and loader errors (src/python_io.rs:20-110, 380-410; the binding's
tests at tests_python/test_bindings.py:189-226). Every case here fails before any row reaches the
device, so the suite needs no GPU."""
import numpy as np
import pytest

from nndex_b200 import NNdex
from nndex_b200._files import _extension


def test_rejects_unsupported_extension():
    with pytest.raises(ValueError, match=r"unsupported file extension for 'matrix.csv', expected .npy, .npz, or .parquet"):
        NNdex.from_file("matrix.csv")


@pytest.mark.parametrize("fmt", ["npz", "parquet"])
def test_requires_key(fmt):
    with pytest.raises(ValueError, match=rf"missing required key for {fmt} file 'matrix.{fmt}'"):
        NNdex.from_file(f"matrix.{fmt}")


def test_backend_checked_before_the_file():
    # parse_index_options runs before load_matrix_from_disk (src/python_bindings.rs:81-83)
    with pytest.raises(ValueError, match="unsupported backend 'vulkan'"):
        NNdex.from_file("matrix.csv", backend="vulkan")


def test_extension_rules_follow_std_path():
    assert _extension("a/b/matrix.NPY") == "NPY"
    assert _extension("a/b.dir/matrix") is None
    assert _extension(".npy") is None
    assert _extension("..npy") == "npy"
    assert _extension("m.tar.npz") == "npz"
    assert _extension("matrix.") == ""
    # the extension is matched case-insensitively
    with pytest.raises(ValueError, match="missing required key for npz file"):
        NNdex.from_file("MATRIX.NPZ")


def test_missing_files(tmp_path):
    with pytest.raises(ValueError, match=r"failed to read .npy matrix from '.*missing.npy': No such file or directory \(os error 2\)"):
        NNdex.from_file(str(tmp_path / "missing.npy"))
    with pytest.raises(ValueError, match=r"could not open '.*missing.npz': No such file"):
        NNdex.from_file(str(tmp_path / "missing.npz"), key="x")
    with pytest.raises(ValueError, match=r"could not open '.*missing.parquet': No such file"):
        NNdex.from_file(str(tmp_path / "missing.parquet"), key="x")


def test_npy_layout_errors(tmp_path):
    p = tmp_path / "m.npy"
    np.save(p, np.ones((4, 3), dtype=np.float64))
    with pytest.raises(ValueError, match=r"failed to read .npy matrix from .*float32"):
        NNdex.from_file(str(p))
    np.save(p, np.ones(5, dtype=np.float32))
    with pytest.raises(ValueError, match=r"failed to read .npy matrix from .*dimensions"):
        NNdex.from_file(str(p))
    np.save(p, np.ones((0, 4), dtype=np.float32))
    with pytest.raises(ValueError, match=r"matrix loaded from '.*m.npy' is empty or has zero dimensions"):
        NNdex.from_file(str(p))
    p.write_bytes(b"not an npy file")
    with pytest.raises(ValueError, match=r"failed to read .npy matrix from"):
        NNdex.from_file(str(p))


def test_npz_key_lookup_errors(tmp_path):
    p = tmp_path / "m.npz"
    np.savez(p, embeddings=np.eye(4, dtype=np.float32), other=np.ones((2, 2), dtype=np.float64))
    with pytest.raises(ValueError, match=r"key 'missing' not found in .npz '.*m.npz'. Available keys: embeddings.npy, other.npy"):
        NNdex.from_file(str(p), key="missing")
    with pytest.raises(ValueError, match=r"failed reading key 'other' from .npz '.*m.npz': .*float32"):
        NNdex.from_file(str(p), key="other")
    np.savez(p, empty=np.ones((3, 0), dtype=np.float32))
    with pytest.raises(ValueError, match=r"matrix loaded from '.*m.npz' is empty"):
        NNdex.from_file(str(p), key="empty.npy")
    bad = tmp_path / "bad.npz"
    bad.write_bytes(b"PK not really")
    with pytest.raises(ValueError, match=r"failed to read .npz archive from '.*bad.npz'"):
        NNdex.from_file(str(bad), key="x")


def _write_parquet(path, column, name="embedding", row_group_size=None):
    pa = pytest.importorskip("pyarrow")
    pq = pytest.importorskip("pyarrow.parquet")
    pq.write_table(pa.table({name: column, "id": pa.array(range(len(column)))}), path,
                   row_group_size=row_group_size)
    return pa


def test_parquet_column_errors(tmp_path):
    pa = pytest.importorskip("pyarrow")
    p = tmp_path / "m.parquet"
    _write_parquet(p, pa.array([[1.0, 2.0], [3.0, 4.0]], type=pa.list_(pa.float32(), 2)))
    with pytest.raises(ValueError, match=r"column 'vectors' was not found in parquet file '.*m.parquet'"):
        NNdex.from_file(str(p), key="vectors")
    with pytest.raises(ValueError, match=r"parquet key 'id' in '.*m.parquet' is not an array/list<f32> column"):
        NNdex.from_file(str(p), key="id")

    _write_parquet(p, pa.array([[1.0, 2.0], None], type=pa.list_(pa.float32(), 2)))
    with pytest.raises(ValueError, match=r"parquet key 'embedding' in '.*' contains null values, which are unsupported"):
        NNdex.from_file(str(p), key="embedding")

    _write_parquet(p, pa.array([[1.0, None], [3.0, 4.0]], type=pa.list_(pa.float32())))
    with pytest.raises(ValueError, match=r"contains null values"):
        NNdex.from_file(str(p), key="embedding")

    _write_parquet(p, pa.array([[1.0, 2.0], [3.0, 4.0, 5.0]], type=pa.list_(pa.float32())))
    with pytest.raises(ValueError, match=r"parquet key 'embedding' in '.*' has inconsistent row dimensions"):
        NNdex.from_file(str(p), key="embedding")

    _write_parquet(p, pa.array([[1.0, 2.0], []], type=pa.list_(pa.float32())))
    with pytest.raises(ValueError, match=r"matrix loaded from '.*m.parquet' is empty or has zero dimensions"):
        NNdex.from_file(str(p), key="embedding")

    _write_parquet(p, pa.array([[1.0, 2.0]], type=pa.list_(pa.float64())))
    with pytest.raises(ValueError, match=r"is not an array/list<f32> column"):
        NNdex.from_file(str(p), key="embedding")

    _write_parquet(p, pa.array([[1.0, 2.0]], type=pa.large_list(pa.float32())))
    with pytest.raises(ValueError, match=r"is not an array/list<f32> column"):
        NNdex.from_file(str(p), key="embedding")

    _write_parquet(p, pa.array([], type=pa.list_(pa.float32())))
    with pytest.raises(ValueError, match=r"matrix loaded from '.*' is empty or has zero dimensions"):
        NNdex.from_file(str(p), key="embedding")

    # the first failing row decides, in the reference's per-row order (nulls, empty, dims)
    _write_parquet(p, pa.array([[1.0, 2.0], [1.0, 2.0, 3.0], []], type=pa.list_(pa.float32())))
    with pytest.raises(ValueError, match=r"inconsistent row dimensions"):
        NNdex.from_file(str(p), key="embedding")

    (tmp_path / "junk.parquet").write_bytes(b"definitely not parquet")
    with pytest.raises(ValueError, match=r"failed to read parquet file '.*junk.parquet'"):
        NNdex.from_file(str(tmp_path / "junk.parquet"), key="embedding")
