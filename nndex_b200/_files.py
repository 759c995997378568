"""Matrix files → a device index, piece by piece (NNdex.from_file).

Restates load_matrix_from_disk (src/python_io.rs:80-377) with its dispatch, key rules and error
messages, but without ever holding the whole matrix on the host: the rows go to the C ABI's
streaming builder (nndex_cuda_builder_*), which uploads each piece through pinned staging while
the next one is read and runs K1 (validation, normalisation, padding, low-precision copies) on the
device. The common .npy layout (little-endian float32, C order) is memory-mapped and streamed by
the library itself (nndex_cuda_create_from_npy).

Every loader error is raised as ValueError with the reference's DiskLoadError Display text
(src/python_io.rs:20-77); errors of the index itself (shape, non-finite values, zero-norm rows)
follow as NNdex::new raises them, after the whole file has been read.
"""
from __future__ import annotations

import ctypes as C
import os
import zipfile

import numpy as np

from . import _lib

# Rows per piece handed to the builder (≈ 64 MB of float32 at 384 dims).
_PIECE_VALUES = 16 << 20


def _io(e: OSError) -> str:
    """std::io::Error's Display: "<description> (os error N)"."""
    if e.errno is not None:
        return f"{e.strerror} (os error {e.errno})"
    return str(e)


def _extension(path: str) -> str | None:
    """std::path::Path::extension: None for no dot, or a name whose only dot leads it."""
    name = os.path.basename(path.rstrip("/"))
    if name in ("", "..") or "." not in name:
        return None
    before, after = name.rsplit(".", 1)
    return None if before == "" else after


class _Builder:
    """nndex_cuda_builder_* over one index; aborted unless finished."""

    def __init__(self, rows: int, dims: int, flags: int, opts):
        h = C.c_void_p()
        st = _lib.lib().nndex_cuda_builder_begin(rows, dims, flags, C.byref(opts), C.byref(h))
        if st != 0:
            raise ValueError(_lib.last_error())
        self.h = h

    def append(self, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype="<f4")
        if v.size == 0:
            return
        st = _lib.lib().nndex_cuda_builder_append(self.h, v.ctypes.data, v.size)
        if st != 0:
            raise ValueError(_lib.last_error())

    def finish(self) -> C.c_void_p:
        out = C.c_void_p()
        h, self.h = self.h, None
        st = _lib.lib().nndex_cuda_builder_finish(h, C.byref(out))
        if st != 0:
            raise ValueError(_lib.last_error())
        return out

    def abort(self) -> None:
        if self.h:
            _lib.lib().nndex_cuda_builder_abort(self.h)
            self.h = None


def _read_header(fp):
    """(shape, fortran_order, dtype) of the .npy stream at fp, left at the first data byte."""
    version = np.lib.format.read_magic(fp)
    if version == (1, 0):
        return np.lib.format.read_array_header_1_0(fp)
    if version == (2, 0):
        return np.lib.format.read_array_header_2_0(fp)
    # format 3.0 differs from 2.0 only in the header's text encoding (utf-8)
    hlen = int.from_bytes(fp.read(4), "little")
    header = fp.read(hlen).decode("utf-8")
    import ast
    d = ast.literal_eval(header)
    return tuple(d["shape"]), bool(d["fortran_order"]), np.dtype(d["descr"])


def _matrix_problem(shape, dtype) -> str | None:
    """Why a .npy array cannot be read as Array2<f32>, or None."""
    if dtype.kind != "f" or dtype.itemsize != 4:
        return f"the array's data type is {dtype.str}, expected float32"
    if len(shape) != 2:
        return f"the array has {len(shape)} dimensions, expected 2"
    return None


def _stream_rows(bld: _Builder, fp, rows: int, dims: int, dtype: np.dtype, fortran: bool, fail) -> None:
    """Appends rows × dims values read from fp (C order), or the whole array (Fortran order)."""
    if fortran:
        raw = fp.read(rows * dims * 4)
        if len(raw) != rows * dims * 4:
            raise fail("the data is truncated")
        a = np.frombuffer(raw, dtype=dtype).reshape((rows, dims), order="F")
        step = max(1, _PIECE_VALUES // dims)
        for r0 in range(0, rows, step):
            bld.append(a[r0:r0 + step])
        return
    step = max(1, _PIECE_VALUES // dims)
    for r0 in range(0, rows, step):
        n = min(step, rows - r0)
        raw = fp.read(n * dims * 4)
        if len(raw) != n * dims * 4:
            raise fail("the data is truncated")
        bld.append(np.frombuffer(raw, dtype=dtype))


def _empty(path: str) -> ValueError:
    return ValueError(f"matrix loaded from '{path}' is empty or has zero dimensions")


def _load_npy(path: str, flags: int, opts):
    """load_npy (src/python_io.rs:112-120)."""
    def fail(why):
        return ValueError(f"failed to read .npy matrix from '{path}': {why}")

    try:
        fp = open(path, "rb")
    except OSError as e:
        raise fail(_io(e)) from None
    with fp:
        try:
            shape, fortran, dtype = _read_header(fp)
        except (ValueError, SyntaxError, KeyError, UnicodeDecodeError) as e:
            raise fail(str(e)) from None
        why = _matrix_problem(shape, dtype)
        if why:
            raise fail(why)
        rows, dims = int(shape[0]), int(shape[1])
        if rows == 0 or dims == 0:
            raise _empty(path)
        if dtype.byteorder in ("<", "=") and not fortran and np.little_endian:
            fp.close()
            h = C.c_void_p()
            st = _lib.lib().nndex_cuda_create_from_npy(os.fsencode(path), flags, C.byref(opts), C.byref(h))
            if st != 0:
                raise ValueError(_lib.last_error())
            return h, rows, dims
        bld = _Builder(rows, dims, flags, opts)
        try:
            _stream_rows(bld, fp, rows, dims, dtype, fortran, fail)
            return bld.finish(), rows, dims
        finally:
            bld.abort()


def _load_npz(path: str, key: str, flags: int, opts):
    """load_npz (src/python_io.rs:122-164): `key` or `key.npy` inside the archive."""
    try:
        fp = open(path, "rb")
    except OSError as e:
        raise ValueError(f"could not open '{path}': {_io(e)}") from None
    with fp:
        try:
            zf = zipfile.ZipFile(fp)
            available = zf.namelist()
        except (zipfile.BadZipFile, OSError, ValueError) as e:
            raise ValueError(f"failed to read .npz archive from '{path}': {e}") from None
        candidate = key if key.endswith(".npy") else f"{key}.npy"
        if candidate in available:
            selected = candidate
        elif key in available:
            selected = key
        else:
            raise ValueError(f"key '{key}' not found in .npz '{path}'. Available keys: {', '.join(available)}")

        def fail(why):
            return ValueError(f"failed reading key '{key}' from .npz '{path}': {why}")

        try:
            member = zf.open(selected)
        except (zipfile.BadZipFile, OSError, NotImplementedError) as e:
            raise fail(str(e)) from None
        with member:
            try:
                shape, fortran, dtype = _read_header(member)
            except (ValueError, SyntaxError, KeyError, UnicodeDecodeError) as e:
                raise fail(str(e)) from None
            why = _matrix_problem(shape, dtype)
            if why:
                raise fail(why)
            rows, dims = int(shape[0]), int(shape[1])
            if rows == 0 or dims == 0:
                raise _empty(path)
            bld = _Builder(rows, dims, flags, opts)
            try:
                try:
                    _stream_rows(bld, member, rows, dims, dtype, fortran, fail)
                except (zipfile.BadZipFile, OSError, EOFError) as e:
                    raise fail(str(e)) from None
                return bld.finish(), rows, dims
            finally:
                bld.abort()


def _fixed_size_rows(col, dims, path, key):
    """append_fixed_size_parquet_column (src/python_io.rs:257-311) → (rows × d array, d)."""
    import pyarrow as pa

    if col.null_count > 0:
        raise ValueError(f"parquet key '{key}' in '{path}' contains null values, which are unsupported")
    d = col.type.list_size
    if d == 0:
        raise _empty(path)
    if col.type.value_type != pa.float32():
        raise ValueError(f"parquet key '{key}' in '{path}' is not an array/list<f32> column")
    flat = col.flatten()
    if flat.null_count > 0:
        raise ValueError(f"parquet key '{key}' in '{path}' contains null values, which are unsupported")
    if dims is not None and dims != d:
        raise ValueError(f"parquet key '{key}' in '{path}' has inconsistent row dimensions")
    return flat.to_numpy(zero_copy_only=False).reshape(len(col), d), d


def _list_rows(col, dims, path, key):
    """append_list_parquet_column (src/python_io.rs:313-366), checked row by row in its order."""
    import pyarrow as pa

    if col.null_count > 0:
        raise ValueError(f"parquet key '{key}' in '{path}' contains null values, which are unsupported")
    n = len(col)
    if n == 0:
        return np.zeros((0, dims or 0), dtype=np.float32), dims
    if col.type.value_type != pa.float32():
        raise ValueError(f"parquet key '{key}' in '{path}' is not an array/list<f32> column")
    offsets = np.asarray(col.offsets, dtype=np.int64)
    lengths = np.diff(offsets)
    flat = col.flatten()
    nulls = np.asarray(flat.is_null(), dtype=np.int64) if flat.null_count > 0 else None
    expect = dims if dims is not None else int(lengths[0])
    bad = (lengths == 0) | (lengths != expect)
    if nulls is not None:
        csum = np.concatenate([[0], np.cumsum(nulls)])
        rel = offsets - offsets[0]
        row_nulls = csum[rel[1:]] - csum[rel[:-1]]
        bad |= row_nulls > 0
    if bad.any():
        i = int(np.argmax(bad))
        if nulls is not None and row_nulls[i] > 0:
            raise ValueError(f"parquet key '{key}' in '{path}' contains null values, which are unsupported")
        if lengths[i] == 0:
            raise _empty(path)
        raise ValueError(f"parquet key '{key}' in '{path}' has inconsistent row dimensions")
    return flat.to_numpy(zero_copy_only=False).reshape(n, expect), expect


def _leaf_nulls(pf, key: str) -> bool:
    """Whether the row groups' statistics count a null under column `key`."""
    md = pf.metadata
    for rg in range(md.num_row_groups):
        g = md.row_group(rg)
        for c in range(g.num_columns):
            col = g.column(c)
            if col.path_in_schema.split(".")[0] == key and col.statistics is not None \
                    and col.statistics.has_null_count and col.statistics.null_count > 0:
                return True
    return False


def _load_parquet(path: str, key: str, flags: int, opts):
    """load_parquet (src/python_io.rs:166-225): a FixedSizeList or List column of float32."""
    try:
        fp = open(path, "rb")
    except OSError as e:
        raise ValueError(f"could not open '{path}': {_io(e)}") from None
    import pyarrow as pa
    import pyarrow.parquet as pq

    with fp:
        try:
            pf = pq.ParquetFile(fp)
            schema = pf.schema_arrow
        except (pa.ArrowException, OSError, ValueError) as e:
            raise ValueError(f"failed to read parquet file '{path}': {e}") from None
        if key not in schema.names:
            raise ValueError(f"column '{key}' was not found in parquet file '{path}'")
        total = int(pf.metadata.num_rows)
        rows, dims, bld = 0, None, None
        try:
            batches = pf.iter_batches(columns=[key])
            while True:
                try:
                    batch = next(batches)
                except StopIteration:
                    break
                except (pa.ArrowException, OSError, ValueError) as e:
                    # pyarrow cannot decode a null entry of a fixed-size list; the column's
                    # statistics still show it, and the reference reports it as a null value
                    if pa.types.is_fixed_size_list(schema.field(key).type) and _leaf_nulls(pf, key):
                        raise ValueError(f"parquet key '{key}' in '{path}' contains null values, which are "
                                         "unsupported") from None
                    raise ValueError(f"failed to read parquet file '{path}': {e}") from None
                col = batch.column(0)
                if pa.types.is_fixed_size_list(col.type):
                    vals, dims = _fixed_size_rows(col, dims, path, key)
                elif pa.types.is_list(col.type):
                    vals, dims = _list_rows(col, dims, path, key)
                else:
                    raise ValueError(f"parquet key '{key}' in '{path}' is not an array/list<f32> column")
                if len(vals) == 0:
                    continue
                if bld is None:
                    bld = _Builder(total, dims, flags, opts)
                bld.append(vals)
                rows += len(vals)
            if rows == 0 or not dims:
                raise _empty(path)
            return bld.finish(), rows, dims
        finally:
            if bld is not None:
                bld.abort()


def load(path: str, key: str | None, flags: int, opts):
    """load_matrix_from_disk (src/python_io.rs:80-110) → (index handle, rows, dims)."""
    ext = _extension(path)
    ext = ext.lower() if ext is not None else None
    if ext == "npy":
        return _load_npy(path, flags, opts)
    if ext == "npz":
        if key is None:
            raise ValueError(f"missing required key for npz file '{path}'")
        return _load_npz(path, key, flags, opts)
    if ext == "parquet":
        if key is None:
            raise ValueError(f"missing required key for parquet file '{path}'")
        return _load_parquet(path, key, flags, opts)
    raise ValueError(f"unsupported file extension for '{path}', expected .npy, .npz, or .parquet")
