"""nndex_b200 — B200 (sm_100a) backend for nndex's cosine top-k search, with nndex's Python API.

``NNdex`` mirrors the reference's PyO3 class (src/python_bindings.rs:31-236): the same
constructor keywords, the same ``search(query, k=10, dataframe=None)`` dispatch (1-D → single
search, 2-D → batch search, one-row 2-D → single search), the same numpy outputs
(``uint64`` indices, ``float32`` similarities, batch rows padded with (0, 0.0)) and the same
exception types (constructor → ValueError, search → RuntimeError, dims mismatch → ValueError).
The only backend is ``"cuda"``: every call goes through libnndex_cuda.so's C ABI
(include/nndex_cuda.h). There is no CPU fallback; a missing library raises at import of the
first index.
"""
from __future__ import annotations

import ctypes as C
from typing import Any

import numpy as np

from . import _lib
from ._lib import (NNDEX_FLAG_APPROX, NNDEX_FLAG_BF16, NNDEX_FLAG_FP8, NNDEX_FLAG_NORMALIZED,
                   NNDEX_PRECISION_AUTO, NNDEX_PRECISION_BF16, NNDEX_PRECISION_FP8, NNDEX_PRECISION_FP32)

__all__ = ["NNdex", "NNdexError", "list_gpu_devices", "kernel_launch_count"]

_PRECISIONS = {
    "auto": NNDEX_PRECISION_AUTO,
    "fp32": NNDEX_PRECISION_FP32,
    "bf16": NNDEX_PRECISION_BF16,
    "fp8": NNDEX_PRECISION_FP8,
}


_IVF_FORMAT = "nndex-cuda-ivf/1"


class NNdexError(RuntimeError):
    """A failed C-ABI call: ``code`` is the NNDEX_ERR_* status, the message NNdexError's Display."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def _parse_backend(raw: str) -> str:
    """src/python_bindings.rs:300-308 parse_backend, with "cuda" as the one backend here."""
    b = str(raw).lower()
    if b == "cuda":
        return b
    raise ValueError(f"unsupported backend '{b}', expected one of: cuda")


def _detect_dataframe_kind(value: Any) -> str | None:
    """src/python_bindings.rs:404-418 detect_dataframe_kind."""
    t = type(value)
    if t.__name__ == "DataFrame" and "pandas" in (t.__module__ or ""):
        return "pandas"
    if t.__name__ == "DataFrame" and "polars" in (t.__module__ or ""):
        return "polars"
    return None


def _parse_input(value: Any) -> np.ndarray:
    """src/python_bindings.rs:311-400 parse_input → a C-contiguous float32 1-D or 2-D array."""
    if hasattr(value, "to_numpy"):
        arr = value.to_numpy()
        if arr is not value:
            return _parse_input(arr)
    if isinstance(value, np.ndarray):
        if value.dtype not in (np.float32, np.float64):
            raise ValueError("unsupported input type: expected list, numpy array, pandas/polars Series, or DataFrame")
        if value.ndim not in (1, 2):
            raise ValueError("only 1D and 2D arrays are supported for inputs")
        return np.ascontiguousarray(value, dtype=np.float32)
    if isinstance(value, (list, tuple)):
        if len(value) == 0:
            raise ValueError("input vector must be non-empty")
        if isinstance(value[0], (list, tuple, np.ndarray)):
            rows = [list(r) for r in value]
            if len(rows[0]) == 0:
                raise ValueError("input matrix must be non-empty")
            dims = len(rows[0])
            if any(len(r) != dims for r in rows):
                raise ValueError("2D list input must have consistent row lengths")
            return np.ascontiguousarray(np.asarray(rows, dtype=np.float32))
        return np.ascontiguousarray(np.asarray(value, dtype=np.float32))
    raise ValueError("unsupported input type: expected list, numpy array, pandas/polars Series, or DataFrame")


def _check(code: int) -> None:
    if code != 0:
        raise NNdexError(code, _lib.last_error())


def list_gpu_devices() -> list[dict]:
    """src/python_bindings.rs:273-289 list_gpu_devices, over CUDA devices."""
    L = _lib.lib()
    cnt = C.c_uint32(0)
    _check(L.nndex_cuda_list_devices(None, 0, C.byref(cnt)))
    n = cnt.value
    if n == 0:
        return []
    arr = (_lib.DevInfo * n)()
    _check(L.nndex_cuda_list_devices(arr, n, C.byref(cnt)))
    return [_devinfo_dict(arr[i]) for i in range(n)]


def kernel_launch_count() -> int:
    """Kernels launched by libnndex_cuda.so in this process so far."""
    return int(_lib.lib().nndex_cuda_kernel_launch_count())


def _devinfo_dict(d: _lib.DevInfo) -> dict:
    return {
        "index": int(d.index),
        "name": d.name.decode(),
        "driver": d.driver.decode(),
        "driver_info": d.driver_info.decode(),
        "backend": d.backend.decode(),
        "device_type": d.device_type.decode(),
        "sm_count": int(d.sm_count),
        "compute_capability": f"{d.cc_major}.{d.cc_minor}",
        "hbm_bytes": int(d.hbm_bytes),
        "l2_bytes": int(d.l2_bytes),
    }


class NNdex:
    """In-memory cosine top-k index on one B200 (src/python_bindings.rs:31-66 PyNNdex)."""

    def __init__(self, data: Any, normalized: bool = False, approx: bool = False, backend: str = "cuda",
                 enable_cache: bool = True, gpu_device_index: int | None = None, *, precision: str = "fp32",
                 nlist: int = 0, nprobe: int = 0, kmeans_iters: int = 0, seed: int | None = None,
                 rerank_width: int = 0, low_precision_copies: tuple = (), ivf: Any = None,
                 autotune: bool = True):
        self._h = None
        flags, opts = self._options(backend, normalized, approx, gpu_device_index, precision, nlist, nprobe,
                                    kmeans_iters, seed, rerank_width, low_precision_copies, ivf)
        arr = _parse_input(data)
        if arr.ndim == 1:
            arr = arr.reshape(1, -1)
        rows, dims = arr.shape
        h = C.c_void_p()
        st = _lib.lib().nndex_cuda_create(arr.ctypes.data, arr.size, rows, dims, flags, C.byref(opts), C.byref(h))
        if st != 0:
            raise ValueError(_lib.last_error())
        self._adopt(h, rows, dims, normalized, approx, enable_cache)
        if not autotune:
            self.set_autotune(False)
        if ivf is not None:
            self.load_ivf(ivf)

    @classmethod
    def from_file(cls, path: str, *, key: str | None = None, normalized: bool = False, approx: bool = False,
                  backend: str = "cuda", enable_cache: bool = True, gpu_device_index: int | None = None,
                  precision: str = "fp32", nlist: int = 0, nprobe: int = 0, kmeans_iters: int = 0,
                  seed: int | None = None, rerank_width: int = 0, low_precision_copies: tuple = (),
                  ivf: Any = None) -> "NNdex":
        """src/python_bindings.rs:67-86 from_file: a .npy, .npz (``key`` names the array) or .parquet
        (``key`` names a list<float32> column) matrix, streamed to the device piece by piece
        (nndex_b200/_files.py); the errors of load_matrix_from_disk (src/python_io.rs:20-77) and of
        NNdex::new, as ValueError."""
        from . import _files
        self = cls.__new__(cls)
        self._h = None
        flags, opts = cls._options(backend, normalized, approx, gpu_device_index, precision, nlist, nprobe,
                                   kmeans_iters, seed, rerank_width, low_precision_copies, ivf)
        h, rows, dims = _files.load(str(path), key, flags, opts)
        self._adopt(h, rows, dims, normalized, approx, enable_cache)
        if ivf is not None:
            self.load_ivf(ivf)
        return self

    @staticmethod
    def _options(backend, normalized, approx, gpu_device_index, precision, nlist, nprobe, kmeans_iters, seed,
                 rerank_width, low_precision_copies, ivf=None):
        """Construction flags and options (parse_index_options, src/python_bindings.rs:239-262).
        With a saved IVF (``ivf``) the index is created without building one."""
        _parse_backend(backend)
        if precision not in _PRECISIONS:
            raise ValueError(f"unsupported precision '{precision}', expected one of: {', '.join(_PRECISIONS)}")
        if ivf is not None and not approx:
            raise ValueError("a saved IVF (ivf=...) needs approx=True")
        flags = 0
        if normalized:
            flags |= NNDEX_FLAG_NORMALIZED
        if approx and ivf is None:
            flags |= NNDEX_FLAG_APPROX
        # "bf16" / "fp8" keep that scoring copy; "auto" keeps a BF16 copy for large batches.
        if precision in ("bf16", "auto"):
            flags |= NNDEX_FLAG_BF16
        if precision == "fp8":
            flags |= NNDEX_FLAG_FP8
        for extra in low_precision_copies:
            flags |= {"bf16": NNDEX_FLAG_BF16, "fp8": NNDEX_FLAG_FP8}[extra]
        opts = _lib.Opts()
        opts.device = -1 if gpu_device_index is None else int(gpu_device_index)
        opts.precision = _PRECISIONS[precision]
        opts.nlist = nlist
        opts.nprobe = nprobe
        opts.kmeans_iters = kmeans_iters
        opts.has_seed = 0 if seed is None else 1
        opts.seed = 0 if seed is None else int(seed)
        opts.rerank_width = rerank_width
        return flags, opts

    def _adopt(self, h, rows, dims, normalized, approx, enable_cache):
        self._backend = "cuda"
        self._enable_cache = enable_cache  # accepted for API parity; the CUDA backend keeps no result cache
        self._h = h
        self._rows = int(rows)
        self._dims = int(dims)
        self._normalized = normalized
        self._approx = approx

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _lib.lib().nndex_cuda_destroy(h)
            self._h = None

    # ---- getters (src/python_bindings.rs:88-123) ----
    @property
    def backend(self) -> str:
        return self._backend

    @property
    def rows(self) -> int:
        return self._rows

    @property
    def dims(self) -> int:
        return self._dims

    @property
    def gpu_info(self) -> dict:
        info = _lib.DevInfo()
        _check(_lib.lib().nndex_cuda_info(self._h, C.byref(info)))
        return _devinfo_dict(info)

    @property
    def handle(self) -> C.c_void_p:
        """The opaque nndex_cuda_index* (for callers that drive the C ABI directly)."""
        return self._h

    def set_precision(self, precision: str, rerank_width: int = 0) -> None:
        """Scan precision for later searches: "fp32", "bf16", "fp8" or "auto" (see __init__)."""
        if precision not in _PRECISIONS:
            raise ValueError(f"unsupported precision '{precision}', expected one of: {', '.join(_PRECISIONS)}")
        _check(_lib.lib().nndex_cuda_set_precision(self._h, _PRECISIONS[precision], int(rerank_width)))

    def last_candidates(self, query_rows: int):
        """(rows, approximate scores, eps, certified) of the last low-precision search's k′ candidates."""
        kp = C.c_uint32(0)
        eps = C.c_float(0.0)
        st = self.last_search_stats()
        kk = int(st["rerank_width"])
        idx = np.zeros((query_rows, max(kk, 1)), dtype=np.uint64)
        sim = np.zeros((query_rows, max(kk, 1)), dtype=np.float32)
        cert = np.zeros(query_rows, dtype=np.uint32)
        _check(_lib.lib().nndex_cuda_last_candidates(self._h, query_rows, idx.ctypes.data, sim.ctypes.data, idx.size,
                                                     C.byref(kp), C.byref(eps), cert.ctypes.data))
        return idx[:, :kp.value], sim[:, :kp.value], float(eps.value), cert.astype(bool)

    def set_autotune(self, enable: bool = True) -> None:
        """Plan choice for later searches: measured once per batch shape (the default) or the fixed
        rules (nndex_cuda_set_autotune). Results are the same either way."""
        _check(_lib.lib().nndex_cuda_set_autotune(self._h, 1 if enable else 0))

    def autotune_export(self) -> str:
        """The autotuner's cache as text (nndex_cuda_autotune_export)."""
        n = C.c_uint64(0)
        _check(_lib.lib().nndex_cuda_autotune_export(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(_lib.lib().nndex_cuda_autotune_export(self._h, buf, n.value, C.byref(n)))
        return buf.value.decode()

    def autotune_import(self, text: str) -> None:
        """Installs a cache exported for the same device model, shape and flags."""
        _check(_lib.lib().nndex_cuda_autotune_import(self._h, text.encode()))

    def set_error_report(self, enable: bool = True) -> None:
        """Record, for every result of later searches, |score − FP64 score| (see
        nndex_cuda_set_error_report); last_score_errors returns them, last_search_stats their max and
        mean."""
        _check(_lib.lib().nndex_cuda_set_error_report(self._h, 1 if enable else 0))

    def last_score_errors(self, query_rows: int, k: int) -> np.ndarray:
        """The last search's per-result score errors, query_rows × min(k, rows) (0 past a query's count)."""
        kk = max(min(int(k), self._rows), 1)
        out = np.zeros((query_rows, kk), dtype=np.float64)
        _check(_lib.lib().nndex_cuda_last_score_errors(self._h, query_rows, int(k), out.ctypes.data))
        return out

    def last_search_stats(self) -> dict:
        s = _lib.SearchStats()
        _check(_lib.lib().nndex_cuda_last_search_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in _lib.SearchStats._fields_}

    def ivf_layout(self) -> dict | None:
        """The IVF of an approx index as ApproxIndex holds it (src/approx.rs:11-25), or None.

        Keys: centroids [nlist × padded_dims] f32, cluster_offsets [nlist + 1], original_indices
        [rows] (reordered position → original row), init_rows [nlist] (the rows k-means++ picked).
        """
        L = _lib.lib()
        n = C.c_uint64(0)
        _check(L.nndex_cuda_ivf_layout(self._h, C.byref(n), None, None, None, None))
        if n.value == 0:
            return None
        nl = n.value
        pd = (self._dims + 7) // 8 * 8
        cent = np.zeros((nl, pd), dtype=np.float32)
        off = np.zeros(nl + 1, dtype=np.uint64)
        orig = np.zeros(self._rows, dtype=np.uint64)
        init = np.zeros(nl, dtype=np.uint64)
        _check(L.nndex_cuda_ivf_layout(self._h, C.byref(n), cent.ctypes.data, off.ctypes.data, orig.ctypes.data,
                                       init.ctypes.data))
        return {"centroids": cent, "cluster_offsets": off, "original_indices": orig, "init_rows": init}

    def set_nprobe(self, nprobe: int) -> None:
        """Lists probed per query by later approx searches (0 = the reference's choose_nprobe)."""
        _check(_lib.lib().nndex_cuda_set_nprobe(self._h, int(nprobe)))

    def checksum(self) -> int:
        """64-bit fingerprint of the stored (validated, normalised) rows (nndex_cuda_base_checksum)."""
        out = C.c_uint64(0)
        _check(_lib.lib().nndex_cuda_base_checksum(self._h, C.byref(out)))
        return int(out.value)

    def save_ivf(self, path: str) -> None:
        """Writes the IVF (ivf_layout) with the matrix's shape and checksum to an .npz file, so that
        a later index over the same matrix can skip the build (``NNdex(..., approx=True, ivf=path)``)."""
        if not self._approx:
            raise ValueError("save_ivf needs an approx index")
        lay = self.ivf_layout()
        if lay is None:
            pd = (self._dims + 7) // 8 * 8
            lay = {"centroids": np.zeros((0, pd), np.float32), "cluster_offsets": np.zeros(0, np.uint64),
                   "original_indices": np.zeros(0, np.uint64), "init_rows": np.zeros(0, np.uint64)}
        with open(path, "wb") as f:
            np.savez(f, format=np.array(_IVF_FORMAT), rows=np.uint64(self._rows), dims=np.uint64(self._dims),
                     normalized=np.bool_(self._normalized), checksum=np.uint64(self.checksum()),
                     nlist=np.uint64(len(lay["init_rows"])), **lay)

    def load_ivf(self, source: Any) -> None:
        """Installs a saved IVF (a path written by save_ivf, or an ivf_layout() dict) instead of
        building one; the index answers approx searches as the index it was saved from."""
        if isinstance(source, dict):
            lay = source
            nl = len(lay["init_rows"]) if lay.get("init_rows") is not None else len(lay["cluster_offsets"]) - 1
        else:
            with np.load(source, allow_pickle=False) as z:
                if "format" not in z.files or str(z["format"]) != _IVF_FORMAT:
                    raise ValueError(f"'{source}' is not a saved nndex IVF")
                if int(z["rows"]) != self._rows or int(z["dims"]) != self._dims:
                    raise ValueError(f"the IVF in '{source}' was saved for a {int(z['rows'])} x {int(z['dims'])} "
                                     f"matrix, this index is {self._rows} x {self._dims}")
                if int(z["checksum"]) != self.checksum():
                    raise ValueError(f"the IVF in '{source}' was saved for a different matrix (checksum mismatch)")
                lay = {k: z[k] for k in ("centroids", "cluster_offsets", "original_indices", "init_rows")}
                nl = int(z["nlist"])
        pd = (self._dims + 7) // 8 * 8
        cent = np.ascontiguousarray(lay["centroids"], dtype=np.float32).reshape(nl, pd) if nl else None
        off = np.ascontiguousarray(lay["cluster_offsets"], dtype=np.uint64)
        orig = np.ascontiguousarray(lay["original_indices"], dtype=np.uint64)
        init = lay.get("init_rows")
        init = np.ascontiguousarray(init, dtype=np.uint64) if init is not None else None
        if nl and (len(off) != nl + 1 or len(orig) != self._rows or (init is not None and len(init) != nl)):
            raise ValueError("IVF layout arrays do not match nlist and the index's rows")
        ptr = lambda a: a.ctypes.data if a is not None else None  # noqa: E731
        _check(_lib.lib().nndex_cuda_ivf_restore(self._h, nl, ptr(cent), ptr(off) if nl else None,
                                                 ptr(orig) if nl else None, ptr(init) if nl else None))
        self._approx = True

    def ivf_stats(self) -> dict:
        s = _lib.IvfStats()
        _check(_lib.lib().nndex_cuda_ivf_stats_get(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in _lib.IvfStats._fields_ if f != "reserved"}

    # ---- search (src/python_bindings.rs:125-236) ----
    def _search_single(self, q: np.ndarray, k: int):
        k = int(k)
        if k < 0:
            raise OverflowError("can't convert negative int to unsigned")
        kk = max(min(k, self._rows), 1)
        idx = np.zeros(kk, dtype=np.uint64)
        sim = np.zeros(kk, dtype=np.float32)
        cnt = C.c_uint64(0)
        st = _lib.lib().nndex_cuda_search(self._h, q.ctypes.data, q.size, k, idx.ctypes.data, sim.ctypes.data,
                                          C.byref(cnt))
        if st != 0:
            raise NNdexError(st, _lib.last_error())
        n = int(cnt.value)
        return idx[:n], sim[:n]

    def _search_batch(self, q: np.ndarray, k: int):
        k = int(k)
        if k < 0:
            raise OverflowError("can't convert negative int to unsigned")
        rows = q.shape[0]
        kk = max(min(k, self._rows), 1)
        idx = np.zeros((rows, kk), dtype=np.uint64)
        sim = np.zeros((rows, kk), dtype=np.float32)
        cnt = np.zeros(rows, dtype=np.uint64)
        st = _lib.lib().nndex_cuda_search_batch(self._h, q.ctypes.data, q.size, rows, k, idx.ctypes.data,
                                                sim.ctypes.data, cnt.ctypes.data)
        if st != 0:
            raise NNdexError(st, _lib.last_error())
        return idx, sim, cnt

    @staticmethod
    def _rectangular(idx, sim, cnt):
        """batch_neighbors_to_numpy (src/python_bindings.rs:465-497): width = the first row's
        length; shorter rows padded with (0, 0.0), longer rows truncated."""
        rows = idx.shape[0]
        cols = int(cnt[0]) if rows else 0
        idx = np.ascontiguousarray(idx[:, :cols])
        sim = np.ascontiguousarray(sim[:, :cols])
        for r in range(rows):
            n = int(cnt[r])
            if n < cols:
                idx[r, n:] = 0
                sim[r, n:] = 0.0
        return idx, sim

    def search(self, query: Any, k: int = 10, dataframe: Any = None):
        out_df = self._resolve_output_dataframe(dataframe)
        query_is_df = _detect_dataframe_kind(query) is not None
        q = _parse_input(query)
        dims = q.shape[-1]
        if q.ndim == 1:
            if not query_is_df and dims != self._dims:
                raise ValueError(f"query dims mismatch: expected {self._dims}, got {dims}")
            if query_is_df and dims != self._dims:
                raise ValueError(f"query dims mismatch: expected {self._dims}, got {dims}")
            res = self._single_or_raise(q, k)
            return self._to_df([res], *out_df) if out_df else res
        if dims != self._dims:
            raise ValueError(f"query dims mismatch: expected {self._dims}, got {dims}")
        # A one-row float32 matrix that is not contiguous takes the batch path in the reference
        # (src/python_bindings.rs:170-198: the single search needs `as_slice`).
        strided_f32 = (not query_is_df and isinstance(query, np.ndarray) and query.dtype == np.float32
                       and query.ndim == 2 and not query.flags.c_contiguous)
        if q.shape[0] == 1 and not strided_f32:
            res = self._single_or_raise(q.reshape(-1), k)
            return self._to_df([res], *out_df) if out_df else res
        try:
            idx, sim, cnt = self._search_batch(q, k)
        except NNdexError as e:
            raise RuntimeError(str(e)) from e
        if out_df:
            # every query's own neighbours (neighbors_to_source_dataframe, src/python_bindings.rs:500-553)
            n = [int(c) for c in cnt]
            return self._to_df([(idx[r, :n[r]], sim[r, :n[r]]) for r in range(idx.shape[0])], *out_df)
        return self._rectangular(idx, sim, cnt)

    def _single_or_raise(self, q: np.ndarray, k: int):
        try:
            return self._search_single(q, k)
        except NNdexError as e:
            raise RuntimeError(str(e)) from e

    # ---- DataFrame output (src/python_bindings.rs:420-553) ----
    def _resolve_output_dataframe(self, dataframe: Any):
        if dataframe is None:
            return None
        kind = _detect_dataframe_kind(dataframe)
        if kind is None:
            raise ValueError("`dataframe` must be a pandas.DataFrame or polars.DataFrame")
        n = int(dataframe.shape[0]) if kind == "pandas" else int(dataframe.height)
        if n != self._rows:
            raise ValueError(
                f"provided dataframe row count must match index rows (index rows={self._rows}, dataframe rows={n})")
        return (kind, dataframe)

    @staticmethod
    def _to_df(batch, kind, source):
        frames = []
        for idx, sim in batch:
            rows = [int(i) for i in idx]
            sims = [float(s) for s in sim]
            if kind == "pandas":
                frames.append(source.take(rows).assign(similarity=sims))
            else:
                import polars as pl  # noqa: PLC0415
                frames.append(source[rows].with_columns(pl.Series("similarity", sims)))
        return frames[0] if len(frames) == 1 else frames


class Server:
    """Continuous-batching request loop over one index (nndex_cuda_server_*; see include/nndex_cuda.h).

    ``submit`` queues a request and returns a ticket at once; ``poll`` returns ``(indices, scores)``
    (or ``None`` while the request runs); ``result`` waits for it. Results have the shape the
    index's own ``search`` gives for a batch (rows × min(k, rows), padded like search_batch).
    The index must outlive the server.
    """

    def __init__(self, index: NNdex, slots: int = 2, max_batch_queries: int = 4096,
                 queue_capacity: int = 1 << 20, slot_bytes: int = 0, latency_budget_ms: int = 0):
        self._index = index  # keeps the index alive while the server runs
        o = _lib.ServerOpts()
        o.slots = slots
        o.max_batch_queries = max_batch_queries
        o.queue_capacity = queue_capacity
        o.slot_bytes = slot_bytes
        o.latency_budget_ms = latency_budget_ms
        h = C.c_void_p()
        _check(_lib.lib().nndex_cuda_server_start(index.handle, C.byref(o), C.byref(h)))
        self._h = h
        self._shapes = {}

    def submit(self, queries: Any, k: int = 10, approx: bool = False, nprobe: int = 0) -> int:
        q = _parse_input(queries)
        if q.ndim == 1:
            q = q.reshape(1, -1)
        t = C.c_uint64(0)
        st = _lib.lib().nndex_cuda_server_submit(self._h, q.ctypes.data, q.shape[0], q.shape[1], int(k),
                                                 NNDEX_FLAG_APPROX if approx else 0, int(nprobe), C.byref(t))
        if st != 0:
            raise NNdexError(st, _lib.last_error())
        self._shapes[t.value] = (q.shape[0], max(min(int(k), self._index.rows), 1))
        return t.value

    def poll(self, ticket: int, timeout: float | None = 0.0, with_info: bool = False):
        rows, kk = self._shapes[ticket]
        idx = np.zeros((rows, kk), dtype=np.uint64)
        sim = np.zeros((rows, kk), dtype=np.float32)
        cnt = np.zeros(rows, dtype=np.uint64)
        info = _lib.RequestInfo()
        ms = -1 if timeout is None else int(timeout * 1000)
        st = _lib.lib().nndex_cuda_server_poll(self._h, ticket, ms, idx.ctypes.data, sim.ctypes.data, cnt.ctypes.data,
                                               C.byref(info))
        if st == _lib.NNDEX_PENDING:
            return None
        del self._shapes[ticket]
        if st != 0:
            raise NNdexError(st, _lib.last_error())
        for r in range(rows):
            n = int(cnt[r])
            idx[r, n:] = 0
            sim[r, n:] = 0.0
        out = (idx, sim)
        if with_info:
            return out, {f: getattr(info, f) for f, _ in _lib.RequestInfo._fields_ if f != "reserved"}
        return out

    def result(self, ticket: int, with_info: bool = False):
        return self.poll(ticket, timeout=None, with_info=with_info)

    def stats(self) -> dict:
        s = _lib.ServerStats()
        _check(_lib.lib().nndex_cuda_server_stats_get(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in _lib.ServerStats._fields_}

    def stop(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().nndex_cuda_server_stop(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()

    def __del__(self):
        self.stop()

