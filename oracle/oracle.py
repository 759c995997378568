"""ctypes view of the CPU oracle (oracle/nndex_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker the CUDA backend is compared against and the timed CPU
baseline. Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this module;
the product package (nndex_b200) never does.

Each wrapper names the reference function (fblissjr/nndex, file:line) the C code restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libnndex_oracle.so")
_lib = None

NNDEX_OK = 0
NNDEX_ERR_SHAPE_MISMATCH = 1
NNDEX_ERR_NON_FINITE = 4
NNDEX_ERR_ZERO_NORM = 5

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u64 = C.c_uint64


def build() -> str:
    """Compile the oracle with its Makefile (system gcc) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE, "CC=gcc"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    sig = {
        "or_dot_unrolled_8": (C.c_float, [_f32p, _f32p, _u64]),
        "or_dot_product": (C.c_float, [_f32p, _f32p, _u64]),
        "or_dot_small": (C.c_float, [_f32p, _f32p, _u64]),
        "or_validate_matrix_shape": (C.c_int, [_u64, _u64, _u64]),
        "or_ensure_finite": (C.c_int, [_f32p, _u64]),
        "or_normalize_rows": (C.c_int, [_f32p, _u64, _u64, _u64, _f32p, C.POINTER(C.c_uint64)]),
        "or_normalize_vector": (C.c_int, [_f32p, _u64, _u64, _f32p]),
        "or_pad_rows": (None, [_f32p, _u64, _u64, _u64, _f32p]),
        "or_padded_dims": (_u64, [_u64]),
        "or_topk_new": (C.c_void_p, [_u64]),
        "or_topk_free": (None, [C.c_void_p]),
        "or_topk_push": (None, [C.c_void_p, _u64, C.c_float]),
        "or_topk_push_slow": (None, [C.c_void_p, _u64, C.c_float]),
        "or_topk_merge": (None, [C.c_void_p, C.c_void_p]),
        "or_topk_into_sorted": (_u64, [C.c_void_p, _u64p, _f32p]),
        "or_topk_threshold": (C.c_float, [C.c_void_p]),
        "or_topk_from_scores": (_u64, [_f32p, _u64, _u64, _u64, _u64p, _f32p]),
        "or_search_exact": (None, [_f32p, _u64, _u64, _f32p, _u64, _u64, _u64p, _f32p]),
        "or_scores_f64": (None, [_f32p, _u64, _u64, _f32p, _f64p]),
        "or_search_f64": (None, [_f32p, _u64, _u64, _f32p, _u64, _u64p, _f64p, C.POINTER(C.c_double)]),
        "or_isqrt": (_u64, [_u64]),
        "or_choose_nlist": (_u64, [_u64]),
        "or_choose_nprobe": (_u64, [_u64, _u64, _u64]),
        "or_pick_medoid_row": (_u64, [_f32p, _u64, _u64]),
        "or_kmeans_plusplus_init": (None, [_f32p, _u64, _u64, _u64, C.c_int, _u64, _f32p, _u64p]),
        "or_spherical_kmeans": (None, [_f32p, _u64, _u64, _u64, _u64, _f32p, _u32p]),
        "or_kmeans_assign_rows": (None, [_f32p, _u64, _u64p, _u64, _f32p, _u64, _u32p]),
        "or_kmeans_update": (None, [_f32p, _u64, _u64, _u64, _u32p, _f32p]),
        "or_ivf_build": (C.c_void_p, [_f32p, _u64, _u64, _u64, _u64, C.c_int, _u64]),
        "or_ivf_from_layout": (C.c_void_p, [_f32p, _u64, _u64, _u64, _f32p, _u64p, _u64p]),
        "or_ivf_free": (None, [C.c_void_p]),
        "or_ivf_nlist": (_u64, [C.c_void_p]),
        "or_ivf_centroids": (C.c_void_p, [C.c_void_p]),
        "or_ivf_offsets": (C.c_void_p, [C.c_void_p]),
        "or_ivf_original": (C.c_void_p, [C.c_void_p]),
        "or_ivf_assign": (C.c_void_p, [C.c_void_p]),
        "or_ivf_init_rows": (C.c_void_p, [C.c_void_p]),
        "or_ivf_provides_speedup": (C.c_int, [C.c_void_p]),
        "or_ivf_probe": (_u64, [C.c_void_p, _f32p, _u64, _u64p, _f32p]),
        "or_ivf_search": (_u64, [C.c_void_p, _f32p, _u64, _u64, _u64p, _f32p]),
        "or_ivf_search_batch": (None, [C.c_void_p, _f32p, _u64, _u64, _u64, _u64p, _f32p, _u64p]),
        "or_num_threads": (C.c_int, []),
        "or_set_num_threads": (None, [C.c_int]),
        "or_bench_search_single": (_u64, [_f32p, _u64, _u64, _f32p, _u64, _u64p, _f32p]),
        "or_bench_search_batch": (None, [_f32p, _u64, _u64, _f32p, _u64, _u64, _u64p, _f32p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


# ---- normalisation (src/lib.rs:433-599) ---------------------------------------------------

def padded_dims(dims: int) -> int:
    """src/lib.rs:192 dims.next_multiple_of(8)."""
    return int(lib().or_padded_dims(dims))


def normalize_rows(values: np.ndarray, rows: int, dims: int, padded: int):
    """src/lib.rs:461-514 normalize_rows → (status, out[rows, padded], bad_row)."""
    v = _c(values, np.float32).reshape(-1)
    out = np.zeros(rows * padded, dtype=np.float32)
    bad = C.c_uint64(0)
    st = lib().or_normalize_rows(v, rows, dims, padded, out, C.byref(bad))
    return st, out.reshape(rows, padded), int(bad.value)


def normalize_vector(values: np.ndarray, padded: int):
    """src/lib.rs:558-575 normalize_vector → (status, out[padded])."""
    v = _c(values, np.float32).reshape(-1)
    out = np.zeros(padded, dtype=np.float32)
    st = lib().or_normalize_vector(v, v.size, padded, out)
    return st, out


def pad_rows(values: np.ndarray, rows: int, dims: int, padded: int) -> np.ndarray:
    v = _c(values, np.float32).reshape(-1)
    out = np.zeros(rows * padded, dtype=np.float32)
    lib().or_pad_rows(v, rows, dims, padded, out)
    return out.reshape(rows, padded)


def ensure_finite(values: np.ndarray) -> int:
    v = _c(values, np.float32).reshape(-1)
    return int(lib().or_ensure_finite(v, v.size))


def prepare_index(matrix: np.ndarray, normalized: bool):
    """NNdex::new's host preparation (src/lib.rs:239-244) → (status, storage[rows, padded])."""
    m = _c(matrix, np.float32)
    rows, dims = m.shape
    pd = padded_dims(dims)
    if normalized:
        st = ensure_finite(m)
        return st, (pad_rows(m, rows, dims, pd) if st == NNDEX_OK else None)
    st, out, _ = normalize_rows(m, rows, dims, pd)
    return st, (out if st == NNDEX_OK else None)


def prepare_query(query: np.ndarray, normalized: bool, padded: int):
    """NNdex::prepare_query (src/lib.rs:404-411) → (status, q[padded])."""
    q = _c(query, np.float32).reshape(-1)
    if normalized:
        st = ensure_finite(q)
        out = np.zeros(padded, dtype=np.float32)
        out[: q.size] = q
        return st, out
    return normalize_vector(q, padded)


def prepare_queries(queries: np.ndarray, normalized: bool, padded: int):
    """NNdex::search_batch's query preparation (src/lib.rs:383-388) → (status, Q[n, padded])."""
    q = _c(queries, np.float32)
    n, dims = q.shape
    if normalized:
        st = ensure_finite(q)
        return st, pad_rows(q, n, dims, padded)
    st, out, _ = normalize_rows(q, n, dims, padded)
    return st, out


# ---- dots ---------------------------------------------------------------------------------

def dot_product(a, b) -> float:
    a = _c(a, np.float32)
    b = _c(b, np.float32)
    return float(lib().or_dot_product(a, b, a.size))


def dot_unrolled_8(a, b) -> float:
    a = _c(a, np.float32)
    b = _c(b, np.float32)
    return float(lib().or_dot_unrolled_8(a, b, a.size))


# ---- top-k (src/topk.rs) ------------------------------------------------------------------

class TopKAccumulator:
    """src/topk.rs:44-152, restated in C."""

    def __init__(self, k: int):
        self.k = k
        self.h = lib().or_topk_new(k)

    def push(self, index: int, sim: float) -> None:
        lib().or_topk_push(self.h, index, sim)

    def push_slow(self, index: int, sim: float) -> None:
        lib().or_topk_push_slow(self.h, index, sim)

    @property
    def min_threshold(self) -> float:
        return float(lib().or_topk_threshold(self.h))

    def merge(self, other: "TopKAccumulator") -> None:
        lib().or_topk_merge(self.h, other.h)
        other.h = None

    def into_sorted_vec(self):
        idx = np.zeros(max(self.k, 1), dtype=np.uint64)
        sim = np.zeros(max(self.k, 1), dtype=np.float32)
        n = lib().or_topk_into_sorted(self.h, idx, sim)
        self.h = None
        return [(int(idx[i]), float(sim[i])) for i in range(n)]

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_topk_free(self.h)
            self.h = None


def topk_from_scores(scores, k: int, row_offset: int = 0):
    """src/topk.rs:169-210."""
    s = _c(scores, np.float32).reshape(-1)
    cap = max(min(k, s.size), 1)
    idx = np.zeros(cap, dtype=np.uint64)
    sim = np.zeros(cap, dtype=np.float32)
    if s.size == 0:
        return []
    n = lib().or_topk_from_scores(s, s.size, k, row_offset, idx, sim)
    return [(int(idx[i]), float(sim[i])) for i in range(n)]


# ---- exact search -------------------------------------------------------------------------

def search_exact(storage: np.ndarray, queries: np.ndarray, k: int):
    """Canonical exact top-k (src/cpu.rs:505-639 semantics, canonical ties) → (idx, sim)."""
    base = _c(storage, np.float32)
    rows, dp = base.shape
    q = _c(queries, np.float32).reshape(-1, dp)
    kk = min(k, rows)
    idx = np.zeros(q.shape[0] * kk, dtype=np.uint64)
    sim = np.zeros(q.shape[0] * kk, dtype=np.float32)
    lib().or_search_exact(base, rows, dp, q, q.shape[0], kk, idx, sim)
    return idx.reshape(-1, kk), sim.reshape(-1, kk)


def scores_f64(storage: np.ndarray, query: np.ndarray) -> np.ndarray:
    base = _c(storage, np.float32)
    rows, dp = base.shape
    out = np.zeros(rows, dtype=np.float64)
    lib().or_scores_f64(base, rows, dp, _c(query, np.float32).reshape(-1), out)
    return out


def search_f64(storage: np.ndarray, query: np.ndarray, k: int):
    """FP64 ground truth → (idx[k], score[k], score of the (k+1)-th)."""
    base = _c(storage, np.float32)
    rows, dp = base.shape
    kk = min(k, rows)
    idx = np.zeros(kk, dtype=np.uint64)
    sc = np.zeros(kk, dtype=np.float64)
    nxt = C.c_double(0.0)
    lib().or_search_f64(base, rows, dp, _c(query, np.float32).reshape(-1), kk, idx, sc, C.byref(nxt))
    return idx, sc, float(nxt.value)


# ---- IVF (src/approx.rs) ------------------------------------------------------------------

def isqrt(n: int) -> int:
    return int(lib().or_isqrt(n))


def choose_nlist(rows: int) -> int:
    return int(lib().or_choose_nlist(rows))


def choose_nprobe(nlist: int, k: int, rows: int) -> int:
    return int(lib().or_choose_nprobe(nlist, k, rows))


def kmeans_plusplus_init(storage: np.ndarray, nlist: int, seed: int | None = None):
    """src/approx.rs:357-406: the first `nlist` k-means++ picks (the medoid first) and their rows.
    The picks do not depend on how many follow, so a small nlist gives a prefix of a larger one's."""
    m = _c(storage, np.float32)
    rows, dims = m.shape
    cent = np.zeros((nlist, dims), np.float32)
    chosen = np.zeros(nlist, np.uint64)
    lib().or_kmeans_plusplus_init(m, rows, dims, nlist, 0 if seed is None else 1, 0 if seed is None else seed,
                                  cent, chosen)
    return chosen, cent


def kmeans_assign_rows(storage: np.ndarray, row_ids: np.ndarray, centroids: np.ndarray) -> np.ndarray:
    """src/approx.rs:446-493: the assignment of the given rows (strict `>` argmax of dot_small)."""
    m = _c(storage, np.float32)
    ids = _c(row_ids, np.uint64)
    cent = _c(centroids, np.float32)
    out = np.zeros(ids.shape[0], np.uint32)
    lib().or_kmeans_assign_rows(m, m.shape[1], ids, ids.shape[0], cent, cent.shape[0], out)
    return out


def kmeans_update(storage: np.ndarray, assign: np.ndarray, nlist: int) -> np.ndarray:
    """src/approx.rs:495-531: the centroids one update makes from an assignment."""
    m = _c(storage, np.float32)
    a = _c(assign, np.uint32)
    out = np.zeros((nlist, m.shape[1]), np.float32)
    lib().or_kmeans_update(m, m.shape[0], m.shape[1], nlist, a, out)
    return out


class IvfIndex:
    """src/approx.rs:46-100 ApproxIndex::build (parameterised), with probe and rerank."""

    def __init__(self, storage: np.ndarray, nlist: int = 0, iters: int = 0, seed: int | None = None,
                 layout: dict | None = None):
        self.base = _c(storage, np.float32)
        self.rows, self.dims = self.base.shape
        if layout is not None:
            cent = _c(layout["centroids"], np.float32)
            self.h = lib().or_ivf_from_layout(self.base, self.rows, self.dims, cent.shape[0], cent,
                                              _c(layout["cluster_offsets"], np.uint64),
                                              _c(layout["original_indices"], np.uint64))
        else:
            self.h = lib().or_ivf_build(self.base, self.rows, self.dims, nlist, iters,
                                        0 if seed is None else 1, 0 if seed is None else seed)
        self.nlist = int(lib().or_ivf_nlist(self.h))

    def _arr(self, fn, ctype, n, dtype):
        p = getattr(lib(), fn)(self.h)
        if not p or n == 0:
            return np.zeros(0, dtype=dtype)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(ctype)), shape=(n,)).astype(dtype).copy()

    @property
    def centroids(self) -> np.ndarray:
        if self.nlist <= 1:
            return np.zeros((0, self.dims), dtype=np.float32)
        return self._arr("or_ivf_centroids", C.c_float, self.nlist * self.dims, np.float32).reshape(self.nlist, self.dims)

    @property
    def offsets(self) -> np.ndarray:
        return self._arr("or_ivf_offsets", C.c_uint64, self.nlist + 1, np.uint64)

    @property
    def original_indices(self) -> np.ndarray:
        return self._arr("or_ivf_original", C.c_uint64, self.rows, np.uint64)

    @property
    def assignments(self) -> np.ndarray:
        return self._arr("or_ivf_assign", C.c_uint32, self.rows, np.uint32)

    @property
    def init_rows(self) -> np.ndarray:
        if self.nlist <= 1:
            return np.zeros(0, dtype=np.uint64)
        return self._arr("or_ivf_init_rows", C.c_uint64, self.nlist, np.uint64)

    def provides_speedup(self) -> bool:
        return bool(lib().or_ivf_provides_speedup(self.h))

    def probe(self, query: np.ndarray, nprobe: int):
        q = _c(query, np.float32).reshape(-1)
        cl = np.zeros(max(nprobe, 1), dtype=np.uint64)
        cs = np.zeros(max(nprobe, 1), dtype=np.float32)
        n = lib().or_ivf_probe(self.h, q, nprobe, cl, cs)
        return cl[:n], cs[:n]

    def search(self, queries: np.ndarray, k: int, nprobe: int = 0):
        q = _c(queries, np.float32).reshape(-1, self.dims)
        nq = q.shape[0]
        kk = min(k, self.rows)
        idx = np.zeros(nq * kk, dtype=np.uint64)
        sim = np.zeros(nq * kk, dtype=np.float32)
        cnt = np.zeros(nq, dtype=np.uint64)
        lib().or_ivf_search_batch(self.h, q, nq, kk, nprobe, idx, sim, cnt)
        return idx.reshape(nq, kk), sim.reshape(nq, kk), cnt

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_ivf_free(self.h)
            self.h = None


# ---- timed CPU baseline -------------------------------------------------------------------

def num_threads() -> int:
    return int(lib().or_num_threads())


def set_num_threads(n: int) -> None:
    lib().or_set_num_threads(n)


def bench_search_single(storage: np.ndarray, query: np.ndarray, k: int):
    base = _c(storage, np.float32)
    rows, dp = base.shape
    kk = min(k, rows)
    idx = np.zeros(kk, dtype=np.uint64)
    sim = np.zeros(kk, dtype=np.float32)
    n = lib().or_bench_search_single(base, rows, dp, _c(query, np.float32).reshape(-1), kk, idx, sim)
    return idx[:n], sim[:n]


def bench_search_batch(storage: np.ndarray, queries: np.ndarray, k: int):
    base = _c(storage, np.float32)
    rows, dp = base.shape
    q = _c(queries, np.float32).reshape(-1, dp)
    kk = min(k, rows)
    idx = np.zeros(q.shape[0] * kk, dtype=np.uint64)
    sim = np.zeros(q.shape[0] * kk, dtype=np.float32)
    lib().or_bench_search_batch(base, rows, dp, q, q.shape[0], kk, idx, sim)
    return idx.reshape(-1, kk), sim.reshape(-1, kk)
