"""ctypes binding of the C ABI in include/nndex_cuda.h (libnndex_cuda.so, built in-tree).

This is the Python-side counterpart of the `extern "C"` block a Rust `CudaIndex` would declare.
Loading fails loudly when the shared object is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnndex_cuda.so")

NNDEX_OK = 0
NNDEX_ERR_SHAPE_MISMATCH = 1
NNDEX_ERR_QUERY_DIMS = 2
NNDEX_ERR_INVALID_TOPK = 3
NNDEX_ERR_NON_FINITE = 4
NNDEX_ERR_ZERO_NORM = 5
NNDEX_ERR_CUDA = 6
NNDEX_ERR_OUT_OF_MEMORY = 7
NNDEX_ERR_TIMEOUT = 8
NNDEX_ERR_ADMISSION = 9
NNDEX_ERR_INVALID_ARGUMENT = 10
NNDEX_ERR_DEVICE_INDEX = 11
NNDEX_ERR_UNSUPPORTED = 12
NNDEX_PENDING = 13  # serving: the request has not finished (not an error)

NNDEX_FLAG_NORMALIZED = 0x1
NNDEX_FLAG_APPROX = 0x2
NNDEX_FLAG_BF16 = 0x4
NNDEX_FLAG_FP8 = 0x8

NNDEX_PRECISION_AUTO = 0
NNDEX_PRECISION_FP32 = 1
NNDEX_PRECISION_BF16 = 2
NNDEX_PRECISION_FP8 = 3


class Opts(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("precision", C.c_uint32),
        ("nlist", C.c_uint32),
        ("nprobe", C.c_uint32),
        ("kmeans_iters", C.c_uint32),
        ("has_seed", C.c_uint32),
        ("seed", C.c_uint64),
        ("rerank_width", C.c_uint32),
        ("reserved", C.c_uint32 * 7),
    ]


class DevInfo(C.Structure):
    _fields_ = [
        ("index", C.c_uint64),
        ("name", C.c_char * 256),
        ("driver", C.c_char * 64),
        ("driver_info", C.c_char * 64),
        ("backend", C.c_char * 32),
        ("device_type", C.c_char * 32),
        ("sm_count", C.c_uint32),
        ("cc_major", C.c_uint32),
        ("cc_minor", C.c_uint32),
        ("hbm_bytes", C.c_uint64),
        ("l2_bytes", C.c_uint64),
    ]


class SearchStats(C.Structure):
    _fields_ = [
        ("path", C.c_uint32),
        ("kernel_launches", C.c_uint32),
        ("rerank_width", C.c_uint32),
        ("certified", C.c_uint32),
        ("second_pass_queries", C.c_uint32),
        ("nprobe", C.c_uint32),
        ("rows_scanned", C.c_uint64),
        ("device_ms", C.c_double),
        ("fp32_fallback_queries", C.c_uint32),
        ("pass1_tile_stride", C.c_uint32),
        ("ivf_rows_streamed", C.c_uint64),
        ("ivf_rows_union", C.c_uint64),
        ("scan_qb", C.c_uint32),
        ("scan_wide", C.c_uint32),
        ("graph", C.c_uint32),
        ("score_errors", C.c_uint32),
        ("max_score_error", C.c_double),
        ("mean_score_error", C.c_double),
        ("tuned", C.c_uint32),
        ("tune_candidates", C.c_uint32),
        ("pass2_rows", C.c_uint64),
        ("pass2_query_blocks", C.c_uint32),
        ("reserved0", C.c_uint32),
    ]


class IvfStats(C.Structure):
    _fields_ = [
        ("nlist", C.c_uint64),
        ("iters", C.c_uint64),
        ("max_list", C.c_uint64),
        ("build_ms", C.c_double),
        ("seed_ms", C.c_double),
        ("kmeans_ms", C.c_double),
        ("layout_ms", C.c_double),
        ("seed_exact_rows", C.c_uint64),
        ("ambiguous_rows", C.c_uint64),
        ("candidate_rows", C.c_uint64),
        ("reserved", C.c_uint64 * 3),
    ]


class ServerOpts(C.Structure):
    _fields_ = [
        ("slots", C.c_uint32),
        ("max_batch_queries", C.c_uint32),
        ("queue_capacity", C.c_uint64),
        ("slot_bytes", C.c_uint64),
        ("latency_budget_ms", C.c_uint32),
        ("reserved", C.c_uint32 * 7),
    ]


class RequestInfo(C.Structure):
    _fields_ = [
        ("submit_ns", C.c_uint64),
        ("start_ns", C.c_uint64),
        ("done_ns", C.c_uint64),
        ("batch_id", C.c_uint64),
        ("batch_queries", C.c_uint32),
        ("slot", C.c_uint32),
        ("path", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("requests_done", C.c_uint64),
        ("queries_done", C.c_uint64),
        ("batches", C.c_uint64),
        ("refused", C.c_uint64),
        ("queued_queries", C.c_uint64),
        ("max_queued_queries", C.c_uint64),
        ("slots", C.c_uint32),
        ("max_batch_queries", C.c_uint32),
        ("slot_bytes", C.c_uint64),
        ("refused_latency", C.c_uint64),
        ("us_per_query", C.c_double),
        ("fp32_fallback_queries", C.c_uint64),
        ("slowest_batch_ms", C.c_double),
        ("slowest_batch_queries", C.c_uint32),
        ("slowest_batch_k", C.c_uint32),
        ("slowest_batch_path", C.c_uint32),
        ("slowest_batch_approx", C.c_uint32),
    ]


_vp = C.c_void_p
_u64 = C.c_uint64
_u32 = C.c_uint32
_i32 = C.c_int

# name → (restype, argtypes); every name here is declared in include/nndex_cuda.h.
SIGNATURES = {
    "nndex_cuda_last_error": (C.c_char_p, []),
    "nndex_cuda_list_devices": (_i32, [C.POINTER(DevInfo), _u32, C.POINTER(_u32)]),
    "nndex_cuda_info": (_i32, [_vp, C.POINTER(DevInfo)]),
    "nndex_cuda_create": (_i32, [_vp, _u64, _u64, _u64, _u32, C.POINTER(Opts), C.POINTER(_vp)]),
    "nndex_cuda_create_from_device": (_i32, [_vp, _u64, _u64, _u64, _u32, C.POINTER(Opts), C.POINTER(_vp)]),
    "nndex_cuda_destroy": (None, [_vp]),
    "nndex_cuda_builder_begin": (_i32, [_u64, _u64, _u32, C.POINTER(Opts), C.POINTER(_vp)]),
    "nndex_cuda_builder_append": (_i32, [_vp, _vp, _u64]),
    "nndex_cuda_builder_finish": (_i32, [_vp, C.POINTER(_vp)]),
    "nndex_cuda_builder_abort": (None, [_vp]),
    "nndex_cuda_create_from_npy": (_i32, [C.c_char_p, _u32, C.POINTER(Opts), C.POINTER(_vp)]),
    "nndex_cuda_rows": (_i32, [_vp, C.POINTER(_u64), C.POINTER(_u64), C.POINTER(_u64)]),
    "nndex_cuda_search": (_i32, [_vp, _vp, _u64, _u64, _vp, _vp, C.POINTER(_u64)]),
    "nndex_cuda_search_batch": (_i32, [_vp, _vp, _u64, _u64, _u64, _vp, _vp, _vp]),
    "nndex_cuda_search_batch_device": (_i32, [_vp, _vp, _u64, _u64, _u64, _vp, _vp, _vp, _vp, _i32]),
    "nndex_cuda_stream_status": (_i32, [_vp]),
    "nndex_cuda_set_precision": (_i32, [_vp, _u32, _u32]),
    "nndex_cuda_last_candidates": (_i32, [_vp, _u64, _vp, _vp, _u64, C.POINTER(_u32), C.POINTER(C.c_float), _vp]),
    "nndex_cuda_last_search_stats": (_i32, [_vp, C.POINTER(SearchStats)]),
    "nndex_cuda_kernel_launch_count": (_u64, []),
    "nndex_cuda_set_scan_timing": (_i32, [_vp, _i32]),
    "nndex_cuda_scan_timing": (_i32, [_vp, C.POINTER(C.c_double), C.POINTER(_u64)]),
    "nndex_cuda_fp64_scores": (_i32, [_vp, _vp, _u64, _vp, _vp, _u64, _vp]),
    "nndex_cuda_set_error_report": (_i32, [_vp, _i32]),
    "nndex_cuda_set_autotune": (_i32, [_vp, _i32]),
    "nndex_cuda_autotune_export": (_i32, [_vp, C.c_char_p, _u64, C.POINTER(_u64)]),
    "nndex_cuda_autotune_import": (_i32, [_vp, C.c_char_p]),
    "nndex_cuda_autotune_validate": (_i32, [C.c_char_p, C.POINTER(_u64)]),
    "nndex_cuda_last_score_errors": (_i32, [_vp, _u64, _u64, _vp]),
    "nndex_cuda_search_batch_device_noalloc": (_i32, [_vp, _vp, _u64, _u64, _u64, _vp, _vp, _vp, _vp]),
    "nndex_cuda_ivf_layout": (_i32, [_vp, C.POINTER(_u64), _vp, _vp, _vp, _vp]),
    "nndex_cuda_ivf_stats_get": (_i32, [_vp, C.POINTER(IvfStats)]),
    "nndex_cuda_set_nprobe": (_i32, [_vp, _u32]),
    "nndex_cuda_set_graphs": (_i32, [_vp, _i32]),
    "nndex_cuda_check_bounded_wait": (_i32, [_vp, _u64]),
    "nndex_cuda_inject_alloc_failures": (None, [_u32]),
    "nndex_cuda_plan_tc_ranges": (_i32, [_u64, _u64, _u32, C.POINTER(_u64), C.POINTER(_u64)]),
    "nndex_cuda_plan_fp32_scan": (_i32, [_u32, _u32, _u32, _u64, _u32, _u64, C.POINTER(_u32), C.POINTER(_u32),
                                         C.POINTER(_u32)]),
    "nndex_cuda_ivf_restore": (_i32, [_vp, _u64, _vp, _vp, _vp, _vp]),
    "nndex_cuda_base_checksum": (_i32, [_vp, C.POINTER(_u64)]),
    "nndex_cuda_server_start": (_i32, [_vp, C.POINTER(ServerOpts), C.POINTER(_vp)]),
    "nndex_cuda_server_submit": (_i32, [_vp, _vp, _u64, _u64, _u64, _u32, _u32, C.POINTER(_u64)]),
    "nndex_cuda_server_poll": (_i32, [_vp, _u64, C.c_int32, _vp, _vp, _vp, C.POINTER(RequestInfo)]),
    "nndex_cuda_server_stats_get": (_i32, [_vp, C.POINTER(ServerStats)]),
    "nndex_cuda_server_stop": (None, [_vp]),
}

NNDEX_NOALLOC_SCRATCH_BYTES = 16 << 20

_lib = None


def lib() -> C.CDLL:
    """Load libnndex_cuda.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `python -m nndex_b200.build`")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return lib().nndex_cuda_last_error().decode("utf-8", "replace")
