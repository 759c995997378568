"""Host-side logic of the Python mirror (no GPU): argument parsing and marshalling rules."""
import ctypes as C

import numpy as np
import pytest

import nndex_b200 as nb
from nndex_b200 import _lib


def test_parse_backend():
    assert nb._parse_backend("CUDA") == "cuda"
    with pytest.raises(ValueError, match="unsupported backend 'cpu', expected one of: cuda"):
        nb._parse_backend("cpu")


def test_parse_input_lists_and_dtypes():
    a = nb._parse_input([[1, 2], [3, 4]])
    assert a.dtype == np.float32 and a.shape == (2, 2)
    b = nb._parse_input(np.arange(4, dtype=np.float64))
    assert b.dtype == np.float32 and b.shape == (4,)
    with pytest.raises(ValueError, match="consistent row lengths"):
        nb._parse_input([[1, 2], [3]])
    with pytest.raises(ValueError, match="non-empty"):
        nb._parse_input([])
    with pytest.raises(ValueError, match="only 1D and 2D"):
        nb._parse_input(np.zeros((2, 2, 2), np.float32))


def test_parse_input_dataframe():
    pd = pytest.importorskip("pandas")
    df = pd.DataFrame(np.eye(3, dtype=np.float32))
    assert nb._detect_dataframe_kind(df) == "pandas"
    assert nb._parse_input(df).shape == (3, 3)


def test_precision_validated_before_device():
    with pytest.raises(ValueError, match="unsupported precision"):
        nb.NNdex(np.eye(8, dtype=np.float32), precision="fp16")
    with pytest.raises(ValueError, match="unsupported backend"):
        nb.NNdex(np.eye(8, dtype=np.float32), backend="gpu")


def test_oracle_ivf_from_layout_equals_built():
    # the CPU baseline times the reference's IVF search on a given layout: same results as the build
    from oracle import oracle as O
    rng = np.random.default_rng(0)
    m = rng.normal(size=(3000, 32)).astype(np.float32)
    st, storage = O.prepare_index(m, False)
    a = O.IvfIndex(storage, nlist=20, iters=3, seed=1)
    lay = {"centroids": a.centroids, "cluster_offsets": a.offsets, "original_indices": a.original_indices}
    b = O.IvfIndex(storage, layout=lay)
    q = storage[:5]
    ra, rb = a.search(q, 10, 4), b.search(q, 10, 4)
    assert np.array_equal(ra[0], rb[0]) and np.array_equal(ra[1], rb[1])


def test_tf32_split_error_term():
    # The TF32 candidate scan's split: x = xb + xs with xb = x's top 10 mantissa bits (exact in
    # TF32) and xs = x - xb (exact in FP32); likewise q. It computes xb·qb + xb·T(qs) + T(xs)·qb,
    # where T keeps 10 mantissa bits (truncation or rounding). Each product is then off by less
    # than 3·2^-20·|x_i q_i|: the split part of the certificate's bound. Checked in exact
    # arithmetic (float64 holds these products exactly) on unit vectors, worst case over T.
    rng = np.random.default_rng(3)

    def head(v):
        return (v.view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)

    def rne10(v):  # round to nearest, 10 mantissa bits
        u = v.view(np.uint32).astype(np.uint64)
        u = (u + 0xFFF + ((u >> 13) & 1)) & 0xFFFFE000
        return u.astype(np.uint32).view(np.float32)

    for _ in range(20):
        x = rng.normal(size=768).astype(np.float32)
        q = rng.normal(size=768).astype(np.float32)
        x /= np.linalg.norm(x)
        q /= np.linalg.norm(q)
        xb, qb = head(x), head(q)
        xs, qs = (x - xb).astype(np.float32), (q - qb).astype(np.float32)
        assert np.array_equal(xb.astype(np.float64) + xs, x.astype(np.float64))  # the split is exact
        for t in (head, rne10):
            prod = (xb.astype(np.float64) * qb + xb.astype(np.float64) * t(qs) + t(xs).astype(np.float64) * qb)
            err = np.abs(prod - x.astype(np.float64) * q.astype(np.float64))
            bound = 3 * 2.0 ** -20 * np.abs(x.astype(np.float64) * q.astype(np.float64))
            assert np.all(err <= bound)
        assert np.abs((x.astype(np.float64) * q).sum()) <= 1 + 1e-6


def test_autotune_cache_text_is_validated_without_a_gpu():
    # the tuner's export format: a header naming device, shape and flags, then one line per shape
    L = _lib.lib()
    n = C.c_uint64(0)
    good = (b"nndex-autotune v2 device=NVIDIA_B200 rows=1000000 dims=768 flags=1\n"
            b"shape ivf=0 nq=16 k=128 precision=0 nprobe=0 plan path=6 stride=0 qb=0 ms=0.512\n"
            b"shape ivf=1 nq=1024 k=16 precision=3 nprobe=32 plan path=5 stride=0 qb=0 ms=2.5\n\n")
    assert L.nndex_cuda_autotune_validate(good, C.byref(n)) == 0 and n.value == 2
    two = good + b"shape ivf=0 nq=256 k=16 precision=1 nprobe=0 plan path=2 stride=8 qb=2 ms=20.5\n"
    assert L.nndex_cuda_autotune_validate(two, C.byref(n)) == 0 and n.value == 3
    pair = two + b"shape ivf=0 nq=512 k=16 precision=1 nprobe=0 plan path=2 stride=8 qb=3 ms=30.5\n"  # CTA pairs
    assert L.nndex_cuda_autotune_validate(pair, C.byref(n)) == 0 and n.value == 4
    bad = [
        b"shape ivf=0 nq=16 k=128 precision=0 nprobe=0 plan path=6 stride=0 qb=0 ms=0.5\n",  # no header
        good + b"shape ivf=0 nq=12 k=128 precision=0 nprobe=0 plan path=1 stride=0 qb=0 ms=1\n",  # nq not 2^n
        good + b"shape ivf=0 nq=16 k=16 precision=0 nprobe=0 plan path=4 stride=0 qb=0 ms=1\n",  # IVF path, exact shape
        good + b"shape ivf=1 nq=16 k=16 precision=0 nprobe=8 plan path=2 stride=0 qb=0 ms=1\n",  # exact path, IVF shape
        good + b"shape ivf=0 nq=16 k=16 precision=0 nprobe=0 plan path=9 stride=0 qb=0 ms=1\n",  # no such path
        good + b"shape ivf=0 nq=16 k=16 precision=0 nprobe=0 plan path=1 stride=0 qb=2 ms=1\n",  # qb off path 2/3
        good + b"shape ivf=0 nq=256 k=16 precision=1 nprobe=0 plan path=2 stride=8 qb=4 ms=1\n",  # qb above 3
        good + b"shape ivf=0 nq=256 k=16 precision=1 nprobe=0 plan path=2 stride=8 ms=1\n",  # no qb field
        good + b"garbage\n",
    ]
    for text in bad:
        assert L.nndex_cuda_autotune_validate(text, C.byref(n)) == _lib.NNDEX_ERR_INVALID_ARGUMENT, text
        assert "autotune text" in _lib.last_error()
    assert L.nndex_cuda_autotune_validate(None, C.byref(n)) == _lib.NNDEX_ERR_INVALID_ARGUMENT


def test_launch_planners_fill_the_sms_in_whole_rounds():
    # The scans' grids, computed on the host without a GPU: one CTA fills an SM, so a launch takes
    # ceil(CTAs / SMs) rounds, and the planners avoid a last round that leaves most SMs idle.
    L = _lib.lib()
    nr, rr = C.c_uint64(), C.c_uint64()

    def ranges(rows, groups, sms=148):
        assert L.nndex_cuda_plan_tc_ranges(rows, groups, sms, C.byref(nr), C.byref(rr)) == 0
        return nr.value, rr.value

    # 4,096 queries (32 blocks) over 10M rows: 37 ranges, 1,184 CTAs in exactly 8 rounds (four ranges
    # per SM gave 19 ranges: 608 CTAs, a fifth round of 16)
    assert ranges(10_000_000, 32) == (37, 270_336)
    assert ranges(10_000_000, 1) == (148, 67_584)  # one block: a range per SM
    assert ranges(12_000, 3) == (6, 2_048)  # a small base: ranges of at least 2,048 rows
    for rows in (3_000, 50_000, 1_000_000, 10_000_000, 123_457):
        for groups in (1, 2, 3, 7, 16, 32, 33, 100, 148, 300, 2_000):
            n, r = ranges(rows, groups)
            assert r % 256 == 0 and (n - 1) * r < rows <= n * r, (rows, groups, n, r)
            tiles = -(-rows // 256)
            old = max(1, min(-(-4 * 148 // groups), -(-rows // 2048)))  # four ranges per SM
            old_r = -(-(-(-rows // old)) // 256) * 256
            old_n = -(-rows // old_r)
            cost = -(-groups * n // 148) * (r // 256)
            assert cost <= -(-groups * old_n // 148) * (old_r // 256), (rows, groups)
            assert n * groups <= max(8 * 148, groups), (rows, groups)  # within the launch's item bound
            assert tiles >= 1
    assert L.nndex_cuda_plan_tc_ranges(0, 1, 148, C.byref(nr), C.byref(rr)) == _lib.NNDEX_ERR_INVALID_ARGUMENT

    qb, groups, ctas = C.c_uint32(), C.c_uint32(), C.c_uint32()

    def fp32(nq, dims, k, rows, sms=148, smem=232_448):
        assert L.nndex_cuda_plan_fp32_scan(nq, dims, k, rows, sms, smem, C.byref(qb), C.byref(groups),
                                           C.byref(ctas)) == 0
        return qb.value, groups.value, ctas.value

    assert fp32(1, 128, 10, 50_000) == (1, 1, 148)  # a single query: one group over every SM
    assert fp32(64, 128, 10, 50_000) == (16, 4, 37)  # C1's batch: the rule's fill, kept
    # 4,096 queries: 256 groups of 16; four CTAs per group take 7 rounds of 148 (1.75 bases) where
    # one took 2 (the second with 40 SMs idle)
    assert fp32(4096, 256, 10, 10_000_000) == (16, 256, 4)
    assert fp32(4096, 256, 10, 5_000)[2] == 1  # too few rows to split: one CTA per group
    assert L.nndex_cuda_plan_fp32_scan(16, 0, 10, 100, 148, 232_448, C.byref(qb), C.byref(groups),
                                       C.byref(ctas)) == _lib.NNDEX_ERR_INVALID_ARGUMENT
