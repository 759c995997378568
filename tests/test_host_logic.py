"""Host-side logic of the Python mirror (no GPU): argument parsing and marshalling rules."""
import numpy as np
import pytest

import nndex_b200 as nb


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
