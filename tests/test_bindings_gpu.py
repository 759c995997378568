"""The Python binding's cases (tests_python/test_bindings.py) on the CUDA backend: list / numpy /
DataFrame inputs, output shapes, DataFrame outputs (src/python_bindings.rs:125-236, 404-553)."""
import numpy as np
import pytest

from nndex_b200 import NNdex

pytestmark = pytest.mark.gpu

EYE = np.eye(8, dtype=np.float32)


def test_list_input_and_search_output_shapes():
    matrix = [[1.0, 0, 0, 0, 0, 0, 0, 0], [0, 1.0, 0, 0, 0, 0, 0, 0], [1.0, 1.0, 0, 0, 0, 0, 0, 0]]
    model = NNdex(matrix, normalized=False, backend="cuda")
    indices, scores = model.search([0.8, 0.6, 0, 0, 0, 0, 0, 0], k=2)
    assert indices.shape == (2,) and scores.shape == (2,)
    assert indices.dtype == np.uint64 and scores.dtype == np.float32
    assert int(indices[0]) == 2
    assert float(scores[0]) > float(scores[1])


def test_numpy_batch_query():
    model = NNdex(EYE, normalized=True)
    indices, scores = model.search(np.vstack([EYE[0], EYE[1]]), k=2)
    assert indices.shape == (2, 2) and scores.shape == (2, 2)
    assert int(indices[0, 0]) == 0 and int(indices[1, 0]) == 1


def test_backend_property_and_approx_flag():
    model = NNdex(EYE, normalized=True, approx=True)
    assert model.backend == "cuda"
    assert int(model.search(EYE[0], k=1)[0][0]) == 0


def test_one_row_matrix_query_is_a_single_search():
    model = NNdex(EYE, normalized=True)
    i, s = model.search(EYE[:1], k=3)
    assert i.shape == (3,)
    # a strided one-row float32 matrix takes the batch path (no contiguous slice)
    strided = np.repeat(EYE[:1], 2, axis=1)[:, ::2]
    assert not strided.flags.c_contiguous
    i2, s2 = model.search(strided, k=3)
    assert i2.shape == (1, 3)
    assert np.array_equal(i2[0], i)


def test_pandas_dataframe_returns_dataframe():
    pd = pytest.importorskip("pandas")
    matrix = pd.DataFrame({c: v for c, v in zip("abcdefgh", [[1.0, 0.0, 1.0], [0.0, 1.0, 1.0]] + [[0.0] * 3] * 6)})
    model = NNdex(matrix, normalized=False)
    result = model.search(matrix.iloc[[0]], k=2, dataframe=matrix)
    assert isinstance(result, pd.DataFrame)
    assert list(result.columns) == [*matrix.columns, "similarity"]
    assert len(result) == 2
    assert float(result.iloc[0]["similarity"]) >= float(result.iloc[1]["similarity"])


def test_pandas_multi_query_returns_list_of_dataframes():
    pd = pytest.importorskip("pandas")
    matrix = pd.DataFrame(EYE)
    model = NNdex(matrix, normalized=True)
    result = model.search(matrix.iloc[[0, 1]], k=2, dataframe=matrix)
    assert isinstance(result, list) and len(result) == 2
    assert all(isinstance(f, pd.DataFrame) and "similarity" in f.columns for f in result)


def test_pandas_query_on_numpy_built_index():
    pd = pytest.importorskip("pandas")
    df = pd.DataFrame(EYE)
    model = NNdex(EYE, normalized=True)
    result = model.search(df, k=1, dataframe=df)
    assert isinstance(result, list) and len(result) == 8
    assert all(len(f) == 1 for f in result)
    with pytest.raises(ValueError, match="row count must match index rows"):
        model.search(EYE[0], k=1, dataframe=df.iloc[:2])
    indices, scores = model.search(pd.DataFrame(EYE[:2]), k=1)
    assert indices.shape == (2, 1) and scores.shape == (2, 1)


def test_ragged_batch_outputs():
    """Approx searches that find fewer than k rows: numpy rows are padded with (0, 0.0) to the
    first row's width (or cut to it), DataFrames keep every query's own neighbours."""
    pd = pytest.importorskip("pandas")
    rng = np.random.default_rng(3)
    base = rng.normal(size=(3_000, 16)).astype(np.float32)
    q = rng.normal(size=(40, 16)).astype(np.float32)
    model = NNdex(base, approx=True, nlist=60, nprobe=1)
    df = pd.DataFrame(base)
    frames = model.search(q, k=200, dataframe=df)
    lengths = [len(f) for f in frames]
    assert len(set(lengths)) > 1 and max(lengths) < 200
    idx, sim = model.search(q, k=200)
    assert idx.shape == (40, lengths[0])
    for r, f in enumerate(frames):
        n = min(lengths[r], lengths[0])
        assert np.array_equal(idx[r, :n], f.index.to_numpy()[:n].astype(np.uint64))
        assert np.array_equal(sim[r, :n], f["similarity"].to_numpy().astype(np.float32)[:n])
        assert not idx[r, n:].any() and not sim[r, n:].any()
