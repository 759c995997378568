"""Parity checks of CUDA results against the FP64 oracle (test helper).

The acceptance rule for exact search: every returned score is within `tol` (1e-5, absolute) of
the FP64 score of its row; indices equal the canonical FP64 top-k (similarity desc, index asc)
wherever the FP64 gap to the neighbouring ranks exceeds `tol`; inside a near-tie group the
returned rows are a valid choice from that group.
"""
from __future__ import annotations

import numpy as np

TOL = 1e-5


def canonical_order(scores: np.ndarray) -> np.ndarray:
    """Row order by score descending, then row index ascending."""
    n = scores.shape[0]
    return np.lexsort((np.arange(n), -scores))


def assert_topk_matches(gidx, gsim, s64, k, tol=TOL, what=""):
    gidx = np.asarray(gidx, dtype=np.int64)
    gsim = np.asarray(gsim, dtype=np.float64)
    n = s64.shape[0]
    kk = min(k, n)
    assert gidx.shape[0] == kk, f"{what}: expected {kk} results, got {gidx.shape[0]}"
    assert len(set(gidx.tolist())) == kk, f"{what}: duplicate rows {gidx}"
    assert np.all((gidx >= 0) & (gidx < n)), f"{what}: row out of range"
    err = np.abs(gsim - s64[gidx])
    assert np.all(err <= tol), f"{what}: score error {err.max():.3g} > {tol}"
    # returned order: similarity desc, ties by index asc
    for j in range(kk - 1):
        a, b = gsim[j], gsim[j + 1]
        assert a > b or (a == b and gidx[j] < gidx[j + 1]), f"{what}: order broken at {j}: {gidx[j:j+2]} {gsim[j:j+2]}"
    order = canonical_order(s64)
    ref = order[:kk]
    rs = s64[ref]
    nxt = s64[order[kk]] if kk < n else -np.inf
    # every returned row is eligible; every clearly-in row is returned
    assert np.all(s64[gidx] >= rs[-1] - tol), f"{what}: returned a row below the k-th score"
    must = ref[rs > nxt + tol]
    missing = set(must.tolist()) - set(gidx.tolist())
    assert not missing, f"{what}: rows {sorted(missing)[:10]} missing"
    # rank consistency and exact positions where isolated
    assert np.all(np.abs(s64[gidx] - rs) <= 2 * tol), f"{what}: rank mismatch"
    for j in range(kk):
        lo_ok = j == 0 or rs[j - 1] - rs[j] > tol
        hi_ok = (rs[j] - (rs[j + 1] if j + 1 < kk else nxt)) > tol
        if lo_ok and hi_ok:
            assert gidx[j] == ref[j], f"{what}: position {j}: got row {gidx[j]}, expected {ref[j]}"
