"""Generates the golden fixtures under tests/golden/ (run in a container that has the reference).

Sources, all read as text from the reference checkout (fblissjr/nndex); nothing of the reference
is executed (it is Rust and cannot be built here):
  * notebooks/python_bindings_demo.ipynb cells 2 and 5 — the published top-5 of the 50,000 × 128
    N(0,1) matrix seeded 42 (also README.md:58-69): parsed from the saved cell output.
  * notebooks/accuracy_vs_numpy.ipynb cells 2 and 4 — seed 7, 50,000 × 128, k=20: top-k overlap
    1.000 and score MAE 0.000000 against NumPy: parsed from the saved cell output.
  * the reference's Rust unit tests — their inputs and expected answers, transcribed into
    reference_unit_cases.json with the file:line each case comes from.
The NumPy re-derivation of the seed-42 data (same generator calls as the notebook) is stored beside
the parsed numbers so the CPU tests can regenerate the matrix without the reference.

Usage:  python tests/golden/make_golden.py [path-to-reference-checkout]
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _cell_output(nb_path: str, cell: int) -> str:
    nb = json.load(open(nb_path))
    out = []
    for o in nb["cells"][cell].get("outputs", []):
        out.append("".join(o.get("text", "")) or "".join(o.get("data", {}).get("text/plain", "")))
    return "\n".join(out)


def _cell_source(nb_path: str, cell: int) -> str:
    return "".join(json.load(open(nb_path))["cells"][cell]["source"])


def demo_golden(ref: str) -> dict:
    nb = os.path.join(ref, "notebooks", "python_bindings_demo.ipynb")
    src = _cell_source(nb, 2)
    assert "default_rng(42)" in src and "rows, dims = 50_000, 128" in src, src
    text = _cell_output(nb, 5)
    idx = json.loads(re.search(r"top-5 indices: (\[[^\]]*\])", text).group(1))
    sim = json.loads(re.search(r"top-5 scores: (\[[^\]]*\])", text).group(1))
    return {
        "source": "notebooks/python_bindings_demo.ipynb cells 2,5; README.md:58-69",
        "generator": "np.random.default_rng(42); matrix = rng.normal(size=(50000,128)).astype(f32); "
                     "query = rng.normal(size=(128,)).astype(f32)",
        "rows": 50000, "dims": 128, "seed": 42, "k": 5, "normalized": False,
        "indices": idx, "similarities": sim,
    }


def accuracy_golden(ref: str) -> dict:
    nb = os.path.join(ref, "notebooks", "accuracy_vs_numpy.ipynb")
    src = _cell_source(nb, 2)
    assert "default_rng(7)" in src and "rows, dims, k = 50_000, 128, 20" in src, src
    text = _cell_output(nb, 4)
    overlap = float(re.search(r"Top-k overlap: ([0-9.]+)", text).group(1))
    mae = float(re.search(r"Score MAE: ([0-9.]+)", text).group(1))
    return {
        "source": "notebooks/accuracy_vs_numpy.ipynb cells 2,4",
        "generator": "np.random.default_rng(7); matrix = rng.normal(size=(50000,128)).astype(f32); "
                     "query = rng.normal(size=(128,)).astype(f32)",
        "rows": 50000, "dims": 128, "seed": 7, "k": 20, "normalized": False,
        "topk_overlap": overlap, "score_mae": mae,
    }


def unit_cases() -> dict:
    """Inputs and expected answers of the reference's Rust unit tests (transcribed)."""
    return {
        "topk": [
            {"src": "src/topk.rs:218-232", "k": 3, "push": [[0, 0.1], [1, 0.9], [2, 0.5], [3, 0.3], [4, 0.7]], "expect_idx": [1, 4, 2]},
            {"src": "src/topk.rs:234-248", "k": 2, "push": [[0, 0.8], [1, 0.9], [2, 0.1], [3, 0.0], [4, -1.0]], "expect_idx": [1, 0]},
            {"src": "src/topk.rs:268-281", "k": 3, "push": [[5, 0.5], [2, 0.5], [8, 0.5]], "expect_idx": [2, 5, 8]},
            {"src": "src/topk.rs:283-297", "k": 2, "push": [[0, 0.5], [1, 0.5], [2, 0.5]], "expect_idx_set": [0, 1]},
            {"src": "src/topk.rs:299-309", "k": 10, "push": [[0, 0.3], [1, 0.7]], "expect_idx": [1, 0]},
            {"src": "src/topk.rs:311-321", "k": 1, "push": [[0, 0.1], [1, 0.9], [2, 0.5]], "expect_idx": [1], "expect_sim": [0.9]},
            {"src": "src/topk.rs:339-350", "k": 2, "push": [[0, -0.9], [1, -0.1], [2, -0.5]], "expect_idx": [1, 2]},
        ],
        "topk_merge": [
            {"src": "src/topk.rs:250-266", "k": 3, "left": [[0, 0.9], [1, 0.1], [2, 0.5]], "right": [[3, 0.8], [4, 0.2], [5, 0.7]], "expect_idx": [0, 3, 5]},
            {"src": "src/topk.rs:323-337", "k": 1, "left": [[0, 0.3]], "right": [[9, 0.7]], "expect_idx": [9], "expect_sim": [0.7]},
        ],
        "topk_from_scores": [
            {"src": "src/topk.rs:367-375", "scores": [0.1, 0.9, 0.5, 0.3, 0.7], "k": 3, "offset": 0, "expect_idx": [1, 4, 2]},
            {"src": "src/topk.rs:377-384", "scores": [0.1, 0.9, 0.5], "k": 2, "offset": 100, "expect_idx": [101, 102]},
            {"src": "src/topk.rs:386-393", "scores": [0.3, 0.7], "k": 10, "offset": 0, "expect_idx": [1, 0]},
            {"src": "src/topk.rs:395-399", "scores": [], "k": 5, "offset": 0, "expect_idx": []},
            {"src": "src/topk.rs:401-408", "scores": [0.5, 0.5, 0.5], "k": 3, "offset": 0, "expect_idx": [0, 1, 2]},
        ],
        "topk_from_scores_generated": [
            {"src": "src/topk.rs:412-425", "n": 200000, "pattern": "i*0.001", "plant": [[150000, 999.0], [175000, 998.0]], "k": 3, "offset": 0, "expect_idx": [150000, 175000, 199999]},
            {"src": "src/topk.rs:427-435", "n": 131072, "pattern": "i", "plant": [], "k": 5, "offset": 0, "expect_idx_prefix": [131071, 131070]},
            {"src": "src/topk.rs:437-445", "n": 131073, "pattern": "i", "plant": [], "k": 5, "offset": 0, "expect_idx_prefix": [131072, 131071]},
            {"src": "src/topk.rs:447-454", "n": 150000, "pattern": "i*0.01", "plant": [], "k": 2, "offset": 1000000, "expect_idx": [1149999, 1149998]},
        ],
        "known_answer": {
            "src": "src/lib.rs:824-851",
            "matrix": [[1, 0, 0, 0, 0, 0, 0, 0], [0, 1, 0, 0, 0, 0, 0, 0], [1, 1, 0, 0, 0, 0, 0, 0]],
            "query": [0.8, 0.6, 0, 0, 0, 0, 0, 0], "k": 2, "normalized": False,
            "expect_idx": [2, 0], "expect_sim": [0.98994946, 0.8], "tol": [1e-5, 1e-6],
        },
        "isqrt": {"src": "src/approx.rs:559-565", "cases": [[0, 0], [1, 1], [4, 2], [10000, 100], [65536, 256]]},
        "choose_nlist": {"src": "src/approx.rs:567-586", "cases": [[100, 1], [200, 1], [10000, 100], [1000000, 512]], "at_least_16": [300]},
        "normalize": [
            {"src": "src/lib.rs:1335-1341", "vector": [3.0, 4.0], "padded": 8, "unit_tol": 1e-6},
            {"src": "src/lib.rs:1344-1351", "rows": [[3.0, 4.0, 0.0, 0.0], [6.0, 8.0, 0.0, 0.0]], "padded": 8, "unit_tol": 1e-5},
        ],
        "pad_rows": {"src": "src/lib.rs:1308-1316", "values": [1, 2, 3, 4, 5, 6], "rows": 2, "dims": 3, "padded": 8,
                     "expect": [1, 2, 3, 0, 0, 0, 0, 0, 4, 5, 6, 0, 0, 0, 0, 0]},
        "errors": [
            {"src": "src/lib.rs:1105-1112", "what": "search k=0", "matrix": "ones(1,8)", "query": "ones(8)", "k": 0, "expect": "InvalidTopK"},
            {"src": "src/lib.rs:1115-1128", "what": "query dims 4 vs 8", "matrix": "ones(2,8)", "query": "ones(4)", "k": 1, "expect": "QueryDimensionalityMismatch", "expected": 8, "found": 4},
            {"src": "src/lib.rs:1131-1135", "what": "10 values as 3x4", "expect": "ShapeMismatch"},
            {"src": "src/lib.rs:1137-1141", "what": "zero rows", "expect": "ShapeMismatch"},
            {"src": "src/lib.rs:1143-1148", "what": "NaN in matrix", "expect": "NonFiniteInput"},
            {"src": "src/lib.rs:1150-1155", "what": "inf in matrix", "expect": "NonFiniteInput"},
            {"src": "src/lib.rs:1157-1162", "what": "zero row", "expect": "ZeroNorm"},
            {"src": "src/lib.rs:1164-1172", "what": "NaN in query", "expect": "NonFiniteInput"},
            {"src": "src/lib.rs:1174-1182", "what": "zero query", "expect": "ZeroNorm"},
            {"src": "src/lib.rs:1184-1192", "what": "batch 16 values as 3 rows", "expect": "ShapeMismatch"},
            {"src": "src/lib.rs:1194-1202", "what": "batch k=0", "expect": "InvalidTopK"},
        ],
        "approx_floors": [
            {"src": "src/lib.rs:962-1021", "rows": 4096, "dims": 64, "k": 20, "min_overlap": 14, "top1_in_exact": True},
            {"src": "src/lib.rs:1205-1297", "rows": 2048, "dims": 64, "k": 10, "queries": 8, "min_overlap": 5, "batch_eq_single_tol": 1e-4},
            {"src": "tests_python/test_accuracy_vs_numpy.py:29-41", "rows": 4096, "dims": 128, "k": 25, "seed": 456, "min_overlap": 15},
        ],
        "exact_vs_numpy": {"src": "tests_python/test_accuracy_vs_numpy.py:15-26", "rows": 4096, "dims": 128, "k": 25, "seed": 123, "atol": 1e-5},
        "naive_parity": {"src": "src/lib.rs:902-959", "rows": 512, "dims": 32, "k": 16, "tol": 1e-5},
    }


def main() -> None:
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the nndex reference checkout>")
    ref = sys.argv[1]
    g = demo_golden(ref)
    rng = np.random.default_rng(42)
    m = rng.normal(size=(50000, 128)).astype(np.float32)
    q = rng.normal(size=(128,)).astype(np.float32)
    # Independent NumPy float64 check that the regenerated data reproduces the parsed answer.
    mn = m.astype(np.float64) / np.linalg.norm(m.astype(np.float64), axis=1, keepdims=True)
    qn = q.astype(np.float64) / np.linalg.norm(q.astype(np.float64))
    s = mn @ qn
    top = np.argsort(-s, kind="stable")[:11]
    assert top[:5].tolist() == g["indices"], (top[:5], g["indices"])
    g["numpy_f64_top10"] = top[:10].tolist()
    g["numpy_f64_top11_scores"] = [float(x) for x in s[top]]
    json.dump(g, open(os.path.join(HERE, "demo_seed42.json"), "w"), indent=1)
    json.dump(accuracy_golden(ref), open(os.path.join(HERE, "accuracy_seed7.json"), "w"), indent=1)
    json.dump(unit_cases(), open(os.path.join(HERE, "reference_unit_cases.json"), "w"), indent=1)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
