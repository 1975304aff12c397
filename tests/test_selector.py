"""The generated selector (selector_tree.inc, fitted on kernel timings
measured on B200) against the exhaustive timing data it was fitted on: the
compiled spmx_select_features reproduces the tree, and picking by it costs
little time over the best of the eight kernels.  Host only."""
import ctypes
import json
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(ROOT, "spmspv-adaptive_b200", "spmx", "data", "selector_b200.jsonl")


def _records():
    return [json.loads(ln) for ln in open(DATA) if ln.strip()]


def test_selector_regret_on_measured_timings():
    from spmx import abi
    recs = _records()
    regret = []
    for r in recs:
        f = (ctypes.c_double * 23)(*r["inputs"])
        k = ctypes.c_int()
        assert abi.lib.spmx_select_features(f, ctypes.byref(k)) == 0
        assert 0 <= k.value < 8
        regret.append(r["us"][k.value] / min(r["us"]))
    regret = np.array(regret)
    assert regret.mean() < 1.05
    assert np.quantile(regret, 0.9) < 1.25


def test_selector_beats_any_single_kernel():
    from spmx import abi
    recs = _records()
    T = np.array([r["us"] for r in recs])
    picks = []
    for r in recs:
        f = (ctypes.c_double * 23)(*r["inputs"])
        k = ctypes.c_int()
        abi.lib.spmx_select_features(f, ctypes.byref(k))
        picks.append(k.value)
    chosen = T[np.arange(len(recs)), picks].sum()
    assert chosen < T.sum(axis=0).min()  # better than always running one kernel


def test_picks_on_the_benchmark_matrix():
    """On the 1M-row Zipf matrix the selector picks a CSC kernel for a sparse x
    and a row (SpMV) kernel for the dense x."""
    from spmx import abi
    recs = [r for r in _records() if r["matrix"] == "zipf-1M"]
    for r in recs:
        f = (ctypes.c_double * 23)(*r["inputs"])
        k = ctypes.c_int()
        abi.lib.spmx_select_features(f, ctypes.byref(k))
        if r["density"] <= 0.01:
            assert k.value in (0, 1, 2, 3), r["density"]
        if r["density"] >= 1.0:
            assert k.value in (6, 7), r["density"]


def test_learner_comparison():
    """The other learners (random forest, gradient boosting, SVM, k nearest)
    are fitted and scored on the same held-out split; every learner beats
    always running the single best kernel, and the exported tree is within a
    few percent of the best of them."""
    pytest.importorskip("sklearn")
    from spmx import selector_train
    out = selector_train.compare(DATA, report=False)
    base = out.pop("always the overall best kernel")["test_regret"]
    for name, r in out.items():
        assert r["test_regret"] < base, name
    best = min(r["test_regret"] for r in out.values())
    assert out["decision tree"]["test_regret"] <= best * 1.05
