"""The tuned default schedules compiled into the library (csrc/azk_tuned.h) are the
tables the autotuner exported with their evidence (apple_b200/tuned_b200.json)."""
import json
import os

import pytest

from apple_b200 import autotune as T

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "apple_b200")


def test_header_matches_exported_tables():
    path = os.path.join(PKG, "tuned_b200.json")
    if not os.path.exists(path):
        pytest.skip("no exported tables")
    doc = json.load(open(path))
    with open(os.path.join(PKG, "csrc", "azk_tuned.h")) as f:
        assert f.read() == T.header_text(doc)


def test_exported_tables_are_valid_depths():
    path = os.path.join(PKG, "tuned_b200.json")
    if not os.path.exists(path):
        pytest.skip("no exported tables")
    doc = json.load(open(path))
    assert set(doc["tables"]) == set(T.TABLE_SHAPES)
    for tab in doc["tables"].values():
        for lg, t in tab.items():
            assert 1 <= t <= min(13, max(1, int(lg)))
    rep = doc["report"]
    assert rep["records"] >= 2000
    # the learned choice beats the fixed-depth heuristic on the held-out sizes
    assert rep["regret_unseen"]["model"]["mean"] < rep["regret_unseen"]["heuristic"]["mean"]
