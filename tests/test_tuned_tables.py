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


def test_plan_store_drift_policy(tmp_path):
    """Live timings near the raced median keep a plan; a sustained shift beyond the
    threshold marks it stale only after the minimum number of samples; a new race
    clears the observation (PlanDatabase.recordLiveObservation semantics)."""
    store = T.PlanStore(str(tmp_path / "p.json"), alpha=0.2, min_samples=8, threshold=0.25)
    shape = (14, 16, 1, 1)
    meas = [{"tile": 9, "threads": 256, "passed_gate": True, "median_gpu_s": 1e-3, "p95_gpu_s": 1.2e-3, "median_submit_s": 1e-5, "runs": 5}]
    store.record_race(shape, meas, 0)
    for k in range(20):
        st = store.record_live(shape, 1e-3 * (1.05 if k % 2 else 0.95), 1e-5)
    assert not st["stale"] and not store.stale_shapes()
    for k in range(7):
        st = store.record_live(shape, 2e-3, 1e-5)
    assert st["stale"]
    fresh = T.PlanStore(str(tmp_path / "q.json"), min_samples=8)
    fresh.record_race(shape, meas, 0)
    for k in range(7):
        assert not fresh.record_live(shape, 5e-3, 1e-5)["stale"]  # fewer samples than the minimum
    assert fresh.record_live(shape, 5e-3, 1e-5)["stale"]
    store.save()
    again = T.PlanStore(str(tmp_path / "p.json"))
    assert again.stale_shapes() == [shape] and again.winner(shape) == (9, 256)
    again.record_race(shape, meas, 0)
    assert not again.stale_shapes()
