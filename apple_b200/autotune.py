"""Autotuner with a learned cost model for the commit kernel's schedule.

The reference's planner races a handful of Merkle schedules (scalar parents vs
treelet depth 3/4) behind a CPU gate and persists winners in SQLite
(Planner/MetalProofPlanner.swift:20-615, PlanDatabase.swift:43-533).  Here:

* `collect()` times the commit kernel (`azk_tuner_time_tree`) over a grid of
  shapes (layer size, leaf bytes, fold-then-hash or not, concurrent trees) and
  schedules (treelet depth, threads per CTA): the exhaustive timed search.
* `CostModel` is an MLP (features -> log seconds per permutation) trained on the
  GPU by the library's own forward/backward/Adam kernels (`azk_mlp_*`).
* `Tuner.choose()` predicts the best schedule for a shape; with a `verify` budget
  it times the model's top candidates and keeps the fastest (the fallback), and
  `regret()` judges its choices against exhaustive search.
* `Tuner.layer_table()` turns choices into the `layer_treelet` table of an
  `azk_schedule`.

Schedules never change results: every schedule hashes the same tree.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import time

import numpy as np

from . import _capi
from ._capi import check, lib

THREADS = (128, 256, 512)
LEAF_BYTES = (16, 64)


def time_tree(ctx, log_leaves, leaf_bytes, fold, concurrent, tile_log, threads, reps=3, group_log=None) -> float:
    sec = ctypes.c_double()
    g = tile_log if group_log is None else group_log
    check(lib().azk_tuner_time_tree(ctx.handle, log_leaves, leaf_bytes, 1 if fold else 0, concurrent, tile_log, g, threads, reps, ctypes.byref(sec)),
          ctx.handle)
    return sec.value


def permutations(log_leaves, leaf_bytes, concurrent) -> int:
    n = 1 << log_leaves
    per_leaf = 1 if leaf_bytes == 16 else 1  # a 64-byte leaf is one permutation too
    return concurrent * (per_leaf * n + n - 1)


def tile_candidates(log_leaves):
    return list(range(2, min(13, log_leaves) + 1)) if log_leaves >= 2 else [1]


def shape_grid(logs=range(6, 23), concurrents=(1, 8, 64), max_leaves=1 << 24):
    shapes = []
    for lg in logs:
        for c in concurrents:
            if (1 << lg) * c > max_leaves:
                continue
            shapes.append((lg, 16, 0, c))
            shapes.append((lg, 16, 1, c))
            if lg <= 20:
                shapes.append((lg, 64, 0, c))
    return shapes


def collect(ctx, shapes=None, threads=THREADS, reps=3, progress=None) -> list:
    """Exhaustive timed search: one record per (shape, schedule)."""
    shapes = shapes if shapes is not None else shape_grid()
    out = []
    for i, (lg, lb, fold, c) in enumerate(shapes):
        for tl in tile_candidates(lg):
            for th in threads:
                t = time_tree(ctx, lg, lb, fold, c, tl, th, reps)
                out.append({"log": lg, "leaf_bytes": lb, "fold": fold, "concurrent": c, "tile": tl, "threads": th, "seconds": t})
        if progress:
            progress(i + 1, len(shapes))
    return out


# ---------------------------------------------------------------------------
# correctness-gated race and randomized validation (the reference's planner:
# Planner/MetalProofPlanner.swift:224-269 races candidates behind a CPU gate,
# :367-418 measures each one, :447-484 validates the winner on fresh inputs)
# ---------------------------------------------------------------------------
def race(ctx, shape, candidates, warmup=1, runs=5, seed=1):
    """Race schedules [(tile, threads), ...] for shape (log, leaf bytes, fold, trees).
    Each candidate commits a seeded random input whose roots the host computes;
    one that differs is dropped untimed.  Returns (measurements, index of the
    winner): per candidate {tile, threads, passed_gate, median_gpu_s, p95_gpu_s,
    median_submit_s, runs}."""
    lg, lb, fold, c = shape
    arr = (_capi.TunerCandidate * len(candidates))(*[_capi.TunerCandidate(t, t, th, 0) for t, th in candidates])
    out = (_capi.TunerMeasurement * len(candidates))()
    win = ctypes.c_uint32()
    check(lib().azk_tuner_race_tree(ctx.handle, lg, lb, 1 if fold else 0, c, arr, len(candidates), warmup, runs, seed, out, ctypes.byref(win)),
          ctx.handle)
    ms = [{"tile": t, "threads": th, "passed_gate": bool(m.passed_gate), "median_gpu_s": m.median_gpu_s, "p95_gpu_s": m.p95_gpu_s,
           "median_submit_s": m.median_submit_s, "runs": m.runs} for (t, th), m in zip(candidates, out)]
    return ms, int(win.value)


def validate(ctx, shape, schedule, batches=3, seed=7):
    """Commit `batches` fresh seeded inputs with `schedule` and compare each root
    with the host's; raises AZKError(correctnessValidationFailed) on a mismatch."""
    lg, lb, fold, c = shape
    t, th = schedule
    cand = _capi.TunerCandidate(t, t, th, 0)
    check(lib().azk_tuner_validate_tree(ctx.handle, lg, lb, 1 if fold else 0, c, ctypes.byref(cand), batches, seed), ctx.handle)


class PlanStore:
    """Persisted race winners and live drift, the reference's plan database
    (Planner/PlanDatabase.swift) as a JSON file: a record per shape (winner, median
    device and submit time, p95, confidence) and an observation per shape that
    keeps exponential moving averages of live timings; once enough samples drift
    more than the threshold from the record, the shape is stale and is raced again
    (recordLiveObservation, PlanDatabase.swift:192-236)."""

    def __init__(self, path=None, alpha=0.2, min_samples=8, threshold=0.25):
        self.path = path
        self.alpha, self.min_samples, self.threshold = alpha, min_samples, threshold
        self.records, self.observations = {}, {}
        if path and os.path.exists(path):
            with open(path) as f:
                doc = json.load(f)
            self.records = doc.get("records", {})
            self.observations = doc.get("observations", {})

    @staticmethod
    def key(shape) -> str:
        return "%d/%d/%d/%d" % tuple(int(v) for v in shape)

    def record_race(self, shape, measurements, winner):
        w = measurements[winner]
        n = w["runs"]
        self.records[self.key(shape)] = {"winner": [w["tile"], w["threads"]], "median_gpu_s": w["median_gpu_s"],
                                         "median_submit_s": w["median_submit_s"], "p95_gpu_s": w["p95_gpu_s"],
                                         "confidence": n / (n + 2.0), "candidates": len(measurements),
                                         "failed_gate": sum(1 for m in measurements if not m["passed_gate"])}
        self.observations.pop(self.key(shape), None)

    def winner(self, shape):
        r = self.records.get(self.key(shape))
        return tuple(r["winner"]) if r else None

    def record_live(self, shape, gpu_s, submit_s) -> dict:
        """Fold one live timing into the shape's moving averages; returns
        {"stale": bool, "samples", "relative_drift"}."""
        rec = self.records.get(self.key(shape))
        if rec is None:
            raise KeyError("no race record for this shape")
        o = self.observations.get(self.key(shape), {"samples": 0, "ema_gpu_s": None, "ema_submit_s": None})
        ema = lambda prev, x: x if prev is None else self.alpha * x + (1 - self.alpha) * prev  # noqa: E731
        o["samples"] += 1
        o["ema_gpu_s"] = ema(o["ema_gpu_s"], gpu_s)
        o["ema_submit_s"] = ema(o["ema_submit_s"], submit_s)
        base = max(1e-12, rec["median_gpu_s"] + rec["median_submit_s"])
        o["relative_drift"] = abs(o["ema_gpu_s"] + o["ema_submit_s"] - base) / base
        o["stale"] = o["samples"] >= self.min_samples and o["relative_drift"] > self.threshold
        self.observations[self.key(shape)] = o
        return {"stale": o["stale"], "samples": o["samples"], "relative_drift": o["relative_drift"]}

    def stale_shapes(self):
        return [tuple(int(v) for v in k.split("/")) for k, o in self.observations.items() if o.get("stale")]

    def save(self, path=None):
        with open(path or self.path, "w") as f:
            json.dump({"version": 1, "records": self.records, "observations": self.observations}, f, indent=1)


# ---------------------------------------------------------------------------
# features
# ---------------------------------------------------------------------------
SM_SLOTS = 148 * 2  # resident 256-thread CTAs of the commit kernel on a B200


def features(log_leaves, leaf_bytes, fold, concurrent, tile, threads) -> list:
    tl = min(tile, log_leaves)
    tiles = concurrent * (1 << (log_leaves - tl))
    waves = tiles / SM_SLOTS
    return [
        log_leaves / 22.0,
        leaf_bytes / 64.0,
        float(fold),
        math.log2(concurrent) / 6.0,
        tl / 13.0,
        math.log2(threads) / 9.0,
        math.log2(tiles) / 20.0,
        math.log2(max(waves, 1e-3)) / 10.0,
        (math.ceil(waves) - waves) if waves >= 1 else (1.0 - waves),  # idle fraction of the last wave
        (log_leaves - tl) / 20.0,
    ]


N_FEATURES = 10


def target(rec) -> float:
    """log seconds per permutation (the quantity the model learns)."""
    return math.log(rec["seconds"] / permutations(rec["log"], rec["leaf_bytes"], rec["concurrent"]))


# ---------------------------------------------------------------------------
# the GPU-trained MLP
# ---------------------------------------------------------------------------
class CostModel:
    def __init__(self, ctx, hidden=(64, 64), seed=1):
        self.ctx = ctx
        self.dims = [N_FEATURES, *hidden, 1]
        self._h = ctypes.c_void_p()
        d = np.array(self.dims, np.uint32)
        check(lib().azk_mlp_create(ctx.handle, len(self.dims) - 1, d.ctypes.data, seed, ctypes.byref(self._h)), ctx.handle)
        self.mu = 0.0
        self.sigma = 1.0

    def close(self):
        if self._h:
            lib().azk_mlp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def param_count(self) -> int:
        return int(lib().azk_mlp_param_count(self._h))

    def params(self) -> np.ndarray:
        p = np.empty(self.param_count, np.float32)
        check(lib().azk_mlp_get_params(self._h, p.ctypes.data, len(p)), self.ctx.handle)
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check(lib().azk_mlp_set_params(self._h, p.ctypes.data, len(p)), self.ctx.handle)

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty(len(x), np.float32)
        check(lib().azk_mlp_forward(self._h, x.ctypes.data, len(x), y.ctypes.data), self.ctx.handle)
        return y

    def gradients(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = ctypes.c_float()
        g = np.empty(self.param_count, np.float32)
        check(lib().azk_mlp_gradients(self._h, x.ctypes.data, y.ctypes.data, len(x), ctypes.byref(loss), g.ctypes.data), self.ctx.handle)
        return loss.value, g

    def train(self, x, y, steps=3000, lr=3e-3) -> float:
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = ctypes.c_float()
        check(lib().azk_mlp_train(self._h, x.ctypes.data, y.ctypes.data, len(x), steps, lr, ctypes.byref(loss)), self.ctx.handle)
        return loss.value

    # standardised target
    def fit(self, records, steps=3000, lr=3e-3) -> float:
        x = np.array([features(r["log"], r["leaf_bytes"], r["fold"], r["concurrent"], r["tile"], r["threads"]) for r in records], np.float32)
        t = np.array([target(r) for r in records], np.float64)
        self.mu, self.sigma = float(t.mean()), float(t.std() or 1.0)
        return self.train(x, ((t - self.mu) / self.sigma).astype(np.float32), steps, lr)

    def predict_seconds(self, shapes_and_schedules) -> np.ndarray:
        x = np.array([features(*s) for s in shapes_and_schedules], np.float32)
        z = self.forward(x).astype(np.float64) * self.sigma + self.mu
        perms = np.array([permutations(s[0], s[1], s[3]) for s in shapes_and_schedules], np.float64)
        return np.exp(z) * perms


# ---------------------------------------------------------------------------
# tuner
# ---------------------------------------------------------------------------
def heuristic_schedule(log_leaves):
    """The schedule without the model: deepest treelet that fits, 256 threads."""
    return (min(12, max(1, log_leaves)), 256)


class Tuner:
    def __init__(self, ctx, records=None, model: CostModel | None = None):
        self.ctx = ctx
        self.records = list(records or [])
        self.model = model
        self._table = {}
        for r in self.records:
            self._table[(r["log"], r["leaf_bytes"], r["fold"], r["concurrent"], r["tile"], r["threads"])] = r["seconds"]
        # candidate thread counts: those the timings cover
        self.threads = tuple(sorted({r["threads"] for r in self.records})) or THREADS

    # exhaustive search over what was measured
    def best_measured(self, shape):
        lg, lb, fold, c = shape
        cands = [(t, th) for t in tile_candidates(lg) for th in self.threads if (lg, lb, fold, c, t, th) in self._table]
        return min(cands, key=lambda s: self._table[(lg, lb, fold, c, s[0], s[1])])

    def measured(self, shape, sched):
        return self._table.get((*shape, *sched))

    def train(self, steps=3000, lr=3e-3, seed=1, hidden=(64, 64), records=None) -> float:
        self.model = CostModel(self.ctx, hidden=hidden, seed=seed)
        return self.model.fit(records if records is not None else self.records, steps=steps, lr=lr)

    def ranked(self, shape, threads=None):
        lg, lb, fold, c = shape
        cands = [(t, th) for t in tile_candidates(lg) for th in (self.threads if threads is None else (threads,))]
        pred = self.model.predict_seconds([(lg, lb, fold, c, t, th) for t, th in cands])
        order = np.argsort(pred)
        return [cands[i] for i in order], pred[order]

    def choose(self, shape, verify: int = 0, threads=None):
        """Model's pick; with verify=k, time its top k candidates and keep the fastest."""
        ranked, _ = self.ranked(shape, threads)
        if verify <= 0:
            return ranked[0]
        lg, lb, fold, c = shape
        timed = []
        for t, th in ranked[:verify]:
            sec = self.measured(shape, (t, th))
            if sec is None:
                sec = time_tree(self.ctx, lg, lb, fold, c, t, th)
                self._table[(*shape, t, th)] = sec
            timed.append((sec, (t, th)))
        return min(timed)[1]

    def plan(self, shape, store: "PlanStore | None" = None, top: int = 4, runs: int = 5, batches: int = 3, seed: int = 1):
        """A schedule for `shape` as the reference's planner makes one, with the model
        in front: the model's `top` candidates race behind the correctness gate, the
        winner is validated on `batches` fresh inputs, and the result is persisted in
        `store`.  A stored winner whose live timings have not drifted is reused."""
        if store is not None:
            w = store.winner(shape)
            if w is not None and tuple(shape) not in store.stale_shapes():
                return w
        cands = self.ranked(shape)[0][:top]
        ms, win = race(self.ctx, shape, cands, runs=runs, seed=seed)
        validate(self.ctx, shape, cands[win], batches=batches, seed=seed + 1)
        if store is not None:
            store.record_race(shape, ms, win)
        return cands[win]

    def regret(self, shapes, verify: int = 0) -> dict:
        """Mean and max of (time of choice / best measured time - 1) over shapes,
        for the model and for the heuristic schedule."""
        out = {"model": [], "heuristic": []}
        for sh in shapes:
            best = self.measured(sh, self.best_measured(sh))
            m = self.measured(sh, self.choose(sh, verify))
            h = self.measured(sh, heuristic_schedule(sh[0]))
            out["model"].append(m / best - 1.0)
            out["heuristic"].append(h / best - 1.0)
        return {k: {"mean": float(np.mean(v)), "max": float(np.max(v)), "n": len(v)} for k, v in out.items()}

    def layer_table(self, concurrent=1, leaf_bytes=16, fold=1, logs=range(1, 27), threads=256) -> dict:
        """{layer log size: treelet depth} for an azk_schedule's layer_treelet (the
        commit kernel's thread count is one per launch, so the table is chosen at a
        fixed `threads`; over the measured shapes that costs at most a few percent)."""
        table = {}
        for lg in logs:
            if lg < 2:
                table[lg] = 1
                continue
            t, _ = self.choose((lg, leaf_bytes, fold, concurrent), threads=threads)
            table[lg] = int(t)
        return table

    def layer_tables(self, concurrent=1, leaf_bytes=16, fold=1, logs=range(1, 27)):
        """({layer log: treelet depth}, {layer log: threads}): the model's pick over
        depth and threads per CTA for each layer size."""
        tiles, threads = {}, {}
        for lg in logs:
            if lg < 2:
                tiles[lg], threads[lg] = 1, 256
                continue
            t, th = self.choose((lg, leaf_bytes, fold, concurrent))
            tiles[lg], threads[lg] = int(t), int(th)
        return tiles, threads

    # persistence (the reference keeps a SQLite plan database; a JSON store here)
    def save(self, path):
        doc = {"version": 1, "device": _device_name(self.ctx), "library": os.path.getmtime(_capi.library_path()), "records": self.records}
        if self.model is not None:
            doc["model"] = {"dims": self.model.dims, "mu": self.model.mu, "sigma": self.model.sigma, "params": self.model.params().tolist()}
        with open(path, "w") as f:
            json.dump(doc, f)

    @classmethod
    def load(cls, ctx, path):
        with open(path) as f:
            doc = json.load(f)
        t = cls(ctx, doc.get("records", []))
        m = doc.get("model")
        if m:
            t.model = CostModel(ctx, hidden=tuple(m["dims"][1:-1]))
            t.model.set_params(np.array(m["params"], np.float32))
            t.model.mu, t.model.sigma = m["mu"], m["sigma"]
        return t


def _device_name(ctx) -> str:
    info = ctx.device_info()
    return f"sm{info['cc'][0]}{info['cc'][1]}-{info['sm_count']}sm"


# Default schedules shipped with the library: per-layer treelet depths chosen by
# the trained model for the commit kernel's common shapes.
TABLE_SHAPES = {
    "pcs_single": dict(concurrent=1, leaf_bytes=16, fold=1),   # one PCS instance: one tree per launch
    "pcs_batch": dict(concurrent=64, leaf_bytes=16, fold=1),   # batched supersteps: many trees per launch
    "merkle_raw64": dict(concurrent=1, leaf_bytes=64, fold=0),  # raw-leaf Merkle plan
}
# Shapes whose threads per CTA stay fixed: a batched commit launch holds layers of
# many sizes, the measured gain of another thread count at 64 concurrent trees is
# at most 1 % (log 6-18), and the largest layers (2^19-2^22 leaves x 64) are
# outside the measured grid, so the depth is chosen at the default 256 threads.
FIXED_THREADS = {"pcs_batch": 256}


def export(tuner: Tuner, report: dict, json_path: str, header_path: str):
    """Write the tables (and the evidence behind them) as JSON and as the C++ header
    the library compiles in (`csrc/azk_tuned.h`): per layer size the treelet depth
    and the threads per CTA the model picks."""
    both = {}
    for name, kw in TABLE_SHAPES.items():
        if name in FIXED_THREADS:
            th = FIXED_THREADS[name]
            tiles = tuner.layer_table(threads=th, **kw)
            both[name] = (tiles, {lg: th for lg in tiles})
        else:
            both[name] = tuner.layer_tables(**kw)
    doc = {"device": _device_name(tuner.ctx), "report": report, "shapes": TABLE_SHAPES, "fixed_threads": FIXED_THREADS,
           "tables": {k: {str(lg): t for lg, t in v[0].items()} for k, v in both.items()},
           "thread_tables": {k: {str(lg): t for lg, t in v[1].items()} for k, v in both.items()}}
    with open(json_path, "w") as f:
        json.dump(doc, f, indent=1)
    with open(header_path, "w") as f:
        f.write(header_text(doc))
    return doc


def header_text(doc) -> str:
    lines = ["// Generated by `python -m apple_b200.autotune --export` from measured commit-kernel",
             "// timings on " + doc["device"] + f" ({doc['report'].get('records', 0)} records) and the cost model trained on them;",
             "// tests/test_tuned_tables.py keeps it equal to apple_b200/tuned_b200.json.",
             "// Entry [k] = treelet depth (kTuned_*) and threads per CTA (kTunedThreads_*) for a layer",
             "// of 2^k leaves (0: not used; the schedule's own value).",
             "#pragma once",
             "#include <stdint.h>",
             "",
             "namespace azk {"]
    for name in TABLE_SHAPES:
        tab = doc["tables"][name]
        vals = [int(tab.get(str(k), 0)) for k in range(32)]
        lines.append(f"static constexpr uint8_t kTuned_{name}[32] = {{{', '.join(str(v) for v in vals)}}};")
    for name in TABLE_SHAPES:
        tab = doc.get("thread_tables", {}).get(name, {})
        vals = [int(tab.get(str(k), 0)) for k in range(32)]
        lines.append(f"static constexpr uint16_t kTunedThreads_{name}[32] = {{{', '.join(str(v) for v in vals)}}};")
    lines += ["}  // namespace azk", ""]
    return "\n".join(lines)


def main():
    import argparse

    import apple_b200 as azk

    ap = argparse.ArgumentParser(description="collect timings, train the cost model, report regret, export default tables")
    ap.add_argument("--out", default="tuner_store.json")
    ap.add_argument("--from-store", default=None, help="reuse the timings of an earlier store instead of collecting")
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--export", action="store_true", help="write the default tables (JSON and C++ header)")
    ap.add_argument("--export-dir", default=None, help="where to write tuned_b200.json and azk_tuned.h (default: in the package)")
    a = ap.parse_args()
    ctx = azk.Context(0)
    t0 = time.time()
    if a.from_store:
        with open(a.from_store) as f:
            recs = json.load(f)["records"]
    else:
        recs = collect(ctx)
    t1 = time.time()
    held = {9, 13, 17, 21}
    train = [r for r in recs if r["log"] not in held]
    tuner = Tuner(ctx, recs)
    loss = tuner.train(steps=a.steps, records=train)
    t2 = time.time()
    test_shapes = sorted({(r["log"], r["leaf_bytes"], r["fold"], r["concurrent"]) for r in recs if r["log"] in held})
    report = {"records": len(recs), "train_records": len(train), "held_out_logs": sorted(held), "collect_s": t1 - t0, "train_s": t2 - t1,
              "train_loss": loss, "regret_unseen": tuner.regret(test_shapes), "regret_unseen_verify3": tuner.regret(test_shapes, verify=3)}
    tuner.save(a.out)
    if a.export:
        # the shipped tables come from a model trained on every record
        final = Tuner(ctx, recs)
        final.train(steps=a.steps)
        here = os.path.dirname(os.path.abspath(__file__))
        jd, hd = (a.export_dir, a.export_dir) if a.export_dir else (here, os.path.join(here, "csrc"))
        export(final, report, os.path.join(jd, "tuned_b200.json"), os.path.join(hd, "azk_tuned.h"))
    print(json.dumps(report))


if __name__ == "__main__":
    main()
