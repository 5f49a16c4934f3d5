"""The autotuner's learned cost model: the MLP's hand-written CUDA forward and
backward kernels against a PyTorch fp32 reference of the same network, training,
and what the trained model gains over the schedule chosen without it."""
import numpy as np
import pytest
import torch

import apple_b200 as azk
from apple_b200 import autotune as T

pytestmark = pytest.mark.gpu

# fp32 tolerance of the gradient check: the GPU sums in a fixed order that differs
# from PyTorch's, so agreement is to rounding (relative 2e-4 of the largest entry).
RTOL = 2e-4


def torch_mlp(dims, params):
    """Unpack the library's parameter layout (per layer: W[out][in], b[out])."""
    ws, off = [], 0
    for i in range(len(dims) - 1):
        n_in, n_out = dims[i], dims[i + 1]
        w = torch.tensor(params[off:off + n_in * n_out].reshape(n_out, n_in), dtype=torch.float32, requires_grad=True)
        off += n_in * n_out
        b = torch.tensor(params[off:off + n_out], dtype=torch.float32, requires_grad=True)
        off += n_out
        ws.append((w, b))
    return ws


def torch_forward(ws, x):
    h = x
    for i, (w, b) in enumerate(ws):
        h = h @ w.T + b
        if i + 1 < len(ws):
            h = torch.relu(h)
    return h[:, 0]


def test_mlp_forward_and_gradients_match_torch(ctx):
    rng = np.random.default_rng(3)
    model = T.CostModel(ctx, hidden=(32, 16), seed=7)
    x = rng.normal(size=(300, T.N_FEATURES)).astype(np.float32)
    y = rng.normal(size=300).astype(np.float32)
    params = model.params()
    ws = torch_mlp(model.dims, params)
    xt = torch.tensor(x)
    pred = torch_forward(ws, xt)
    np.testing.assert_allclose(model.forward(x), pred.detach().numpy(), rtol=1e-5, atol=1e-5)
    loss_t = ((pred - torch.tensor(y)) ** 2).mean()
    loss_t.backward()
    want = np.concatenate([np.concatenate([w.grad.numpy().ravel(), b.grad.numpy().ravel()]) for w, b in ws])
    loss, got = model.gradients(x, y)
    assert abs(loss - loss_t.item()) <= RTOL * abs(loss_t.item())
    assert np.max(np.abs(got - want)) <= RTOL * np.max(np.abs(want))


def test_mlp_training_fits_a_smooth_function(ctx):
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, size=(1024, T.N_FEATURES)).astype(np.float32)
    y = (np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2]).astype(np.float32)
    model = T.CostModel(ctx, hidden=(64, 64), seed=2)
    start, _ = model.gradients(x, y)
    final = model.train(x, y, steps=1500, lr=3e-3)
    assert final < 0.05 * start


def test_tuner_gain_over_heuristic_on_unseen_shapes(ctx, tmp_path):
    logs = range(8, 19)
    shapes = [(lg, 16, 1, c) for lg in logs for c in (1, 16)]
    recs = T.collect(ctx, shapes, threads=(256,), reps=3)
    held = {11, 15}
    tuner = T.Tuner(ctx, recs)
    tuner.train(steps=2000, records=[r for r in recs if r["log"] not in held])
    unseen = [s for s in shapes if s[0] in held]
    r = tuner.regret(unseen, verify=3)
    # the model, checked by timing its top 3 candidates, stays within 5 % of the
    # exhaustive optimum on shapes it never saw, and loses less than the heuristic
    assert r["model"]["mean"] <= 0.05
    assert r["model"]["mean"] <= r["heuristic"]["mean"] + 1e-9
    # persistence round trip
    path = tmp_path / "store.json"
    tuner.save(path)
    again = T.Tuner.load(ctx, path)
    for sh in unseen:
        assert again.choose(sh) == tuner.choose(sh)


def test_layer_table_schedules_give_identical_proofs(ctx, oracle):
    from tests import generators as G

    rng = np.random.default_rng(12)
    ev = rng.integers(0, G.P, size=(1 << 14, 4), dtype=np.uint32)
    pub = bytes(range(32))
    table = {lg: max(1, lg - 4) for lg in range(1, 15)}
    p = azk.CirclePCSFRIProver(ctx, 14, 2, 16, 8, schedule=dict(layer_treelet=table))
    assert p.prove_evaluations(ev, pub) == oracle.prove(14, ev, 2, 16, pub, 8).proof


@pytest.mark.parametrize("shape", [(10, 16, 1, 1), (12, 16, 0, 8), (11, 64, 0, 2)])
def test_race_gates_on_host_roots_and_validates_winner(ctx, shape):
    """Every candidate schedule reproduces the host's roots (none fails the gate),
    the winner has the lowest device-plus-submit median, and it survives randomized
    validation on fresh inputs."""
    cands = [(t, th) for t in (2, min(6, shape[0]), min(9, shape[0])) for th in (128, 256, 512)]
    ms, win = T.race(ctx, shape, cands, warmup=1, runs=5, seed=3)
    assert all(m["passed_gate"] and m["runs"] == 5 for m in ms)
    score = [m["median_gpu_s"] + m["median_submit_s"] for m in ms]
    assert win == int(np.argmin(score))
    assert all(m["p95_gpu_s"] >= m["median_gpu_s"] > 0 for m in ms)
    T.validate(ctx, shape, cands[win], batches=3, seed=11)


def test_plan_races_model_candidates_and_persists(ctx, tmp_path):
    shapes = [(lg, 16, 1, 1) for lg in (8, 9, 10, 11, 12)]
    recs = T.collect(ctx, shapes, threads=(128, 256), reps=2)
    tuner = T.Tuner(ctx, recs)
    tuner.train(steps=800)
    store = T.PlanStore(str(tmp_path / "plans.json"))
    got = tuner.plan((10, 16, 1, 1), store=store, top=3)
    assert store.winner((10, 16, 1, 1)) == tuple(got)
    rec = store.records[store.key((10, 16, 1, 1))]
    assert rec["candidates"] == 3 and rec["failed_gate"] == 0
    store.save()
    again = T.PlanStore(str(tmp_path / "plans.json"))
    assert tuner.plan((10, 16, 1, 1), store=again) == tuple(got)  # reused, no race
    # sustained slower live timings make the record stale; the next plan races again
    for _ in range(again.min_samples):
        again.record_live((10, 16, 1, 1), 3 * rec["median_gpu_s"], rec["median_submit_s"])
    assert (10, 16, 1, 1) in again.stale_shapes()
    tuner.plan((10, 16, 1, 1), store=again, top=2)
    assert again.records[again.key((10, 16, 1, 1))]["candidates"] == 2 and not again.stale_shapes()
