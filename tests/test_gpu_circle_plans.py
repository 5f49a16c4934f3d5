"""GPU parity of the Circle plan handles: CircleDomainMaterializationPlan (points,
FFT twiddles, QM31 inverse-domain layers), CircleFRIFoldPlan, CircleFRIFoldChainPlan
and CircleFRIMerkleTranscriptFoldChainPlan (host, resident, materialised-layer and
precomputed-first-commitment forms), against the CPU oracle
(CircleDomainMaterializationPlan.swift:52-219, CircleFRIFoldPlan.swift:5-518)."""
import numpy as np
import pytest

import apple_b200 as azk
from tests import generators as G

pytestmark = pytest.mark.gpu


def _qm31(rng, n):
    return rng.integers(0, G.P, size=(n, 4), dtype=np.uint32)


def _dev(ctx, arr):
    b = ctx.alloc(max(16, np.asarray(arr).nbytes))
    b.upload(np.ascontiguousarray(arr))
    return b


def _q_from(buf, count, offset=0):
    return np.frombuffer(buf.download(16 * count, offset), np.uint32).reshape(-1, 4)


@pytest.mark.parametrize("log_size,rounds", [(1, 1), (5, 3), (12, 12), (16, 10)])
def test_domain_plan_tables(ctx, oracle, log_size, rounds):
    plan = azk.CircleDomainMaterializationPlan(ctx, log_size, True, True, rounds)
    assert np.array_equal(plan.read_domain_points(), oracle.domain_points(log_size))
    assert np.array_equal(plan.read_codeword_twiddles(), oracle.fft_twiddles(log_size))
    layers = plan.read_inverse_domain_layers()
    want = oracle.inverse_layers(log_size, rounds)
    assert len(layers) == rounds
    for got, w in zip(layers, want):
        assert np.array_equal(got[:, 0], w) and not got[:, 1:].any()
    pts, tw, inv = plan.buffers()
    assert pts and tw and inv
    assert plan.output_count == (1 << log_size) >> rounds
    assert plan.materialization_stats.gpu_s >= 0


def test_domain_plan_partial_and_rejections(ctx):
    plan = azk.CircleDomainMaterializationPlan(ctx, 8, False, False, 2)
    pts, tw, inv = plan.buffers()
    assert pts is None and tw is None and inv
    for read in (plan.read_domain_points, plan.read_codeword_twiddles):
        with pytest.raises(azk.AZKError) as e:
            read()
        assert e.value.name == "invalidInputLayout"
    for args in [(8, False, False, 0), (8, False, False, 9), (0, True, False, 0)]:
        with pytest.raises(azk.AZKError) as e:
            azk.CircleDomainMaterializationPlan(ctx, *args)
        assert e.value.name == "invalidInputLayout"


@pytest.mark.parametrize("log_size", [1, 6, 14, 20])
def test_circle_fold_plan(ctx, oracle, log_size):
    rng = np.random.default_rng(log_size)
    n = 1 << log_size
    ev, ch = _qm31(rng, n), _qm31(rng, 1)
    want = oracle.circle_fold_chain(log_size, ev, ch)
    plan = azk.CircleFRIFoldPlan(ctx, log_size)
    assert np.array_equal(plan.execute(ev, ch), want)
    d_ev, d_out = _dev(ctx, ev), ctx.alloc(8 * n + 32)
    plan.execute_resident(d_ev.ptr, d_out.ptr, ch, out_offset=32)
    assert np.array_equal(_q_from(d_out, n // 2, 32), want)
    inv = plan.read_inverse_y_twiddles()
    assert np.array_equal(inv[:, 0], oracle.inverse_layers(log_size, 1)[0]) and not inv[:, 1:].any()
    plan.clear_reusable_buffers()


@pytest.mark.parametrize("log_size,rounds", [(3, 3), (10, 4), (16, 10), (20, 14)])
def test_circle_fold_chain_plan(ctx, oracle, log_size, rounds):
    rng = np.random.default_rng(100 + log_size)
    n = 1 << log_size
    ev, ch = _qm31(rng, n), _qm31(rng, rounds)
    want = oracle.circle_fold_chain(log_size, ev, ch)
    plan = azk.CircleFRIFoldChainPlan(ctx, log_size, rounds)
    assert np.array_equal(plan.execute(ev, ch), want)
    d_ev, d_out = _dev(ctx, ev), ctx.alloc(16 * (n >> rounds) + 48)
    plan.execute_resident(d_ev.ptr, d_out.ptr, ch, final_offset=48)
    assert np.array_equal(_q_from(d_out, n >> rounds, 48), want)
    layers = plan.read_inverse_domain_layers()
    for got, w in zip(layers, oracle.inverse_layers(log_size, rounds)):
        assert np.array_equal(got[:, 0], w)
    # the final layer may not overlap the evaluations
    with pytest.raises(azk.AZKError) as e:
        plan.execute_resident(d_ev.ptr, d_ev.ptr, ch)
    assert e.value.name == "invalidInputLayout"


@pytest.mark.parametrize("log_size,rounds,queries", [(6, 3, 4), (14, 8, 16), (18, 12, 64)])
def test_circle_merkle_chain_plan(ctx, oracle, log_size, rounds, queries):
    rng = np.random.default_rng(200 + log_size)
    n = 1 << log_size
    ev = _qm31(rng, n)
    pub = bytes(rng.integers(0, 256, 32, dtype=np.uint8))
    ref = oracle.prove(log_size, ev, 1, queries, pub, rounds)
    plan = azk.CircleFRIMerkleTranscriptFoldChainPlan(ctx, log_size, 1, queries, pub, rounds)
    fin, cm, ch = plan.execute(ev)
    assert np.array_equal(fin, ref.final_layer)
    assert cm == ref.commitments
    assert np.array_equal(ch, ref.challenges)
    # same results as the single-call entry point
    fin2, cm2, ch2 = azk.circle_merkle_fold_chain(ctx, log_size, ev, 1, queries, pub, rounds)
    assert np.array_equal(fin, fin2) and cm == cm2 and np.array_equal(ch, ch2)
    # resident, strided commitments
    stride = 48
    d_ev, d_cm, d_fin = _dev(ctx, ev), ctx.alloc(stride * rounds), ctx.alloc(16 * plan.output_count)
    plan.execute_resident(d_ev.ptr, d_cm.ptr, d_fin.ptr, commitment_stride=stride)
    raw = d_cm.download()
    assert [raw[stride * k:stride * k + 32] for k in range(rounds)] == cm
    assert np.array_equal(_q_from(d_fin, plan.output_count), fin)
    assert np.array_equal(plan.challenges(), ch)
    # materialised committed layers: round k's input layer at the layer-log offset
    d_log = ctx.alloc(16 * plan.total_committed_layer_count)
    plan.execute_resident(d_ev.ptr, d_cm.ptr, d_fin.ptr, dev_committed_layers=d_log.ptr, commitment_stride=stride)
    log = _q_from(d_log, plan.total_committed_layer_count)
    assert np.array_equal(log[:n], ev)
    off = 0
    for k, c in enumerate(plan.committed_layer_counts):
        # each committed layer's 16-byte-leaf Merkle root is that round's commitment
        assert oracle.merkle_root(log[off:off + c].tobytes(), c, 16, 16) == cm[k]
        off += c
    assert np.array_equal(log[n:n + n // 2], oracle.circle_fold_chain(log_size, ev, ch[:1]))
    # with round 0's commitment given: the same chain
    d_first = _dev(ctx, np.frombuffer(cm[0], np.uint8))
    d_fin3 = ctx.alloc(16 * plan.output_count)
    plan.execute_resident(d_ev.ptr, d_cm.ptr, d_fin3.ptr, dev_committed_layers=d_log.ptr, dev_first_commitment=d_first.ptr, commitment_stride=stride)
    assert np.array_equal(_q_from(d_fin3, plan.output_count), fin)
    assert np.array_equal(plan.challenges(), ch)


@pytest.mark.parametrize("log_count", [0, 1, 5, 12, 17])
def test_prehashed_merkle_plan(ctx, oracle, log_count):
    """SHA3PrehashedLeavesMerkleCommitPlan: host and resident commits equal the
    oracle's prehashed root; a misaligned or out-of-range resident buffer and a
    count that is not a power of two are rejected."""
    rng = np.random.default_rng(300 + log_count)
    n = 1 << log_count
    dig = rng.integers(0, 256, 32 * n, dtype=np.uint8).tobytes()
    want = oracle.merkle_root_prehashed(dig)
    plan = azk.SHA3PrehashedLeavesMerkleCommitPlan(ctx, n)
    assert plan.commit(dig) == want
    buf = ctx.alloc(32 * n + 64)
    buf.upload(np.frombuffer(dig, np.uint8), 64)
    assert plan.commit_resident(buf.ptr, 64) == want
    assert plan.commit_resident(buf.ptr, 64) == want  # counters reset themselves
    for off in (8, 96):
        with pytest.raises(azk.AZKError) as e:
            plan.commit_resident(buf.ptr, off)
        assert e.value.name == "invalidInputLayout"
    with pytest.raises(azk.AZKError) as e:
        azk.SHA3PrehashedLeavesMerkleCommitPlan(ctx, 3)
    assert e.value.name == "invalidLeafCount"
