"""GPU parity of the fold plan handles (QM31FRIFoldPlan, QM31FRIFoldChainPlan in
its explicit, transcript-derived and Merkle-bound modes, host and resident forms)
and of the resident query extractor (CircleFRIResidentQueryExtractorV1), against
the CPU oracle and the GPU prover's own proof bytes; resident range and aliasing
rejections follow QM31FRIFold.swift:1236-1294, 2707-2909."""
import numpy as np
import pytest

import apple_b200 as azk
from tests import generators as G

pytestmark = pytest.mark.gpu


def _qm31(rng, n, nonzero=False):
    v = rng.integers(0, G.P, size=(n, 4), dtype=np.uint32)
    if nonzero:
        v[:, 0] |= 1
    return v


def _inverse_layers(rng, n, rounds):
    return [_qm31(rng, (n >> r) // 2, nonzero=True) for r in range(rounds)]


def _dev(ctx, arr):
    b = ctx.alloc(max(16, np.asarray(arr).nbytes))
    b.upload(np.ascontiguousarray(arr))
    return b


def _oracle_chain(oracle, ev, inv_layers, challenges):
    cur = ev
    for layer, ch in zip(inv_layers, challenges):
        cur = oracle.fold(cur, layer, ch)
    return cur


@pytest.mark.parametrize("n", [2, 6, 1 << 12, 1 << 17])
def test_qm31_fold_plan_host_and_resident(ctx, oracle, n):
    rng = np.random.default_rng(n)
    ev, inv = _qm31(rng, n), _qm31(rng, n // 2, nonzero=True)
    ch = _qm31(rng, 1)[0]
    want = oracle.fold(ev, inv, ch)
    plan = azk.QM31FRIFoldPlan(ctx, n)
    assert np.array_equal(plan.execute(ev, inv, ch), want)
    dev, dinv, dout = _dev(ctx, ev), _dev(ctx, inv), ctx.alloc(8 * n + 64)
    plan.execute_resident(dev.ptr, dinv.ptr, dout.ptr, ch, out_offset=64)
    got = np.frombuffer(dout.download(8 * n, 64), np.uint32).reshape(-1, 4)
    assert np.array_equal(got, want)


def test_qm31_fold_plan_rejections(ctx):
    rng = np.random.default_rng(1)
    n = 64
    plan = azk.QM31FRIFoldPlan(ctx, n)
    ev, inv, ch = _qm31(rng, n), _qm31(rng, n // 2, nonzero=True), _qm31(rng, 1)[0]
    bad = inv.copy()
    bad[3] = 0
    for args in [(ev, bad, ch), (np.where(ev == ev, G.P, 0).astype(np.uint32), inv, ch)]:
        with pytest.raises(azk.AZKError) as e:
            plan.execute(*args)
        assert e.value.name == "invalidInputLayout"
    with pytest.raises(azk.AZKError):
        azk.QM31FRIFoldPlan(ctx, 7)
    big = ctx.alloc(32 * n)
    big.upload(np.concatenate([ev, inv]))
    # output overlapping the evaluations
    with pytest.raises(azk.AZKError) as e:
        plan.execute_resident(big.ptr, big.ptr, big.ptr, ch, inverse_offset=16 * n, out_offset=16 * n - 16)
    assert e.value.name == "invalidInputLayout"
    # a range running past the end of its allocation
    small = ctx.alloc(8 * n)
    with pytest.raises(azk.AZKError) as e:
        plan.execute_resident(big.ptr, big.ptr, small.ptr, ch, inverse_offset=16 * n, out_offset=16)
    assert e.value.name == "invalidInputLayout"


@pytest.mark.parametrize("n,rounds", [(8, 3), (12, 2), (1 << 10, 5), (1 << 16, 10)])
def test_chain_explicit_and_transcript_modes(ctx, oracle, n, rounds):
    rng = np.random.default_rng(n + rounds)
    ev, invs = _qm31(rng, n), _inverse_layers(rng, n, rounds)
    chs = _qm31(rng, rounds)
    plan = azk.QM31FRIFoldChainPlan(ctx, n, rounds)
    assert plan.output_count == n >> rounds and plan.total_inverse_domain_count == sum(len(l) for l in invs)
    want = _oracle_chain(oracle, ev, invs, chs)
    assert np.array_equal(plan.execute(ev, invs, chs), want)
    dev, dinv = _dev(ctx, ev), _dev(ctx, np.concatenate(invs))
    dout = ctx.alloc(16 * plan.output_count)
    plan.execute_resident(dev.ptr, dinv.ptr, dout.ptr, chs)
    assert np.array_equal(np.frombuffer(dout.download(), np.uint32).reshape(-1, 4), want)
    # challenges from given commitments (QM31FRIFoldTranscriptOracle)
    cms = [bytes(rng.integers(0, 256, 32, dtype=np.uint8)) for _ in range(rounds)]
    tch = oracle.qm31_transcript_challenges(n, cms)
    want_t = _oracle_chain(oracle, ev, invs, tch)
    out, ch = plan.execute_transcript_derived(ev, invs, cms)
    assert np.array_equal(ch, tch) and np.array_equal(out, want_t)
    # resident commitments at a 48-byte stride
    stride = 48
    cbuf = np.zeros(stride * rounds, np.uint8)
    for r, c in enumerate(cms):
        cbuf[stride * r:stride * r + 32] = np.frombuffer(c, np.uint8)
    dcm = _dev(ctx, cbuf)
    plan.execute_transcript_derived_resident(dev.ptr, dinv.ptr, dcm.ptr, dout.ptr, commitment_stride=stride)
    assert np.array_equal(np.frombuffer(dout.download(), np.uint32).reshape(-1, 4), want_t)
    assert np.array_equal(plan.challenges(), tch)


@pytest.mark.parametrize("logn,rounds", [(3, 2), (10, 4), (16, 10)])
def test_chain_merkle_modes(ctx, oracle, logn, rounds):
    n = 1 << logn
    rng = np.random.default_rng(logn * 31 + rounds)
    ev, invs = _qm31(rng, n), _inverse_layers(rng, n, rounds)
    fin, cms, chs = oracle.qm31_merkle_fold_chain(ev, invs)
    plan = azk.QM31FRIFoldChainPlan(ctx, n, rounds)
    out, cm, ch = plan.execute_merkle_transcript_derived(ev, invs)
    assert np.array_equal(out, fin) and cm == cms and np.array_equal(ch, chs)
    dev, dinv = _dev(ctx, ev), _dev(ctx, np.concatenate(invs))
    out, cm, ch = plan.execute_merkle_transcript_derived_readback(dev.ptr, dinv.ptr)
    assert np.array_equal(out, fin) and cm == cms and np.array_equal(ch, chs)
    # fully resident, with a layer log and strided commitments
    stride = 64
    dcm, dfin = ctx.alloc(stride * rounds), ctx.alloc(16 * plan.output_count)
    dlog = ctx.alloc(16 * plan.layer_log_count)
    plan.execute_merkle_transcript_derived_resident(dev.ptr, dinv.ptr, dcm.ptr, dfin.ptr, dev_layer_log=dlog.ptr, commitment_stride=stride)
    assert np.array_equal(np.frombuffer(dfin.download(), np.uint32).reshape(-1, 4), fin)
    raw = dcm.download()
    assert [raw[stride * r:stride * r + 32] for r in range(rounds)] == cms
    log = np.frombuffer(dlog.download(), np.uint32).reshape(-1, 4)
    layer, off = ev, 0
    for r in range(rounds):
        assert np.array_equal(log[off:off + len(layer)], layer), r
        off += len(layer)
        layer = oracle.fold(layer, invs[r], chs[r])
    # precomputed first commitment, the layer log's first layer being the evaluations
    log_with_input = ctx.alloc(16 * plan.layer_log_count)
    log_with_input.upload(ev)
    first = _dev(ctx, np.frombuffer(cms[0], np.uint8))
    dcm2 = ctx.alloc(32 * rounds)
    plan.execute_merkle_transcript_derived_resident(log_with_input.ptr, dinv.ptr, dcm2.ptr, dfin.ptr, dev_layer_log=log_with_input.ptr,
                                                   dev_first_commitment=first.ptr)
    assert np.array_equal(np.frombuffer(dfin.download(), np.uint32).reshape(-1, 4), fin)
    assert dcm2.download() == b"".join(cms)
    assert np.array_equal(plan.challenges(), chs)


def test_chain_rejections(ctx):
    rng = np.random.default_rng(2)
    with pytest.raises(azk.AZKError):
        azk.QM31FRIFoldChainPlan(ctx, 12, 3)  # 12 -> 6 -> 3: the third round's input is odd
    plan = azk.QM31FRIFoldChainPlan(ctx, 12, 2)
    ev, invs = _qm31(rng, 12), _inverse_layers(rng, 12, 2)
    with pytest.raises(azk.AZKError) as e:
        plan.execute_merkle_transcript_derived(ev, invs)  # not a power of two
    assert e.value.name == "invalidInputLayout"
    n, rounds = 64, 3
    plan = azk.QM31FRIFoldChainPlan(ctx, n, rounds)
    ev, invs = _qm31(rng, n), _inverse_layers(rng, n, rounds)
    dev, dinv = _dev(ctx, ev), _dev(ctx, np.concatenate(invs))
    dcm, dfin, dlog = ctx.alloc(32 * rounds), ctx.alloc(16 * plan.output_count), ctx.alloc(16 * plan.layer_log_count)
    cases = [
        dict(dev_commitments=dev.ptr),                      # commitments over the evaluations
        dict(dev_layer_log=dev.ptr),                        # layer log over the evaluations, no precomputed root
        dict(dev_layer_log=dlog.ptr, dev_final=dlog.ptr),   # final layer inside the layer log
        dict(commitment_stride=16),                         # stride below 32 bytes
        dict(dev_first_commitment=dcm.ptr),                 # precomputed root without a layer log
    ]
    for case in cases:
        kw = dict(dev_commitments=dcm.ptr, dev_final=dfin.ptr)
        kw.update(case)
        with pytest.raises(azk.AZKError) as e:
            plan.execute_merkle_transcript_derived_resident(dev.ptr, dinv.ptr, **kw)
        assert e.value.name == "invalidInputLayout", case


@pytest.mark.parametrize("logn,rounds,queries", [(6, 3, 5), (12, 6, 16), (16, 10, 32)])
def test_query_extractor_matches_proof_bytes(ctx, oracle, logn, rounds, queries):
    """Openings extracted from the committed layers equal the query section of the
    prover's proof for the same layers, commitments and query pairs."""
    rng = np.random.default_rng(logn)
    n = 1 << logn
    ev = _qm31(rng, n)
    pub = bytes(range(32))
    prover = azk.CirclePCSFRIProver(ctx, logn, 2, queries, rounds)
    proof = prover.prove_evaluations(ev, pub)
    cms, chs, _, pairs = prover.trace()
    layers = [ev] + [oracle.circle_fold_chain(logn, ev, chs[:k]) for k in range(1, rounds)]
    dlayers = _dev(ctx, np.concatenate(layers))
    ex = azk.CircleFRIResidentQueryExtractor(ctx, logn, rounds)
    got = ex.extract_queries(dlayers.ptr, cms, pairs)
    fcnt = n >> rounds
    hdr = 8 + 4 + 4 + 4 + 44 + 16 + 4 + 32 + 4 + 32 * rounds + 8 + 16 * fcnt + 4
    assert got == proof[hdr:hdr + queries * ex.query_bytes]
    # a layer whose root is not the committed one is refused
    bad = list(cms)
    bad[rounds - 1] = bytes(32)
    with pytest.raises(azk.AZKError) as e:
        ex.extract_queries(dlayers.ptr, bad, pairs)
    assert e.value.name == "correctnessValidationFailed"
    with pytest.raises(azk.AZKError) as e:
        ex.extract_queries(dlayers.ptr, cms, [n // 2])
    assert e.value.name == "invalidInputLayout"
