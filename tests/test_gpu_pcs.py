"""GPU parity: the Circle PCS/FRI prover (single instance and batched) produces
the oracle's proof bytes, the reference's golden proof digests and corpus bytes,
and the oracle verifier accepts them (CircleDomainTests.swift:1497-1830)."""
import os

import numpy as np
import pytest

import apple_b200 as azk
from tests import generators as G

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_first_fold_and_three_round_proof_digests(ctx, oracle, golden):
    v = golden["circle_first_fold_proof_log4"]
    pub = bytes(0x10 + i for i in range(32))
    p = azk.CirclePCSFRIProver(ctx, 4, 2, 3, 1)
    proof = p.prove_evaluations(G.stable_circle_evaluations(16), pub)
    assert oracle.sha3_256(proof).hex() == v["hex"]
    v = golden["circle_3round_proof_log5"]
    pub = bytes(0x50 + i for i in range(32))
    p = azk.CirclePCSFRIProver(ctx, 5, 2, 5, 3)
    proof = p.prove_evaluations(G.stable_circle_evaluations(32), pub)
    assert oracle.sha3_256(proof).hex() == v["hex"]
    assert oracle.verify(proof, pub)


@pytest.mark.parametrize("log_size", [10, 14])
def test_codeword_prover_golden_proof(ctx, oracle, golden, log_size):
    """FFT-basis coefficients -> codeword -> commit/fold -> proof: the reference's digest."""
    v = golden[f"bench_codeword_prover_log{log_size}"]
    x, y = G.bench_codeword_polynomial(1 << log_size)
    coeffs = oracle.fft_basis_coefficients(log_size, x, y)
    pub = bytes(0xA0 + i for i in range(32))
    p = azk.CirclePCSFRIProver(ctx, log_size, 2, 4, 3)
    proof = p.prove_coefficients(coeffs, pub)
    assert len(proof) == v["proof_bytes"]
    assert oracle.sha3_256(proof).hex() == v["proof_hex"]
    assert oracle.verify(proof, pub)


def test_corpus_proof_on_gpu(ctx, oracle, golden):
    c = golden["corpus"]
    valid = open(os.path.join(GOLDEN, c["valid_file"]), "rb").read()

    def q(hexes):
        return np.array([[int.from_bytes(bytes.fromhex(h)[4 * k:4 * k + 4], "little") for k in range(4)] for h in hexes], np.uint32)

    x, y = q(c["x_hex"]), q(c["y_hex"])
    prof = c["profile"]
    ev = azk.CircleCodewordPlan(ctx, c["log"]).execute(x, y)
    assert np.array_equal(ev, oracle.evaluate_direct(c["log"], x, y))
    p = azk.CirclePCSFRIProver(ctx, c["log"], prof["logBlowupFactor"], prof["queryCount"], c["rounds"], prof["grindingBits"])
    proof = p.prove_evaluations(ev, bytes.fromhex(c["public_digest"]), claimed_indices=c["claimed"])
    assert proof == valid


@pytest.mark.parametrize("log_size,rounds,queries", [(1, 1, 1), (2, 2, 3), (6, 6, 7), (9, 3, 16), (12, 6, 64), (17, 11, 64)])
def test_prover_matches_oracle(ctx, oracle, log_size, rounds, queries):
    rng = np.random.default_rng(log_size * 7 + rounds)
    ev = rng.integers(0, G.P, size=(1 << log_size, 4), dtype=np.uint32)
    pub = rng.integers(0, 256, size=32, dtype=np.uint8).tobytes()
    p = azk.CirclePCSFRIProver(ctx, log_size, 2, queries, rounds)
    proof = p.prove_evaluations(ev, pub)
    r = oracle.prove(log_size, ev, 2, queries, pub, rounds)
    assert proof == r.proof
    cm, ch, fl, qp = p.trace()
    assert cm == r.commitments and np.array_equal(ch, r.challenges) and np.array_equal(fl, r.final_layer) and qp == r.query_pairs


@pytest.mark.parametrize("schedule", [dict(treelet_log=3, group_log=2, threads=256, persistent_trees=1),
                                      dict(treelet_log=11, group_log=5, threads=512, persistent_trees=1),
                                      dict(layer_treelet={15: 9, 14: 9, 13: 7}, layer_threads={15: 512, 14: 128, 12: 512}),
                                      dict(treelet_log=1, group_log=1, threads=128), dict(treelet_log=5, group_log=3, threads=256),
                                      dict(treelet_log=11, group_log=11, threads=512), dict(treelet_log=8, group_log=2, threads=256),
                                      dict(treelet_log=13, group_log=13, threads=256), dict(treelet_log=2, group_log=1, threads=512)])
def test_prover_schedules_do_not_change_bytes(ctx, oracle, schedule):
    rng = np.random.default_rng(99)
    log_size, rounds = 15, 9
    ev = rng.integers(0, G.P, size=(1 << log_size, 4), dtype=np.uint32)
    pub = bytes(range(32))
    p = azk.CirclePCSFRIProver(ctx, log_size, 2, 20, rounds, schedule=schedule)
    assert p.prove_evaluations(ev, pub) == oracle.prove(log_size, ev, 2, 20, pub, rounds).proof


def test_prover_grinding(ctx, oracle):
    rng = np.random.default_rng(4)
    ev = rng.integers(0, G.P, size=(1 << 8, 4), dtype=np.uint32)
    pub = bytes(32)
    p = azk.CirclePCSFRIProver(ctx, 8, 2, 5, 4, grinding_bits=8)
    proof = p.prove_evaluations(ev, pub)
    r = oracle.prove(8, ev, 2, 5, pub, 4, grinding_bits=8)
    assert proof == r.proof and oracle.verify(proof, pub)


def test_prover_rejects_non_canonical(ctx):
    ev = np.zeros((16, 4), np.uint32)
    ev[3, 2] = G.P
    p = azk.CirclePCSFRIProver(ctx, 4, 2, 3, 1)
    with pytest.raises(azk.AZKError) as e:
        p.prove_evaluations(ev, bytes(32))
    assert e.value.name == "invalidInputLayout"


def test_prover_rejects_bad_parameters(ctx):
    for args in [(0, 2, 4, 1), (5, 0, 4, 1), (5, 2, 0, 1), (5, 2, 4, 6), (5, 2, 4, 0)]:
        with pytest.raises(azk.AZKError):
            azk.CirclePCSFRIProver(ctx, *args)
    with pytest.raises(azk.AZKError):
        azk.CirclePCSFRIProver(ctx, 5, 2, 4, 1, grinding_bits=21)


def _batch_inputs(logs, seed):
    rng = np.random.default_rng(seed)
    coeffs, offsets, counts = [], [], []
    pos = 0
    for lg in logs:
        n = (1 << lg) // 4
        c = rng.integers(0, G.P, size=(n, 4), dtype=np.uint32)
        coeffs.append(c)
        offsets.append(pos)
        counts.append(n)
        pos += n
    return np.concatenate(coeffs), offsets, counts


@pytest.mark.parametrize("plain", [False, True])
def test_batch_matches_oracle_uneven(ctx, oracle, plain):
    logs = [10, 13, 7, 12, 10, 15, 8, 11]
    rounds = [lg - 6 if lg > 6 else 1 for lg in logs]
    flat, offs, cnts = _batch_inputs(logs, 5)
    b = azk.BatchProver(ctx, logs, rounds, 2, 16, schedule=dict(treelet_log=8))
    b.upload(flat, offs, cnts)
    pubs = bytes((i * 7) & 0xFF for i in range(32 * len(logs)))
    b.prove(pubs, plain=plain)
    proofs = b.proofs()
    for i, lg in enumerate(logs):
        n = 1 << lg
        coeffs = np.zeros((n, 4), np.uint32)
        coeffs[: cnts[i]] = flat[offs[i]:offs[i] + cnts[i]]
        ev = oracle.fft_evaluate(lg, coeffs)
        r = oracle.prove(lg, ev, 2, 16, pubs[32 * i:32 * i + 32], rounds[i])
        assert proofs[i] == r.proof, i


def test_batch_persistent_trees_graph_replay(ctx, oracle):
    """The persistent work-queue commit launches (counters reset by the last CTA out)
    give the oracle's proofs, and again on graph replay and in the plain form."""
    logs = [12, 9, 14, 10, 11, 13]
    rounds = [lg - 6 for lg in logs]
    flat, offs, cnts = _batch_inputs(logs, 21)
    b = azk.BatchProver(ctx, logs, rounds, 2, 8, schedule=dict(group_log=12, threads=256, use_graph=1, persistent_trees=1))
    b.upload(flat, offs, cnts)
    pubs = bytes((3 * i) & 0xFF for i in range(32 * len(logs)))
    b.prove(pubs)
    first = b.proofs()
    for i, lg in enumerate(logs):
        c = np.zeros((1 << lg, 4), np.uint32)
        c[: cnts[i]] = flat[offs[i]:offs[i] + cnts[i]]
        assert first[i] == oracle.prove(lg, oracle.fft_evaluate(lg, c), 2, 8, pubs[32 * i:32 * i + 32], rounds[i]).proof
    b.prove(pubs)
    b.prove(pubs)
    assert b.proofs() == first
    b.prove(pubs, plain=True)
    assert b.proofs() == first


def test_batch_graph_replay_and_plain_agree(ctx):
    logs = [12, 9, 14, 10]
    rounds = [lg - 6 for lg in logs]
    flat, offs, cnts = _batch_inputs(logs, 8)
    b = azk.BatchProver(ctx, logs, rounds, 2, 8)
    b.upload(flat, offs, cnts)
    pubs = bytes(32 * len(logs))
    b.prove(pubs)
    first = b.proofs()
    b.prove(pubs)  # graph replay
    assert b.proofs() == first
    b.prove(pubs, plain=True)
    assert b.proofs() == first


def test_batch_upload_rejects_non_canonical(ctx):
    logs = [10, 11]
    flat, offs, cnts = _batch_inputs(logs, 3)
    b = azk.BatchProver(ctx, logs, [4, 5], 2, 8)
    b.upload(flat, offs, cnts)
    bad = flat.copy()
    bad[offs[1] + cnts[1] - 1, 2] = G.P
    with pytest.raises(azk.AZKError) as e:
        b.upload(bad, offs, cnts)
    assert e.value.name == "invalidInputLayout"


@pytest.mark.parametrize("log_size,count_log,rounds", [(5, 3, 2), (12, 10, 6), (13, 11, 7), (16, 14, 9), (20, 18, 14), (23, 21, 17)])
def test_lifted_m31_coefficients_match_oracle(ctx, oracle, log_size, count_log, rounds):
    """Coefficients with zero b, c, d limbs and a zero tail take the FFT's M31 path
    (one limb between passes, tail reads skipped); proofs stay the oracle's."""
    rng = np.random.default_rng(log_size * 3 + 1)
    count = 1 << count_log
    coeffs = np.zeros((count, 4), np.uint32)
    coeffs[:, 0] = rng.integers(0, G.P, size=count, dtype=np.uint32)
    pub = rng.integers(0, 256, size=32, dtype=np.uint8).tobytes()
    p = azk.CirclePCSFRIProver(ctx, log_size, 2, 8, rounds)
    proof = p.prove_coefficients(coeffs, pub)
    full = np.zeros((1 << log_size, 4), np.uint32)
    full[:count] = coeffs
    ev = oracle.fft_evaluate(log_size, full)
    assert proof == oracle.prove(log_size, ev, 2, 8, pub, rounds).proof
    # one nonzero upper limb anywhere switches the same prover back to QM31 arithmetic
    coeffs[count - 1, 3] = 5
    full[:count] = coeffs
    proof = p.prove_coefficients(coeffs, pub)
    assert proof == oracle.prove(log_size, oracle.fft_evaluate(log_size, full), 2, 8, pub, rounds).proof


@pytest.mark.parametrize("log_size", [4, 5, 12, 13, 14, 15, 16, 18, 19, 22])
def test_lifted_m31_prefix_counts_match_oracle(ctx, oracle, log_size):
    """Lifted-M31 inputs whose nonzero prefix is at most N/4 skip the two copy-only top
    stages of the first FFT pass; longer prefixes run every stage.  Prefixes of 1,
    N/4 - 1, N/4, N/4 + 1, N/2 and N coefficients, at sizes whose first pass covers 1,
    2 and 3+ stages (and single-pass sizes), give the oracle's proofs."""
    N = 1 << log_size
    if log_size == 22:
        counts = [N // 4, N // 4 + 1]
    else:
        counts = sorted({1, max(1, N // 4 - 1), max(1, N // 4), N // 4 + 1, N // 2, N})
    rounds = max(1, log_size - 4)
    rng = np.random.default_rng(0xC0 + log_size)
    offs = np.cumsum([0] + counts[:-1]).tolist()
    flat = np.zeros((sum(counts), 4), np.uint32)
    flat[:, 0] = rng.integers(0, G.P, size=len(flat), dtype=np.uint32)
    b = azk.BatchProver(ctx, [log_size] * len(counts), [rounds] * len(counts), 2, 8)
    b.upload(flat, offs, counts)
    pubs = rng.integers(0, 256, size=32 * len(counts), dtype=np.uint8).tobytes()
    b.prove(pubs)
    proofs = b.proofs()
    for i, c in enumerate(counts):
        full = np.zeros((N, 4), np.uint32)
        full[:c] = flat[offs[i]:offs[i] + c]
        want = oracle.prove(log_size, oracle.fft_evaluate(log_size, full), 2, 8, pubs[32 * i:32 * i + 32], rounds).proof
        assert proofs[i] == want, (log_size, c)


def test_batch_mixes_m31_and_qm31_instances(ctx, oracle):
    logs = [14, 13, 9, 15]
    rounds = [lg - 6 for lg in logs]
    rng = np.random.default_rng(21)
    flat, offs, cnts = _batch_inputs(logs, 9)
    flat[offs[0]:offs[0] + cnts[0], 1:] = 0   # instance 0: lifted M31
    flat[offs[2]:offs[2] + cnts[2], 1:] = 0   # instance 2: lifted M31 (single pass)
    b = azk.BatchProver(ctx, logs, rounds, 2, 8)
    b.upload(flat, offs, cnts)
    pubs = rng.integers(0, 256, size=32 * len(logs), dtype=np.uint8).tobytes()
    b.prove(pubs)
    proofs = b.proofs()
    for i, lg in enumerate(logs):
        full = np.zeros((1 << lg, 4), np.uint32)
        full[:cnts[i]] = flat[offs[i]:offs[i] + cnts[i]]
        assert proofs[i] == oracle.prove(lg, oracle.fft_evaluate(lg, full), 2, 8, pubs[32 * i:32 * i + 32], rounds[i]).proof, i
    # writing through the input pointer makes the batch forget the upload's description
    import ctypes
    ptr = b.input_pointer(0)
    full = rng.integers(0, G.P, size=(1 << logs[0], 4), dtype=np.uint32)
    azk._capi.check(azk.lib().azk_buf_upload(ctx.handle, ctypes.c_void_p(ptr), 0, full.ctypes.data, full.nbytes), ctx.handle)
    b.prove(pubs)
    want = oracle.prove(logs[0], oracle.fft_evaluate(logs[0], full), 2, 8, pubs[:32], rounds[0]).proof
    assert b.proofs()[0] == want


@pytest.mark.parametrize("plain", [False, True])
def test_batch_64_byte_leaves_match_oracle(ctx, oracle, plain):
    """64-byte Merkle leaves (4 QM31 per leaf): commitments, challenges and final layers
    of every instance equal the oracle's chain; no proof bytes exist for this layout."""
    logs = [14, 9, 12, 7, 16, 11]
    rounds = [lg - 6 if lg > 7 else 1 for lg in logs]
    flat, offs, cnts = _batch_inputs(logs, 64)
    flat[offs[1]:offs[1] + cnts[1], 1:] = 0  # one lifted-M31 instance
    b = azk.BatchProver(ctx, logs, rounds, 2, 16, leaf_bytes=64)
    b.upload(flat, offs, cnts)
    pubs = bytes((3 * i + 1) & 0xFF for i in range(32 * len(logs)))
    b.prove(pubs, plain=plain)
    for i, lg in enumerate(logs):
        full = np.zeros((1 << lg, 4), np.uint32)
        full[:cnts[i]] = flat[offs[i]:offs[i] + cnts[i]]
        cm, ch, fl = oracle.commit_fold_chain_leaf64(lg, oracle.fft_evaluate(lg, full), 2, 16, pubs[32 * i:32 * i + 32], rounds[i])
        gcm, gch, gfl, _ = b.trace(i)
        assert gcm == cm, i
        assert np.array_equal(gch, ch), i
        assert np.array_equal(gfl, fl), i
    assert b.proof_total == 0
    with pytest.raises(azk.AZKError):
        b.proofs()


def test_batch_64_byte_leaves_need_four_values_per_layer(ctx):
    with pytest.raises(azk.AZKError):
        azk.BatchProver(ctx, [8], [8], 2, 4, leaf_bytes=64)
    with pytest.raises(azk.AZKError):
        azk.BatchProver(ctx, [8], [2], 2, 4, leaf_bytes=32)
