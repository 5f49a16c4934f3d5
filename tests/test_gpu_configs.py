"""GPU parity at the benchmark configurations' own sizes.

C1: SHA3 Merkle commitment over 2^16 leaves of 64 uniform bytes plus 16 openings.
C2: 2^24 raw Keccak-f[1600] permutations; SHA3-256 over 2^24 messages of 32, 64, 128
    and 136 bytes; SHA3 Merkle over 2^24 leaves of 64 bytes plus 1024 openings.
C3: one Circle PCS/FRI proof of a log-22 codeword (blowup 4, 16 folds to log 6,
    64 queries).
C4: the batched superstep's 512 uneven instances (log sizes U[10, 22]).

Every output is compared byte for byte with the CPU oracle at full size (the
oracle runs on all host threads), and proofs go through the oracle's verifier
(CircleProofFormat.swift:1397-1546), like the reference's *Verified entry points
(CircleCodeword.swift:1152-1177) and its bench's exit on mismatch (main.swift:20).
"""
import ctypes
import hashlib

import numpy as np
import pytest

import apple_b200 as azk
from tests import generators as G

pytestmark = pytest.mark.gpu

N24 = 1 << 24


def _download(ctx, buf, nbytes):
    out = np.empty(nbytes, np.uint8)
    azk._capi.check(azk.lib().azk_buf_download(ctx.handle, ctypes.c_void_p(out.ctypes.data), buf.ptr, 0, nbytes), ctx.handle)
    return out


def test_c1_exact(ctx, oracle):
    n = 1 << 16
    leaves, idx = G.config_c1()
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, n, 64, 64)
    root = plan.commit(leaves)
    got = plan.open_resident(idx)
    oroot, want = oracle.merkle_openings(leaves, n, 64, 64, idx)
    assert root == oroot and got == want
    for k, i in enumerate(idx.tolist()):
        leaf = leaves[64 * i:64 * i + 64].tobytes()
        assert oracle.merkle_verify(leaf, i, got[k], root)
        # level-0 sibling = SHA3-256 of the neighbouring leaf (hashlib cross-check)
        j = i ^ 1
        assert got[k][0] == hashlib.sha3_256(leaves[64 * j:64 * j + 64].tobytes()).digest()
    # the reference's per-opening path (commit + open one leaf) agrees, and so does its
    # literal full-rebuild oracle
    for i in idx[:4].tolist():
        leaf, sib, r = plan.open_raw_leaf(leaves, i)
        lroot, lsib = oracle.merkle_opening_literal(leaves, n, 64, 64, i)
        assert r == root == lroot and sib == lsib and leaf == leaves[64 * i:64 * i + 64].tobytes()


def test_c2_keccak_f1600_2e24(ctx, oracle):
    states = G.config_bytes(G.C2_SEED, N24 * 200)
    din, dout = ctx.alloc(N24 * 200), ctx.alloc(N24 * 200)
    din.upload(states)
    plan = azk.KeccakF1600PermutationPlan(ctx, N24)
    plan.permute_resident(din.ptr, dout.ptr)
    got = _download(ctx, dout, N24 * 200)
    din.free()
    dout.free()
    want = oracle.keccak_f1600(states)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("length", [32, 64, 128, 136])
def test_c2_sha3_2e24(ctx, oracle, length):
    msgs = G.config_bytes(G.C2_SEED + length, N24 * length)
    din, dout = ctx.alloc(N24 * length), ctx.alloc(N24 * 32)
    din.upload(msgs)
    plan = azk.SHA3FixedOneBlockHashPlan(ctx, N24, length, length)
    plan.hash_resident(din.ptr, dout.ptr)
    got = _download(ctx, dout, N24 * 32)
    din.free()
    dout.free()
    want = np.frombuffer(oracle.hash_batch(msgs, N24, length, length), np.uint8)
    assert np.array_equal(got, want)
    for i in (0, 1, N24 // 2, N24 - 1):
        assert got[32 * i:32 * i + 32].tobytes() == hashlib.sha3_256(msgs[length * i:length * (i + 1)].tobytes()).digest()


def test_c2_merkle_2e24_1024_openings(ctx, oracle):
    leaves = G.config_bytes(G.C2_SEED ^ 0x3E, N24 * 64)
    idx = G.config_indices(G.C2_SEED, 1024, N24)
    dl = ctx.alloc(N24 * 64)
    dl.upload(leaves)
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, N24, 64, 64)
    root = plan.commit_resident(dl.ptr)
    got = plan.open_resident(idx)
    dl.free()
    oroot, want = oracle.merkle_openings(leaves, N24, 64, 64, idx)
    assert root == oroot
    assert got == want
    for k in (0, 511, 1023):
        i = int(idx[k])
        assert oracle.merkle_verify(leaves[64 * i:64 * i + 64].tobytes(), i, got[k], root)


def test_c3_log22_16_rounds_64_queries_verify(ctx, oracle):
    log_size, rounds, queries = 22, 16, 64
    coeffs, pub = G.config_c3(log_size)
    p = azk.CirclePCSFRIProver(ctx, log_size, 2, queries, rounds)
    proof = p.prove_coefficients(coeffs, pub)
    full = np.zeros((1 << log_size, 4), np.uint32)
    full[: len(coeffs)] = coeffs
    r = oracle.prove(log_size, oracle.fft_evaluate(log_size, full), 2, queries, pub, rounds)
    assert len(proof) == len(r.proof) == azk.pcs_proof_size(log_size, rounds, queries)
    assert proof == r.proof
    cm, ch, fl, qp = p.trace()
    assert cm == r.commitments and np.array_equal(ch, r.challenges) and np.array_equal(fl, r.final_layer) and qp == r.query_pairs
    assert oracle.verify(proof, pub)


def test_c4_batched_superstep_512_instances(ctx, oracle):
    """The bench's workload: every one of the 512 proofs is accepted by the oracle's
    verifier, and one instance of each log size (10 ... 22) equals the oracle's
    proof byte for byte; the plain per-instance form gives the same bytes."""
    import bench

    logs, rounds, counts, offsets = bench.workload()
    rows = bench.coefficient_rows(counts)
    pubs = bench.public_digests(len(logs))
    b = azk.BatchProver(ctx, logs, rounds, 2, 64, schedule=dict(group_log=12, threads=256, use_graph=1))
    b.upload(rows, offsets, counts)
    b.prove(pubs)
    proofs = b.proofs()
    for i in range(len(logs)):
        assert oracle.verify(proofs[i], pubs[32 * i:32 * i + 32]), i
    for i in bench.stratified_sample(logs):
        n = 1 << logs[i]
        c = np.zeros((n, 4), np.uint32)
        c[: counts[i]] = rows[offsets[i]:offsets[i] + counts[i]]
        want = oracle.prove(logs[i], oracle.fft_evaluate(logs[i], c), 2, 64, pubs[32 * i:32 * i + 32], rounds[i]).proof
        assert proofs[i] == want, (i, logs[i])
    b.prove(pubs, plain=True)
    assert b.proofs() == proofs
