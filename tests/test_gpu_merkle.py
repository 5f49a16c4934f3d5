"""GPU parity: SHA3 Merkle commitment and openings against the CPU oracle and the
reference's golden roots (MerkleTests.swift:119-585)."""
import numpy as np
import pytest

import apple_b200 as azk
from tests import generators as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("length", [0, 32, 136])
def test_merkle_matches_oracle_small(ctx, oracle, length):
    leaves = G.make_leaves(16, length, length)
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, 16, length, length)
    assert plan.commit(leaves) == oracle.merkle_root(leaves, 16, length, length)


def test_golden_roots(ctx, golden):
    leaves = G.make_leaves(8, 32, 32)
    assert azk.SHA3RawLeavesMerkleCommitPlan(ctx, 8, 32, 32).commit(leaves).hex() == golden["merkle_root_8x32"]["hex"]
    leaves = G.make_leaves(1024, 32, 32, salt=71)
    assert azk.SHA3RawLeavesMerkleCommitPlan(ctx, 1024, 32, 32).commit(leaves).hex() == golden["merkle_root_1024x32_salt71"]["hex"]
    for length, want in golden["bench_merkle_roots_16384"]["roots_by_leaf_length"].items():
        length = int(length)
        leaves = G.make_bench_leaves(16384, length)
        assert azk.SHA3RawLeavesMerkleCommitPlan(ctx, 16384, length, length).commit(leaves).hex() == want, length


@pytest.mark.parametrize("treelet_log", [1, 2, 3, 4, 6, 8, 10, 11, 12, 13])
@pytest.mark.parametrize("length,stride", [(0, 5), (64, 72), (128, 136), (135, 144), (136, 144), (32, 40)])
def test_treelet_depths_and_strides(ctx, oracle, treelet_log, length, stride):
    count = 256 if treelet_log < 9 else (4096 if treelet_log < 12 else 32768)
    leaves = G.make_leaves(count, stride, length, salt=length + treelet_log)
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, count, stride, length, treelet_log=treelet_log)
    assert plan.commit(leaves) == oracle.merkle_root(leaves, count, stride, length)


@pytest.mark.parametrize("log_count", [0, 1, 2, 9, 10, 11, 12, 17])
def test_tree_sizes_across_upper_levels(ctx, oracle, log_count):
    count = 1 << log_count
    rng = np.random.default_rng(log_count)
    leaves = rng.integers(0, 256, size=count * 64, dtype=np.uint8).tobytes()
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, count, 64, 64, treelet_log=4)
    r1 = plan.commit(leaves)
    assert r1 == oracle.merkle_root(leaves, count, 64, 64)
    # counters reset themselves: a second commit of new leaves is right too
    leaves2 = rng.integers(0, 256, size=count * 64, dtype=np.uint8).tobytes()
    assert plan.commit(leaves2) == oracle.merkle_root(leaves2, count, 64, 64)


def test_openings_match_oracle_and_verify(ctx, oracle):
    leaves = G.make_leaves(128, 144, 135, salt=131)
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, 128, 144, 135, treelet_log=4)
    assert plan.tree_depth == 7
    for idx in [0, 1, 63, 64, 127]:
        leaf, sib, root = plan.open_raw_leaf(leaves, idx)
        oroot, [osib] = oracle.merkle_openings(leaves, 128, 144, 135, [idx])
        assert root == oroot and sib == osib and leaf == leaves[idx * 144:idx * 144 + 135]
        assert oracle.merkle_verify(leaf, idx, sib, root)


def test_open_resident_many(ctx, oracle):
    count = 1 << 14
    rng = np.random.default_rng(3)
    leaves = rng.integers(0, 256, size=count * 64, dtype=np.uint8).tobytes()
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, count, 64, 64)
    root = plan.commit(leaves)
    idx = rng.integers(0, count, size=64)
    got = plan.open_resident(idx)
    oroot, want = oracle.merkle_openings(leaves, count, 64, 64, idx)
    assert root == oroot and got == want


def test_single_leaf_tree(ctx, oracle):
    leaves = G.make_leaves(1, 32, 32, salt=5)
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, 1, 32, 32)
    leaf, sib, root = plan.open_raw_leaf(leaves, 0)
    assert sib == [] and root == oracle.sha3_256(leaf)


def test_prehashed_root(ctx, oracle):
    rng = np.random.default_rng(11)
    for n in (1, 2, 512, 4096):
        d = rng.integers(0, 256, size=32 * n, dtype=np.uint8).tobytes()
        assert azk.commit_prehashed_leaves(ctx, d) == oracle.merkle_root_prehashed(d)
    with pytest.raises(azk.AZKError) as e:
        azk.commit_prehashed_leaves(ctx, b"\0" * 96)
    assert e.value.name == "invalidLeafCount"


def test_merkle_rejections(ctx):
    cases = [((3, 32, 32), "invalidLeafCount"), ((2, 137, 137), "unsupportedOneBlockLength"), ((2, 31, 32), "invalidInputLayout"),
             ((1 << 32, 0, 0), "invalidInputLayout")]
    for args, name in cases:
        with pytest.raises(azk.AZKError) as e:
            azk.SHA3RawLeavesMerkleCommitPlan(ctx, *args)
        assert e.value.name == name
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, 8, 32, 32)
    with pytest.raises(azk.AZKError) as e:
        plan.open_raw_leaf(G.make_leaves(8, 32, 32), 8)
    assert e.value.name == "invalidInputLayout"
