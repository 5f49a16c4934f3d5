"""GPU parity: the M31 multilinear sum-check prover (M31MultilinearSumcheckProofBuilderV1,
SumcheckOracle.swift:797-868) gives the oracle's round sums, challenges, claimed sum,
final evaluation and statement digest, bit for bit."""
import numpy as np
import pytest

import apple_b200 as azk

pytestmark = pytest.mark.gpu
P = (1 << 31) - 1


def _same(g, o):
    assert g["claimed_sum"] == o["claimed_sum"]
    assert g["initial_digest"] == o["initial_digest"]
    assert np.array_equal(g["r0"], o["r0"])
    assert np.array_equal(g["r1"], o["r1"])
    assert np.array_equal(g["challenges"], o["challenges"])
    assert g["final"] == o["final"]


# 2^1..2^6 cover the digest's tail-only and first-block paths; 2^7.. the full
# 136-byte blocks assembled from words
@pytest.mark.parametrize("log_n", [1, 2, 3, 5, 6, 7, 8, 10, 13, 16])
def test_sumcheck_matches_oracle(ctx, oracle, log_n):
    rng = np.random.default_rng(0x5C + log_n)
    ev = rng.integers(0, P, 1 << log_n, dtype=np.uint32)
    _same(azk.sumcheck_prove(ctx, ev), oracle.sumcheck_multilinear(ev))


def test_sumcheck_serving_size(ctx, oracle):
    """The serving mix's sum-check jobs are 2^20 evaluations."""
    rng = np.random.default_rng(20)
    ev = rng.integers(0, P, 1 << 20, dtype=np.uint32)
    _same(azk.sumcheck_prove(ctx, ev), oracle.sumcheck_multilinear(ev))


def test_sumcheck_edge_values(ctx, oracle):
    for ev in (np.full(64, P - 1, np.uint32), np.zeros(32, np.uint32), np.arange(1 << 9, dtype=np.uint32)):
        _same(azk.sumcheck_prove(ctx, ev), oracle.sumcheck_multilinear(ev))


def test_sumcheck_rejects_bad_inputs(ctx):
    with pytest.raises(azk.AZKError):
        azk.sumcheck_prove(ctx, np.zeros(3, np.uint32))
    with pytest.raises(azk.AZKError):
        azk.sumcheck_prove(ctx, np.zeros(1, np.uint32))
    with pytest.raises(azk.AZKError):
        azk.sumcheck_prove(ctx, np.full(4, P, np.uint32))
