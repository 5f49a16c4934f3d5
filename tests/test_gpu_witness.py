"""GPU parity: witness columns -> Circle FFT-basis coefficients
(CircleWitnessToFFTBasisPlanV1, CircleWitnessFFTBasis.swift:226-590) equals the
oracle's monomial -> Chebyshev -> line-basis conversion (CircleCodeword.swift:187-263)
for every column length, and feeds the prover like the reference's pipeline."""
import numpy as np
import pytest

import apple_b200 as azk
from tests import generators as G

pytestmark = pytest.mark.gpu


def _cols(rng, nx, ny):
    return (rng.integers(0, G.P, size=(nx, 4), dtype=np.uint32), rng.integers(0, G.P, size=(ny, 4), dtype=np.uint32))


@pytest.mark.parametrize("log_size,nx,ny", [(1, 1, 1), (2, 2, 0), (3, 1, 4), (5, 16, 9), (8, 128, 128), (11, 1000, 3), (12, 2048, 2048),
                                            (13, 4096, 4096), (15, 7000, 9000)])
def test_witness_transform_matches_oracle(ctx, oracle, log_size, nx, ny):
    rng = np.random.default_rng(log_size * 100 + nx)
    x, y = _cols(rng, nx, ny)
    plan = azk.CircleWitnessToFFTBasisPlan(ctx, log_size)
    got = plan.execute(x, y)
    assert np.array_equal(got, oracle.fft_basis_coefficients(log_size, x, y))


def test_witness_transform_golden_proof(ctx, oracle, golden):
    """Bench polynomial of the log-14 golden proof: witness plan -> PCS prover
    reproduces the reference's proof digest."""
    v = golden["bench_codeword_prover_log14"]
    x, y = G.bench_codeword_polynomial(1 << 14)
    coeffs = azk.CircleWitnessToFFTBasisPlan(ctx, 14).execute(x, y)
    assert np.array_equal(coeffs, oracle.fft_basis_coefficients(14, x, y))
    pub = bytes(0xA0 + i for i in range(32))
    proof = azk.CirclePCSFRIProver(ctx, 14, 2, 4, 3).prove_coefficients(coeffs, pub)
    assert oracle.sha3_256(proof).hex() == v["proof_hex"]


def test_witness_resident_and_rejections(ctx, oracle):
    rng = np.random.default_rng(5)
    x, y = _cols(rng, 40, 33)
    plan = azk.CircleWitnessToFFTBasisPlan(ctx, 7)
    dx, dy, do = ctx.alloc(16 * 40), ctx.alloc(16 * 33), ctx.alloc(16 * 128)
    dx.upload(x)
    dy.upload(y)
    plan.execute_resident(dx.ptr, 40, dy.ptr, 33, do.ptr)
    got = np.frombuffer(do.download(), np.uint32).reshape(-1, 4)
    assert np.array_equal(got, oracle.fft_basis_coefficients(7, x, y))
    with pytest.raises(azk.AZKError):  # output over a column
        plan.execute_resident(dx.ptr, 40, dy.ptr, 33, dx.ptr)
    with pytest.raises(azk.AZKError):  # too many coefficients
        plan.execute(np.zeros((65, 4), np.uint32), y)
    with pytest.raises(azk.AZKError):  # both empty
        plan.execute(np.zeros((0, 4), np.uint32), np.zeros((0, 4), np.uint32))
    bad = x.copy()
    bad[3, 2] = G.P
    with pytest.raises(azk.AZKError):
        plan.execute(bad, y)


def test_prover_from_polynomial_golden_and_resident(ctx, oracle, golden):
    """prove(polynomial:) and proveResidentWitnessCoefficients: the monomial columns of
    the log-14 golden proof go through the prover's own device conversion and give
    the reference's proof digest, from host and from resident columns."""
    v = golden["bench_codeword_prover_log14"]
    x, y = G.bench_codeword_polynomial(1 << 14)
    pub = bytes(0xA0 + i for i in range(32))
    prover = azk.CirclePCSFRIProver(ctx, 14, 2, 4, 3)
    proof = prover.prove_polynomial(x, y, pub)
    assert oracle.sha3_256(proof).hex() == v["proof_hex"]
    x, y = np.asarray(x, np.uint32).reshape(-1, 4), np.asarray(y, np.uint32).reshape(-1, 4)
    dx, dy = ctx.alloc(max(16, x.nbytes)), ctx.alloc(max(16, y.nbytes))
    dx.upload(x)
    dy.upload(y)
    dproof = ctx.alloc(len(proof))
    n = prover.prove_resident_witness(dx.ptr, len(x), dy.ptr, len(y), pub, dproof.ptr)
    assert n == len(proof) and dproof.download(n) == proof
    # random columns: the same proof as from the oracle's FFT-basis coefficients
    rng = np.random.default_rng(77)
    xs, ys = _cols(rng, 300, 211)
    p2 = azk.CirclePCSFRIProver(ctx, 11, 1, 8, 5)
    want = p2.prove_coefficients(oracle.fft_basis_coefficients(11, xs, ys), pub)
    assert p2.prove_polynomial(xs, ys, pub) == want
