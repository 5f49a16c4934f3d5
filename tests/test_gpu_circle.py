"""GPU parity: circle domain tables, Circle FFT codeword, folds and fold chains
against the CPU oracle and the reference's golden digests
(CircleDomainTests.swift:129-148, 1200-1240, 1318-2084; bench reports)."""
import numpy as np
import pytest

import apple_b200 as azk
from tests import generators as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_size", [1, 2, 3, 5, 8, 13, 16])
def test_domain_tables_match_oracle(ctx, oracle, log_size):
    assert np.array_equal(azk.circle_domain_points(ctx, log_size), oracle.domain_points(log_size))
    assert np.array_equal(azk.circle_fft_twiddles(ctx, log_size), oracle.fft_twiddles(log_size))
    got = azk.circle_inverse_layers(ctx, log_size, log_size)
    want = oracle.inverse_layers(log_size, log_size)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_domain_log5_golden_digests(ctx, oracle, golden):
    v = golden["circle_log5_digests"]
    assert oracle.sha3_256(azk.circle_domain_points(ctx, 5).astype("<u4").tobytes()).hex() == v["points"]
    assert oracle.sha3_256(azk.circle_fft_twiddles(ctx, 5).astype("<u4").tobytes()).hex() == v["fft_twiddles"]
    layers = azk.circle_inverse_layers(ctx, 5, 4)
    q = np.concatenate([np.stack([l, 0 * l, 0 * l, 0 * l], axis=1) for l in layers]).astype("<u4")
    assert oracle.sha3_256(q.tobytes()).hex() == v["inverse_layers_4"]


@pytest.mark.parametrize("log_size", [1, 2, 4, 6, 11, 12, 13, 15, 18, 22, 23])
def test_codeword_fft_matches_oracle(ctx, oracle, log_size):
    n = 1 << log_size
    rng = np.random.default_rng(log_size)
    coeffs = rng.integers(0, G.P, size=(n, 4), dtype=np.uint32)
    plan = azk.CircleCodewordPlan(ctx, log_size)
    got = plan.execute_coefficients(coeffs)
    assert np.array_equal(got, oracle.fft_evaluate(log_size, coeffs))


@pytest.mark.parametrize("log_size", [1, 3, 6])
def test_codeword_polynomial_matches_direct(ctx, oracle, log_size):
    half = 1 << (log_size - 1)
    x = G.deterministic_qm31_coefficients(half, 0x40)
    y = G.deterministic_qm31_coefficients(half, 0x80)
    plan = azk.CircleCodewordPlan(ctx, log_size)
    assert np.array_equal(plan.execute(x, y), oracle.evaluate_direct(log_size, x, y))
    assert np.array_equal(plan.execute(x[:1]), oracle.evaluate_direct(log_size, x[:1], []))


@pytest.mark.parametrize("log_size,nx,ny", [(12, 2048, 2048), (14, 8192, 8192), (14, 5000, 1), (16, 3, 700)])
def test_codeword_polynomial_long_columns(ctx, oracle, log_size, nx, ny):
    """execute(polynomial:) converts monomials to the FFT basis on the device (the
    witness kernels); the codeword equals the oracle's conversion + FFT, for full
    half-domain columns as well as ragged ones."""
    rng = np.random.default_rng(log_size * 100 + nx)
    x = rng.integers(0, G.P, size=(nx, 4), dtype=np.uint32)
    y = rng.integers(0, G.P, size=(ny, 4), dtype=np.uint32)
    want = oracle.fft_evaluate(log_size, oracle.fft_basis_coefficients(log_size, x, y))
    assert np.array_equal(azk.CircleCodewordPlan(ctx, log_size).execute(x, y), want)


@pytest.mark.parametrize("log_size", [10, 14])
def test_codeword_golden_digest(ctx, oracle, golden, log_size):
    v = golden[f"bench_codeword_prover_log{log_size}"]
    x, y = G.bench_codeword_polynomial(1 << log_size)
    cw = azk.CircleCodewordPlan(ctx, log_size).execute(x, y)
    assert oracle.sha3_256(cw.astype("<u4").tobytes()).hex() == v["codeword_hex"]


def test_codeword_prefix_coefficients_zero_filled(ctx, oracle):
    log_size = 14
    n = 1 << log_size
    rng = np.random.default_rng(1)
    coeffs = np.zeros((n, 4), np.uint32)
    coeffs[: n // 4] = rng.integers(0, G.P, size=(n // 4, 4), dtype=np.uint32)
    plan = azk.CircleCodewordPlan(ctx, log_size)
    assert np.array_equal(plan.execute_coefficients(coeffs[: n // 4]), oracle.fft_evaluate(log_size, coeffs))


def test_qm31_fold_matches_oracle(ctx, oracle):
    rng = np.random.default_rng(2)
    n = 1 << 12
    ev = rng.integers(0, G.P, size=(n, 4), dtype=np.uint32)
    inv = rng.integers(1, G.P, size=(n // 2, 4), dtype=np.uint32)
    ch = rng.integers(0, G.P, size=4, dtype=np.uint32)
    assert np.array_equal(azk.qm31_fold(ctx, ev, inv, ch), oracle.fold(ev, inv, ch))
    bad = inv.copy()
    bad[5] = 0
    with pytest.raises(azk.AZKError):
        azk.qm31_fold(ctx, ev, bad, ch)


def test_bench_first_fold_and_explicit_chain_log14(ctx, oracle, golden):
    v = golden["bench_circle_first_fold_log14"]
    ev = G.deterministic_qm31(1 << 14, v["salts"])
    out = azk.circle_fold_chain(ctx, 14, ev, np.array([v["challenge"]], np.uint32))
    assert oracle.sha3_256(out.astype("<u4").tobytes()).hex() == v["hex"]
    v = golden["bench_circle_fold_chain_explicit_log14"]
    ev = G.deterministic_qm31(1 << 14, v["salts"])
    out = azk.circle_fold_chain(ctx, 14, ev, G.circle_fri_challenges(3))
    assert oracle.sha3_256(out.astype("<u4").tobytes()).hex() == v["hex"]


@pytest.mark.parametrize("log_size,rounds", [(4, 1), (8, 8), (16, 10)])
def test_circle_fold_chain_matches_oracle(ctx, oracle, log_size, rounds):
    rng = np.random.default_rng(log_size)
    ev = rng.integers(0, G.P, size=(1 << log_size, 4), dtype=np.uint32)
    ch = rng.integers(0, G.P, size=(rounds, 4), dtype=np.uint32)
    assert np.array_equal(azk.circle_fold_chain(ctx, log_size, ev, ch), oracle.circle_fold_chain(log_size, ev, ch))


def test_qm31_merkle_fold_chain_matches_oracle(ctx, oracle):
    rng = np.random.default_rng(9)
    n, rounds = 1 << 12, 5
    ev = rng.integers(0, G.P, size=(n, 4), dtype=np.uint32)
    inv = [rng.integers(1, G.P, size=(n >> (r + 1), 4), dtype=np.uint32) for r in range(rounds)]
    fin, cm, ch = azk.qm31_merkle_fold_chain(ctx, ev, inv)
    ofin, ocm, och = oracle.qm31_merkle_fold_chain(ev, inv)
    assert cm == ocm and np.array_equal(ch, och) and np.array_equal(fin, ofin)
    assert np.array_equal(azk.qm31_transcript_challenges(ctx, n, cm), oracle.qm31_transcript_challenges(n, cm))


def test_circle_merkle_fold_chain_golden_log14(ctx, oracle, golden):
    v = golden["bench_circle_fold_chain_merkle_log14"]
    ev = G.deterministic_qm31(1 << 14, v["salts"])
    pub = bytes(0x90 + i for i in range(32))
    fin, cm, ch = azk.circle_merkle_fold_chain(ctx, 14, ev, 2, 4, pub, 3)
    assert oracle.sha3_256(fin.astype("<u4").tobytes()).hex() == v["hex"]
    r = oracle.prove(14, ev, 2, 4, pub, 3)
    assert cm == r.commitments and np.array_equal(ch, r.challenges)


def test_canonical_gate(ctx):
    buf = ctx.alloc(4 * 1024)
    words = np.arange(1024, dtype=np.uint32)
    buf.upload(words)
    from apple_b200 import _capi
    import ctypes

    flag = ctypes.c_uint32(7)
    _capi.check(_capi.lib().azk_check_canonical(ctx.handle, buf.ptr, 1024, ctypes.byref(flag)))
    assert flag.value == 0
    words[900] = G.P
    buf.upload(words)
    _capi.check(_capi.lib().azk_check_canonical(ctx.handle, buf.ptr, 1024, ctypes.byref(flag)))
    assert flag.value == 1


@pytest.mark.parametrize("log_size", [5, 13])
def test_codeword_plan_resident_ranges(ctx, oracle, log_size):
    """executeResident (CircleCodeword.swift:517-545): coefficients and codeword in
    device buffers at byte offsets equal the host form; a range past its allocation
    or an output over the coefficients is rejected."""
    rng = np.random.default_rng(log_size)
    n = 1 << log_size
    coeffs = rng.integers(0, G.P, size=(n, 4), dtype=np.uint32)
    plan = azk.CircleCodewordPlan(ctx, log_size)
    want = plan.execute_coefficients(coeffs)
    din, dout = ctx.alloc(16 * n + 32), ctx.alloc(16 * n + 64)
    din.upload(coeffs, 32)
    plan.execute_resident(din.ptr, dout.ptr, in_offset=32, out_offset=64)
    assert np.array_equal(np.frombuffer(dout.download(16 * n, 64), np.uint32).reshape(-1, 4), want)
    for args in [dict(in_offset=48), dict(out_offset=80)]:
        with pytest.raises(azk.AZKError) as e:
            plan.execute_resident(din.ptr, dout.ptr, **args)
        assert e.value.name == "invalidInputLayout"
    with pytest.raises(azk.AZKError) as e:
        plan.execute_resident(din.ptr, din.ptr, in_offset=32, out_offset=16)
    assert e.value.name == "invalidInputLayout"
