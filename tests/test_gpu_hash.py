"""GPU parity: Keccak-f[1600] batch and SHA3-256 / Keccak-256 fixed-rate batch
hashing against the CPU oracle (SHA3OracleTests.swift:130-760)."""
import hashlib

import numpy as np
import pytest

import apple_b200 as azk
from tests import generators as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("count,in_stride,out_stride", [(6, 216, 224), (5, 200, 200), (7, 200, 200), (1000, 200, 200), (129, 208, 200)])
def test_keccak_permutation_plan_matches_oracle(ctx, oracle, count, in_stride, out_stride):
    states = G.make_permutation_states(count, in_stride, salt=0x91)
    plan = azk.KeccakF1600PermutationPlan(ctx, count, in_stride, out_stride)
    out = np.frombuffer(plan.permute(states), np.uint8)
    want = oracle.keccak_f1600(states, in_stride)
    for i in range(count):
        assert out[i * out_stride:i * out_stride + 200].tobytes() == want[i * in_stride:i * in_stride + 200].tobytes(), i
        assert not out[i * out_stride + 200:(i + 1) * out_stride].any()


def test_keccak_plan_reuse_and_clear(ctx, oracle):
    plan = azk.KeccakF1600PermutationPlan(ctx, 5)
    for salt in (0x11, 0x203):
        st = G.make_permutation_states(5, 200, salt)
        assert plan.permute(st) == oracle.keccak_f1600(st).tobytes()
        plan.clear_reusable_buffers()


def test_keccak_large_random_batch(ctx, oracle):
    rng = np.random.default_rng(7)
    st = rng.integers(0, 256, size=200 * 100003, dtype=np.uint8)
    plan = azk.KeccakF1600PermutationPlan(ctx, 100003)
    assert plan.permute(st) == oracle.keccak_f1600(st).tobytes()


def test_keccak_plan_rejects_invalid_layouts(ctx):
    for args in [(0, 200, 200), (1, 199, 200), (1, 200, 201), (1 << 32, 200, 200)]:
        with pytest.raises(azk.AZKError) as e:
            azk.KeccakF1600PermutationPlan(ctx, *args)
        assert e.value.name == "invalidInputLayout"
    with pytest.raises(azk.AZKError) as e:
        azk.KeccakF1600PermutationPlan(ctx, 1, threads=7)
    assert e.value.name == "invalidKernelConfiguration"


@pytest.mark.parametrize("keccak", [False, True])
@pytest.mark.parametrize("length", [0, 1, 31, 32, 64, 128, 135, 136])
def test_hash_plan_matches_oracle(ctx, oracle, keccak, length):
    count = 9
    stride = length + 3 if length else 0
    msgs = G.make_batch_messages(count, stride, length, salt=length * 13)
    plan = azk.SHA3FixedOneBlockHashPlan(ctx, count, stride, length, 40, keccak=keccak)
    out = plan.hash(msgs)
    want = oracle.hash_batch(msgs, count, stride, length, 40, keccak=keccak)
    assert out == want
    if not keccak:
        for i in range(count):
            assert out[i * 40:i * 40 + 32] == hashlib.sha3_256(msgs[i * stride:i * stride + length]).digest()


@pytest.mark.parametrize("length", [32, 64, 128, 136])
def test_hash_plan_contiguous_large(ctx, oracle, length):
    count = 1 << 16
    rng = np.random.default_rng(length)
    msgs = rng.integers(0, 256, size=count * length, dtype=np.uint8).tobytes()
    plan = azk.SHA3FixedOneBlockHashPlan(ctx, count, length, length)
    assert plan.hash(msgs) == oracle.hash_batch(msgs, count, length, length)


def test_hash_plan_padding_zeroed_and_reuse(ctx, oracle):
    plan = azk.SHA3FixedOneBlockHashPlan(ctx, 4, 37, 32, 40)
    for salt in (0, 17):
        msgs = G.make_batch_messages(4, 37, 32, salt)
        out = plan.hash(msgs)
        assert out == oracle.hash_batch(msgs, 4, 37, 32, 40)
        plan.clear_reusable_buffers()


def test_hash_plan_rejections(ctx):
    with pytest.raises(azk.AZKError) as e:
        azk.SHA3FixedOneBlockHashPlan(ctx, 1, 137, 137)
    assert e.value.name == "unsupportedOneBlockLength"
    with pytest.raises(azk.AZKError) as e:
        azk.SHA3FixedOneBlockHashPlan(ctx, (1 << 32), 0, 0)
    assert e.value.name == "invalidInputLayout"
    with pytest.raises(azk.AZKError) as e:
        azk.SHA3FixedOneBlockHashPlan(ctx, 1, 32, 32, 31)
    assert e.value.name == "invalidInputLayout"
