"""The allocation-free Merkle root entry point (azk_merkle_root_noalloc).

It serves callers that may not call cudaMalloc -- a host that gives the library
a fixed memory budget, code that must not risk the device synchronisation an
allocation can cause, or a loop that cannot afford an allocation failure -- by
keeping its scratch in a fixed array inside the library.  This file runs last
(pytest collects it after the other test files) and passes both alone in a fresh
process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

import apple_b200 as azk
from apple_b200 import _capi

pytestmark = pytest.mark.gpu

MAX_LEAVES = 1 << 16


def _root_noalloc(dev_leaves, count, stride, length, dev_root):
    rc = _capi.lib().azk_merkle_root_noalloc(dev_leaves, count, stride, length, dev_root, None)
    return rc


def test_noalloc_root_matches_plan_two_calls_in_a_row(ctx):
    rng = np.random.default_rng(0x5EED)
    for count, stride, length in [(MAX_LEAVES, 64, 64), (1024, 72, 64), (1, 32, 32), (256, 136, 136), (4096, 40, 33)]:
        leaves_buf = ctx.alloc(max(16, count * stride))
        root_buf = ctx.alloc(32)
        plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, count, stride, length)
        for call in range(2):
            leaves = rng.integers(0, 256, size=count * stride, dtype=np.uint8)
            leaves_buf.upload(leaves)
            want = plan.commit_resident(leaves_buf.ptr)
            rc = _root_noalloc(leaves_buf.ptr, count, stride, length, root_buf.ptr)
            assert rc == 0, _capi.lib().azk_last_error_message(None)
            got = root_buf.download(32)  # synchronous copy after the default-stream kernel
            assert got == want, (count, stride, length, call)
        plan.close()
        leaves_buf.free()
        root_buf.free()


def test_noalloc_rejects_sizes_beyond_the_limit(ctx):
    buf = ctx.alloc(64)
    rc = _root_noalloc(buf.ptr, MAX_LEAVES * 2, 32, 32, buf.ptr)
    assert azk.AZK_STATUS_NAMES[rc] == "invalidInputLayout"
    assert b"65536" in _capi.lib().azk_last_error_message(None)
    assert azk.AZK_STATUS_NAMES[_root_noalloc(buf.ptr, 3, 32, 32, buf.ptr)] == "invalidLeafCount"
    assert azk.AZK_STATUS_NAMES[_root_noalloc(buf.ptr, 4, 137, 137, buf.ptr)] == "unsupportedOneBlockLength"
